// gf_tc_kernel.cu -- the far-lag part of the in-loop GF extrapolation on the
// tensor cores (tcgen05.mma, kind::tf32, accumulators in tensor memory).
//
// extrapolate_pv_from_pin! and extrapolate_p_from_pin
// (src/kernels/extrapolation.jl:139-193) sum, for step it and driven source o,
//     sum_r sum_lag G[lag, o, r] * pin[it-1-lag, r].
// In the block-causal form (adf_gf_far_kernel in fdtd_kernels.cu) the lags
// older than the current block of kGfBlock steps are summed once per block.
// Per receiver r that is a matrix product: the source x lag slice of the map
// (A: 128 sources x 16 lags per chunk) times the block's masked Toeplitz
// window of the input history (B: 32 steps x 16 lags, B[b][l] =
// pin[it0-1+b-lag, r] on the far lags of step b, zero elsewhere).  Here that
// product runs on tcgen05.mma with FP32 accumulation in tensor memory.  Every
// Float32 map entry and Float64 history sample is split into a TF32 part
// (rounded to nearest, ties away) and the remainder, and hi*hi + hi*lo +
// lo*hi is accumulated: the dropped lo*lo term is below 2^-22 of the
// product and each remainder, read by the tensor cores at TF32 width, loses
// below 2^-21, so a product is within 5 * 2^-22 of g*h (the products of
// TF32 parts are exact in FP32).  After the last chunk of a receiver its
// accumulator is added into Float64 sums in shared memory (two accumulator
// sets in tensor memory alternate, so one is drained while the next
// receiver's products run), so the sum over receivers stays in Float64.  The result agrees with the
// Float64 sum to about 1e-6 relative, Float32 level: an opt-in contraction
// (ADF_GF_CONTRACT_TF32X3); the default path keeps the Float64 FMAs of the
// reference's accumulation.
//
// Data path: the two tensors of the map are split and packed once per map
// (adf_gf_tc_pack_kernel) into 32 KB tiles (receiver, 16-lag chunk,
// 128-source tile; TF32 parts and remainders of both tensors) laid out as
// the MMA's K-major, no-swizzle operands (8-row x 16-byte core matrices), so
// one bulk copy (cp.async.bulk, completing on an mbarrier, no multicast)
// stages a chunk's A operands where the MMAs read them, and a second one on
// the same mbarrier brings the chunk's rows of the input history; four chunks
// are staged, the next two in flight while two are in use.  Warps are
// specialised and hand work over on mbarriers, with no CTA barrier inside
// the loop: warps 0-3 (the owners of the 128 tensor-memory lanes) build each
// chunk's history operand (double-buffered) and drain the accumulators; one
// thread of warp 4 waits for a chunk's tile and operand, issues its 12 MMAs,
// commits them to the slot's mbarrier and refills the slot of the chunk two
// back.  One CTA (160 threads, 204 KB of shared memory, 128 tensor-memory
// columns) per SM and (source tile, receiver split); every wait is bounded
// and a wait that gives up sets the solve's error word (ADF_E_TIMEOUT), ends
// every role's loop, lets the copies and products in flight land, frees the
// tensor memory and leaves the partials unwritten.
#include <atomic>

#include "adf_internal.h"
#include "ptx_util.h"

namespace adf {

constexpr int kMaxDevices = 64;  // devices a process can launch this kernel on

constexpr int kTcM = 128;              // sources per CTA = tensor-memory lanes
constexpr int kTcL = 16;               // lags per chunk (two MMA k-steps of 8)
constexpr int kTcN = kGfBlock;         // steps of a block (MMA N)
constexpr int kTcStages = 4;           // staged map tiles in flight
constexpr int kTcTile = kTcL * kTcM;   // floats of one tensor's tile (8 KB)
constexpr int kTcBTile = kTcN * kTcL;  // floats of one history window operand (2 KB)
constexpr int kTcThreads = 160;        // warps 0-3: history operand, drains; warp 4: MMAs, copies
constexpr int kTcIssuer = 128;         // the thread that issues the MMAs and the bulk copies
constexpr int kTcWinD = 64;            // doubles per staged history window (50 at most used)
// shared memory (bytes): staged operand tiles [kTcStages][tensor][hi, lo]
// [kTcTile] f32 (read by the MMAs where they land), history windows
// [kTcStages][kTcWinD] f64, B operands [2 buffers][hi, lo][kTcBTile] f32,
// Float64 sums [tensor x step][source]
constexpr int kTcStgOff = 0;
constexpr int kTcWinOff = kTcStgOff + kTcStages * 4 * kTcTile * 4;
constexpr int kTcBOff = kTcWinOff + kTcStages * kTcWinD * 8;
constexpr int kTcSumOff = kTcBOff + 2 * 2 * kTcBTile * 4;
constexpr int kTcSmemBytes = kTcSumOff + 2 * kTcN * kTcM * 8;
constexpr size_t kTcDynSmem = kTcSmemBytes + 1024;  // + alignment to 1 KB
constexpr uint32_t kTcCols = 128;  // tensor-memory columns: 2 sets x 2 tensors x 32 steps
static_assert(kTcM == 128 && kTcN % 16 == 0 && kTcN <= 256, "MMA shape M=128, N=32");
static_assert(kTcCols >= 4 * kTcN, "two accumulator sets of two tensors");
// Instruction descriptor of kind::tf32: D Float32 (bit 4), A and B TF32
// (bits 7-9, 10-12), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) |
                              ((uint32_t)(kTcN >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
// Operand layouts (K-major, no swizzle): core matrix (row group g, k-block
// kb of 4 lags) at byte (kb * groups + g) * 128, its 8 rows 16 B apart.
constexpr uint32_t kTcALbo = (kTcM / 8) * 128;  // next k-block of A
constexpr uint32_t kTcBLbo = (kTcN / 8) * 128;  // next k-block of B
constexpr uint32_t kTcSbo = 128;                // next row group
constexpr uint32_t kTcWaitLimit = 1u << 22;     // polls of a bounded wait

// Shared-memory matrix descriptor (tcgen05): start, leading and stride byte
// offsets (>> 4), descriptor version 1 at bit 46, no swizzle, base offset 0.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__device__ __forceinline__ void tc_mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(kTcIdesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   mbar)
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// 16 consecutive 32-bit columns of this warp's 32 tensor-memory lanes
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
// x rounded to TF32 (10 stored mantissa bits, ties away from zero) by two
// integer operations; x - tf32_hi(x) is exact in Float32
__device__ __forceinline__ float tf32_hi(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// Packs the two tensors of an input-history map (layout as in
// adf_gf_far_kernel: PVFromPin element lag + ngf*(o + n1*r), PFromPin
// lag + ngf*(r + n1*o)) into tiles (r, chunk c, source tile ot) of
// [tensor][TF32 part, remainder][kb][g][row][4]: source ot*128 + 8g + row,
// lag 16c + 1 + 4kb + col, zero beyond the map.  Set-up, once per map.
__global__ void adf_gf_tc_pack_kernel(const float* t0, const float* t1, float* out, int kind,
                                      int ngf, int n1, int nout, int nin, int nch, int notile) {
  const long long per_tile = 4LL * kTcTile;
  const long long total = (long long)nin * nch * notile * per_tile;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(i % per_tile);
    long long tile = i / per_tile;
    const int ot = (int)(tile % notile);
    tile /= notile;
    const int c = (int)(tile % nch);
    const int r = (int)(tile / nch);
    const int t = e / (2 * kTcTile), part = (e / kTcTile) & 1, w = e % kTcTile;
    const int kb = w / (kTcM * 4), rem = w - kb * (kTcM * 4);
    const int g = rem >> 5, row = (rem >> 2) & 7, col = rem & 3;
    const int o = ot * kTcM + g * 8 + row, lag = kTcL * c + 1 + 4 * kb + col;
    float v = 0.f;
    if (o < nout && lag < ngf) {
      const long long idx = kind == ADF_GF_PV_FROM_PIN_ ? lag + (long long)ngf * (o + (long long)n1 * r)
                                                        : lag + (long long)ngf * (r + (long long)n1 * o);
      v = (t == 0 ? t0 : t1)[idx];
    }
    const float hi = tf32_hi(v);
    out[i] = part == 0 ? hi : __fsub_rn(v, hi);
  }
}

// Far-lag sums of the block of kGfBlock steps that starts at this launch-step
// (the same partials as adf_gf_far_kernel: gf_far[o][receiver split][step of
// the block][2], added over the splits by adf_gf_far_combine_kernel).
// blockIdx.x = source tile * gf_rs + receiver split, blockIdx.y = solve.
__global__ void __launch_bounds__(kTcThreads, 1) adf_gf_far_tc_kernel(const EpiParams p) {
  const SolveDev& S = p.solves[blockIdx.y];
  const int it0 = S.it_base + p.step;
  if (!(S.flags & SF_GF) || !(S.flags & SF_GF_TC) || S.gf_rs <= 0 || it0 > S.it_stop ||
      it0 >= S.nt)
    return;
  const int rsn = S.gf_rs, nout = S.gf_nout;
  const int ot = blockIdx.x / rsn, rsi = blockIdx.x - ot * rsn;
  if (ot * kTcM >= nout) return;
  const int nt = S.nt, ngf = S.gf_nt, nin = S.gf_nin, notile = (nout + kTcM - 1) / kTcM;
  const int r0 = (int)((long long)nin * rsi / rsn), r1 = (int)((long long)nin * (rsi + 1) / rsn);
  const int lag_hi = min(it0 + kGfBlock - 1, ngf) - 1;  // largest lag any step of the block uses
  const int nch = lag_hi >= 1 ? (lag_hi + kTcL - 1) / kTcL : 0;  // chunks this block needs
  const int Q = (r1 - r0) * nch;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int o = ot * kTcM + tid;  // threads 0..127: this source = this tensor-memory lane
  if (Q == 0) {  // no far lag in this block (uniform across the CTA)
    if (tid < kTcM && o < nout) {
      double* pp = S.gf_far + ((long long)o * rsn + rsi) * kGfBlock * 2;
      for (int k = 0; k < 2 * kTcN; ++k) pp[k] = 0.0;
    }
    return;
  }

  extern __shared__ unsigned char tc_smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  float* stg = reinterpret_cast<float*>(base + kTcStgOff);
  double* win = reinterpret_cast<double*>(base + kTcWinOff);
  float* opB = reinterpret_cast<float*>(base + kTcBOff);
  double* sums = reinterpret_cast<double*>(base + kTcSumOff);
  __shared__ __align__(8) uint64_t full[kTcStages];  // staged tile and window landed
  __shared__ __align__(8) uint64_t mmad[kTcStages];  // products of a staged chunk done
  __shared__ __align__(8) uint64_t bready[2];        // history operand of a buffer built
  __shared__ __align__(8) uint64_t drained[2];       // accumulator set added into the sums
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  for (int i = tid; i < 2 * kTcN * kTcM; i += kTcThreads) sums[i] = 0.0;
  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s) mbar_init(smem_u32(&full[s]), 1);
    for (int s = 0; s < kTcStages; ++s) mbar_init(smem_u32(&mmad[s]), 1);
    for (int s = 0; s < 2; ++s) {
      mbar_init(smem_u32(&bready[s]), 4);   // one arrival per builder warp
      mbar_init(smem_u32(&drained[s]), 4);
    }
    fence_mbar_init();
    s_abort = 0;
  }
  if (warp == 0) {  // one warp allocates (and later frees) the accumulators
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&s_tmem)),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = s_tmem;

  // solve fields used in the loop, read once (the loop's fences would
  // otherwise reload them from global memory every chunk)
  const float* gtc = S.gf_tc;
  const double* gpin = S.gf_pin;
  int* gerr = S.err;
  const long long cstride = (long long)notile * 4 * kTcTile;  // floats per 16-lag chunk
  const long long rstride = (long long)S.gf_tc_nch * cstride;  // floats per receiver
  // history window of chunk (receiver r0+rr, chunk c): the input-history
  // rows its far lags read, [max(0, it0-1-16(c+1)), min(it0-2, it0+29-16c)],
  // copied from the even element at or below the first (16-B aligned source)
  // for an even count of doubles; cnt = 0 when the chunk reads no row
  auto win_of = [&](int rr, int c, long long& gs, int& cnt) {
    const int lo = max(0, it0 - 1 - kTcL * (c + 1)), hi = min(it0 - 2, it0 + kTcN - 3 - kTcL * c);
    gs = 0;
    cnt = 0;
    if (hi < lo) return;
    const long long g0 = (long long)(r0 + rr) * nt;
    gs = (g0 + lo) & ~1LL;
    cnt = (int)((g0 + hi - gs + 2) & ~1LL);
  };
  // issuer: the next chunk to stage, as (receiver offset, chunk)
  int staged = 0, srr = 0, sc = 0;
  auto stage_next = [&]() {
    const int s = staged % kTcStages;
    long long gs;
    int cnt;
    win_of(srr, sc, gs, cnt);
    fence_proxy_async_smem();  // the slot was last read through the generic proxy
    const uint32_t tb = (uint32_t)(4 * kTcTile * sizeof(float));
    mbar_expect_tx(smem_u32(&full[s]), tb + (uint32_t)cnt * 8u);
    bulk_load(smem_u32(stg + s * 4 * kTcTile),
              gtc + (long long)(r0 + srr) * rstride + sc * cstride + ot * (4LL * kTcTile), tb,
              smem_u32(&full[s]));
    if (cnt > 0)
      bulk_load(smem_u32(win + s * kTcWinD), gpin + gs, (uint32_t)cnt * 8u, smem_u32(&full[s]));
    ++staged;
    if (++sc == nch) {
      sc = 0;
      ++srr;
    }
  };
  if (tid == kTcIssuer)
    while (staged < min(Q, kTcStages)) stage_next();
  auto abort_seen = [&]() { return *reinterpret_cast<volatile int*>(&s_abort) != 0; };
  // once any wait has given up, no later wait of the loops blocks again: a
  // wait that does not complete on its first try returns when the abort flag
  // is set, and each role leaves its loop at its next abort check
  auto bounded = [&](uint64_t* bar, int phase) {
    const uint32_t a = smem_u32(bar), par = (uint32_t)phase & 1u;
    if (mbar_try_wait(a, par) || abort_seen()) return;
    if (!mbar_wait(a, par, kTcWaitLimit)) {
      atomicOr(gerr, 4);  // reported as ADF_E_TIMEOUT
      s_abort = 1;         // every role leaves its loop
    }
  };
  // warps 0-3: adds accumulator set `set` of this warp's lanes into the
  // Float64 sums (step-major, source fastest)
  auto drain = [&](int set) {
    const uint32_t ta = tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)(set * 2 * kTcN);
#pragma unroll
    for (int t = 0; t < 2; ++t)
#pragma unroll
      for (int h = 0; h < kTcN / 16; ++h) {
        uint32_t v[16];
        tmem_ld16(ta + t * kTcN + h * 16, v);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          double* a = sums + (t * kTcN + h * 16 + j) * kTcM + tid;
          *a = __dadd_rn(*a, (double)__uint_as_float(v[j]));
        }
      }
  };
  const uint64_t descA = umma_desc(smem_u32(stg), kTcALbo, kTcSbo);
  const uint64_t descB = umma_desc(smem_u32(opB), kTcBLbo, kTcSbo);

  // Warps 0-3 build each chunk's history operand and hand it over on
  // bready; the issuer waits for the staged tile and the operand, issues the
  // chunk's products and commits them to mmad; no CTA barrier inside the
  // loop, so building, issuing and the tensor cores overlap across chunks.
  const int lane = tid & 31;
  int q = 0;  // the chunk this thread's role stopped at
  if (warp < 4) {
    int rr = 0, c = 0;  // chunk q = chunk c of receiver r0 + rr
    for (; q < Q; ++q, c = (c + 1 == nch ? 0 : c + 1), rr += (c == 0)) {
      const int s = q % kTcStages, buf = q & 1, r = r0 + rr;
      if (c == 0 && q > 0) {  // the previous receiver's products into Float64
        bounded(&mmad[(q - 1) % kTcStages], (q - 1) / kTcStages);
        tc_fence_after();
        drain((rr - 1) & 1);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&drained[(rr - 1) & 1]));
      }
      if (q >= 2) bounded(&mmad[(q - 2) % kTcStages], (q - 2) / kTcStages);  // B buffer of q-2
      bounded(&full[s], q / kTcStages);
      // the block's far-lag window of receiver r's input history: thread ->
      // step b = tid/4, lags 4(tid%4) .. +3 of the chunk (one core-matrix row)
      {
        long long gs;
        int cnt;
        win_of(rr, c, gs, cnt);
        const double* w = win + s * kTcWinD;
        const long long row0 = (long long)r * nt - gs;  // window index of history row 0
        const int b = tid >> 2, kb = tid & 3;
        const int lim = min(it0 + b, ngf);
        float hv[4], lv[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int lag = kTcL * c + 1 + 4 * kb + j;
          const double h = (lag > b && lag < lim) ? w[row0 + it0 - 1 + b - lag] : 0.0;
          hv[j] = tf32_hi((float)h);
          lv[j] = (float)(h - (double)hv[j]);
        }
        float* B = opB + buf * 2 * kTcBTile;
        const int off = (kb * (kTcN / 8) + (b >> 3)) * 32 + (b & 7) * 4;
        *reinterpret_cast<float4*>(B + off) = make_float4(hv[0], hv[1], hv[2], hv[3]);
        *reinterpret_cast<float4*>(B + kTcBTile + off) = make_float4(lv[0], lv[1], lv[2], lv[3]);
      }
      fence_proxy_async_smem();  // the B operand is read by the tensor cores (async proxy)
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&bready[buf]));
      if (abort_seen()) break;
    }
    if (q == Q && !abort_seen()) {  // the last receiver's products
      bounded(&mmad[(Q - 1) % kTcStages], (Q - 1) / kTcStages);
      tc_fence_after();
      drain(((Q - 1) / nch) & 1);
    }
  } else if (tid == kTcIssuer) {
    int rr = 0, c = 0;
    for (; q < Q; ++q, c = (c + 1 == nch ? 0 : c + 1), rr += (c == 0)) {
      const int s = q % kTcStages, buf = q & 1;
      bounded(&full[s], q / kTcStages);
      bounded(&bready[buf], q >> 1);
      if (c == 0 && rr >= 2) bounded(&drained[rr & 1], (rr - 2) >> 1);  // set of receiver rr-2
      if (abort_seen()) break;
      tc_fence_after();
      const uint32_t set = (uint32_t)((rr & 1) * 2 * kTcN);
      const uint64_t a0 = descA + (uint64_t)((s * 4 * kTcTile * 4) >> 4);
      const uint64_t b0 = descB + (uint64_t)((buf * 2 * kTcBTile * 4) >> 4);
#pragma unroll
      for (int ks = 0; ks < kTcL / 8; ++ks) {
        const uint64_t bh = b0 + ((ks * 2 * kTcBLbo) >> 4);
        const uint64_t bl = bh + ((kTcBTile * 4) >> 4);
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          const uint32_t d = tbase + set + (uint32_t)(t * kTcN);
          const uint64_t ah = a0 + (((2 * t) * kTcTile * 4 + ks * 2 * kTcALbo) >> 4);
          const uint64_t al = ah + ((kTcTile * 4) >> 4);
          tc_mma_tf32(d, ah, bh, (c > 0 || ks > 0) ? 1u : 0u);  // a receiver's first product overwrites
          tc_mma_tf32(d, ah, bl, 1u);
          tc_mma_tf32(d, al, bh, 1u);
        }
      }
      tc_commit(smem_u32(&mmad[s]));
      // the slot of chunk q-2 is free once its products are done: chunk q+2
      // (never staged over products that are not known to be done)
      if (q >= 2 && staged < Q) {
        bounded(&mmad[(q - 2) % kTcStages], (q - 2) / kTcStages);
        if (abort_seen()) {
          ++q;  // chunk q's products were issued: the clean-up waits for them
          break;
        }
        stage_next();
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (s_abort) {
    // let the copies and products in flight land before the CTA exits
    // (bounded again); no partial is written, the host reports the error
    if (tid == kTcIssuer) {
      for (int k = q; k < staged; ++k)
        mbar_wait(smem_u32(&full[k % kTcStages]), (uint32_t)(k / kTcStages) & 1u, kTcWaitLimit);
      if (q > 0)
        mbar_wait(smem_u32(&mmad[(q - 1) % kTcStages]), (uint32_t)((q - 1) / kTcStages) & 1u,
                  kTcWaitLimit);
    }
  } else if (tid < kTcM && o < nout) {
    double* pp = S.gf_far + ((long long)o * rsn + rsi) * kGfBlock * 2;
#pragma unroll 4
    for (int b = 0; b < kTcN; ++b) {
      pp[2 * b] = sums[b * kTcM + tid];
      pp[2 * b + 1] = sums[(kTcN + b) * kTcM + tid];
    }
  }
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(kTcCols)
                 : "memory");
  }
}

int64_t gf_tc_chunks(int64_t nt_gf) { return nt_gf > 1 ? (nt_gf - 1 + kTcL - 1) / kTcL : 1; }
size_t gf_tc_packed_floats(int64_t nt_gf, int64_t n_src, int64_t n_rec) {
  return (size_t)n_rec * gf_tc_chunks(nt_gf) * ((n_src + kTcM - 1) / kTcM) * 4 * kTcTile;
}
int gf_tc_sources_per_tile() { return kTcM; }

cudaError_t launch_gf_tc_pack(const SolveDev& d, float* out, cudaStream_t s) {
  const int notile = (d.gf_nout + kTcM - 1) / kTcM;
  adf_gf_tc_pack_kernel<<<8 * 148, 256, 0, s>>>(d.gf_t[0], d.gf_t[1], out, d.gf_kind, d.gf_nt,
                                                d.gf_n1, d.gf_nout, d.gf_nin, d.gf_tc_nch, notile);
  return cudaGetLastError();
}

cudaError_t launch_gf_far_tc(const EpiParams& p, int max_blocks, cudaStream_t s) {
  // the first launch on each device raises the kernel's shared-memory limit
  // there (contexts on several devices or threads may launch concurrently)
  static std::atomic<bool> attr_set[kMaxDevices];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  if (!attr_set[dev].load(std::memory_order_acquire)) {
    e = cudaFuncSetAttribute((const void*)adf_gf_far_tc_kernel,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcDynSmem);
    if (e != cudaSuccess) return e;
    attr_set[dev].store(true, std::memory_order_release);
  }
  adf_gf_far_tc_kernel<<<dim3(max_blocks > 0 ? max_blocks : 1, p.n_solves), kTcThreads, kTcDynSmem,
                         s>>>(p);
  return cudaGetLastError();
}

}  // namespace adf
