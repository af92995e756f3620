// kh_kernel.cu -- Kirchhoff-Helmholtz pressure at far-field targets.
//
// Two-way KH sum (part3_kh_extrapolation.jl:168-185) with the monopole and
// dipole kernels of eval_one_kernel (src/kh_kernels.jl:106-157):
//
//   out[t, r] = aq * sum_s sum_k p_p(k; s, r) in_q[t - k, s]
//             + af * sum_s sum_k p_v(k; s, r) in_f[t - k, s]
//   p_p(k) = dfg(tau_k) / (4 pi d)
//   p_v(k) = cos_s * (fg(tau_k) / (4 pi d^2) + dfg(tau_k) / (4 pi d c0))
//   tau_k  = k dt - d / c0,  fg = Gaussian(sigma),  dfg = fg'
//
// which is what direct_kh_accumulate! (src/kh_kernels.jl:256-296) computes
// from a materialised kernel K(nt_K, N_s, N_r).  Here K is never stored: the
// kernel is a fractional-delay Gaussian, so only the taps within
// +-window_sigmas*sigma of the delay are non-negligible and each (target,
// surface point) pair's taps are evaluated on the fly from its geometry.
//
// Work decomposition (CUDA cores, FP32 FMA bound):
//   CTA   = 16 targets x one block of 32*T output samples, 16 warps
//   warp  = KH_RW targets (default 1); lane = T consecutive output samples
//           of each (T odd: 13 or 17, chosen per call by the padded cost)
//   loop  = surface points in chunks of SC.  One thread stages chunk c+1's
//           input windows into shared memory with bulk async copies while
//           the CTA works on chunk c (double buffer, mbarrier completion);
//           the input columns are zero-padded on the device so that every
//           window is one aligned, in-bounds copy.  Each chunk's pair
//           geometry is computed in FP64, each pair's 2*LM taps are
//           evaluated one per lane into a per-warp buffer, and every lane
//           forms its T outputs with LM*T paired FMAs (__ffma2_rn: the
//           monopole and dipole channel in one instruction) from a window
//           of T+LM-1 samples per channel.  Lanes start T samples apart, an
//           odd stride, so the 32 lanes of a window load hit 32 banks.
//   The partial sums of KH_G consecutive surface points are added to the
//   output accumulators with a compensated (Kahan) FP32 sum, so the sum over
//   thousands of surface points keeps FP32 round-off at the level of a
//   few additions.
#include <cmath>
#include <cstring>
#include <vector>

#include "ptx_util.h"
#include "runtime.h"

namespace adf {

namespace {

#ifndef KH_NWARPS
#define KH_NWARPS 16
#endif
#ifndef KH_NRW
#define KH_NRW 1
#endif
#ifndef KH_NG
#define KH_NG 8
#endif
constexpr int KH_WARPS = KH_NWARPS;
constexpr int KH_THREADS = 32 * KH_WARPS;
constexpr int KH_RW = KH_NRW;            // targets per warp
constexpr int KH_G = KH_NG;              // surface points summed before each compensated add
constexpr int KH_RT = KH_WARPS * KH_RW;  // targets per CTA
constexpr int KH_SC_MAX = 32;            // surface points per staged chunk
// Output samples per lane, T, is a template parameter: 17 (128 registers)
// costs about 8 % less per sample than 13 (112 registers) on long traces, but
// its CTAs cover 544 samples against 416, so short traces pad more.  The
// launcher takes the one with the smaller padded cost.
constexpr int KH_T_LONG = 17, KH_T_SHORT = 13;
constexpr double KH_T_LONG_COST = 0.917;  // per-sample cost of 17 relative to 13

int kh_samples_per_lane(int nt) {
  const double c17 = KH_T_LONG_COST * (double)((nt + 32 * KH_T_LONG - 1) / (32 * KH_T_LONG)) *
                     (32 * KH_T_LONG);
  const double c13 = (double)((nt + 32 * KH_T_SHORT - 1) / (32 * KH_T_SHORT)) * (32 * KH_T_SHORT);
  return c17 < c13 ? KH_T_LONG : KH_T_SHORT;
}

struct KhParams {
  int ns, nr, nt;
  int sc;           // surface points per chunk
  int rowpad;       // staged floats per channel and surface point (multiple of 4)
  int pad;          // zero samples in front of each padded input column
  long long pitch;  // floats per padded input column (multiple of 4)
  double inv_c0dt;  // 1 / (c0 dt)
  double hw;        // window half width in samples
  double aq, af;    // channel scales
  double C;         // 1 / (sqrt(2 pi) sigma)
  double dts2;      // dt / sigma^2
  double c0, inv_rho;
  float a;          // dt^2 / (2 sigma^2)
  float dt_sigma;   // dt / sigma (argument scale of the Gaussian CDF)
  const double* sp;  // (ns,3) column-major
  const double* sn;
  const double* rp;  // (nr,3)
  const double* rn;  // (nr,3) target normals (velocity output)
  const int2* tile_lo;  // per target tile: {lo_min, lo_max}
  const float* in_qf;   // (2 pitch, ns): zero-padded columns of {in_q, in_f} pairs,
                        // the pair of sample t at 2 (pad + t)
  const float* cs_f;    // running sum of in_f, same layout (velocity output)
  float* out;           // (nt, nr)
  int* err;
  unsigned wait_limit;  // polls of a chunk's bounded wait (kWaitLimit)
  int skip_chunk;       // test hook: chunk whose copies are not issued (-1: none)
};

}  // namespace

// KIND 0: pressure (p_p on in_q, p_v on in_f).  KIND 1: normal velocity
// (v_p on in_q, v_v on in_f); v_v's Gaussian-CDF term tends to a constant,
// so beyond each pair's window it is that constant times the running sum of
// in_f (staged as a third row per surface point).
template <int LM, int KIND, int T>
__global__ void __launch_bounds__(KH_THREADS, 1) adf_kh_pressure_kernel(KhParams p) {
  static_assert(T % 2 == 1, "lanes must start an odd number of samples apart");
  constexpr int XN = T + LM - 1;
  extern __shared__ __align__(128) float smem[];
  __shared__ __align__(8) uint64_t full[2];
  __shared__ int s_abort;  // a chunk's bounded wait gave up
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tile = blockIdx.x;
  const int tb = blockIdx.y * (32 * T);
  const int r_base = tile * KH_RT;
  const int2 lob = p.tile_lo[tile];
  const int lo_min = lob.x, lo_max = lob.y;
  // first staged sample, rounded down to a 16-B boundary of the padded column
  const int g0 = tb - lo_max - (LM - 1);
  const int col0 = p.pad + g0;
  const int shift = col0 & 3;
  const float* colqf = p.in_qf + 2 * (col0 - shift);
  const float* colc = KIND ? p.cs_f + (col0 - shift) : nullptr;
  const int npair = KH_RT * p.sc;
  constexpr int NROW = KIND ? 3 : 2;  // staged rows per surface point
  constexpr int NPAR = 8;             // lo, n, wb, 5 coefficients

  // shared memory: 2 window buffers [sc][NROW][rowpad] (per surface point a
  // row of rowpad {q, f} pairs, then for KIND 1 the running-sum row), 2 pair-parameter
  // buffers [NPAR][RT*sc], per-warp taps [warps][RW][LM][2]
  const int wbuf = p.sc * NROW * p.rowpad;
  float* const par0 = smem + 2 * wbuf;
  float* taps = par0 + 2 * NPAR * npair;
  float* my_taps = taps + warp * (KH_RW * 2 * LM);

  const int nchunks = (p.ns + p.sc - 1) / p.sc;
  if (threadIdx.x == 0) {
    mbar_init(smem_u32(&full[0]), 1);
    mbar_init(smem_u32(&full[1]), 1);
    fence_mbar_init();
    s_abort = 0;
  }
  __syncthreads();

  // bulk copies of chunk c (one thread)
  auto stage = [&](int c) {
    const int s0 = c * p.sc;
    const int nsc = min(p.sc, p.ns - s0);
    const uint32_t mb = smem_u32(&full[c & 1]);
    const uint32_t row_bytes = (uint32_t)p.rowpad * 4u;
    // the buffer's previous contents were read through the generic proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(mb, row_bytes * (uint32_t)NROW * (uint32_t)nsc);
    // test hook: the bytes are expected but never arrive, so this chunk's
    // wait runs out with no copy in flight
    if (c == p.skip_chunk) return;
    float* w = smem + (c & 1) * wbuf;
    for (int sl = 0; sl < nsc; ++sl) {
      const size_t off = (size_t)(s0 + sl) * p.pitch;
      bulk_load(smem_u32(w + (size_t)(NROW * sl) * p.rowpad), colqf + 2 * off, 2 * row_bytes, mb);
      if (KIND)
        bulk_load(smem_u32(w + (size_t)(NROW * sl + 2) * p.rowpad), colc + off, row_bytes, mb);
    }
  };
  // pair geometry of chunk c in FP64 (all threads)
  auto params = [&](int c) {
    const int s0 = c * p.sc;
    const int nsc = min(p.sc, p.ns - s0);
    float* pb = par0 + (c & 1) * NPAR * npair;
    int* pr_lo = reinterpret_cast<int*>(pb);
    int* pr_n = pr_lo + npair;
    float* pr_wb = pb + 2 * npair;
    float* pr_c = pb + 3 * npair;  // 5 coefficient arrays
    for (int idx = threadIdx.x; idx < KH_RT * nsc; idx += KH_THREADS) {
      const int rr = idx % KH_RT, sl = idx / KH_RT;
      const int r = r_base + rr, s = s0 + sl;
      int lo = lo_max, n = 0;
      float wb = 0.f, k0 = 0.f, k1 = 0.f, k2 = 0.f, k3 = 0.f, k4 = 0.f;
      if (r < p.nr) {
        const double dx = p.rp[r] - p.sp[s];
        const double dy = p.rp[r + p.nr] - p.sp[s + p.ns];
        const double dz = p.rp[r + 2 * p.nr] - p.sp[s + 2 * p.ns];
        const double d = sqrt(dx * dx + dy * dy + dz * dz);
        const double cs = (p.sn[s] * dx + p.sn[s + p.ns] * dy + p.sn[s + 2 * p.ns] * dz) / d;
        const double u = d * p.inv_c0dt;                 // delay in samples
        const double lod = ceil(u - p.hw);
        const double hid = floor(u + p.hw);
        const int l = lod < 0.0 ? 0 : (lod > 2.0e9 ? 2000000000 : (int)lod);
        const int h = hid > 2.0e9 ? 2000000000 : (int)hid;
        if (l <= p.nt - 1 && h >= l) {
          if (l < lo_min || l > lo_max) {
            atomicOr(p.err, 1);  // window bound violated: drop the pair
          } else {
            lo = l;
            n = min(h - l + 1, LM);
            const double i1 = 1.0 / (4.0 * M_PI * d);
            const double i2 = 1.0 / (4.0 * M_PI * (d * d));
            wb = (float)((double)l - u);
            // taps, w = k - delay in samples, e = exp(-a w^2):
            //   KIND 0: q = k0 w e,          f = (k1 + k2 w) e
            //   KIND 1: q = (k0 + k1 w) e,   f = (k2 + k3 w) e + k4 F(w dt)
            if (KIND == 0) {
              k0 = (float)(-p.aq * p.C * p.dts2 * i1);                 // p_p
              k1 = (float)(p.af * p.C * cs * i2);                      // p_v
              k2 = (float)(-p.af * p.C * p.dts2 / p.c0 * cs * i1);
            } else {
              const double cr =
                  (p.rn[r] * dx + p.rn[r + p.nr] * dy + p.rn[r + 2 * p.nr] * dz) / d;
              const double i3 = 1.0 / (4.0 * M_PI * (d * d * d));
              const double qr = p.aq * cr * p.inv_rho, fr = p.af * cr * cs * p.inv_rho;
              k0 = (float)(qr * p.C * i2);                              // v_p
              k1 = (float)(-qr * p.C * p.dts2 / p.c0 * i1);
              k2 = (float)(fr * p.C * 2.0 * i2 / p.c0);                 // v_v
              k3 = (float)(-fr * p.C * p.dts2 / (p.c0 * p.c0) * i1);
              k4 = (float)(fr * 2.0 * i3);                              // F term, pedestal
            }
          }
        }
      }
      const int pi = sl * KH_RT + rr;
      pr_lo[pi] = lo;
      pr_n[pi] = n;
      pr_wb[pi] = wb;
      pr_c[pi] = k0;
      pr_c[npair + pi] = k1;
      pr_c[2 * npair + pi] = k2;
      pr_c[3 * npair + pi] = k3;
      pr_c[4 * npair + pi] = k4;
    }
  };

  float sum[KH_RW][T], comp[KH_RW][T];
#pragma unroll
  for (int r = 0; r < KH_RW; ++r)
#pragma unroll
    for (int j = 0; j < T; ++j) sum[r][j] = comp[r][j] = 0.f;

  if (threadIdx.x == 0) stage(0);
  params(0);
  __syncthreads();
  bool ok = true;
  int failed = -1;  // chunk whose wait gave up (the same in every thread after a barrier)
  for (int c = 0; c < nchunks; ++c) {
    // a wait of the previous chunk gave up: stage nothing more
    if (s_abort) {
      failed = c - 1;
      break;
    }
    // chunk c+1's buffers were last read in chunk c-1, which every thread
    // has finished (barrier at the end of the previous iteration)
    if (c + 1 < nchunks) {
      if (threadIdx.x == 0) stage(c + 1);
      params(c + 1);
    }
    if (!mbar_wait(smem_u32(&full[c & 1]), (uint32_t)(c >> 1) & 1u, p.wait_limit)) {
      atomicOr(p.err, 2);
      s_abort = 1;  // read by every thread after the barrier below
      ok = false;
    }
    const int nsc = min(p.sc, p.ns - c * p.sc);
    const float* win = smem + (c & 1) * wbuf;
    const float* pb = par0 + (c & 1) * NPAR * npair;
    const int* pr_lo = reinterpret_cast<const int*>(pb);
    const int* pr_n = pr_lo + npair;
    const float* pr_wb = pb + 2 * npair;
    const float* pr_c = pb + 3 * npair;
    // partial sums of up to KH_G surface points, then one compensated add
    float2 c2[KH_RW][T];
#pragma unroll
    for (int rho = 0; rho < KH_RW; ++rho)
#pragma unroll
      for (int j = 0; j < T; ++j) c2[rho][j] = make_float2(0.f, 0.f);
    for (int sl = 0; ok && sl < nsc; ++sl) {
      // this point's {q, f} pairs from the first needed sample, and its
      // running-sum row
      const float2* wqf = reinterpret_cast<const float2*>(win + (size_t)(NROW * sl) * p.rowpad) + shift;
      const float* wc = win + (size_t)(NROW * sl + 2) * p.rowpad + shift;
      // taps of this warp's targets: lane-parallel, one exp per tap
#pragma unroll
      for (int rho = 0; rho < KH_RW; ++rho) {
        const int pi = sl * KH_RT + warp * KH_RW + rho;
        const float wb = pr_wb[pi];
        const int n = pr_n[pi];
#pragma unroll
        for (int kk = lane; kk < 2 * LM; kk += 32) {
          const int kp = kk % LM;
          const float w = wb + (float)kp;
          const float e = expf(-p.a * (w * w));
          float v;
          if (KIND == 0) {
            v = kk < LM ? pr_c[pi] * w * e : (pr_c[npair + pi] + pr_c[2 * npair + pi] * w) * e;
          } else if (kk < LM) {
            v = (pr_c[pi] + pr_c[npair + pi] * w) * e;
          } else {
            v = (pr_c[2 * npair + pi] + pr_c[3 * npair + pi] * w) * e +
                pr_c[4 * npair + pi] * normcdff(w * p.dt_sigma);
          }
          // interleaved {monopole, dipole} per tap for the paired FMA
          my_taps[rho * 2 * LM + 2 * kp + (kk >= LM)] = kp < n ? v : 0.f;
        }
      }
      __syncwarp();
#pragma unroll
      for (int rho = 0; rho < KH_RW; ++rho) {
        const int pi = sl * KH_RT + warp * KH_RW + rho;
        const int base = T * lane + (lo_max - pr_lo[pi]);
        // {monopole, dipole} input pairs: one paired FMA per tap and sample
        float2 x2[XN];
#pragma unroll
        for (int i = 0; i < XN; ++i) x2[i] = wqf[base + i];
        const float4* t4p = reinterpret_cast<const float4*>(my_taps + rho * 2 * LM);
#pragma unroll
        for (int k2 = 0; k2 < LM / 2; ++k2) {
          const float4 t4 = t4p[k2];
          const float2 ta = make_float2(t4.x, t4.y), tb2 = make_float2(t4.z, t4.w);
#pragma unroll
          for (int j = 0; j < T; ++j)
            c2[rho][j] = __ffma2_rn(ta, x2[j + LM - 1 - 2 * k2], c2[rho][j]);
#pragma unroll
          for (int j = 0; j < T; ++j)
            c2[rho][j] = __ffma2_rn(tb2, x2[j + LM - 2 - 2 * k2], c2[rho][j]);
        }
        if (KIND == 1) {  // lags past the window: v_v's constant times the running sum
          const float ped = pr_c[4 * npair + pi];
          const int cb = base + LM - 1 - pr_n[pi];
#pragma unroll
          for (int j = 0; j < T; ++j) c2[rho][j].y = __fmaf_rn(ped, wc[cb + j], c2[rho][j].y);
        }
      }
      // compensated accumulation over groups of surface points
      if (sl % KH_G == KH_G - 1 || sl == nsc - 1) {
#pragma unroll
        for (int rho = 0; rho < KH_RW; ++rho)
#pragma unroll
          for (int j = 0; j < T; ++j) {
            const float cj = __fadd_rn(c2[rho][j].x, c2[rho][j].y);
            const float y = __fsub_rn(cj, comp[rho][j]);
            const float t = __fadd_rn(sum[rho][j], y);
            comp[rho][j] = __fsub_rn(__fsub_rn(t, sum[rho][j]), y);
            sum[rho][j] = t;
            c2[rho][j] = make_float2(0.f, 0.f);
          }
      }
      __syncwarp();  // taps of the next surface point overwrite the buffer
    }
    __syncthreads();
  }
  if (failed < 0 && s_abort) failed = nchunks - 1;
  if (failed >= 0) {
    // The chunk after the failed one was staged before the failure: its
    // copies write into this CTA's shared memory, so let them land (again a
    // bounded wait) before the CTA exits.  No output is written; the host
    // reports ADF_E_TIMEOUT.
    const int c = failed + 1;
    if (threadIdx.x == 0 && c < nchunks && c != p.skip_chunk)
      mbar_wait(smem_u32(&full[c & 1]), (uint32_t)(c >> 1) & 1u);
    return;
  }

  // outputs: lane owns samples tb + T*lane .. +T-1 of each of its targets
#pragma unroll
  for (int rho = 0; rho < KH_RW; ++rho) {
    const int r = r_base + warp * KH_RW + rho;
    if (r >= p.nr) continue;
    const int t0 = tb + T * lane;
    float* o = p.out + (size_t)r * p.nt + t0;
#pragma unroll
    for (int j = 0; j < T; ++j)
      if (t0 + j < p.nt) o[j] = sum[rho][j];
  }
}

// FP32 FMA throughput probe: 8 independent chains per thread, enough warps
// per SM to keep every FMA pipe busy.  2 FLOP per FMA.
__global__ void __launch_bounds__(256) adf_fma_peak_kernel(float* out, int iters, float a, float b) {
  float x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-3f + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u)
#pragma unroll
      for (int k = 0; k < 8; ++k) x[k] = fmaf(x[k], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == 1234.5f) out[blockIdx.x] = s;  // keeps the chains live
}

// FP64 FMA throughput probe (the roofline of the in-loop GF contraction,
// which accumulates in Float64): the same chains in double.
__global__ void __launch_bounds__(256) adf_fma64_peak_kernel(double* out, int iters, double a,
                                                             double b) {
  double x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-3 + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u)
#pragma unroll
      for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == 1234.5) out[blockIdx.x] = s;  // keeps the chains live
}

namespace {

template <typename T>
struct DevBuf {  // device scratch from the context's pool, freed in stream order
  T* p = nullptr;
  cudaStream_t s = nullptr;
  explicit DevBuf(const adf_ctx* ctx) : s(ctx->stream), pool(ctx->pool) {}
  ~DevBuf() {
    if (p) cudaFreeAsync(p, s);
  }
  bool alloc(size_t n) {
    if (cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), n * sizeof(T), pool, s) == cudaSuccess)
      return true;
    cudaGetLastError();
    p = nullptr;
    return false;
  }

 private:
  cudaMemPool_t pool;
};

}  // namespace

}  // namespace adf

using namespace adf;

// kind 0: pressure, kind 1: normal velocity (adf_kh_pressure / adf_kh_velocity)
// {q, f} pairs of the padded input columns, so that a window's two channels
// are read with one 64-bit load
__global__ void adf_kh_interleave_kernel(const float* q, const float* f, float2* qf, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    qf[i] = make_float2(q[i], f[i]);
}

// Columns cols[s] of two [nt][ntx] trace arrays in HBM (a solve's recorded
// v_n and p, transceiver fastest) into the zero-padded KH input columns
// dq[s][pad + t], df[s][pad + t]: a 32 x 32 tiled transpose per array.
__global__ void adf_kh_gather_kernel(const float* q, const float* f, int ntx, int nt,
                                     const int* cols, int ns, float* dq, float* df,
                                     long long pitch, int pad) {
  __shared__ float tq[32][33], tf[32][33];
  const int s0 = blockIdx.x * 32, t0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {  // rows t, columns s: coalesced reads
    const int t = t0 + i, sl = s0 + threadIdx.x;
    float a = 0.f, b = 0.f;
    if (t < nt && sl < ns) {
      const long long o = (long long)t * ntx + cols[sl];
      a = q[o];
      b = f[o];
    }
    tq[i][threadIdx.x] = a;
    tf[i][threadIdx.x] = b;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {  // rows s, samples t: coalesced writes
    const int sl = s0 + i, t = t0 + threadIdx.x;
    if (sl < ns && t < nt) {
      dq[(long long)sl * pitch + pad + t] = tq[threadIdx.x][i];
      df[(long long)sl * pitch + pad + t] = tf[threadIdx.x][i];
    }
  }
}

// in_q / in_f either host arrays (nt, ns) or, with `dev`, columns of
// device-resident traces (pressure only).
static int kh_run(adf_ctx* ctx, const adf_kh_desc* d, const float* in_q, const float* in_f,
                  float* out, int kind, const KhDevSrc* dev = nullptr) {
  if (!ctx || !d || (!dev && (!in_q || !in_f)) || !out || !d->s_pts || !d->s_nrm || !d->r_pts)
    return fail(ADF_E_ARG, "adf_kh_pressure: null argument");
  if (dev && (kind != 0 || !dev->q || !dev->f || !dev->cols || dev->ntx < 1))
    return fail(ADF_E_ARG, "KH from device traces: pressure only, traces and columns required");
  if (kind == 1 && (!d->r_nrm || !(d->rho > 0)))
    return fail(ADF_E_ARG, "adf_kh_velocity: target normals and a positive rho are required");
  if (d->ns < 1 || d->nr < 1 || d->nt < 1 || !(d->dt > 0) || !(d->sigma > 0) || !(d->c0 > 0))
    return fail(ADF_E_ARG, "adf_kh_pressure: ns, nr, nt, dt, sigma and c0 must be positive");
  if (d->ns > (1 << 30) || d->nr > (1 << 30) || d->nt > (1 << 28))
    return fail(ADF_E_ARG, "adf_kh_pressure: sizes out of range");
  const double ws = d->window_sigmas > 0 ? d->window_sigmas : 6.0;
  const double hw = ws * d->sigma / d->dt;
  const int taps = (int)std::floor(2.0 * hw) + 1;
  int lm = 0;
  if (taps <= 16) lm = 16;
  else if (taps <= 24) lm = 24;  // e.g. +-6 sigma at 20 kHz and dt = 2.1 us: 19 taps
  else if (taps <= 32) lm = 32;
  else
    return fail(ADF_E_ARG, "adf_kh_pressure: the +-" + std::to_string(ws) +
                               " sigma window spans " + std::to_string(taps) +
                               " samples; at most 32 are supported");
  const int ns = (int)d->ns, nr = (int)d->nr, nt = (int)d->nt;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));

  // delay bounds of each target tile from the surface's bounding sphere
  double cx = 0, cy = 0, cz = 0;
  for (int s = 0; s < ns; ++s) {
    cx += d->s_pts[s];
    cy += d->s_pts[s + ns];
    cz += d->s_pts[s + 2 * ns];
  }
  cx /= ns; cy /= ns; cz /= ns;
  double rs = 0;
  for (int s = 0; s < ns; ++s) {
    const double ex = d->s_pts[s] - cx, ey = d->s_pts[s + ns] - cy, ez = d->s_pts[s + 2 * ns] - cz;
    rs = std::max(rs, std::sqrt(ex * ex + ey * ey + ez * ez));
  }
  rs = rs * (1 + 1e-12) + 1e-12;
  const double inv_c0dt = 1.0 / (d->c0 * d->dt);
  const int T = kh_samples_per_lane(nt), TB = 32 * T;  // output samples per lane, per CTA
  const int ntiles = (nr + KH_RT - 1) / KH_RT;
  std::vector<int2> tlo((size_t)ntiles);
  int wmax = 0, lo_all = 0;
  for (int t = 0; t < ntiles; ++t) {
    double dmin = 1e300, dmax = 0;
    for (int r = t * KH_RT; r < std::min(nr, (t + 1) * KH_RT); ++r) {
      const double ex = d->r_pts[r] - cx, ey = d->r_pts[r + nr] - cy, ez = d->r_pts[r + 2 * nr] - cz;
      const double dc = std::sqrt(ex * ex + ey * ey + ez * ez);
      dmin = std::min(dmin, std::max(0.0, dc - rs));
      dmax = std::max(dmax, dc + rs);
    }
    const double lmin = std::ceil(dmin * inv_c0dt - hw) - 2;
    const double lmax = std::ceil(dmax * inv_c0dt - hw) + 2;
    int lo_min = (int)std::max(0.0, std::min(lmin, (double)nt + 1));
    int lo_max = (int)std::max(0.0, std::min(lmax, (double)nt + 1));
    lo_min = std::min(lo_min, lo_max);
    tlo[(size_t)t] = make_int2(lo_min, lo_max);
    wmax = std::max(wmax, TB + (lo_max - lo_min) + lm - 1);
    lo_all = std::max(lo_all, lo_max);
  }
  // multiple of 4 floats so the tap buffer behind the rows stays 16-B aligned
  // A staged row starts up to 3 samples early (16-B aligned source) and is a
  // multiple of 4 floats, so every bulk copy and the tap buffer stay aligned.
  const int rowpad = (wmax + 3 + 3) / 4 * 4;
  const size_t tap_bytes = (size_t)KH_WARPS * KH_RW * 2 * lm * 4;
  const int nrow = kind ? 3 : 2;  // staged rows per surface point
  // double-buffered windows and pair parameters (lo, n, wb, 5 coefficients)
  const size_t per_s = 2 * ((size_t)nrow * rowpad * 4 + (size_t)8 * KH_RT * 4);
  const size_t smem_cap = (size_t)ctx->smem_optin - 256;  // static mbarriers
  int sc = KH_SC_MAX;
  while (sc > 1 && per_s * sc + tap_bytes > smem_cap) --sc;
  const size_t smem = per_s * sc + tap_bytes;
  // Input columns are zero-padded so that every staged window lies inside
  // its column: pad zeros before sample 0 cover the earliest window start,
  // the tail covers the last time block's window end.
  const int nblk = (nt + TB - 1) / TB;
  const int pad = (lo_all + lm + 4 + 3) / 4 * 4;
  const long long pitch = ((long long)pad + (long long)nblk * TB + lo_all + 16 + 3) / 4 * 4;
  if (smem > smem_cap)
    return fail(ADF_E_ARG, "adf_kh_pressure: the targets' delay spread needs a " +
                               std::to_string(wmax) + "-sample window, more than shared memory holds");

  // scratch from the context's pool: after the first call of a size the
  // memory stays mapped and later calls take it without driver allocations
  DevBuf<double> dsp(ctx), dsn(ctx), drp(ctx), drn(ctx);
  DevBuf<float> dq(ctx), df(ctx), dqf(ctx), dc(ctx), dout(ctx);
  DevBuf<int2> dtlo(ctx);
  DevBuf<int> derr(ctx);
  if (!dsp.alloc((size_t)3 * ns) || !dsn.alloc((size_t)3 * ns) || !drp.alloc((size_t)3 * nr) ||
      !dq.alloc((size_t)pitch * ns) || !df.alloc((size_t)pitch * ns) ||
      !dqf.alloc((size_t)2 * pitch * ns) ||
      !dout.alloc((size_t)nt * nr) ||
      !dtlo.alloc((size_t)ntiles) || !derr.alloc(1) ||
      (kind && (!drn.alloc((size_t)3 * nr) || !dc.alloc((size_t)pitch * ns))))
    return fail(ADF_E_NOMEM, "adf_kh_pressure: device allocation failed");
  std::vector<float> csum;
  if (kind) {  // running sum of in_f per surface point, in Float64, stored Float32
    csum.resize((size_t)nt * ns);
    for (int s = 0; s < ns; ++s) {
      double a = 0.0;
      for (int t = 0; t < nt; ++t) {
        a += (double)in_f[(size_t)s * nt + t];
        csum[(size_t)s * nt + t] = (float)a;
      }
    }
  }
  cudaStream_t st = ctx->stream;
  cudaMemcpyAsync(dsp.p, d->s_pts, (size_t)24 * ns, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dsn.p, d->s_nrm, (size_t)24 * ns, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(drp.p, d->r_pts, (size_t)24 * nr, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(dq.p, 0, (size_t)4 * pitch * ns, st);
  cudaMemsetAsync(df.p, 0, (size_t)4 * pitch * ns, st);
  if (dev) {
    const dim3 gg((unsigned)((ns + 31) / 32), (unsigned)((nt + 31) / 32));
    adf_kh_gather_kernel<<<gg, dim3(32, 8), 0, st>>>(dev->q, dev->f, dev->ntx, nt, dev->cols, ns,
                                                      dq.p, df.p, pitch, pad);
  } else {
    cudaMemcpy2DAsync(dq.p + pad, (size_t)4 * pitch, in_q, (size_t)4 * nt, (size_t)4 * nt, ns,
                      cudaMemcpyHostToDevice, st);
    cudaMemcpy2DAsync(df.p + pad, (size_t)4 * pitch, in_f, (size_t)4 * nt, (size_t)4 * nt, ns,
                      cudaMemcpyHostToDevice, st);
  }
  adf_kh_interleave_kernel<<<ctx->nsm * 8, 256, 0, st>>>(dq.p, df.p,
                                                         reinterpret_cast<float2*>(dqf.p),
                                                         (long long)pitch * ns);
  if (kind) {
    cudaMemcpyAsync(drn.p, d->r_nrm, (size_t)24 * nr, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(dc.p, 0, (size_t)4 * pitch * ns, st);
    cudaMemcpy2DAsync(dc.p + pad, (size_t)4 * pitch, csum.data(), (size_t)4 * nt,
                      (size_t)4 * nt, ns, cudaMemcpyHostToDevice, st);
  }
  cudaMemcpyAsync(dtlo.p, tlo.data(), sizeof(int2) * ntiles, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(derr.p, 0, sizeof(int), st);

  KhParams p;
  p.ns = ns; p.nr = nr; p.nt = nt;
  p.sc = sc; p.rowpad = rowpad;
  p.pad = pad; p.pitch = pitch;
  p.inv_c0dt = inv_c0dt;
  p.hw = hw;
  const double C = 1.0 / (std::sqrt(2.0 * M_PI) * d->sigma);
  const double s2 = d->sigma * d->sigma;
  p.aq = d->aq;
  p.af = d->af;
  p.C = C;
  p.dts2 = d->dt / s2;
  p.c0 = d->c0;
  p.inv_rho = kind ? 1.0 / d->rho : 0.0;
  p.a = (float)(d->dt * d->dt / (2.0 * s2));
  p.dt_sigma = (float)(d->dt / d->sigma);
  p.sp = dsp.p; p.sn = dsn.p; p.rp = drp.p; p.rn = drn.p;
  p.tile_lo = dtlo.p;
  p.in_qf = dqf.p; p.cs_f = dc.p; p.out = dout.p;
  p.err = derr.p;
  // the one-shot test hook of adf_kh_test_fault
  p.wait_limit = ctx->kh_wait_limit ? ctx->kh_wait_limit : kWaitLimit;
  p.skip_chunk = ctx->kh_skip_chunk;
  ctx->kh_wait_limit = 0;
  ctx->kh_skip_chunk = -1;

  // the instantiation for (taps, kind, samples per lane)
  using KhFn = void (*)(KhParams);
  // (taps past the window are zero, so a wider instantiation gives the same
  // sums with more FMAs: the narrowest that holds the window is taken)
  static const KhFn kfn[3][2][2] = {
      {{adf_kh_pressure_kernel<16, 0, KH_T_SHORT>, adf_kh_pressure_kernel<16, 0, KH_T_LONG>},
       {adf_kh_pressure_kernel<16, 1, KH_T_SHORT>, adf_kh_pressure_kernel<16, 1, KH_T_LONG>}},
      {{adf_kh_pressure_kernel<24, 0, KH_T_SHORT>, adf_kh_pressure_kernel<24, 0, KH_T_LONG>},
       {adf_kh_pressure_kernel<24, 1, KH_T_SHORT>, adf_kh_pressure_kernel<24, 1, KH_T_LONG>}},
      {{adf_kh_pressure_kernel<32, 0, KH_T_SHORT>, adf_kh_pressure_kernel<32, 0, KH_T_LONG>},
       {adf_kh_pressure_kernel<32, 1, KH_T_SHORT>, adf_kh_pressure_kernel<32, 1, KH_T_LONG>}}};
  const KhFn fn = kfn[lm == 16 ? 0 : (lm == 24 ? 1 : 2)][kind ? 1 : 0][T == KH_T_LONG ? 1 : 0];
  e = cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, std::string("kh smem: ") + cudaGetErrorString(e));
  const dim3 grid((unsigned)ntiles, (unsigned)((nt + TB - 1) / TB));
  cudaEventRecord(ctx->ev0, st);
  fn<<<grid, KH_THREADS, smem, st>>>(p);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, std::string("kh launch: ") + cudaGetErrorString(e));
  cudaEventRecord(ctx->ev1, st);
  int herr = 0;
  cudaMemcpyAsync(out, dout.p, (size_t)4 * nt * nr, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&herr, derr.p, sizeof(int), cudaMemcpyDeviceToHost, st);
  e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaGetLastError();  // a download refused when it was enqueued
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  ctx->last_ms = ms;
  ctx->kh_ms = ms;
  ctx->launches = 1;
  ctx->h2d_bytes = (int64_t)48 * ns + (kind ? 48 : 24) * (int64_t)nr +
                   (dev ? 0 : (int64_t)(kind ? 12 : 8) * nt * ns);
  ctx->d2h_bytes = (int64_t)4 * nt * nr;
  if (herr & 2) return fail(ADF_E_TIMEOUT, "KH: a bounded wait for a staged chunk gave up");
  if (herr) return fail(ADF_E_STATE, "KH: a pair's delay fell outside its tile bound");
  return ADF_OK;
}

namespace adf {
int kh_pressure_dev(adf_ctx* ctx, const adf_kh_desc* d, const KhDevSrc& src, float* out) {
  return kh_run(ctx, d, nullptr, nullptr, out, 0, &src);
}
}  // namespace adf

extern "C" int adf_kh_pressure(adf_ctx* ctx, const adf_kh_desc* d, const float* in_q,
                               const float* in_f, float* out) {
  return kh_run(ctx, d, in_q, in_f, out, 0);
}

extern "C" int adf_kh_velocity(adf_ctx* ctx, const adf_kh_desc* d, const float* in_q,
                               const float* in_f, float* out) {
  return kh_run(ctx, d, in_q, in_f, out, 1);
}

extern "C" int adf_kh_test_fault(adf_ctx* ctx, int skip_chunk, uint32_t poll_limit) {
  if (!ctx || skip_chunk < -1 || poll_limit == 0)
    return fail(ADF_E_ARG, "adf_kh_test_fault: skip_chunk >= -1 and poll_limit > 0");
  ctx->kh_skip_chunk = skip_chunk;
  ctx->kh_wait_limit = poll_limit;
  return ADF_OK;
}

extern "C" int adf_fp64_fma_peak(adf_ctx* ctx, double* tflops, double* ms_out) {
  if (!ctx || !tflops) return fail(ADF_E_ARG, "adf_fp64_fma_peak: null argument");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  const int blocks = ctx->nsm * 8, iters = 1024;
  DevBuf<double> o(ctx);
  if (!o.alloc((size_t)blocks)) return fail(ADF_E_NOMEM, "adf_fp64_fma_peak: allocation failed");
  adf_fma64_peak_kernel<<<blocks, 256, 0, ctx->stream>>>(o.p, 16, 0.999, 1e-4);  // warm-up
  cudaEventRecord(ctx->ev0, ctx->stream);
  adf_fma64_peak_kernel<<<blocks, 256, 0, ctx->stream>>>(o.p, iters, 0.999, 1e-4);
  cudaEventRecord(ctx->ev1, ctx->stream);
  e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  const double flop = 2.0 * 128.0 * iters * (double)blocks * 256;
  *tflops = flop / (ms * 1e-3) / 1e12;
  if (ms_out) *ms_out = ms;
  return ADF_OK;
}

extern "C" int adf_fp32_fma_peak(adf_ctx* ctx, double* tflops, double* ms_out) {
  if (!ctx || !tflops) return fail(ADF_E_ARG, "adf_fp32_fma_peak: null argument");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  const int blocks = ctx->nsm * 8, iters = 4096;
  DevBuf<float> o(ctx);
  if (!o.alloc((size_t)blocks)) return fail(ADF_E_NOMEM, "adf_fp32_fma_peak: allocation failed");
  adf_fma_peak_kernel<<<blocks, 256, 0, ctx->stream>>>(o.p, 64, 0.999f, 1e-4f);  // warm-up
  cudaEventRecord(ctx->ev0, ctx->stream);
  adf_fma_peak_kernel<<<blocks, 256, 0, ctx->stream>>>(o.p, iters, 0.999f, 1e-4f);
  cudaEventRecord(ctx->ev1, ctx->stream);
  e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  const double flop = 2.0 * 128.0 * iters * (double)blocks * 256;
  *tflops = flop / (ms * 1e-3) / 1e12;
  if (ms_out) *ms_out = ms;
  return ADF_OK;
}
