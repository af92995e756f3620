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
//   CTA   = 32 targets x one block of 256 output samples, 8 warps
//   warp  = 4 targets; lane = 8 consecutive output samples of each
//   loop  = surface points in chunks of SC: the chunk's input windows are
//           staged in shared memory (skewed by one word per eight so that
//           lanes reading 8 samples apart hit distinct banks), the chunk's
//           pair geometry is computed in FP64, each pair's 2*LM taps are
//           evaluated one per lane into a per-warp buffer, and every lane
//           forms its 8 outputs with 2*LM*8 register FMAs.
//   The per-pair partial sums are added to the output accumulators with a
//   compensated (Kahan) FP32 sum, so the sum over thousands of surface
//   points keeps FP32 round-off at the level of a single addition.
#include <cmath>
#include <cstring>
#include <vector>

#include "runtime.h"

namespace adf {

namespace {

constexpr int KH_T = 8;                 // output samples per lane
constexpr int KH_WARPS = 8;
constexpr int KH_THREADS = 32 * KH_WARPS;
constexpr int KH_TB = 32 * KH_T;        // output samples per CTA
constexpr int KH_RW = 4;                // targets per warp
constexpr int KH_RT = KH_WARPS * KH_RW; // targets per CTA
constexpr int KH_SC_MAX = 32;           // surface points per staged chunk

struct KhParams {
  int ns, nr, nt;
  int sc;           // surface points per chunk
  int wlen;         // staged samples per channel and surface point
  int rowpad;       // floats per staged row (skewed)
  double inv_c0dt;  // 1 / (c0 dt)
  double hw;        // window half width in samples
  double cq;        // -aq C dt / sigma^2            (C = 1/(sqrt(2 pi) sigma))
  double cf1;       //  af C
  double cf2;       // -af C dt / (sigma^2 c0)
  float a;          // dt^2 / (2 sigma^2)
  const double* sp;  // (ns,3) column-major
  const double* sn;
  const double* rp;  // (nr,3)
  const int2* tile_lo;  // per target tile: {lo_min, lo_max}
  const float* in_q;    // (nt, ns)
  const float* in_f;
  float* out;           // (nt, nr)
  int* err;
};

// Loads 8+LM-1 consecutive staged samples.  The staged address of sample m
// is m + m/8; a lane's window starts at m0 = 8*(lane+q) + rho, so with the
// base at 9*(lane+q) the offsets are compile-time for each rho.
template <int XN, int RHO>
__device__ __forceinline__ void kh_load_win(const float* __restrict__ b, float* x) {
#pragma unroll
  for (int i = 0; i < XN; ++i) x[i] = b[RHO + i + ((RHO + i) >> 3)];
}

template <int XN>
__device__ __forceinline__ void kh_load(const float* b, int rho, float* x) {
  switch (rho) {
    case 0: kh_load_win<XN, 0>(b, x); break;
    case 1: kh_load_win<XN, 1>(b, x); break;
    case 2: kh_load_win<XN, 2>(b, x); break;
    case 3: kh_load_win<XN, 3>(b, x); break;
    case 4: kh_load_win<XN, 4>(b, x); break;
    case 5: kh_load_win<XN, 5>(b, x); break;
    case 6: kh_load_win<XN, 6>(b, x); break;
    default: kh_load_win<XN, 7>(b, x); break;
  }
}

}  // namespace

template <int LM>
__global__ void __launch_bounds__(KH_THREADS, 1) adf_kh_pressure_kernel(KhParams p) {
  constexpr int XN = KH_T + LM - 1;
  extern __shared__ __align__(16) float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tile = blockIdx.x;
  const int tb = blockIdx.y * KH_TB;
  const int r_base = tile * KH_RT;
  const int2 lob = p.tile_lo[tile];
  const int lo_min = lob.x, lo_max = lob.y;
  const int g0 = tb - lo_max - (LM - 1);

  float* win = smem;                                     // [sc][2][rowpad]
  int* pr_lo = reinterpret_cast<int*>(win + (size_t)p.sc * 2 * p.rowpad);
  int* pr_n = pr_lo + KH_RT * p.sc;
  float* pr_wb = reinterpret_cast<float*>(pr_n + KH_RT * p.sc);
  float* pr_q = pr_wb + KH_RT * p.sc;
  float* pr_f1 = pr_q + KH_RT * p.sc;
  float* pr_f2 = pr_f1 + KH_RT * p.sc;
  float* taps = pr_f2 + KH_RT * p.sc;                    // [warps][RW][2][LM]
  float* my_taps = taps + warp * (KH_RW * 2 * LM);

  float sum[KH_RW][KH_T], comp[KH_RW][KH_T];
#pragma unroll
  for (int r = 0; r < KH_RW; ++r)
#pragma unroll
    for (int j = 0; j < KH_T; ++j) sum[r][j] = comp[r][j] = 0.f;

  for (int s0 = 0; s0 < p.ns; s0 += p.sc) {
    const int nsc = min(p.sc, p.ns - s0);
    __syncthreads();  // the previous chunk's readers are done
    // stage the chunk's input windows, zero outside [0, nt)
    const int per_row = p.wlen;
    const int total = nsc * 2 * per_row;
    for (int idx = threadIdx.x; idx < total; idx += KH_THREADS) {
      const int row = idx / per_row;
      const int m = idx - row * per_row;
      const int sl = row >> 1;
      const int g = g0 + m;
      float v = 0.f;
      if (g >= 0 && g < p.nt) {
        const float* src = (row & 1) ? p.in_f : p.in_q;
        v = __ldg(src + (size_t)(s0 + sl) * p.nt + g);
      }
      win[(size_t)row * p.rowpad + m + (m >> 3)] = v;
    }
    // pair geometry in FP64
    for (int idx = threadIdx.x; idx < KH_RT * nsc; idx += KH_THREADS) {
      const int rr = idx % KH_RT, sl = idx / KH_RT;
      const int r = r_base + rr, s = s0 + sl;
      int lo = lo_max, n = 0;
      float wb = 0.f, q = 0.f, f1 = 0.f, f2 = 0.f;
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
            q = (float)(p.cq * i1);
            f1 = (float)(p.cf1 * cs * i2);
            f2 = (float)(p.cf2 * cs * i1);
          }
        }
      }
      const int pi = sl * KH_RT + rr;
      pr_lo[pi] = lo;
      pr_n[pi] = n;
      pr_wb[pi] = wb;
      pr_q[pi] = q;
      pr_f1[pi] = f1;
      pr_f2[pi] = f2;
    }
    __syncthreads();

    for (int sl = 0; sl < nsc; ++sl) {
      const float* wq = win + (size_t)(2 * sl) * p.rowpad;
      const float* wf = wq + p.rowpad;
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
          const float v = kk < LM ? pr_q[pi] * w * e : (pr_f1[pi] + pr_f2[pi] * w) * e;
          my_taps[rho * 2 * LM + kk] = kp < n ? v : 0.f;
        }
      }
      __syncwarp();
#pragma unroll
      for (int rho = 0; rho < KH_RW; ++rho) {
        const int pi = sl * KH_RT + warp * KH_RW + rho;
        const int d = lo_max - pr_lo[pi];
        const int base = 9 * (lane + (d >> 3));
        float xq[XN], xf[XN];
        kh_load<XN>(wq + base, d & 7, xq);
        kh_load<XN>(wf + base, d & 7, xf);
        float c[KH_T];
#pragma unroll
        for (int j = 0; j < KH_T; ++j) c[j] = 0.f;
        const float4* tq = reinterpret_cast<const float4*>(my_taps + rho * 2 * LM);
        const float4* tf = tq + LM / 4;
#pragma unroll
        for (int k4 = 0; k4 < LM / 4; ++k4) {
          const float4 a4 = tq[k4];
          const float4 b4 = tf[k4];
          const float av[4] = {a4.x, a4.y, a4.z, a4.w};
          const float bv[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int k = 4 * k4 + q;
#pragma unroll
            for (int j = 0; j < KH_T; ++j) {
              c[j] = fmaf(av[q], xq[j + LM - 1 - k], c[j]);
              c[j] = fmaf(bv[q], xf[j + LM - 1 - k], c[j]);
            }
          }
        }
        // compensated accumulation over surface points
#pragma unroll
        for (int j = 0; j < KH_T; ++j) {
          const float y = __fsub_rn(c[j], comp[rho][j]);
          const float t = __fadd_rn(sum[rho][j], y);
          comp[rho][j] = __fsub_rn(__fsub_rn(t, sum[rho][j]), y);
          sum[rho][j] = t;
        }
      }
      __syncwarp();  // taps of the next surface point overwrite the buffer
    }
  }

  // outputs: lane owns samples tb + 8*lane .. +7 of each of its targets
#pragma unroll
  for (int rho = 0; rho < KH_RW; ++rho) {
    const int r = r_base + warp * KH_RW + rho;
    if (r >= p.nr) continue;
    const int t0 = tb + KH_T * lane;
    float* o = p.out + (size_t)r * p.nt + t0;
    if (t0 + KH_T <= p.nt && ((p.nt & 3) == 0)) {
      reinterpret_cast<float4*>(o)[0] = make_float4(sum[rho][0], sum[rho][1], sum[rho][2], sum[rho][3]);
      reinterpret_cast<float4*>(o)[1] = make_float4(sum[rho][4], sum[rho][5], sum[rho][6], sum[rho][7]);
    } else {
#pragma unroll
      for (int j = 0; j < KH_T; ++j)
        if (t0 + j < p.nt) o[j] = sum[rho][j];
    }
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

namespace {

template <typename T>
struct DevBuf {
  T* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  bool alloc(size_t n) { return cudaMalloc(&p, n * sizeof(T)) == cudaSuccess; }
};

}  // namespace

}  // namespace adf

using namespace adf;

extern "C" int adf_kh_pressure(adf_ctx* ctx, const adf_kh_desc* d, const float* in_q,
                               const float* in_f, float* out) {
  if (!ctx || !d || !in_q || !in_f || !out || !d->s_pts || !d->s_nrm || !d->r_pts)
    return fail(ADF_E_ARG, "adf_kh_pressure: null argument");
  if (d->ns < 1 || d->nr < 1 || d->nt < 1 || !(d->dt > 0) || !(d->sigma > 0) || !(d->c0 > 0))
    return fail(ADF_E_ARG, "adf_kh_pressure: ns, nr, nt, dt, sigma and c0 must be positive");
  if (d->ns > (1 << 30) || d->nr > (1 << 30) || d->nt > (1 << 28))
    return fail(ADF_E_ARG, "adf_kh_pressure: sizes out of range");
  const double ws = d->window_sigmas > 0 ? d->window_sigmas : 6.0;
  const double hw = ws * d->sigma / d->dt;
  const int taps = (int)std::floor(2.0 * hw) + 1;
  int lm = 0;
  if (taps <= 16) lm = 16;
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
  const int ntiles = (nr + KH_RT - 1) / KH_RT;
  std::vector<int2> tlo((size_t)ntiles);
  int wmax = 0;
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
    wmax = std::max(wmax, KH_TB + (lo_max - lo_min) + lm - 1);
  }
  // multiple of 4 floats so the tap buffer behind the rows stays 16-B aligned
  const int rowpad = ((wmax - 1) + ((wmax - 1) >> 3) + 1 + 3) / 4 * 4;
  const size_t tap_bytes = (size_t)KH_WARPS * KH_RW * 2 * lm * 4;
  const size_t per_s = (size_t)2 * rowpad * 4 + (size_t)6 * KH_RT * 4;
  int sc = KH_SC_MAX;
  while (sc > 1 && per_s * sc + tap_bytes > (size_t)ctx->smem_optin) --sc;
  const size_t smem = per_s * sc + tap_bytes;
  if (smem > (size_t)ctx->smem_optin)
    return fail(ADF_E_ARG, "adf_kh_pressure: the targets' delay spread needs a " +
                               std::to_string(wmax) + "-sample window, more than shared memory holds");

  DevBuf<double> dsp, dsn, drp;
  DevBuf<float> dq, df, dout;
  DevBuf<int2> dtlo;
  DevBuf<int> derr;
  if (!dsp.alloc((size_t)3 * ns) || !dsn.alloc((size_t)3 * ns) || !drp.alloc((size_t)3 * nr) ||
      !dq.alloc((size_t)nt * ns) || !df.alloc((size_t)nt * ns) || !dout.alloc((size_t)nt * nr) ||
      !dtlo.alloc((size_t)ntiles) || !derr.alloc(1))
    return fail(ADF_E_NOMEM, "adf_kh_pressure: device allocation failed");
  cudaStream_t st = ctx->stream;
  cudaMemcpyAsync(dsp.p, d->s_pts, (size_t)24 * ns, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dsn.p, d->s_nrm, (size_t)24 * ns, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(drp.p, d->r_pts, (size_t)24 * nr, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dq.p, in_q, (size_t)4 * nt * ns, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(df.p, in_f, (size_t)4 * nt * ns, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dtlo.p, tlo.data(), sizeof(int2) * ntiles, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(derr.p, 0, sizeof(int), st);

  KhParams p;
  p.ns = ns; p.nr = nr; p.nt = nt;
  p.sc = sc; p.wlen = wmax; p.rowpad = rowpad;
  p.inv_c0dt = inv_c0dt;
  p.hw = hw;
  const double C = 1.0 / (std::sqrt(2.0 * M_PI) * d->sigma);
  const double s2 = d->sigma * d->sigma;
  p.cq = -d->aq * C * d->dt / s2;
  p.cf1 = d->af * C;
  p.cf2 = -d->af * C * d->dt / (s2 * d->c0);
  p.a = (float)(d->dt * d->dt / (2.0 * s2));
  p.sp = dsp.p; p.sn = dsn.p; p.rp = drp.p;
  p.tile_lo = dtlo.p;
  p.in_q = dq.p; p.in_f = df.p; p.out = dout.p;
  p.err = derr.p;

  const void* fn = lm == 16 ? (const void*)adf_kh_pressure_kernel<16>
                            : (const void*)adf_kh_pressure_kernel<32>;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, std::string("kh smem: ") + cudaGetErrorString(e));
  const dim3 grid((unsigned)ntiles, (unsigned)((nt + KH_TB - 1) / KH_TB));
  cudaEventRecord(ctx->ev0, st);
  if (lm == 16)
    adf_kh_pressure_kernel<16><<<grid, KH_THREADS, smem, st>>>(p);
  else
    adf_kh_pressure_kernel<32><<<grid, KH_THREADS, smem, st>>>(p);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, std::string("kh launch: ") + cudaGetErrorString(e));
  cudaEventRecord(ctx->ev1, st);
  int herr = 0;
  cudaMemcpyAsync(out, dout.p, (size_t)4 * nt * nr, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&herr, derr.p, sizeof(int), cudaMemcpyDeviceToHost, st);
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  ctx->last_ms = ms;
  ctx->launches = 1;
  ctx->h2d_bytes = (int64_t)48 * ns + 24 * (int64_t)nr + (int64_t)8 * nt * ns;
  ctx->d2h_bytes = (int64_t)4 * nt * nr;
  if (herr) return fail(ADF_E_STATE, "adf_kh_pressure: a pair's delay fell outside its tile bound");
  return ADF_OK;
}

extern "C" int adf_fp32_fma_peak(adf_ctx* ctx, double* tflops, double* ms_out) {
  if (!ctx || !tflops) return fail(ADF_E_ARG, "adf_fp32_fma_peak: null argument");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  const int blocks = ctx->nsm * 8, iters = 4096;
  DevBuf<float> o;
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
