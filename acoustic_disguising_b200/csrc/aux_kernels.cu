// aux_kernels.cu -- FP64 set-up kernels (compiled with --fmad=false so no
// multiply-add is contracted: the reference evaluates every product and sum
// separately in Float64).
//
//  * CPML damping profiles: calc_Kab_CPML (src/kernels/cpmlcoeffs.jl:65-126)
//  * scatterer update mask -> 4-bit-per-cell bitmask: _outside_predicate +
//    build_scatterer + build_update_mask (src/geometry.jl:86-176, 250-280)
//  * C_f / C_q injection coefficients: C_for_N
//    (diagnostics/_check_inject_kh/injection_coefficients.jl:467-472)
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/adfdtd.h"

namespace adf {

// One thread per profile entry.  t in [0, 2n) ongrd (left then right),
// [2n, 2n + 2(n+1)) halfgrd.  Output order a_l a_r a_hl a_hr b_l b_r b_hl b_hr.
__global__ void adf_cpml_profile_kernel(int n, double vel_max, double dt, double rcoef,
                                        double thickness, double f0, float* out32,
                                        double* out64) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int total = 2 * n + 2 * (n + 1);
  if (t >= total) return;
  const bool half = t >= 2 * n;
  const int m = half ? n + 1 : n;           // Kab_size
  const int u = half ? t - 2 * n : t;
  const bool right = u >= m;
  const int i = right ? u - m : u;          // 0-based element
  const double shift = half ? 0.5 : 0.0;
  const double alpha_max = 3.141592653589793 * f0;
  const double npower = 2.0;
  double d0 = -(npower + 1) * vel_max * log(rcoef) / (2.0 * thickness);
  if (n == 0) d0 = 0.0;
  // LinRange(0 - shift, m - shift - 1, m)[k] = (1-t)*a + t*b, t = (k-1)/max(1,m-1)
  auto dist = [&](int k0) {
    if (half && k0 == 0) return 0.0;  // dist[1] = 0 on the half grid
    const double a = 0 - shift, b = (double)m - shift - 1;
    const double tt = (double)k0 / (double)(m > 1 ? m - 1 : 1);
    return (1 - tt) * a + tt * b;
  };
  double nd = right ? dist(i) : dist(m - 1 - i);
  if (n != 0) nd = nd / (double)n;
  const double dd = d0 * (nd * nd);
  const double alpha = alpha_max * (1.0 - nd);
  const double b = exp(-(dd / 1.0 + alpha) * dt);
  const double a = dd * (b - 1.0) / (1.0 * (dd + 1.0 * alpha));
  // offsets of the eight arrays
  const int oa = half ? 2 * n + (right ? n + 1 : 0) : (right ? n : 0);
  const int ob = 4 * n + 2 + oa;
  out32[oa + i] = (float)a;
  out32[ob + i] = (float)b;
  if (out64) {
    out64[oa + i] = a;
    out64[ob + i] = b;
  }
}

struct ShapeDev {
  int kind;
  double p[6];
};

// `true` when (x,y,z) lies strictly outside the scatterer (geometry.jl:86-143)
__device__ __forceinline__ bool outside(const ShapeDev& s, double x, double y, double z) {
  switch (s.kind) {
    case 1: {  // sphere: x^2 + y^2 + z^2 > r^2 (centre 0 reproduces the reference)
      double r = s.p[0], xx = x - s.p[1], yy = y - s.p[2], zz = z - s.p[3];
      return xx * xx + yy * yy + zz * zz > r * r;
    }
    case 2: {  // cube: |x| > l/2 || |y| > l/2 || |z| > l/2
      double r = s.p[0], xx = x - s.p[1], yy = y - s.p[2], zz = z - s.p[3];
      return fabs(xx) > r / 2 || fabs(yy) > r / 2 || fabs(zz) > r / 2;
    }
    case 3: {  // 3-D Greek cross
      double l = s.p[0], h = l / 2, sl = 2.0 * l / 3;
      auto in = [h](double a, double b, double c) {
        return fabs(a) < h && fabs(b) < h && fabs(c) < h;
      };
      if (!in(x, y, z)) return true;
      if (in(x + sl, y + sl, z) || in(x - sl, y - sl, z) || in(x + sl, y - sl, z) ||
          in(x - sl, y + sl, z))
        return true;
      if (in(x + sl, y, z + sl) || in(x - sl, y, z - sl) || in(x + sl, y, z - sl) ||
          in(x - sl, y, z + sl))
        return true;
      if (in(x, y + sl, z + sl) || in(x, y - sl, z - sl) || in(x, y + sl, z - sl) ||
          in(x, y - sl, z + sl))
        return true;
      return false;
    }
    case 4: {  // ellipsoid (extension), same strict cell-centre rule
      double xx = (x - s.p[3]) / s.p[0], yy = (y - s.p[4]) / s.p[1], zz = (z - s.p[5]) / s.p[2];
      return xx * xx + yy * yy + zz * zz > 1.0;
    }
    default:
      return true;
  }
}

// One thread per mask word (8 cells along x).  bits per cell: 0 P open
// (fluid), 1 Vx face open, 2 Vy, 3 Vz (both neighbours fluid; the first
// index strip along the face's axis stays closed).  Optionally also writes
// the reference's (nx,ny,nz,4) Bool layout.
__global__ void adf_mask_kernel(ShapeDev s, const double* __restrict__ xs,
                                const double* __restrict__ ys, const double* __restrict__ zs,
                                int nx, int ny, int nz, int mw, uint32_t* bits,
                                uint8_t* jl) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long total = (long long)mw * ny * nz;
  if (t >= total) return;
  const int w = (int)(t % mw);
  const long long jk = t / mw;
  const int j = (int)(jk % ny), k = (int)(jk / ny);
  uint32_t word = 0;
  const long long N = (long long)nx * ny * nz;
  bool prev_solid = false;
  if (8 * w >= 1 && 8 * w - 1 < nx) prev_solid = !outside(s, xs[8 * w - 1], ys[j], zs[k]);
  for (int e = 0; e < 8; ++e) {
    const int i = 8 * w + e;
    if (i >= nx) break;
    const bool sd = !outside(s, xs[i], ys[j], zs[k]);
    const bool sy = j >= 1 ? !outside(s, xs[i], ys[j - 1], zs[k]) : true;
    const bool sz = k >= 1 ? !outside(s, xs[i], ys[j], zs[k - 1]) : true;
    const bool p = !sd;
    const bool vx = i >= 1 && !prev_solid && !sd;
    const bool vy = j >= 1 && !sy && !sd;
    const bool vz = k >= 1 && !sz && !sd;
    word |= (uint32_t)(p | (vx << 1) | (vy << 2) | (vz << 3)) << (4 * e);
    prev_solid = sd;
    if (jl) {
      const long long o = i + (long long)nx * (j + (long long)ny * k);
      jl[o] = p;
      jl[o + N] = vx;
      jl[o + 2 * N] = vy;
      jl[o + 3 * N] = vz;
    }
  }
  bits[t] = word;
}

// Pack a reference Bool mask (nx,ny,nz,4) into the bitmask layout.
__global__ void adf_pack_mask_kernel(const uint8_t* __restrict__ jl, int nx, int ny, int nz,
                                     int mw, uint32_t* bits) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long total = (long long)mw * ny * nz;
  if (t >= total) return;
  const int w = (int)(t % mw);
  const long long jk = t / mw;
  const int j = (int)(jk % ny), k = (int)(jk / ny);
  const long long N = (long long)nx * ny * nz;
  uint32_t word = 0;
  for (int e = 0; e < 8; ++e) {
    const int i = 8 * w + e;
    if (i >= nx) break;
    const long long o = i + (long long)nx * (j + (long long)ny * k);
    uint32_t nib = (jl[o] ? 1u : 0u) | (jl[o + N] ? 2u : 0u) | (jl[o + 2 * N] ? 4u : 0u) |
                   (jl[o + 3 * N] ? 8u : 0u);
    word |= nib << (4 * e);
  }
  bits[t] = word;
}

// C_for_N: dS = 4 pi R^2 / N (fib_sphere_area), C_f = dS dt / (rho dx^3),
// C_q = C_f z0^2
__global__ void adf_injection_coef_kernel(double radius, long long n, double dt, double rho,
                                          double dx, double z0, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double pi = 3.141592653589793;
  const double dS = 4 * pi * (radius * radius) / (double)n;
  const double cf = dS * dt / (rho * (dx * dx * dx));
  out[0] = cf;
  out[1] = cf * (z0 * z0);
  out[2] = dS;
}

// Scale traces by a Float64 coefficient and round to Float32:
// Float32.(C * trace) as inject_inner_sources! stores it (fdtd_runners.jl:39-45)
__global__ void adf_scale_traces_kernel(const float* __restrict__ in, float* out, long long n,
                                        const double* coef, int which) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) out[t] = (float)(coef[which] * (double)in[t]);
}

cudaError_t launch_cpml_profiles(int n, double vel_max, double dt, double rcoef, double thickness,
                                 double f0, float* out32, double* out64, cudaStream_t s) {
  int total = 4 * n + 2;
  adf_cpml_profile_kernel<<<(total + 63) / 64, 64, 0, s>>>(n, vel_max, dt, rcoef, thickness, f0,
                                                           out32, out64);
  return cudaGetLastError();
}

cudaError_t launch_mask(int kind, const double* params, const double* xs, const double* ys,
                        const double* zs, int nx, int ny, int nz, int mw, uint32_t* bits,
                        uint8_t* jl, cudaStream_t s) {
  ShapeDev sd;
  sd.kind = kind;
  for (int i = 0; i < 6; ++i) sd.p[i] = params ? params[i] : 0.0;
  long long total = (long long)mw * ny * nz;
  adf_mask_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(sd, xs, ys, zs, nx, ny, nz, mw,
                                                                 bits, jl);
  return cudaGetLastError();
}

cudaError_t launch_pack_mask(const uint8_t* jl, int nx, int ny, int nz, int mw, uint32_t* bits,
                             cudaStream_t s) {
  long long total = (long long)mw * ny * nz;
  adf_pack_mask_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(jl, nx, ny, nz, mw, bits);
  return cudaGetLastError();
}

cudaError_t launch_injection_coef(double radius, long long n, double dt, double rho, double dx,
                                  double z0, double* out, cudaStream_t s) {
  adf_injection_coef_kernel<<<1, 32, 0, s>>>(radius, n, dt, rho, dx, z0, out);
  return cudaGetLastError();
}

cudaError_t launch_scale_traces(const float* in, float* out, long long n, const double* coef,
                                int which, cudaStream_t s) {
  adf_scale_traces_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(in, out, n, coef, which);
  return cudaGetLastError();
}

// ---- impulsive_gfs post-processing (src/greens.jl:174-190, resample.jl:32-76,
// greens_io.jl:195-205), one source's traces (nt_in, ncol) column-major.
// Prefilter: one thread per column -- denoise at 1e-4 of the column's
// (signed) maximum, then the natural cubic B-spline coefficients
// c_0..c_{n+1} of Line(OnGrid()) ends: c_1 = y_1, c_n = y_n and
// (c_{i-1} + 4 c_i + c_{i+1}) / 6 = y_i in between (Thomas algorithm; the
// pivots cpv depend only on i and are shared by all columns).
__global__ void adf_gf_prefilter_kernel(int ncol, int n, const float* __restrict__ in,
                                        const double* __restrict__ cpv, double* coef,
                                        int denoise) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  const float* a = in + (long long)n * c;
  double* cf = coef + (long long)(n + 2) * c;
  float mx = a[0];
  for (int t = 1; t < n; ++t) mx = fmaxf(mx, a[t]);
  const double thr = 1e-4 * (double)mx;
  auto y = [&](int t1) {  // 1-based sample, denoised
    const float v = a[t1 - 1];
    return (denoise && (double)fabsf(v) < thr) ? 0.0 : (double)v;
  };
  cf[1] = y(1);
  cf[n] = y(n);
  // forward sweep: cf[i] holds d'_i
  for (int i = 2; i <= n - 1; ++i) {
    double rhs = 6.0 * y(i);
    if (i == 2) rhs -= cf[1];
    if (i == n - 1) rhs -= cf[n];
    const double b = 4.0 - (i > 2 ? cpv[i - 1] : 0.0);
    cf[i] = (rhs - (i > 2 ? cf[i - 1] : 0.0)) / b;
  }
  for (int i = n - 2; i >= 2; --i) cf[i] = cf[i] - cpv[i] * cf[i + 1];
  cf[0] = 2.0 * cf[1] - cf[2];
  cf[n + 1] = 2.0 * cf[n] - cf[n - 1];
}

// Evaluation: one thread per output sample and column; Flat() outside the
// input axis, times dt_out/dt_in, rounded to Float32, divided by unit32.
__global__ void adf_gf_resample_kernel(int ncol, int n, int nt_out, double t_in0, double dt_in,
                                       double t_out0, double dt_out, const double* coef,
                                       float* out, float unit32) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= (long long)nt_out * ncol) return;
  const int c = (int)(k / nt_out), j = (int)(k - (long long)c * nt_out);
  const double* cf = coef + (long long)(n + 2) * c;
  const double tt = t_out0 + (double)j * dt_out;
  double x = (tt - t_in0) / dt_in + 1.0;
  x = fmin(fmax(x, 1.0), (double)n);
  int i = (int)floor(x);
  if (i > n - 1) i = n - 1;
  const double d = x - (double)i, e = 1.0 - d;
  const double w0 = e * e * e / 6.0, w3 = d * d * d / 6.0;
  const double w1 = (3.0 * d * d * d - 6.0 * d * d + 4.0) / 6.0;
  const double w2 = (-3.0 * d * d * d + 3.0 * d * d + 3.0 * d + 1.0) / 6.0;
  const double v = cf[i - 1] * w0 + cf[i] * w1 + cf[i + 1] * w2 + cf[i + 2] * w3;
  out[k] = __fdiv_rn((float)(v * (dt_out / dt_in)), unit32);
}

cudaError_t launch_gf_postprocess(int ncol, int n, int nt_out, double t_in0, double dt_in,
                                  double t_out0, double dt_out, const float* in,
                                  const double* cpv, double* coef, float* out, float unit32,
                                  int denoise, cudaStream_t s) {
  adf_gf_prefilter_kernel<<<(ncol + 127) / 128, 128, 0, s>>>(ncol, n, in, cpv, coef, denoise);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const long long tot = (long long)nt_out * ncol;
  adf_gf_resample_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(
      ncol, n, nt_out, t_in0, dt_in, t_out0, dt_out, coef, out, unit32);
  return cudaGetLastError();
}

// Fixed scratch for adf_cpml_profiles_static: room for the profiles of
// npml <= kStaticCpmlMaxNpml (8*npml+4 values) in Float64 followed by Float32.
// Nothing in it has to start at zero: the profile kernel writes every value
// that the copies back to the host read.
constexpr int kStaticCpmlMaxNpml = ADF_STATIC_CPML_MAX_NPML;
constexpr int kStaticCpmlMaxVals = 8 * kStaticCpmlMaxNpml + 4;
static __device__ __align__(256) double g_cpml_scratch[kStaticCpmlMaxVals + kStaticCpmlMaxVals / 2 + 1];

int static_cpml_max_npml() { return kStaticCpmlMaxNpml; }
extern "C" int adf_static_cpml_max_npml(void) { return kStaticCpmlMaxNpml; }

// Device address of the scratch on the current device.  Taking it is the one
// set-up step (it may load this module onto the device), so callers do it
// once per device and keep the pointer.
cudaError_t static_cpml_scratch(double** d64, float** d32) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_cpml_scratch);
  if (e != cudaSuccess) return e;
  *d64 = static_cast<double*>(p);
  *d32 = reinterpret_cast<float*>(static_cast<double*>(p) + kStaticCpmlMaxVals);
  return cudaSuccess;
}

}  // namespace adf
