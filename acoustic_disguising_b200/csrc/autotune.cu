// autotune.cu -- per-grid-size choice of the step kernel's tile shape.
//
// For one grid size, runs a short batch of synthetic impulsive GF solves
// (CPML, a centred rigid sphere, a point source and a receiver shell: the
// work mix of the serving stream) once per candidate (tile rows, z-chunk
// depth), times the fused step kernel with per-launch CUDA events, and stores
// the fastest shape in the tune table that later solves of that size read.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "runtime.h"

using namespace adf;

extern "C" int adf_autotune(adf_ctx* ctx, int64_t nx, int64_t ny, int64_t nz, int64_t npml,
                            int n_solves, int steps, int* best_ty, int* best_nzc,
                            double* best_ms) {
  if (!ctx || nx < 8 || ny < 8 || nz < 8 || npml < 0 || n_solves < 1 || steps < 4)
    return fail(ADF_E_ARG, "adf_autotune: bad arguments");
  const double dx = 0.005, c0 = 343.0, rho = 1.2;
  const double dt = 0.5 * dx / c0 / std::sqrt(3.0);
  adf_domain d;
  int rc = adf_domain_make((steps - 0.5) * dt, (nx - 1) * dx / 2, (ny - 1) * dx / 2,
                           (nz - 1) * dx / 2, nx, ny, nz, c0, rho, 0.5, &d);
  if (rc) return rc;
  if (d.nt != steps) return fail(ADF_E_STATE, "adf_autotune: step count mismatch");
  const double rmin = std::min(d.xmax, std::min(d.ymax, d.zmax));
  // Gaussian pulse source, 64-point receiver shell (Fibonacci sphere)
  std::vector<double> tf((size_t)steps);
  for (int t = 0; t < steps; ++t) tf[t] = std::exp(-0.5 * std::pow((t - 20.0) / 5.0, 2));
  const int nrec = 64;
  std::vector<double> rp(3 * nrec), rn(3 * nrec);
  for (int i = 0; i < nrec; ++i) {
    const double z = 1.0 - (2.0 * i + 1.0) / nrec, rxy = std::sqrt(std::max(0.0, 1 - z * z));
    const double th = M_PI * (3.0 - std::sqrt(5.0)) * i;
    const double n[3] = {rxy * std::cos(th), rxy * std::sin(th), z};
    for (int a = 0; a < 3; ++a) {
      rn[3 * i + a] = n[a];
      rp[3 * i + a] = 0.6 * rmin * n[a];
    }
  }
  std::vector<float> out_p((size_t)n_solves * steps * nrec), out_vn(out_p.size());
  std::vector<adf_gf_request> reqs((size_t)n_solves);
  for (int k = 0; k < n_solves; ++k) {
    adf_gf_request& r = reqs[(size_t)k];
    std::memset(&r, 0, sizeof(r));
    r.dom = d;
    r.npml = npml;
    r.pml_rcoef = 1e-4;
    r.pml_fc = 2000.0;
    r.shape = ADF_SHAPE_SPHERE;
    r.shape_params[0] = 0.1 * rmin;
    const double a = 2 * M_PI * k / n_solves;
    r.src_point[0] = 0.8 * rmin * std::cos(a);
    r.src_point[1] = 0.8 * rmin * std::sin(a);
    r.src_dir[0] = 1.0;
    r.src_tf = tf.data();
    r.n_rec = nrec;
    r.rec_points = rp.data();
    r.rec_normals = rn.data();
    r.flags = ADF_ARITH_PROMOTE;
    r.out_p = out_p.data() + (size_t)k * steps * nrec;
    r.out_vn = out_vn.data() + (size_t)k * steps * nrec;
  }
  std::vector<std::pair<int, int>> cand;
  const int tys[] = {3, 5, 7};
  const int nzcs[] = {8, 16, 32};
  for (int ty : tys)
    for (int nzc : nzcs)
      if (ty <= ny && nzc <= nz) cand.push_back({ty, nzc});
  const bool timing_was = ctx->kernel_timing;
  adf_set_kernel_timing(ctx, 1);
  double best = 1e300;
  int bty = 0, bnzc = 0;
  std::string last_err;
  for (auto [ty, nzc] : cand) {
    tune_force(Tune{ty, nzc});
    adf_kernel_timing(ctx, nullptr, nullptr, 1);
    const int r = adf_gf_solve_batch(ctx, n_solves, reqs.data(), 1);
    double ms = 0;
    int64_t n = 0;
    adf_kernel_timing(ctx, &ms, &n, 1);
    if (r != ADF_OK || n == 0) {  // shape does not fit this grid: skip it
      char buf[256];
      adf_last_error(buf, sizeof(buf));
      last_err = buf;
      continue;
    }
    const double per = ms / (double)n;
    if (per < best) {
      best = per;
      bty = ty;
      bnzc = nzc;
    }
  }
  tune_force(Tune{0, 0});
  adf_set_kernel_timing(ctx, timing_was ? 1 : 0);
  if (bty == 0) return fail(ADF_E_STATE, "adf_autotune: no candidate ran: " + last_err);
  if (tune_store((int)nx, (int)ny, (int)nz, Tune{bty, bnzc}) != ADF_OK)
    return fail(ADF_E_ARG, "adf_autotune: cannot write the tune table");
  if (best_ty) *best_ty = bty;
  if (best_nzc) *best_nzc = bnzc;
  if (best_ms) *best_ms = best;
  return ADF_OK;
}
