// setup.cu -- solve set-up helpers: device mask construction and the
// host-side transceiver packing of transceiversToGrid.
#include <cstring>
#include <vector>

#include "runtime.h"

namespace adf {
cudaError_t launch_mask(int kind, const double* params, const double* xs, const double* ys,
                        const double* zs, int nx, int ny, int nz, int mw, uint32_t* bits,
                        uint8_t* jl, cudaStream_t s);

// Cell-centre coordinates are the reference's Float64 range values
// (geometry.jl:162-165); the predicate runs in FP64 on the device.
int build_mask_device(adf_ctx* ctx, const adf_domain& d, int shape, const double* params, int mw,
                      uint32_t** bits, uint8_t** jl) {
  hm::Dom dom;
  dom.xmax = d.xmax; dom.ymax = d.ymax; dom.zmax = d.zmax;
  dom.nx = d.nx; dom.ny = d.ny; dom.nz = d.nz;
  dom.dx = d.dx; dom.dy = d.dy; dom.dz = d.dz;
  std::vector<double> xyz((size_t)(d.nx + d.ny + d.nz));
  for (int a = 0; a < 3; ++a) {
    hm::Range r = hm::axis_range(dom, a, 0);
    double* o = xyz.data() + (a == 0 ? 0 : a == 1 ? d.nx : d.nx + d.ny);
    for (int64_t i = 1; i <= r.len; ++i) o[i - 1] = r.at(i);
  }
  double* dxyz = nullptr;
  if (cudaMalloc(&dxyz, xyz.size() * 8) != cudaSuccess) return fail(ADF_E_NOMEM, "alloc");
  const size_t words = (size_t)mw * d.ny * d.nz;
  if (cudaMalloc((void**)bits, words * 4) != cudaSuccess) {
    cudaFree(dxyz);
    return fail(ADF_E_NOMEM, "alloc");
  }
  if (jl && cudaMalloc((void**)jl, (size_t)4 * d.nx * d.ny * d.nz) != cudaSuccess) {
    cudaFree(dxyz);
    cudaFree(*bits);
    return fail(ADF_E_NOMEM, "alloc");
  }
  cudaError_t e =
      cudaMemcpyAsync(dxyz, xyz.data(), xyz.size() * 8, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = launch_mask(shape, params, dxyz, dxyz + d.nx, dxyz + d.nx + d.ny, (int)d.nx, (int)d.ny,
                    (int)d.nz, mw, *bits, jl ? *jl : nullptr, ctx->stream);
  const cudaError_t es = cudaStreamSynchronize(ctx->stream);  // xyz outlives its copy
  if (e == cudaSuccess) e = es;
  cudaFree(dxyz);
  if (e != cudaSuccess) {
    cudaFree(*bits);
    *bits = nullptr;
    if (jl) {
      cudaFree(*jl);
      *jl = nullptr;
    }
    cudaGetLastError();
    return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  }
  return ADF_OK;
}

// transceiversToGrid (simulation.jl:387-431): indices and weights stored as
// Float32, src = Float32(tf * direction[c]), rec = Float32(src * 0).
int pack_transceivers_host(const hm::Dom& d, const double* points, const double* dirs,
                           const double* tf, adf_txgrid* o) {
  const int64_t ntx = o->ntx, nt = o->nt;
  for (int64_t is = 0; is < ntx; ++is) {
    int64_t idx[12];
    double w[32];
    if (!hm::trilinear(d, points + 3 * is, idx, w))
      return fail(ADF_E_ARG, "transceiver " + std::to_string(is) + " lies outside the grid");
    for (int c = 0; c < 4; ++c) {
      for (int q = 0; q < 3; ++q) o->idx[c][3 * is + q] = (float)idx[3 * c + q];
      for (int q = 0; q < 8; ++q) o->w[c][8 * is + q] = (float)w[8 * c + q];
      const double dc = dirs[4 * is + c];
      for (int64_t t = 0; t < nt; ++t) {
        const double v = tf[t + nt * is] * dc;
        o->src[c][t + nt * is] = (float)v;
        o->rec[c][t + nt * is] = (float)(v * 0);
      }
    }
    for (int q = 0; q < 4; ++q) o->dir[4 * is + q] = (float)dirs[4 * is + q];
    for (int64_t t = 0; t < nt; ++t) {
      o->vn_src[t + nt * is] = 0.0f;
      o->vn_rec[t + nt * is] = 0.0f;
    }
  }
  return ADF_OK;
}

}  // namespace adf
