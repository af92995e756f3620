// runtime.cu -- host runtime behind the C-ABI (include/adfdtd.h).
//
// Owns device memory, builds the per-solve descriptors, entry lists and work
// items, and drives the fused step kernel.  Layout conversions between
// the reference's Julia arrays and the HBM layout (see adf_internal.h) happen
// here, once per call.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/adfdtd.h"
#include "adf_internal.h"
#include "host_math.h"
#include <cuda.h>
#include <cudaTypedefs.h>

#include "runtime.h"

namespace adf {
cudaError_t launch_cpml_profiles(int n, double vel_max, double dt, double rcoef, double thickness,
                                 double f0, float* out32, double* out64, cudaStream_t s);
cudaError_t launch_mask(int kind, const double* params, const double* xs, const double* ys,
                        const double* zs, int nx, int ny, int nz, int mw, uint32_t* bits,
                        uint8_t* jl, cudaStream_t s);
cudaError_t launch_pack_mask(const uint8_t* jl, int nx, int ny, int nz, int mw, uint32_t* bits,
                             cudaStream_t s);
cudaError_t launch_injection_coef(double radius, long long n, double dt, double rho, double dx,
                                  double z0, double* out, cudaStream_t s);
cudaError_t launch_gf_postprocess(int ncol, int n, int nt_out, double t_in0, double dt_in,
                                  double t_out0, double dt_out, const float* in,
                                  const double* cpv, double* coef, float* out, float unit32,
                                  int denoise, cudaStream_t s);
int static_cpml_max_npml();
cudaError_t static_cpml_scratch(double** d64, float** d32);

thread_local std::string g_err;
int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}


// ---------------------------------------------------------------------------
// Solve: device resources of one FDTD solve
// ---------------------------------------------------------------------------
Solve::~Solve() { release(); }

void Solve::release() {
  for (void* p : allocs)
    if (p) {
      if (alloc_stream)
        cudaFreeAsync(p, alloc_stream);
      else
        cudaFree(p);
    }
  allocs.clear();
}

template <typename T>
static T* dalloc(Solve& s, size_t n, int& rc) {
  void* p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = s.alloc_stream
                      ? cudaMallocFromPoolAsync(&p, n * sizeof(T), s.alloc_pool, s.alloc_stream)
                      : cudaMalloc(&p, n * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    rc = fail(ADF_E_NOMEM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
    return nullptr;
  }
  s.allocs.push_back(p);
  s.bytes += n * sizeof(T);
  return static_cast<T*>(p);
}

void choose_tiles(int nx, int ny, int nz, int& nxp, int& ty, int& nzc, int& mw) {
  nxp = (nx + 3) / 4 * 4;
  mw = ((nx + 7) / 8 + 3) / 4 * 4;
  const Tune t = tune_lookup(nx, ny, nz);
  ty = t.ty;
  nzc = t.nzc;
  if (ty < 2) ty = 2;
  if (ty > step_max_ty()) ty = step_max_ty();
  if (ty > ny) ty = ny;
  if (nzc < 2) nzc = 2;
  if (nzc > nz) nzc = nz;
}

size_t solve_bytes_estimate(int64_t nx, int64_t ny, int64_t nz, int64_t npml, int64_t ntx,
                            int64_t nt, bool mask) {
  int nxp, ty, nzc, mw;
  choose_tiles((int)nx, (int)ny, (int)nz, nxp, ty, nzc, mw);
  size_t b = 2ull * 4 * nz * ny * nxp * 4;
  if (mask) b += (size_t)mw * ny * nz * 4;
  size_t n = npml;
  b += 2ull * 2 * 4 * (nz * ny * n + nz * n * nxp + n * ny * nxp);
  b += 2ull * 2 * 4 * (nz * ny * (n + 1) + nz * (n + 1) * nxp + (n + 1) * ny * nxp);
  b += 10ull * nt * ntx * 4;
  b += (size_t)ntx * 4 * 8 * 4 * 3;  // contributions + entries
  b += (size_t)((ny + ty - 1) / ty) * nz * 4 * 4;
  return b + (1 << 20);
}

// Entry lists for interp_trilinear! (derivatives.jl:30-60): every in-bounds
// (channel, transceiver) contributes its 8 stencil corners; corners are
// grouped by (y tile, plane, channel) and, inside a cell, kept in
// transceiver order (the order of the sequential reference loop).  P
// corners on the last row of a tile are duplicated (slot -1) into the next
// tile's halo row so that tile's velocity update sees the injection.
static int build_entries(Solve& s, const float* const idx[4], const float* const w[4],
                         const int* src_col) {
  SolveDev& d = s.dev;
  const int ntx = d.ntx, nx = d.nx, ny = d.ny, nz = d.nz, ty = d.ty, nxp = d.nxp;
  struct E {
    long long key;  // bucket * 2^32 + cell
    int tx;
    int slot;
    float w;
    int col;        // src column, -1 when the transceiver never injects
  };
  std::vector<E> es;
  es.reserve((size_t)ntx * 36);
  std::vector<unsigned char> inb((size_t)4 * ntx, 0);
  for (int c = 0; c < 4; ++c)
    for (int tx = 0; tx < ntx; ++tx) {
      const int I = (int)idx[c][3 * tx], J = (int)idx[c][3 * tx + 1], K = (int)idx[c][3 * tx + 2];
      const bool ok = I >= 1 && I < nx && J >= 1 && J < ny && K >= 1 && K < nz;
      inb[(size_t)c * ntx + tx] = ok;
      if (!ok) continue;
      for (int n = 0; n < 8; ++n) {
        const int ii = n & 1, jj = (n >> 1) & 1, kk = n >> 2;
        const int i = I - 1 + ii, j = J - 1 + jj, k = K - 1 + kk;
        const float wv = w[c][8 * tx + n];
        const int T = j / ty, r = j - T * ty + 1;
        const long long bucket = ((long long)T * nz + k) * 4 + c;
        const int col = src_col ? src_col[tx] : tx;
        es.push_back({(bucket << 32) | (long long)(r * nxp + i), tx, (c * ntx + tx) * 8 + n, wv,
                      col});
        if (c == 0 && (j + 1) % ty == 0 && j + 1 < ny) {
          const long long b2 = ((long long)((j + 1) / ty) * nz + k) * 4;
          es.push_back({(b2 << 32) | (long long)i, tx, -1, wv, col});
        }
      }
    }
  std::stable_sort(es.begin(), es.end(), [](const E& a, const E& b) {
    return a.key < b.key || (a.key == b.key && a.tx < b.tx);
  });
  const long long nb = (long long)d.nty * nz * 4;
  std::vector<int> off((size_t)nb + 1, 0);
  std::vector<int4> seg;
  std::vector<float> ew;
  std::vector<int> etx, eslot;
  ew.reserve(es.size());
  etx.reserve(es.size());
  eslot.reserve(es.size());
  size_t i = 0;
  long long cur_b = 0;
  for (; i < es.size();) {
    const long long b = es[i].key >> 32;
    while (cur_b <= b) off[(size_t)cur_b++] = (int)seg.size();
    size_t j = i;
    while (j < es.size() && es[j].key == es[i].key) ++j;
    // {cell | count<<16, ...}: one entry inline {w, slot, src column},
    // more than one {first entry, 0, 0} into the entry arrays
    const int cell = (int)(es[i].key & 0xffffffffLL);
    const int cnt = (int)(j - i);
    int4 sg;
    sg.x = cell | (cnt << 16);
    if (cnt == 1) {
      std::memcpy(&sg.y, &es[i].w, 4);
      sg.z = es[i].slot;
      sg.w = es[i].col;
    } else {
      sg.y = (int)ew.size();
      sg.z = 0;
      sg.w = 0;
      for (size_t k = i; k < j; ++k) {
        ew.push_back(es[k].w);
        etx.push_back(es[k].col);
        eslot.push_back(es[k].slot);
      }
    }
    seg.push_back(sg);
    i = j;
  }
  while (cur_b <= nb) off[(size_t)cur_b++] = (int)seg.size();
  int rc = ADF_OK;
  int* d_off = dalloc<int>(s, off.size(), rc);
  int4* d_seg = dalloc<int4>(s, seg.size(), rc);
  float* d_w = dalloc<float>(s, ew.size(), rc);
  int* d_tx = dalloc<int>(s, etx.size(), rc);
  int* d_slot = dalloc<int>(s, eslot.size(), rc);
  unsigned char* d_inb = dalloc<unsigned char>(s, inb.size(), rc);
  float* d_contrib = dalloc<float>(s, (size_t)4 * ntx * 8, rc);
  if (rc) return rc;
  cudaStream_t st = s.stream;
  cudaMemcpyAsync(d_off, off.data(), off.size() * 4, cudaMemcpyHostToDevice, st);
  if (!seg.empty())
    cudaMemcpyAsync(d_seg, seg.data(), seg.size() * sizeof(int4), cudaMemcpyHostToDevice, st);
  if (!ew.empty()) {
    cudaMemcpyAsync(d_w, ew.data(), ew.size() * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_tx, etx.data(), etx.size() * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_slot, eslot.data(), eslot.size() * 4, cudaMemcpyHostToDevice, st);
  }
  cudaMemcpyAsync(d_inb, inb.data(), inb.size(), cudaMemcpyHostToDevice, st);
  s.h2d += (int64_t)(off.size() * 4 + seg.size() * sizeof(int4) + ew.size() * 12 + inb.size());
  cudaMemsetAsync(d_contrib, 0, (size_t)4 * ntx * 8 * 4, st);
  // the vectors must outlive the async copies; a failed copy is sticky in
  // the stream or the thread's last error
  cudaError_t e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, std::string("entry upload: ") + cudaGetErrorString(e));
  d.tp_off = d_off;
  d.seg = d_seg;
  d.ent_w = d_w;
  d.ent_tx = d_tx;
  d.ent_slot = d_slot;
  d.inb = d_inb;
  d.contrib = d_contrib;
  s.n_entries = (long long)es.size();
  return ADF_OK;
}

template <typename T>
T* solve_dalloc(Solve& s, size_t n, int& rc) {
  return dalloc<T>(s, n, rc);
}
template float* solve_dalloc<float>(Solve&, size_t, int&);
template int* solve_dalloc<int>(Solve&, size_t, int&);
template double* solve_dalloc<double>(Solve&, size_t, int&);

// The step kernel's TMA descriptors of the two field buffers: 4D tiled maps
// (x: nxp, y: ny, z: nz, channel: 4) with the staged boxes (kStageW, ty+2, 1, 3)
// for P, Vx, Vy and (kStageW, ty+2, 1, 1) for Vz, zero fill outside the grid.  cuTensorMapEncodeTiled comes from the
// driver through the runtime's entry-point query (no link against libcuda).
static int make_field_maps(Solve& s) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    cudaGetLastError();
  });
  if (!encode) return fail(ADF_E_DEVICE, "cuTensorMapEncodeTiled is not available");
  SolveDev& d = s.dev;
  const cuuint64_t dims[4] = {(cuuint64_t)d.nxp, (cuuint64_t)d.ny, (cuuint64_t)d.nz, 4};
  const cuuint64_t strides[3] = {(cuuint64_t)d.nxp * 4, (cuuint64_t)d.nxp * d.ny * 4,
                                 (cuuint64_t)d.chan_stride * 4};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  for (int m4 = 0; m4 < 4; ++m4) {  // buffer b = m4 / 2; box of 3 channels or of Vz
    const int b = m4 / 2;
    const cuuint32_t box[4] = {(cuuint32_t)kStageW, (cuuint32_t)(d.ty + 2), 1,
                               (cuuint32_t)(m4 % 2 ? 1 : 3)};
    CUtensorMap* m = reinterpret_cast<CUtensorMap*>(s.fmap_host + 128 * m4);
    const CUresult r = encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, d.field + b * d.buf_stride,
                              dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
      return fail(ADF_E_DEVICE, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  }
  int rc = ADF_OK;
  void* dm = dalloc<unsigned char>(s, sizeof(s.fmap_host), rc);
  if (rc) return rc;
  if (cudaMemcpyAsync(dm, s.fmap_host, sizeof(s.fmap_host), cudaMemcpyHostToDevice, s.stream) !=
      cudaSuccess) {
    cudaGetLastError();
    return fail(ADF_E_DEVICE, "tensor map upload failed");
  }
  d.fmap = dm;
  return ADF_OK;
}

// Allocates everything except traces; field/psi zeroed.
int solve_alloc(adf_ctx* ctx, Solve& s, const hm::Dom& dom, int npml, bool has_mask, int arith,
                int ntx) {
  SolveDev& d = s.dev;
  std::memset(&d, 0, sizeof(d));
  s.stream = ctx->stream;
  choose_tiles((int)dom.nx, (int)dom.ny, (int)dom.nz, d.nxp, d.ty, s.nzc, d.mw);
  d.nx = (int)dom.nx;
  d.ny = (int)dom.ny;
  d.nz = (int)dom.nz;
  d.nty = (d.ny + d.ty - 1) / d.ty;
  d.npml = npml;
  d.nt = (int)dom.nt;
  d.ntx = ntx;
  d.flags = (has_mask ? SF_MASK : 0) | ((npml > 1 || (has_mask && npml >= 1)) ? SF_PCPML : 0) |
            (npml >= 1 ? SF_VCPML : 0) | (arith == ADF_ARITH_FP32 ? SF_FP32 : 0);
  d.fq = dom.fact_m0;
  d.fv = dom.fact_m1;
  d.rdx = 1.0 / dom.dx;
  d.rdy = 1.0 / dom.dy;
  d.rdz = 1.0 / dom.dz;
  d.fqf = (float)dom.fact_m0;
  d.fvf = (float)dom.fact_m1;
  d.rdxf = 1.0f / (float)dom.dx;
  d.rdyf = 1.0f / (float)dom.dy;
  d.rdzf = 1.0f / (float)dom.dz;
  d.chan_stride = (long long)d.nz * d.ny * d.nxp;
  d.buf_stride = 4 * d.chan_stride;
  int rc = ADF_OK;
  d.field = dalloc<float>(s, (size_t)2 * d.buf_stride, rc);
  if (rc) return rc;
  cudaMemsetAsync(d.field, 0, (size_t)2 * d.buf_stride * 4, s.stream);
  if (has_mask) {
    s.mask_bits = dalloc<uint32_t>(s, (size_t)d.mw * d.ny * d.nz, rc);
    if (rc) return rc;
    d.mask_bits = s.mask_bits;
  }
  rc = make_field_maps(s);
  if (rc) return rc;
  const long long n = npml, nm = npml + 1, nxp = d.nxp, ny = d.ny, nz = d.nz;
  // x-slab rows: side 1 starts at the quad holding its first cell
  d.xs1p = std::max(0, d.nx - npml) / 4 * 4;
  d.xs1v = std::max(0, d.nx - npml - 1) / 4 * 4;
  d.npp = std::max((npml + 3) / 4 * 4, d.nxp - d.xs1p);
  d.nvp = std::max((npml + 1 + 3) / 4 * 4, d.nxp - d.xs1v);
  const long long ps[3] = {nz * ny * d.npp, nz * n * nxp, n * ny * nxp};
  const long long vs[3] = {nz * ny * d.nvp, nz * nm * nxp, nm * ny * nxp};
  for (int a = 0; a < 3; ++a) {
    d.psi_p_side[a] = ps[a];
    d.psi_p_buf[a] = 2 * ps[a];
    d.psi_v_side[a] = vs[a];
    d.psi_v_buf[a] = 2 * vs[a];
    if (npml > 0) {
      d.psi_p[a] = dalloc<float>(s, (size_t)4 * ps[a], rc);
      d.psi_v[a] = dalloc<float>(s, (size_t)4 * vs[a], rc);
      if (rc) return rc;
      cudaMemsetAsync(d.psi_p[a], 0, (size_t)4 * ps[a] * 4, s.stream);
      cudaMemsetAsync(d.psi_v[a], 0, (size_t)4 * vs[a] * 4, s.stream);
    }
  }
  float* coef = dalloc<float>(s, (size_t)8 * n + 4, rc);
  if (rc) return rc;
  cudaMemsetAsync(coef, 0, ((size_t)8 * n + 4) * 4, s.stream);
  d.coef = coef;
  s.coef_dev = coef;
  int* e = dalloc<int>(s, 1, rc);
  if (rc) return rc;
  cudaMemsetAsync(e, 0, 4, s.stream);
  d.err = e;
  return ADF_OK;
}

int solve_alloc_traces(Solve& s, bool need_vsrc) {
  SolveDev& d = s.dev;
  const size_t n = (size_t)d.nt * d.ntx;
  d.src_ntx = d.ntx;
  int rc = ADF_OK;
  for (int c = 0; c < 4; ++c) {
    d.rec[c] = dalloc<float>(s, n, rc);
    if (rc) return rc;
    cudaMemsetAsync(d.rec[c], 0, n * 4, s.stream);
  }
  for (int c = 0; c < 4; ++c) {
    d.src[c] = dalloc<float>(s, n, rc);
    if (rc) return rc;
    cudaMemsetAsync(d.src[c], 0, n * 4, s.stream);
  }
  d.vn_src = dalloc<float>(s, n, rc);
  d.vn_rec = dalloc<float>(s, n, rc);
  float* dir = dalloc<float>(s, (size_t)4 * d.ntx, rc);
  if (rc) return rc;
  cudaMemsetAsync(d.vn_src, 0, n * 4, s.stream);
  cudaMemsetAsync(d.vn_rec, 0, n * 4, s.stream);
  d.dir = dir;
  s.dir_dev = dir;
  (void)need_vsrc;
  return ADF_OK;
}

int solve_finalize(adf_ctx* ctx, Solve& s, const float* const idx[4], const float* const w[4],
                   const int* src_col) {
  int rc = build_entries(s, idx, w, src_col);
  if (rc) return rc;
  // work items {solve, y tile | x tile << 16, z0, z1}: z chunks outer, then
  // y tiles, x tiles inner, so that tiles sharing halo rows run together and
  // the halo hits L2
  s.items.clear();
  const int xt = step_x_tile(), nxt = (s.dev.nxp + xt - 1) / xt;
  for (int z0 = 0; z0 < s.dev.nz; z0 += s.nzc)
    for (int t = 0; t < s.dev.nty; ++t)
      for (int x = 0; x < nxt; ++x)
        s.items.push_back(make_int4(0, t | (x << 16), z0, std::min(z0 + s.nzc, s.dev.nz)));
  return ADF_OK;
}

// ---------------------------------------------------------------------------
// Batch: a set of solves advanced by one launch per step
// ---------------------------------------------------------------------------
Batch::~Batch() { release(); }
void Batch::release() {
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  graph_exec = nullptr;
  graph_steps = 0;
  if (d_solves) cudaFree(d_solves);
  if (d_items) cudaFree(d_items);
  d_solves = nullptr;
  d_items = nullptr;
  cap_solves = cap_items = 0;
}

int Batch::setup(adf_ctx* ctx, const std::vector<Solve*>& list) {
  solves = list;
  const int ns = (int)list.size();
  std::vector<SolveDev> sd(ns);
  std::vector<int4> items;
  max_ty = 1;
  max_ntx = 0;
  max_gf_nsrc = 0;
  max_gf_blocks = 0;
  max_gf_far_blocks = 0;
  max_gf_tc_blocks = 0;
  gf_reduce = false;
  for (int i = 0; i < ns; ++i) {
    sd[i] = list[i]->dev;
    if (sd[i].flags & SF_GF) {
      max_gf_nsrc = std::max(max_gf_nsrc, sd[i].gf_nout);
      max_gf_blocks = std::max(max_gf_blocks, sd[i].gf_nout * sd[i].gf_ks);
      gf_reduce = gf_reduce || sd[i].gf_ks > 1;
      if (sd[i].gf_rs > 0 && (sd[i].flags & SF_GF_TC))
        max_gf_tc_blocks = std::max(max_gf_tc_blocks,
                                    (sd[i].gf_nout + gf_tc_sources_per_tile() - 1) /
                                        gf_tc_sources_per_tile() * sd[i].gf_rs);
      else if (sd[i].gf_rs > 0)
        max_gf_far_blocks = std::max(max_gf_far_blocks, (sd[i].gf_nout + 63) / 64 * sd[i].gf_rs);
    }
    const SolveDev& d = list[i]->dev;
    max_ty = std::max(max_ty, d.ty);
    max_ntx = std::max(max_ntx, d.ntx);
  }
  // interleave items of different solves so the batch stays balanced
  {
    std::vector<size_t> pos(ns, 0);
    bool any = true;
    while (any) {
      any = false;
      for (int i = 0; i < ns; ++i) {
        // a few consecutive items per solve keep neighbouring tiles together
        for (int k = 0; k < 8 && pos[i] < list[i]->items.size(); ++k) {
          int4 it = list[i]->items[pos[i]++];
          it.x = i;
          items.push_back(it);
          any = true;
        }
      }
    }
  }
  n_items = (int)items.size();
  if (ns > cap_solves || n_items > cap_items) {
    release();
    cap_solves = std::max(ns, 1);
    cap_items = std::max(n_items, 1);
    if (cudaMalloc(&d_solves, sizeof(SolveDev) * cap_solves) != cudaSuccess ||
        cudaMalloc(&d_items, sizeof(int4) * cap_items) != cudaSuccess) {
      cudaGetLastError();
      return fail(ADF_E_NOMEM, "batch descriptor allocation failed");
    }
  }
  cudaStream_t st = ctx->stream;
  cudaMemcpyAsync(d_solves, sd.data(), sizeof(SolveDev) * ns, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_items, items.data(), sizeof(int4) * n_items, cudaMemcpyHostToDevice, st);
  {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();  // a copy refused when it was enqueued
    if (e != cudaSuccess)
      return fail(ADF_E_DEVICE, std::string("batch descriptor upload: ") + cudaGetErrorString(e));
  }
  // step + epilogue; GF solves add the extrapolation and its reduction when
  // a source's receivers are split
  per_step = max_gf_nsrc > 0 ? (gf_reduce ? 4 : 3) : 2;
  if (max_ty > step_max_ty()) return fail(ADF_E_ARG, "tile taller than the step kernel's rows");
  grid = n_items;
  if (graph_exec) {
    cudaGraphExecDestroy(graph_exec);
    graph_exec = nullptr;
    graph_steps = 0;
  }
  return ADF_OK;
}

int Batch::launch_step(adf_ctx* ctx, int step) {
  StepParams p;
  p.solves = d_solves;
  p.items = d_items;
  p.n_items = n_items;
  p.step = step;
  const bool timed = ctx->kernel_timing && 2 * step + 1 < (int)ctx->kev.size();
  // inside stream capture an event record must be an external node to be
  // a timing point on every replay
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (timed) cudaStreamIsCapturing(ctx->stream, &cap);
  const unsigned evf =
      cap == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
  if (timed && cudaEventRecordWithFlags(ctx->kev[2 * step], ctx->stream, evf) != cudaSuccess)
    return fail(ADF_E_DEVICE, std::string("event record: ") + cudaGetErrorString(cudaGetLastError()));
  cudaError_t e = adf::launch_step(p, grid, max_ty, ctx->stream);
  if (e != cudaSuccess)
    return fail(ADF_E_DEVICE, std::string("step launch failed: ") + cudaGetErrorString(e) +
                                  " (grid " + std::to_string(grid) + ")");
  if (timed && cudaEventRecordWithFlags(ctx->kev[2 * step + 1], ctx->stream, evf) != cudaSuccess)
    return fail(ADF_E_DEVICE, std::string("event record: ") + cudaGetErrorString(cudaGetLastError()));
  EpiParams ep;
  ep.solves = d_solves;
  ep.n_solves = (int)solves.size();
  ep.step = step;
  cudaError_t e2;
  if ((e2 = launch_epilogue(ep, max_ntx, ctx->stream)) != cudaSuccess)
    return fail(ADF_E_DEVICE, std::string("epilogue launch failed: ") + cudaGetErrorString(e2));
  if (max_gf_nsrc > 0) {  // in-loop GF extrapolation, then vn2v! of those solves
    // the far lags of a block of steps, at the block's first launch-step
    if (max_gf_tc_blocks > 0 && step % kGfBlock == 0 &&
        (e2 = launch_gf_far_tc(ep, max_gf_tc_blocks, ctx->stream)) != cudaSuccess)
      return fail(ADF_E_DEVICE, std::string("GF launch failed: ") + cudaGetErrorString(e2));
    if ((max_gf_far_blocks > 0 || max_gf_tc_blocks > 0) && step % kGfBlock == 0 &&
        (e2 = launch_gf_far(ep, max_gf_far_blocks, max_gf_nsrc, ctx->stream)) != cudaSuccess)
      return fail(ADF_E_DEVICE, std::string("GF launch failed: ") + cudaGetErrorString(e2));
    if ((e2 = launch_gf_extrapolate(ep, max_gf_blocks, max_gf_nsrc, gf_reduce, ctx->stream)) !=
        cudaSuccess)
      return fail(ADF_E_DEVICE, std::string("GF launch failed: ") + cudaGetErrorString(e2));
  }
  return ADF_OK;
}

// Runs `nsteps` launch-steps with step indices step0..step0+nsteps-1.  When
// `use_graph`, chunks of `chunk` steps are captured once into a CUDA graph
// whose last node advances it_base, and the graph is replayed.
int Batch::run(adf_ctx* ctx, int nsteps, bool use_graph, int chunk) {
  if (!use_graph || nsteps < 2 * chunk) {
    for (int s = 0; s < nsteps; ++s) {
      int rc = launch_step(ctx, s);
      if (rc) return rc;
      ctx->launches += per_step;
    }
    return ADF_OK;
  }
  if (!graph_exec || graph_steps != chunk) {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    graph_exec = nullptr;
    cudaGraph_t g;
    if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      return fail(ADF_E_DEVICE, "graph capture failed");
    for (int s = 0; s < chunk; ++s) launch_step(ctx, s);
    launch_advance(d_solves, (int)solves.size(), chunk, ctx->stream);
    if (cudaStreamEndCapture(ctx->stream, &g) != cudaSuccess)
      return fail(ADF_E_DEVICE, "graph capture failed");
    if (cudaGraphInstantiate(&graph_exec, g, 0) != cudaSuccess) {
      cudaGraphDestroy(g);
      return fail(ADF_E_DEVICE, "graph instantiate failed");
    }
    cudaGraphDestroy(g);
    graph_steps = chunk;
  }
  int done = 0;
  while (nsteps - done >= chunk) {
    if (cudaGraphLaunch(graph_exec, ctx->stream) != cudaSuccess)
      return fail(ADF_E_DEVICE, "graph launch failed");
    ctx->launches += per_step * chunk + 1 + far_launches() * chunk / kGfBlock;
    done += chunk;
    if (ctx->kernel_timing) {  // measurement mode: the replay's per-launch events, before reuse
      cudaStreamSynchronize(ctx->stream);
      collect_kernel_times(ctx, chunk);
    }
  }
  for (int s = 0; s < nsteps - done; ++s) {
    int rc = launch_step(ctx, s);
    if (rc) return rc;
    ctx->launches += per_step;
  }
  // restore it_base on the host-side copy's semantics: the caller re-uploads
  return ADF_OK;
}

// One chunk of `n` launch-steps followed by the it_base advance: replayed from
// a captured graph when n == chunk, launched directly otherwise.
int Batch::run_chunk(adf_ctx* ctx, int n, int chunk) {
  if (n == chunk) {
    if (!graph_exec || graph_steps != chunk) {
      if (graph_exec) cudaGraphExecDestroy(graph_exec);
      graph_exec = nullptr;
      cudaGraph_t g;
      if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return fail(ADF_E_DEVICE, "graph capture failed");
      for (int s = 0; s < chunk; ++s) launch_step(ctx, s);
      launch_advance(d_solves, (int)solves.size(), chunk, ctx->stream);
      if (cudaStreamEndCapture(ctx->stream, &g) != cudaSuccess)
        return fail(ADF_E_DEVICE, "graph capture failed");
      if (cudaGraphInstantiate(&graph_exec, g, 0) != cudaSuccess) {
        cudaGraphDestroy(g);
        return fail(ADF_E_DEVICE, "graph instantiate failed");
      }
      cudaGraphDestroy(g);
      graph_steps = chunk;
    }
    if (cudaGraphLaunch(graph_exec, ctx->stream) != cudaSuccess)
      return fail(ADF_E_DEVICE, "graph launch failed");
    ctx->launches += per_step * chunk + 1 + far_launches() * chunk / kGfBlock;
    return ADF_OK;
  }
  for (int s = 0; s < n; ++s) {
    int rc = launch_step(ctx, s);
    if (rc) return rc;
  }
  launch_advance(d_solves, (int)solves.size(), n, ctx->stream);
  ctx->launches += per_step * n + 1;
  return ADF_OK;
}

int Batch::run_advance(adf_ctx* ctx, int n) {
  if (launch_advance(d_solves, (int)solves.size(), n, ctx->stream) != cudaSuccess)
    return fail(ADF_E_DEVICE, "advance launch failed");
  ctx->launches += 1;
  return ADF_OK;
}

void Batch::collect_kernel_times(adf_ctx* ctx, int n) {
  if (!ctx->kernel_timing) return;
  for (int s = 0; s < n && 2 * s + 1 < (int)ctx->kev.size(); ++s) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, ctx->kev[2 * s], ctx->kev[2 * s + 1]) == cudaSuccess) {
      ctx->kernel_ms += ms;
      ++ctx->kernel_launches;
    } else {
      cudaGetLastError();  // a missing sample is not a device error of the next call
    }
  }
}

// Waits for the batch's work and reports any device error it raised.
int Batch::check_error(adf_ctx* ctx) {
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, std::string("device error: ") + cudaGetErrorString(e));
  // per-solve error words written by the kernels (bit 2: a bounded wait for
  // a staged plane gave up)
  for (Solve* s : solves) {
    int w = 0;
    if (s->dev.err && cudaMemcpy(&w, s->dev.err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      return fail(ADF_E_DEVICE, "error word read failed");
    if (w & 4) return fail(ADF_E_TIMEOUT, "step kernel: a bounded wait for a staged plane gave up");
    if (w) return fail(ADF_E_STATE, "step kernel error word " + std::to_string(w));
  }
  return ADF_OK;
}

}  // namespace adf

using namespace adf;

// ---------------------------------------------------------------------------
// layout helpers
// ---------------------------------------------------------------------------
// Julia (nt, ntx) time-fastest  <->  device [nt][ntx] transceiver-fastest
static void transpose_to_dev_layout(const float* jl, float* out, int64_t nt, int64_t ntx) {
  const int64_t B = 64;
  for (int64_t t0 = 0; t0 < nt; t0 += B)
    for (int64_t x0 = 0; x0 < ntx; x0 += B)
      for (int64_t x = x0; x < std::min(ntx, x0 + B); ++x)
        for (int64_t t = t0; t < std::min(nt, t0 + B); ++t) out[t * ntx + x] = jl[t + nt * x];
}
static void transpose_to_julia(const float* dv, float* jl, int64_t nt, int64_t ntx) {
  const int64_t B = 64;
  for (int64_t x0 = 0; x0 < ntx; x0 += B)
    for (int64_t t0 = 0; t0 < nt; t0 += B)
      for (int64_t t = t0; t < std::min(nt, t0 + B); ++t)
        for (int64_t x = x0; x < std::min(ntx, x0 + B); ++x) jl[t + nt * x] = dv[t * ntx + x];
}

// Uploads on stream `st`, so the kernels that follow on it are ordered after
// them; the staging vector is reused only once its copy has completed.
static cudaError_t upload_traces(Solve& s, const adf_txgrid* txs, cudaStream_t st) {
  SolveDev& d = s.dev;
  const int64_t nt = d.nt, ntx = d.ntx;
  std::vector<float> tmp((size_t)(nt * ntx));
  cudaError_t e = cudaSuccess;
  auto up = [&](const float* jl, float* dst) {
    if (e != cudaSuccess) return;
    transpose_to_dev_layout(jl, tmp.data(), nt, ntx);
    e = cudaMemcpyAsync(dst, tmp.data(), tmp.size() * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  };
  for (int c = 0; c < 4; ++c) {
    up(txs->src[c], d.src[c]);
    up(txs->rec[c], d.rec[c]);
  }
  up(txs->vn_src, d.vn_src);
  up(txs->vn_rec, d.vn_rec);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s.dir_dev, txs->dir, (size_t)4 * ntx * 4, cudaMemcpyHostToDevice, st);
  return e;
}

// Device (step-major) traces -> the caller's Julia (nt, ntx) arrays.  Stops at
// the first failed copy and returns its error; nothing is transposed from it.
static cudaError_t download_trace(Solve& s, std::vector<float>& tmp, const float* src, float* jl) {
  const cudaError_t e = cudaMemcpy(tmp.data(), src, tmp.size() * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) transpose_to_julia(tmp.data(), jl, s.dev.nt, s.dev.ntx);
  return e;
}

static cudaError_t download_traces(Solve& s, adf_txgrid* txs) {
  SolveDev& d = s.dev;
  std::vector<float> tmp((size_t)(d.nt * d.ntx));
  cudaError_t e = cudaSuccess;
  for (int c = 0; c < 4 && e == cudaSuccess; ++c) {
    e = download_trace(s, tmp, d.rec[c], txs->rec[c]);
    if (c > 0 && e == cudaSuccess) e = download_trace(s, tmp, d.src[c], txs->src[c]);
  }
  if (e == cudaSuccess) e = download_trace(s, tmp, d.vn_rec, txs->vn_rec);
  return e;
}

// the GF extrapolation writes p_src and vn_src rows: both come back too
static cudaError_t download_gf_sources(Solve& s, adf_txgrid* txs) {
  SolveDev& d = s.dev;
  std::vector<float> tmp((size_t)(d.nt * d.ntx));
  cudaError_t e = download_trace(s, tmp, d.src[0], txs->src[0]);
  if (e == cudaSuccess) e = download_trace(s, tmp, d.vn_src, txs->vn_src);
  return e;
}

// psi: Julia (npml,ny,nz,2) / (nx,npml,nz,2) / (nx,ny,npml,2) <-> device.
// Uploads are stream-ordered on `st`; downloads are synchronous copies taken
// after the caller has synchronised the stream that wrote the memory.
static cudaError_t psi_copy(Solve& s, int axis, bool vside, float* host, bool upload, int buffer,
                            cudaStream_t st) {
  SolveDev& d = s.dev;
  const long long n = vside ? d.npml + 1 : d.npml;
  float* base = vside ? d.psi_v[axis] : d.psi_p[axis];
  const long long side = vside ? d.psi_v_side[axis] : d.psi_p_side[axis];
  float* dev = base + (long long)buffer * 2 * side;
  if (axis == 0) {  // rows of n values per side; device pitch npp / nvp, side 1 offset
    const size_t pitch = (size_t)(vside ? d.nvp : d.npp) * 4;
    const size_t rows = (size_t)d.ny * d.nz;
    const long long first1 = vside ? d.nx - d.npml - 1 : d.nx - d.npml;  // side 1's first cell
    // (a grid narrower than npml+1 cells never uses side 1: any in-row offset does)
    const long long off1 = first1 < 0 ? 0 : first1 - (vside ? d.xs1v : d.xs1p);
    for (int sd = 0; sd < 2; ++sd) {
      float* dv = dev + sd * side + (sd ? off1 : 0);
      float* hs = host + (size_t)sd * rows * n;
      const cudaError_t e =
          upload ? cudaMemcpy2DAsync(dv, pitch, hs, (size_t)n * 4, (size_t)n * 4, rows,
                                     cudaMemcpyHostToDevice, st)
                 : cudaMemcpy2D(hs, (size_t)n * 4, dv, pitch, (size_t)n * 4, rows,
                                cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  const size_t rows = axis == 1 ? (size_t)n * d.nz * 2 : (size_t)d.ny * n * 2;
  if (upload)
    return cudaMemcpy2DAsync(dev, (size_t)d.nxp * 4, host, (size_t)d.nx * 4, (size_t)d.nx * 4,
                             rows, cudaMemcpyHostToDevice, st);
  return cudaMemcpy2D(host, (size_t)d.nx * 4, dev, (size_t)d.nxp * 4, (size_t)d.nx * 4, rows,
                      cudaMemcpyDeviceToHost);
}

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" {

int adf_version(void) { return 10000; }

int adf_last_error(char* buf, size_t n) {
  if (!buf || n == 0) return ADF_E_ARG;
  std::snprintf(buf, n, "%s", g_err.c_str());
  return ADF_OK;
}

int adf_ctx_create(int device, size_t hbm_budget, adf_ctx** out) {
  if (!out) return fail(ADF_E_ARG, "out is NULL");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(ADF_E_DEVICE, "no CUDA device available: this library has no CPU fallback");
  }
  if (device < 0 || device >= ndev) return fail(ADF_E_ARG, "bad device index");
  if (cudaSetDevice(device) != cudaSuccess) return fail(ADF_E_DEVICE, "cudaSetDevice failed");
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  if (prop.major < 10) return fail(ADF_E_DEVICE, "this library is built for sm_100a (B200)");
  auto* c = new adf_ctx();
  c->device = device;
  c->nsm = prop.multiProcessorCount;
  c->smem_per_sm = (int)prop.sharedMemPerMultiprocessor;
  c->smem_optin = (int)prop.sharedMemPerBlockOptin;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return fail(ADF_E_DEVICE, "stream creation failed");
  }
  cudaEventCreate(&c->ev0);
  cudaEventCreate(&c->ev1);
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  c->budget = hbm_budget ? hbm_budget : (size_t)(0.9 * (double)fr);
  {  // the context's own pool (device memory, no release back to the driver
     // while the context lives); admission keeps its size within the budget
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    uint64_t keep = UINT64_MAX;
    if (cudaMemPoolCreate(&c->pool, &props) != cudaSuccess ||
        cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
      cudaGetLastError();
      if (c->pool) cudaMemPoolDestroy(c->pool);
      cudaEventDestroy(c->ev0);
      cudaEventDestroy(c->ev1);
      cudaStreamDestroy(c->stream);
      delete c;
      return fail(ADF_E_DEVICE, "memory pool creation failed");
    }
  }
  *out = c;
  return ADF_OK;
}

int adf_ctx_destroy(adf_ctx* c) {
  if (!c) return ADF_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (auto& e : c->kev) cudaEventDestroy(e);
  cudaEventDestroy(c->ev0);
  cudaEventDestroy(c->ev1);
  cudaStreamDestroy(c->stream);
  if (c->pool) cudaMemPoolDestroy(c->pool);
  delete c;
  return ADF_OK;
}

int adf_domain_make(double tmax, double xmax, double ymax, double zmax, int64_t nx, int64_t ny,
                    int64_t nz, double c0, double r0, double cf, adf_domain* o) {
  if (!o || nx < 2 || ny < 2 || nz < 2 || !(c0 > 0) || !(cf > 0))
    return fail(ADF_E_ARG, "bad domain arguments");
  o->tmax = tmax; o->xmax = xmax; o->ymax = ymax; o->zmax = zmax;
  o->nx = nx; o->ny = ny; o->nz = nz;
  o->c0 = c0; o->r0 = r0; o->cf = cf;
  o->dx = 2 * xmax / (double)(nx - 1);
  o->dy = 2 * ymax / (double)(ny - 1);
  o->dz = 2 * zmax / (double)(nz - 1);
  o->dt = cf * std::min(o->dx, std::min(o->dy, o->dz)) / c0 / std::sqrt(3.0);
  o->nt = (int64_t)std::ceil(tmax / o->dt);
  o->fact_m0 = o->dt * r0 * (c0 * c0);
  o->fact_m1 = o->dt / r0;
  o->z0 = r0 * c0;
  return ADF_OK;
}

int adf_coords(const adf_domain* d, int axis, int chan, double* out) {
  if (!d || !out || axis < 0 || axis > 2 || chan < 0 || chan > 3)
    return fail(ADF_E_ARG, "bad coords arguments");
  hm::Range r = hm::axis_range(to_dom(*d), axis, chan);
  for (int64_t i = 1; i <= r.len; ++i) out[i - 1] = r.at(i);
  return ADF_OK;
}

int adf_time_axis(const adf_domain* d, double* out) {
  if (!d || !out || d->nt < 1) return fail(ADF_E_ARG, "bad time axis arguments");
  hm::Range r = hm::make_range(0.0, d->tmax, d->nt);
  for (int64_t i = 1; i <= d->nt; ++i) out[i - 1] = r.at(i);
  return ADF_OK;
}

int adf_cpml_profiles(adf_ctx* ctx, int64_t npml, double vel_max, double dt, double rcoef,
                      double thickness, double fc, float* out32, double* out64) {
  if (!ctx || npml < 0 || !out32) return fail(ADF_E_ARG, "bad cpml arguments");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  cudaGetLastError();  // the checks below see only this call's errors
  const size_t n = (size_t)(8 * npml + 4);
  float* d32 = nullptr;
  double* d64 = nullptr;
  if (cudaMalloc(&d32, n * 4) != cudaSuccess || cudaMalloc(&d64, n * 8) != cudaSuccess) {
    cudaFree(d32);  // whichever was allocated (cudaFree(nullptr) is a no-op)
    cudaGetLastError();
    return fail(ADF_E_NOMEM, "cudaMalloc failed");
  }
  e = launch_cpml_profiles((int)npml, vel_max, dt, rcoef, thickness, fc, d32, d64, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out32, d32, n * 4, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && out64)
    e = cudaMemcpyAsync(out64, d64, n * 8, cudaMemcpyDeviceToHost, ctx->stream);
  const cudaError_t es = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) e = es;
  cudaFree(d32);
  cudaFree(d64);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  return ADF_OK;
}

// adf_cpml_profiles with its scratch in a fixed device array instead of
// cudaMalloc/cudaFree.  The scratch address is taken once per device, on the
// first call with that device current, and cached.
int adf_cpml_profiles_static(adf_ctx* ctx, int64_t npml, double vel_max, double dt,
                             double rcoef, double thickness, double fc, float* out32,
                             double* out64) {
  static std::mutex mu;
  static int n_dev = -1;
  static std::vector<double*> dev64;
  static std::vector<float*> dev32;
  if (!ctx || npml < 0 || !out32) return fail(ADF_E_ARG, "bad cpml arguments");
  const int max_npml = static_cpml_max_npml();
  if (npml > max_npml)
    return fail(ADF_E_ARG, "npml " + std::to_string(npml) +
                               " exceeds the fixed scratch of adf_cpml_profiles_static (max " +
                               std::to_string(max_npml) + "); use adf_cpml_profiles");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  cudaGetLastError();  // a leftover error of an earlier call is not this call's
  double* d64 = nullptr;
  float* d32 = nullptr;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (n_dev < 0) {
      e = cudaGetDeviceCount(&n_dev);
      if (e != cudaSuccess) {
        n_dev = -1;
        return fail(ADF_E_DEVICE, cudaGetErrorString(e));
      }
      dev64.assign((size_t)n_dev, nullptr);
      dev32.assign((size_t)n_dev, nullptr);
    }
    if (ctx->device < 0 || ctx->device >= n_dev) return fail(ADF_E_ARG, "bad device");
    if (!dev64[(size_t)ctx->device]) {
      e = static_cpml_scratch(&d64, &d32);
      if (e != cudaSuccess)
        return fail(ADF_E_DEVICE, std::string("scratch address: ") + cudaGetErrorString(e));
      dev64[(size_t)ctx->device] = d64;
      dev32[(size_t)ctx->device] = d32;
    }
    d64 = dev64[(size_t)ctx->device];
    d32 = dev32[(size_t)ctx->device];
  }
  const size_t n = (size_t)(8 * npml + 4);
  e = launch_cpml_profiles((int)npml, vel_max, dt, rcoef, thickness, fc, d32, d64, ctx->stream);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  e = cudaMemcpyAsync(out32, d32, n * 4, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && out64)
    e = cudaMemcpyAsync(out64, d64, n * 8, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  return ADF_OK;
}

int adf_build_mask(adf_ctx* ctx, const adf_domain* d, int shape, const double* params,
                   uint8_t* out_bool) {
  if (!ctx || !d) return fail(ADF_E_ARG, "bad mask arguments");
  if (shape == ADF_SHAPE_NONE) return 1;
  if (shape < 0 || shape > 4) return fail(ADF_E_ARG, "unknown shape");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  cudaGetLastError();
  uint32_t* bits = nullptr;
  uint8_t* jl = nullptr;
  const int mw = (int)(((d->nx + 7) / 8 + 3) / 4 * 4);
  int rc = build_mask_device(ctx, *d, shape, params, mw, &bits, out_bool ? &jl : nullptr);
  if (rc) return rc;
  if (out_bool)
    e = cudaMemcpyAsync(out_bool, jl, (size_t)4 * d->nx * d->ny * d->nz, cudaMemcpyDeviceToHost,
                        ctx->stream);
  const cudaError_t es = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) e = es;
  cudaFree(bits);
  if (jl) cudaFree(jl);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  return ADF_OK;
}

int adf_pack_transceivers(const adf_domain* d, const double* points, const double* dirs,
                          const double* tf, adf_txgrid* o) {
  if (!d || !points || !dirs || !tf || !o) return fail(ADF_E_ARG, "NULL argument");
  if (o->nt != d->nt) return fail(ADF_E_ARG, "txgrid nt must equal dom.nt");
  return pack_transceivers_host(to_dom(*d), points, dirs, tf, o);
}

// The KH extrapolation that follows a run on the recorded traces of some of
// its transceivers (adf_run_fdtd_kh), or none.
struct KhAfter {
  const adf_kh_desc* desc = nullptr;
  const int64_t* cols = nullptr;  // 1-based transceiver indices, desc->ns of them
  float* out = nullptr;
};

static int run_fdtd_impl(adf_ctx* ctx, const adf_domain* d, float* field, adf_txgrid* txs,
                         adf_cpml* cpml, const uint8_t* mask, int64_t start_step,
                         int64_t stop_step, int flags, const adf_gfmap* gf, adf_step_cb cb,
                         void* user, const KhAfter& kh = KhAfter()) {
  if (!ctx || !d || !field || !txs) return fail(ADF_E_ARG, "NULL argument");
  if (kh.desc) {
    if (!kh.cols || !kh.out) return fail(ADF_E_ARG, "KH: surface columns and output required");
    if (kh.desc->nt < 1 || kh.desc->nt > stop_step)
      return fail(ADF_E_ARG, "KH: nt must lie in 1..stop_step (recorded rows)");
    if (!(std::fabs(kh.desc->dt - d->dt) <= 1e-12 * d->dt))
      return fail(ADF_E_ARG, "KH: dt must equal the domain's time step");
    for (int64_t k = 0; k < kh.desc->ns; ++k)
      if (kh.cols[k] < 1 || kh.cols[k] > txs->ntx)
        return fail(ADF_E_ARG, "KH: surface column outside 1..ntx");
  }
  const bool use_gf = gf && !gf->discard;
  int ntens = 0;
  if (gf) {
    if (gf->kind < ADF_GF_PV_FROM_PIN || gf->kind > ADF_GF_PV_FROM_PV)
      return fail(ADF_E_ARG, "unknown gf map kind");
    ntens = gf->kind == ADF_GF_PV_FROM_PV ? 4 : 2;
    // driven sources and read receivers per kind (extrapolation.jl:36-87)
    const int64_t nout = gf->kind == ADF_GF_PV_FROM_PIN ? gf->n1 : gf->n2;
    const int64_t nin = gf->kind == ADF_GF_PV_FROM_PIN ? gf->n2 : gf->n1;
    if (gf->nt_gf < 1 || gf->n1 < 1 || gf->n2 < 1 || !gf->i_src || !gf->i_rec)
      return fail(ADF_E_ARG, "bad gf map");
    if (gf->n_src != nout || gf->n_rec != nin)
      return fail(ADF_E_ARG, "gf map: iSrc/iRec lengths do not match the tensor dimensions");
    for (int k = 0; use_gf && k < ntens; ++k)
      if (!gf->t[k]) return fail(ADF_E_ARG, "gf map: missing tensor");
    for (int64_t k = 0; k < gf->n_src; ++k)
      if (gf->i_src[k] < 1 || gf->i_src[k] > txs->ntx)
        return fail(ADF_E_ARG, "gf map iSrc outside 1..ntx");
    for (int64_t k = 0; k < gf->n_rec; ++k)
      if (gf->i_rec[k] < 1 || gf->i_rec[k] > txs->ntx)
        return fail(ADF_E_ARG, "gf map iRec outside 1..ntx");
  }
  if (use_gf && gf->contraction != ADF_GF_CONTRACT_FP64 &&
      gf->contraction != ADF_GF_CONTRACT_TF32X3)
    return fail(ADF_E_ARG, "gf map contraction must be ADF_GF_CONTRACT_FP64 or _TF32X3");
  if (use_gf && gf->contraction == ADF_GF_CONTRACT_TF32X3 && gf->kind == ADF_GF_PV_FROM_PV)
    return fail(ADF_E_ARG, "the tensor-core contraction applies to PVFromPin and PFromPin maps");
  const bool use_tc = use_gf && gf->contraction == ADF_GF_CONTRACT_TF32X3;
  if (txs->nt != d->nt) return fail(ADF_E_ARG, "txs.nt must equal dom.nt");
  if (start_step < 1 || stop_step > d->nt) return fail(ADF_E_ARG, "step range outside 1..nt");
  if (d->nx < 4 || d->ny < 4 || d->nz < 4) return fail(ADF_E_ARG, "grid must be at least 4^3");
  if (d->nx > 512) return fail(ADF_E_ARG, "nx > 512 is not supported");
  if (flags != ADF_ARITH_PROMOTE && flags != ADF_ARITH_FP32) return fail(ADF_E_ARG, "bad flags");
  const int64_t npml = cpml ? cpml->npml : 0;
  if (npml < 0 || (npml > 0 && !cpml->coef)) return fail(ADF_E_ARG, "bad cpml");
  if (npml > 63) return fail(ADF_E_ARG, "npml > 63 is not supported");
  if (stop_step < start_step) return ADF_OK;
  cudaSetDevice(ctx->device);
  cudaGetLastError();  // the checks below see only this call's errors
  size_t need = solve_bytes_estimate(d->nx, d->ny, d->nz, npml, txs->ntx, d->nt, mask);
  if (use_gf) {
    need += (size_t)4 * ntens * gf->nt_gf * gf->n1 * gf->n2 + (size_t)8 * gf->n_rec * d->nt +
            (size_t)4 * (gf->n_src + gf->n_rec + txs->ntx);
    if (gf->kind != ADF_GF_PV_FROM_PV)  // near-lag copy and history ring of the blocked kinds
      need += (size_t)4 * 2 * std::min<int64_t>(kGfBlock, gf->nt_gf) * gf->n1 * gf->n2 +
              (size_t)8 * kGfRing * gf->n_rec;
    if (use_tc) need += sizeof(float) * gf_tc_packed_floats(gf->nt_gf, gf->n_src, gf->n_rec);
  }
  if (need > ctx->budget) return fail(ADF_E_BUDGET, "solve exceeds the context's HBM budget");
  auto s = std::make_unique<Solve>();
  const hm::Dom dom = to_dom(*d);
  int rc = solve_alloc(ctx, *s, dom, (int)npml, mask != nullptr, flags, (int)txs->ntx);
  if (!rc) rc = solve_alloc_traces(*s, true);
  if (rc) return rc;
  // Every upload below is a stream-ordered copy on the context stream: the
  // zeroing above, the copies, the set-up kernels and the steps run in that
  // order.  A pageable source is staged before cudaMemcpyAsync returns.
  cudaStream_t st = ctx->stream;
  SolveDev& sd = s->dev;
  cudaError_t ue = cudaSuccess;  // the first failed upload
  auto up = [&](cudaError_t e) {
    if (ue == cudaSuccess && e != cudaSuccess) ue = e;
  };
  // field -> buffer 0 (input of step start_step)
  up(cudaMemcpy2DAsync(sd.field, (size_t)sd.nxp * 4, field, (size_t)d->nx * 4, (size_t)d->nx * 4,
                       (size_t)d->ny * d->nz * 4, cudaMemcpyHostToDevice, st));
  if (mask) {
    uint8_t* jl = nullptr;
    const size_t mb = (size_t)4 * d->nx * d->ny * d->nz;
    if (cudaMalloc(&jl, mb) != cudaSuccess) {
      cudaGetLastError();
      return fail(ADF_E_NOMEM, "mask staging alloc failed");
    }
    up(cudaMemcpyAsync(jl, mask, mb, cudaMemcpyHostToDevice, st));
    up(launch_pack_mask(jl, sd.nx, sd.ny, sd.nz, sd.mw, s->mask_bits, st));
    up(cudaStreamSynchronize(st));
    cudaFree(jl);
  }
  if (npml > 0) {
    up(cudaMemcpyAsync(s->coef_dev, cpml->coef, (size_t)(8 * npml + 4) * 4,
                       cudaMemcpyHostToDevice, st));
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 2; ++b) {
        if (cpml->mv[a]) up(psi_copy(*s, a, false, cpml->mv[a], true, b, st));
        if (cpml->mp[a]) up(psi_copy(*s, a, true, cpml->mp[a], true, b, st));
      }
  }
  up(upload_traces(*s, txs, st));
  if (use_gf) {  // GF tensors, 0-based columns, Float64 pin history
    const size_t ng = (size_t)gf->nt_gf * gf->n1 * gf->n2;
    for (int k = 0; k < ntens && !rc; ++k) {
      float* t = solve_dalloc<float>(*s, ng, rc);
      if (!rc) up(cudaMemcpyAsync(t, gf->t[k], ng * 4, cudaMemcpyHostToDevice, st));
      sd.gf_t[k] = t;
    }
    int* isrc = rc ? nullptr : solve_dalloc<int>(*s, (size_t)gf->n_src, rc);
    int* gcol = rc ? nullptr : solve_dalloc<int>(*s, (size_t)txs->ntx, rc);
    int* irec = rc ? nullptr : solve_dalloc<int>(*s, (size_t)gf->n_rec, rc);
    double* pin = rc ? nullptr : solve_dalloc<double>(*s, (size_t)gf->n_rec * d->nt, rc);
    // receiver splits of the per-step kernel: about eight 256-thread blocks
    // per SM in all; one per source when the far lags are blocked (it then
    // sums at most kGfBlock lags per receiver)
    const int ks = gf->kind != ADF_GF_PV_FROM_PV
                       ? 1
                       : (int)std::max<int64_t>(
                             1, std::min<int64_t>(gf->n_rec, (int64_t)8 * ctx->nsm /
                                                                 std::max<int64_t>(1, gf->n_src)));
    double* part = rc ? nullptr : solve_dalloc<double>(*s, (size_t)gf->n_src * ks * 2, rc);
    // block-causal far lags for the input-history kinds: receiver splits for
    // about two 256-thread blocks per SM over the 64-source tiles
    int rs = 0;
    double* far = nullptr;
    if (gf->kind != ADF_GF_PV_FROM_PV && !rc) {
      if (use_tc) {  // one 128-source CTA per SM over the source tiles
        const int64_t otiles = (gf->n_src + gf_tc_sources_per_tile() - 1) / gf_tc_sources_per_tile();
        rs = (int)std::max<int64_t>(1, std::min<int64_t>(gf->n_rec, (ctx->nsm + otiles - 1) / otiles));
      } else {
        const int64_t otiles = (gf->n_src + 63) / 64;
        rs = (int)std::max<int64_t>(1, std::min<int64_t>(gf->n_rec, (2 * ctx->nsm + otiles - 1) / otiles));
      }
      far = solve_dalloc<double>(*s, (size_t)gf->n_src * rs * kGfBlock * 2, rc);
    }
    float* tc = nullptr;
    if (use_tc && !rc) tc = solve_dalloc<float>(*s, gf_tc_packed_floats(gf->nt_gf, gf->n_src, gf->n_rec), rc);
    // the blocked kinds' per-step sum reads lags 0..kGfBlock-1 from a
    // receiver-major copy and the recent history from a receiver-major ring
    float* near = nullptr;
    double* ring = nullptr;
    const int nl = (int)std::min<int64_t>(kGfBlock, gf->nt_gf);
    if (rs > 0 && !rc) {
      near = solve_dalloc<float>(*s, (size_t)2 * nl * gf->n1 * gf->n2, rc);
      if (!rc) ring = solve_dalloc<double>(*s, (size_t)kGfRing * gf->n_rec, rc);
    }
    if (rc) return rc;
    sd.gf_part = part;
    sd.gf_ks = ks;
    sd.gf_far = far;
    sd.gf_rs = rs;
    sd.gf_ring = ring;
    sd.gf_nl = nl;
    std::vector<int> cs((size_t)gf->n_src), cr((size_t)gf->n_rec);
    for (int64_t k = 0; k < gf->n_src; ++k) cs[(size_t)k] = (int)(gf->i_src[k] - 1);
    for (int64_t k = 0; k < gf->n_rec; ++k) cr[(size_t)k] = (int)(gf->i_rec[k] - 1);
    up(cudaMemcpyAsync(isrc, cs.data(), cs.size() * 4, cudaMemcpyHostToDevice, st));
    {  // driven columns: the last source writing each one applies its vn2v!
      std::vector<int> col((size_t)txs->ntx, 0);
      for (int64_t k = 0; k < gf->n_src; ++k) col[(size_t)cs[(size_t)k]] = (int)k + 1;
      up(cudaMemcpyAsync(gcol, col.data(), col.size() * 4, cudaMemcpyHostToDevice, st));
      up(cudaStreamSynchronize(st));  // before `col` goes out of scope
      sd.gf_col = gcol;
    }
    up(cudaMemcpyAsync(irec, cr.data(), cr.size() * 4, cudaMemcpyHostToDevice, st));
    sd.gf_isrc = isrc;
    sd.gf_irec = irec;
    sd.gf_pin = pin;
    sd.gf_z0 = gf->z0;
    sd.gf_kind = gf->kind;
    sd.gf_nt = (int)gf->nt_gf;
    sd.gf_n1 = (int)gf->n1;
    sd.gf_n2 = (int)gf->n2;
    sd.gf_nout = (int)gf->n_src;
    sd.gf_nin = (int)gf->n_rec;
    sd.flags |= SF_GF;
    if (near) {
      cudaError_t e = launch_gf_near_pack(sd, near, ctx->stream);
      if (e != cudaSuccess)
        return fail(ADF_E_DEVICE, std::string("GF pack launch failed: ") + cudaGetErrorString(e));
      sd.gf_near = near;
    }
    if (tc) {  // the far lags' operand tiles for the tensor cores
      sd.gf_tc_nch = (int)gf_tc_chunks(gf->nt_gf);
      cudaError_t e = launch_gf_tc_pack(sd, tc, ctx->stream);
      if (e != cudaSuccess)
        return fail(ADF_E_DEVICE, std::string("GF pack launch failed: ") + cudaGetErrorString(e));
      sd.gf_tc = tc;
      sd.flags |= SF_GF_TC;
    }
    // pin rows recorded before start_step (a resumed run) from the host traces
    if (start_step > 1 && gf->kind != ADF_GF_PV_FROM_PV) {
      std::vector<double> h((size_t)gf->n_rec * d->nt, 0.0);
      for (int64_t r = 0; r < gf->n_rec; ++r)
        for (int64_t t = 0; t < start_step - 1; ++t) {
          const int64_t o = t + d->nt * cr[(size_t)r];
          h[(size_t)(r * d->nt + t)] =
              ((double)txs->rec[0][o] - (double)txs->vn_rec[o] * gf->z0) / 2.0;
        }
      up(cudaMemcpyAsync(pin, h.data(), h.size() * 8, cudaMemcpyHostToDevice, st));
      up(cudaStreamSynchronize(st));  // before `h` goes out of scope
    }
    up(cudaStreamSynchronize(st));  // before `cs` and `cr` go out of scope
  }
  const float* idx[4] = {txs->idx[0], txs->idx[1], txs->idx[2], txs->idx[3]};
  const float* w[4] = {txs->w[0], txs->w[1], txs->w[2], txs->w[3]};
  up(cudaStreamSynchronize(st));
  if (ue != cudaSuccess) {
    cudaGetLastError();
    return fail(ADF_E_DEVICE, std::string("upload: ") + cudaGetErrorString(ue));
  }
  rc = solve_finalize(ctx, *s, idx, w, nullptr);
  if (rc) return rc;
  sd.it_first = (int)start_step;
  sd.it_base = (int)start_step;
  sd.it_stop = (int)stop_step;
  Batch b;
  rc = b.setup(ctx, {s.get()});
  if (rc) return rc;
  const int nsteps = (int)(stop_step - start_step + 1);
  ctx->launches = 0;
  {
    const int64_t ntr = (int64_t)d->nt * txs->ntx * 4;
    ctx->h2d_bytes = (int64_t)d->nx * d->ny * d->nz * 16 + 10 * ntr + txs->ntx * 16 +
                     (mask ? 4 * d->nx * d->ny * d->nz : 0) + s->h2d;
    ctx->d2h_bytes = (int64_t)d->nx * d->ny * d->nz * 16 + 8 * ntr;
    if (npml > 0) {
      const int64_t psi = 2 * 2 * npml * (d->ny * d->nz + d->nx * d->nz + d->nx * d->ny) * 4 +
                          2 * 2 * (npml + 1) * (d->ny * d->nz + d->nx * d->nz + d->nx * d->ny) * 4;
      ctx->h2d_bytes += psi + (8 * npml + 4) * 4;
      ctx->d2h_bytes += psi / 2;
    }
  }
  ctx->cur = s.get();
  cudaEventRecord(ctx->ev0, ctx->stream);
  if (!cb) {
    rc = b.run(ctx, nsteps, true, kGraphChunk);
  } else {
    for (int k = 0; k < nsteps && !rc; ++k) {
      rc = b.launch_step(ctx, k);
      ctx->launches += b.per_step;
      if (rc) break;
      ctx->cur_it = start_step + k;
      cudaStreamSynchronize(ctx->stream);
      if (cb(start_step + k, user)) rc = fail(ADF_E_CANCELLED, "cancelled by callback");
    }
  }
  cudaEventRecord(ctx->ev1, ctx->stream);
  int rc2 = b.check_error(ctx);
  if (!rc) rc = rc2;
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  ctx->last_ms = ms;
  ctx->cur = nullptr;
  if (rc) return rc;
  if (kh.desc) {  // KH on the recorded v_n (monopole) and p (dipole) columns, in HBM
    std::vector<int> c0((size_t)kh.desc->ns);
    for (int64_t k = 0; k < kh.desc->ns; ++k) c0[(size_t)k] = (int)(kh.cols[k] - 1);
    int* dcols = solve_dalloc<int>(*s, c0.size(), rc);
    if (rc) return rc;
    if (cudaMemcpyAsync(dcols, c0.data(), c0.size() * 4, cudaMemcpyHostToDevice, st) !=
        cudaSuccess) {
      cudaGetLastError();
      return fail(ADF_E_DEVICE, "KH column upload failed");
    }
    KhDevSrc src{sd.vn_rec, sd.rec[0], sd.ntx, dcols};
    rc = kh_pressure_dev(ctx, kh.desc, src, kh.out);
    ctx->last_ms = ms;  // the run's own time; KH's is ctx->kh_ms
    if (rc) return rc;
  }
  // output buffer of the last executed step
  const int fb = (int)((stop_step - start_step + 1) & 1);
  cudaError_t e = cudaMemcpy2D(field, (size_t)d->nx * 4, sd.field + (size_t)fb * sd.buf_stride,
                               (size_t)sd.nxp * 4, (size_t)d->nx * 4,
                               (size_t)d->ny * d->nz * 4, cudaMemcpyDeviceToHost);
  if (npml > 0)
    for (int a = 0; a < 3 && e == cudaSuccess; ++a) {
      if (cpml->mv[a]) e = psi_copy(*s, a, false, cpml->mv[a], false, fb, st);
      if (cpml->mp[a] && e == cudaSuccess) e = psi_copy(*s, a, true, cpml->mp[a], false, fb, st);
    }
  if (e == cudaSuccess) e = download_traces(*s, txs);
  if (use_gf && e == cudaSuccess) e = download_gf_sources(*s, txs);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(ADF_E_DEVICE, std::string("download: ") + cudaGetErrorString(e));
  }
  return ADF_OK;
}

int adf_run_fdtd(adf_ctx* ctx, const adf_domain* d, float* field, adf_txgrid* txs,
                 adf_cpml* cpml, const uint8_t* mask, int64_t start_step, int64_t stop_step,
                 int flags, adf_step_cb cb, void* user) {
  return run_fdtd_impl(ctx, d, field, txs, cpml, mask, start_step, stop_step, flags, nullptr,
                       cb, user);
}

int adf_run_fdtd_kh(adf_ctx* ctx, const adf_domain* d, float* field, adf_txgrid* txs,
                    adf_cpml* cpml, const uint8_t* mask, int64_t start_step, int64_t stop_step,
                    int flags, const adf_kh_desc* kh, const int64_t* kh_cols, float* kh_out) {
  if (!kh) return fail(ADF_E_ARG, "NULL KH descriptor");
  KhAfter a;
  a.desc = kh;
  a.cols = kh_cols;
  a.out = kh_out;
  return run_fdtd_impl(ctx, d, field, txs, cpml, mask, start_step, stop_step, flags, nullptr,
                       nullptr, nullptr, a);
}

int adf_last_kh_ms(adf_ctx* ctx, double* ms) {
  if (!ctx || !ms) return fail(ADF_E_ARG, "bad arguments");
  *ms = ctx->kh_ms;
  return ADF_OK;
}

int adf_run_fdtd_gf(adf_ctx* ctx, const adf_domain* d, float* field, adf_txgrid* txs,
                    adf_cpml* cpml, const uint8_t* mask, int64_t start_step, int64_t stop_step,
                    int flags, const adf_gfmap* gf, adf_step_cb cb, void* user) {
  if (!gf) return fail(ADF_E_ARG, "NULL gf map");
  return run_fdtd_impl(ctx, d, field, txs, cpml, mask, start_step, stop_step, flags, gf, cb,
                       user);
}

int adf_read_field(adf_ctx* ctx, int chan, float* out) {
  if (!ctx || !out || chan < 0 || chan > 3) return fail(ADF_E_ARG, "bad arguments");
  if (!ctx->cur) return fail(ADF_E_STATE, "adf_read_field is only valid inside a step callback");
  const SolveDev& sd = ctx->cur->dev;
  const int fb = (int)((ctx->cur_it - sd.it_first + 1) & 1);
  const cudaError_t e = cudaMemcpy2D(
      out, (size_t)sd.nx * 4, sd.field + (size_t)fb * sd.buf_stride + (size_t)chan * sd.chan_stride,
      (size_t)sd.nxp * 4, (size_t)sd.nx * 4, (size_t)sd.ny * sd.nz, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, std::string("adf_read_field: ") + cudaGetErrorString(e));
  return ADF_OK;
}

int adf_last_timing(adf_ctx* ctx, double* ms, int64_t* launches) {
  if (!ctx) return fail(ADF_E_ARG, "NULL ctx");
  if (ms) *ms = ctx->last_ms;
  if (launches) *launches = ctx->launches;
  return ADF_OK;
}

int adf_set_kernel_timing(adf_ctx* ctx, int on) {
  if (!ctx) return fail(ADF_E_ARG, "NULL ctx");
  ctx->kernel_timing = on != 0;
  if (on && ctx->kev.empty()) {
    ctx->kev.resize(2 * kGraphChunk);
    for (auto& e : ctx->kev) cudaEventCreate(&e);
  }
  // graphs captured without (or with) event nodes are re-captured lazily
  return ADF_OK;
}

int adf_host_pin(void* ptr, size_t bytes) {
  if (!ptr || !bytes) return fail(ADF_E_ARG, "adf_host_pin: empty buffer");
  const cudaError_t e = cudaHostRegister(ptr, bytes, cudaHostRegisterDefault);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(ADF_E_DEVICE, std::string("adf_host_pin: ") + cudaGetErrorString(e));
  }
  return ADF_OK;
}

int adf_host_unpin(void* ptr) {
  if (!ptr) return fail(ADF_E_ARG, "adf_host_unpin: NULL pointer");
  const cudaError_t e = cudaHostUnregister(ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(ADF_E_DEVICE, std::string("adf_host_unpin: ") + cudaGetErrorString(e));
  }
  return ADF_OK;
}

int adf_last_io_bytes(adf_ctx* ctx, int64_t* h2d, int64_t* d2h) {
  if (!ctx) return fail(ADF_E_ARG, "NULL ctx");
  if (h2d) *h2d = ctx->h2d_bytes;
  if (d2h) *d2h = ctx->d2h_bytes;
  return ADF_OK;
}

int adf_kernel_timing(adf_ctx* ctx, double* ms, int64_t* n, int reset) {
  if (!ctx) return fail(ADF_E_ARG, "NULL ctx");
  if (ms) *ms = ctx->kernel_ms;
  if (n) *n = ctx->kernel_launches;
  if (reset) {
    ctx->kernel_ms = 0.0;
    ctx->kernel_launches = 0;
  }
  return ADF_OK;
}

int adf_gf_postprocess(adf_ctx* ctx, int64_t ncol, int64_t nt_in, double t_in0, double dt_in,
                       int64_t nt_out, double t_out0, double dt_out, const float* in,
                       float* out, double unit, int denoise) {
  if (!ctx || !in || !out || ncol < 1 || nt_in < 4 || nt_out < 1 || !(dt_in > 0) ||
      !(dt_out > 0) || !(unit != 0) || ncol > (1 << 28) || nt_in > (1 << 28) ||
      nt_out > (1 << 28))
    return fail(ADF_E_ARG, "adf_gf_postprocess: bad arguments");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  const int n = (int)nt_in;
  std::vector<double> cpv((size_t)n + 1, 0.0);  // Thomas pivots of (1, 4, 1)
  for (int i = 2; i <= n - 1; ++i) cpv[(size_t)i] = 1.0 / (4.0 - (i > 2 ? cpv[(size_t)i - 1] : 0.0));
  float* din = nullptr;
  float* dout = nullptr;
  double* dcoef = nullptr;
  double* dcp = nullptr;
  auto release = [&]() {
    cudaFree(din);
    cudaFree(dout);
    cudaFree(dcoef);
    cudaFree(dcp);
  };
  if (cudaMalloc(&din, (size_t)4 * n * ncol) != cudaSuccess ||
      cudaMalloc(&dout, (size_t)4 * nt_out * ncol) != cudaSuccess ||
      cudaMalloc(&dcoef, (size_t)8 * (n + 2) * ncol) != cudaSuccess ||
      cudaMalloc(&dcp, (size_t)8 * (n + 1)) != cudaSuccess) {
    release();
    cudaGetLastError();
    return fail(ADF_E_NOMEM, "adf_gf_postprocess: device allocation failed");
  }
  cudaStream_t st = ctx->stream;
  cudaMemcpyAsync(din, in, (size_t)4 * n * ncol, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dcp, cpv.data(), (size_t)8 * (n + 1), cudaMemcpyHostToDevice, st);
  cudaEventRecord(ctx->ev0, st);
  e = launch_gf_postprocess((int)ncol, n, (int)nt_out, t_in0, dt_in, t_out0, dt_out, din, dcp,
                            dcoef, dout, (float)unit, denoise ? 1 : 0, st);
  cudaEventRecord(ctx->ev1, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, dout, (size_t)4 * nt_out * ncol, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  float ms = 0.f;
  if (e == cudaSuccess) cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  release();
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  ctx->last_ms = ms;
  ctx->launches = 2;
  ctx->h2d_bytes = (int64_t)4 * n * ncol;
  ctx->d2h_bytes = (int64_t)4 * nt_out * ncol;
  return ADF_OK;
}

int adf_injection_coefficients(adf_ctx* ctx, const adf_domain* d, double radius, int64_t n,
                               double* out) {
  if (!ctx || !d || !out || n <= 0) return fail(ADF_E_ARG, "bad arguments");
  cudaSetDevice(ctx->device);
  double* dv = nullptr;
  if (cudaMalloc(&dv, 3 * sizeof(double)) != cudaSuccess) return fail(ADF_E_NOMEM, "alloc");
  launch_injection_coef(radius, n, d->dt, d->r0, d->dx, d->z0, dv, ctx->stream);
  cudaMemcpyAsync(out, dv, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  cudaFree(dv);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  return ADF_OK;
}

}  // extern "C"
