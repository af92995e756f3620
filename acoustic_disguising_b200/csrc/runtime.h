// runtime.h -- host-side objects behind the C-ABI.
#pragma once

#include <string>
#include <vector>

#include "../../include/adfdtd.h"
#include "adf_internal.h"
#include "host_math.h"

namespace adf {
struct Solve;
}

struct adf_ctx {
  int device = 0;
  int nsm = 148;
  int smem_per_sm = 233472;
  int smem_optin = 232448;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // stream-ordered pool of the GF engine's solve memory; it keeps freed
  // blocks mapped, so a solve admitted after another one retires reuses its
  // memory instead of mapping fresh gigabytes
  cudaMemPool_t pool = nullptr;
  size_t budget = 0;
  struct adf::Solve* cur = nullptr;  // solve whose field adf_read_field reads
  int64_t cur_it = 0;
  double last_ms = 0.0;
  double kh_ms = 0.0;  // kernel time of the last KH extrapolation
  int64_t launches = 0;
  // per-launch timing of the step kernel
  int64_t h2d_bytes = 0, d2h_bytes = 0;  // traffic of the last call
  bool kernel_timing = false;
  // one-shot test hook of the next KH call (adf_kh_test_fault)
  int kh_skip_chunk = -1;
  uint32_t kh_wait_limit = 0;
  std::vector<cudaEvent_t> kev;  // 2 per launch-step of a chunk
  double kernel_ms = 0.0;
  int64_t kernel_launches = 0;
};

namespace adf {

constexpr int kGraphChunk = 32;  // steps per captured CUDA graph
static_assert(kGraphChunk % kGfBlock == 0, "a graph chunk holds whole GF blocks");

int fail(int code, const std::string& msg);

inline hm::Dom to_dom(const adf_domain& d) {
  hm::Dom o;
  o.tmax = d.tmax; o.xmax = d.xmax; o.ymax = d.ymax; o.zmax = d.zmax;
  o.nx = d.nx; o.ny = d.ny; o.nz = d.nz;
  o.c0 = d.c0; o.r0 = d.r0; o.cf = d.cf;
  o.dx = d.dx; o.dy = d.dy; o.dz = d.dz;
  o.fact_m0 = d.fact_m0; o.fact_m1 = d.fact_m1; o.dt = d.dt; o.nt = d.nt; o.z0 = d.z0;
  return o;
}

// Tile shape per grid size: rows per tile and z-chunk depth.  Chosen by the
// autotuner (tune.cpp) and cached in a JSON table beside the library.
struct Tune {
  int ty;
  int nzc;
};
Tune tune_lookup(int nx, int ny, int nz);
int tune_store(int nx, int ny, int nz, Tune t);
void tune_force(Tune t);  // {0,0} releases

struct Solve {
  SolveDev dev;
  unsigned char fmap_host[4 * 128];  // the tensor maps of dev.fmap (copied to the device)
  std::vector<void*> allocs;
  size_t bytes = 0;
  int nzc = 32;
  uint32_t* mask_bits = nullptr;
  float* coef_dev = nullptr;
  float* dir_dev = nullptr;
  float* stage = nullptr;  // output staging of GF solves
  int64_t h2d = 0;         // bytes uploaded while setting this solve up
  long long n_entries = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t alloc_stream = nullptr;  // stream-ordered allocation from alloc_pool when set
  cudaMemPool_t alloc_pool = nullptr;
  std::vector<int4> items;  // {0, y tile | x tile << 16, z0, z1}
  ~Solve();
  void release();
};

struct Batch {
  std::vector<Solve*> solves;
  SolveDev* d_solves = nullptr;
  int4* d_items = nullptr;
  int cap_solves = 0, cap_items = 0;
  int n_items = 0, grid = 1, max_ntx = 0;
  int max_ty = 1;            // tallest tile in the batch: the block is (32, max_ty + 1)
  int max_gf_nsrc = 0;       // > 0: some solve runs the in-loop GF extrapolation
  int max_gf_blocks = 0;     // (source, receiver split) blocks of the GF kernel
  int max_gf_far_blocks = 0; // (source tile, receiver split) blocks of the far-lag kernel
  int max_gf_tc_blocks = 0;  // the same for the tensor-core far-lag kernel
  // far-lag kernels launched per block of kGfBlock steps (FP64, tensor-core, combine)
  int far_launches() const {
    const int k = (max_gf_far_blocks > 0) + (max_gf_tc_blocks > 0);
    return k > 0 ? k + 1 : 0;
  }
  bool gf_reduce = false;    // some GF solve splits a source's receivers over blocks
  int per_step = 2;          // kernel launches per launch-step
  cudaGraphExec_t graph_exec = nullptr;
  int graph_steps = 0;
  ~Batch();
  void release();
  int setup(adf_ctx* ctx, const std::vector<Solve*>& list);
  int launch_step(adf_ctx* ctx, int step);
  int run(adf_ctx* ctx, int nsteps, bool use_graph, int chunk);
  int run_chunk(adf_ctx* ctx, int n, int chunk);
  void collect_kernel_times(adf_ctx* ctx, int n);
  int run_advance(adf_ctx* ctx, int n);  // after the stream is synchronised
  int check_error(adf_ctx* ctx);
};

void choose_tiles(int nx, int ny, int nz, int& nxp, int& ty, int& nzc, int& mw);
size_t solve_bytes_estimate(int64_t nx, int64_t ny, int64_t nz, int64_t npml, int64_t ntx,
                            int64_t nt, bool mask);
int solve_alloc(adf_ctx* ctx, Solve& s, const hm::Dom& dom, int npml, bool has_mask, int arith,
                int ntx);
int solve_alloc_traces(Solve& s, bool need_vsrc);
int solve_finalize(adf_ctx* ctx, Solve& s, const float* const idx[4], const float* const w[4],
                   const int* src_col);
template <typename T>
T* solve_dalloc(Solve& s, size_t n, int& rc);

// set-up helpers (setup.cu)
int build_mask_device(adf_ctx* ctx, const adf_domain& d, int shape, const double* params, int mw,
                      uint32_t** bits, uint8_t** jl);
int pack_transceivers_host(const hm::Dom& d, const double* points, const double* dirs,
                           const double* tf, adf_txgrid* o);

// KH pressure on columns of device-resident traces (kh_kernel.cu): q and f
// are [nt][ntx] arrays in HBM (a solve's vn_rec and p_rec), cols the ns
// 0-based columns in device memory; out (nt, nr) on the host.
struct KhDevSrc {
  const float* q;
  const float* f;
  int ntx;
  const int* cols;
};
int kh_pressure_dev(adf_ctx* ctx, const adf_kh_desc* d, const KhDevSrc& src, float* out);

// kernels (fdtd_kernels.cu)
cudaError_t launch_advance(SolveDev* solves, int n, int by, cudaStream_t s);

}  // namespace adf
