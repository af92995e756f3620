// server.cu -- impulsive Green's-function solves: batched engine, plain
// path and the continuous-batching serving loop.
//
// One request is one FDTD solve of impulsive_gfs (src/greens.jl:143-199):
// field and CPML memory start at zero, a point source fires `src_tf`, and
// p / v_n are recorded at the receivers for nt steps.  The engine keeps every
// admitted solve resident (field, psi, traces) and advances all of them with
// one step launch per time step over a (solve, tile) work list, in chunks
// captured as CUDA graphs.  Between chunks it retires finished solves
// (outputs copied out, memory freed) and admits queued ones while the HBM
// budget and the slot count allow.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "runtime.h"

namespace adf {
cudaError_t launch_cpml_profiles(int n, double vel_max, double dt, double rcoef, double thickness,
                                 double f0, float* out32, double* out64, cudaStream_t s);
cudaError_t launch_mask(int kind, const double* params, const double* xs, const double* ys,
                        const double* zs, int nx, int ny, int nz, int mw, uint32_t* bits,
                        uint8_t* jl, cudaStream_t s);

// rec [nt][ntx] -> out (nt, ntx - skip) Julia layout, dropping the first
// `skip` transceiver columns (the source's self-record, greens.jl:169-173)
__global__ void adf_extract_kernel(const float* __restrict__ rec, int nt, int ntx, int skip,
                                   float* __restrict__ out) {
  __shared__ float tile[32][33];
  const int n = ntx - skip;
  const int t0 = blockIdx.y * 32, r0 = blockIdx.x * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int t = t0 + k, r = r0 + threadIdx.x;
    tile[k][threadIdx.x] = (t < nt && r < n) ? rec[(long long)t * ntx + skip + r] : 0.f;
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = r0 + k, t = t0 + threadIdx.x;
    if (t < nt && r < n) out[(long long)r * nt + t] = tile[threadIdx.x][k];
  }
}

static cudaError_t launch_extract(const float* rec, int nt, int ntx, int skip, float* out,
                                  cudaStream_t s) {
  dim3 grid((ntx - skip + 31) / 32, (nt + 31) / 32);
  adf_extract_kernel<<<grid, dim3(32, 8), 0, s>>>(rec, nt, ntx, skip, out);
  return cudaGetLastError();
}

struct GfJob {
  adf_gf_request req;
  int64_t id = 0;
  std::chrono::steady_clock::time_point t_submit, t_done;
  int status = 0;  // 0 queued, 1 resident, 2 done, <0 error
  bool cancel = false;
  std::unique_ptr<Solve> solve;
  size_t est = 0;
  long long items = 0;  // step-kernel work items (CTAs per step launch)
};

// Work items one step launch runs for this request's grid (as solve_finalize
// builds them: x tiles x y tiles x z chunks).
static long long gf_items(const adf_gf_request& r) {
  int nxp, ty, nzc, mw;
  choose_tiles((int)r.dom.nx, (int)r.dom.ny, (int)r.dom.nz, nxp, ty, nzc, mw);
  const long long xt = step_x_tile();
  return (nxp + xt - 1) / xt * ((r.dom.ny + ty - 1) / ty) * ((r.dom.nz + nzc - 1) / nzc);
}

static size_t gf_bytes(const adf_gf_request& r) {
  int nxp, ty, nzc, mw;
  choose_tiles((int)r.dom.nx, (int)r.dom.ny, (int)r.dom.nz, nxp, ty, nzc, mw);
  const size_t nx = r.dom.nx, ny = r.dom.ny, nz = r.dom.nz, n = r.npml, nt = r.dom.nt;
  const size_t ntx = 1 + r.n_rec;
  size_t b = 2ull * 4 * nz * ny * nxp * 4;
  if (r.shape != ADF_SHAPE_NONE) b += (size_t)mw * ny * nz * 4;
  b += 2ull * 2 * 4 * (nz * ny * n + nz * n * nxp + n * ny * nxp);
  b += 2ull * 2 * 4 * (nz * ny * (n + 1) + nz * (n + 1) * nxp + (n + 1) * ny * nxp);
  b += 2ull * nt * ntx * 4 + 4ull * nt * 4;  // p/vn records + source columns
  b += 2ull * nt * (ntx - 1) * 4;            // output staging
  b += ntx * 4 * 8 * 4 * 4;                  // contributions + entries
  b += (size_t)((ny + ty - 1) / ty) * nz * 16;
  (void)nx;
  return b + (1 << 20);
}

// Device set-up of one GF solve on the context stream.
static int gf_setup(adf_ctx* ctx, GfJob& j) {
  const adf_gf_request& r = j.req;
  const adf_domain& dd = r.dom;
  if (dd.nx < 4 || dd.ny < 4 || dd.nz < 4 || dd.nx > 512 || dd.nt < 1 || r.n_rec < 0 ||
      r.npml < 0 || r.npml > 63 || !r.src_tf || (r.n_rec > 0 && (!r.rec_points || !r.rec_normals)) ||
      !r.out_p || !r.out_vn)
    return fail(ADF_E_ARG, "bad GF request");
  auto s = std::make_unique<Solve>();
  s->alloc_stream = ctx->stream;
  s->alloc_pool = ctx->pool;
  const hm::Dom dom = to_dom(dd);
  const bool has_mask = r.shape != ADF_SHAPE_NONE;
  const int ntx = 1 + (int)r.n_rec;
  int rc = solve_alloc(ctx, *s, dom, (int)r.npml, has_mask, r.flags, ntx);
  if (rc) return rc;
  SolveDev& d = s->dev;
  const size_t nt = (size_t)dd.nt;
  // traces: p and v_n records of every transceiver, source columns of tx 0
  d.rec[0] = solve_dalloc<float>(*s, nt * ntx, rc);
  d.vn_rec = solve_dalloc<float>(*s, nt * ntx, rc);
  float* srcs = solve_dalloc<float>(*s, 4 * nt, rc);
  float* dir = solve_dalloc<float>(*s, (size_t)4 * ntx, rc);
  float* stage = solve_dalloc<float>(*s, 2 * nt * (size_t)std::max(1, ntx - 1), rc);
  if (rc) return rc;
  cudaStream_t st = ctx->stream;
  cudaMemsetAsync(d.rec[0], 0, nt * ntx * 4, st);
  cudaMemsetAsync(d.vn_rec, 0, nt * ntx * 4, st);
  for (int c = 0; c < 4; ++c) d.src[c] = srcs + c * nt;
  d.src_ntx = 1;
  d.vn_src = nullptr;
  d.dir = dir;
  s->dir_dev = dir;
  s->stage = stage;
  // host packing: transceiversToGrid of [source, receivers...]
  std::vector<float> idx[4], w[4];
  for (int c = 0; c < 4; ++c) {
    idx[c].resize((size_t)3 * ntx);
    w[c].resize((size_t)8 * ntx);
  }
  std::vector<float> dirs((size_t)4 * ntx, 0.0f);
  for (int tx = 0; tx < ntx; ++tx) {
    double pt[3], dv[4];
    if (tx == 0) {
      for (int q = 0; q < 3; ++q) pt[q] = r.src_point[q];
      for (int q = 0; q < 4; ++q) dv[q] = r.src_dir[q];
    } else {
      for (int q = 0; q < 3; ++q) pt[q] = r.rec_points[3 * (tx - 1) + q];
      dv[0] = 0.0;
      for (int q = 0; q < 3; ++q) dv[q + 1] = r.rec_normals[3 * (tx - 1) + q];
    }
    int64_t ii[12];
    double ww[32];
    if (!hm::trilinear(dom, pt, ii, ww))
      return fail(ADF_E_ARG, "transceiver " + std::to_string(tx) + " lies outside the grid");
    for (int c = 0; c < 4; ++c) {
      for (int q = 0; q < 3; ++q) idx[c][3 * tx + q] = (float)ii[3 * c + q];
      for (int q = 0; q < 8; ++q) w[c][8 * tx + q] = (float)ww[8 * c + q];
    }
    for (int q = 0; q < 4; ++q) dirs[4 * tx + q] = (float)dv[q];
  }
  std::vector<float> sv(4 * nt);
  for (int c = 0; c < 4; ++c)
    for (size_t t = 0; t < nt; ++t) sv[c * nt + t] = (float)(r.src_tf[t] * r.src_dir[c]);
  cudaError_t ue = cudaSuccess;  // the first failed set-up copy or launch
  auto up = [&](cudaError_t e) {
    if (ue == cudaSuccess && e != cudaSuccess) ue = e;
  };
  up(cudaMemcpyAsync(srcs, sv.data(), sv.size() * 4, cudaMemcpyHostToDevice, st));
  up(cudaMemcpyAsync(dir, dirs.data(), dirs.size() * 4, cudaMemcpyHostToDevice, st));
  s->h2d += (int64_t)(sv.size() * 4 + dirs.size() * 4);
  // CPML profiles in FP64 on the device: Cpml(dom; npml, rcoef, fc)
  if (r.npml > 0)
    up(launch_cpml_profiles((int)r.npml, dd.c0, dd.dt, r.pml_rcoef, dd.dx * (double)r.npml,
                            r.pml_fc, s->coef_dev, nullptr, st));
  // scatterer mask straight into the bitmask
  double* xyz = nullptr;
  if (has_mask) {
    std::vector<double> c((size_t)(dd.nx + dd.ny + dd.nz));
    for (int a = 0; a < 3; ++a) {
      hm::Range rr = hm::axis_range(dom, a, 0);
      double* o = c.data() + (a == 0 ? 0 : a == 1 ? dd.nx : dd.nx + dd.ny);
      for (int64_t i = 1; i <= rr.len; ++i) o[i - 1] = rr.at(i);
    }
    if (cudaMallocFromPoolAsync((void**)&xyz, c.size() * 8, ctx->pool, st) != cudaSuccess)
      return fail(ADF_E_NOMEM, "alloc");
    up(cudaMemcpyAsync(xyz, c.data(), c.size() * 8, cudaMemcpyHostToDevice, st));
    s->h2d += (int64_t)(c.size() * 8);
    up(launch_mask(r.shape, r.shape_params, xyz, xyz + dd.nx, xyz + dd.nx + dd.ny, (int)dd.nx,
                   (int)dd.ny, (int)dd.nz, d.mw, s->mask_bits, nullptr, st));
    up(cudaStreamSynchronize(st));  // before `c` goes out of scope
    cudaFreeAsync(xyz, st);
  }
  std::vector<int> col(ntx, -1);
  col[0] = 0;
  const float* ip[4] = {idx[0].data(), idx[1].data(), idx[2].data(), idx[3].data()};
  const float* wp[4] = {w[0].data(), w[1].data(), w[2].data(), w[3].data()};
  rc = solve_finalize(ctx, *s, ip, wp, col.data());
  if (rc) return rc;
  up(cudaStreamSynchronize(st));  // sv and dirs outlive their copies
  if (ue != cudaSuccess) {
    cudaGetLastError();
    return fail(ADF_E_DEVICE, std::string("GF set-up: ") + cudaGetErrorString(ue));
  }
  ctx->h2d_bytes += s->h2d;
  d.it_first = 1;
  d.it_base = 1;
  d.it_stop = (int)dd.nt;
  j.solve = std::move(s);
  return ADF_OK;
}

// Outputs of a finished solve into the request's buffers (synchronises).
static int gf_extract(adf_ctx* ctx, GfJob& j) {
  Solve& s = *j.solve;
  const SolveDev& d = s.dev;
  const int n = d.ntx - 1;
  const size_t nt = (size_t)d.nt;
  cudaStream_t st = ctx->stream;
  cudaError_t e = cudaSuccess;
  if (n > 0) {
    e = launch_extract(d.rec[0], d.nt, d.ntx, 1, s.stage, st);
    if (e == cudaSuccess) e = launch_extract(d.vn_rec, d.nt, d.ntx, 1, s.stage + nt * n, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(j.req.out_p, s.stage, nt * n * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(j.req.out_vn, s.stage + nt * n, nt * n * 4, cudaMemcpyDeviceToHost, st);
    ctx->d2h_bytes += (int64_t)(2 * nt * n * 4);
  }
  // the stream is synchronised even after a failed enqueue: the host
  // buffers may still be targets of copies already issued
  const cudaError_t es = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = es;
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(ADF_E_DEVICE, std::string("GF output download: ") + cudaGetErrorString(e));
  }
  return ADF_OK;
}

class Engine {
 public:
  Engine(adf_ctx* ctx, size_t budget, int max_resident, int chunk)
      : ctx_(ctx), budget_(budget), max_resident_(max_resident), chunk_(chunk) {}

  void enqueue(GfJob* j) { pending_.push_back(j); }
  // Admission by work: a request joins only while the resident solves' step
  // work items stay within max_items (one solve is always admitted); 0 = no cap.
  void set_work_cap(long long max_items) { max_items_.store(max_items); }
  bool idle() const { return pending_.empty() && resident_.empty(); }
  size_t resident() const { return resident_.size(); }

  // admit -> run one chunk -> retire; returns an error only for device failure
  int tick(std::vector<GfJob*>* finished) {
    admit(finished);
    if (resident_.empty()) return ADF_OK;
    if (dirty_) {
      std::vector<Solve*> list;
      for (GfJob* j : resident_) list.push_back(j->solve.get());
      int rc = batch_.setup(ctx_, list);
      if (rc) return rc;
      dirty_ = false;
    }
    int max_rem = 0;
    for (GfJob* j : resident_)
      max_rem = std::max(max_rem, j->solve->dev.it_stop - j->solve->dev.it_base + 1);
    const int n = std::min(chunk_, max_rem);
    // Requests still queued after admit() cannot join before a resident
    // solve finishes (memory, work cap or slots are exhausted): replay full
    // chunks back to back up to the first such retirement and synchronise
    // once, instead of returning to the host after every chunk.  With the
    // queue empty, one chunk per tick keeps new arrivals' admission prompt.
    int reps = 1;
    if (!pending_.empty() && n == chunk_ && !ctx_->kernel_timing) {
      int min_rem = max_rem;
      for (GfJob* j : resident_)
        min_rem = std::min(min_rem, j->solve->dev.it_stop - j->solve->dev.it_base + 1);
      reps = std::max(1, (min_rem + chunk_ - 1) / chunk_);
    }
    int rc = ADF_OK;
    for (int r = 0; r < reps; ++r) {
      rc = batch_.run_chunk(ctx_, n, chunk_);
      if (rc) return rc;
      for (GfJob* j : resident_) j->solve->dev.it_base += n;
    }
    rc = batch_.check_error(ctx_);  // synchronises the stream
    if (rc) return rc;
    batch_.collect_kernel_times(ctx_, n);
    retire(finished);
    return ADF_OK;
  }

 private:
  void admit(std::vector<GfJob*>* finished) {
    while (!pending_.empty() && (int)resident_.size() < max_resident_) {
      GfJob* j = pending_.front();
      if (j->cancel) {
        pending_.pop_front();
        j->status = ADF_E_CANCELLED;
        j->t_done = std::chrono::steady_clock::now();
        finished->push_back(j);
        continue;
      }
      if (!j->est) j->est = gf_bytes(j->req);
      if (j->est > budget_) {  // can never fit
        pending_.pop_front();
        fail(ADF_E_BUDGET, "GF request exceeds the HBM budget");
        j->status = ADF_E_BUDGET;
        j->t_done = std::chrono::steady_clock::now();
        finished->push_back(j);
        continue;
      }
      if (used_ + j->est > budget_) break;  // wait for memory to free up
      if (!j->items) j->items = gf_items(j->req);
      const long long cap = max_items_.load();
      if (cap > 0 && !resident_.empty() && items_ + j->items > cap) break;  // GPU full
      pending_.pop_front();
      int rc = gf_setup(ctx_, *j);
      if (rc) {
        j->solve.reset();
        j->status = rc;
        j->t_done = std::chrono::steady_clock::now();
        finished->push_back(j);
        continue;
      }
      used_ += j->est;
      items_ += j->items;
      j->status = 1;
      resident_.push_back(j);
      dirty_ = true;
    }
  }

  void retire(std::vector<GfJob*>* finished) {
    std::vector<GfJob*> keep;
    for (GfJob* j : resident_) {
      const SolveDev& d = j->solve->dev;
      if (j->cancel || d.it_base > d.it_stop) {
        int rc = j->cancel ? ADF_E_CANCELLED : gf_extract(ctx_, *j);
        j->solve.reset();
        used_ -= j->est;
        items_ -= j->items;
        j->status = rc ? rc : 2;
        j->t_done = std::chrono::steady_clock::now();
        finished->push_back(j);
        dirty_ = true;
      } else {
        keep.push_back(j);
      }
    }
    resident_.swap(keep);
  }

  adf_ctx* ctx_;
  size_t budget_;
  int max_resident_;
  int chunk_;
  size_t used_ = 0;
  std::atomic<long long> max_items_{0};
  long long items_ = 0;
  std::deque<GfJob*> pending_;
  std::vector<GfJob*> resident_;
  Batch batch_;
  bool dirty_ = true;
};

}  // namespace adf

using namespace adf;

struct adf_server {
  adf_ctx* ctx = nullptr;
  std::unique_ptr<Engine> eng;
  std::thread th;
  std::mutex mu;
  std::condition_variable cv, cv_done;
  std::deque<GfJob*> inbox;
  std::unordered_map<int64_t, std::unique_ptr<GfJob>> jobs;
  int64_t next_id = 1;
  int64_t outstanding = 0;
  bool stop = false;
  int dev_error = 0;
};

static void server_loop(adf_server* s) {
  cudaSetDevice(s->ctx->device);
  std::vector<GfJob*> done;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (s->eng->idle() && s->inbox.empty()) {
        if (s->stop) break;
        s->cv.wait_for(lk, std::chrono::milliseconds(50));
        if (s->stop && s->inbox.empty() && s->eng->idle()) break;
      }
      while (!s->inbox.empty()) {
        s->eng->enqueue(s->inbox.front());
        s->inbox.pop_front();
      }
    }
    done.clear();
    int rc = s->eng->tick(&done);
    std::lock_guard<std::mutex> lk(s->mu);
    for (GfJob* j : done) --s->outstanding;
    if (rc) {
      s->dev_error = rc;
      s->stop = true;
    }
    if (!done.empty() || rc) s->cv_done.notify_all();
    if (rc) break;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  s->cv_done.notify_all();
}

extern "C" {

int adf_gf_solve_batch(adf_ctx* ctx, int64_t n, adf_gf_request* reqs, int batched) {
  if (!ctx || n < 0 || (n > 0 && !reqs)) return fail(ADF_E_ARG, "bad arguments");
  cudaSetDevice(ctx->device);
  std::vector<std::unique_ptr<GfJob>> jobs;
  for (int64_t i = 0; i < n; ++i) {
    jobs.emplace_back(new GfJob());
    jobs.back()->req = reqs[i];
    jobs.back()->id = i;
  }
  ctx->launches = 0;
  ctx->h2d_bytes = 0;
  ctx->d2h_bytes = 0;
  double dev_ms = 0.0;
  int rc = ADF_OK;
  if (batched) {
    Engine eng(ctx, ctx->budget, 1 << 20, kGraphChunk);
    for (auto& j : jobs) eng.enqueue(j.get());
    std::vector<GfJob*> done;
    cudaEventRecord(ctx->ev0, ctx->stream);
    while (!eng.idle() && !rc) rc = eng.tick(&done);
    cudaEventRecord(ctx->ev1, ctx->stream);
    cudaEventSynchronize(ctx->ev1);
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    dev_ms = ms;
  } else {
    // plain path: one solve at a time, one launch (plus trace epilogue) per step
    for (auto& jp : jobs) {
      GfJob& j = *jp;
      rc = gf_setup(ctx, j);
      if (rc) break;
      Batch b;
      rc = b.setup(ctx, {j.solve.get()});
      if (rc) break;
      cudaEventRecord(ctx->ev0, ctx->stream);
      const int nt = j.solve->dev.nt;
      for (int s0 = 0; s0 < nt && !rc; s0 += kGraphChunk) {
        const int n = std::min(kGraphChunk, nt - s0);
        for (int s = 0; s < n && !rc; ++s) {
          rc = b.launch_step(ctx, s);
          ctx->launches += 2;
        }
        if (!rc) rc = b.run_advance(ctx, n);
        if (!rc && ctx->kernel_timing) {
          cudaStreamSynchronize(ctx->stream);
          b.collect_kernel_times(ctx, n);
        }
      }
      cudaEventRecord(ctx->ev1, ctx->stream);
      if (!rc) rc = b.check_error(ctx);
      float ms = 0;
      cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
      dev_ms += ms;
      j.solve->dev.it_base = nt + 1;
      if (!rc) rc = gf_extract(ctx, j);
      j.solve.reset();
      j.status = rc ? rc : 2;
      if (rc) break;
    }
  }
  ctx->last_ms = dev_ms;
  if (rc) return rc;
  for (auto& j : jobs)
    if (j->status != 2) return j->status < 0 ? j->status : fail(ADF_E_STATE, "request not run");
  return ADF_OK;
}

int adf_server_start(adf_ctx* ctx, size_t hbm_budget, int max_resident, adf_server** out) {
  if (!ctx || !out) return fail(ADF_E_ARG, "NULL argument");
  auto* s = new adf_server();
  s->ctx = ctx;
  const size_t budget = hbm_budget ? std::min(hbm_budget, ctx->budget) : ctx->budget;
  s->eng.reset(new Engine(ctx, budget, max_resident > 0 ? max_resident : 1 << 20, kGraphChunk));
  s->th = std::thread(server_loop, s);
  *out = s;
  return ADF_OK;
}

int adf_server_set_work_cap(adf_server* s, int64_t max_items) {
  if (!s || max_items < 0) return fail(ADF_E_ARG, "adf_server_set_work_cap: bad arguments");
  s->eng->set_work_cap((long long)max_items);
  return ADF_OK;
}

int adf_step_resident_ctas(adf_ctx* ctx, int64_t* n) {
  if (!ctx || !n) return fail(ADF_E_ARG, "NULL argument");
  int per_sm = 0;
  const cudaError_t e = step_ctas_per_sm(&per_sm);
  if (e != cudaSuccess) return fail(ADF_E_DEVICE, cudaGetErrorString(e));
  *n = (int64_t)per_sm * ctx->nsm;
  return ADF_OK;
}

int adf_server_submit(adf_server* s, const adf_gf_request* req, int64_t* id) {
  if (!s || !req || !id) return fail(ADF_E_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return fail(ADF_E_STATE, s->dev_error ? "server stopped on a device error"
                                                     : "server is stopping");
  auto j = std::make_unique<GfJob>();
  j->req = *req;
  j->id = s->next_id++;
  j->t_submit = std::chrono::steady_clock::now();
  *id = j->id;
  s->inbox.push_back(j.get());
  s->jobs[j->id] = std::move(j);
  ++s->outstanding;
  s->cv.notify_all();
  return ADF_OK;
}

int adf_server_poll(adf_server* s, int64_t id, int* status, double* latency_ms) {
  if (!s || !status) return fail(ADF_E_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return fail(ADF_E_NOTFOUND, "unknown request id");
  GfJob& j = *it->second;
  *status = j.status == 2 ? 1 : (j.status < 0 ? j.status : 0);
  if (latency_ms)
    *latency_ms = j.status == 2 || j.status < 0
                      ? std::chrono::duration<double, std::milli>(j.t_done - j.t_submit).count()
                      : 0.0;
  return ADF_OK;
}

int adf_server_cancel(adf_server* s, int64_t id) {
  if (!s) return fail(ADF_E_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return fail(ADF_E_NOTFOUND, "unknown request id");
  it->second->cancel = true;
  return ADF_OK;
}

int adf_server_drain(adf_server* s) {
  if (!s) return fail(ADF_E_ARG, "NULL argument");
  std::unique_lock<std::mutex> lk(s->mu);
  s->cv_done.wait(lk, [s] { return s->outstanding == 0 || s->dev_error != 0; });
  if (s->dev_error) return fail(s->dev_error, "server stopped on a device error");
  return ADF_OK;
}

int adf_server_stop(adf_server* s) {
  if (!s) return ADF_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (auto& kv : s->jobs)
      if (kv.second->status <= 1) kv.second->cancel = true;
    s->cv.notify_all();
  }
  if (s->th.joinable()) s->th.join();
  int err = s->dev_error;
  delete s;
  return err ? fail(err, "server stopped on a device error") : ADF_OK;
}

}  // extern "C"
