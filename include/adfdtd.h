/*
 * adfdtd.h -- C-ABI of the B200 FDTD + Kirchhoff-Helmholtz library
 * (libadfdtd.so).  This is the drop-in boundary that the reference's Julia
 * host code binds with `ccall`; each entry point names the reference
 * routine it replaces (paths are inside the AcousticDisguising project).
 *
 * Conventions
 *  - Arrays crossing this boundary use the reference's Julia layout:
 *    column-major, first index fastest, the shapes the reference uses.
 *    Indices stored in arrays are 1-based exactly as the reference packs
 *    them (Float32 in TransceiverGrid); plain C pointers and sizes only.
 *  - Every function returns int: 0 (ADF_OK) or a negative ADF_E_* code.
 *    A message for the last failure on the calling thread is available
 *    from adf_last_error().  Nothing aborts the process and no device code
 *    traps: device-side waits are bounded and report ADF_E_TIMEOUT.
 *  - An adf_ctx owns one CUDA device's streams and buffers.  A context is
 *    not shared between host threads without external locking; any number
 *    of contexts may exist.  The serving calls (adf_server_*) are
 *    thread-safe.
 */
#ifndef ADFDTD_H
#define ADFDTD_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define ADF_OK 0
#define ADF_E_ARG (-1)        /* bad argument / shape                       */
#define ADF_E_NOMEM (-2)      /* device allocation failed                   */
#define ADF_E_BUDGET (-3)     /* request exceeds the context's HBM budget   */
#define ADF_E_CANCELLED (-4)  /* cancelled by callback / server stop       */
#define ADF_E_DEVICE (-5)     /* CUDA error                                 */
#define ADF_E_TIMEOUT (-6)    /* a bounded device-side wait gave up         */
#define ADF_E_STATE (-7)      /* call not valid in the current state        */
#define ADF_E_NOTFOUND (-8)   /* unknown request id                         */

/* run flags (adf_run_fdtd / GF requests) */
#define ADF_ARITH_PROMOTE 0   /* Float32 storage, Float64 intermediates, as
                                 Julia promotes the Float64 Domain scalars  */
#define ADF_ARITH_FP32 1      /* Float32 arithmetic throughout              */

/* scatterer shapes: geometry.jl:86-143 (+ centred/ellipsoid extensions) */
#define ADF_SHAPE_NONE 0
#define ADF_SHAPE_SPHERE 1    /* params {radius, cx, cy, cz}                */
#define ADF_SHAPE_CUBE 2      /* params {length, cx, cy, cz}                */
#define ADF_SHAPE_CROSS 3     /* params {length}                            */
#define ADF_SHAPE_ELLIPSOID 4 /* params {ax, ay, az, cx, cy, cz}            */

/* Mirror of `struct Domain` (src/simulation.jl:25-44). */
typedef struct {
  double tmax, xmax, ymax, zmax;
  int64_t nx, ny, nz;
  double c0, r0, cf;
  double dx, dy, dz;
  double fact_m0, fact_m1;
  double dt;
  int64_t nt;
  double z0;
} adf_domain;

/* Mirror of `TransceiverGrid` / `ChannelBuffers` (src/simulation.jl:354-378);
 * host arrays in Julia layout, channel order 0=p 1=vx 2=vy 3=vz.
 *   idx[c] (3,ntx) Float32 1-based; w[c] (2,2,2,ntx); src[c], rec[c] (nt,ntx)
 *   dir (4,ntx); vn_src, vn_rec (nt,ntx).                                    */
typedef struct {
  int64_t ntx, nt;
  float* idx[4];
  float* w[4];
  float* src[4];
  float* rec[4];
  float* dir;
  float* vn_src;
  float* vn_rec;
} adf_txgrid;

/* Mirror of `Cpml` (src/simulation.jl:200-227), Julia layout host arrays:
 *   mv[0] (npml,ny,nz,2) mv[1] (nx,npml,nz,2) mv[2] (nx,ny,npml,2)
 *   mp[d]: the same with npml+1 along axis d.
 *   coef: Float32 a_l[n] a_r[n] a_hl[n+1] a_hr[n+1] b_l[n] b_r[n] b_hl[n+1] b_hr[n+1]
 * mv/mp may be NULL when npml == 0.                                         */
typedef struct {
  int64_t npml;
  float* mv[3];
  float* mp[3];
  const float* coef;
} adf_cpml;

typedef struct adf_ctx adf_ctx;

/* Called after each completed step `it` (1-based) when passed to
 * adf_run_fdtd; the `on_step(it, field)` hook of run_fdtd!
 * (src/simulation.jl:551-553).  Return nonzero to cancel.  Inside the
 * callback adf_read_field() reads the current field.                       */
typedef int (*adf_step_cb)(int64_t it, void* user);

int adf_version(void);
/* Copies the calling thread's last error message (NUL-terminated). */
int adf_last_error(char* buf, size_t n);

/* Context: one device, one HBM budget (bytes, 0 = 90% of free memory). */
int adf_ctx_create(int device, size_t hbm_budget, adf_ctx** out);
int adf_ctx_destroy(adf_ctx* ctx);

/* Domain(; tmax, xmax, ymax, zmax, nx, ny, nz, c0, r0, cf)
 * (src/simulation.jl:46-79); host arithmetic, identical to the reference. */
int adf_domain_make(double tmax, double xmax, double ymax, double zmax, int64_t nx,
                    int64_t ny, int64_t nz, double c0, double r0, double cf, adf_domain* out);

/* coords(d)[axis][chan] (src/simulation.jl:86-115): the Float64 values of
 * Julia's range(-xmax; stop=xmax, length=n) (minus d/2 on the staggered
 * axis), reproduced in twice-precision arithmetic.  Host.                  */
int adf_coords(const adf_domain* d, int axis, int chan, double* out);
/* t(d) = range(0; stop=tmax, length=nt) (src/simulation.jl:86), host. */
int adf_time_axis(const adf_domain* d, double* out);

/* compute_CPML_coefficients! + calc_Kab_CPML (src/kernels/cpmlcoeffs.jl:36-126),
 * evaluated in FP64 on the GPU and rounded to Float32 as Data.Array stores
 * them.  out32: 8 arrays as in adf_cpml.coef (8*npml+4 floats); out64 may be
 * NULL or receive the same arrays in Float64.                              */
int adf_cpml_profiles(adf_ctx* ctx, int64_t npml, double vel_max, double dt, double rcoef,
                      double thickness, double fc, float* out32, double* out64);

/* adf_cpml_profiles without any device allocation; no counterpart in the
 * reference.  For callers that must not allocate or free device memory while
 * work is in flight: cudaFree synchronizes the whole device (stalling solves
 * running on other streams), and a serving process may have handed all of
 * HBM to its solve budget.  Scratch is a fixed device array sized for
 * npml <= 63 (the largest npml the step kernel accepts); larger npml returns
 * ADF_E_ARG.  The first call on each device does a one-time set-up (it takes
 * the array's address, which may load the module), so make it before any
 * stream capture.  Nothing has to be zeroed first.  Calls that overlap on
 * one device share the array and race: serialize them.  Results equal
 * adf_cpml_profiles bit for bit.                                          */
int adf_cpml_profiles_static(adf_ctx* ctx, int64_t npml, double vel_max, double dt,
                             double rcoef, double thickness, double fc, float* out32,
                             double* out64);
/* The largest npml adf_cpml_profiles_static accepts, for callers that
 * cannot read the macro (ccall, ctypes).  Always ADF_STATIC_CPML_MAX_NPML. */
#define ADF_STATIC_CPML_MAX_NPML 63
int adf_static_cpml_max_npml(void);

/* build_update_mask (src/geometry.jl:250-280), evaluated on the GPU.
 * out_bool: (nx,ny,nz,4) uint8 Julia layout, or NULL.  Returns 1 (writing
 * nothing) for ADF_SHAPE_NONE, as the reference returns `nothing`.        */
int adf_build_mask(adf_ctx* ctx, const adf_domain* d, int shape, const double* params,
                   uint8_t* out_bool);

/* transceiversToGrid (src/simulation.jl:387-431) for transceivers built by
 * Transceiver(d; point, direction, tf) (src/simulation.jl:176-186).
 * points (3,ntx), dirs (4,ntx), tf (nt,ntx) Float64; fills the caller's
 * arrays of *out (ntx, nt set by the caller).  Host.                       */
int adf_pack_transceivers(const adf_domain* d, const double* points, const double* dirs,
                          const double* tf, adf_txgrid* out);

/* run_fdtd!(dom, field, txs, cpml, va; start_step, on_step)
 * (src/simulation.jl:542-557) / forward_onestep! (src/kernels/forward.jl:13-139)
 * for it = start_step .. stop_step (1-based, stop_step <= nt).
 * field (nx,ny,nz,4) Float32 host array, updated in place; txs rec/src/
 * vn_rec and cpml memory are updated in place as the reference does.
 * mask: build_update_mask's (nx,ny,nz,4) Bool array as uint8, or NULL.
 * flags: ADF_ARITH_*.  cb may be NULL.                                    */
int adf_run_fdtd(adf_ctx* ctx, const adf_domain* d, float* field, adf_txgrid* txs,
                 adf_cpml* cpml, const uint8_t* mask, int64_t start_step, int64_t stop_step,
                 int flags, adf_step_cb cb, void* user);

/* GFMap of run_fdtd!(...; gf_map) (src/kernels/extrapolation.jl:36-87).
 * Tensors are (nt_gf, n1, n2) Float32 in Julia layout; i_src/i_rec are
 * 1-based transceiver indices (iSrc, iRec).
 *   ADF_GF_PV_FROM_PIN  t = {p_pin, v_pin}, n1 = #iSrc, n2 = #iRec
 *   ADF_GF_P_FROM_PIN   t = {pos, neg},     n1 = #iRec, n2 = #iSrc
 *   ADF_GF_PV_FROM_PV   t = {pp, pv, vp, vv}, n1 = #iRec, n2 = #iSrc       */
#define ADF_GF_PV_FROM_PIN 0
#define ADF_GF_P_FROM_PIN 1
#define ADF_GF_PV_FROM_PV 2
typedef struct {
  int kind;
  int64_t nt_gf, n1, n2;
  const float* t[4];
  const int64_t* i_src;
  int64_t n_src;
  const int64_t* i_rec;
  int64_t n_rec;
  double z0;
  int discard;  /* 1: as the reference ships (extrapolate! writes into slice
                   copies, extrapolation.jl:215-216, 228-229, 246-247, so the
                   sources never change); 0: the documented intent, the
                   extrapolated samples are written into txs's sources     */
  int contraction; /* ADF_GF_CONTRACT_FP64 (0): every lag summed with Float64
                      FMAs, as the reference accumulates; ADF_GF_CONTRACT_TF32X3
                      (1): the *FromPin kinds sum the lags older than the
                      current 32-step block on the tensor cores (TF32 split
                      into three products, FP32 per receiver, Float64 over
                      receivers), within about 1e-6 of the Float64 sums; the
                      map is kept again as packed operand tiles of twice
                      its size (TF32 parts and remainders)               */
} adf_gfmap;
#define ADF_GF_CONTRACT_FP64 0
#define ADF_GF_CONTRACT_TF32X3 1

/* run_fdtd! with a gf_map (src/simulation.jl:542-557, forward.jl:123-128):
 * adf_run_fdtd plus, after v2vn! of each step it < nt, extrapolate!
 * (extrapolation.jl:204-249) on the device: rows it-T+1..it of the recorded
 * p / v_n (T = min(it, nt_gf)), pin = (p_rec - z0 vn_rec)/2 in Float64 for
 * the two *FromPin kinds, sums over receivers and lags accumulated in
 * Float64, p_src[it+1, iSrc] and vn_src[it+1, iSrc] set before vn2v!.
 * txs->src[0] and txs->vn_src come back updated.                          */
int adf_run_fdtd_gf(adf_ctx* ctx, const adf_domain* d, float* field, adf_txgrid* txs,
                    adf_cpml* cpml, const uint8_t* mask, int64_t start_step, int64_t stop_step,
                    int flags, const adf_gfmap* gf, adf_step_cb cb, void* user);

/* Inside an adf_step_cb: copy channel c (0=P..3=Vz) of the current field,
 * (nx,ny,nz) Float32 Julia layout, to host memory.                        */
int adf_read_field(adf_ctx* ctx, int chan, float* out);

/* Device time (ms, CUDA events on the context's stream) of the step launches
 * of the most recent adf_run_fdtd / adf_gf_solve_batch call, and the number
 * of kernels that call launched.                                           */
int adf_last_timing(adf_ctx* ctx, double* device_ms, int64_t* kernel_launches);

/* Per-launch CUDA-event timing of the fused step kernel (events recorded on
 * the context stream around every step launch, inside captured graphs
 * too).  Off by default.  adf_kernel_timing returns the summed device time
 * and launch count since the last reset.                                   */
int adf_set_kernel_timing(adf_ctx* ctx, int on);
/* Host->device and device->host bytes copied by the most recent
 * adf_run_fdtd / adf_gf_solve_batch call.                                  */
int adf_last_io_bytes(adf_ctx* ctx, int64_t* h2d, int64_t* d2h);
int adf_kernel_timing(adf_ctx* ctx, double* step_kernel_ms, int64_t* step_launches, int reset);

/* Page-locks (pins) a caller's host buffer so that later calls copy to and
 * from it by DMA, without staging; adf_host_unpin releases it before the
 * caller frees the memory.  No reference counterpart: a host-memory helper
 * for callers that reuse their trace buffers across calls.                 */
int adf_host_pin(void* ptr, size_t bytes);
int adf_host_unpin(void* ptr);

/* ---- Impulsive Green's-function solves (impulsive_gfs, src/greens.jl:48-234) ----
 * One request = one FDTD solve: a point source at `src_point` with
 * direction {q,fx,fy,fz} driven by `src_tf` (nt Float64), recording p and
 * v_n at n_rec receivers (direction {0, normal}) for nt steps, optionally
 * inside a scatterer mask.  Outputs p_rec and vn_rec (nt, n_rec) Float32,
 * Julia layout, the receiver columns of p_rec/vn_rec after run_fdtd!
 * (greens.jl:169-173; the source's self-record column is dropped).       */
typedef struct {
  adf_domain dom;
  int64_t npml;
  double pml_rcoef, pml_fc;
  int shape;
  double shape_params[6];
  double src_point[3];
  double src_dir[4];
  const double* src_tf;      /* (nt)                                      */
  int64_t n_rec;
  const double* rec_points;  /* (3, n_rec)                                */
  const double* rec_normals; /* (3, n_rec)                                */
  int flags;                 /* ADF_ARITH_*                               */
  float* out_p;              /* (nt, n_rec)                               */
  float* out_vn;             /* (nt, n_rec)                               */
} adf_gf_request;

/* Runs n requests.  batched=1: all requests that fit the HBM budget advance
 * together, one step-kernel launch per time step over all of their (solve,
 * tile, z chunk) work items, the step loop captured in CUDA graphs.  batched=0: the plain path,
 * one solve at a time, one launch per step.                               */
int adf_gf_solve_batch(adf_ctx* ctx, int64_t n, adf_gf_request* reqs, int batched);

/* Autotuner of the fused step kernel's tile shape for one grid size; no
 * counterpart in the reference.  Times n_solves synthetic GF solves of
 * `steps` steps (CPML npml, centred rigid sphere, point source, receiver
 * shell) for each candidate (tile rows, z-chunk depth), keeps the fastest
 * in the tune table next to the library (or $ADF_TUNE_TABLE) that later
 * solves of this size use, and returns it with its mean step-kernel time.  */
int adf_autotune(adf_ctx* ctx, int64_t nx, int64_t ny, int64_t nz, int64_t npml, int n_solves,
                 int steps, int* best_ty, int* best_nzc, double* best_ms);

/* ---- Serving loop: continuous batching of GF solves ----------------------
 * A host thread owns the device work: requests submitted while others are
 * on the GPU are admitted as slots and HBM budget free up, and all resident
 * solves advance together.  submit/poll/cancel are thread-safe.           */
typedef struct adf_server adf_server;
int adf_server_start(adf_ctx* ctx, size_t hbm_budget, int max_resident, adf_server** out);
/* The request's pointers (src_tf, points, outputs) must stay valid until the
 * request completes.  *id receives a request id.                          */
/* Admission by work, with no reference counterpart: a queued request joins
 * only while the resident solves' step-kernel work items (CTAs per step
 * launch) stay within max_items, so that each step launch keeps the GPU
 * full without spreading it over more solves than that needs; one solve is
 * always admitted.  0 (the default) = HBM budget and slot count only.
 * adf_step_resident_ctas gives the CTAs the GPU runs at once (one wave).  */
int adf_server_set_work_cap(adf_server* s, int64_t max_items);
int adf_step_resident_ctas(adf_ctx* ctx, int64_t* n);
int adf_server_submit(adf_server* s, const adf_gf_request* req, int64_t* id);
/* status: 0 pending/running, 1 done (outputs written), <0 error code.
 * latency_ms (optional): submit-to-completion wall time once done.        */
int adf_server_poll(adf_server* s, int64_t id, int* status, double* latency_ms);
int adf_server_cancel(adf_server* s, int64_t id);
/* Blocks until every submitted request has completed. */
int adf_server_drain(adf_server* s);
int adf_server_stop(adf_server* s);

/* ---- Kirchhoff-Helmholtz extrapolation (src/kh_kernels.jl) ----------------
 * Two-way KH pressure at targets (part3_kh_extrapolation.jl:168-185,216-265):
 *   out[t,r] = aq * sum_s p_p(s,r) (*) in_q[:,s] + af * sum_s p_v(s,r) (*) in_f[:,s]
 * with the kernels of eval_one_kernel (kh_kernels.jl:106-157), evaluated on
 * the fly (Gaussian wavelet sigma, taps within +-window_sigmas*sigma of the
 * delay r/c0) instead of materialising K (nt_K, N_s, N_r).  FP32 taps and
 * FP32 compensated (two-sum) accumulation over surface points.
 * s_pts, s_nrm (ns,3), r_pts (nr,3) Float64 column-major; in_q, in_f
 * (nt, ns) Float32; out (nt, nr) Float32.                                  */
typedef struct {
  int64_t ns, nr, nt;
  double dt, sigma, c0, rho;
  double aq, af;
  double window_sigmas;      /* 0 -> default 6                            */
  const double* s_pts;
  const double* s_nrm;
  const double* r_pts;
  const double* r_nrm;       /* (nr,3) target normals, adf_kh_velocity only */
} adf_kh_desc;
int adf_kh_pressure(adf_ctx* ctx, const adf_kh_desc* desc, const float* in_q,
                    const float* in_f, float* out);
/* Two-way KH normal velocity at targets (part3_kh_extrapolation.jl:151,
 * 180-265): out[t,r] = aq * sum_s v_p(s,r) (*) in_q[:,s]
 *                    + af * sum_s v_v(s,r) (*) in_f[:,s]
 * with v_p, v_v of eval_one_kernel (kh_kernels.jl:106-157).  v_v's
 * Gaussian-CDF term does not decay; beyond each pair's window it is added
 * as its limit times the running sum of in_f (the K_dc pedestal of
 * direct_kh_accumulate!, kh_kernels.jl:256-296), so the result is the
 * convolution with the untruncated kernel.  Needs desc->r_nrm and rho.    */
int adf_kh_velocity(adf_ctx* ctx, const adf_kh_desc* desc, const float* in_q,
                    const float* in_f, float* out);

/* Hologram synthesis and its extrapolation in one call: build_hologram's
 * run_fdtd! (src/hologram.jl:141, 248) with a distributed C_f / C_q
 * injection already written into txs's sources
 * (diagnostics/_check_inject_kh/fdtd_runners.jl:39-45), followed by the
 * two-way KH pressure of part3_kh_extrapolation.jl:168-185 on the recorded
 * shell: in_q = the v_n traces and in_f = the p traces of the transceivers
 * kh_cols[0..kh->ns-1] (1-based), rows 1..kh->nt.  Everything of
 * adf_run_fdtd is returned as there; the recorded traces go from HBM into
 * the KH kernel without a host round trip.  kh->dt must equal d->dt and
 * kh->nt <= stop_step; kh_out is (kh->nt, kh->nr) Float32.                 */
int adf_run_fdtd_kh(adf_ctx* ctx, const adf_domain* d, float* field, adf_txgrid* txs,
                    adf_cpml* cpml, const uint8_t* mask, int64_t start_step, int64_t stop_step,
                    int flags, const adf_kh_desc* kh, const int64_t* kh_cols, float* kh_out);
/* Kernel time (ms) of the last KH extrapolation on ctx; a measurement
 * helper with no reference counterpart.                                   */
int adf_last_kh_ms(adf_ctx* ctx, double* ms);

/* Measured FP32 FMA throughput of the device (TFLOP/s, 2 FLOP per FMA): the
 * roofline denominator of adf_kh_pressure.  Measurement helper with no
 * reference counterpart; ms (optional) receives the probe's duration.      */
int adf_fp32_fma_peak(adf_ctx* ctx, double* tflops, double* ms);
/* The same probe in Float64: the roofline denominator of the in-loop GF
 * extrapolation's contraction, which accumulates in Float64.             */
int adf_fp64_fma_peak(adf_ctx* ctx, double* tflops, double* ms);

/* Test hook with no reference counterpart: arms the next adf_kh_pressure /
 * adf_kh_velocity call on ctx (one shot) so that its bounded waits give up
 * after poll_limit polls and the bulk copies of staged chunk skip_chunk
 * (0-based; -1 none) are never issued.  Nothing is then in flight when that
 * chunk's wait runs out: the call returns ADF_E_TIMEOUT with the context
 * still usable, which is how a test shows that a device wait ends in an
 * error code instead of a hang.                                           */
int adf_kh_test_fault(adf_ctx* ctx, int skip_chunk, uint32_t poll_limit);

/* impulsive_gfs post-processing of recorded GF traces (src/greens.jl:174-190,
 * src/resample.jl:32-76, src/greens_io.jl:195-205), on the GPU, per column
 * of in (nt_in, ncol) Float32: values below 1e-4 of the column maximum set
 * to zero (denoise != 0); cubic B-spline resampling (Interpolations.jl
 * BSpline(Cubic(Line(OnGrid()))), Flat() extrapolation) from the axis
 * t_in0 + k dt_in to t_out0 + k dt_out, times dt_out/dt_in; rounded to
 * Float32 and divided by Float32(unit) (gf_to_physical's C_p or C_v, 1 for
 * raw units).  out (nt_out, ncol).  For impulsive_gfs: t_in0 = -timeshift,
 * dt_in = dom.dt, t_out0 = 0, dt_out = tmax/(nt_gf-1).                    */
int adf_gf_postprocess(adf_ctx* ctx, int64_t ncol, int64_t nt_in, double t_in0, double dt_in,
                       int64_t nt_out, double t_out0, double dt_out, const float* in,
                       float* out, double unit, int denoise);

/* C_for_N (diagnostics/_check_inject_kh/injection_coefficients.jl:467-472)
 * with fib_sphere_area (src/io.jl:131), in FP64 on the GPU:
 * out[0]=C_f, out[1]=C_q, out[2]=dS.                                       */
int adf_injection_coefficients(adf_ctx* ctx, const adf_domain* d, double radius,
                               int64_t n_points, double* out);

#ifdef __cplusplus
}
#endif
#endif
