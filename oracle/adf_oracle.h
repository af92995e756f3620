/*
 * adf_oracle.h -- CPU oracle for the AcousticDisguising FDTD + KH hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain C++17 (std::thread)
 * restatement of the reference's CPU ("Threads" backend) arithmetic.  Only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg / reference
 * arm may load it, and only as the checker or as the timed CPU baseline.  The
 * product path (acoustic_disguising_b200) never links or calls it.
 *
 * Parity status: the reference is Julia and no Julia runtime exists where
 * this was written, so the oracle could not be run side by side with the
 * reference.  It is pinned against (a) the reference's own known-answer
 * tests restated with their exact setups (test/test_reciprocity.jl:18-69;
 * test/test_extrapolation_writecount.jl:354-393), (b) exact rational
 * arithmetic for the range coordinates, and (c) closed-form checks (CPML
 * profile formulae, Fibonacci points, wavelet normalisation).  Beyond those
 * anchors the element-level arithmetic is "parity unpinned".
 *
 * Array conventions follow the reference (Julia column-major, first index
 * fastest); indices stored in buffers are 1-based, exactly as the reference
 * packs them.  All functions return 0 on success, negative on bad input.
 */
#ifndef ADF_ORACLE_H
#define ADF_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Domain  (src/simulation.jl:25-79) */
typedef struct {
  double tmax, xmax, ymax, zmax;
  int64_t nx, ny, nz;
  double c0, r0, cf;
  double dx, dy, dz;
  double fact_m0, fact_m1;
  double dt;
  int64_t nt;
  double z0;
} or_domain;

/* TransceiverGrid / ChannelBuffers (src/simulation.jl:354-431), Julia layout.
 * channel order 0=p, 1=vx, 2=vy, 3=vz.
 *   idx[c]: (3, ntx)  Float32, 1-based lower-corner indices
 *   w[c]  : (2,2,2, ntx) Float32
 *   src[c], rec[c]: (nt, ntx) Float32
 *   dir   : (4, ntx) Float32   [q, nx, ny, nz]
 *   vn_src, vn_rec: (nt, ntx) Float32                                       */
typedef struct {
  int64_t ntx, nt;
  float* idx[4];
  float* w[4];
  float* src[4];
  float* rec[4];
  float* dir;
  float* vn_src;
  float* vn_rec;
} or_txgrid;

/* Cpml (src/simulation.jl:200-227): memory variables in Julia layout.
 *   mv[0]: (npml, ny, nz, 2)   mv[1]: (nx, npml, nz, 2)   mv[2]: (nx, ny, npml, 2)
 *   mp[d]: same with npml+1 along axis d.
 *   coef: a_l[n] a_r[n] a_hl[n+1] a_hr[n+1] b_l[n] b_r[n] b_hl[n+1] b_hr[n+1]
 *         as Float32 (the reference stores them in Data.Array = Float32).   */
typedef struct {
  int64_t npml;
  float* mv[3];
  float* mp[3];
  const float* coef;
} or_cpml;

/* The same buffers in Float64, for the FP64 run (or_run_fdtd64).  idx stays
 * Float32: its values are small integers, exact in either type.          */
typedef struct {
  int64_t ntx, nt;
  float* idx[4];
  double* w[4];
  double* src[4];
  double* rec[4];
  double* dir;
  double* vn_src;
  double* vn_rec;
} or_txgrid64;
typedef struct {
  int64_t npml;
  double* mv[3];
  double* mp[3];
  const double* coef;
} or_cpml64;

enum { OR_MODE_PROMOTE = 0, OR_MODE_FP32 = 1 };
enum { OR_SHAPE_NONE = 0, OR_SHAPE_SPHERE = 1, OR_SHAPE_CUBE = 2, OR_SHAPE_CROSS = 3,
       OR_SHAPE_ELLIPSOID = 4 };

int or_domain_make(double tmax, double xmax, double ymax, double zmax, int64_t nx,
                   int64_t ny, int64_t nz, double c0, double r0, double cf, or_domain* out);
/* Elements of Julia's range(start; stop=stop, length=len) minus `shift`
 * (shift applied to the range's twice-precision reference, as the broadcast
 * `r .- shift` on a StepRangeLen does).  shift=0 gives the plain range. */
int or_range(double start, double stop, int64_t len, double shift, double* out);
/* coords(d)[axis][chan]   axis 0..2, chan 0=p 1=vx 2=vy 3=vz */
int or_coords(const or_domain* d, int axis, int chan, double* out);
int or_time_axis(const or_domain* d, double* out);
/* compute_CPML_coefficients! + calc_Kab_CPML (src/kernels/cpmlcoeffs.jl:36-126)
 * out: 8 arrays concatenated in Float64 (a_l,a_r,a_hl,a_hr,b_l,b_r,b_hl,b_hr) */
int or_cpml_coefficients(int64_t npml, double vel_max, double dt, double rcoef,
                         double thickness, double f0, double* out);
/* build_update_mask (src/geometry.jl:250-280); out (nx,ny,nz,4) uint8.
 * returns 1 (and writes nothing) for SHAPE_NONE, matching `nothing`.
 * params: sphere {r}; cube {l}; cross {l}; ellipsoid {cx,cy,cz,ax,ay,az}. */
int or_build_update_mask(const or_domain* d, int shape, const double* params, uint8_t* out);
int or_build_scatterer(const or_domain* d, int shape, const double* params, uint8_t* out);
int or_fibonacci_sphere(int64_t n, double radius, double* points, double* normals);
int or_impulsive_wavelet(const or_domain* d, double f3db, double* tf, double* timeshift);
int or_ricker_wavelet(const or_domain* d, double fc, int injection, double* tf);
/* trilinearInterpolation: idx (3,4) 1-based Int, w (2,2,2,4) Float64 */
int or_trilinear(const or_domain* d, const double* point, int64_t* idx, double* w);
/* transceiversToGrid: points (3,ntx), dirs (4,ntx), tf (nt,ntx) Float64.
 * Fills the caller-allocated arrays of *out (ntx and nt must be set).   */
int or_pack_transceivers(const or_domain* d, const double* points, const double* dirs,
                         const double* tf, or_txgrid* out);
/* run_fdtd!(dom, field, txs, cpml, va; start_step) for it in start..stop
 * (1-based, inclusive).  field (nx,ny,nz,4) Float32; mask (nx,ny,nz,4)
 * uint8 or NULL.  mode: OR_MODE_PROMOTE (Julia promotion of the Float64
 * Domain scalars) or OR_MODE_FP32.  nthreads<=0: OpenMP default.          */
int or_run_fdtd(const or_domain* d, float* field, or_txgrid* txs, or_cpml* cpml,
                const uint8_t* mask, int64_t start_step, int64_t stop_step, int mode,
                int nthreads);
/* run_fdtd! in Float64 throughout (field, memory, coefficients, weights,
 * traces): the reference's algorithm without any Float32 rounding, which
 * the error statements of the Float32 paths are measured against.        */
int or_run_fdtd64(const or_domain* d, double* field, or_txgrid64* txs, or_cpml64* cpml,
                  const uint8_t* mask, int64_t start_step, int64_t stop_step, int nthreads);

/* In-loop GF extrapolation of run_fdtd!(...; gf_map) (src/kernels/
 * extrapolation.jl:36-87, 91-249; forward.jl:123-128), after v2vn! of each
 * step it < nt, T = min(it, nt_gf), rows it-T+1..it of the traces:
 *  kind 0 PVFromPin  t = {p_pin, v_pin} (nt_gf, nsrc, nrec), iRec -> nrec,
 *    pin = (p_rec - z0*vn_rec)/2 (Float64); per s: psum/vsum = Float64 sums
 *    of p_pin/v_pin[T-tt+1, s, r] * pin; p_src[it+1, iSrc[s]] = vsum,
 *    vn_src[it+1, iSrc[s]] = psum (extrapolate_pv_from_pin!, :139-170).
 *  kind 1 PFromPin   t = {pos, neg} (nt_gf, nrec, nsrc); pos[s], neg[s] =
 *    Float64 sums of g[T-tt+1, r, s] * pin rounded to Float32;
 *    p_src = pos - neg, vn_src = (pos + neg)/z0 (extrapolate_p_from_pin,
 *    :172-193 and :237-249).
 *  kind 2 PVFromPV   t = {pp, pv, vp, vv} (nt_gf, nm, nrec), iRec -> nm
 *    columns of p_rec / vn_rec, per r: psum += pv*p + pp*vn, vsum += vv*p +
 *    vp*vn (Float32 products and pair sum, accumulated sequentially in
 *    Float32 as the reference does, :91-137); p_src[it+1, iSrc[r]] = vsum,
 *    vn_src[it+1, iSrc[r]] = psum (:204-218).
 * discard = 1 reproduces the shipped code, whose slice copies drop the
 * writes.  i_src, i_rec are 1-based transceiver indices.                  */
typedef struct {
  int kind;
  int64_t nt_gf, n1, n2;  /* tensor dims (nt_gf, n1, n2) */
  const float* t[4];
  const int64_t* i_src;
  int64_t n_src;
  const int64_t* i_rec;
  int64_t n_rec;
  double z0;
  int discard;
} or_gfmap;
int or_run_fdtd_gf(const or_domain* d, float* field, or_txgrid* txs, or_cpml* cpml,
                   const uint8_t* mask, int64_t start_step, int64_t stop_step, int mode,
                   const or_gfmap* gf, int nthreads);

/* ---- Kirchhoff-Helmholtz (src/kh_kernels.jl) ----
 * which: 0=p_p 1=p_v 2=v_p 3=v_v.  Points (n,3) column-major Float64.   */
int or_kh_eval_kernel(int which, int64_t n_outer, const double* outer_pts,
                      const double* outer_nrm, int64_t n_inner, const double* inner_pts,
                      const double* inner_nrm, int64_t ntk, const double* t_grid,
                      double sigma, double c0, double rho, float* K /*(ntk,n_outer,n_inner)*/,
                      int nthreads);
/* direct_kh_accumulate! (kh_kernels.jl:256-296): out (nt,n_inner) Float64 */
int or_kh_accumulate(double* out, int64_t nt, const float* K, int64_t ntk, int64_t n_outer,
                     int64_t n_inner, const float* in, double alpha, const float* K_dc,
                     const double* cumsum_in, int nthreads);
/* Two-way KH pressure at targets: out[t, r] = aq*sum_s p_p(s,r) (*) in_q[., s]
 *                                            + af*sum_s p_v(s,r) (*) in_f[., s]
 * evaluated with the kernel formulae of eval_one_kernel (kh_kernels.jl:106-157)
 * on the time grid t_k = (k-1)*dt, k=1..ntk, directly in FP64 (no Float32
 * kernel storage): the FP64 oracle for the on-the-fly GPU KH.  Targets
 * [r_begin, r_end) only; out is (nt, r_end-r_begin).  mode 1 = FP64; mode 0
 * stores taps as Float32 and multiplies in Float32 with a Float64
 * accumulator, as direct_kh_accumulate! does.                               */
int or_kh_pressure(int64_t ns, const double* s_pts, const double* s_nrm, int64_t nr,
                   const double* r_pts, int64_t nt, int64_t ntk, double dt, double sigma,
                   double c0, const float* in_q, const float* in_f, double aq, double af,
                   int mode, int64_t r_begin, int64_t r_end, double* out, int nthreads);

/* Two-way KH normal velocity at targets (part3_kh_extrapolation.jl:151,
 * 180-265): out[t, r] = aq*sum_s v_p(s,r) (*) in_q[., s]
 *                    + af*sum_s v_v(s,r) (*) in_f[., s]
 * with v_p, v_v of eval_one_kernel (kh_kernels.jl:106-157) in FP64: taps
 * within +-12 sigma of the delay, plus, for the non-decaying F-term of v_v
 * (its tau -> inf value (cos_r cos_s / rho) 2/(4 pi d^3)), that value times
 * the running sum of in_f beyond the window, which makes the sum equal to
 * the convolution with the full, untruncated kernel.  r_nrm (nr,3) are the
 * target normals.  Targets [r_begin, r_end); out (nt, r_end-r_begin).     */
int or_kh_velocity(int64_t ns, const double* s_pts, const double* s_nrm, int64_t nr,
                   const double* r_pts, const double* r_nrm, int64_t nt, double dt,
                   double sigma, double c0, double rho, const float* in_q, const float* in_f,
                   double aq, double af, int64_t r_begin, int64_t r_end, double* out,
                   int nthreads);

/* impulsive_gfs post-processing of one source's traces (src/greens.jl:
 * 174-190, src/resample.jl:32-76, src/greens_io.jl:195-205), per column of
 * in (nt_in, ncol) Float32:
 *   denoise  (denoise != 0): values with |a| < 1e-4 * (column maximum) -> 0
 *   resample : cubic B-spline, Line(OnGrid()) ends (zero second derivative),
 *              Flat() extrapolation, from t_in0 + k dt_in to t_out0 + k
 *              dt_out, times dt_out / dt_in, rounded to Float32
 *   physical : divided by Float32(unit) (gf_to_physical's C_p or C_v; 1
 *              leaves the raw units)
 * into out (nt_out, ncol).  FP64 throughout before the final roundings.
 * The B-spline prefilter follows Interpolations.jl 0.16.2's published
 * algorithm, which is not part of the reference tree: parity unpinned.   */
int or_gf_postprocess(int64_t ncol, int64_t nt_in, double t_in0, double dt_in, int64_t nt_out,
                      double t_out0, double dt_out, const float* in, float* out, double unit,
                      int denoise);

/* extrapolate_pv_from_pin! (src/kernels/extrapolation.jl:139-170), 1-based it.
 * pin (nt, nrec), p_src/v_src (nt, nsrc), pp/vp (nt_gf, nsrc, nrec).      */
int or_extrapolate_pv_from_pin(const float* pin, int64_t nt, int64_t nrec, float* p_src,
                               float* v_src, int64_t nsrc, const float* pp, const float* vp,
                               int64_t nt_gf, int64_t it);

int or_version(void);

#ifdef __cplusplus
}
#endif
#endif
