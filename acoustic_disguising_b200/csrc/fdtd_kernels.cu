// fdtd_kernels.cu -- the fused staggered-grid FDTD step for sm_100a.
//
// One launch advances every active solve of a batch by one time step
// (forward_onestep!, src/kernels/forward.jl:13-139).  The step reads field
// buffer `rb` and writes buffer `wb`, so the pressure update, the q-channel
// injection/recording, the three velocity updates, the f-channel
// injection/recording and the rigid mirrors all happen in a single pass over
// HBM: 16 B read + 16 B written per cell, plus psi traffic on CPML slabs and
// half a byte of mask per cell.
//
// Work decomposition: a persistent CTA walks (solve, y tile, z chunk) items.
// A tile spans the full x extent (nxp <= 512), `ty` rows and a run of
// planes.  A producer warp streams planes into a ring of shared-memory slots
// with TMA (cp.async.bulk.tensor, no multicast): each slot holds P, Vx, Vy
// for rows j0-1 .. j0+ty and plane k, Vz for planes k and k+1, and the mask
// nibbles.  Eight consumer warps compute, per plane:
//   P phase : P_new on rows j0-1 .. j0+ty-1 (row j0-1 is the halo that the
//             velocity update of row j0 needs; it is recomputed, not
//             exchanged), into a triple-buffered shared plane;
//   Q phase : q-channel inject/record entries of this (tile, plane), if any;
//   V phase : Vx/Vy/Vz_new from P_new (x-1 and y-1 from shared memory, z-1
//             from the previous plane still in shared memory);
//   F phase : f-channel entries, if any;  then 128-bit stores of all four.
// A z chunk starting at z0 > 0 first recomputes P_new on plane z0-1
// (prologue plane: no stores, no records) for Vz at z0.
//
// Arithmetic: Arith<double> reproduces Julia's promotion (Float32 storage,
// Float64 Domain scalars, src/kernels/updates.jl) with explicit round-to-
// nearest intrinsics so that nothing is contracted; the one deliberate
// difference is x*(1/dx) in place of x/dx.  Arith<float> is the all-Float32
// variant.  Injection/recording (derivatives.jl:30-60) is pure Float32 with
// separate multiply and add, as the reference computes it.
#include "adf_internal.h"
#include "ptx_util.h"

namespace adf {

#ifndef ADF_NCT
#define ADF_NCT 256
#endif
constexpr int NCT = ADF_NCT;      // consumer threads
constexpr int NCW = NCT / 32;     // consumer warps
constexpr int NTHREADS = NCT + 32;
constexpr int kMaxStages = 8;
constexpr int kPnBufs = 3;
constexpr int kMaxCoef = 8 * 63 + 4;  // CPML coefficients for npml <= 63

int consumer_threads() { return NCT; }

// ---------------------------------------------------------------------------
// TMA tensor loads (no multicast)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* map, uint32_t mbar,
                                            int c0, int c1, int c2, int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(dst),
      "l"((uint64_t)map), "r"(mbar), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
      : "memory");
}
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, uint32_t mbar,
                                            int c0, int c1, int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(dst),
      "l"((uint64_t)map), "r"(mbar), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, uint32_t mbar,
                                            int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
      "l"((uint64_t)map), "r"(mbar), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
__device__ __forceinline__ void tmap_acquire(const CUtensorMap* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"((uint64_t)map)
               : "memory");
}
__device__ __forceinline__ void consumer_bar() {
  asm volatile("bar.sync 1, %0;" ::"n"(NCT) : "memory");
}

// ---------------------------------------------------------------------------
// Arithmetic policies
// ---------------------------------------------------------------------------
template <typename R>
struct Arith;
template <>
struct Arith<double> {
  static __device__ __forceinline__ double cv(float x) { return (double)x; }
  static __device__ __forceinline__ float rn(double x) { return __double2float_rn(x); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double fq(const SolveDev& s) { return s.fq; }
  static __device__ __forceinline__ double fv(const SolveDev& s) { return s.fv; }
  static __device__ __forceinline__ double rdx(const SolveDev& s) { return s.rdx; }
  static __device__ __forceinline__ double rdy(const SolveDev& s) { return s.rdy; }
  static __device__ __forceinline__ double rdz(const SolveDev& s) { return s.rdz; }
};
template <>
struct Arith<float> {
  static __device__ __forceinline__ float cv(float x) { return x; }
  static __device__ __forceinline__ float rn(float x) { return x; }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float fq(const SolveDev& s) { return s.fqf; }
  static __device__ __forceinline__ float fv(const SolveDev& s) { return s.fvf; }
  static __device__ __forceinline__ float rdx(const SolveDev& s) { return s.rdxf; }
  static __device__ __forceinline__ float rdy(const SolveDev& s) { return s.rdyf; }
  static __device__ __forceinline__ float rdz(const SolveDev& s) { return s.rdzf; }
};

// CPML memory update m = b*m + a*d; d += m  (updates.jl:46-61): b*m is a
// Float32 product, a*d is promoted, the sum is rounded to Float32 on store
// and re-added.  `m` is updated in place; the caller stores it.
template <typename R>
__device__ __forceinline__ void cpml_apply(R& dv, float& m, float a, float b) {
  using A = Arith<R>;
  const float bm = __fmul_rn(b, m);
  m = A::rn(A::add(A::cv(bm), A::mul(A::cv(a), dv)));
  dv = A::add(dv, A::cv(m));
}

struct PlaneCtx {
  const float* sP;
  const float* sVx;
  const float* sVy;
  const float* sVz;   // plane k rows, plane k+1 at + R*nxp
  const uint32_t* sM;
  const float* sXp;   // x-slab psi, p side: [side][R][npp]
  const float* sXv;   // x-slab psi, v side: [side][R][nvp]
  const float* yP;    // y-slab psi rows of side ysP (p) / ysV (v): [R][nxp]
  const float* yV;
  const float* zP;    // z-slab psi of this plane (p / v side): [R][nxp]
  const float* zV;
  int ysP, ysV;
  const float* co;    // CPML coefficients staged in shared memory
  float* pn_cur;
  const float* pn_prev;
  int j0, R, pl, rb, wb;
  bool has_mask;
};

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ float f4get(const float4& v, int e) {
  return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w;
}
__device__ __forceinline__ void f4set(float4& v, int e, float x) {
  if (e == 0) v.x = x; else if (e == 1) v.y = x; else if (e == 2) v.z = x; else v.w = x;
}

// Per-item scalars held in registers for the fast paths (the descriptor
// lives in shared memory; re-reading it per quad costs a load per field).
template <typename R>
struct Regs {
  int nxp, R2;  // row pitch, rows per ring region (ty+2)
  R fq, fv, rdx, rdy, rdz;
};

// ---------------------------------------------------------------------------
// Boundary path, pressure: rigid planes, the i = nx plane, CPML slabs.  Row-
// and plane-wide conditions are uniform branches; per-cell conditions (the x
// slab, the last x cells) are selects, so the four cells' dependency chains
// interleave.  CPML memory comes from the ring slot (x and staged y/z slabs).
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ float p_cell_slow(float P, float dx_in, float dy_in, float dz_in,
                                             const Regs<R>& g, bool upd, bool open, bool xs,
                                             float& mx, float ax, float bx, bool ys, float& my,
                                             float ay, float by, bool zs, float& mz, float az,
                                             float bz) {
  using A = Arith<R>;
  R dvx = A::mul(A::cv(dx_in), g.rdx);
  R dvy = A::mul(A::cv(dy_in), g.rdy);
  R dvz = A::mul(A::cv(dz_in), g.rdz);
  {  // x slab: computed for every cell, kept where the cell is in the slab
    R d2 = dvx;
    float m2 = mx;
    cpml_apply<R>(d2, m2, ax, bx);
    if (xs) { dvx = d2; mx = m2; }
  }
  if (ys) cpml_apply<R>(dvy, my, ay, by);
  if (zs) cpml_apply<R>(dvz, mz, az, bz);
  const float n = A::rn(A::sub(A::cv(P), A::mul(g.fq, A::add(A::add(dvx, dvy), dvz))));
  return (upd && open) ? n : P;
}

template <typename R>
__device__ __forceinline__ void p_quad(const SolveDev& S, const Regs<R>& g, const PlaneCtx& c,
                                       int r, int q, bool owned) {
  const int nxp = g.nxp, nx = S.nx, ny = S.ny, nz = S.nz, npml = S.npml, npp = S.npp;
  const int x0 = 4 * q;
  const int j = c.j0 - 1 + r;
  const int pl = c.pl;
  const float* base = c.sP + r * nxp + x0;
  const float4 P4 = ld4(base);
  const float4 X4 = ld4(c.sVx + r * nxp + x0);
  const float X5 = (x0 + 4 < nxp) ? c.sVx[r * nxp + x0 + 4] : 0.f;
  const float4 Y0 = ld4(c.sVy + r * nxp + x0);
  const float4 Y1 = ld4(c.sVy + (r + 1) * nxp + x0);
  const float4 Z0 = ld4(c.sVz + r * nxp + x0);
  const float4 Z1 = ld4(c.sVz + (c.R + r) * nxp + x0);
  uint32_t nib = 0xFFFFu;
  const bool rigid_y = (j == ny - 1), rigid_z = (pl == nz - 1);
  // rigid planes use update_p! (updates.jl:122-136): -2V/d at the wall, no
  // CPML, no mask; the (ny, nz) corner is not updated at all
  const bool plain_rigid = rigid_y || rigid_z;
  if (c.has_mask && !plain_rigid) nib = (c.sM[r * S.mw + (q >> 1)] >> ((q & 1) * 16)) & 0xFFFFu;
  const bool pc = (S.flags & SF_PCPML) != 0 && !plain_rigid;
  const float* co = c.co;
  int ysd = -1, yl = 0, zsd = -1, zl = 0;
  if (pc) {
    if (j < npml) { ysd = 0; yl = j; }
    else if (j >= ny - npml) { ysd = 1; yl = j - (ny - npml); }
    if (pl < npml) { zsd = 0; zl = pl; }
    else if (pl >= nz - npml) { zsd = 1; zl = pl - (nz - npml); }
  }
  long long oy = 0, oz = 0;
  float4 my = make_float4(0.f, 0.f, 0.f, 0.f), mz = my;
  float ay = 0.f, by = 0.f, az = 0.f, bz = 0.f;
  if (ysd >= 0) {  // staged with the plane unless the tile straddles both y slabs
    oy = (long long)ysd * S.psi_p_side[1] + ((long long)pl * npml + yl) * nxp + x0;
    my = ysd == c.ysP ? ld4(c.yP + r * nxp + x0) : ldg4(S.psi_p[1] + c.rb * S.psi_p_buf[1] + oy);
    ay = co[ysd * npml + yl];
    by = co[4 * npml + 2 + ysd * npml + yl];
  }
  if (zsd >= 0) {
    oz = (long long)zsd * S.psi_p_side[2] + ((long long)zl * ny + j) * nxp + x0;
    mz = (S.flags & SF_YZG) ? ldg4(S.psi_p[2] + c.rb * S.psi_p_buf[2] + oz)
                            : ld4(c.zP + r * nxp + x0);
    az = co[zsd * npml + zl];
    bz = co[4 * npml + 2 + zsd * npml + zl];
  }
  // x slab: side and depth of each cell, memory from the slot
  float mx[4], ax[4], bx[4];
  bool xs[4];
  int xside[4], xl[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int x = x0 + e;
    int side = -1, l = 0;
    if (pc) {
      side = x < npml ? 0 : (x >= nx - npml ? 1 : -1);
      l = side == 0 ? x : x - (nx - npml);
    }
    xs[e] = side >= 0;
    const int sd = xs[e] ? side : 0, ll = xs[e] ? l : 0;
    xside[e] = sd;
    xl[e] = ll;
    mx[e] = c.sXp[(sd * c.R + r) * npp + ll];
    ax[e] = xs[e] ? co[sd * npml + ll] : 0.f;
    bx[e] = xs[e] ? co[4 * npml + 2 + sd * npml + ll] : 0.f;
  }
  const float dyv[4] = {rigid_y ? __fmul_rn(-2.0f, Y0.x) : __fsub_rn(Y1.x, Y0.x),
                        rigid_y ? __fmul_rn(-2.0f, Y0.y) : __fsub_rn(Y1.y, Y0.y),
                        rigid_y ? __fmul_rn(-2.0f, Y0.z) : __fsub_rn(Y1.z, Y0.z),
                        rigid_y ? __fmul_rn(-2.0f, Y0.w) : __fsub_rn(Y1.w, Y0.w)};
  const float dzv[4] = {rigid_z ? __fmul_rn(-2.0f, Z0.x) : __fsub_rn(Z1.x, Z0.x),
                        rigid_z ? __fmul_rn(-2.0f, Z0.y) : __fsub_rn(Z1.y, Z0.y),
                        rigid_z ? __fmul_rn(-2.0f, Z0.z) : __fsub_rn(Z1.z, Z0.z),
                        rigid_z ? __fmul_rn(-2.0f, Z0.w) : __fsub_rn(Z1.w, Z0.w)};
  const float dxv[4] = {__fsub_rn(X4.y, X4.x), __fsub_rn(X4.z, X4.y), __fsub_rn(X4.w, X4.z),
                        __fsub_rn(X5, X4.w)};
  const bool corner = rigid_y && rigid_z;
  const float Pv[4] = {P4.x, P4.y, P4.z, P4.w};
  float myv[4] = {my.x, my.y, my.z, my.w}, mzv[4] = {mz.x, mz.y, mz.z, mz.w};
  float o[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const bool upd = (x0 + e <= nx - 2) && !corner;
    float myc = myv[e], mzc = mzv[e], mxc = mx[e];
    o[e] = p_cell_slow<R>(Pv[e], dxv[e], dyv[e], dzv[e], g, upd, (nib >> (4 * e)) & 1u,
                          xs[e] && upd, mxc, ax[e], bx[e], ysd >= 0, myc, ay, by, zsd >= 0, mzc,
                          az, bz);
    if (upd) { myv[e] = myc; mzv[e] = mzc; mx[e] = mxc; }
  }
  st4(c.pn_cur + r * nxp + x0, make_float4(o[0], o[1], o[2], o[3]));
  if (owned) {  // cells of the quad that were not updated keep their loaded value
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (xs[e] && (x0 + e <= nx - 2) && !corner)
        S.psi_p[0][c.wb * S.psi_p_buf[0] + xside[e] * S.psi_p_side[0] +
                   ((long long)pl * ny + j) * npp + xl[e]] = mx[e];
    if (ysd >= 0)
      st4(S.psi_p[1] + c.wb * S.psi_p_buf[1] + oy, make_float4(myv[0], myv[1], myv[2], myv[3]));
    if (zsd >= 0)
      st4(S.psi_p[2] + c.wb * S.psi_p_buf[2] + oz, make_float4(mzv[0], mzv[1], mzv[2], mzv[3]));
  }
}

// Boundary path, velocities: grid edges (Vx at i=1, Vy at j=1, Vz at k=1 are
// not updated) and CPML slabs with the half-grid coefficients (npml+1).
template <typename R>
__device__ __forceinline__ float v_cell_slow(float V, float dp_in, R fv, R rd, bool upd,
                                             bool open, bool sl, float& m, float a, float b) {
  using A = Arith<R>;
  R dp = A::mul(A::cv(dp_in), rd);
  R d2 = dp;
  float m2 = m;
  cpml_apply<R>(d2, m2, a, b);
  if (sl) { dp = d2; m = m2; }
  const float n = A::rn(A::sub(A::cv(V), A::mul(fv, dp)));
  return (upd && open) ? n : V;
}

template <typename R>
__device__ __forceinline__ void v_quad(const SolveDev& S, const Regs<R>& g, const PlaneCtx& c,
                                       int r, int q, float4& vxo, float4& vyo, float4& vzo) {
  const int nxp = g.nxp, nx = S.nx, ny = S.ny, nz = S.nz, npml = S.npml, nvp = S.nvp;
  const int nm = npml + 1;
  const int x0 = 4 * q;
  const int j = c.j0 - 1 + r;
  const int pl = c.pl;
  const float4 Pc = ld4(c.pn_cur + r * nxp + x0);
  const float Pxm = x0 > 0 ? c.pn_cur[r * nxp + x0 - 1] : 0.f;
  const float4 Pym = ld4(c.pn_cur + (r - 1) * nxp + x0);
  const float4 Pzm = ld4(c.pn_prev + r * nxp + x0);
  const float4 VX = ld4(c.sVx + r * nxp + x0);
  const float4 VY = ld4(c.sVy + r * nxp + x0);
  const float4 VZ = ld4(c.sVz + r * nxp + x0);
  uint32_t nib = 0xFFFFu;
  if (c.has_mask) nib = (c.sM[r * S.mw + (q >> 1)] >> ((q & 1) * 16)) & 0xFFFFu;
  const bool vc = (S.flags & SF_VCPML) != 0;
  const float* co = c.co;
  int ysd = -1, yl = 0, zsd = -1, zl = 0;
  if (vc && j >= 1) {
    if (j <= npml) { ysd = 0; yl = j; }
    else if (j >= ny - npml - 1) { ysd = 1; yl = j - (ny - npml - 1); }
  }
  if (vc && pl >= 1) {
    if (pl <= npml) { zsd = 0; zl = pl; }
    else if (pl >= nz - npml - 1) { zsd = 1; zl = pl - (nz - npml - 1); }
  }
  long long oy = 0, oz = 0;
  float4 my = make_float4(0.f, 0.f, 0.f, 0.f), mz = my;
  float ay = 0.f, by = 0.f, az = 0.f, bz = 0.f;
  if (ysd >= 0) {
    oy = (long long)ysd * S.psi_v_side[1] + ((long long)pl * nm + yl) * nxp + x0;
    my = ysd == c.ysV ? ld4(c.yV + r * nxp + x0) : ldg4(S.psi_v[1] + c.rb * S.psi_v_buf[1] + oy);
    ay = co[2 * npml + ysd * nm + yl];
    by = co[6 * npml + 2 + ysd * nm + yl];
  }
  if (zsd >= 0) {
    oz = (long long)zsd * S.psi_v_side[2] + ((long long)zl * ny + j) * nxp + x0;
    mz = (S.flags & SF_YZG) ? ldg4(S.psi_v[2] + c.rb * S.psi_v_buf[2] + oz)
                            : ld4(c.zV + r * nxp + x0);
    az = co[2 * npml + zsd * nm + zl];
    bz = co[6 * npml + 2 + zsd * nm + zl];
  }
  const float Pv[4] = {Pc.x, Pc.y, Pc.z, Pc.w};
  const float Pl[4] = {Pxm, Pc.x, Pc.y, Pc.z};
  const float Py[4] = {Pym.x, Pym.y, Pym.z, Pym.w};
  const float Pz[4] = {Pzm.x, Pzm.y, Pzm.z, Pzm.w};
  const float Vx[4] = {VX.x, VX.y, VX.z, VX.w};
  const float Vy[4] = {VY.x, VY.y, VY.z, VY.w};
  const float Vz[4] = {VZ.x, VZ.y, VZ.z, VZ.w};
  float myv[4] = {my.x, my.y, my.z, my.w}, mzv[4] = {mz.x, mz.y, mz.z, mz.w};
  float ox[4], oy4[4], oz4[4], mx[4];
  bool xs[4];
  int xside[4], xl[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int x = x0 + e;
    const bool in = x < nx;
    // Vx over i = 2..nx (update_vx!, updates.jl:192-218), x slab with npml+1
    int side = -1, l = 0;
    if (vc) {
      side = x <= npml ? 0 : (x >= nx - npml - 1 ? 1 : -1);
      l = side == 0 ? x : x - (nx - npml - 1);
    }
    const bool updx = in && x >= 1;
    xs[e] = side >= 0 && updx;
    const int sd = side >= 0 ? side : 0, ll = side >= 0 ? l : 0;
    xside[e] = sd;
    xl[e] = ll;
    mx[e] = c.sXv[(sd * c.R + r) * nvp + ll];
    const float axe = side >= 0 ? co[2 * npml + sd * nm + ll] : 0.f;
    const float bxe = side >= 0 ? co[6 * npml + 2 + sd * nm + ll] : 0.f;
    ox[e] = v_cell_slow<R>(Vx[e], __fsub_rn(Pv[e], Pl[e]), g.fv, g.rdx, updx,
                           (nib >> (4 * e + 1)) & 1u, xs[e], mx[e], axe, bxe);
    // Vy over j = 2..ny
    float myc = myv[e];
    oy4[e] = v_cell_slow<R>(Vy[e], __fsub_rn(Pv[e], Py[e]), g.fv, g.rdy, in && j >= 1,
                            (nib >> (4 * e + 2)) & 1u, ysd >= 0 && in, myc, ay, by);
    if (in) myv[e] = myc;
    // Vz over k = 2..nz
    float mzc = mzv[e];
    oz4[e] = v_cell_slow<R>(Vz[e], __fsub_rn(Pv[e], Pz[e]), g.fv, g.rdz, in && pl >= 1,
                            (nib >> (4 * e + 3)) & 1u, zsd >= 0 && in, mzc, az, bz);
    if (in) mzv[e] = mzc;
  }
  vxo = make_float4(ox[0], ox[1], ox[2], ox[3]);
  vyo = make_float4(oy4[0], oy4[1], oy4[2], oy4[3]);
  vzo = make_float4(oz4[0], oz4[1], oz4[2], oz4[3]);
#pragma unroll
  for (int e = 0; e < 4; ++e)
    if (xs[e])
      S.psi_v[0][c.wb * S.psi_v_buf[0] + xside[e] * S.psi_v_side[0] +
                 ((long long)pl * ny + j) * nvp + xl[e]] = mx[e];
  if (ysd >= 0)
    st4(S.psi_v[1] + c.wb * S.psi_v_buf[1] + oy, make_float4(myv[0], myv[1], myv[2], myv[3]));
  if (zsd >= 0)
    st4(S.psi_v[2] + c.wb * S.psi_v_buf[2] + oz, make_float4(mzv[0], mzv[1], mzv[2], mzv[3]));
}

// ---- one cell of a boundary quad on an ordinary tile-plane: no rigid plane
// and no y/z slab here, only the x slab and the last x cells.  Same
// arithmetic as p_quad / v_quad for that cell.
template <typename R>
__device__ __forceinline__ void p_xcell(const SolveDev& S, const Regs<R>& g, const PlaneCtx& c,
                                        int r, int x, bool owned) {
  const int nxp = g.nxp, nx = S.nx, npml = S.npml;
  const int o = r * nxp + x;
  const float P = c.sP[o];
  const float X0 = c.sVx[o];
  const float X1 = (x + 1 < nxp) ? c.sVx[o + 1] : 0.f;
  const float dy = __fsub_rn(c.sVy[o + nxp], c.sVy[o]);
  const float dz = __fsub_rn(c.sVz[o + c.R * nxp], c.sVz[o]);
  uint32_t open = 1u;
  if (c.has_mask) open = (c.sM[r * S.mw + (x >> 3)] >> (4 * (x & 7))) & 1u;
  const bool upd = x <= nx - 2;
  int side = -1, l = 0;
  if (S.flags & SF_PCPML) {
    side = x < npml ? 0 : (x >= nx - npml ? 1 : -1);
    l = side == 0 ? x : x - (nx - npml);
  }
  const bool xs = side >= 0 && upd;
  const int sd = side >= 0 ? side : 0, ll = side >= 0 ? l : 0;
  float mx = c.sXp[(sd * c.R + r) * S.npp + ll];
  const float ax = side >= 0 ? c.co[sd * npml + ll] : 0.f;
  const float bx = side >= 0 ? c.co[4 * npml + 2 + sd * npml + ll] : 0.f;
  float my = 0.f, mz = 0.f;
  c.pn_cur[o] = p_cell_slow<R>(P, __fsub_rn(X1, X0), dy, dz, g, upd, open, xs, mx, ax, bx, false,
                               my, 0.f, 0.f, false, mz, 0.f, 0.f);
  if (owned && xs) {
    const int j = c.j0 - 1 + r;
    S.psi_p[0][c.wb * S.psi_p_buf[0] + sd * S.psi_p_side[0] +
               ((long long)c.pl * S.ny + j) * S.npp + ll] = mx;
  }
}

template <typename R>
__device__ __forceinline__ void v_xcell(const SolveDev& S, const Regs<R>& g, const PlaneCtx& c,
                                        int r, int x, float& vx, float& vy, float& vz) {
  const int nxp = g.nxp, nx = S.nx, npml = S.npml, nm = npml + 1;
  const int j = c.j0 - 1 + r;
  const int o = r * nxp + x;
  const float Pc = c.pn_cur[o];
  const float Pxm = x > 0 ? c.pn_cur[o - 1] : 0.f;
  const float Pym = c.pn_cur[o - nxp];
  const float Pzm = c.pn_prev[o];
  uint32_t nib = 0xFu;
  if (c.has_mask) nib = (c.sM[r * S.mw + (x >> 3)] >> (4 * (x & 7))) & 0xFu;
  const bool in = x < nx;
  int side = -1, l = 0;
  if (S.flags & SF_VCPML) {
    side = x <= npml ? 0 : (x >= nx - npml - 1 ? 1 : -1);
    l = side == 0 ? x : x - (nx - npml - 1);
  }
  const bool updx = in && x >= 1;
  const bool xs = side >= 0 && updx;
  const int sd = side >= 0 ? side : 0, ll = side >= 0 ? l : 0;
  float mx = c.sXv[(sd * c.R + r) * S.nvp + ll];
  const float axe = side >= 0 ? c.co[2 * npml + sd * nm + ll] : 0.f;
  const float bxe = side >= 0 ? c.co[6 * npml + 2 + sd * nm + ll] : 0.f;
  vx = v_cell_slow<R>(c.sVx[o], __fsub_rn(Pc, Pxm), g.fv, g.rdx, updx, (nib >> 1) & 1u, xs, mx,
                      axe, bxe);
  float dm = 0.f;
  vy = v_cell_slow<R>(c.sVy[o], __fsub_rn(Pc, Pym), g.fv, g.rdy, in && j >= 1, (nib >> 2) & 1u,
                      false, dm, 0.f, 0.f);
  vz = v_cell_slow<R>(c.sVz[o], __fsub_rn(Pc, Pzm), g.fv, g.rdz, in && c.pl >= 1,
                      (nib >> 3) & 1u, false, dm, 0.f, 0.f);
  if (xs)
    S.psi_v[0][c.wb * S.psi_v_buf[0] + sd * S.psi_v_side[0] +
               ((long long)c.pl * S.ny + j) * S.nvp + ll] = mx;
}

// ---- fast paths: every cell of the quad is an interior cell of its update
// (no rigid plane, no CPML slab, no grid edge); branch-free 4-wide code.
template <typename R>
__device__ __forceinline__ float p_cell(float P, float dvx, float dvy, float dvz, R fq, R rdx,
                                        R rdy, R rdz, uint32_t open) {
  using A = Arith<R>;
  const R s = A::add(A::add(A::mul(A::cv(dvx), rdx), A::mul(A::cv(dvy), rdy)),
                     A::mul(A::cv(dvz), rdz));
  const float n = A::rn(A::sub(A::cv(P), A::mul(fq, s)));
  return open ? n : P;
}

template <typename R>
__device__ __forceinline__ float v_cell(float V, float dp, R fv, R rd, uint32_t open) {
  using A = Arith<R>;
  const float n = A::rn(A::sub(A::cv(V), A::mul(fv, A::mul(A::cv(dp), rd))));
  return open ? n : V;
}

template <typename R>
__device__ __forceinline__ void p_quad_fast(const Regs<R>& g, const float* __restrict__ sp,
                                            const float* __restrict__ sx,
                                            const float* __restrict__ sy,
                                            const float* __restrict__ sz,
                                            float* __restrict__ out, uint32_t nib) {
  const int nxp = g.nxp;
  const float4 P4 = ld4(sp), X4 = ld4(sx), Y0 = ld4(sy), Y1 = ld4(sy + nxp), Z0 = ld4(sz),
               Z1 = ld4(sz + g.R2 * nxp);
  const float X5 = sx[4];
  float4 o;
  o.x = p_cell<R>(P4.x, __fsub_rn(X4.y, X4.x), __fsub_rn(Y1.x, Y0.x), __fsub_rn(Z1.x, Z0.x),
                  g.fq, g.rdx, g.rdy, g.rdz, nib & 1u);
  o.y = p_cell<R>(P4.y, __fsub_rn(X4.z, X4.y), __fsub_rn(Y1.y, Y0.y), __fsub_rn(Z1.y, Z0.y),
                  g.fq, g.rdx, g.rdy, g.rdz, nib & 0x10u);
  o.z = p_cell<R>(P4.z, __fsub_rn(X4.w, X4.z), __fsub_rn(Y1.z, Y0.z), __fsub_rn(Z1.z, Z0.z),
                  g.fq, g.rdx, g.rdy, g.rdz, nib & 0x100u);
  o.w = p_cell<R>(P4.w, __fsub_rn(X5, X4.w), __fsub_rn(Y1.w, Y0.w), __fsub_rn(Z1.w, Z0.w),
                  g.fq, g.rdx, g.rdy, g.rdz, nib & 0x1000u);
  st4(out, o);
}

template <typename R>
__device__ __forceinline__ void v_quad_fast(const Regs<R>& g, const float* __restrict__ pc,
                                            const float* __restrict__ pz,
                                            const float* __restrict__ sx,
                                            const float* __restrict__ sy,
                                            const float* __restrict__ sz, uint32_t nib,
                                            float4& vx, float4& vy, float4& vz) {
  const float4 Pc = ld4(pc), Pym = ld4(pc - g.nxp), Pzm = ld4(pz);
  const float Pxm = pc[-1];
  const float4 VX = ld4(sx), VY = ld4(sy), VZ = ld4(sz);
  vx.x = v_cell<R>(VX.x, __fsub_rn(Pc.x, Pxm), g.fv, g.rdx, nib & 0x2u);
  vx.y = v_cell<R>(VX.y, __fsub_rn(Pc.y, Pc.x), g.fv, g.rdx, nib & 0x20u);
  vx.z = v_cell<R>(VX.z, __fsub_rn(Pc.z, Pc.y), g.fv, g.rdx, nib & 0x200u);
  vx.w = v_cell<R>(VX.w, __fsub_rn(Pc.w, Pc.z), g.fv, g.rdx, nib & 0x2000u);
  vy.x = v_cell<R>(VY.x, __fsub_rn(Pc.x, Pym.x), g.fv, g.rdy, nib & 0x4u);
  vy.y = v_cell<R>(VY.y, __fsub_rn(Pc.y, Pym.y), g.fv, g.rdy, nib & 0x40u);
  vy.z = v_cell<R>(VY.z, __fsub_rn(Pc.z, Pym.z), g.fv, g.rdy, nib & 0x400u);
  vy.w = v_cell<R>(VY.w, __fsub_rn(Pc.w, Pym.w), g.fv, g.rdy, nib & 0x4000u);
  vz.x = v_cell<R>(VZ.x, __fsub_rn(Pc.x, Pzm.x), g.fv, g.rdz, nib & 0x8u);
  vz.y = v_cell<R>(VZ.y, __fsub_rn(Pc.y, Pzm.y), g.fv, g.rdz, nib & 0x80u);
  vz.z = v_cell<R>(VZ.z, __fsub_rn(Pc.z, Pzm.z), g.fv, g.rdz, nib & 0x800u);
  vz.w = v_cell<R>(VZ.w, __fsub_rn(Pc.w, Pzm.w), g.fv, g.rdz, nib & 0x8000u);
}

// interp_trilinear! entries of one (tile, plane, channel) in transceiver
// order per cell: rec += w*f (stored per entry, summed by the epilogue in
// corner order), then f += w*src[it].  A segment with one entry carries it
// inline {cell | 1<<16, w, slot, src column}; longer ones point at the
// entry arrays {cell | n<<16, first entry, 0, 0}.
__device__ __forceinline__ void process_entries(const SolveDev& S, int b, int e, int chan,
                                                float* cells, bool records, int it) {
  const float* src = S.src[chan] + (long long)(it - 1) * S.src_ntx;
  for (int si = b + (int)threadIdx.x; si < e; si += NCT) {
    const int4 sg = __ldg(S.seg + si);
    const int cell = sg.x & 0xFFFF, cnt = (int)((unsigned)sg.x >> 16);
    float v = cells[cell];
    if (cnt == 1) {
      const float w = __int_as_float(sg.y);
      if (records && sg.z >= 0) S.contrib[sg.z] = __fmul_rn(w, v);
      if (sg.w >= 0) v = __fadd_rn(v, __fmul_rn(w, __ldg(src + sg.w)));
    } else {
      for (int k = sg.y; k < sg.y + cnt; ++k) {
        const float w = __ldg(S.ent_w + k);
        const int slot = __ldg(S.ent_slot + k);
        if (records && slot >= 0) S.contrib[slot] = __fmul_rn(w, v);
        const int col = __ldg(S.ent_tx + k);
        if (col >= 0) v = __fadd_rn(v, __fmul_rn(w, __ldg(src + col)));  // receivers: src == 0
      }
    }
    cells[cell] = v;
  }
}

__device__ __forceinline__ void store_outputs(const SolveDev& S, const PlaneCtx& c, int r, int q,
                                              float4 P4, float4 vx, float4 vy, float4 vz) {
  const int j = c.j0 - 1 + r;
  const int pl = c.pl;
  float* out = S.field + (long long)c.wb * S.buf_stride;
  const long long row = ((long long)pl * S.ny + j) * S.nxp + 4 * q;
  st4(out + row, P4);
  st4(out + S.chan_stride + row, vx);
  // rigid mirrors (forward.jl:134-137): Vy[:,1,:] = -Vy[:,2,:], Vz[:,:,1] = -Vz[:,:,2]
  if (j != 0) st4(out + 2 * S.chan_stride + row, vy);
  if (j == 1)
    st4(out + 2 * S.chan_stride + row - S.nxp, make_float4(-vy.x, -vy.y, -vy.z, -vy.w));
  if (pl != 0) st4(out + 3 * S.chan_stride + row, vz);
  if (pl == 1)
    st4(out + 3 * S.chan_stride + row - (long long)S.ny * S.nxp,
        make_float4(-vz.x, -vz.y, -vz.z, -vz.w));
}

__device__ __forceinline__ void store_cell(const SolveDev& S, const PlaneCtx& c, int r, int x,
                                           float P, float vx, float vy, float vz) {
  const int j = c.j0 - 1 + r;
  const int pl = c.pl;
  float* out = S.field + (long long)c.wb * S.buf_stride;
  const long long cell = ((long long)pl * S.ny + j) * S.nxp + x;
  out[cell] = P;
  out[S.chan_stride + cell] = vx;
  if (j != 0) out[2 * S.chan_stride + cell] = vy;
  if (j == 1) out[2 * S.chan_stride + cell - S.nxp] = -vy;
  if (pl != 0) out[3 * S.chan_stride + cell] = vz;
  if (pl == 1) out[3 * S.chan_stride + cell - (long long)S.ny * S.nxp] = -vz;
}

// Work index -> (row, quad, cell) for an ordinary tile-plane.  Boundary quads
// (the first nl and the last nb-nl quads of a row) are split into their four
// cells, one cell per thread, so that the longer boundary update is spread
// over several warps instead of making one warp the critical path of the
// plane.  Work units: the interior quads of every row, then the boundary
// cells.  Division by the per-row counts uses a 32.32 reciprocal (exact for
// u, divisor < 2^16).
struct XSplit {
  int nl, ni, nb, na, na_pad, total;
  unsigned long long mb, mi;
  // u -> (row, quad, cell); cell = -1 for an interior quad (all four cells).
  // Interior quads come first, so the threads whose unit is a boundary cell
  // are the ones without a second unit in phases with more units than
  // threads.
  __device__ __forceinline__ void map(int u, int& row, int& q, int& e) const {
    const int nint = total - na_pad;
    if (u < nint) {
      row = (int)(((unsigned long long)u * mi) >> 32);
      q = nl + u - row * ni;
      e = -1;
      return;
    }
    u -= nint;
    if (u >= na) { row = -1; e = 0; return; }
    row = (int)(((unsigned long long)u * mb) >> 32);
    const int k = u - row * 4 * nb;
    const int kq = k >> 2;
    q = kq < nl ? kq : kq + ni;
    e = k & 3;
  }
};
__device__ __forceinline__ XSplit make_split(int xmin, int xmax, int nq, int nrows) {
  XSplit s;
  s.nl = (xmin + 3) / 4;                     // quads with x0 < xmin
  const int qhi = xmax >= 3 ? (xmax - 3) / 4 : -1;  // last quad with x0+3 <= xmax
  s.ni = max(0, min(qhi, nq - 1) - s.nl + 1);
  s.nb = nq - s.ni;
  s.na = nrows * s.nb * 4;
  s.na_pad = (s.na + 31) / 32 * 32;
  s.total = s.na_pad + nrows * s.ni;
  s.mb = s.nb ? ((1ull << 32) + 4 * s.nb - 1) / (4 * s.nb) : 0;
  s.mi = s.ni ? ((1ull << 32) + s.ni - 1) / s.ni : 0;
  return s;
}

template <typename R>
__device__ bool consume_item(const StepParams& p, const SolveDev& S, int4 item, int it,
                             uint64_t* full, uint64_t* empty, float* ring, float* pn, int& n,
                             volatile int* s_fail, const float* s_co) {
  using A = Arith<R>;
  const int rb = (it - S.it_first) & 1;
  const int ty = S.ty, nxp = S.nxp, nq = nxp / 4;
  const int j0 = item.y * ty;
  const int Rr = ty + 2;
  const bool has_mask = (S.flags & SF_MASK) != 0;
  const bool pcpml = (S.flags & SF_PCPML) != 0, vcpml = (S.flags & SF_VCPML) != 0;
  const SlotLayout L = slot_layout(ty, nxp, has_mask ? S.mw : 0, pcpml ? S.npp : 0,
                                   vcpml ? S.nvp : 0, !(S.flags & SF_YZG));
  const int pz0 = item.z > 0 ? item.z - 1 : 0;
  const int tid = threadIdx.x;
  Regs<R> g;
  g.nxp = nxp;
  g.R2 = Rr;
  g.fq = A::fq(S);
  g.fv = A::fv(S);
  g.rdx = A::rdx(S);
  g.rdy = A::rdy(S);
  g.rdz = A::rdz(S);
  const int nx = S.nx, ny = S.ny, nz = S.nz, npml = S.npml, mw = S.mw;
  // thread -> (row, quad) walk: stride NCT over rows of nq quads
  const int dr = NCT / nq, dq = NCT - (NCT / nq) * nq;
  const int r_first = tid / nq, q_first = tid - r_first * nq;
  // x ranges where every cell of a quad takes the plain update
  const int p_xmin = pcpml ? npml : 0;
  const int p_xmax = pcpml ? min(nx - 2, nx - npml - 1) : nx - 2;
  const int v_xmin = vcpml ? npml + 1 : 1;
  const int v_xmax = vcpml ? nx - npml - 2 : nx - 1;
  // Ordinary tile-planes: boundary quads (x slab / x edges) are packed into
  // whole warps ahead of the interior quads, so interior warps never diverge
  // into the boundary path.  Row range and x classes per phase:
  const int rP0 = j0 == 0 ? 1 : 0, rP1 = min(ty, ny - j0);
  const int rV1 = min(ty, ny - j0);
  bool tileP = rP1 >= rP0, tileV = rV1 >= 1;
  for (int r = rP0; r <= rP1; ++r) {
    const int j = j0 - 1 + r;
    tileP = tileP && (j != ny - 1) && (!pcpml || (j >= npml && j < ny - npml));
  }
  for (int r = 1; r <= rV1; ++r) {
    const int j = j0 - 1 + r;
    tileV = tileV && j >= 1 && (!vcpml || (j > npml && j < ny - npml - 1));
  }
  const XSplit sP = make_split(p_xmin, p_xmax, nq, rP1 - rP0 + 1);
  const XSplit sV = make_split(v_xmin, v_xmax, nq, rV1);
  tileP = tileP && sP.ni > 0;
  tileV = tileV && sV.ni > 0;
  for (int pl = pz0; pl < item.w; ++pl, ++n) {
    const int slot = n % p.stages;
    const int round = n / p.stages;
    // every consumer thread waits; a thread that gives up skips the P phase
    // and the abort is decided uniformly after the barrier below, so no
    // thread is ever left alone in bar.sync
    const bool landed = mbar_wait(smem_u32(&full[slot]), round & 1);
    if (!landed) *s_fail = 1;
    const bool prologue = pl < item.z;
    float* base = ring + (long long)slot * p.stage_floats;
    PlaneCtx c;
    c.sP = base;
    c.sVx = base + L.reg;
    c.sVy = base + 2 * L.reg;
    c.sVz = base + L.off_vz;
    c.sM = reinterpret_cast<const uint32_t*>(base + L.off_m);
    c.sXp = base + L.off_xp;
    c.sXv = base + L.off_xv;
    c.yP = base + L.off_py;
    c.yV = base + L.off_vy;
    c.zP = base + L.off_pz;
    c.zV = base + L.off_vz2;
    c.co = s_co;
    c.ysP = (pcpml && !(S.flags & SF_YZG)) ? tile_yside(j0, ty, ny, npml) : -1;
    c.ysV = (vcpml && !(S.flags & SF_YZG)) ? tile_yside(j0, ty, ny, npml + 1) : -1;
    c.pn_cur = pn + (n % kPnBufs) * p.pn_floats;
    c.pn_prev = pn + ((n + kPnBufs - 1) % kPnBufs) * p.pn_floats;
    c.j0 = j0;
    c.R = Rr;
    c.pl = pl;
    c.rb = rb;
    c.wb = rb ^ 1;
    c.has_mask = has_mask;
    // ---- P phase: rows j0-1 .. j0+ty-1 ----
    if (landed) {
      const bool pl_plain = !(pl == nz - 1) && (!pcpml || (pl >= npml && pl < nz - npml));
      auto p_work = [&](int r, int q, bool fast) {
        if (fast) {
          uint32_t nib = 0xFFFFu;
          if (has_mask) nib = (c.sM[r * mw + (q >> 1)] >> ((q & 1) * 16)) & 0xFFFFu;
          const int o = r * nxp + 4 * q;
          p_quad_fast<R>(g, c.sP + o, c.sVx + o, c.sVy + o, c.sVz + o, c.pn_cur + o, nib);
        } else {
          p_quad<R>(S, g, c, r, q, !prologue && r >= 1);
        }
      };
      if (pl_plain && tileP) {
        for (int u = tid; u < sP.total; u += NCT) {
          int row, q, e;
          sP.map(u, row, q, e);
          if (row < 0) continue;
          if (e < 0)
            p_work(rP0 + row, q, true);
          else
            p_xcell<R>(S, g, c, rP0 + row, 4 * q + e, !prologue && rP0 + row >= 1);
        }
      } else {
        for (int r = r_first, q = q_first; r <= ty; q += dq, r += dr) {
          if (q >= nq) { q -= nq; ++r; if (r > ty) break; }
          const int j = j0 - 1 + r;
          if (j < 0 || j >= ny) continue;
          const int x0 = 4 * q;
          const bool row_plain = (j != ny - 1) && (!pcpml || (j >= npml && j < ny - npml));
          p_work(r, q, pl_plain && row_plain && x0 + 3 <= p_xmax && x0 >= p_xmin);
        }
      }
    }
    consumer_bar();
    if (*s_fail) {
      if (tid == 0) atomicExch(p.err, KERR_FULL_TIMEOUT);
      return false;
    }
    // ---- Q phase: q-channel inject/record on P (forward.jl:92) ----
    const int* hdr = reinterpret_cast<const int*>(base + p.stage_floats - 32);
    const int off0 = hdr[0], off1 = hdr[1], off2 = hdr[2], off3 = hdr[3], off4 = hdr[4];
    if (off0 < off1) {
      process_entries(S, off0, off1, 0, c.pn_cur, !prologue, it);
      consumer_bar();
    }
    if (!prologue) {
      const bool has_f = off1 < off4;
      const bool pl_vplain = pl >= 1 && (!vcpml || (pl > npml && pl < nz - npml - 1));
      auto v_work = [&](int r, int q, bool fast) {
        float4 vx, vy, vz;
        const int o = r * nxp + 4 * q;
        if (fast) {
          uint32_t nib = 0xFFFFu;
          if (has_mask) nib = (c.sM[r * mw + (q >> 1)] >> ((q & 1) * 16)) & 0xFFFFu;
          v_quad_fast<R>(g, c.pn_cur + o, c.pn_prev + o, c.sVx + o, c.sVy + o, c.sVz + o, nib,
                         vx, vy, vz);
        } else {
          v_quad<R>(S, g, c, r, q, vx, vy, vz);
        }
        if (has_f) {  // stage into this slot's own rows (only this thread reads them)
          st4(const_cast<float*>(c.sVx) + o, vx);
          st4(const_cast<float*>(c.sVy) + o, vy);
          st4(const_cast<float*>(c.sVz) + o, vz);
        } else {
          store_outputs(S, c, r, q, ld4(c.pn_cur + o), vx, vy, vz);
        }
      };
      if (pl_vplain && tileV) {
        for (int u = tid; u < sV.total; u += NCT) {
          int row, q, e;
          sV.map(u, row, q, e);
          if (row < 0) continue;
          if (e < 0) {
            v_work(1 + row, q, true);
          } else {
            const int r = 1 + row, x = 4 * q + e, o = r * nxp + x;
            float vx, vy, vz;
            v_xcell<R>(S, g, c, r, x, vx, vy, vz);
            if (has_f) {  // stage into this slot's own row cells (only this thread reads them)
              const_cast<float*>(c.sVx)[o] = vx;
              const_cast<float*>(c.sVy)[o] = vy;
              const_cast<float*>(c.sVz)[o] = vz;
            } else {
              store_cell(S, c, r, x, c.pn_cur[o], vx, vy, vz);
            }
          }
        }
      } else {
        for (int r = 1 + r_first, q = q_first; r <= ty; q += dq, r += dr) {
          if (q >= nq) { q -= nq; ++r; if (r > ty) break; }
          const int j = j0 - 1 + r;
          if (j >= ny) continue;
          const int x0 = 4 * q;
          const bool row_vplain = j >= 1 && (!vcpml || (j > npml && j < ny - npml - 1));
          v_work(r, q, pl_vplain && row_vplain && x0 >= v_xmin && x0 + 3 <= v_xmax);
        }
      }
      if (has_f) {
        consumer_bar();
        // ---- F phase: f-channel inject/record (forward.jl:111-115) ----
        if (off1 < off2) process_entries(S, off1, off2, 1, const_cast<float*>(c.sVx), true, it);
        if (off2 < off3) process_entries(S, off2, off3, 2, const_cast<float*>(c.sVy), true, it);
        if (off3 < off4) process_entries(S, off3, off4, 3, const_cast<float*>(c.sVz), true, it);
        consumer_bar();
        for (int r = 1 + r_first, q = q_first; r <= ty; q += dq, r += dr) {
          if (q >= nq) { q -= nq; ++r; if (r > ty) break; }
          const int j = j0 - 1 + r;
          if (j >= ny) continue;
          const int o = r * nxp + 4 * q;
          store_outputs(S, c, r, q, ld4(c.pn_cur + o), ld4(c.sVx + o), ld4(c.sVy + o),
                        ld4(c.sVz + o));
        }
        // generic-proxy writes to the slot must be ordered before the next
        // TMA write into it
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      }
    }
    __syncwarp();
    if ((tid & 31) == 0) mbar_arrive(smem_u32(&empty[slot]));
  }
  return true;
}

// MINB = CTAs per SM the launch is sized for: 2 caps registers so two CTAs
// fit, 1 gives the kernel the registers it needs without spilling.
template <int MINB>
__global__ void __launch_bounds__(NTHREADS, MINB) adf_fdtd_step_kernel(const StepParams p) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw);
  uint64_t* empty = full + kMaxStages;
  float* ring = reinterpret_cast<float*>(smem_raw + 256);
  float* pn = ring + (long long)p.stages * p.stage_floats;
  __shared__ int s_fail;
  const int tid = threadIdx.x;
  if (tid == 0) {
    s_fail = 0;
    for (int s = 0; s < p.stages; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), NCW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();

  if (tid >= NCT) {
    // ---------------- producer warp: TMA loads into the ring ----------------
    if (tid != NCT) return;
    int n = 0;
    int last_round[kMaxStages];
    for (int s = 0; s < kMaxStages; ++s) last_round[s] = -1;
    int cur = -1;
    for (int i = blockIdx.x; i < p.n_items; i += gridDim.x) {
      if (*(volatile int*)p.err) break;
      const int4 item = p.items[i];
      const SolveDev& S = p.solves[item.x];
      const int it = S.it_base + p.step;
      if (it > S.it_stop) continue;
      const int rb = (it - S.it_first) & 1;
      const CUtensorMap* tm = p.tmaps + kTmaps * item.x;
      if (item.x != cur) {
        for (int k = 0; k < kTmaps; ++k) tmap_acquire(tm + k);
        cur = item.x;
      }
      const int ty = S.ty, nxp = S.nxp, Rr = ty + 2;
      const int j0 = item.y * ty;
      const bool has_mask = (S.flags & SF_MASK) != 0;
      const bool pcpml = (S.flags & SF_PCPML) != 0, vcpml = (S.flags & SF_VCPML) != 0;
      const bool stage_yz = !(S.flags & SF_YZG);
      const SlotLayout L = slot_layout(ty, nxp, has_mask ? S.mw : 0, pcpml ? S.npp : 0,
                                       vcpml ? S.nvp : 0, stage_yz);
      const uint32_t bytes0 =
          (uint32_t)(5 * Rr * nxp * 4 + (has_mask ? Rr * S.mw * 4 : 0) +
                     (pcpml ? 2 * Rr * S.npp * 4 : 0) + (vcpml ? 2 * Rr * S.nvp * 4 : 0));
      const uint32_t box_bytes = (uint32_t)(Rr * nxp * 4);
      const int ny = S.ny, nz = S.nz, npml = S.npml;
      const int ysP = (pcpml && stage_yz) ? tile_yside(j0, ty, ny, npml) : -1;
      const int ysV = (vcpml && stage_yz) ? tile_yside(j0, ty, ny, npml + 1) : -1;
      const int pz0 = item.z > 0 ? item.z - 1 : 0;
      bool ok = true;
      for (int pl = pz0; pl < item.w; ++pl, ++n) {
        const int slot = n % p.stages, round = n / p.stages;
        if (!mbar_wait(smem_u32(&empty[slot]), (round & 1) ^ 1)) {
          atomicExch(p.err, KERR_EMPTY_TIMEOUT);
          ok = false;
          break;
        }
        const uint32_t mb = smem_u32(&full[slot]);
        float* base = ring + (long long)slot * p.stage_floats;
        // bulk copies first (the transaction count may dip below zero until
        // the arrive below adds the expected bytes; the phase cannot complete
        // before that arrive)
        tma_load_5d(smem_u32(base), tm, mb, 0, 0, j0 - 1, pl, 4 * rb + 0);
        tma_load_5d(smem_u32(base + L.reg), tm, mb, 0, 0, j0 - 1, pl, 4 * rb + 1);
        tma_load_5d(smem_u32(base + 2 * L.reg), tm, mb, 0, 0, j0 - 1, pl, 4 * rb + 2);
        tma_load_5d(smem_u32(base + L.off_vz), tm + 1, mb, 0, 0, j0 - 1, pl, 4 * rb + 3);
        if (has_mask) tma_load_3d(smem_u32(base + L.off_m), tm + 2, mb, 0, j0 - 1, pl);
        // x-slab CPML memory of both sides: box (np, R, 1, 2) at (0, j0-1, pl, 2*rb)
        if (pcpml) tma_load_4d(smem_u32(base + L.off_xp), tm + 3, mb, 0, j0 - 1, pl, 2 * rb);
        if (vcpml) tma_load_4d(smem_u32(base + L.off_xv), tm + 4, mb, 0, j0 - 1, pl, 2 * rb);
        // y-slab rows of the tile (rows outside the slab arrive as zeros) and
        // the z-slab plane, p and v sides
        uint32_t bytes = bytes0;
        if (ysP >= 0) {
          const int l0 = ysP == 0 ? j0 - 1 : j0 - 1 - (ny - npml);
          tma_load_5d(smem_u32(base + L.off_py), tm + 5, mb, 0, 0, l0, pl, 2 * rb + ysP);
          bytes += box_bytes;
        }
        if (ysV >= 0) {
          const int l0 = ysV == 0 ? j0 - 1 : j0 - 1 - (ny - npml - 1);
          tma_load_5d(smem_u32(base + L.off_vy), tm + 6, mb, 0, 0, l0, pl, 2 * rb + ysV);
          bytes += box_bytes;
        }
        if (pcpml && stage_yz) {
          const int zs = plane_zside(pl, nz, npml);
          if (zs >= 0) {
            const int l = zs == 0 ? pl : pl - (nz - npml);
            tma_load_5d(smem_u32(base + L.off_pz), tm + 7, mb, 0, 0, j0 - 1, l, 2 * rb + zs);
            bytes += box_bytes;
          }
        }
        if (vcpml && stage_yz) {
          const int zs = plane_zside(pl, nz, npml + 1);
          if (zs >= 0) {
            const int l = zs == 0 ? pl : pl - (nz - npml - 1);
            tma_load_5d(smem_u32(base + L.off_vz2), tm + 8, mb, 0, 0, j0 - 1, l, 2 * rb + zs);
            bytes += box_bytes;
          }
        }
        {  // entry-list offsets of this (tile, plane), staged for the consumers
          int* hdr = reinterpret_cast<int*>(base + p.stage_floats - 32);
          const int tb = (item.y * S.nz + pl) * 4;
          const int4 o4 = *reinterpret_cast<const int4*>(S.tp_off + tb);
          hdr[0] = o4.x; hdr[1] = o4.y; hdr[2] = o4.z; hdr[3] = o4.w;
          hdr[4] = S.tp_off[tb + 4];
        }
        mbar_expect_tx(mb, bytes);  // release: the header is visible after the wait
        last_round[slot] = round;
      }
      if (!ok) break;
    }
    // never leave while a bulk copy into this CTA's shared memory is in flight
    for (int s = 0; s < p.stages; ++s)
      if (last_round[s] >= 0 && !mbar_wait(smem_u32(&full[s]), last_round[s] & 1))
        atomicExch(p.err, KERR_DRAIN_TIMEOUT);
    return;
  }

  // ---------------- consumer warps ----------------
  // the solve descriptor is read from shared memory inside the hot loops
  __shared__ __align__(16) SolveDev s_desc[2];
  __shared__ float s_coef[2][kMaxCoef];
  int n = 0, k_item = 0;
  for (int i = blockIdx.x; i < p.n_items; i += gridDim.x) {
    const int4 item = p.items[i];
    const SolveDev& G = p.solves[item.x];
    const int it = G.it_base + p.step;
    if (it > G.it_stop) continue;
    SolveDev& S = s_desc[k_item & 1];
    float* co = s_coef[k_item & 1];
    ++k_item;
    {
      const int* src = reinterpret_cast<const int*>(&G);
      int* dst = reinterpret_cast<int*>(&S);
      for (int w = tid; w < (int)(sizeof(SolveDev) / 4); w += NCT) dst[w] = src[w];
      const int ncoef = 8 * G.npml + 4;
      for (int w = tid; w < ncoef; w += NCT) co[w] = G.coef[w];
      consumer_bar();
    }
    bool ok;
    if (S.flags & SF_FP32)
      ok = consume_item<float>(p, S, item, it, full, empty, ring, pn, n, &s_fail, co);
    else
      ok = consume_item<double>(p, S, item, it, full, empty, ring, pn, n, &s_fail, co);
    if (!ok) return;
    // items run in lock-step with the producer; if it stopped on an error
    // flag the next full-barrier wait times out and returns here
  }
}

// Per-step trace assembly (derivatives.jl:51-56 record sums in corner order,
// v2vn! :85-90, vn2v! :92-97 into row it+1).
__global__ void adf_fdtd_epilogue_kernel(const EpiParams p) {
  const SolveDev& S = p.solves[blockIdx.y];
  const int it = S.it_base + p.step;
  if (it > S.it_stop) return;
  const int ntx = S.ntx;
  const bool gf = (S.flags & SF_GF) != 0;
  if (p.phase == 2) {  // vn2v! of a GF solve, after the extrapolation wrote vn_src[it+1]
    if (!gf || !S.vn_src || it >= S.nt) return;
    for (int tx = blockIdx.x * blockDim.x + threadIdx.x; tx < ntx; tx += gridDim.x * blockDim.x) {
      const long long nr = (long long)it * ntx + tx;
      const float* d = S.dir + 4 * tx;
      const float vs = S.vn_src[nr];
#pragma unroll
      for (int c = 1; c <= 3; ++c) S.src[c][nr] = __fadd_rn(S.src[c][nr], __fmul_rn(vs, d[c]));
    }
    return;
  }
  for (int tx = blockIdx.x * blockDim.x + threadIdx.x; tx < ntx; tx += gridDim.x * blockDim.x) {
    const long long row = (long long)(it - 1) * ntx + tx;
    float r[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      // a record buffer that is not kept starts every row at zero, as the
      // reference's freshly packed rec (= src*0) does
      r[c] = S.rec[c] ? S.rec[c][row] : 0.0f;
      if (S.inb[c * ntx + tx]) {
        const float* cb = S.contrib + ((long long)c * ntx + tx) * 8;
#pragma unroll
        for (int k = 0; k < 8; ++k) r[c] = __fadd_rn(r[c], cb[k]);
        if (S.rec[c]) S.rec[c][row] = r[c];
      }
    }
    const float* d = S.dir + 4 * tx;
    S.vn_rec[row] =
        __fadd_rn(__fadd_rn(__fmul_rn(r[1], d[1]), __fmul_rn(r[2], d[2])), __fmul_rn(r[3], d[3]));
    if (S.vn_src && it < S.nt && !gf) {
      const long long nr = row + ntx;
      const float vs = S.vn_src[nr];
#pragma unroll
      for (int c = 1; c <= 3; ++c) S.src[c][nr] = __fadd_rn(S.src[c][nr], __fmul_rn(vs, d[c]));
    }
  }
}

// Advances it_base of every solve by `by` steps: the last node of a captured
// chunk of steps, so replaying the graph continues where it stopped.
// In-loop GF extrapolation, extrapolate! (src/kernels/extrapolation.jl:204-249)
// after v2vn! of step it < nt, for every driven source o:
//   PVFromPin (:139-170): pin[t, r] = (p_rec - z0 vn_rec)/2 (Float64);
//     ps/vs = sum_r sum_tt p_pin/v_pin[T-tt+1, o, r] * pin[it-T+tt, r];
//     p_src[it+1, iSrc[o]] = vs, vn_src[it+1, iSrc[o]] = ps.
//   PFromPin (:172-193, 237-249): pos/neg[o] = sums of pos/neg[., r, o] * pin,
//     rounded to Float32; p_src = pos - neg, vn_src = (pos + neg) / z0.
//   PVFromPV (:91-137, 204-218): ps += pv*p + pp*vn, vs += vv*p + vp*vn over
//     the recorded p / v_n of the iRec columns (Float32 terms).
// Sums are accumulated in Float64 (the Float32 zero of the reference is
// promoted by the first Float64 add for the *FromPin kinds).  The receiver
// range of each source is split over gf_ks blocks (blockIdx.x = o*ks + part)
// whose partial sums the reduce kernel adds in a fixed order.  Rows before
// `it` of pin come from gf_pin; row `it` is formed here and block 0 files it.
__global__ void __launch_bounds__(256) adf_gf_extrapolate_kernel(const EpiParams p) {
  const SolveDev& S = p.solves[blockIdx.y];
  const int it = S.it_base + p.step;
  if (it > S.it_stop || it >= S.nt || !(S.flags & SF_GF)) return;
  const int ks = S.gf_ks;
  const int o = blockIdx.x / ks, part = blockIdx.x - (blockIdx.x / ks) * ks;
  if (o >= S.gf_nout) return;
  const int nt = S.nt, ntx = S.ntx, ngf = S.gf_nt, n1 = S.gf_n1, nin = S.gf_nin;
  const int kind = S.gf_kind;
  const int T = min(it, ngf);
  const int t0 = it - T;  // 0-based row of tt = 1
  const long long cur = (long long)(it - 1) * ntx;
  auto pin_now = [&](int r) {
    const int col = S.gf_irec[r];
    return ((double)S.rec[0][cur + col] - (double)S.vn_rec[cur + col] * S.gf_z0) / 2.0;
  };
  if (blockIdx.x == 0 && kind != ADF_GF_PV_FROM_PV_)
    for (int r = threadIdx.x; r < nin; r += blockDim.x)
      S.gf_pin[(long long)r * nt + (it - 1)] = pin_now(r);
  const int rb = (int)((long long)nin * part / ks), re = (int)((long long)nin * (part + 1) / ks);
  double a = 0.0, b = 0.0;
  // (r, tt) walk over this block's receivers, tt fastest: contiguous tensor
  // and pin reads, the index stepped instead of divided
  int r = rb + (int)threadIdx.x / T, tt = (int)threadIdx.x - ((int)threadIdx.x / T) * T;
  const int step_r = (int)blockDim.x / T, step_t = (int)blockDim.x - step_r * T;
  for (; r < re;) {
    const int row = t0 + tt;
    // tensor element [T-tt, ., .] (1-based lag) for this receiver and output
    const long long g = (long long)(T - 1 - tt) +
                        (long long)ngf * (kind == ADF_GF_PV_FROM_PIN_ ? o + (long long)n1 * r
                                                                      : r + (long long)n1 * o);
    if (kind == ADF_GF_PV_FROM_PV_) {
      const int col = S.gf_irec[r];
      const float pt = S.rec[0][(long long)row * ntx + col];
      const float vt = S.vn_rec[(long long)row * ntx + col];
      const float ps = __fadd_rn(__fmul_rn(S.gf_t[1][g], pt), __fmul_rn(S.gf_t[0][g], vt));
      const float vs = __fadd_rn(__fmul_rn(S.gf_t[3][g], pt), __fmul_rn(S.gf_t[2][g], vt));
      a = __dadd_rn(a, (double)ps);
      b = __dadd_rn(b, (double)vs);
    } else {
      const double pin = row == it - 1 ? pin_now(r) : S.gf_pin[(long long)r * nt + row];
      a = __dadd_rn(a, __dmul_rn((double)S.gf_t[0][g], pin));
      b = __dadd_rn(b, __dmul_rn((double)S.gf_t[1][g], pin));
    }
    r += step_r;
    tt += step_t;
    if (tt >= T) {
      tt -= T;
      ++r;
    }
  }
  __shared__ double red[2][8];
#pragma unroll
  for (int w = 16; w > 0; w >>= 1) {
    a = __dadd_rn(a, __shfl_down_sync(0xffffffffu, a, w));
    b = __dadd_rn(b, __shfl_down_sync(0xffffffffu, b, w));
  }
  const int wi = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    red[0][wi] = a;
    red[1][wi] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sa = 0.0, sb = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      sa = __dadd_rn(sa, red[0][k]);
      sb = __dadd_rn(sb, red[1][k]);
    }
    double* pp = S.gf_part + ((long long)o * ks + part) * 2;
    pp[0] = sa;
    pp[1] = sb;
  }
}

// Adds each source's partial sums in split order and writes its p_src and
// vn_src samples of row it+1.
__global__ void adf_gf_reduce_kernel(const EpiParams p) {
  const SolveDev& S = p.solves[blockIdx.y];
  const int it = S.it_base + p.step;
  if (it > S.it_stop || it >= S.nt || !(S.flags & SF_GF)) return;
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= S.gf_nout) return;
  double sa = 0.0, sb = 0.0;
  for (int k = 0; k < S.gf_ks; ++k) {
    const double* pp = S.gf_part + ((long long)o * S.gf_ks + k) * 2;
    sa = __dadd_rn(sa, pp[0]);
    sb = __dadd_rn(sb, pp[1]);
  }
  const int col = S.gf_isrc[o];
  float ps, vs;
  if (S.gf_kind == ADF_GF_P_FROM_PIN_) {
    const float pos = (float)sa, neg = (float)sb;
    ps = (float)((double)__fadd_rn(pos, neg) / S.gf_z0);  // vn_src
    vs = __fsub_rn(pos, neg);                              // p_src
  } else {
    ps = (float)sa;  // vn_src <- p_pin / (pv, pp)-derived
    vs = (float)sb;  // p_src  <- v_pin / (vv, vp)-derived
  }
  S.src[0][(long long)it * S.src_ntx + col] = vs;
  S.vn_src[(long long)it * S.ntx + col] = ps;
}

__global__ void adf_advance_kernel(SolveDev* solves, int n, int by) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) solves[i].it_base += by;
}

cudaError_t launch_advance(SolveDev* solves, int n, int by, cudaStream_t s) {
  adf_advance_kernel<<<(n + 127) / 128, 128, 0, s>>>(solves, n, by);
  return cudaGetLastError();
}

const void* step_kernel_ptr(bool two_per_sm) {
  return two_per_sm ? (const void*)adf_fdtd_step_kernel<2> : (const void*)adf_fdtd_step_kernel<1>;
}

cudaError_t step_kernel_attributes(size_t smem, bool two_per_sm) {
  return cudaFuncSetAttribute(step_kernel_ptr(two_per_sm),
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

cudaError_t launch_step(const StepParams& p, int grid, int block, size_t smem, cudaStream_t s,
                        bool two_per_sm) {
  if (two_per_sm)
    adf_fdtd_step_kernel<2><<<grid, block, smem, s>>>(p);
  else
    adf_fdtd_step_kernel<1><<<grid, block, smem, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_gf_extrapolate(const EpiParams& p, int max_blocks, int max_nsrc,
                                  cudaStream_t s) {
  // (source, receiver split) blocks of the largest map in the batch, then
  // the fixed-order reduction of the splits
  adf_gf_extrapolate_kernel<<<dim3(max_blocks > 0 ? max_blocks : 1, p.n_solves), 256, 0, s>>>(p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  adf_gf_reduce_kernel<<<dim3((max_nsrc + 127) / 128, p.n_solves), 128, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_epilogue(const EpiParams& p, int max_ntx, cudaStream_t s) {
  int threads = 128;
  int gx = (max_ntx + threads - 1) / threads;
  if (gx < 1) gx = 1;
  dim3 grid(gx, p.n_solves);
  adf_fdtd_epilogue_kernel<<<grid, threads, 0, s>>>(p);
  return cudaGetLastError();
}

}  // namespace adf
