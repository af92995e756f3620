// fdtd_kernels.cu -- the fused staggered-grid FDTD step for sm_100a.
//
// One launch advances every active solve of a batch by one time step
// (forward_onestep!, src/kernels/forward.jl:13-139).  The step reads field
// buffer `rb` and writes buffer `wb`, so the pressure update, the q-channel
// injection/recording, the three velocity updates, the f-channel
// injection/recording and the rigid mirrors all happen in a single pass over
// HBM: 16 B read + 16 B written per cell, plus the CPML memory on the slabs
// and half a byte of mask per cell.
//
// Work decomposition (2.5D): a CTA owns a tile of 7 rows x 64 cells of one
// solve and a run of planes; each warp holds 16 cells of all the tile's rows
// (plus the halo row), its lanes 4-cell quads, and the CTA walks the planes
// in z keeping the z-neighbours in registers.  The new P of a plane goes
// through shared memory for the x-1 / y-1 neighbours of the velocity update;
// the halo row and column are recomputed, not exchanged.  Grids of many
// such CTAs (eight per SM) keep HBM busy: the update is a short,
// memory-bound stencil.
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

constexpr int kMaxCoef = 8 * 63 + 4;  // CPML coefficients for npml <= 63

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


__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
// field stores: evict-first (the next step reads them back from HBM, and the
// halo rows that neighbouring tiles re-read are loads, which keep normal
// priority)
__device__ __forceinline__ void stcs4(float* p, float4 v) { __stcs(reinterpret_cast<float4*>(p), v); }
__device__ __forceinline__ float4 neg4(float4 v) { return make_float4(-v.x, -v.y, -v.z, -v.w); }

template <typename R>
struct Sc {  // per-solve update scalars in registers
  R fq, fv, rdx, rdy, rdz;
};

// Per-(row, plane) geometry shared by the cells of a quad, uniform across a warp.
struct RowCtx {
  int nx, ny, nz, npml, nxp, j, k, rb, wb;
  bool pcpml, vcpml;
};

// ---------------------------------------------------------------------------
// Pressure update of the quad x0..x0+3 of row j, plane k (update_p_cpml!,
// update_p_mask!, update_p! on the rigid planes; updates.jl:21-136).
// Inputs are the plane's P, Vx (x0..x0+4), Vy (rows j, j+1) and Vz (planes
// k, k+1) from the input buffer.  Row- and plane-wide conditions (rigid
// planes, y/z slabs) are warp-uniform branches; the x slab is a per-cell
// block taken only by quads that touch it.  `owned` stores the new CPML
// memory; recomputed halo cells and the prologue plane leave it alone.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ float4 p_update_quad(const SolveDev& S, const RowCtx& rc, const Sc<R>& g,
                                                const float* co, int x0, bool owned, float4 P4,
                                                float4 X4, float X5, float4 Y0, float4 Y1,
                                                float4 Z0, float4 Z1, uint32_t nib) {
  using A = Arith<R>;
  const int nx = rc.nx, ny = rc.ny, nz = rc.nz, npml = rc.npml, j = rc.j, k = rc.k;
  const bool rigid_y = j == ny - 1, rigid_z = k == nz - 1;
  // rigid planes use update_p! (-2V/d at the wall, no CPML, no mask); the
  // (ny, nz) corner is not updated at all
  const bool plain_rigid = rigid_y || rigid_z;
  const bool corner = rigid_y && rigid_z;
  if (plain_rigid) nib = 0xFFFFu;
  const float Pv[4] = {P4.x, P4.y, P4.z, P4.w};
  const float dxv[4] = {__fsub_rn(X4.y, X4.x), __fsub_rn(X4.z, X4.y), __fsub_rn(X4.w, X4.z),
                        __fsub_rn(X5, X4.w)};
  const float dyv[4] = {rigid_y ? __fmul_rn(-2.0f, Y0.x) : __fsub_rn(Y1.x, Y0.x),
                        rigid_y ? __fmul_rn(-2.0f, Y0.y) : __fsub_rn(Y1.y, Y0.y),
                        rigid_y ? __fmul_rn(-2.0f, Y0.z) : __fsub_rn(Y1.z, Y0.z),
                        rigid_y ? __fmul_rn(-2.0f, Y0.w) : __fsub_rn(Y1.w, Y0.w)};
  const float dzv[4] = {rigid_z ? __fmul_rn(-2.0f, Z0.x) : __fsub_rn(Z1.x, Z0.x),
                        rigid_z ? __fmul_rn(-2.0f, Z0.y) : __fsub_rn(Z1.y, Z0.y),
                        rigid_z ? __fmul_rn(-2.0f, Z0.z) : __fsub_rn(Z1.z, Z0.z),
                        rigid_z ? __fmul_rn(-2.0f, Z0.w) : __fsub_rn(Z1.w, Z0.w)};
  R dvx[4], dvy[4], dvz[4];
  bool upd[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    dvx[e] = A::mul(A::cv(dxv[e]), g.rdx);
    dvy[e] = A::mul(A::cv(dyv[e]), g.rdy);
    dvz[e] = A::mul(A::cv(dzv[e]), g.rdz);
    upd[e] = x0 + e <= nx - 2 && !corner;
  }
  if (rc.pcpml && !plain_rigid) {
    const bool s0 = x0 < npml, s1 = x0 + 3 >= nx - npml;
    // x slab: the quad's memory of a side is one aligned float4 (both sides
    // only on grids narrower than two slabs and a quad: one after the other)
    const long long row = ((long long)k * ny + j) * S.npp;
    for (int sd = 0; sd < 2; ++sd) {
      if (!(sd == 0 ? s0 : s1)) continue;
      const long long o = sd == 0 ? row + x0 : S.psi_p_side[0] + row + (x0 - S.xs1p);
      const float4 t = ld4(S.psi_p[0] + rc.rb * S.psi_p_buf[0] + o);
      float m[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int x = x0 + e;
        const int side = x < npml ? 0 : (x >= nx - npml ? 1 : -1);
        if (side == sd && upd[e]) {
          const int l = side == 0 ? x : x - (nx - npml);
          cpml_apply<R>(dvx[e], m[e], co[side * npml + l], co[4 * npml + 2 + side * npml + l]);
        }
      }
      // cells outside the slab or not updated write back what they read
      if (owned) st4(S.psi_p[0] + rc.wb * S.psi_p_buf[0] + o, make_float4(m[0], m[1], m[2], m[3]));
    }
    const int ysd = j < npml ? 0 : (j >= ny - npml ? 1 : -1);
    if (ysd >= 0) {  // y slab: the whole quad, cells that are not updated keep their memory
      const int yl = ysd == 0 ? j : j - (ny - npml);
      const long long o = ysd * S.psi_p_side[1] + ((long long)k * npml + yl) * rc.nxp + x0;
      const float4 m4 = ld4(S.psi_p[1] + rc.rb * S.psi_p_buf[1] + o);
      float m[4] = {m4.x, m4.y, m4.z, m4.w};
      const float a = co[ysd * npml + yl], b = co[4 * npml + 2 + ysd * npml + yl];
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (upd[e]) cpml_apply<R>(dvy[e], m[e], a, b);
      if (owned) st4(S.psi_p[1] + rc.wb * S.psi_p_buf[1] + o, make_float4(m[0], m[1], m[2], m[3]));
    }
    const int zsd = k < npml ? 0 : (k >= nz - npml ? 1 : -1);
    if (zsd >= 0) {
      const int zl = zsd == 0 ? k : k - (nz - npml);
      const long long o = zsd * S.psi_p_side[2] + ((long long)zl * ny + j) * rc.nxp + x0;
      const float4 m4 = ld4(S.psi_p[2] + rc.rb * S.psi_p_buf[2] + o);
      float m[4] = {m4.x, m4.y, m4.z, m4.w};
      const float a = co[zsd * npml + zl], b = co[4 * npml + 2 + zsd * npml + zl];
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (upd[e]) cpml_apply<R>(dvz[e], m[e], a, b);
      if (owned) st4(S.psi_p[2] + rc.wb * S.psi_p_buf[2] + o, make_float4(m[0], m[1], m[2], m[3]));
    }
  }
  float o[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const float n =
        A::rn(A::sub(A::cv(Pv[e]), A::mul(g.fq, A::add(A::add(dvx[e], dvy[e]), dvz[e]))));
    o[e] = (upd[e] && ((nib >> (4 * e)) & 1u)) ? n : Pv[e];
  }
  return make_float4(o[0], o[1], o[2], o[3]);
}

// The same update for one cell (the halo column x = xb-1 of an x tile), from
// the staged plane `st` (P, Vx, Vy of plane k; `c` the cell's offset in a
// channel, `cst` the channel stride) and Vz of planes k and k+1 (Z0, Z1).
template <typename R>
__device__ __forceinline__ float p_update_cell(const SolveDev& S, const RowCtx& rc, const Sc<R>& g,
                                               const float* co, const float* st, float Z0,
                                               float Z1, int c, int cst, int x) {
  using A = Arith<R>;
  const int nx = rc.nx, ny = rc.ny, nz = rc.nz, npml = rc.npml, j = rc.j, k = rc.k, nxp = rc.nxp;
  const bool rigid_y = j == ny - 1, rigid_z = k == nz - 1;
  const bool plain_rigid = rigid_y || rigid_z;
  const bool upd = x <= nx - 2 && !(rigid_y && rigid_z);
  const float P = st[c];
  if (!upd) return P;
  const float X0 = st[cst + c], X1 = st[cst + c + 1];
  const float Y0 = st[2 * cst + c];
  const float dy = rigid_y ? __fmul_rn(-2.0f, Y0) : __fsub_rn(st[2 * cst + c + kStageW], Y0);
  const float dz = rigid_z ? __fmul_rn(-2.0f, Z0) : __fsub_rn(Z1, Z0);
  R dvx = A::mul(A::cv(__fsub_rn(X1, X0)), g.rdx);
  R dvy = A::mul(A::cv(dy), g.rdy);
  R dvz = A::mul(A::cv(dz), g.rdz);
  bool open = true;
  if (!plain_rigid) {
    if (S.flags & SF_MASK) open = (S.mask_bits[((long long)k * ny + j) * S.mw + (x >> 3)] >> (4 * (x & 7))) & 1u;
    if (rc.pcpml) {
      const int xs = x < npml ? 0 : (x >= nx - npml ? 1 : -1);
      if (xs >= 0) {
        const int l = xs == 0 ? x : x - (nx - npml);
        float m = S.psi_p[0][rc.rb * S.psi_p_buf[0] + xs * S.psi_p_side[0] +
                             ((long long)k * ny + j) * S.npp + (xs == 0 ? x : x - S.xs1p)];
        cpml_apply<R>(dvx, m, co[xs * npml + l], co[4 * npml + 2 + xs * npml + l]);
      }
      const int ysd = j < npml ? 0 : (j >= ny - npml ? 1 : -1);
      if (ysd >= 0) {
        const int yl = ysd == 0 ? j : j - (ny - npml);
        float m = S.psi_p[1][rc.rb * S.psi_p_buf[1] + ysd * S.psi_p_side[1] +
                             ((long long)k * npml + yl) * nxp + x];
        cpml_apply<R>(dvy, m, co[ysd * npml + yl], co[4 * npml + 2 + ysd * npml + yl]);
      }
      const int zsd = k < npml ? 0 : (k >= nz - npml ? 1 : -1);
      if (zsd >= 0) {
        const int zl = zsd == 0 ? k : k - (nz - npml);
        float m = S.psi_p[2][rc.rb * S.psi_p_buf[2] + zsd * S.psi_p_side[2] +
                             ((long long)zl * ny + j) * nxp + x];
        cpml_apply<R>(dvz, m, co[zsd * npml + zl], co[4 * npml + 2 + zsd * npml + zl]);
      }
    }
  }
  const float n = A::rn(A::sub(A::cv(P), A::mul(g.fq, A::add(A::add(dvx, dvy), dvz))));
  return open ? n : P;
}

// ---------------------------------------------------------------------------
// Velocity updates of the quad (update_vx!/vy!/vz! and their masked forms,
// updates.jl:192-274, 380-500): Vx over x >= 1, Vy over j >= 1, Vz over k >= 1,
// x < nx; CPML with the half-grid coefficients (npml+1 layers).
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void v_update_quad(const SolveDev& S, const RowCtx& rc, const Sc<R>& g,
                                              const float* co, int x0, float4 Pc, float Pxm,
                                              float4 Pym, float4 Pzm, float4 VX, float4 VY,
                                              float4 VZ, uint32_t nib, float4& vxo, float4& vyo,
                                              float4& vzo) {
  using A = Arith<R>;
  const int nx = rc.nx, ny = rc.ny, nz = rc.nz, npml = rc.npml, nm = npml + 1, j = rc.j, k = rc.k;
  const float Pv[4] = {Pc.x, Pc.y, Pc.z, Pc.w};
  const float Pl[4] = {Pxm, Pc.x, Pc.y, Pc.z};
  const float Py[4] = {Pym.x, Pym.y, Pym.z, Pym.w};
  const float Pz[4] = {Pzm.x, Pzm.y, Pzm.z, Pzm.w};
  const float Vx[4] = {VX.x, VX.y, VX.z, VX.w};
  const float Vy[4] = {VY.x, VY.y, VY.z, VY.w};
  const float Vz[4] = {VZ.x, VZ.y, VZ.z, VZ.w};
  R dx[4], dy[4], dz[4];
  bool in[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    dx[e] = A::mul(A::cv(__fsub_rn(Pv[e], Pl[e])), g.rdx);
    dy[e] = A::mul(A::cv(__fsub_rn(Pv[e], Py[e])), g.rdy);
    dz[e] = A::mul(A::cv(__fsub_rn(Pv[e], Pz[e])), g.rdz);
    in[e] = x0 + e < nx;
  }
  if (rc.vcpml) {
    const bool s0 = x0 <= npml, s1 = x0 + 3 >= nx - npml - 1;
    // x slab: one aligned float4 per side, the sides one after the other
    const long long row = ((long long)k * ny + j) * S.nvp;
    for (int sd = 0; sd < 2; ++sd) {
      if (!(sd == 0 ? s0 : s1)) continue;
      const long long o = sd == 0 ? row + x0 : S.psi_v_side[0] + row + (x0 - S.xs1v);
      const float4 t = ld4(S.psi_v[0] + rc.rb * S.psi_v_buf[0] + o);
      float m[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int x = x0 + e;
        const int side = x <= npml ? 0 : (x >= nx - npml - 1 ? 1 : -1);
        if (side == sd && in[e] && x >= 1) {
          const int l = side == 0 ? x : x - (nx - npml - 1);
          cpml_apply<R>(dx[e], m[e], co[2 * npml + side * nm + l], co[6 * npml + 2 + side * nm + l]);
        }
      }
      st4(S.psi_v[0] + rc.wb * S.psi_v_buf[0] + o, make_float4(m[0], m[1], m[2], m[3]));
    }
    const int ysd = j < 1 ? -1 : (j <= npml ? 0 : (j >= ny - npml - 1 ? 1 : -1));
    if (ysd >= 0) {
      const int yl = ysd == 0 ? j : j - (ny - npml - 1);
      const long long o = ysd * S.psi_v_side[1] + ((long long)k * nm + yl) * rc.nxp + x0;
      const float4 m4 = ld4(S.psi_v[1] + rc.rb * S.psi_v_buf[1] + o);
      float m[4] = {m4.x, m4.y, m4.z, m4.w};
      const float a = co[2 * npml + ysd * nm + yl], b = co[6 * npml + 2 + ysd * nm + yl];
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (in[e]) cpml_apply<R>(dy[e], m[e], a, b);
      st4(S.psi_v[1] + rc.wb * S.psi_v_buf[1] + o, make_float4(m[0], m[1], m[2], m[3]));
    }
    const int zsd = k < 1 ? -1 : (k <= npml ? 0 : (k >= nz - npml - 1 ? 1 : -1));
    if (zsd >= 0) {
      const int zl = zsd == 0 ? k : k - (nz - npml - 1);
      const long long o = zsd * S.psi_v_side[2] + ((long long)zl * ny + j) * rc.nxp + x0;
      const float4 m4 = ld4(S.psi_v[2] + rc.rb * S.psi_v_buf[2] + o);
      float m[4] = {m4.x, m4.y, m4.z, m4.w};
      const float a = co[2 * npml + zsd * nm + zl], b = co[6 * npml + 2 + zsd * nm + zl];
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (in[e]) cpml_apply<R>(dz[e], m[e], a, b);
      st4(S.psi_v[2] + rc.wb * S.psi_v_buf[2] + o, make_float4(m[0], m[1], m[2], m[3]));
    }
  }
  float ox[4], oy[4], oz[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const bool ux = in[e] && x0 + e >= 1 && ((nib >> (4 * e + 1)) & 1u);
    const bool uy = in[e] && j >= 1 && ((nib >> (4 * e + 2)) & 1u);
    const bool uz = in[e] && k >= 1 && ((nib >> (4 * e + 3)) & 1u);
    const float nxv = A::rn(A::sub(A::cv(Vx[e]), A::mul(g.fv, dx[e])));
    const float nyv = A::rn(A::sub(A::cv(Vy[e]), A::mul(g.fv, dy[e])));
    const float nzv = A::rn(A::sub(A::cv(Vz[e]), A::mul(g.fv, dz[e])));
    ox[e] = ux ? nxv : Vx[e];
    oy[e] = uy ? nyv : Vy[e];
    oz[e] = uz ? nzv : Vz[e];
  }
  vxo = make_float4(ox[0], ox[1], ox[2], ox[3]);
  vyo = make_float4(oy[0], oy[1], oy[2], oy[3]);
  vzo = make_float4(oz[0], oz[1], oz[2], oz[3]);
}

// ---------------------------------------------------------------------------
// interp_trilinear! entries of one (y tile, plane, channel) bucket
// (derivatives.jl:30-60).  Segments are cells {cell = r*nxp + x | n << 16};
// inside a cell the entries are in transceiver order: rec += w*f (stored per
// entry, summed by the epilogue in corner order), then f += w*src[it].  The
// CTA handles the cells of its x range [x_lo, x_hi) and records only those
// it owns (row >= 1, x >= xb; the P bucket also carries the tile's halo row
// with slot -1).  `cells` maps (r, x) -> shared memory.
// ---------------------------------------------------------------------------
template <typename CellAt>
__device__ __forceinline__ void apply_entries(const SolveDev& S, int b, int e, int chan, int nxp,
                                              int x_lo, int x_hi, int xb, bool records, int it,
                                              int tid, int nthr, CellAt cell_at) {
  const float* src = S.src[chan] + (long long)(it - 1) * S.src_ntx;
  for (int si = b + tid; si < e; si += nthr) {
    const int4 sg = __ldg(S.seg + si);
    const int cell = sg.x & 0xFFFF, cnt = (int)((unsigned)sg.x >> 16);
    const int r = cell / nxp, x = cell - r * nxp;
    if (x < x_lo || x >= x_hi) continue;
    const bool rec = records && r >= 1 && x >= xb;
    float* c = cell_at(r, x);
    float v = *c;
    if (cnt == 1) {
      const float w = __int_as_float(sg.y);
      if (rec && sg.z >= 0) S.contrib[sg.z] = __fmul_rn(w, v);
      if (sg.w >= 0) v = __fadd_rn(v, __fmul_rn(w, __ldg(src + sg.w)));
    } else {
      for (int kk = sg.y; kk < sg.y + cnt; ++kk) {
        const float w = __ldg(S.ent_w + kk);
        const int slot = __ldg(S.ent_slot + kk);
        if (rec && slot >= 0) S.contrib[slot] = __fmul_rn(w, v);
        const int col = __ldg(S.ent_tx + kk);
        if (col >= 0) v = __fadd_rn(v, __fmul_rn(w, __ldg(src + col)));  // receivers: src == 0
      }
    }
    *c = v;
  }
}

// ---- plain quads: every cell interior for its update (no rigid plane, no
// CPML slab, no grid edge); the same arithmetic as the general functions
// for such cells, without their conditions.
template <typename R>
__device__ __forceinline__ float p_plain(float P, float dx, float dy, float dz, const Sc<R>& g) {
  using A = Arith<R>;
  const R s = A::add(A::add(A::mul(A::cv(dx), g.rdx), A::mul(A::cv(dy), g.rdy)),
                     A::mul(A::cv(dz), g.rdz));
  return A::rn(A::sub(A::cv(P), A::mul(g.fq, s)));
}
template <typename R>
__device__ __forceinline__ float v_plain(float V, float dp, R rd, const Sc<R>& g) {
  using A = Arith<R>;
  return A::rn(A::sub(A::cv(V), A::mul(g.fv, A::mul(A::cv(dp), rd))));
}
template <typename R, bool MASK>
__device__ __forceinline__ float4 p_plain_quad(const Sc<R>& g, float4 P4, float4 X4, float X5,
                                               float4 Y0, float4 Y1, float4 Z0, float4 Z1,
                                               uint32_t nib) {
  float4 n;
  n.x = p_plain<R>(P4.x, __fsub_rn(X4.y, X4.x), __fsub_rn(Y1.x, Y0.x), __fsub_rn(Z1.x, Z0.x), g);
  n.y = p_plain<R>(P4.y, __fsub_rn(X4.z, X4.y), __fsub_rn(Y1.y, Y0.y), __fsub_rn(Z1.y, Z0.y), g);
  n.z = p_plain<R>(P4.z, __fsub_rn(X4.w, X4.z), __fsub_rn(Y1.z, Y0.z), __fsub_rn(Z1.z, Z0.z), g);
  n.w = p_plain<R>(P4.w, __fsub_rn(X5, X4.w), __fsub_rn(Y1.w, Y0.w), __fsub_rn(Z1.w, Z0.w), g);
  if (MASK) {
    n.x = (nib & 1u) ? n.x : P4.x;
    n.y = (nib & 0x10u) ? n.y : P4.y;
    n.z = (nib & 0x100u) ? n.z : P4.z;
    n.w = (nib & 0x1000u) ? n.w : P4.w;
  }
  return n;
}
template <typename R, bool MASK>
__device__ __forceinline__ void v_plain_quad(const Sc<R>& g, float4 Pc, float Pxm, float4 Pym,
                                             float4 Pzm, float4 VX, float4 VY, float4 VZ,
                                             uint32_t nib, float4& vx, float4& vy, float4& vz) {
  vx.x = v_plain<R>(VX.x, __fsub_rn(Pc.x, Pxm), g.rdx, g);
  vx.y = v_plain<R>(VX.y, __fsub_rn(Pc.y, Pc.x), g.rdx, g);
  vx.z = v_plain<R>(VX.z, __fsub_rn(Pc.z, Pc.y), g.rdx, g);
  vx.w = v_plain<R>(VX.w, __fsub_rn(Pc.w, Pc.z), g.rdx, g);
  vy.x = v_plain<R>(VY.x, __fsub_rn(Pc.x, Pym.x), g.rdy, g);
  vy.y = v_plain<R>(VY.y, __fsub_rn(Pc.y, Pym.y), g.rdy, g);
  vy.z = v_plain<R>(VY.z, __fsub_rn(Pc.z, Pym.z), g.rdy, g);
  vy.w = v_plain<R>(VY.w, __fsub_rn(Pc.w, Pym.w), g.rdy, g);
  vz.x = v_plain<R>(VZ.x, __fsub_rn(Pc.x, Pzm.x), g.rdz, g);
  vz.y = v_plain<R>(VZ.y, __fsub_rn(Pc.y, Pzm.y), g.rdz, g);
  vz.z = v_plain<R>(VZ.z, __fsub_rn(Pc.z, Pzm.z), g.rdz, g);
  vz.w = v_plain<R>(VZ.w, __fsub_rn(Pc.w, Pzm.w), g.rdz, g);
  if (MASK) {
    vx.x = (nib & 0x2u) ? vx.x : VX.x;
    vx.y = (nib & 0x20u) ? vx.y : VX.y;
    vx.z = (nib & 0x200u) ? vx.z : VX.z;
    vx.w = (nib & 0x2000u) ? vx.w : VX.w;
    vy.x = (nib & 0x4u) ? vy.x : VY.x;
    vy.y = (nib & 0x40u) ? vy.y : VY.y;
    vy.z = (nib & 0x400u) ? vy.z : VY.z;
    vy.w = (nib & 0x4000u) ? vy.w : VY.w;
    vz.x = (nib & 0x8u) ? vz.x : VZ.x;
    vz.y = (nib & 0x80u) ? vz.y : VZ.y;
    vz.z = (nib & 0x800u) ? vz.z : VZ.z;
    vz.w = (nib & 0x8000u) ? vz.w : VZ.w;
  }
}

// ---------------------------------------------------------------------------
// The step kernel.  One CTA per work item {solve, y tile | x tile << 16, z0,
// z1}: a tile of ty <= 7 rows j0..j0+ty-1 and the kXT = 64 cells
// xb..xb+63 of one solve, and the planes z0..z1-1.  blockDim = (32, 4): warp
// w holds the 4 quads 4w..4w+3 (16 cells) of all 8 tile rows
// r = j - j0 + 1 = 0..7 (lane = 4r + quad).  Row r = 0 is the halo row
// j0-1, whose new P the Vy update of row j0 needs: it is recomputed, not
// exchanged.  The lanes of quad 0 also recompute the halo column x = xb-1
// (for Vx at xb).  With this shape the x-slab quads of a grid sit in one
// warp of each x-edge tile and the tiles between hold none, so few warps
// take the CPML branch and few CTAs wait for such a warp at their barrier.
// Per plane, after a prologue plane z0-1 (new P only, for Vz at z0) when
// z0 > 0:
//   loads  : P, Vx, Vy of plane k and Vz of plane k+1 (Vz of plane k and the
//            new P of plane k-1 are carried in registers), 128-bit, coalesced;
//   P      : new P into a double-buffered shared plane; barrier;
//   q      : injection/recording on P (only planes with entries; barrier);
//   V      : Vx/Vy/Vz from the new P (x-1 and y-1 neighbours from shared
//            memory);
//   f      : injection/recording on V (only planes with entries: staged in
//            shared memory between two barriers);
//   stores : 128-bit stores of the four channels and the rigid mirrors.
// A warp whose quads are all plain for this plane (the bulk of the grid)
// takes the plain functions (warp-uniform branch); the rest the general
// ones.  Several CTAs per SM keep enough independent warps in flight to
// cover the latency of the float/double chains and of HBM.
// ---------------------------------------------------------------------------
constexpr int kMaxTy = 7;           // rows per tile (plus the halo row: 8 per warp)
constexpr int kXT = 64;             // cells per x tile (4 warps)
constexpr int kPnPitch = kXT + 4;   // shared new-P row: [3] = halo column, [4..] = cells
constexpr int kStepThreads = 32 * kXT / 16;  // warps of 4 quads x 8 rows

// One stage: P, Vx, Vy of a plane ([3][ty+2][kStageW]) and, from the next
// 128-B boundary on (TMA destinations must be 128-B aligned), Vz of the next
// plane ([ty+2][kStageW]).
__host__ __device__ constexpr int stage_vz_offset(int cst) { return (3 * cst + 31) / 32 * 32; }
constexpr int kStageFloats =
    (stage_vz_offset((kMaxTy + 2) * kStageW) + (kMaxTy + 2) * kStageW + 31) / 32 * 32;
// Polls of a staged plane's bounded wait: a plane lands within microseconds,
// so a limit far below kWaitLimit keeps a lost copy from stalling the GPU
constexpr uint32_t kStepWaitLimit = 1u << 20;
static_assert((kStageFloats * 4) % 128 == 0, "stages stay 128-B aligned");
static_assert((stage_vz_offset(5 * kStageW) * 4) % 128 == 0, "Vz boxes start 128-B aligned");

template <typename R>
__device__ __forceinline__ void step_item(const StepParams& p, const SolveDev& S, int4 item, int it,
                                          float* sPn, float* sV, const float* co, float* ring,
                                          uint64_t* rbar) {
  const int lane = threadIdx.x, wid = threadIdx.y;
  const int tid = wid * 32 + lane, nthr = blockDim.x * blockDim.y;
  const int nx = S.nx, ny = S.ny, nz = S.nz, nxp = S.nxp, ty = S.ty, npml = S.npml;
  const int T = item.y & 0xFFFF, X = item.y >> 16;
  const int j0 = T * ty, xb = X * kXT;
  // this thread's tile row r (0 = halo row) and quad qx; its warp's quads
  const int qx = 4 * wid + (lane & 3), r = lane >> 2;
  const int wq0 = 4 * wid, wnq = 4, wr0 = 0, wnr = kMaxTy + 1;
  const int j = j0 - 1 + r, x0 = xb + 4 * qx;
  const bool row_ok = r <= ty && j >= 0 && j < ny;
  const bool act = row_ok && x0 < nxp;  // this thread updates a quad
  const bool vrow = act && r >= 1;      // ... and owns it (velocity update, stores)
  const int rb = (it - S.it_first) & 1, wb = rb ^ 1;
  const long long cs = S.chan_stride, plane = (long long)ny * nxp;
  float* fout = S.field + wb * S.buf_stride;
  const bool has_mask = (S.flags & SF_MASK) != 0;
  const bool pcp = (S.flags & SF_PCPML) != 0, vcp = (S.flags & SF_VCPML) != 0;
  Sc<R> g;
  g.fq = Arith<R>::fq(S);
  g.fv = Arith<R>::fv(S);
  g.rdx = Arith<R>::rdx(S);
  g.rdy = Arith<R>::rdy(S);
  g.rdz = Arith<R>::rdz(S);
  RowCtx rc;
  rc.nx = nx;
  rc.ny = ny;
  rc.nz = nz;
  rc.npml = npml;
  rc.nxp = nxp;
  rc.j = j;
  rc.rb = rb;
  rc.wb = wb;
  rc.pcpml = pcp;
  rc.vcpml = vcp;
  // warp-uniform: do all of the warp's rows and x cells take the plain P
  // (and, rows >= 1, V) updates?  The plane is checked per plane below.
  bool wplain_rx;
  {
    const int wj0 = j0 - 1 + wr0, wj1 = wj0 + wnr - 1;  // rows: P on all, V from wj0 + 1
    const int wx0 = xb + 4 * wq0, wx1 = wx0 + 4 * wnq - 1;
    const int p_xmin = pcp ? npml : 0, p_xmax = pcp ? min(nx - 2, nx - npml - 1) : nx - 2;
    const int v_xmin = vcp ? npml + 1 : 1, v_xmax = vcp ? nx - npml - 2 : nx - 1;
    bool ok = wr0 + wnr - 1 <= ty && wj0 >= 0 && wx1 < nxp;
    ok = ok && wj1 < ny - 1 && (!pcp || (wj0 >= npml && wj1 < ny - npml));
    ok = ok && wx0 >= p_xmin && wx1 <= p_xmax;
    ok = ok && wj0 + 1 >= 1 && (!vcp || (wj0 + 1 > npml && wj1 < ny - npml - 1));
    ok = ok && wx0 >= v_xmin && wx1 <= v_xmax;
    wplain_rx = ok;
  }
  const long long rowoff = (long long)(row_ok ? j : 0) * nxp + x0;
  const int pq = r * kPnPitch + 4 + 4 * qx;  // this quad in a shared new-P plane
  const int z0 = item.z, z1 = item.w;
  const int kfirst = z0 > 0 ? z0 - 1 : z0;
  // The stage of plane k, staged by TMA into a ring of kStepRing slots, holds
  // P, Vx, Vy of plane k and Vz of plane k+1 (channel slot 3; not loaded for
  // k = nz-1, where the loop supplies the zeros itself), rows j0-1 .. j0+ty,
  // x = xb-4 .. xb+67, zero outside the grid.  Vz of plane k is carried in
  // registers from the previous stage.
  const int cst = (ty + 2) * kStageW;         // channel stride in a stage
  const int vzo = stage_vz_offset(cst);       // Vz of the next plane in a stage
  const int so = r * kStageW + 4 + 4 * qx;    // this quad in a stage channel
  const char* maps = static_cast<const char*>(S.fmap) + rb * 256;  // {P,Vx,Vy box; Vz box}
  auto slot_of = [&](int k) { return (k - kfirst) % kStepRing; };
  auto issue = [&](int k) {  // one thread
    const int sl = slot_of(k);
    fence_proxy_async_smem();  // the slot was last read through the generic proxy
    const uint32_t bar = smem_u32(rbar + sl);
    const bool vz = k + 1 < nz;
    mbar_expect_tx(bar, (uint32_t)((vz ? 16 : 12) * cst));
    float* dst = ring + sl * kStageFloats;
    tma_load_4d(smem_u32(dst), maps, xb - 4, j0 - 1, k, 0, bar);
    if (vz) tma_load_4d(smem_u32(dst + vzo), maps + 128, xb - 4, j0 - 1, k + 1, 3, bar);
  };
  auto wait = [&](int k) {
    const int u = k - kfirst;
    if (!mbar_wait(smem_u32(rbar + u % kStepRing), (uint32_t)(u / kStepRing) & 1u, kStepWaitLimit))
      atomicOr(S.err, 4);  // reported as ADF_E_TIMEOUT; the values read are wrong
  };
  if (tid == 0)
    for (int k = kfirst; k < min(z1, kfirst + kStepRing); ++k) issue(k);
  // Vz of plane kfirst (the stages carry the next plane's), and of the halo
  // column for its single-cell update
  float4 Z0 = make_float4(0.f, 0.f, 0.f, 0.f), Pzm = Z0;
  const bool hcol = qx == 0 && r >= 1 && row_ok && xb > 0;
  float Zh = 0.f;
  {
    const float* vz0 = S.field + rb * S.buf_stride + 3 * cs + kfirst * plane + rowoff;
    if (act) Z0 = ldg4(vz0);
    if (hcol) Zh = __ldg(vz0 - 1);
  }
  const int* tp = S.tp_off + (long long)T * nz * 4;
  for (int k = kfirst; k < z1; ++k) {
    const bool prologue = k < z0;
    rc.k = k;
    float* pn = sPn + (k & 1) * (kMaxTy + 1) * kPnPitch;
    const float* st = ring + slot_of(k) * kStageFloats;
    wait(k);
    const int off0 = __ldg(tp + 4 * k), off1 = __ldg(tp + 4 * k + 1), off4 = __ldg(tp + 4 * k + 4);
    const bool pplane = k != nz - 1 && (!pcp || (k >= npml && k < nz - npml));
    const bool vplane = k >= 1 && (!vcp || (k > npml && k < nz - npml - 1));
    const bool wplain = wplain_rx && pplane && (prologue || vplane);
    float4 Pn = make_float4(0.f, 0.f, 0.f, 0.f), X4 = Pn, Y0 = Pn, Z1 = Pn;
    uint32_t nib = 0xFFFFu;
    if (act) {
      const float4 P4 = ld4(st + so);
      X4 = ld4(st + cst + so);
      Y0 = ld4(st + 2 * cst + so);
      const float X5 = st[cst + so + 4];
      const float4 Y1 = ld4(st + 2 * cst + so + kStageW);
      Z1 = k + 1 < nz ? ld4(st + vzo + so) : Pn;
      if (has_mask)
        nib = (__ldg(S.mask_bits + ((long long)k * ny + j) * S.mw + (x0 >> 3)) >> ((x0 & 4) * 4)) &
              0xFFFFu;
      if (wplain)
        Pn = has_mask ? p_plain_quad<R, true>(g, P4, X4, X5, Y0, Y1, Z0, Z1, nib)
                      : p_plain_quad<R, false>(g, P4, X4, X5, Y0, Y1, Z0, Z1, nib);
      else
        Pn = p_update_quad<R>(S, rc, g, co, x0, vrow && !prologue, P4, X4, X5, Y0, Y1, Z0, Z1, nib);
      st4(pn + pq, Pn);
    }
    if (hcol) {
      const float Zh1 = k + 1 < nz ? st[vzo + so - 1] : 0.f;
      pn[pq - 1] = p_update_cell<R>(S, rc, g, co, st, Zh, Zh1, so - 1, cst, xb - 1);
      Zh = Zh1;
    }
    __syncthreads();
    // every read of plane k's stage is done: refill its slot
    if (tid == 0 && k + kStepRing < z1) issue(k + kStepRing);
    // ---- q channel: inject/record on the new P (forward.jl:92) ----
    if (off0 < off1) {
      apply_entries(S, off0, off1, 0, nxp, xb - 1, xb + kXT, xb, !prologue, it, tid, nthr,
                    [&](int rr, int x) { return pn + rr * kPnPitch + (x - xb + 4); });
      __syncthreads();
      if (act) Pn = ld4(pn + pq);
    }
    if (!prologue) {
      float4 vx = Pn, vy = Pn, vz = Pn;
      if (vrow) {
        const float Pxm = pn[pq - 1];
        const float4 Pym = ld4(pn + pq - kPnPitch);
        if (wplain) {
          if (has_mask)
            v_plain_quad<R, true>(g, Pn, Pxm, Pym, Pzm, X4, Y0, Z0, nib, vx, vy, vz);
          else
            v_plain_quad<R, false>(g, Pn, Pxm, Pym, Pzm, X4, Y0, Z0, nib, vx, vy, vz);
        } else {
          v_update_quad<R>(S, rc, g, co, x0, Pn, Pxm, Pym, Pzm, X4, Y0, Z0, nib, vx, vy, vz);
        }
      }
      // ---- f channel: inject/record on the new V (forward.jl:111-115) ----
      if (off1 < off4) {
        float* sVx = sV;
        float* sVy = sV + kMaxTy * kXT;
        float* sVz = sV + 2 * kMaxTy * kXT;
        const int so = (r - 1) * kXT + 4 * qx;
        if (vrow) {
          st4(sVx + so, vx);
          st4(sVy + so, vy);
          st4(sVz + so, vz);
        }
        __syncthreads();
        for (int c = 1; c <= 3; ++c) {
          const int b = __ldg(tp + 4 * k + c), e = __ldg(tp + 4 * k + c + 1);
          if (b < e)
            apply_entries(S, b, e, c, nxp, xb, xb + kXT, xb, true, it, tid, nthr,
                          [&](int rr, int x) {
                            return sV + (c - 1) * kMaxTy * kXT + (rr - 1) * kXT + (x - xb);
                          });
        }
        __syncthreads();
        if (vrow) {
          vx = ld4(sVx + so);
          vy = ld4(sVy + so);
          vz = ld4(sVz + so);
        }
      }
      if (vrow) {
        float* o = fout + k * plane + rowoff;
        stcs4(o, Pn);
        stcs4(o + cs, vx);
        // rigid mirrors (forward.jl:134-137): Vy[:,1,:] = -Vy[:,2,:], Vz[:,:,1] = -Vz[:,:,2]
        if (j != 0) stcs4(o + 2 * cs, vy);
        if (j == 1) st4(o + 2 * cs - nxp, neg4(vy));
        if (k != 0) stcs4(o + 3 * cs, vz);
        if (k == 1) st4(o + 3 * cs - plane, neg4(vz));
      }
    }
    Pzm = Pn;
    Z0 = Z1;
  }
}

// Shared memory: the staged-plane ring (dynamic, kStepRing * kStageFloats
// floats) plus the new-P planes, the f-channel staging and the descriptor:
// 33.4 KB per CTA; five CTAs per SM (the register budget: 102 per thread,
// no spills; six CTAs at 80 registers spill and measured slower).
#ifndef ADF_STEP_CTAS_PER_SM
#define ADF_STEP_CTAS_PER_SM 5
#endif
constexpr int kStepCtasPerSm = ADF_STEP_CTAS_PER_SM;  // register budget: 65536 / (128 x this)
// (+128 B so that the ring can start on a 128-B boundary, as TMA destinations must)
constexpr size_t kStepDynSmem = sizeof(float) * kStepRing * kStageFloats + 128;

__global__ void __launch_bounds__(kStepThreads, kStepCtasPerSm) adf_fdtd_step_kernel(const StepParams p) {
  extern __shared__ __align__(128) float dyn_smem[];
  float* ring = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(dyn_smem) + 127) &
                                         ~static_cast<uintptr_t>(127));
  __shared__ __align__(8) uint64_t rbar[kStepRing];
  __shared__ __align__(16) float sPn[2 * (kMaxTy + 1) * kPnPitch];
  __shared__ __align__(16) float sV[3 * kMaxTy * kXT];
  __shared__ float s_co[kMaxCoef];
  __shared__ __align__(16) SolveDev S;  // the solve descriptor, read in the hot loop
  const int4 item = p.items[blockIdx.x];
  const SolveDev& G = p.solves[item.x];
  const int it = G.it_base + p.step;
  if (it > G.it_stop) return;
  const int tid = threadIdx.y * 32 + threadIdx.x, nthr = blockDim.x * blockDim.y;
  {
    const int* src = reinterpret_cast<const int*>(&G);
    int* dst = reinterpret_cast<int*>(&S);
    for (int w = tid; w < (int)(sizeof(SolveDev) / 4); w += nthr) dst[w] = src[w];
    const int ncoef = 8 * G.npml + 4;
    for (int w = tid; w < ncoef; w += nthr) s_co[w] = G.coef[w];
    if (tid == 0) {
      for (int q = 0; q < kStepRing; ++q) mbar_init(smem_u32(rbar + q), 1);
      fence_mbar_init();
    }
  }
  __syncthreads();
  if (S.flags & SF_FP32)
    step_item<float>(p, S, item, it, sPn, sV, s_co, ring, rbar);
  else
    step_item<double>(p, S, item, it, sPn, sV, s_co, ring, rbar);
}

// Per-step trace assembly (derivatives.jl:51-56 record sums in corner order,
// v2vn! :85-90, vn2v! :92-97 into row it+1).
__global__ void adf_fdtd_epilogue_kernel(const EpiParams p) {
  const SolveDev& S = p.solves[blockIdx.y];
  const int it = S.it_base + p.step;
  if (it > S.it_stop) return;
  const int ntx = S.ntx;
  const bool gf = (S.flags & SF_GF) != 0;
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
    // vn2v! into row it+1; a GF solve's driven columns get it when the
    // extrapolation has written their vn_src (gf_finish)
    if (S.vn_src && it < S.nt && (!gf || S.gf_col[tx] == 0)) {
      const long long nr = row + ntx;
      const float vs = S.vn_src[nr];
#pragma unroll
      for (int c = 1; c <= 3; ++c) S.src[c][nr] = __fadd_rn(S.src[c][nr], __fmul_rn(vs, d[c]));
    }
  }
}

// Advances it_base of every solve by `by` steps: the last node of a captured
// chunk of steps, so replaying the graph continues where it stopped.
// Completes source o of step it from its summed lags: adds the far lags
// summed at the block's start (block-causal kinds), writes the p_src and
// vn_src samples of row it+1 (extrapolation.jl:215-216, 228-229, 246-247)
// and applies vn2v! to the column.
__device__ __forceinline__ void gf_finish(const SolveDev& S, int o, int it, int step, double sa,
                                          double sb) {
  if (S.gf_rs > 0) {
    const double* pp = S.gf_far + ((long long)o * S.gf_rs * kGfBlock + step % kGfBlock) * 2;
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
  if (S.gf_col[col] == o + 1) {  // vn2v! of the column (derivatives.jl:92-97), once
    const long long nr = (long long)it * S.ntx + col;
    const float* d = S.dir + 4 * col;
#pragma unroll
    for (int c = 1; c <= 3; ++c) S.src[c][nr] = __fadd_rn(S.src[c][nr], __fmul_rn(ps, d[c]));
  }
}

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
// whose partial sums the reduce kernel adds in a fixed order; with one block
// per source (ks = 1) that block completes the source itself.  Rows before
// `it` of pin come from gf_pin; row `it` is formed here and block 0 files it.
__global__ void __launch_bounds__(256, 4) adf_gf_extrapolate_kernel(const EpiParams p) {
  const SolveDev& S = p.solves[blockIdx.y];
  const int it = S.it_base + p.step;
  if (it > S.it_stop || it >= S.nt || !(S.flags & SF_GF)) return;
  const int ks = S.gf_ks;
  const int o = blockIdx.x / ks, part = blockIdx.x - (blockIdx.x / ks) * ks;
  if (o >= S.gf_nout) return;
  const int nt = S.nt, ntx = S.ntx, ngf = S.gf_nt, n1 = S.gf_n1, nin = S.gf_nin;
  const int kind = S.gf_kind;
  // lags 0..T-1 (T = min(it, ngf)); with blocking only 0..b, b = this step's
  // place in its block, the older lags coming from adf_gf_far_kernel
  const int T = S.gf_rs > 0 ? min(min(it, ngf), p.step % kGfBlock + 1) : min(it, ngf);
  const int t0 = it - T;  // 0-based row of tt = 1
  const long long cur = (long long)(it - 1) * ntx;
  auto pin_now = [&](int r) {
    const int col = S.gf_irec[r];
    return ((double)S.rec[0][cur + col] - (double)S.vn_rec[cur + col] * S.gf_z0) / 2.0;
  };
  double a = 0.0, b = 0.0;
  if (S.gf_near) {
    // blocked kinds (one block per source): lags 0..T-1 <= b from the
    // near-lag copy and the history ring, both receiver-major, so every lag
    // is one coalesced row of each; thread t sums receivers t, t+256, ...
    // Block 0 files row it-1 into the history and the ring; the other rows
    // come from earlier launches.
    const int nl = S.gf_nl;
    const float* g0 = S.gf_near + (long long)o * nl * nin;
    const float* g1 = g0 + (long long)S.gf_nout * nl * nin;
    for (int r = threadIdx.x; r < nin; r += blockDim.x) {
      const double h0 = pin_now(r);
      if (blockIdx.x == 0) {
        S.gf_pin[(long long)r * nt + (it - 1)] = h0;
        S.gf_ring[(long long)((it - 1) % kGfRing) * nin + r] = h0;
      }
      a = __fma_rn((double)g0[r], h0, a);
      b = __fma_rn((double)g1[r], h0, b);
#pragma unroll 4
      for (int lag = 1; lag < T; ++lag) {
        const double h = S.gf_ring[(long long)((it - 1 - lag) % kGfRing) * nin + r];
        a = __fma_rn((double)g0[(long long)lag * nin + r], h, a);
        b = __fma_rn((double)g1[(long long)lag * nin + r], h, b);
      }
    }
  } else {
  if (blockIdx.x == 0 && kind != ADF_GF_PV_FROM_PV_)
    for (int r = threadIdx.x; r < nin; r += blockDim.x)
      S.gf_pin[(long long)r * nt + (it - 1)] = pin_now(r);
  const int rb = (int)((long long)nin * part / ks), re = (int)((long long)nin * (part + 1) / ks);
  // (r, tt) walk over this block's receivers, tt fastest: contiguous tensor
  // and pin reads, the index stepped instead of divided.  GF_U elements per
  // round: all their loads are issued before the first is accumulated, so
  // each thread keeps GF_U loads in flight; the accumulation order of a
  // thread is the walk order either way.
  constexpr int GF_U = 4;
  int r = rb + (int)threadIdx.x / T, tt = (int)threadIdx.x - ((int)threadIdx.x / T) * T;
  const int step_r = (int)blockDim.x / T, step_t = (int)blockDim.x - step_r * T;
  const long long so = kind == ADF_GF_PV_FROM_PIN_ ? (long long)ngf * o : (long long)ngf * n1 * o;
  const long long sr = kind == ADF_GF_PV_FROM_PIN_ ? (long long)ngf * n1 : (long long)ngf;
  while (r < re) {
    int ru[GF_U], tu[GF_U];
#pragma unroll
    for (int u = 0; u < GF_U; ++u) {
      ru[u] = r;
      tu[u] = tt;
      r += step_r;
      tt += step_t;
      if (tt >= T) {
        tt -= T;
        ++r;
      }
    }
    if (kind == ADF_GF_PV_FROM_PV_) {
      float g0[GF_U], g1[GF_U], g2[GF_U], g3[GF_U], pt[GF_U], vt[GF_U];
#pragma unroll
      for (int u = 0; u < GF_U; ++u) {
        if (ru[u] < re) {
          // tensor element [T-tt, ., .] (1-based lag) for this receiver and output
          const long long g = (long long)(T - 1 - tu[u]) + so + sr * ru[u];
          const int col = S.gf_irec[ru[u]];
          const long long e = (long long)(t0 + tu[u]) * ntx + col;
          g0[u] = S.gf_t[0][g];
          g1[u] = S.gf_t[1][g];
          g2[u] = S.gf_t[2][g];
          g3[u] = S.gf_t[3][g];
          pt[u] = S.rec[0][e];
          vt[u] = S.vn_rec[e];
        }
      }
#pragma unroll
      for (int u = 0; u < GF_U; ++u) {
        if (ru[u] < re) {
          const float ps = __fadd_rn(__fmul_rn(g1[u], pt[u]), __fmul_rn(g0[u], vt[u]));
          const float vs = __fadd_rn(__fmul_rn(g3[u], pt[u]), __fmul_rn(g2[u], vt[u]));
          a = __dadd_rn(a, (double)ps);
          b = __dadd_rn(b, (double)vs);
        }
      }
    } else {
      float g0[GF_U], g1[GF_U];
      double pin[GF_U];
#pragma unroll
      for (int u = 0; u < GF_U; ++u) {
        if (ru[u] < re) {
          const long long g = (long long)(T - 1 - tu[u]) + so + sr * ru[u];
          const int row = t0 + tu[u];
          g0[u] = S.gf_t[0][g];
          g1[u] = S.gf_t[1][g];
          pin[u] = row == it - 1 ? pin_now(ru[u]) : S.gf_pin[(long long)ru[u] * nt + row];
        }
      }
#pragma unroll
      for (int u = 0; u < GF_U; ++u) {
        if (ru[u] < re) {
          a = __dadd_rn(a, __dmul_rn((double)g0[u], pin[u]));
          b = __dadd_rn(b, __dmul_rn((double)g1[u], pin[u]));
        }
      }
    }
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
    if (ks == 1) {
      gf_finish(S, o, it, p.step, sa, sb);
    } else {
      double* pp = S.gf_part + ((long long)o * ks + part) * 2;
      pp[0] = sa;
      pp[1] = sb;
    }
  }
}

// Far-lag part of the in-loop GF extrapolation (extrapolation.jl:139-170),
// block-causal form.  For the block of kGfBlock steps it0 .. it0+B-1 that
// starts at this launch-step, step it0+b needs lags 0 .. T_b-1 of the map
// (T_b = min(it0+b, ngf)).  Lags b+1 .. T_b-1 read input-history rows
// it0-1+b-lag <= it0-2, all complete before the block starts, so they are
// summed here once for the whole block: a contraction over (receiver, lag)
// of the block's 32 steps x 32 sources, which reads each tensor slice once
// per block instead of once per step.  Lags 0..b, whose rows appear during
// the block, stay in adf_gf_extrapolate_kernel.  FP64 fused multiply-adds;
// one partial per (source, receiver split, step), added in split order by
// adf_gf_reduce_kernel.  Input-history kinds only.
constexpr int kGfLC = 32;  // lags per staged chunk
constexpr int kGfOT = 64;  // sources per tile (two per thread)
__global__ void __launch_bounds__(256) adf_gf_far_kernel(const EpiParams p) {
  const SolveDev& S = p.solves[blockIdx.y];
  const int it0 = S.it_base + p.step;
  if (S.gf_rs <= 0 || it0 > S.it_stop || it0 >= S.nt || !(S.flags & SF_GF) || (S.flags & SF_GF_TC))
    return;  // (tensor-core solves: adf_gf_far_tc_kernel)
  const int rsn = S.gf_rs, nout = S.gf_nout;
  const int ot = blockIdx.x / rsn, rsi = blockIdx.x - ot * rsn;
  if (ot * kGfOT >= nout) return;
  const int nt = S.nt, ngf = S.gf_nt, n1 = S.gf_n1, nin = S.gf_nin;
  const bool pv = S.gf_kind == ADF_GF_PV_FROM_PIN_;
  const int r0 = (int)((long long)nin * rsi / rsn), r1 = (int)((long long)nin * (rsi + 1) / rsn);
  // thread: sources ol and ol+32 of the tile, steps b = bg + 8q of the block
  const int ol = (int)threadIdx.x & 31, bg = (int)threadIdx.x >> 5;
  __shared__ double sG[2][kGfLC][kGfOT + 1];   // lag-major, Float64, padded against conflicts
  __shared__ double sH[kGfLC + kGfBlock - 1];  // history rows of the chunk
  double acc[2][2][4];
#pragma unroll
  for (int t = 0; t < 2; ++t)
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[t][h][q] = 0.0;
  const int lag_hi = min(it0 + kGfBlock - 1, ngf) - 1;  // largest lag any step of the block uses
  for (int r = r0; r < r1; ++r) {
    const double* hist = S.gf_pin + (long long)r * nt;
    for (int l0 = 1; l0 <= lag_hi; l0 += kGfLC) {
      __syncthreads();  // the previous chunk has been used
      for (int i = threadIdx.x; i < kGfOT * kGfLC; i += blockDim.x) {
        const int oo = i / kGfLC, ll = i - oo * kGfLC;  // lag fastest: coalesced reads
        const int lag = l0 + ll, og = ot * kGfOT + oo;
        float v0 = 0.f, v1 = 0.f;
        if (lag <= lag_hi && og < nout) {
          const long long col = pv ? (long long)ngf * (og + (long long)n1 * r)
                                   : (long long)ngf * (r + (long long)n1 * og);
          v0 = S.gf_t[0][col + lag];
          v1 = S.gf_t[1][col + lag];
        }
        sG[0][ll][oo] = (double)v0;
        sG[1][ll][oo] = (double)v1;
      }
      // rows it0-1+b-lag of this chunk lie in [hlo, hlo + kGfLC + kGfBlock - 2]
      const int hlo = it0 - l0 - kGfLC;
      for (int i = threadIdx.x; i < kGfLC + kGfBlock - 1; i += blockDim.x) {
        const int row = hlo + i;
        sH[i] = (row >= 0 && row < nt) ? hist[row] : 0.0;
      }
      __syncthreads();
      const bool full = l0 >= kGfBlock && l0 + kGfLC <= min(it0, ngf);
      for (int ll = 0; ll < kGfLC; ++ll) {
        const int lag = l0 + ll;
        const double g00 = sG[0][ll][ol], g01 = sG[0][ll][ol + 32];
        const double g10 = sG[1][ll][ol], g11 = sG[1][ll][ol + 32];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int b = bg + 8 * q;
          // past every step of the block and below every step's T, or checked
          if (full || (lag > b && lag < min(it0 + b, ngf))) {
            const double h = sH[b + kGfLC - 1 - ll];
            acc[0][0][q] = __fma_rn(g00, h, acc[0][0][q]);
            acc[0][1][q] = __fma_rn(g01, h, acc[0][1][q]);
            acc[1][0][q] = __fma_rn(g10, h, acc[1][0][q]);
            acc[1][1][q] = __fma_rn(g11, h, acc[1][1][q]);
          }
        }
      }
    }
  }
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int o = ot * kGfOT + ol + 32 * h;
    if (o >= nout) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      double* pp = S.gf_far + (((long long)o * rsn + rsi) * kGfBlock + bg + 8 * q) * 2;
      pp[0] = acc[0][h][q];
      pp[1] = acc[1][h][q];
    }
  }
}

// Sums the far-lag partials of each (source, step of the block) over the
// receiver splits, in split order, into split 0's slot.
__global__ void adf_gf_far_combine_kernel(const EpiParams p) {
  const SolveDev& S = p.solves[blockIdx.y];
  const int it0 = S.it_base + p.step;
  if (S.gf_rs <= 0 || it0 > S.it_stop || it0 >= S.nt || !(S.flags & SF_GF)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // (source, step of the block)
  if (i >= S.gf_nout * kGfBlock) return;
  const int o = i / kGfBlock, b = i - o * kGfBlock;
  double sa = 0.0, sb = 0.0;
  for (int k = 0; k < S.gf_rs; ++k) {
    const double* pp = S.gf_far + (((long long)o * S.gf_rs + k) * kGfBlock + b) * 2;
    sa = __dadd_rn(sa, pp[0]);
    sb = __dadd_rn(sb, pp[1]);
  }
  double* out = S.gf_far + ((long long)o * S.gf_rs * kGfBlock + b) * 2;
  out[0] = sa;
  out[1] = sb;
}

// Adds each source's partial sums in split order and writes its p_src and
// vn_src samples of row it+1 (solves with more than one block per source).
__global__ void adf_gf_reduce_kernel(const EpiParams p) {
  const SolveDev& S = p.solves[blockIdx.y];
  const int it = S.it_base + p.step;
  if (it > S.it_stop || it >= S.nt || !(S.flags & SF_GF) || S.gf_ks == 1) return;
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= S.gf_nout) return;
  double sa = 0.0, sb = 0.0;
  for (int k = 0; k < S.gf_ks; ++k) {
    const double* pp = S.gf_part + ((long long)o * S.gf_ks + k) * 2;
    sa = __dadd_rn(sa, pp[0]);
    sb = __dadd_rn(sb, pp[1]);
  }
  gf_finish(S, o, it, p.step, sa, sb);
}

__global__ void adf_advance_kernel(SolveDev* solves, int n, int by) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) solves[i].it_base += by;
}

cudaError_t launch_advance(SolveDev* solves, int n, int by, cudaStream_t s) {
  adf_advance_kernel<<<(n + 127) / 128, 128, 0, s>>>(solves, n, by);
  return cudaGetLastError();
}

cudaError_t launch_step(const StepParams& p, int grid, int max_ty, cudaStream_t s) {
  (void)max_ty;  // the block always holds kMaxTy rows; shorter tiles idle the rest
  adf_fdtd_step_kernel<<<grid, dim3(32, kXT / 16), kStepDynSmem, s>>>(p);
  return cudaGetLastError();
}

int step_max_ty() { return kMaxTy; }
cudaError_t step_ctas_per_sm(int* n) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, adf_fdtd_step_kernel, kStepThreads,
                                                       kStepDynSmem);
}
int step_x_tile() { return kXT; }

cudaError_t launch_gf_extrapolate(const EpiParams& p, int max_blocks, int max_nsrc, bool reduce,
                                  cudaStream_t s) {
  // (source, receiver split) blocks of the largest map in the batch, then,
  // when some solve splits its receivers, the fixed-order reduction
  adf_gf_extrapolate_kernel<<<dim3(max_blocks > 0 ? max_blocks : 1, p.n_solves), 256, 0, s>>>(p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !reduce) return e;
  adf_gf_reduce_kernel<<<dim3((max_nsrc + 127) / 128, p.n_solves), 128, 0, s>>>(p);
  return cudaGetLastError();
}

// Copies lags 0..nl-1 of the two tensors of an input-history map into the
// receiver-major near-lag layout [2][n_out][nl][n_in] (set-up, once per map).
__global__ void adf_gf_near_pack_kernel(const float* t0, const float* t1, float* near, int kind,
                                        int ngf, int n1, int nout, int nin, int nl) {
  const long long per = (long long)nout * nl * nin;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 2 * per;
       i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i / per);
    long long q = i - k * per;
    const int r = (int)(q % nin);
    q /= nin;
    const int lag = (int)(q % nl);
    const int o = (int)(q / nl);
    const long long g = kind == ADF_GF_PV_FROM_PIN_
                            ? lag + (long long)ngf * (o + (long long)n1 * r)
                            : lag + (long long)ngf * (r + (long long)n1 * o);
    near[i] = (k == 0 ? t0 : t1)[g];
  }
}

cudaError_t launch_gf_near_pack(const SolveDev& d, float* near, cudaStream_t s) {
  adf_gf_near_pack_kernel<<<4 * 148, 256, 0, s>>>(d.gf_t[0], d.gf_t[1], near, d.gf_kind, d.gf_nt,
                                                  d.gf_n1, d.gf_nout, d.gf_nin, d.gf_nl);
  return cudaGetLastError();
}

cudaError_t launch_gf_far(const EpiParams& p, int max_blocks, int max_nsrc, cudaStream_t s) {
  if (max_blocks > 0) {  // 0: every blocked solve of the batch is on the tensor cores
    adf_gf_far_kernel<<<dim3(max_blocks, p.n_solves), 256, 0, s>>>(p);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  adf_gf_far_combine_kernel<<<dim3((max_nsrc * kGfBlock + 255) / 256, p.n_solves), 256, 0, s>>>(p);
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
