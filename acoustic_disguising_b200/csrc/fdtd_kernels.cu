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

namespace adf {

constexpr int NCT = 256;          // consumer threads
constexpr int NCW = NCT / 32;     // consumer warps
constexpr int NTHREADS = NCT + 32;
constexpr int kMaxStages = 8;
constexpr int kPnBufs = 3;
constexpr uint32_t kWaitLimit = 1u << 22;

int consumer_threads() { return NCT; }

// ---------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t a) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after kWaitLimit polls (about a second) so that a
// logic error surfaces as an error code instead of a hung GPU.
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity) {
  for (uint32_t i = 0; i < kWaitLimit; ++i) {
    if (mbar_try_wait(a, parity)) return true;
    if (i >= 8) __nanosleep(64);
  }
  return false;
}
__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* map, uint32_t mbar,
                                            int c0, int c1, int c2, int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(dst),
      "l"((uint64_t)map), "r"(mbar), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
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
// and re-added.  Only the owning tile stores (halo/prologue cells read).
template <typename R>
__device__ __forceinline__ void cpml_step(R& dv, const float* rd, float* wr, long long off,
                                          float a, float b, bool owned) {
  using A = Arith<R>;
  float m = rd[off];
  float bm = __fmul_rn(b, m);
  R nm = A::add(A::cv(bm), A::mul(A::cv(a), dv));
  float mf = A::rn(nm);
  if (owned) wr[off] = mf;
  dv = A::add(dv, A::cv(mf));
}

struct PlaneCtx {
  const float* sP;
  const float* sVx;
  const float* sVy;
  const float* sVz;  // plane k rows, plane k+1 at + R*nxp
  const uint32_t* sM;
  float* pn_cur;
  const float* pn_prev;
  int j0, R, pl, rb, wb;
  bool has_mask;
};

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float f4get(const float4& v, int e) {
  return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w;
}

// Pressure update of one quad (4 cells along x) of row r (global row j0-1+r)
template <typename R>
__device__ __forceinline__ void p_quad(const SolveDev& S, const PlaneCtx& c, int r, int q,
                                       bool owned) {
  using A = Arith<R>;
  const int nxp = S.nxp, nx = S.nx, ny = S.ny, nz = S.nz, npml = S.npml;
  const int x0 = 4 * q;
  const int j = c.j0 - 1 + r;
  const int pl = c.pl;
  const float4 P4 = ld4(c.sP + r * nxp + x0);
  const float4 X4 = ld4(c.sVx + r * nxp + x0);
  const float X5 = (x0 + 4 < nxp) ? c.sVx[r * nxp + x0 + 4] : 0.f;
  const float4 Y0 = ld4(c.sVy + r * nxp + x0);
  const float4 Y1 = ld4(c.sVy + (r + 1) * nxp + x0);
  const float4 Z0 = ld4(c.sVz + r * nxp + x0);
  const float4 Z1 = ld4(c.sVz + (c.R + r) * nxp + x0);
  uint32_t nib = 0xFFFFu;
  if (c.has_mask) nib = (c.sM[r * S.mw + (q >> 1)] >> ((q & 1) * 16)) & 0xFFFFu;
  const R fq = A::fq(S), rdx = A::rdx(S), rdy = A::rdy(S), rdz = A::rdz(S);
  const bool rigid_y = (j == ny - 1), rigid_z = (pl == nz - 1);
  const bool pc = (S.flags & SF_PCPML) != 0;
  float out[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int x = x0 + e;
    const float P = f4get(P4, e);
    const float xa = f4get(X4, e), xb = (e < 3) ? f4get(X4, e + 1) : X5;
    if (x > nx - 2 || (rigid_y && rigid_z)) {  // i = nx plane / (ny,nz) corner: not updated
      out[e] = P;
      continue;
    }
    R dvx = A::mul(A::cv(__fsub_rn(xb, xa)), rdx);
    R dvy, dvz;
    if (rigid_y) {  // update_p! on the plane j = ny (updates.jl:122-136)
      dvy = A::mul(A::cv(__fmul_rn(-2.0f, f4get(Y0, e))), rdy);
      dvz = A::mul(A::cv(__fsub_rn(f4get(Z1, e), f4get(Z0, e))), rdz);
      out[e] = A::rn(A::sub(A::cv(P), A::mul(fq, A::add(A::add(dvx, dvy), dvz))));
      continue;
    }
    if (rigid_z) {  // update_p! on the plane k = nz
      dvy = A::mul(A::cv(__fsub_rn(f4get(Y1, e), f4get(Y0, e))), rdy);
      dvz = A::mul(A::cv(__fmul_rn(-2.0f, f4get(Z0, e))), rdz);
      out[e] = A::rn(A::sub(A::cv(P), A::mul(fq, A::add(A::add(dvx, dvy), dvz))));
      continue;
    }
    dvy = A::mul(A::cv(__fsub_rn(f4get(Y1, e), f4get(Y0, e))), rdy);
    dvz = A::mul(A::cv(__fsub_rn(f4get(Z1, e), f4get(Z0, e))), rdz);
    if (pc) {
      const float* co = S.coef;
      // x slab (getBoundaryIndex(i, nx, npml), derivatives.jl:66-79)
      int side = -1, l = 0;
      if (x < npml) { side = 0; l = x; }
      else if (x >= nx - npml) { side = 1; l = x - (nx - npml); }
      if (side >= 0) {
        long long off = (long long)side * S.psi_p_side[0] + ((long long)pl * ny + j) * npml + l;
        cpml_step<R>(dvx, S.psi_p[0] + c.rb * S.psi_p_buf[0], S.psi_p[0] + c.wb * S.psi_p_buf[0],
                     off, __ldg(co + side * npml + l), __ldg(co + 4 * npml + 2 + side * npml + l),
                     owned);
      }
      side = -1;
      if (j < npml) { side = 0; l = j; }
      else if (j >= ny - npml) { side = 1; l = j - (ny - npml); }
      if (side >= 0) {
        long long off = (long long)side * S.psi_p_side[1] + ((long long)pl * npml + l) * nxp + x;
        cpml_step<R>(dvy, S.psi_p[1] + c.rb * S.psi_p_buf[1], S.psi_p[1] + c.wb * S.psi_p_buf[1],
                     off, __ldg(co + side * npml + l), __ldg(co + 4 * npml + 2 + side * npml + l),
                     owned);
      }
      side = -1;
      if (pl < npml) { side = 0; l = pl; }
      else if (pl >= nz - npml) { side = 1; l = pl - (nz - npml); }
      if (side >= 0) {
        long long off = (long long)side * S.psi_p_side[2] + ((long long)l * ny + j) * nxp + x;
        cpml_step<R>(dvz, S.psi_p[2] + c.rb * S.psi_p_buf[2], S.psi_p[2] + c.wb * S.psi_p_buf[2],
                     off, __ldg(co + side * npml + l), __ldg(co + 4 * npml + 2 + side * npml + l),
                     owned);
      }
    }
    if ((nib >> (4 * e)) & 1u)
      out[e] = A::rn(A::sub(A::cv(P), A::mul(fq, A::add(A::add(dvx, dvy), dvz))));
    else
      out[e] = P;  // coeff = fq * false: the cell is frozen (updates.jl:314-316)
  }
  st4(c.pn_cur + r * nxp + x0, make_float4(out[0], out[1], out[2], out[3]));
}

// Velocity update of one quad of tile row r (global row j0-1+r)
template <typename R>
__device__ __forceinline__ void v_quad(const SolveDev& S, const PlaneCtx& c, int r, int q,
                                       float4& vxo, float4& vyo, float4& vzo) {
  using A = Arith<R>;
  const int nxp = S.nxp, nx = S.nx, ny = S.ny, nz = S.nz, npml = S.npml;
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
  const R fv = A::fv(S), rdx = A::rdx(S), rdy = A::rdy(S), rdz = A::rdz(S);
  const bool vc = (S.flags & SF_VCPML) != 0;
  const float* co = S.coef;
  float ox[4], oy[4], oz[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int x = x0 + e;
    const float pc = f4get(Pc, e);
    const float vx = f4get(VX, e), vy = f4get(VY, e), vz = f4get(VZ, e);
    // Vx over i = 2..nx (update_vx!, updates.jl:192-218)
    if (x == 0 || x >= nx) {
      ox[e] = vx;
    } else {
      const float pm = e > 0 ? f4get(Pc, e - 1) : Pxm;
      R dp = A::mul(A::cv(__fsub_rn(pc, pm)), rdx);
      if (vc) {
        int side = -1, l = 0;
        if (x <= npml) { side = 0; l = x; }
        else if (x >= nx - npml - 1) { side = 1; l = x - (nx - npml - 1); }
        if (side >= 0) {
          long long off = (long long)side * S.psi_v_side[0] + ((long long)pl * ny + j) * nm + l;
          cpml_step<R>(dp, S.psi_v[0] + c.rb * S.psi_v_buf[0], S.psi_v[0] + c.wb * S.psi_v_buf[0],
                       off, __ldg(co + 2 * npml + side * nm + l),
                       __ldg(co + 6 * npml + 2 + side * nm + l), true);
        }
      }
      ox[e] = ((nib >> (4 * e + 1)) & 1u) ? A::rn(A::sub(A::cv(vx), A::mul(fv, dp))) : vx;
    }
    // Vy over j = 2..ny
    if (j == 0 || x >= nx) {
      oy[e] = vy;
    } else {
      R dp = A::mul(A::cv(__fsub_rn(pc, f4get(Pym, e))), rdy);
      if (vc) {
        int side = -1, l = 0;
        if (j <= npml) { side = 0; l = j; }
        else if (j >= ny - npml - 1) { side = 1; l = j - (ny - npml - 1); }
        if (side >= 0) {
          long long off = (long long)side * S.psi_v_side[1] + ((long long)pl * nm + l) * nxp + x;
          cpml_step<R>(dp, S.psi_v[1] + c.rb * S.psi_v_buf[1], S.psi_v[1] + c.wb * S.psi_v_buf[1],
                       off, __ldg(co + 2 * npml + side * nm + l),
                       __ldg(co + 6 * npml + 2 + side * nm + l), true);
        }
      }
      oy[e] = ((nib >> (4 * e + 2)) & 1u) ? A::rn(A::sub(A::cv(vy), A::mul(fv, dp))) : vy;
    }
    // Vz over k = 2..nz
    if (pl == 0 || x >= nx) {
      oz[e] = vz;
    } else {
      R dp = A::mul(A::cv(__fsub_rn(pc, f4get(Pzm, e))), rdz);
      if (vc) {
        int side = -1, l = 0;
        if (pl <= npml) { side = 0; l = pl; }
        else if (pl >= nz - npml - 1) { side = 1; l = pl - (nz - npml - 1); }
        if (side >= 0) {
          long long off = (long long)side * S.psi_v_side[2] + ((long long)l * ny + j) * nxp + x;
          cpml_step<R>(dp, S.psi_v[2] + c.rb * S.psi_v_buf[2], S.psi_v[2] + c.wb * S.psi_v_buf[2],
                       off, __ldg(co + 2 * npml + side * nm + l),
                       __ldg(co + 6 * npml + 2 + side * nm + l), true);
        }
      }
      oz[e] = ((nib >> (4 * e + 3)) & 1u) ? A::rn(A::sub(A::cv(vz), A::mul(fv, dp))) : vz;
    }
  }
  vxo = make_float4(ox[0], ox[1], ox[2], ox[3]);
  vyo = make_float4(oy[0], oy[1], oy[2], oy[3]);
  vzo = make_float4(oz[0], oz[1], oz[2], oz[3]);
}

// interp_trilinear! entries of one (tile, plane, channel) in transceiver
// order per cell: rec += w*f (stored per entry, summed by the epilogue in
// corner order), then f += w*src[it].
__device__ __forceinline__ void process_entries(const SolveDev& S, int b, int e, int chan,
                                                float* cells, bool records, int it) {
  const float* src = S.src[chan] + (long long)(it - 1) * S.src_ntx;
  for (int si = b + (int)threadIdx.x; si < e; si += NCT) {
    const int4 sg = S.seg[si];
    float v = cells[sg.x];
    for (int k = sg.y; k < sg.y + sg.z; ++k) {
      const float w = S.ent_w[k];
      const int slot = S.ent_slot[k];
      if (records && slot >= 0) S.contrib[slot] = __fmul_rn(w, v);
      const int col = S.ent_tx[k];
      if (col >= 0) v = __fadd_rn(v, __fmul_rn(w, src[col]));  // receivers: src == 0
    }
    cells[sg.x] = v;
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

template <typename R>
__device__ bool consume_item(const StepParams& p, const SolveDev& S, int4 item, int it,
                             uint64_t* full, uint64_t* empty, float* ring, float* pn, int& n,
                             volatile int* s_fail) {
  const int rb = (it - S.it_first) & 1;
  const int ty = S.ty, nxp = S.nxp, nq = nxp / 4;
  const int j0 = item.y * ty;
  const int Rr = ty + 2;
  const int reg = slot_region(ty, nxp);
  const int reg2 = round32(2LL * Rr * nxp);
  const int pz0 = item.z > 0 ? item.z - 1 : 0;
  const int tid = threadIdx.x;
  const bool has_mask = (S.flags & SF_MASK) != 0;
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
    c.sVx = base + reg;
    c.sVy = base + 2 * reg;
    c.sVz = base + 3 * reg;
    c.sM = reinterpret_cast<const uint32_t*>(base + 3 * reg + reg2);
    c.pn_cur = pn + (n % kPnBufs) * p.pn_floats;
    c.pn_prev = pn + ((n + kPnBufs - 1) % kPnBufs) * p.pn_floats;
    c.j0 = j0;
    c.R = Rr;
    c.pl = pl;
    c.rb = rb;
    c.wb = rb ^ 1;
    c.has_mask = has_mask;
    // ---- P phase ----
    const int nP = (ty + 1) * nq;
    if (landed) {
      for (int u = tid; u < nP; u += NCT) {
        const int r = u / nq, q = u - r * nq;
        const int j = j0 - 1 + r;
        if (j < 0 || j >= S.ny) continue;
        p_quad<R>(S, c, r, q, !prologue && r >= 1);
      }
    }
    consumer_bar();
    if (*s_fail) {
      if (tid == 0) atomicExch(p.err, KERR_FULL_TIMEOUT);
      return false;
    }
    // ---- Q phase: q-channel inject/record on P (forward.jl:92) ----
    const int tb = (item.y * S.nz + pl) * 4;
    {
      const int b = S.tp_off[tb], e = S.tp_off[tb + 1];
      if (b < e) {
        process_entries(S, b, e, 0, c.pn_cur, !prologue, it);
        consumer_bar();
      }
    }
    if (!prologue) {
      const int fb = S.tp_off[tb + 1], fe = S.tp_off[tb + 4];
      const bool has_f = fb < fe;
      const int nV = ty * nq;
      for (int u = tid; u < nV; u += NCT) {
        const int r = 1 + u / nq, q = u - (r - 1) * nq;
        const int j = j0 - 1 + r;
        if (j >= S.ny) continue;
        float4 vx, vy, vz;
        v_quad<R>(S, c, r, q, vx, vy, vz);
        if (has_f) {  // stage into this slot's own rows (only this thread reads them)
          st4(const_cast<float*>(c.sVx) + r * nxp + 4 * q, vx);
          st4(const_cast<float*>(c.sVy) + r * nxp + 4 * q, vy);
          st4(const_cast<float*>(c.sVz) + r * nxp + 4 * q, vz);
        } else {
          store_outputs(S, c, r, q, ld4(c.pn_cur + r * nxp + 4 * q), vx, vy, vz);
        }
      }
      if (has_f) {
        consumer_bar();
        // ---- F phase: f-channel inject/record (forward.jl:111-115) ----
        for (int ch = 1; ch <= 3; ++ch) {
          const int b = S.tp_off[tb + ch], e = S.tp_off[tb + ch + 1];
          float* cells = const_cast<float*>(ch == 1 ? c.sVx : ch == 2 ? c.sVy : c.sVz);
          if (b < e) process_entries(S, b, e, ch, cells, true, it);
        }
        consumer_bar();
        for (int u = tid; u < nV; u += NCT) {
          const int r = 1 + u / nq, q = u - (r - 1) * nq;
          const int j = j0 - 1 + r;
          if (j >= S.ny) continue;
          store_outputs(S, c, r, q, ld4(c.pn_cur + r * nxp + 4 * q), ld4(c.sVx + r * nxp + 4 * q),
                        ld4(c.sVy + r * nxp + 4 * q), ld4(c.sVz + r * nxp + 4 * q));
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

__global__ void __launch_bounds__(NTHREADS, 2) adf_fdtd_step_kernel(const StepParams p) {
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
      const CUtensorMap* tm = p.tmaps + 3 * item.x;
      if (item.x != cur) {
        tmap_acquire(tm);
        tmap_acquire(tm + 1);
        tmap_acquire(tm + 2);
        cur = item.x;
      }
      const int ty = S.ty, nxp = S.nxp, Rr = ty + 2;
      const int j0 = item.y * ty;
      const int reg = slot_region(ty, nxp);
      const int reg2 = round32(2LL * Rr * nxp);
      const bool has_mask = (S.flags & SF_MASK) != 0;
      const uint32_t bytes = (uint32_t)(5 * Rr * nxp * 4 + (has_mask ? Rr * S.mw * 4 : 0));
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
        mbar_expect_tx(mb, bytes);
        float* base = ring + (long long)slot * p.stage_floats;
        tma_load_5d(smem_u32(base), tm, mb, 0, 0, j0 - 1, pl, 4 * rb + 0);
        tma_load_5d(smem_u32(base + reg), tm, mb, 0, 0, j0 - 1, pl, 4 * rb + 1);
        tma_load_5d(smem_u32(base + 2 * reg), tm, mb, 0, 0, j0 - 1, pl, 4 * rb + 2);
        tma_load_5d(smem_u32(base + 3 * reg), tm + 1, mb, 0, 0, j0 - 1, pl, 4 * rb + 3);
        if (has_mask) tma_load_3d(smem_u32(base + 3 * reg + reg2), tm + 2, mb, 0, j0 - 1, pl);
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
  int n = 0;
  for (int i = blockIdx.x; i < p.n_items; i += gridDim.x) {
    const int4 item = p.items[i];
    const SolveDev& S = p.solves[item.x];
    const int it = S.it_base + p.step;
    if (it > S.it_stop) continue;
    bool ok;
    if (S.flags & SF_FP32)
      ok = consume_item<float>(p, S, item, it, full, empty, ring, pn, n, &s_fail);
    else
      ok = consume_item<double>(p, S, item, it, full, empty, ring, pn, n, &s_fail);
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
    if (S.vn_src && it < S.nt) {
      const long long nr = row + ntx;
      const float vs = S.vn_src[nr];
#pragma unroll
      for (int c = 1; c <= 3; ++c) S.src[c][nr] = __fadd_rn(S.src[c][nr], __fmul_rn(vs, d[c]));
    }
  }
}

// Advances it_base of every solve by `by` steps: the last node of a captured
// chunk of steps, so replaying the graph continues where it stopped.
__global__ void adf_advance_kernel(SolveDev* solves, int n, int by) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) solves[i].it_base += by;
}

cudaError_t launch_advance(SolveDev* solves, int n, int by, cudaStream_t s) {
  adf_advance_kernel<<<(n + 127) / 128, 128, 0, s>>>(solves, n, by);
  return cudaGetLastError();
}

const void* step_kernel_ptr() { return (const void*)adf_fdtd_step_kernel; }

cudaError_t step_kernel_attributes(size_t smem, bool) {
  return cudaFuncSetAttribute(adf_fdtd_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem);
}

cudaError_t launch_step(const StepParams& p, int grid, int block, size_t smem, cudaStream_t s,
                        bool) {
  adf_fdtd_step_kernel<<<grid, block, smem, s>>>(p);
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
