// adf_oracle.cpp -- CPU oracle (test infrastructure only; see adf_oracle.h).
//
// Every function restates one reference routine; the reference file:line is
// given beside it.  Arithmetic follows Julia's promotion rules: the Domain
// scalars (dx, fact_m0, fact_m1) are Float64 while the field, CPML memory,
// CPML coefficients, weights and traces are Float32, so in OR_MODE_PROMOTE
// `(Float32 - Float32) / Float64` is evaluated in double and rounded to
// float only on store.  Build with -ffp-contract=off so that no multiply-add
// is fused (Julia never contracts without @fastmath / muladd).
#include "adf_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <type_traits>
#include <vector>

namespace {

// Static-schedule parallel loop over [b, e) (the reference's Threads backend
// splits the outermost index across threads the same way).
int g_threads = 0;
template <typename F>
void pfor(int64_t b, int64_t e, F&& fn) {
  int64_t n = e - b;
  if (n <= 0) return;
  int nt = g_threads > 0 ? g_threads : (int)std::max(1u, std::thread::hardware_concurrency());
  if (nt > n) nt = (int)n;
  if (nt <= 1) {
    for (int64_t i = b; i < e; ++i) fn(i);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(nt);
  for (int t = 0; t < nt; ++t) {
    int64_t lo = b + n * t / nt, hi = b + n * (t + 1) / nt;
    th.emplace_back([lo, hi, &fn]() {
      for (int64_t i = lo; i < hi; ++i) fn(i);
    });
  }
  for (auto& x : th) x.join();
}

// ---------------------------------------------------------------------------
// Julia Base range arithmetic (StepRangeLen with a twice-precision reference
// and step).  Restated from the published double-double algorithm that Julia's
// base/twiceprecision.jl implements; used by x(d)/xv(d)/t(d) in
// src/simulation.jl:86-100, which masks and transceiver indices depend on.
// ---------------------------------------------------------------------------
struct TP {
  double hi, lo;
};

inline void canonicalize2(double big, double little, double& h, double& l) {
  h = big + little;
  l = (big - h) + little;
}
inline void add12(double x, double y, double& h, double& l) {
  if (std::fabs(y) > std::fabs(x)) std::swap(x, y);
  canonicalize2(x, y, h, l);
}
inline void mul12(double x, double y, double& h, double& l) {
  h = x * y;
  l = std::isfinite(h) ? std::fma(x, y, -h) : h;
}
inline TP tp_div(TP x, TP y) {
  double hi = x.hi / y.hi;
  double uh, ul;
  mul12(hi, y.hi, uh, ul);
  double lo = ((((x.hi - uh) - ul) + x.lo) - hi * y.lo) / y.hi;
  TP r;
  canonicalize2(hi, lo, r.hi, r.lo);
  if (x.hi == 0.0 || !std::isfinite(hi)) r = TP{hi, hi};
  return r;
}
inline TP tp_from_int(__int128 i) {
  double hi = (double)i;
  __int128 rest = i - (__int128)hi;
  TP r;
  canonicalize2(hi, (double)rest, r.hi, r.lo);
  return r;
}
inline double truncbits(double x, int nb) {
  uint64_t u;
  std::memcpy(&u, &x, 8);
  u &= (~(uint64_t)0) << nb;
  std::memcpy(&x, &u, 8);
  return x;
}
inline TP twiceprecision(TP v, int nb) {
  double hi = truncbits(v.hi, nb);
  return TP{hi, (v.hi - hi) + v.lo};
}
inline int top_set_bit(int64_t x) {
  int n = 0;
  while (x > 0) {
    ++n;
    x >>= 1;
  }
  return n;
}
inline int nbitslen(int64_t len, int64_t offset) {
  if (len < 2) return 0;
  int64_t m = std::max(offset - 1, len - offset);
  int v = top_set_bit(m - 1) + 1;
  return std::min(27, v);  // cld(precision(Float64), 2) = 27
}
inline int64_t round_half_even(double x) { return (int64_t)std::nearbyint(x); }

// Continued-fraction rational approximation `rat` (Julia base/twiceprecision.jl)
inline void rat(double x, int64_t& num, int64_t& den) {
  double y = x;
  int64_t a = 1, d = 1, b = 0, c = 0;
  const double m = 16777216.0;  // maxintfloat(Float32, Int)
  while (std::fabs(y) <= m) {
    int64_t f = (int64_t)std::trunc(y);
    y -= (double)f;
    int64_t na = f * a + c, nc = a;
    int64_t nb = f * b + d, nd = b;
    a = na;
    c = nc;
    b = nb;
    d = nd;
    if (!(std::max(std::llabs(a), std::llabs(b)) <= (int64_t)m)) {
      num = c;
      den = d;
      return;
    }
    if ((double)a / (double)b == x) break;
    y = 1.0 / y;
  }
  num = a;
  den = b;
}

struct JRange {
  TP ref, step;
  int64_t len, offset;
  double at(int64_t i) const {  // 1-based, unsafe_getindex
    double u = (double)(i - offset);
    double shift_hi = u * step.hi, shift_lo = u * step.lo;
    double x_hi, x_lo;
    add12(ref.hi, shift_hi, x_hi, x_lo);
    return x_hi + (x_lo + (shift_lo + ref.lo));
  }
};

inline int64_t gcd64(int64_t a, int64_t b) {
  a = std::llabs(a);
  b = std::llabs(b);
  while (b) {
    int64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}

JRange linspace_rational(int64_t start_n, int64_t stop_n, int64_t len, int64_t den) {
  JRange r;
  r.len = len;
  if (start_n == stop_n) {
    r.ref = tp_div(tp_from_int(start_n), tp_from_int(den));
    r.step = tp_div(tp_from_int(0), tp_from_int(den));
    r.offset = 1;
    return r;
  }
  double tmin = -(double)start_n / ((double)stop_n - (double)start_n);
  int64_t imin = round_half_even(tmin * (double)(len - 1) + 1.0);
  imin = std::min(std::max(imin, (int64_t)1), len);
  __int128 ref_num = (__int128)(len - imin) * start_n + (__int128)(imin - 1) * stop_n;
  __int128 ref_den = (__int128)(len - 1) * den;
  r.ref = tp_div(tp_from_int(ref_num), tp_from_int(ref_den));
  TP st = tp_div(tp_from_int((__int128)stop_n - (__int128)start_n), tp_from_int(ref_den));
  r.step = twiceprecision(st, nbitslen(len, imin));
  r.offset = imin;
  return r;
}

JRange linspace_float(double start, double stop, int64_t len) {
  JRange r;
  r.len = len;
  double delta = stop - start;
  double dfac = 1.0;
  if (!std::isfinite(delta)) {
    delta = stop / (double)len - start / (double)len;
    dfac = (double)len;
  }
  double tmin = -(start / delta) / dfac;
  int64_t imin = round_half_even(tmin * (double)(len - 1) + 1.0);
  double ref, step;
  if (1 < imin && imin < len) {
    double t = (double)(imin - 1) / (double)(len - 1);
    ref = (1.0 - t) * start + t * stop;
    step = (imin - 1 < len - imin) ? (ref - start) / (double)(imin - 1)
                                   : (stop - ref) / (double)(len - imin);
  } else if (imin <= 1) {
    imin = 1;
    ref = start;
    step = (delta / (double)(len - 1)) * dfac;
  } else {
    imin = len;
    ref = stop;
    step = (delta / (double)(len - 1)) * dfac;
  }
  const double mx = std::nextafter(1.7976931348623157e308, 0.0);
  double k = (double)std::max(imin - 1, len - imin);
  double lo_c = std::max(-(mx + ref) / k, (-mx + ref) / k);
  double hi_c = std::min((mx - ref) / k, (mx + ref) / k);
  double step_hi_pre = std::min(std::max(step, lo_c), hi_c);
  int nb = nbitslen(len, imin);
  double step_hi = truncbits(step_hi_pre, nb);
  double x1_hi, x1_lo, x2_hi, x2_lo;
  add12((double)(1 - imin) * step_hi, ref, x1_hi, x1_lo);
  add12((double)(len - imin) * step_hi, ref, x2_hi, x2_lo);
  double a = (start - x1_hi) - x1_lo, b = (stop - x2_hi) - x2_lo;
  double step_lo = (b - a) / (double)(len - 1);
  double ref_lo = a - (double)(1 - imin) * step_lo;
  r.ref = TP{ref, ref_lo};
  r.step = TP{step_hi, step_lo};
  r.offset = imin;
  return r;
}

// range(start; stop, length) for Float64 endpoints (range_start_stop_length)
JRange julia_range(double start, double stop, int64_t len) {
  if (len < 2) {
    JRange r;
    r.ref = TP{start, 0.0};
    r.step = TP{len == 1 ? 0.0 : stop - start, 0.0};
    r.len = len;
    r.offset = 1;
    return r;
  }
  if (start == stop) {
    JRange r;
    r.ref = TP{start, 0.0};
    r.step = TP{0.0, 0.0};
    r.len = len;
    r.offset = 1;
    return r;
  }
  int64_t sn, sd, en, ed;
  rat(start, sn, sd);
  rat(stop, en, ed);
  if (sd != 0 && ed != 0) {
    int64_t g = gcd64(sd, ed);
    int64_t den = sd * (ed / g);  // lcm_unchecked
    const double m = 9007199254740992.0;  // maxintfloat(Float64, Int)
    if (den != 0 && std::fabs((double)den * start) <= m && std::fabs((double)den * stop) <= m) {
      int64_t start_n = round_half_even((double)den * start);
      int64_t stop_n = round_half_even((double)den * stop);
      if ((double)start_n / (double)den == start && (double)stop_n / (double)den == stop)
        return linspace_rational(start_n, stop_n, len, den);
    }
  }
  return linspace_float(start, stop, len);
}

// r .- shift on a StepRangeLen: ref + (-shift) in twice precision
JRange range_shift(JRange r, double shift) {
  double s_hi, s_lo;
  add12(r.ref.hi, -shift, s_hi, s_lo);
  TP nr;
  canonicalize2(s_hi, s_lo + r.ref.lo, nr.hi, nr.lo);
  r.ref = nr;
  return r;
}

JRange axis_range(const or_domain* d, int axis, bool staggered) {
  double mx = axis == 0 ? d->xmax : axis == 1 ? d->ymax : d->zmax;
  int64_t n = axis == 0 ? d->nx : axis == 1 ? d->ny : d->nz;
  double h = axis == 0 ? d->dx : axis == 1 ? d->dy : d->dz;
  JRange r = julia_range(-mx, mx, n);
  if (staggered) r = range_shift(r, h / 2);
  return r;
}

// coords(d) (simulation.jl:109-115): channel c is staggered along axis c-1
inline bool is_staggered(int axis, int chan) { return chan >= 1 && chan - 1 == axis; }

inline int64_t findlast_less(const JRange& r, double xp) {
  // findlast(xk .< xp) over an increasing range; 0 means `nothing`
  int64_t ans = 0;
  for (int64_t i = 1; i <= r.len; ++i)
    if (r.at(i) < xp) ans = i;
  return ans;
}

// ---------------------------------------------------------------------------
// Scatterer predicates (src/geometry.jl:86-143) plus the centred/ellipsoid
// extensions used by the serving stream (centre 0 reduces to the reference).
// ---------------------------------------------------------------------------
struct Shape {
  int kind;
  double p[6];
  bool outside(double x, double y, double z) const {
    switch (kind) {
      case OR_SHAPE_NONE:
        return true;
      case OR_SHAPE_SPHERE: {
        double r = p[0];
        double xx = x - p[1], yy = y - p[2], zz = z - p[3];
        return xx * xx + yy * yy + zz * zz > r * r;
      }
      case OR_SHAPE_CUBE: {
        double r = p[0];
        double xx = x - p[1], yy = y - p[2], zz = z - p[3];
        return std::fabs(xx) > r / 2 || std::fabs(yy) > r / 2 || std::fabs(zz) > r / 2;
      }
      case OR_SHAPE_CROSS: {
        double l = p[0];
        double s = l / 2;
        double sl = 2.0 * l / 3;
        auto in = [s](double a, double b, double c) {
          return std::fabs(a) < s && std::fabs(b) < s && std::fabs(c) < s;
        };
        if (in(x, y, z)) {
          if (in(x + sl, y + sl, z) || in(x - sl, y - sl, z) || in(x + sl, y - sl, z) ||
              in(x - sl, y + sl, z))
            return true;
          if (in(x + sl, y, z + sl) || in(x - sl, y, z - sl) || in(x + sl, y, z - sl) ||
              in(x - sl, y, z + sl))
            return true;
          if (in(x, y + sl, z + sl) || in(x, y - sl, z - sl) || in(x, y + sl, z - sl) ||
              in(x, y - sl, z + sl))
            return true;
          return false;
        }
        return true;
      }
      case OR_SHAPE_ELLIPSOID: {
        double xx = (x - p[3]) / p[0], yy = (y - p[4]) / p[1], zz = (z - p[5]) / p[2];
        return xx * xx + yy * yy + zz * zz > 1.0;
      }
    }
    return true;
  }
};

// ---------------------------------------------------------------------------
// getBoundaryIndex (src/kernels/derivatives.jl:66-79), 1-based
// ---------------------------------------------------------------------------
inline void boundary_index(int64_t i, int64_t ndim, int64_t npml, int64_t& l, int& side) {
  side = 0;
  if (i <= npml) {
    side = 1;
    l = i;
  } else {
    l = i - (ndim - npml);
    if (l > 0) side = 2;
  }
}

template <typename R>
struct Scal {
  R fq, fv, dx, dy, dz;
};

// Field view over storage S: float (the reference's Float32 arrays) or
// double (the FP64 error-statement run, every array in Float64).
template <typename S>
struct ViewT {
  int64_t nx, ny, nz;
  S* f;
  inline S& P(int64_t i, int64_t j, int64_t k) { return f[idx(i, j, k, 0)]; }
  inline int64_t idx(int64_t i, int64_t j, int64_t k, int c) const {
    return (i - 1) + nx * ((j - 1) + ny * ((k - 1) + nz * (int64_t)c));
  }
};

// update_p! (updates.jl:105-142) for one cell, used on the rigid planes and
// on the npml==0 unmasked interior
template <typename R, typename S>
inline void update_p_plain(ViewT<S>& v, const Scal<R>& s, int64_t i, int64_t j, int64_t k) {
  S* f = v.f;
  const S m2 = -2;
  R dvx, dvy, dvz;
  if (i == v.nx)
    dvx = (R)(m2 * f[v.idx(i, j, k, 1)]) / s.dx;
  else
    dvx = (R)(f[v.idx(i + 1, j, k, 1)] - f[v.idx(i, j, k, 1)]) / s.dx;
  if (j == v.ny)
    dvy = (R)(m2 * f[v.idx(i, j, k, 2)]) / s.dy;
  else
    dvy = (R)(f[v.idx(i, j + 1, k, 2)] - f[v.idx(i, j, k, 2)]) / s.dy;
  if (k == v.nz)
    dvz = (R)(m2 * f[v.idx(i, j, k, 3)]) / s.dz;
  else
    dvz = (R)(f[v.idx(i, j, k + 1, 3)] - f[v.idx(i, j, k, 3)]) / s.dz;
  S& P = f[v.idx(i, j, k, 0)];
  P = (S)((R)P - s.fq * (dvx + dvy + dvz));
}

// CPML memory update `m = b*m + a*d; d += m` (updates.jl:46-61).  b*m is a
// Float32 product; a*d promotes to R.
template <typename R, typename S>
inline void cpml_apply(R& dv, S* m, S a, S b) {
  S bm = b * (*m);
  R nm = (R)bm + (R)a * dv;
  *m = (S)nm;
  dv = dv + (R)(*m);
}

// update_p_cpml! (updates.jl:21-103) / update_p_cpml_mask! (:320-378) /
// update_p_mask! (:288-318) for one interior cell
template <typename R, typename S, typename CP>
inline void update_p_interior(ViewT<S>& v, const Scal<R>& s, CP* cp, const uint8_t* mask,
                              bool guard, int64_t i, int64_t j, int64_t k) {
  S* f = v.f;
  const int64_t nx = v.nx, ny = v.ny, nz = v.nz;
  R dvx = (R)(f[v.idx(i + 1, j, k, 1)] - f[v.idx(i, j, k, 1)]) / s.dx;
  R dvy = (R)(f[v.idx(i, j + 1, k, 2)] - f[v.idx(i, j, k, 2)]) / s.dy;
  R dvz = (R)(f[v.idx(i, j, k + 1, 3)] - f[v.idx(i, j, k, 3)]) / s.dz;
  const int64_t npml = cp ? cp->npml : 0;
  if (cp && npml > 0 && (!guard || npml > 1)) {
    const S* co = cp->coef;
    const S* A[2] = {co, co + npml};
    const S* B[2] = {co + 4 * npml + 2, co + 5 * npml + 2};
    int64_t l;
    int side;
    boundary_index(i, nx, npml, l, side);
    if (side > 0) {
      S* m = cp->mv[0] + (l - 1) + npml * ((j - 1) + ny * ((k - 1) + nz * (side - 1)));
      cpml_apply(dvx, m, A[side - 1][l - 1], B[side - 1][l - 1]);
    }
    boundary_index(j, ny, npml, l, side);
    if (side > 0) {
      S* m = cp->mv[1] + (i - 1) + nx * ((l - 1) + npml * ((k - 1) + nz * (side - 1)));
      cpml_apply(dvy, m, A[side - 1][l - 1], B[side - 1][l - 1]);
    }
    boundary_index(k, nz, npml, l, side);
    if (side > 0) {
      S* m = cp->mv[2] + (i - 1) + nx * ((j - 1) + ny * ((l - 1) + npml * (side - 1)));
      cpml_apply(dvz, m, A[side - 1][l - 1], B[side - 1][l - 1]);
    }
  }
  S& P = f[v.idx(i, j, k, 0)];
  if (mask) {
    R coeff = s.fq * (R)(mask[v.idx(i, j, k, 0)] ? 1 : 0);
    P = (S)((R)P - coeff * (dvx + dvy + dvz));
  } else {
    P = (S)((R)P - s.fq * (dvx + dvy + dvz));
  }
}

// update_vx!/vy!/vz! (updates.jl:192-274) and the _mask variants (:380-501)
template <typename R, typename S, typename CP>
inline void update_v(ViewT<S>& v, const Scal<R>& s, CP* cp, const uint8_t* mask, int axis,
                     int64_t i, int64_t j, int64_t k) {
  S* f = v.f;
  const int64_t nx = v.nx, ny = v.ny, nz = v.nz;
  const int c = axis + 1;
  R h = axis == 0 ? s.dx : axis == 1 ? s.dy : s.dz;
  int64_t im = i - (axis == 0), jm = j - (axis == 1), km = k - (axis == 2);
  R dp = (R)(f[v.idx(i, j, k, 0)] - f[v.idx(im, jm, km, 0)]) / h;
  const int64_t npml = cp ? cp->npml : 0;
  const int64_t nm = npml + 1;  // size(mp_*, axis)
  if (cp && nm > 1) {
    const S* co = cp->coef;
    const S* A[2] = {co + 2 * npml, co + 3 * npml + 1};
    const S* B[2] = {co + 6 * npml + 2, co + 7 * npml + 3};
    int64_t ii = axis == 0 ? i : axis == 1 ? j : k;
    int64_t nd = axis == 0 ? nx : axis == 1 ? ny : nz;
    int64_t l;
    int side;
    boundary_index(ii, nd, nm, l, side);
    if (side > 0) {
      S* m;
      if (axis == 0)
        m = cp->mp[0] + (l - 1) + nm * ((j - 1) + ny * ((k - 1) + nz * (side - 1)));
      else if (axis == 1)
        m = cp->mp[1] + (i - 1) + nx * ((l - 1) + nm * ((k - 1) + nz * (side - 1)));
      else
        m = cp->mp[2] + (i - 1) + nx * ((j - 1) + ny * ((l - 1) + nm * (side - 1)));
      cpml_apply(dp, m, A[side - 1][l - 1], B[side - 1][l - 1]);
    }
  }
  S& V = f[v.idx(i, j, k, c)];
  if (mask) {
    R coeff = s.fv * (R)(mask[v.idx(i, j, k, c)] ? 1 : 0);
    V = (S)((R)V - coeff * dp);
  } else {
    V = (S)((R)V - s.fv * dp);
  }
}

// interp_trilinear! (derivatives.jl:30-60) with transceivers in ascending
// order (the reference's parallel order is undefined where stencils overlap)
template <typename S>
inline void interp_trilinear(ViewT<S>& v, int c, int64_t it, const float* idx, const S* w,
                             const S* src, S* rec, int64_t ntx, int64_t nt) {
  for (int64_t is = 0; is < ntx; ++is) {
    int64_t I = (int64_t)idx[3 * is + 0];
    int64_t J = (int64_t)idx[3 * is + 1];
    int64_t K = (int64_t)idx[3 * is + 2];
    bool inb = I >= 1 && I < v.nx && J >= 1 && J < v.ny && K >= 1 && K < v.nz;
    if (!inb) continue;
    S s = src[(it - 1) + nt * is];
    S& r = rec[(it - 1) + nt * is];
    for (int kk = 0; kk < 2; ++kk)
      for (int jj = 0; jj < 2; ++jj)
        for (int ii = 0; ii < 2; ++ii) {
          S wv = w[ii + 2 * jj + 4 * kk + 8 * is];
          S& fv = v.f[v.idx(I + ii, J + jj, K + kk, c)];
          r += wv * fv;
          fv += wv * s;
        }
  }
}

// extrapolate! (extrapolation.jl:204-249) with its three kernels, step it
void gf_extrapolate(const or_gfmap* g, or_txgrid* txs, int64_t nt, int64_t it) {
  const int64_t T = std::min(it, g->nt_gf);
  const int64_t t_off = it - T + 1;
  auto pin = [&](int64_t row, int64_t col) {  // row 1-based, col 0-based
    return ((double)txs->rec[0][(row - 1) + nt * col] -
            (double)txs->vn_rec[(row - 1) + nt * col] * g->z0) / 2.0;
  };
  if (g->kind == 0) {  // PVFromPin, extrapolate_pv_from_pin! (:139-170)
    pfor(0, g->n1, [&](int64_t s) {
      double psum = 0.0, vsum = 0.0;  // Float32 zero promoted by the first Float64 add
      for (int64_t r = 0; r < g->n2; ++r) {
        const int64_t col = g->i_rec[r] - 1;
        for (int64_t tt = 1; tt <= T; ++tt) {
          const double pt = pin(t_off + tt - 1, col);
          const size_t k = (size_t)(T - tt) + (size_t)g->nt_gf * (size_t)(s + g->n1 * r);
          psum += (double)g->t[0][k] * pt;
          vsum += (double)g->t[1][k] * pt;
        }
      }
      if (!g->discard) {
        const int64_t col = g->i_src[s] - 1;
        txs->src[0][it + nt * col] = (float)vsum;  // p_src <- v_pin-derived
        txs->vn_src[it + nt * col] = (float)psum;  // vn_src <- p_pin-derived
      }
    });
  } else if (g->kind == 1) {  // PFromPin, extrapolate_p_from_pin (:172-193)
    pfor(0, g->n2, [&](int64_t s) {
      float pn[2];
      for (int h = 0; h < 2; ++h) {
        double sum = 0.0;
        for (int64_t r = 0; r < g->n1; ++r) {
          const int64_t col = g->i_rec[r] - 1;
          for (int64_t tt = 1; tt <= T; ++tt) {
            const size_t k = (size_t)(T - tt) + (size_t)g->nt_gf * (size_t)(r + g->n1 * s);
            sum += (double)g->t[h][k] * pin(t_off + tt - 1, col);
          }
        }
        pn[h] = (float)sum;  // out = zeros(Float32, nsrc)
      }
      if (!g->discard) {
        const int64_t col = g->i_src[s] - 1;
        txs->src[0][it + nt * col] = pn[0] - pn[1];
        txs->vn_src[it + nt * col] = (float)((double)(pn[0] + pn[1]) / g->z0);
      }
    });
  } else {  // PVFromPV, extrapolate_pv_from_pv (:91-137)
    pfor(0, g->n2, [&](int64_t r) {
      float psum = 0.0f, vsum = 0.0f;
      for (int64_t m = 0; m < g->n1; ++m) {
        const int64_t col = g->i_rec[m] - 1;
        for (int64_t tt = 1; tt <= T; ++tt) {
          const int64_t row = t_off + tt - 1;
          const float p_t = txs->rec[0][(row - 1) + nt * col];
          const float vn_t = txs->vn_rec[(row - 1) + nt * col];
          const size_t k = (size_t)(T - tt) + (size_t)g->nt_gf * (size_t)(m + g->n1 * r);
          psum += g->t[1][k] * p_t + g->t[0][k] * vn_t;  // pv*p + pp*vn
          vsum += g->t[3][k] * p_t + g->t[2][k] * vn_t;  // vv*p + vp*vn
        }
      }
      if (!g->discard) {
        const int64_t col = g->i_src[r] - 1;
        txs->src[0][it + nt * col] = vsum;
        txs->vn_src[it + nt * col] = psum;
      }
    });
  }
}

// R: arithmetic of the updates; S, TX, CP: storage of the field, the
// transceiver buffers and the CPML memory (Float32, or Float64 throughout
// for the FP64 run, which has no GF map).
template <typename R, typename S, typename TX, typename CP>
int run_fdtd_t(const or_domain* d, S* field, TX* txs, CP* cp, const uint8_t* mask, int64_t start,
               int64_t stop, const or_gfmap* gf = nullptr) {
  ViewT<S> v{d->nx, d->ny, d->nz, field};
  Scal<R> s{(R)d->fact_m0, (R)d->fact_m1, (R)d->dx, (R)d->dy, (R)d->dz};
  const int64_t nx = d->nx, ny = d->ny, nz = d->nz, nt = d->nt;
  const int64_t npml = cp ? cp->npml : 0;
  for (int64_t it = start; it <= stop; ++it) {
    // forward.jl:64-70 rigid planes j=ny and k=nz (update_p!, no CPML/mask)
    pfor(1, (nz - 1) + 1, [&](int64_t k) {
      for (int64_t i = 1; i <= nx - 1; ++i) update_p_plain<R>(v, s, i, ny, k);
    });
    pfor(1, (ny - 1) + 1, [&](int64_t j) {
      for (int64_t i = 1; i <= nx - 1; ++i) update_p_plain<R>(v, s, i, j, nz);
    });
    // forward.jl:76-89 interior
    if (!mask && npml == 0) {
      pfor(1, (nz - 1) + 1, [&](int64_t k) {
        for (int64_t j = 1; j <= ny - 1; ++j)
          for (int64_t i = 1; i <= nx - 1; ++i) update_p_plain<R>(v, s, i, j, k);
      });
    } else {
      CP* cpu = npml == 0 ? nullptr : cp;
      bool guard = (mask == nullptr);  // update_p_cpml! guards npml>1, the mask variant does not
      pfor(1, (nz - 1) + 1, [&](int64_t k) {
        for (int64_t j = 1; j <= ny - 1; ++j)
          for (int64_t i = 1; i <= nx - 1; ++i)
            update_p_interior<R>(v, s, cpu, mask, guard, i, j, k);
      });
    }
    // forward.jl:92 q-channel injection/recording on P
    interp_trilinear(v, 0, it, txs->idx[0], txs->w[0], txs->src[0], txs->rec[0], txs->ntx, nt);
    // forward.jl:99-107 velocity updates (read the updated P)
    pfor(1, (nz) + 1, [&](int64_t k) {
      for (int64_t j = 1; j <= ny; ++j)
        for (int64_t i = 1; i <= nx; ++i) {
          if (i >= 2) update_v<R>(v, s, cp, mask, 0, i, j, k);
          if (j >= 2) update_v<R>(v, s, cp, mask, 1, i, j, k);
          if (k >= 2) update_v<R>(v, s, cp, mask, 2, i, j, k);
        }
    });
    // forward.jl:111-115 f-channel injection/recording
    for (int c = 1; c <= 3; ++c)
      interp_trilinear(v, c, it, txs->idx[c], txs->w[c], txs->src[c], txs->rec[c], txs->ntx,
                       nt);
    // forward.jl:120 v2vn!
    for (int64_t is = 0; is < txs->ntx; ++is) {
      const S* n = txs->dir + 4 * is;
      int64_t o = (it - 1) + nt * is;
      txs->vn_rec[o] = txs->rec[1][o] * n[1] + txs->rec[2][o] * n[2] + txs->rec[3][o] * n[3];
    }
    // forward.jl:123-128 in-loop GF extrapolation
    if constexpr (std::is_same<TX, or_txgrid>::value) {
      if (gf && it < nt) gf_extrapolate(gf, txs, nt, it);
    }
    // forward.jl:130-132 vn2v! into row it+1
    if (it < nt) {
      for (int64_t is = 0; is < txs->ntx; ++is) {
        const S* n = txs->dir + 4 * is;
        int64_t o = it + nt * is;
        S vn = txs->vn_src[o];
        txs->src[1][o] += vn * n[1];
        txs->src[2][o] += vn * n[2];
        txs->src[3][o] += vn * n[3];
      }
    }
    // forward.jl:134-137 rigid mirrors
    pfor(1, (nz) + 1, [&](int64_t k) {
      for (int64_t i = 1; i <= nx; ++i) field[v.idx(i, 1, k, 2)] = -field[v.idx(i, 2, k, 2)];
    });
    pfor(1, (ny) + 1, [&](int64_t j) {
      for (int64_t i = 1; i <= nx; ++i) field[v.idx(i, j, 1, 3)] = -field[v.idx(i, j, 2, 3)];
    });
  }
  return 0;
}

// KH wavelet helpers (kh_kernels.jl:19-28)
inline double kh_erf(double x) {
  double s = (x > 0) - (x < 0), ax = std::fabs(x);
  double t = 1.0 / (1.0 + 0.3275911 * ax);
  double y = 1.0 - (((((1.061405429 * t - 1.453152027) * t) + 1.421413741) * t - 0.284496736) * t +
                    0.254829592) *
                       t * std::exp(-ax * ax);
  return s * y;
}
inline double kh_fg(double tau, double sg) {
  return (1.0 / (std::sqrt(2.0 * M_PI) * sg)) * std::exp(-(tau * tau) / (2.0 * (sg * sg)));
}
inline double kh_dfg(double tau, double sg) { return -(tau / (sg * sg)) * kh_fg(tau, sg); }
inline double kh_Fg(double tau, double sg) { return 0.5 * (1.0 + kh_erf(tau / (sg * std::sqrt(2.0)))); }

inline void set_threads(int n) { g_threads = n; }

}  // namespace

extern "C" {

int or_version(void) { return 1; }

// Domain constructor (simulation.jl:46-79)
int or_domain_make(double tmax, double xmax, double ymax, double zmax, int64_t nx, int64_t ny,
                   int64_t nz, double c0, double r0, double cf, or_domain* o) {
  if (!o || nx < 2 || ny < 2 || nz < 2) return -1;
  o->tmax = tmax;
  o->xmax = xmax;
  o->ymax = ymax;
  o->zmax = zmax;
  o->nx = nx;
  o->ny = ny;
  o->nz = nz;
  o->c0 = c0;
  o->r0 = r0;
  o->cf = cf;
  o->dx = 2 * xmax / (double)(nx - 1);
  o->dy = 2 * ymax / (double)(ny - 1);
  o->dz = 2 * zmax / (double)(nz - 1);
  o->dt = cf * std::min(o->dx, std::min(o->dy, o->dz)) / c0 / std::sqrt(3.0);
  o->nt = (int64_t)std::ceil(tmax / o->dt);
  o->fact_m0 = o->dt * r0 * (c0 * c0);
  o->fact_m1 = o->dt / r0;
  o->z0 = r0 * c0;
  return 0;
}

int or_range(double start, double stop, int64_t len, double shift, double* out) {
  if (len < 1 || !out) return -1;
  JRange r = julia_range(start, stop, len);
  if (shift != 0.0) r = range_shift(r, shift);
  for (int64_t i = 1; i <= len; ++i) out[i - 1] = r.at(i);
  return 0;
}

int or_coords(const or_domain* d, int axis, int chan, double* out) {
  if (!d || axis < 0 || axis > 2 || chan < 0 || chan > 3) return -1;
  JRange r = axis_range(d, axis, is_staggered(axis, chan));
  for (int64_t i = 1; i <= r.len; ++i) out[i - 1] = r.at(i);
  return 0;
}

int or_time_axis(const or_domain* d, double* out) {
  JRange r = julia_range(0.0, d->tmax, d->nt);
  for (int64_t i = 1; i <= d->nt; ++i) out[i - 1] = r.at(i);
  return 0;
}

// compute_CPML_coefficients! / calc_Kab_CPML (cpmlcoeffs.jl:36-126), K_max = nothing
int or_cpml_coefficients(int64_t halo, double vel_max, double dt, double rcoef, double thickness,
                         double f0, double* out) {
  if (halo < 0 || !out) return -1;
  const double alpha_max = M_PI * f0;
  const double npower = 2.0;
  double d0 = -(npower + 1) * vel_max * std::log(rcoef) / (2.0 * thickness);
  if (halo == 0) d0 = 0.0;
  double* a_l = out;
  double* a_r = a_l + halo;
  double* a_hl = a_r + halo;
  double* a_hr = a_hl + halo + 1;
  double* b_l = a_hr + halo + 1;
  double* b_r = b_l + halo;
  double* b_hl = b_r + halo;
  double* b_hr = b_hl + halo + 1;
  for (int pass = 0; pass < 2; ++pass) {
    const bool half = pass == 1;
    int64_t n = halo + (half ? 1 : 0);
    double shift = half ? 0.5 : 0.0;
    std::vector<double> dist(n);
    // collect(LinRange(0 - shift, n - shift - 1, n)): element i is
    // lerpi(i-1, lendiv, a, b) = (1-t)*a + t*b with t = (i-1)/lendiv and
    // lendiv = max(1, n-1)
    double lr0 = 0 - shift, lr1 = (double)n - shift - 1;
    int64_t lendiv = std::max<int64_t>(1, n - 1);
    for (int64_t i = 1; i <= n; ++i) {
      double t = (double)(i - 1) / (double)lendiv;
      dist[i - 1] = (1 - t) * lr0 + t * lr1;
    }
    if (half) dist[0] = 0;
    double* al = half ? a_hl : a_l;
    double* ar = half ? a_hr : a_r;
    double* bl = half ? b_hl : b_l;
    double* br = half ? b_hr : b_r;
    for (int64_t i = 0; i < n; ++i) {
      double ndl = halo != 0 ? dist[n - 1 - i] / (double)halo : dist[n - 1 - i];
      double ndr = halo != 0 ? dist[i] / (double)halo : dist[i];
      // normdist .^ 2.0: Julia's Float64 power by squaring returns RN(x*x)
      double dl = d0 * (ndl * ndl);
      double alphal = alpha_max * (1.0 - ndl);
      double bL = std::exp(-(dl / 1.0 + alphal) * dt);
      double aL = dl * (bL - 1.0) / (1.0 * (dl + 1.0 * alphal));
      double dr = d0 * (ndr * ndr);
      double alphar = alpha_max * (1.0 - ndr);
      double bR = std::exp(-(dr / 1.0 + alphar) * dt);
      double aR = dr * (bR - 1.0) / (1.0 * (dr + 1.0 * alphar));
      al[i] = aL;
      bl[i] = bL;
      ar[i] = aR;
      br[i] = bR;
    }
  }
  return 0;
}

int or_build_scatterer(const or_domain* d, int shape, const double* params, uint8_t* out) {
  if (!d || !out) return -1;
  Shape sh;
  sh.kind = shape;
  for (int i = 0; i < 6; ++i) sh.p[i] = params ? params[i] : 0.0;
  if (shape == OR_SHAPE_ELLIPSOID && (!params || params[0] <= 0 || params[1] <= 0 || params[2] <= 0))
    return -1;
  std::vector<double> xp(d->nx), yp(d->ny), zp(d->nz);
  or_coords(d, 0, 0, xp.data());
  or_coords(d, 1, 0, yp.data());
  or_coords(d, 2, 0, zp.data());
  const int64_t nx = d->nx, ny = d->ny, nz = d->nz;
  if (shape == OR_SHAPE_NONE) {
    std::memset(out, 0, (size_t)(nx * ny * nz));
    return 0;
  }
  pfor(0, nz, [&](int64_t k) {
    for (int64_t j = 0; j < ny; ++j)
      for (int64_t i = 0; i < nx; ++i)
        out[i + nx * (j + ny * k)] = !sh.outside(xp[i], yp[j], zp[k]);
  });
  return 0;
}

// build_update_mask (geometry.jl:250-280)
int or_build_update_mask(const or_domain* d, int shape, const double* params, uint8_t* out) {
  if (!d || !out) return -1;
  if (shape == OR_SHAPE_NONE) return 1;
  const int64_t nx = d->nx, ny = d->ny, nz = d->nz, N = nx * ny * nz;
  std::vector<uint8_t> s((size_t)N);
  int rc = or_build_scatterer(d, shape, params, s.data());
  if (rc) return rc;
  std::memset(out, 0, (size_t)(4 * N));
  pfor(0, nz, [&](int64_t k) {
    for (int64_t j = 0; j < ny; ++j)
      for (int64_t i = 0; i < nx; ++i) {
        int64_t o = i + nx * (j + ny * k);
        out[o] = !s[o];
        if (i >= 1) out[o + N] = !s[o - 1] && !s[o];
        if (j >= 1) out[o + 2 * N] = !s[o - nx] && !s[o];
        if (k >= 1) out[o + 3 * N] = !s[o - nx * ny] && !s[o];
      }
  });
  return 0;
}

// fibonacci_sphere (illumination.jl:19-46); points, normals (n,3) column-major
int or_fibonacci_sphere(int64_t n, double radius, double* pts, double* nrm) {
  if (n <= 0) return -1;
  const double golden = M_PI * (3.0 - std::sqrt(5.0));
  for (int64_t i = 1; i <= n; ++i) {
    double z = 1.0 - (2.0 * (double)(i - 1) + 1.0) / (double)n;
    double rxy = std::sqrt(std::max(0.0, 1.0 - z * z));
    double th = golden * (double)(i - 1);
    double nx = rxy * std::cos(th), ny = rxy * std::sin(th), nz = z;
    nrm[(i - 1)] = nx;
    nrm[(i - 1) + n] = ny;
    nrm[(i - 1) + 2 * n] = nz;
    pts[(i - 1)] = radius * nx;
    pts[(i - 1) + n] = radius * ny;
    pts[(i - 1) + 2 * n] = radius * nz;
  }
  return 0;
}

// impulsive_wavelet (illumination.jl:167-184)
int or_impulsive_wavelet(const or_domain* d, double f3db, double* tf, double* timeshift) {
  double sig = std::sqrt(std::log(2.0)) / (2 * M_PI * f3db);
  int64_t plen = round_half_even(10 * sig / d->dt);
  int64_t pl = std::min(plen, d->nt);
  double pc = (double)pl / 2, pw = (double)pl / 10;
  for (int64_t i = 0; i < d->nt; ++i) tf[i] = 0.0;
  for (int64_t i = 1; i <= pl; ++i) {
    double u = (double)i - pc;
    tf[i - 1] = std::exp(-(u * u) / (2 * (pw * pw)));
  }
  // sum(tf): Julia's sum over a Vector{Float64} uses pairwise summation
  // (blocks of 1024 summed sequentially); restated here.
  struct PS {
    static double sum(const double* a, int64_t n) {
      if (n <= 1024) {
        double s = 0.0;
        if (n == 0) return 0.0;
        // Base.mapreduce_impl: sequential within a block, 4-way unrolled by
        // @simd is permitted to reassociate; plain order here.
        for (int64_t i = 0; i < n; ++i) s += a[i];
        return s;
      }
      int64_t h = n >> 1;
      return sum(a, h) + sum(a + h, n - h);
    }
  };
  double s = PS::sum(tf, d->nt) * d->dt;
  for (int64_t i = 0; i < d->nt; ++i) tf[i] /= s;
  if (timeshift) *timeshift = pc * d->dt;
  return 0;
}

// ricker_wavelet (illumination.jl:199-207)
int or_ricker_wavelet(const or_domain* d, double fc, int injection, double* tf) {
  std::vector<double> t((size_t)d->nt);
  or_time_axis(d, t.data());
  for (int64_t i = 0; i < d->nt; ++i) {
    double wn = M_PI * fc * (t[i] - 1.0 / fc);
    tf[i] = (1.0 - 2.0 * (wn * wn)) * std::exp(-(wn * wn));
  }
  if (injection) {
    double acc = 0.0;
    double sc = d->dt / d->dx;
    for (int64_t i = 0; i < d->nt; ++i) {
      acc += tf[i];
      tf[i] = acc * sc;
    }
  }
  return 0;
}

// trilinearInterpolation (simulation.jl:254-287) + bilinearInterpolation (:310-341)
int or_trilinear(const or_domain* d, const double* point, int64_t* idx, double* w) {
  const double xp = point[0], yp = point[1], zp = point[2];
  const double ds = d->dx * d->dy;
  // bilinear stencils for p, vx, vy; vz reuses p's
  int64_t bix[3], biy[3];
  double bw[3][4];
  for (int ch = 0; ch < 3; ++ch) {
    JRange xr = axis_range(d, 0, is_staggered(0, ch));
    JRange yr = axis_range(d, 1, is_staggered(1, ch));
    int64_t ix = findlast_less(xr, xp), iy = findlast_less(yr, yp);
    if (ix == 0 || iy == 0) return -2;  // `nothing` -> the reference throws
    double* ww = bw[ch];
    ww[0] = ww[1] = ww[2] = ww[3] = 0.0;
    if (ix < d->nx && iy < d->ny) {
      double x1 = xr.at(ix), x2 = xr.at(ix + 1), y1 = yr.at(iy), y2 = yr.at(iy + 1);
      double dx0 = xp - x1, dx1 = x2 - xp, dy0 = yp - y1, dy1 = y2 - yp;
      ww[0] = dx1 * dy1;  // w[1,1]
      ww[1] = dx0 * dy1;  // w[2,1]
      ww[2] = dx1 * dy0;  // w[1,2]
      ww[3] = dx0 * dy0;  // w[2,2]
      for (int q = 0; q < 4; ++q) ww[q] /= ds;
    }
    bix[ch] = ix;
    biy[ch] = iy;
  }
  const int src_xy[4] = {0, 1, 2, 0};
  for (int c = 0; c < 4; ++c) {
    JRange zr = axis_range(d, 2, is_staggered(2, c));
    int64_t iz = findlast_less(zr, zp);
    if (iz == 0) return -2;
    const double* wxy = bw[src_xy[c]];
    double* w3 = w + 8 * c;
    for (int q = 0; q < 8; ++q) w3[q] = 0.0;
    if (iz < d->nz) {
      double z1 = zr.at(iz), z2 = zr.at(iz + 1);
      for (int q = 0; q < 4; ++q) {
        w3[q] = wxy[q] * (z2 - zp);
        w3[q + 4] = wxy[q] * (zp - z1);
      }
      for (int q = 0; q < 8; ++q) w3[q] /= d->dz;
    }
    idx[3 * c + 0] = bix[src_xy[c]];
    idx[3 * c + 1] = biy[src_xy[c]];
    idx[3 * c + 2] = iz;
  }
  return 0;
}

// transceiversToGrid (simulation.jl:387-431)
int or_pack_transceivers(const or_domain* d, const double* points, const double* dirs,
                         const double* tf, or_txgrid* o) {
  const int64_t ntx = o->ntx, nt = o->nt;
  if (nt != d->nt) return -1;
  for (int64_t is = 0; is < ntx; ++is) {
    int64_t idx[12];
    double w[32];
    int rc = or_trilinear(d, points + 3 * is, idx, w);
    if (rc) return rc;
    for (int c = 0; c < 4; ++c) {
      for (int q = 0; q < 3; ++q) o->idx[c][3 * is + q] = (float)idx[3 * c + q];
      for (int q = 0; q < 8; ++q) o->w[c][8 * is + q] = (float)w[8 * c + q];
      double dc = dirs[4 * is + c];
      for (int64_t t = 0; t < nt; ++t) {
        o->src[c][t + nt * is] = (float)(tf[t + nt * is] * dc);
        o->rec[c][t + nt * is] = (float)((tf[t + nt * is] * dc) * 0);
      }
    }
    for (int q = 0; q < 4; ++q) o->dir[4 * is + q] = (float)dirs[4 * is + q];
    for (int64_t t = 0; t < nt; ++t) {
      o->vn_src[t + nt * is] = 0.0f;
      o->vn_rec[t + nt * is] = 0.0f;
    }
  }
  return 0;
}

int or_run_fdtd_gf(const or_domain* d, float* field, or_txgrid* txs, or_cpml* cpml,
                   const uint8_t* mask, int64_t start_step, int64_t stop_step, int mode,
                   const or_gfmap* gf, int nthreads) {
  if (!d || !field || !txs || !gf) return -1;
  if (start_step < 1 || stop_step > d->nt) return -1;
  if (gf->kind < 0 || gf->kind > 2) return -1;
  // output count and receiver columns per kind
  const int64_t nout = gf->kind == 0 ? gf->n1 : gf->n2;
  const int64_t nin = gf->kind == 0 ? gf->n2 : gf->n1;
  if (gf->n_src != nout || gf->n_rec != nin) return -1;
  for (int64_t s = 0; s < gf->n_src; ++s)
    if (gf->i_src[s] < 1 || gf->i_src[s] > txs->ntx) return -1;
  for (int64_t r = 0; r < gf->n_rec; ++r)
    if (gf->i_rec[r] < 1 || gf->i_rec[r] > txs->ntx) return -1;
  set_threads(nthreads);
  if (mode == OR_MODE_FP32)
    return run_fdtd_t<float>(d, field, txs, cpml, mask, start_step, stop_step, gf);
  return run_fdtd_t<double>(d, field, txs, cpml, mask, start_step, stop_step, gf);
}

int or_run_fdtd(const or_domain* d, float* field, or_txgrid* txs, or_cpml* cpml,
                const uint8_t* mask, int64_t start_step, int64_t stop_step, int mode,
                int nthreads) {
  if (!d || !field || !txs) return -1;
  if (start_step < 1) return -1;
  if (stop_step > d->nt) return -1;
  set_threads(nthreads);
  if (mode == OR_MODE_FP32)
    return run_fdtd_t<float>(d, field, txs, cpml, mask, start_step, stop_step);
  return run_fdtd_t<double>(d, field, txs, cpml, mask, start_step, stop_step);
}

// run_fdtd! with every array in Float64: the FP64 run the error statements
// of the Float32 paths are measured against.  Same operation order as the
// Float32 restatement; coefficients, weights and sources unrounded.
int or_run_fdtd64(const or_domain* d, double* field, or_txgrid64* txs, or_cpml64* cpml,
                  const uint8_t* mask, int64_t start_step, int64_t stop_step, int nthreads) {
  if (!d || !field || !txs) return -1;
  if (start_step < 1) return -1;
  if (stop_step > d->nt) return -1;
  set_threads(nthreads);
  return run_fdtd_t<double>(d, field, txs, cpml, mask, start_step, stop_step);
}

// eval_one_kernel (kh_kernels.jl:106-157)
int or_kh_eval_kernel(int which, int64_t n_outer, const double* op, const double* on,
                      int64_t n_inner, const double* ip, const double* in_, int64_t ntk,
                      const double* tg, double sg, double c0, double rho, float* K,
                      int nthreads) {
  if (which < 0 || which > 3) return -1;
  set_threads(nthreads);
  pfor(0, n_inner, [&](int64_t ir) {
 {
    for (int64_t is = 0; is < n_outer; ++is) {
      double dx = ip[ir] - op[is], dy = ip[ir + n_inner] - op[is + n_outer],
             dz = ip[ir + 2 * n_inner] - op[is + 2 * n_outer];
      double r = std::sqrt(dx * dx + dy * dy + dz * dz);
      double ihx = dx / r, ihy = dy / r, ihz = dz / r;
      double cr = in_[ir] * ihx + in_[ir + n_inner] * ihy + in_[ir + 2 * n_inner] * ihz;
      double cs = on[is] * ihx + on[is + n_outer] * ihy + on[is + 2 * n_outer] * ihz;
      double retard = r / c0;
      double i1 = 1 / (4 * M_PI * r), i2 = 1 / (4 * M_PI * (r * r)),
             i3 = 1 / (4 * M_PI * (r * r * r));
      float* out = K + ntk * (is + n_outer * ir);
      for (int64_t it = 0; it < ntk; ++it) {
        double tau = tg[it] - retard;
        double v;
        if (which == 0) {
          v = kh_dfg(tau, sg) * i1;
        } else if (which == 1) {
          v = cs * (kh_fg(tau, sg) * i2 + kh_dfg(tau, sg) * i1 / c0);
        } else if (which == 2) {
          v = (cr / rho) * (kh_fg(tau, sg) * i2 + kh_dfg(tau, sg) * i1 / c0);
        } else {
          v = (cr * cs / rho) * (2 * kh_Fg(tau, sg) * i3 + 2 * kh_fg(tau, sg) * i2 / c0 +
                                 kh_dfg(tau, sg) * i1 / (c0 * c0));
        }
        out[it] = (float)v;
      }
    }
  }
  });
  return 0;
}

// direct_kh_accumulate! (kh_kernels.jl:256-296)
int or_kh_accumulate(double* out, int64_t nt, const float* K, int64_t ntk, int64_t n_outer,
                     int64_t n_inner, const float* in, double alpha, const float* K_dc,
                     const double* cumsum_in, int nthreads) {
  if (ntk > nt) return -1;
  if ((K_dc == nullptr) != (cumsum_in == nullptr)) return -1;
  set_threads(nthreads);
  pfor(0, n_inner, [&](int64_t s) {
 {
    for (int64_t r = 0; r < n_outer; ++r) {
      const float* Kp = K + ntk * (r + n_outer * s);
      const float* ip = in + nt * r;
      for (int64_t t = 1; t <= nt; ++t) {
        double acc = 0.0;
        int64_t m = std::min(t, ntk);
        for (int64_t tt = 1; tt <= m; ++tt) acc += (double)(Kp[tt - 1] * ip[t - tt]);
        out[(t - 1) + nt * s] += alpha * acc;
      }
    }
  }
  });
  if (K_dc) {
    pfor(0, n_inner, [&](int64_t s) {
      for (int64_t r = 0; r < n_outer; ++r) {
        float k = K_dc[r + n_outer * s];
        if (k == 0) continue;
        double ak = alpha * (double)k;
        for (int64_t t = 0; t < nt; ++t) out[t + nt * s] += ak * cumsum_in[t + nt * r];
      }
    });
  }
  return 0;
}

int or_kh_pressure(int64_t ns, const double* sp, const double* sn, int64_t nr,
                   const double* rp, int64_t nt, int64_t ntk, double dt, double sg, double c0,
                   const float* in_q, const float* in_f, double aq, double af, int mode,
                   int64_t r0, int64_t r1, double* out, int nthreads) {
  if (r0 < 0 || r1 > nr || r1 < r0 || ntk > nt) return -1;
  set_threads(nthreads);
  const int64_t nrr = r1 - r0;
  pfor(0, nrr, [&](int64_t rr) {
    std::vector<double> kq((size_t)ntk), kf((size_t)ntk);
    {
      int64_t ir = r0 + rr;
      double* o = out + nt * rr;
      for (int64_t t = 0; t < nt; ++t) o[t] = 0.0;
      for (int64_t is = 0; is < ns; ++is) {
        double dx = rp[ir] - sp[is], dy = rp[ir + nr] - sp[is + ns],
               dz = rp[ir + 2 * nr] - sp[is + 2 * ns];
        double r = std::sqrt(dx * dx + dy * dy + dz * dz);
        double ihx = dx / r, ihy = dy / r, ihz = dz / r;
        double cs = sn[is] * ihx + sn[is + ns] * ihy + sn[is + 2 * ns] * ihz;
        double retard = r / c0;
        double i1 = 1 / (4 * M_PI * r), i2 = 1 / (4 * M_PI * (r * r));
        // taps with |tau| > 12 sigma are below 1e-31 of the peak (exp(-72))
        // and are dropped; every other tap is evaluated in full
        int64_t lo = std::max<int64_t>(0, (int64_t)std::floor((retard - 12 * sg) / dt));
        int64_t hi = std::min<int64_t>(ntk - 1, (int64_t)std::ceil((retard + 12 * sg) / dt));
        for (int64_t k = lo; k <= hi; ++k) {
          double tau = (double)k * dt - retard;
          double f = kh_fg(tau, sg), df = kh_dfg(tau, sg);
          double vq = df * i1;
          double vf = cs * (f * i2 + df * i1 / c0);
          kq[k] = mode == 0 ? (double)(float)vq : vq;
          kf[k] = mode == 0 ? (double)(float)vf : vf;
        }
        const float* q = in_q + nt * is;
        const float* fsig = in_f + nt * is;
        for (int64_t t = 1; t <= nt; ++t) {
          double aq_s = 0.0, af_s = 0.0;
          int64_t kmax = std::min(hi, t - 1);
          for (int64_t k = lo; k <= kmax; ++k) {
            if (mode == 0) {
              aq_s += (double)((float)kq[k] * q[t - 1 - k]);
              af_s += (double)((float)kf[k] * fsig[t - 1 - k]);
            } else {
              aq_s += kq[k] * (double)q[t - 1 - k];
              af_s += kf[k] * (double)fsig[t - 1 - k];
            }
          }
          o[t - 1] += aq * aq_s + af * af_s;
        }
      }
    }
  });
  return 0;
}

int or_kh_velocity(int64_t ns, const double* sp, const double* sn, int64_t nr,
                   const double* rp, const double* rn, int64_t nt, double dt, double sg,
                   double c0, double rho, const float* in_q, const float* in_f, double aq,
                   double af, int64_t r0, int64_t r1, double* out, int nthreads) {
  if (r0 < 0 || r1 > nr || r1 < r0 || nt < 1) return -1;
  set_threads(nthreads);
  const int64_t nrr = r1 - r0;
  // running sums of in_f per surface point (FP64): cs[t] = sum_{j <= t} in_f[j]
  std::vector<double> cs((size_t)(nt * ns));
  for (int64_t s = 0; s < ns; ++s) {
    double a = 0.0;
    for (int64_t t = 0; t < nt; ++t) {
      a += (double)in_f[t + nt * s];
      cs[(size_t)(t + nt * s)] = a;
    }
  }
  pfor(0, nrr, [&](int64_t rr) {
    const int64_t ir = r0 + rr;
    double* o = out + nt * rr;
    for (int64_t t = 0; t < nt; ++t) o[t] = 0.0;
    std::vector<double> kq, kf;
    for (int64_t is = 0; is < ns; ++is) {
      const double dx = rp[ir] - sp[is], dy = rp[ir + nr] - sp[is + ns],
                   dz = rp[ir + 2 * nr] - sp[is + 2 * ns];
      const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
      const double ihx = dx / r, ihy = dy / r, ihz = dz / r;
      const double cr = rn[ir] * ihx + rn[ir + nr] * ihy + rn[ir + 2 * nr] * ihz;
      const double cs_ = sn[is] * ihx + sn[is + ns] * ihy + sn[is + 2 * ns] * ihz;
      const double retard = r / c0;
      const double i1 = 1 / (4 * M_PI * r), i2 = 1 / (4 * M_PI * (r * r)),
                   i3 = 1 / (4 * M_PI * (r * r * r));
      const int64_t lo = std::max<int64_t>(0, (int64_t)std::floor((retard - 12 * sg) / dt));
      const int64_t hi = (int64_t)std::ceil((retard + 12 * sg) / dt);
      kq.assign((size_t)(hi - lo + 1), 0.0);
      kf.assign((size_t)(hi - lo + 1), 0.0);
      for (int64_t k = lo; k <= hi; ++k) {
        const double tau = (double)k * dt - retard;
        const double f = kh_fg(tau, sg), df = kh_dfg(tau, sg), F = kh_Fg(tau, sg);
        kq[(size_t)(k - lo)] = (cr / rho) * (f * i2 + df * i1 / c0);  // v_p
        kf[(size_t)(k - lo)] =
            (cr * cs_ / rho) * (2 * F * i3 + 2 * f * i2 / c0 + df * i1 / (c0 * c0));  // v_v
      }
      const double ped = (cr * cs_ / rho) * 2 * i3;  // v_v for tau -> inf
      const float* q = in_q + nt * is;
      const float* fs = in_f + nt * is;
      for (int64_t t = 0; t < nt; ++t) {
        double aq_s = 0.0, af_s = 0.0;
        const int64_t kmax = std::min(hi, t);
        for (int64_t k = lo; k <= kmax; ++k) {
          aq_s += kq[(size_t)(k - lo)] * (double)q[t - k];
          af_s += kf[(size_t)(k - lo)] * (double)fs[t - k];
        }
        // lags k > hi: the kernel is its tau -> inf value
        if (t - hi - 1 >= 0) af_s += ped * cs[(size_t)(t - hi - 1 + nt * is)];
        o[t] += aq * aq_s + af * af_s;
      }
    }
  });
  return 0;
}

int or_gf_postprocess(int64_t ncol, int64_t n, double t_in0, double dt_in, int64_t nt_out,
                      double t_out0, double dt_out, const float* in, float* out, double unit,
                      int denoise) {
  if (ncol < 0 || n < 4 || nt_out < 1 || !(dt_in > 0) || !(dt_out > 0) || !(unit != 0))
    return -1;
  const float unit32 = (float)unit;
  const double amp = dt_out / dt_in;  // resample_time's scale_amplitude
  pfor(0, ncol, [&](int64_t c) {
    const float* a = in + n * c;
    std::vector<double> y((size_t)n + 1), cf((size_t)n + 2), cp((size_t)n + 1), dp((size_t)n + 1);
    // greens.jl:178-179: maximum over time (signed), threshold 1e-4 * max
    float mx = a[0];
    for (int64_t t = 1; t < n; ++t) mx = std::max(mx, a[t]);
    for (int64_t t = 1; t <= n; ++t) {
      const float v = a[t - 1];
      y[(size_t)t] = (denoise && (double)std::fabs(v) < 1e-4 * (double)mx) ? 0.0 : (double)v;
    }
    // natural cubic B-spline coefficients c_0..c_{n+1}: c_1 = y_1, c_n = y_n,
    // (c_{i-1} + 4 c_i + c_{i+1}) / 6 = y_i for i = 2..n-1, then the end rows
    cf[1] = y[1];
    cf[(size_t)n] = y[(size_t)n];
    // Thomas algorithm on i = 2..n-1 with rhs 6 y_i and known c_1, c_n
    for (int64_t i = 2; i <= n - 1; ++i) {
      double rhs = 6.0 * y[(size_t)i];
      if (i == 2) rhs -= cf[1];
      if (i == n - 1) rhs -= cf[(size_t)n];
      const double b = 4.0 - (i > 2 ? cp[(size_t)i - 1] : 0.0);
      cp[(size_t)i] = 1.0 / b;
      dp[(size_t)i] = (rhs - (i > 2 ? dp[(size_t)i - 1] : 0.0)) / b;
    }
    for (int64_t i = n - 1; i >= 2; --i)
      cf[(size_t)i] = dp[(size_t)i] - (i < n - 1 ? cp[(size_t)i] * cf[(size_t)i + 1] : 0.0);
    cf[0] = 2.0 * cf[1] - cf[2];
    cf[(size_t)n + 1] = 2.0 * cf[(size_t)n] - cf[(size_t)n - 1];
    for (int64_t k = 0; k < nt_out; ++k) {
      const double tt = t_out0 + (double)k * dt_out;
      double x = (tt - t_in0) / dt_in + 1.0;  // 1-based sample coordinate
      x = std::min(std::max(x, 1.0), (double)n);  // Flat()
      int64_t i = (int64_t)std::floor(x);
      if (i > n - 1) i = n - 1;
      const double d = x - (double)i, e = 1.0 - d;
      const double w0 = e * e * e / 6.0, w3 = d * d * d / 6.0;
      const double w1 = (3.0 * d * d * d - 6.0 * d * d + 4.0) / 6.0;
      const double w2 = (-3.0 * d * d * d + 3.0 * d * d + 3.0 * d + 1.0) / 6.0;
      const double v = cf[(size_t)i - 1] * w0 + cf[(size_t)i] * w1 + cf[(size_t)i + 1] * w2 +
                       cf[(size_t)i + 2] * w3;
      out[k + nt_out * c] = (float)(v * amp) / unit32;
    }
  });
  return 0;
}

// extrapolate_pv_from_pin! (extrapolation.jl:139-170)
int or_extrapolate_pv_from_pin(const float* pin, int64_t nt, int64_t nrec, float* p_src,
                               float* v_src, int64_t nsrc, const float* pp, const float* vp,
                               int64_t nt_gf, int64_t it) {
  int64_t T = std::min(it, nt_gf);
  int64_t t_off = it - T + 1;
  if (it + 1 > nt) return -1;
  for (int64_t s = 0; s < nsrc; ++s) {
    float psum = 0.0f, vsum = 0.0f;
    for (int64_t r = 0; r < nrec; ++r)
      for (int64_t tt = 1; tt <= T; ++tt) {
        int64_t g = T - tt + 1;
        float pv = pin[(t_off + tt - 1 - 1) + nt * r];
        psum += pp[(g - 1) + nt_gf * (s + nsrc * r)] * pv;
        vsum += vp[(g - 1) + nt_gf * (s + nsrc * r)] * pv;
      }
    p_src[it + nt * s] = vsum;
    v_src[it + nt * s] = psum;
  }
  return 0;
}

}  // extern "C"
