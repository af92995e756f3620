// host_math.h -- host-side geometry of the reference's simulation core.
//
// Domain (src/simulation.jl:46-79), coordinate ranges (simulation.jl:86-115)
// and trilinear transceiver stencils (simulation.jl:254-341).  The
// coordinates are Julia StepRangeLen values with a twice-precision
// reference and step (the double-double algorithm of Julia Base's
// twiceprecision.jl: rational endpoints are detected with a continued
// fraction and the range is evaluated as ref + (i-offset)*step in
// double-double).  Scatterer masks and `findlast(xk .< xp)` depend on the
// last bit of these values, so they are reproduced exactly rather than
// approximated by -xmax + (i-1)*dx.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

namespace adf {
namespace hm {

struct DD {
  double hi, lo;
};

inline void canon2(double big, double little, double& h, double& l) {
  h = big + little;
  l = (big - h) + little;
}
inline void add12(double x, double y, double& h, double& l) {
  if (std::fabs(y) > std::fabs(x)) std::swap(x, y);
  canon2(x, y, h, l);
}
inline DD dd_div(DD x, DD y) {
  double hi = x.hi / y.hi;
  double uh = hi * y.hi;
  double ul = std::isfinite(uh) ? std::fma(hi, y.hi, -uh) : uh;
  double lo = ((((x.hi - uh) - ul) + x.lo) - hi * y.lo) / y.hi;
  DD r;
  canon2(hi, lo, r.hi, r.lo);
  if (x.hi == 0.0 || !std::isfinite(hi)) r = DD{hi, hi};
  return r;
}
inline DD dd_int(__int128 v) {
  double hi = (double)v;
  DD r;
  canon2(hi, (double)(v - (__int128)hi), r.hi, r.lo);
  return r;
}
inline double clear_low_bits(double x, int nb) {
  uint64_t u;
  std::memcpy(&u, &x, 8);
  u &= (~(uint64_t)0) << nb;
  std::memcpy(&x, &u, 8);
  return x;
}
inline int len_bits(int64_t len, int64_t offset) {
  if (len < 2) return 0;
  int64_t m = std::max(offset - 1, len - offset) - 1;
  int b = 0;
  while (m > 0) {
    ++b;
    m >>= 1;
  }
  return std::min(27, b + 1);
}
inline int64_t rne(double x) { return (int64_t)std::nearbyint(x); }

// continued-fraction search for a/b with Float64(a)/Float64(b) == x,
// numerator and denominator bounded by 2^24
inline void cf_rational(double x, int64_t& num, int64_t& den) {
  double y = x;
  int64_t a = 1, d = 1, b = 0, c = 0;
  const double lim = 16777216.0;
  while (std::fabs(y) <= lim) {
    int64_t f = (int64_t)std::trunc(y);
    y -= (double)f;
    int64_t na = f * a + c, nb = f * b + d;
    c = a;
    d = b;
    a = na;
    b = nb;
    if (std::max(std::llabs(a), std::llabs(b)) > (int64_t)lim) {
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

struct Range {
  DD ref, step;
  int64_t len, offset;
  double at(int64_t i) const {  // 1-based element
    double u = (double)(i - offset);
    double sh = u * step.hi, sl = u * step.lo;
    double xh, xl;
    add12(ref.hi, sh, xh, xl);
    return xh + (xl + (sl + ref.lo));
  }
  Range shifted(double s) const {  // r .- s
    Range r = *this;
    double h, l;
    add12(ref.hi, -s, h, l);
    canon2(h, l + ref.lo, r.ref.hi, r.ref.lo);
    return r;
  }
  // findlast(r .< x) for an increasing range; 0 = nothing
  int64_t findlast_less(double x) const {
    int64_t lo = 0, hi = len;  // invariant: at(lo) < x (lo=0 sentinel), at(hi+1) >= x
    // elements are monotone; binary search then verify neighbours
    while (lo < hi) {
      int64_t mid = (lo + hi + 1) / 2;
      if (at(mid) < x)
        lo = mid;
      else
        hi = mid - 1;
    }
    return lo;
  }
};

inline Range make_range(double a, double b, int64_t len) {
  Range r;
  r.len = len;
  r.offset = 1;
  if (len < 2 || a == b) {
    r.ref = DD{a, 0.0};
    r.step = DD{len < 2 ? 0.0 : 0.0, 0.0};
    return r;
  }
  int64_t an, ad, bn, bd;
  cf_rational(a, an, ad);
  cf_rational(b, bn, bd);
  if (ad != 0 && bd != 0) {
    int64_t g = ad, h = bd;
    g = std::llabs(g);
    h = std::llabs(h);
    while (h) {
      int64_t t = g % h;
      g = h;
      h = t;
    }
    int64_t den = ad * (bd / g);
    const double m = 9007199254740992.0;
    if (den != 0 && std::fabs((double)den * a) <= m && std::fabs((double)den * b) <= m) {
      int64_t s_n = rne((double)den * a), e_n = rne((double)den * b);
      if ((double)s_n / (double)den == a && (double)e_n / (double)den == b) {
        if (s_n == e_n) {
          r.ref = dd_div(dd_int(s_n), dd_int(den));
          r.step = dd_div(dd_int(0), dd_int(den));
          return r;
        }
        double tmin = -(double)s_n / ((double)e_n - (double)s_n);
        int64_t imin = std::min(std::max(rne(tmin * (double)(len - 1) + 1.0), (int64_t)1), len);
        __int128 rnum = (__int128)(len - imin) * s_n + (__int128)(imin - 1) * e_n;
        __int128 rden = (__int128)(len - 1) * den;
        r.ref = dd_div(dd_int(rnum), dd_int(rden));
        DD st = dd_div(dd_int((__int128)e_n - (__int128)s_n), dd_int(rden));
        double sh = clear_low_bits(st.hi, len_bits(len, imin));
        r.step = DD{sh, (st.hi - sh) + st.lo};
        r.offset = imin;
        return r;
      }
    }
  }
  // non-rational endpoints
  double delta = b - a, fac = 1.0;
  if (!std::isfinite(delta)) {
    delta = b / (double)len - a / (double)len;
    fac = (double)len;
  }
  double tmin = -(a / delta) / fac;
  int64_t imin = rne(tmin * (double)(len - 1) + 1.0);
  double ref, step;
  if (1 < imin && imin < len) {
    double t = (double)(imin - 1) / (double)(len - 1);
    ref = (1.0 - t) * a + t * b;
    step = (imin - 1 < len - imin) ? (ref - a) / (double)(imin - 1) : (b - ref) / (double)(len - imin);
  } else if (imin <= 1) {
    imin = 1;
    ref = a;
    step = (delta / (double)(len - 1)) * fac;
  } else {
    imin = len;
    ref = b;
    step = (delta / (double)(len - 1)) * fac;
  }
  const double big = std::nextafter(1.7976931348623157e308, 0.0);
  double k = (double)std::max(imin - 1, len - imin);
  double clo = std::max(-(big + ref) / k, (-big + ref) / k);
  double chi = std::min((big - ref) / k, (big + ref) / k);
  double shi = clear_low_bits(std::min(std::max(step, clo), chi), len_bits(len, imin));
  double x1h, x1l, x2h, x2l;
  add12((double)(1 - imin) * shi, ref, x1h, x1l);
  add12((double)(len - imin) * shi, ref, x2h, x2l);
  double lo1 = (a - x1h) - x1l, lo2 = (b - x2h) - x2l;
  double slo = (lo2 - lo1) / (double)(len - 1);
  r.ref = DD{ref, lo1 - (double)(1 - imin) * slo};
  r.step = DD{shi, slo};
  r.offset = imin;
  return r;
}

struct Dom {
  double tmax, xmax, ymax, zmax;
  int64_t nx, ny, nz;
  double c0, r0, cf, dx, dy, dz, fact_m0, fact_m1, dt;
  int64_t nt;
  double z0;
};

// coords(d)[axis][chan]: chan c (1..3 = vx..vz) is staggered along axis c-1
inline Range axis_range(const Dom& d, int axis, int chan) {
  double mx = axis == 0 ? d.xmax : axis == 1 ? d.ymax : d.zmax;
  int64_t n = axis == 0 ? d.nx : axis == 1 ? d.ny : d.nz;
  double h = axis == 0 ? d.dx : axis == 1 ? d.dy : d.dz;
  Range r = make_range(-mx, mx, n);
  if (chan >= 1 && chan - 1 == axis) r = r.shifted(h / 2);
  return r;
}

// trilinearInterpolation: idx (3,4) 1-based, w (2,2,2,4); returns false
// where the reference would throw (a coordinate below the first node)
inline bool trilinear(const Dom& d, const double* pt, int64_t* idx, double* w) {
  const double xp = pt[0], yp = pt[1], zp = pt[2];
  const double ds = d.dx * d.dy;
  int64_t bx[3], by[3];
  double bw[3][4];
  for (int ch = 0; ch < 3; ++ch) {
    Range xr = axis_range(d, 0, ch), yr = axis_range(d, 1, ch);
    int64_t ix = xr.findlast_less(xp), iy = yr.findlast_less(yp);
    if (ix == 0 || iy == 0) return false;
    double* ww = bw[ch];
    ww[0] = ww[1] = ww[2] = ww[3] = 0.0;
    if (ix < d.nx && iy < d.ny) {
      double x1 = xr.at(ix), x2 = xr.at(ix + 1), y1 = yr.at(iy), y2 = yr.at(iy + 1);
      double dx0 = xp - x1, dx1 = x2 - xp, dy0 = yp - y1, dy1 = y2 - yp;
      ww[0] = dx1 * dy1;
      ww[1] = dx0 * dy1;
      ww[2] = dx1 * dy0;
      ww[3] = dx0 * dy0;
      for (int q = 0; q < 4; ++q) ww[q] /= ds;
    }
    bx[ch] = ix;
    by[ch] = iy;
  }
  const int xy_of[4] = {0, 1, 2, 0};  // vz reuses p's x-y stencil
  for (int c = 0; c < 4; ++c) {
    Range zr = axis_range(d, 2, c);
    int64_t iz = zr.findlast_less(zp);
    if (iz == 0) return false;
    const double* wxy = bw[xy_of[c]];
    double* w3 = w + 8 * c;
    for (int q = 0; q < 8; ++q) w3[q] = 0.0;
    if (iz < d.nz) {
      double z1 = zr.at(iz), z2 = zr.at(iz + 1);
      for (int q = 0; q < 4; ++q) {
        w3[q] = wxy[q] * (z2 - zp);
        w3[q + 4] = wxy[q] * (zp - z1);
      }
      for (int q = 0; q < 8; ++q) w3[q] /= d.dz;
    }
    idx[3 * c] = bx[xy_of[c]];
    idx[3 * c + 1] = by[xy_of[c]];
    idx[3 * c + 2] = iz;
  }
  return true;
}

}  // namespace hm
}  // namespace adf
