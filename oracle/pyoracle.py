"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, as the checker or as the timed CPU restatement of the
reference.  The product (acoustic_disguising_b200) never imports it.

Arrays follow the reference's Julia layout: numpy arrays in Fortran order
with the same shapes the reference uses, e.g. the field is (nx, ny, nz, 4).
Parity status: see the header of adf_oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

SHAPES = {"none": 0, "sphere": 1, "cube": 2, "cross": 3, "ellipsoid": 4}
MODES = {"promote": 0, "fp32": 1}


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class Domain(C.Structure):
    """Mirror of `Domain` (src/simulation.jl:25-44)."""

    _fields_ = [
        ("tmax", C.c_double), ("xmax", C.c_double), ("ymax", C.c_double), ("zmax", C.c_double),
        ("nx", C.c_int64), ("ny", C.c_int64), ("nz", C.c_int64),
        ("c0", C.c_double), ("r0", C.c_double), ("cf", C.c_double),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("fact_m0", C.c_double), ("fact_m1", C.c_double),
        ("dt", C.c_double), ("nt", C.c_int64), ("z0", C.c_double),
    ]


class _TxGrid(C.Structure):
    _fields_ = [
        ("ntx", C.c_int64), ("nt", C.c_int64),
        ("idx", C.c_void_p * 4), ("w", C.c_void_p * 4),
        ("src", C.c_void_p * 4), ("rec", C.c_void_p * 4),
        ("dir", C.c_void_p), ("vn_src", C.c_void_p), ("vn_rec", C.c_void_p),
    ]


class _Cpml(C.Structure):
    _fields_ = [("npml", C.c_int64), ("mv", C.c_void_p * 3), ("mp", C.c_void_p * 3),
                ("coef", C.c_void_p)]


# the Float64 run's buffers have the same fields (pointer types differ only)
_TxGrid64 = _TxGrid
_Cpml64 = _Cpml


class _GfMap(C.Structure):
    _fields_ = [("kind", C.c_int), ("nt_gf", C.c_int64), ("n1", C.c_int64), ("n2", C.c_int64),
                ("t", C.c_void_p * 4), ("i_src", C.c_void_p), ("n_src", C.c_int64),
                ("i_rec", C.c_void_p), ("n_rec", C.c_int64), ("z0", C.c_double),
                ("discard", C.c_int)]


GF_KINDS = {"PVFromPin": 0, "PFromPin": 1, "PVFromPV": 2}


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        dp = C.POINTER(Domain)
        L.or_domain_make.argtypes = [C.c_double] * 4 + [C.c_int64] * 3 + [C.c_double] * 3 + [dp]
        L.or_range.argtypes = [C.c_double, C.c_double, C.c_int64, C.c_double, C.c_void_p]
        L.or_coords.argtypes = [dp, C.c_int, C.c_int, C.c_void_p]
        L.or_time_axis.argtypes = [dp, C.c_void_p]
        L.or_cpml_coefficients.argtypes = [C.c_int64, C.c_double, C.c_double, C.c_double,
                                           C.c_double, C.c_double, C.c_void_p]
        L.or_build_update_mask.argtypes = [dp, C.c_int, C.c_void_p, C.c_void_p]
        L.or_build_scatterer.argtypes = [dp, C.c_int, C.c_void_p, C.c_void_p]
        L.or_fibonacci_sphere.argtypes = [C.c_int64, C.c_double, C.c_void_p, C.c_void_p]
        L.or_impulsive_wavelet.argtypes = [dp, C.c_double, C.c_void_p, C.c_void_p]
        L.or_ricker_wavelet.argtypes = [dp, C.c_double, C.c_int, C.c_void_p]
        L.or_trilinear.argtypes = [dp, C.c_void_p, C.c_void_p, C.c_void_p]
        L.or_pack_transceivers.argtypes = [dp, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.POINTER(_TxGrid)]
        L.or_run_fdtd.argtypes = [dp, C.c_void_p, C.POINTER(_TxGrid), C.POINTER(_Cpml),
                                  C.c_void_p, C.c_int64, C.c_int64, C.c_int, C.c_int]
        L.or_run_fdtd64.argtypes = [dp, C.c_void_p, C.POINTER(_TxGrid64), C.POINTER(_Cpml64),
                                    C.c_void_p, C.c_int64, C.c_int64, C.c_int]
        L.or_run_fdtd_gf.argtypes = [dp, C.c_void_p, C.POINTER(_TxGrid), C.POINTER(_Cpml),
                                     C.c_void_p, C.c_int64, C.c_int64, C.c_int,
                                     C.POINTER(_GfMap), C.c_int]
        L.or_kh_eval_kernel.argtypes = [C.c_int, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64,
                                        C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                        C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_int]
        L.or_kh_accumulate.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int64,
                                       C.c_int64, C.c_void_p, C.c_double, C.c_void_p,
                                       C.c_void_p, C.c_int]
        L.or_kh_pressure.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                     C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double,
                                     C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_int,
                                     C.c_int64, C.c_int64, C.c_void_p, C.c_int]
        L.or_kh_velocity.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                     C.c_void_p, C.c_int64, C.c_double, C.c_double, C.c_double,
                                     C.c_double, C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                     C.c_int64, C.c_int64, C.c_void_p, C.c_int]
        L.or_gf_postprocess.argtypes = [C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_int64,
                                        C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                        C.c_double, C.c_int]
        L.or_extrapolate_pv_from_pin.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p,
                                                 C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                                 C.c_int64, C.c_int64]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _chk(rc, what):
    if rc < 0:
        raise RuntimeError(f"oracle {what} failed rc={rc}")
    return rc


def domain(tmax=10e-4, xmax=1.0, ymax=None, zmax=None, nx=201, ny=None, nz=None,
           c0=1500.0, r0=1000.0, cf=0.25) -> Domain:
    ymax = xmax if ymax is None else ymax
    zmax = xmax if zmax is None else zmax
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    d = Domain()
    _chk(lib().or_domain_make(tmax, xmax, ymax, zmax, nx, ny, nz, c0, r0, cf, C.byref(d)),
         "domain")
    return d


def julia_range(start, stop, n, shift=0.0):
    out = np.empty(n, np.float64)
    _chk(lib().or_range(start, stop, n, shift, _p(out)), "range")
    return out


def coords(d: Domain, axis: int, chan: int):
    n = [d.nx, d.ny, d.nz][axis]
    out = np.empty(n, np.float64)
    _chk(lib().or_coords(C.byref(d), axis, chan, _p(out)), "coords")
    return out


def time_axis(d: Domain):
    out = np.empty(d.nt, np.float64)
    lib().or_time_axis(C.byref(d), _p(out))
    return out


def cpml_coefficients(npml, c0, dt, rcoef, thickness, fc):
    """Float64 profiles (a_l, a_r, a_hl, a_hr, b_l, b_r, b_hl, b_hr)."""
    n = npml
    out = np.zeros(8 * n + 4, np.float64)
    _chk(lib().or_cpml_coefficients(n, c0, dt, rcoef, thickness, fc, _p(out)), "cpml")
    sizes = [n, n, n + 1, n + 1, n, n, n + 1, n + 1]
    res, o = [], 0
    for s in sizes:
        res.append(out[o:o + s].copy())
        o += s
    return tuple(res)


def shape_params(shape: str, **kw):
    p = np.zeros(6, np.float64)
    if shape in ("sphere",):
        p[0] = kw["radius"]
        p[1:4] = kw.get("center", (0.0, 0.0, 0.0))
    elif shape == "cube":
        p[0] = kw["length"]
        p[1:4] = kw.get("center", (0.0, 0.0, 0.0))
    elif shape == "cross":
        p[0] = kw["length"]
    elif shape == "ellipsoid":
        p[0:3] = kw["semi_axes"]
        p[3:6] = kw.get("center", (0.0, 0.0, 0.0))
    return p


def build_update_mask(d: Domain, shape: str, **kw):
    """(nx,ny,nz,4) uint8 in Fortran order, or None for shape 'none'."""
    out = np.zeros((d.nx, d.ny, d.nz, 4), np.uint8, order="F")
    rc = _chk(lib().or_build_update_mask(C.byref(d), SHAPES[shape], _p(shape_params(shape, **kw)),
                                         _p(out)), "mask")
    return None if rc == 1 else out


def fibonacci_sphere(n, radius=1.0):
    pts = np.zeros((n, 3), np.float64, order="F")
    nrm = np.zeros((n, 3), np.float64, order="F")
    _chk(lib().or_fibonacci_sphere(n, radius, _p(pts), _p(nrm)), "fibonacci")
    return pts, nrm


def impulsive_wavelet(d: Domain, f_3db_hz):
    tf = np.zeros(d.nt, np.float64)
    ts = C.c_double()
    lib().or_impulsive_wavelet(C.byref(d), f_3db_hz, _p(tf), C.byref(ts))
    return tf, ts.value


def ricker_wavelet(d: Domain, fc=18000.0, injection=True):
    tf = np.zeros(d.nt, np.float64)
    lib().or_ricker_wavelet(C.byref(d), fc, int(injection), _p(tf))
    return tf


def trilinear(d: Domain, point):
    idx = np.zeros((3, 4), np.int64, order="F")
    w = np.zeros((2, 2, 2, 4), np.float64, order="F")
    pt = np.ascontiguousarray(point, np.float64)
    _chk(lib().or_trilinear(C.byref(d), _p(pt), _p(idx), _p(w)), "trilinear")
    return idx, w


@dataclass
class TxGrid:
    """TransceiverGrid (src/simulation.jl:370-378) in Julia layout."""

    idx: list
    w: list
    src: list
    rec: list
    dir: np.ndarray
    vn_src: np.ndarray
    vn_rec: np.ndarray

    @property
    def ntx(self):
        return self.dir.shape[1]

    @property
    def nt(self):
        return self.vn_src.shape[0]

    def copy(self):
        return TxGrid([a.copy(order="F") for a in self.idx], [a.copy(order="F") for a in self.w],
                      [a.copy(order="F") for a in self.src], [a.copy(order="F") for a in self.rec],
                      self.dir.copy(order="F"), self.vn_src.copy(order="F"),
                      self.vn_rec.copy(order="F"))

    def _c(self):
        g = _TxGrid()
        g.ntx, g.nt = self.ntx, self.nt
        for c in range(4):
            g.idx[c] = self.idx[c].ctypes.data
            g.w[c] = self.w[c].ctypes.data
            g.src[c] = self.src[c].ctypes.data
            g.rec[c] = self.rec[c].ctypes.data
        g.dir = self.dir.ctypes.data
        g.vn_src = self.vn_src.ctypes.data
        g.vn_rec = self.vn_rec.ctypes.data
        return g


def transceivers_to_grid(d: Domain, points, directions, tfs) -> TxGrid:
    """points (ntx,3), directions (ntx,4), tfs (ntx, nt) Float64."""
    points = np.asarray(points, np.float64)
    directions = np.asarray(directions, np.float64)
    ntx = points.shape[0]
    nt = d.nt
    tfs = np.asarray(tfs, np.float64)
    P = np.ascontiguousarray(points.reshape(ntx, 3))          # (3, ntx) col-major
    D = np.ascontiguousarray(directions.reshape(ntx, 4))      # (4, ntx) col-major
    T = np.asfortranarray(tfs.reshape(ntx, nt).T)             # (nt, ntx)
    g = TxGrid([np.zeros((3, ntx), np.float32, order="F") for _ in range(4)],
               [np.zeros((2, 2, 2, ntx), np.float32, order="F") for _ in range(4)],
               [np.zeros((nt, ntx), np.float32, order="F") for _ in range(4)],
               [np.zeros((nt, ntx), np.float32, order="F") for _ in range(4)],
               np.zeros((4, ntx), np.float32, order="F"),
               np.zeros((nt, ntx), np.float32, order="F"),
               np.zeros((nt, ntx), np.float32, order="F"))
    cg = g._c()
    _chk(lib().or_pack_transceivers(C.byref(d), _p(P), _p(D), _p(T), C.byref(cg)), "pack")
    return g


class CpmlState:
    """Cpml memory variables (src/simulation.jl:200-227) in Julia layout."""

    def __init__(self, d: Domain, npml: int, rcoef=1e-4, fc=3e3):
        self.npml = npml
        dims = [d.nx, d.ny, d.nz]
        self.mv, self.mp = [], []
        for ax in range(3):
            sv = dims.copy(); sv[ax] = npml
            sp = dims.copy(); sp[ax] = npml + 1
            self.mv.append(np.zeros(sv + [2], np.float32, order="F"))
            self.mp.append(np.zeros(sp + [2], np.float32, order="F"))
        prof = cpml_coefficients(npml, d.c0, d.dt, rcoef, d.dx * npml, fc)
        self.profiles64 = prof
        self.coef = np.concatenate([p.astype(np.float32) for p in prof])

    def copy(self):
        c = object.__new__(CpmlState)
        c.npml = self.npml
        c.mv = [a.copy(order="F") for a in self.mv]
        c.mp = [a.copy(order="F") for a in self.mp]
        c.profiles64 = self.profiles64
        c.coef = self.coef.copy()
        return c

    def _c(self):
        s = _Cpml()
        s.npml = self.npml
        for a in range(3):
            s.mv[a] = self.mv[a].ctypes.data
            s.mp[a] = self.mp[a].ctypes.data
        s.coef = self.coef.ctypes.data
        return s


def run_fdtd(d: Domain, field, txs: TxGrid, cpml: CpmlState, mask=None, start_step=1,
             stop_step=None, mode="promote", nthreads=0):
    """run_fdtd! (src/simulation.jl:542-557): advances field/txs/cpml in place."""
    stop_step = d.nt if stop_step is None else stop_step
    assert field.flags.f_contiguous and field.dtype == np.float32
    assert field.shape == (d.nx, d.ny, d.nz, 4)
    cg = txs._c()
    cc = cpml._c() if cpml is not None else None
    _chk(lib().or_run_fdtd(C.byref(d), _p(field), C.byref(cg), C.byref(cc) if cc else None,
                           _p(mask) if mask is not None else None, start_step, stop_step,
                           MODES[mode], nthreads), "run_fdtd")
    return field


def transceivers_to_grid64(d: Domain, points, directions, tfs) -> TxGrid:
    """transceiversToGrid with Float64 weights and sources (the FP64 run's
    inputs): the weights of trilinearInterpolation and tf * direction
    unrounded; indices as in the Float32 grid."""
    points = np.asarray(points, np.float64).reshape(-1, 3)
    directions = np.asarray(directions, np.float64).reshape(-1, 4)
    ntx, nt = points.shape[0], d.nt
    tfs = np.asarray(tfs, np.float64).reshape(ntx, nt)
    idx = [np.zeros((3, ntx), np.float32, order="F") for _ in range(4)]
    w = [np.zeros((2, 2, 2, ntx), np.float64, order="F") for _ in range(4)]
    for i in range(ntx):
        ii, ww = trilinear(d, points[i])
        for c in range(4):
            idx[c][:, i] = ii[:, c]
            w[c][..., i] = ww[..., c]
    src = [np.asfortranarray((tfs * directions[:, c:c + 1]).T) for c in range(4)]
    rec = [np.zeros((nt, ntx), np.float64, order="F") for _ in range(4)]
    return TxGrid(idx, w, src, rec, np.asfortranarray(directions.T),
                  np.zeros((nt, ntx), np.float64, order="F"),
                  np.zeros((nt, ntx), np.float64, order="F"))


class CpmlState64(CpmlState):
    """Cpml memory and coefficients in Float64 (the FP64 run)."""

    def __init__(self, d: Domain, npml: int, rcoef=1e-4, fc=3e3):
        super().__init__(d, npml, rcoef, fc)
        self.mv = [a.astype(np.float64, order="F") for a in self.mv]
        self.mp = [a.astype(np.float64, order="F") for a in self.mp]
        self.coef = np.concatenate([np.asarray(p, np.float64) for p in self.profiles64])


def run_fdtd64(d: Domain, field, txs: TxGrid, cpml: CpmlState64, mask=None, start_step=1,
               stop_step=None, nthreads=0):
    """run_fdtd! with every array in Float64 (or_run_fdtd64): the reference
    algorithm without Float32 rounding, for error statements."""
    stop_step = d.nt if stop_step is None else stop_step
    assert field.flags.f_contiguous and field.dtype == np.float64
    assert field.shape == (d.nx, d.ny, d.nz, 4)
    assert txs.w[0].dtype == np.float64 and txs.src[0].dtype == np.float64
    cg = txs._c()
    cc = cpml._c() if cpml is not None else None
    if cc is not None:
        assert cpml.coef.dtype == np.float64 and cpml.mv[0].dtype == np.float64
    _chk(lib().or_run_fdtd64(C.byref(d), _p(field), C.byref(cg), C.byref(cc) if cc else None,
                             _p(mask) if mask is not None else None, start_step, stop_step,
                             nthreads), "run_fdtd64")
    return field


def run_fdtd_gf(d: Domain, field, txs: TxGrid, cpml: CpmlState, mask, kind, tensors, i_src,
                i_rec, z0, discard=False, start_step=1, stop_step=None, mode="promote",
                nthreads=0):
    """run_fdtd!(...; gf_map) with the in-loop GF extrapolation
    (extrapolation.jl:36-249).  kind: "PVFromPin" (tensors p_pin, v_pin),
    "PFromPin" (pos, neg) or "PVFromPV" (pp, pv, vp, vv), each (nt_gf, n1, n2)
    float32; i_src, i_rec 1-based transceiver indices."""
    stop_step = d.nt if stop_step is None else stop_step
    assert field.flags.f_contiguous and field.dtype == np.float32
    ts = [np.asfortranarray(t, np.float32) for t in tensors]
    isr = np.ascontiguousarray(i_src, np.int64)
    irc = np.ascontiguousarray(i_rec, np.int64)
    g = _GfMap(kind=GF_KINDS[kind], nt_gf=ts[0].shape[0], n1=ts[0].shape[1], n2=ts[0].shape[2],
               i_src=isr.ctypes.data, n_src=isr.size, i_rec=irc.ctypes.data, n_rec=irc.size,
               z0=z0, discard=int(bool(discard)))
    for k, t in enumerate(ts):
        g.t[k] = t.ctypes.data
    cg = txs._c()
    cc = cpml._c() if cpml is not None else None
    _chk(lib().or_run_fdtd_gf(C.byref(d), _p(field), C.byref(cg), C.byref(cc) if cc else None,
                              _p(mask) if mask is not None else None, start_step, stop_step,
                              MODES[mode], C.byref(g), nthreads), "run_fdtd_gf")
    return field


def kh_eval_kernel(which, outer_pts, outer_nrm, inner_pts, inner_nrm, t_grid, sigma, c0, rho,
                   nthreads=0):
    no, ni, ntk = outer_pts.shape[0], inner_pts.shape[0], len(t_grid)
    K = np.zeros((ntk, no, ni), np.float32, order="F")
    f = lambda a: np.asfortranarray(a, np.float64)
    _chk(lib().or_kh_eval_kernel(which, no, _p(f(outer_pts)), _p(f(outer_nrm)), ni,
                                 _p(f(inner_pts)), _p(f(inner_nrm)), ntk,
                                 _p(np.ascontiguousarray(t_grid, np.float64)), sigma, c0, rho,
                                 _p(K), nthreads), "kh_eval")
    return K


def kh_accumulate(out, K, inp, alpha=1.0, K_dc=None, cumsum_in=None, nthreads=0):
    ntk, no, ni = K.shape
    nt = out.shape[0]
    _chk(lib().or_kh_accumulate(_p(out), nt, _p(K), ntk, no, ni, _p(inp), alpha,
                                _p(K_dc) if K_dc is not None else None,
                                _p(cumsum_in) if cumsum_in is not None else None, nthreads),
         "kh_acc")
    return out


def kh_pressure(s_pts, s_nrm, r_pts, in_q, in_f, dt, sigma, c0, aq, af, ntk=None, r_begin=0,
                r_end=None, mode=1, nthreads=0):
    """FP64 oracle of the two-way KH pressure sum; in_q/in_f are (nt, ns) Float32."""
    ns, nr = s_pts.shape[0], r_pts.shape[0]
    nt = in_q.shape[0]
    ntk = nt if ntk is None else ntk
    r_end = nr if r_end is None else r_end
    out = np.zeros((nt, r_end - r_begin), np.float64, order="F")
    f = lambda a: np.asfortranarray(a, np.float64)
    g = lambda a: np.asfortranarray(a, np.float32)
    _chk(lib().or_kh_pressure(ns, _p(f(s_pts)), _p(f(s_nrm)), nr, _p(f(r_pts)), nt, ntk, dt,
                              sigma, c0, _p(g(in_q)), _p(g(in_f)), aq, af, mode, r_begin, r_end,
                              _p(out), nthreads), "kh_pressure")
    return out


def kh_velocity(s_pts, s_nrm, r_pts, r_nrm, in_q, in_f, dt, sigma, c0, rho, aq, af, r_begin=0,
                r_end=None, nthreads=0):
    """FP64 oracle of the two-way KH normal velocity (v_p, v_v kernels with the
    v_v pedestal); in_q/in_f are (nt, ns) Float32."""
    ns, nr = s_pts.shape[0], r_pts.shape[0]
    nt = in_q.shape[0]
    r_end = nr if r_end is None else r_end
    out = np.zeros((nt, r_end - r_begin), np.float64, order="F")
    f = lambda a: np.asfortranarray(a, np.float64)
    g = lambda a: np.asfortranarray(a, np.float32)
    _chk(lib().or_kh_velocity(ns, _p(f(s_pts)), _p(f(s_nrm)), nr, _p(f(r_pts)), _p(f(r_nrm)), nt,
                              dt, sigma, c0, rho, _p(g(in_q)), _p(g(in_f)), aq, af, r_begin, r_end,
                              _p(out), nthreads), "kh_velocity")
    return out


def gf_postprocess(a, t_in0, dt_in, nt_out, t_out0, dt_out, unit=1.0, denoise=True):
    """impulsive_gfs post-processing (denoise, cubic B-spline resample,
    physical units) of a (nt_in, ncol) float32 array -> (nt_out, ncol)."""
    a = np.asfortranarray(a, np.float32)
    out = np.zeros((nt_out, a.shape[1]), np.float32, order="F")
    _chk(lib().or_gf_postprocess(a.shape[1], a.shape[0], t_in0, dt_in, nt_out, t_out0, dt_out,
                                 _p(a), _p(out), unit, int(bool(denoise))), "gf_postprocess")
    return out


def extrapolate_pv_from_pin(pin, p_src, v_src, pp, vp, it):
    nt, nrec = pin.shape
    nt_gf, nsrc, _ = pp.shape
    _chk(lib().or_extrapolate_pv_from_pin(_p(pin), nt, nrec, _p(p_src), _p(v_src), nsrc,
                                          _p(pp), _p(vp), nt_gf, it), "extrapolate")
