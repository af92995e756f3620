"""Python mirror of the reference's FDTD/KH entry points over libadfdtd.so.

Names, argument meaning and array layouts follow the reference Julia API
(AcousticDisguising: src/simulation.jl, src/geometry.jl, src/illumination.jl,
src/greens.jl, src/kh_kernels.jl) so that host code reads the same way:
numpy arrays are Fortran-ordered with the reference's shapes, e.g. the field
is (nx, ny, nz, 4) Float32 and trace buffers are (nt, ntx).

Every compute call goes through the C-ABI; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import math
import mmap
import threading
import weakref
from dataclasses import dataclass, field as dc_field

import numpy as np

from . import _lib as L

_ctx_lock = threading.Lock()
_ctx = None


class Context:
    """One adf_ctx (device, stream, HBM budget)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        h = C.c_void_p()
        L.check(L.lib().adf_ctx_create(device, hbm_budget, C.byref(h)), "adf_ctx_create")
        self.h = h

    def close(self):
        if self.h:
            L.lib().adf_ctx_destroy(self.h)
            self.h = None

    def set_kernel_timing(self, on: bool):
        L.check(L.lib().adf_set_kernel_timing(self.h, int(bool(on))), "set_kernel_timing")

    def kernel_timing(self, reset: bool = False):
        ms = C.c_double()
        n = C.c_int64()
        L.check(L.lib().adf_kernel_timing(self.h, C.byref(ms), C.byref(n), int(reset)),
                "kernel_timing")
        return ms.value, n.value

    def last_io_bytes(self):
        h = C.c_int64()
        d = C.c_int64()
        L.check(L.lib().adf_last_io_bytes(self.h, C.byref(h), C.byref(d)), "last_io_bytes")
        return h.value, d.value

    def last_timing(self):
        ms = C.c_double()
        n = C.c_int64()
        L.check(L.lib().adf_last_timing(self.h, C.byref(ms), C.byref(n)), "adf_last_timing")
        return ms.value, n.value

    def step_resident_ctas(self) -> int:
        """Step-kernel CTAs the GPU holds at once (one wave)."""
        n = C.c_int64()
        L.check(L.lib().adf_step_resident_ctas(self.h, C.byref(n)), "step_resident_ctas")
        return n.value

    def last_kh_ms(self) -> float:
        """Kernel time of the last KH extrapolation on this context."""
        ms = C.c_double()
        L.check(L.lib().adf_last_kh_ms(self.h, C.byref(ms)), "adf_last_kh_ms")
        return ms.value


def default_context() -> Context:
    global _ctx
    with _ctx_lock:
        if _ctx is None:
            _ctx = Context(0)
        return _ctx


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------------------
# Domain and coordinates (src/simulation.jl:25-115)
# ---------------------------------------------------------------------------
def Domain(tmax=10e-4, xmax=1.0, ymax=None, zmax=None, nx=201, ny=None, nz=None, c0=1500.0,
           r0=1000.0, cf=0.25) -> L.Domain:
    ymax = xmax if ymax is None else ymax
    zmax = xmax if zmax is None else zmax
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    d = L.Domain()
    L.check(L.lib().adf_domain_make(float(tmax), float(xmax), float(ymax), float(zmax), int(nx),
                                    int(ny), int(nz), float(c0), float(r0), float(cf),
                                    C.byref(d)), "Domain")
    return d


def coord(d: L.Domain, axis: int, chan: int) -> np.ndarray:
    """coords(d)[axis][chan]; axis 0..2 = x,y,z, chan 0..3 = p,vx,vy,vz."""
    n = [d.nx, d.ny, d.nz][axis]
    out = np.empty(n, np.float64)
    L.check(L.lib().adf_coords(C.byref(d), axis, chan, _p(out)), "coords")
    return out


def coords(d: L.Domain) -> dict:
    keys = ("p", "vx", "vy", "vz")
    return {ax: {k: coord(d, a, c) for c, k in enumerate(keys)}
            for a, ax in enumerate(("x", "y", "z"))}


def t(d: L.Domain) -> np.ndarray:
    """t(d) = range(0; stop=tmax, length=nt) (simulation.jl:86), the Julia
    range values.  The step is tmax/(nt-1), not dt, as in the reference."""
    out = np.empty(int(d.nt), np.float64)
    L.check(L.lib().adf_time_axis(C.byref(d), _p(out)), "t")
    return out


# ---------------------------------------------------------------------------
# Illumination helpers (src/illumination.jl)
# ---------------------------------------------------------------------------
def fibonacci_sphere(n: int, radius: float = 1.0):
    """fibonacci_sphere (illumination.jl:19-46): (points, normals), (n,3)."""
    i = np.arange(n, dtype=np.float64)
    z = 1.0 - (2.0 * i + 1.0) / n
    rxy = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    th = (math.pi * (3.0 - math.sqrt(5.0))) * i
    nrm = np.stack([rxy * np.cos(th), rxy * np.sin(th), z], axis=1)
    return radius * nrm, nrm


def impulsive_wavelet(d: L.Domain, f_3db_hz: float):
    """impulsive_wavelet (illumination.jl:167-184): (tf, timeshift)."""
    sig = math.sqrt(math.log(2.0)) / (2 * math.pi * float(f_3db_hz))
    plen = int(round(10 * sig / d.dt))
    pl = min(plen, int(d.nt))
    pc, pw = pl / 2, pl / 10
    tf = np.zeros(int(d.nt), np.float64)
    u = np.arange(1, pl + 1, dtype=np.float64) - pc
    tf[:pl] = np.exp(-(u * u) / (2 * (pw * pw)))
    tf /= tf.sum() * d.dt
    return tf, pc * d.dt


def ricker_wavelet(d: L.Domain, fc: float = 18_000.0, injection: bool = True):
    """ricker_wavelet (illumination.jl:199-207)."""
    wn = math.pi * fc * (t(d) - 1.0 / fc)
    tf = (1.0 - 2.0 * wn * wn) * np.exp(-(wn * wn))
    if injection:
        tf = np.cumsum(tf) * (d.dt / d.dx)
    return tf


def fib_sphere_area(radius: float, n_points: int) -> float:
    """fib_sphere_area (src/io.jl:131)."""
    return 4 * math.pi * radius ** 2 / n_points


# ---------------------------------------------------------------------------
# CPML (src/simulation.jl:200-241, src/kernels/cpmlcoeffs.jl)
# ---------------------------------------------------------------------------
def cpml_profiles(npml: int, vel_max: float, dt: float, rcoef: float, thickness: float, fc: float,
                  ctx: Context | None = None):
    """compute_CPML_coefficients! on the GPU in FP64; returns (float32[8n+4],
    float64[8n+4]) in the order a_l a_r a_hl a_hr b_l b_r b_hl b_hr."""
    ctx = ctx or default_context()
    o32 = np.zeros(8 * npml + 4, np.float32)
    o64 = np.zeros(8 * npml + 4, np.float64)
    L.check(L.lib().adf_cpml_profiles(ctx.h, npml, vel_max, dt, rcoef, thickness, fc, _p(o32),
                                      _p(o64)), "cpml_profiles")
    return o32, o64


def static_cpml_max_npml() -> int:
    """The largest npml cpml_profiles_static accepts (read from the library)."""
    return int(L.lib().adf_static_cpml_max_npml())


def cpml_profiles_static(npml: int, vel_max: float, dt: float, rcoef: float, thickness: float,
                         fc: float, ctx: Context | None = None):
    """cpml_profiles through adf_cpml_profiles_static: the same values, computed
    with fixed device scratch (npml <= static_cpml_max_npml()) and no device
    allocation.  The first call per device sets the scratch up, so make it
    before any stream capture; concurrent calls on one device race."""
    ctx = ctx or default_context()
    o32 = np.zeros(8 * npml + 4, np.float32)
    o64 = np.zeros(8 * npml + 4, np.float64)
    L.check(L.lib().adf_cpml_profiles_static(ctx.h, npml, vel_max, dt, rcoef, thickness, fc,
                                             _p(o32), _p(o64)), "cpml_profiles_static")
    return o32, o64


def split_profiles(flat: np.ndarray, npml: int) -> dict:
    n = npml
    sizes = [("a_l", n), ("a_r", n), ("a_hl", n + 1), ("a_hr", n + 1), ("b_l", n), ("b_r", n),
             ("b_hl", n + 1), ("b_hr", n + 1)]
    out, o = {}, 0
    for k, s in sizes:
        out[k] = flat[o:o + s]
        o += s
    return out


class Cpml:
    """`Cpml(d; npml, rcoef, fc)`: memory variables (Julia layout) + Float32
    coefficients.  `mv[a]`/`mp[a]` are the reference's `cpml.v[a]`/`cpml.p[a]`."""

    def __init__(self, d: L.Domain, npml: int, rcoef: float = 1e-4, fc: float = 3e3,
                 ctx: Context | None = None):
        self.n = npml
        dims = [d.nx, d.ny, d.nz]
        self.mv, self.mp = [], []
        for a in range(3):
            sv = list(dims); sv[a] = npml
            sp = list(dims); sp[a] = npml + 1
            self.mv.append(np.zeros(sv + [2], np.float32, order="F"))
            self.mp.append(np.zeros(sp + [2], np.float32, order="F"))
        self.coef, self.coef64 = cpml_profiles(npml, d.c0, d.dt, rcoef, d.dx * npml, fc, ctx)

    def reset(self):
        """resetCPMLmemory! (simulation.jl:235-241)."""
        for a in self.mv + self.mp:
            a[...] = 0

    def _c(self):
        s = L.CpmlC()
        s.npml = self.n
        for a in range(3):
            s.mv[a] = self.mv[a].ctypes.data
            s.mp[a] = self.mp[a].ctypes.data
        s.coef = self.coef.ctypes.data
        return s


# ---------------------------------------------------------------------------
# Geometry (src/geometry.jl)
# ---------------------------------------------------------------------------
def shape_params(scatterer: str, radius=None, length=None, semi_axes=None,
                 center=(0.0, 0.0, 0.0)) -> np.ndarray:
    p = np.zeros(6, np.float64)
    if scatterer == "sphere":
        p[0] = radius
        p[1:4] = center
    elif scatterer == "cube":
        p[0] = length
        p[1:4] = center
    elif scatterer == "cross":
        p[0] = length
    elif scatterer == "ellipsoid":
        p[0:3] = semi_axes
        p[3:6] = center
    return p


def build_update_mask(d: L.Domain, scatterer: str, ctx: Context | None = None, **kw):
    """build_update_mask (geometry.jl:250-280) -> (nx,ny,nz,4) bool or None."""
    if scatterer == "none":
        return None
    ctx = ctx or default_context()
    out = np.zeros((d.nx, d.ny, d.nz, 4), np.uint8, order="F")
    L.check(L.lib().adf_build_mask(ctx.h, C.byref(d), L.SHAPES[scatterer],
                                   _p(shape_params(scatterer, **kw)), _p(out)), "build_update_mask")
    return out.astype(bool)


# ---------------------------------------------------------------------------
# Transceivers (src/simulation.jl:168-187, 347-452)
# ---------------------------------------------------------------------------
@dataclass
class Transceiver:
    """Transceiver(d; point, direction, tf); direction = [q, fx, fy, fz]."""

    point: np.ndarray
    direction: np.ndarray
    tf: np.ndarray


@dataclass
class TransceiverGrid:
    """Packed per-channel buffers, Julia layout (channel order p, vx, vy, vz)."""

    idx: list
    w: list
    src: list
    rec: list
    direction: np.ndarray
    vn_src: np.ndarray
    vn_rec: np.ndarray

    @property
    def ntx(self):
        return self.direction.shape[1]

    @property
    def nt(self):
        return self.vn_src.shape[0]

    def _c(self):
        g = L.TxGridC()
        g.ntx, g.nt = self.ntx, self.nt
        for c in range(4):
            g.idx[c] = self.idx[c].ctypes.data
            g.w[c] = self.w[c].ctypes.data
            g.src[c] = self.src[c].ctypes.data
            g.rec[c] = self.rec[c].ctypes.data
        g.dir = self.direction.ctypes.data
        g.vn_src = self.vn_src.ctypes.data
        g.vn_rec = self.vn_rec.ctypes.data
        return g

    def copy(self):
        cp = lambda a: a.copy(order="F")
        return TransceiverGrid([cp(a) for a in self.idx], [cp(a) for a in self.w],
                               [cp(a) for a in self.src], [cp(a) for a in self.rec],
                               cp(self.direction), cp(self.vn_src), cp(self.vn_rec))


def transceivers_to_grid(d: L.Domain, txs) -> TransceiverGrid:
    """transceiversToGrid (simulation.jl:387-431)."""
    ntx, nt = len(txs), int(d.nt)
    pts = np.ascontiguousarray([np.asarray(x.point, np.float64) for x in txs]).reshape(ntx, 3)
    dirs = np.ascontiguousarray([np.asarray(x.direction, np.float64) for x in txs]).reshape(ntx, 4)
    tf = np.asfortranarray(np.stack([np.asarray(x.tf, np.float64) for x in txs], axis=1))
    g = TransceiverGrid([np.zeros((3, ntx), np.float32, order="F") for _ in range(4)],
                        [np.zeros((2, 2, 2, ntx), np.float32, order="F") for _ in range(4)],
                        [np.zeros((nt, ntx), np.float32, order="F") for _ in range(4)],
                        [np.zeros((nt, ntx), np.float32, order="F") for _ in range(4)],
                        np.zeros((4, ntx), np.float32, order="F"),
                        np.zeros((nt, ntx), np.float32, order="F"),
                        np.zeros((nt, ntx), np.float32, order="F"))
    cg = g._c()
    L.check(L.lib().adf_pack_transceivers(C.byref(d), _p(pts), _p(dirs), _p(tf), C.byref(cg)),
            "transceiversToGrid")
    return g


def p_src(g: TransceiverGrid):
    return g.src[0]


def p_rec(g: TransceiverGrid):
    return g.rec[0]


def vn_src(g: TransceiverGrid):
    return g.vn_src


def vn_rec(g: TransceiverGrid):
    return g.vn_rec


# ---------------------------------------------------------------------------
# Time stepping (src/simulation.jl:542-557)
# ---------------------------------------------------------------------------
@dataclass
class GfMap:
    """A GFMap of run_fdtd!(...; gf_map) (src/kernels/extrapolation.jl:36-87).
    kind "PVFromPin": tensors (p_pin, v_pin), each (nt_gf, #iSrc, #iRec);
    kind "PFromPin": (pos, neg), each (nt_gf, #iRec, #iSrc);
    kind "PVFromPV": (pp, pv, vp, vv), each (nt_gf, #iRec, #iSrc).
    i_src / i_rec are 1-based transceiver indices.  discard=True reproduces
    the reference as shipped, whose extrapolate! writes into slice copies so
    the sources never change.  contraction "fp64" (default) sums every lag
    with Float64 FMAs, as the reference accumulates; "tf32x3" sums the lags
    older than the current 32-step block on the tensor cores (the two
    *FromPin kinds; TF32 split into three products, within about 1e-6 of the
    Float64 sums), keeping the map a second time as operand tiles."""

    kind: str
    tensors: tuple
    i_src: np.ndarray
    i_rec: np.ndarray
    discard: bool = False
    contraction: str = "fp64"

    def _c(self, z0: float):
        self._t = [np.asfortranarray(t, np.float32) for t in self.tensors]
        self._is = np.ascontiguousarray(self.i_src, np.int64)
        self._ir = np.ascontiguousarray(self.i_rec, np.int64)
        want = 4 if self.kind == "PVFromPV" else 2
        if len(self._t) != want or any(t.shape != self._t[0].shape or t.ndim != 3
                                         for t in self._t):
            raise ValueError(f"{self.kind} takes {want} tensors of one shape (nt_gf, n1, n2)")
        g = L.GfMapC(kind=L.GF_KINDS[self.kind], nt_gf=self._t[0].shape[0],
                     n1=self._t[0].shape[1], n2=self._t[0].shape[2], i_src=self._is.ctypes.data,
                     n_src=self._is.size, i_rec=self._ir.ctypes.data, n_rec=self._ir.size,
                     z0=float(z0), discard=int(bool(self.discard)),
                     contraction=L.GF_CONTRACTIONS[self.contraction])
        for k, t in enumerate(self._t):
            g.t[k] = t.ctypes.data
        return g


def PVFromPin(p_pin, v_pin, i_src, i_rec, discard=False, contraction="fp64") -> GfMap:
    return GfMap("PVFromPin", (p_pin, v_pin), i_src, i_rec, discard, contraction)


def PFromPin(pos, neg, i_src, i_rec, discard=False, contraction="fp64") -> GfMap:
    return GfMap("PFromPin", (pos, neg), i_src, i_rec, discard, contraction)


def PVFromPV(pp, pv, vp, vv, i_src, i_rec, discard=False) -> GfMap:
    return GfMap("PVFromPV", (pp, pv, vp, vv), i_src, i_rec, discard)


def run_fdtd(d: L.Domain, field: np.ndarray, txs: TransceiverGrid, cpml: Cpml | None, va=None,
             start_step: int = 1, on_step=None, stop_step: int | None = None,
             arith: str = "promote", ctx: Context | None = None,
             gf_map: GfMap | None = None) -> np.ndarray:
    """run_fdtd!(dom, field, txs, cpml, va; start_step, on_step, gf_map):
    advances `field` (and the trace buffers and CPML memory) in place on the
    GPU.  on_step(it, read) is called after each step; read(c) returns
    channel c.  gf_map drives the in-loop GF extrapolation."""
    ctx = ctx or default_context()
    stop_step = int(d.nt) if stop_step is None else int(stop_step)
    if field.dtype != np.float32 or not field.flags.f_contiguous:
        raise ValueError("field must be a Fortran-ordered float32 array")
    if field.shape != (d.nx, d.ny, d.nz, 4):
        raise ValueError("field shape must be (nx, ny, nz, 4)")
    mask = None
    if va is not None:
        mask = np.asfortranarray(va, dtype=np.uint8)
    cg = txs._c()
    cc = cpml._c() if cpml is not None else None
    cb = L.STEP_CB()
    if on_step is not None:
        def _cb(it, _user):
            def read(c):
                out = np.zeros((d.nx, d.ny, d.nz), np.float32, order="F")
                L.check(L.lib().adf_read_field(ctx.h, c, _p(out)), "adf_read_field")
                return out
            try:
                r = on_step(int(it), read)
            except Exception:  # a failing callback cancels the run
                return 1
            return 1 if r is False else 0
        cb = L.STEP_CB(_cb)
    if gf_map is not None:
        gm = gf_map._c(d.z0)
        L.check(L.lib().adf_run_fdtd_gf(ctx.h, C.byref(d), _p(field), C.byref(cg),
                                        C.byref(cc) if cc is not None else None, _p(mask),
                                        int(start_step), stop_step, L.ARITH[arith],
                                        C.byref(gm), cb, None), "run_fdtd_gf")
        return field
    L.check(L.lib().adf_run_fdtd(ctx.h, C.byref(d), _p(field), C.byref(cg),
                                 C.byref(cc) if cc is not None else None, _p(mask),
                                 int(start_step), stop_step, L.ARITH[arith], cb, None),
            "run_fdtd")
    return field


def run_fdtd_kh(d: L.Domain, field: np.ndarray, txs: TransceiverGrid, cpml: Cpml | None,
                va, surface_cols, s_pts, s_nrm, r_pts, sigma: float, aq: float, af: float,
                nt: int | None = None, window_sigmas: float = 6.0, arith: str = "promote",
                ctx: Context | None = None, out: np.ndarray | None = None) -> np.ndarray:
    """build_hologram's run_fdtd! followed by the two-way KH pressure of its
    recorded shell (part3_kh_extrapolation.jl:168-185) in one call:
    out[t, r] = aq sum_s p_p(s,r) (*) vn[:, s] + af sum_s p_v(s,r) (*) p[:, s]
    over the transceivers `surface_cols` (1-based; s_pts, s_nrm their points
    and outward normals), targets r_pts, rows 1..nt (default dom.nt).  The
    traces stay in HBM between the two.  `field`, `txs` and `cpml` are
    advanced in place as by run_fdtd.  Returns out (nt, nr) Float32."""
    ctx = ctx or default_context()
    if field.dtype != np.float32 or not field.flags.f_contiguous:
        raise ValueError("field must be a Fortran-ordered float32 array")
    if field.shape != (d.nx, d.ny, d.nz, 4):
        raise ValueError("field shape must be (nx, ny, nz, 4)")
    nt = int(d.nt) if nt is None else int(nt)
    cols = np.ascontiguousarray(surface_cols, np.int64)
    sp = np.asfortranarray(s_pts, np.float64)
    sn = np.asfortranarray(s_nrm, np.float64)
    rp = np.asfortranarray(r_pts, np.float64)
    ns, nr = sp.shape[0], rp.shape[0]
    if cols.shape != (ns,) or sn.shape != (ns, 3) or rp.shape[1] != 3:
        raise ValueError("run_fdtd_kh: shape mismatch")
    desc = L.KhDescC(ns=ns, nr=nr, nt=nt, dt=d.dt, sigma=sigma, c0=d.c0, rho=d.r0, aq=aq, af=af,
                     window_sigmas=window_sigmas, s_pts=sp.ctypes.data, s_nrm=sn.ctypes.data,
                     r_pts=rp.ctypes.data)
    out = _kh_out(out, nt, nr, "run_fdtd_kh")
    mask = None if va is None else np.asfortranarray(va, dtype=np.uint8)
    cg = txs._c()
    cc = cpml._c() if cpml is not None else None
    L.check(L.lib().adf_run_fdtd_kh(ctx.h, C.byref(d), _p(field), C.byref(cg),
                                    C.byref(cc) if cc is not None else None, _p(mask), 1,
                                    int(d.nt), L.ARITH[arith], C.byref(desc), _p(cols), _p(out)),
            "run_fdtd_kh")
    return out


def injection_coefficients(d: L.Domain, radius: float, n_points: int,
                           ctx: Context | None = None):
    """C_for_N on the GPU in FP64 -> (C_f, C_q, dS)."""
    ctx = ctx or default_context()
    out = np.zeros(3, np.float64)
    L.check(L.lib().adf_injection_coefficients(ctx.h, C.byref(d), float(radius), int(n_points),
                                               _p(out)), "injection_coefficients")
    return float(out[0]), float(out[1]), float(out[2])


# ---------------------------------------------------------------------------
# Kirchhoff-Helmholtz extrapolation (src/kh_kernels.jl:106-157, 256-296)
# ---------------------------------------------------------------------------
def _kh_out(out, nt, nr, name):
    """The caller's output array, or a new one (nt, nr) Float32 column-major."""
    if out is None:
        return np.zeros((nt, nr), np.float32, order="F")
    if out.dtype != np.float32 or out.shape != (nt, nr) or not out.flags.f_contiguous:
        raise ValueError(f"{name}: out must be a Fortran-ordered float32 ({nt}, {nr}) array")
    return out


def kh_pressure(s_pts, s_nrm, r_pts, in_q, in_f, dt: float, sigma: float, c0: float,
                aq: float, af: float, rho: float = 1.2, window_sigmas: float = 6.0,
                ctx: Context | None = None, out: np.ndarray | None = None) -> np.ndarray:
    """Two-way KH pressure at targets:
    out[t, r] = aq sum_s p_p(s,r) (*) in_q[:, s] + af sum_s p_v(s,r) (*) in_f[:, s]
    with the Gaussian kernels of eval_one_kernel (kh_kernels.jl:106-157).
    s_pts, s_nrm (ns, 3), r_pts (nr, 3) Float64; in_q, in_f (nt, ns) Float32.
    Returns out (nt, nr) Float32, Julia (column-major) layout (written into
    `out` when given, e.g. a pinned_zeros buffer reused across calls)."""
    ctx = ctx or default_context()
    f64 = lambda a: np.asfortranarray(a, np.float64)
    f32 = lambda a: np.asfortranarray(a, np.float32)
    sp, sn, rp = f64(s_pts), f64(s_nrm), f64(r_pts)
    q, f = f32(in_q), f32(in_f)
    ns, nr, nt = sp.shape[0], rp.shape[0], q.shape[0]
    if sn.shape != (ns, 3) or rp.shape[1] != 3 or q.shape != (nt, ns) or f.shape != (nt, ns):
        raise ValueError("kh_pressure: shape mismatch")
    desc = L.KhDescC(ns=ns, nr=nr, nt=nt, dt=dt, sigma=sigma, c0=c0, rho=rho, aq=aq, af=af,
                     window_sigmas=window_sigmas, s_pts=sp.ctypes.data, s_nrm=sn.ctypes.data,
                     r_pts=rp.ctypes.data)
    out = _kh_out(out, nt, nr, "kh_pressure")
    L.check(L.lib().adf_kh_pressure(ctx.h, C.byref(desc), _p(q), _p(f), _p(out)), "kh_pressure")
    return out


def kh_test_fault(skip_chunk: int, poll_limit: int, ctx: Context | None = None) -> None:
    """Arms the next kh_pressure / kh_velocity call on ctx (one shot): its
    device waits give up after `poll_limit` polls and the copies of staged
    chunk `skip_chunk` are never issued, so that chunk's wait runs out with
    nothing in flight and the call raises ADF_E_TIMEOUT (a test hook)."""
    ctx = ctx or default_context()
    L.check(L.lib().adf_kh_test_fault(ctx.h, int(skip_chunk), int(poll_limit)), "kh_test_fault")


def kh_velocity(s_pts, s_nrm, r_pts, r_nrm, in_q, in_f, dt: float, sigma: float, c0: float,
                aq: float, af: float, rho: float = 1.2, window_sigmas: float = 6.0,
                ctx: Context | None = None, out: np.ndarray | None = None) -> np.ndarray:
    """Two-way KH normal velocity at targets with normals r_nrm:
    out[t, r] = aq sum_s v_p(s,r) (*) in_q[:, s] + af sum_s v_v(s,r) (*) in_f[:, s]
    (eval_one_kernel's v_p, v_v, kh_kernels.jl:106-157; the non-decaying part
    of v_v is carried as its limit times the running sum of in_f)."""
    ctx = ctx or default_context()
    f64 = lambda a: np.asfortranarray(a, np.float64)
    f32 = lambda a: np.asfortranarray(a, np.float32)
    sp, sn, rp, rn = f64(s_pts), f64(s_nrm), f64(r_pts), f64(r_nrm)
    q, f = f32(in_q), f32(in_f)
    ns, nr, nt = sp.shape[0], rp.shape[0], q.shape[0]
    if (sn.shape != (ns, 3) or rp.shape[1] != 3 or rn.shape != rp.shape or
            q.shape != (nt, ns) or f.shape != (nt, ns)):
        raise ValueError("kh_velocity: shape mismatch")
    desc = L.KhDescC(ns=ns, nr=nr, nt=nt, dt=dt, sigma=sigma, c0=c0, rho=rho, aq=aq, af=af,
                     window_sigmas=window_sigmas, s_pts=sp.ctypes.data, s_nrm=sn.ctypes.data,
                     r_pts=rp.ctypes.data, r_nrm=rn.ctypes.data)
    out = _kh_out(out, nt, nr, "kh_velocity")
    L.check(L.lib().adf_kh_velocity(ctx.h, C.byref(desc), _p(q), _p(f), _p(out)), "kh_velocity")
    return out


def gf_postprocess(a, t_in0: float, dt_in: float, nt_out: int, t_out0: float, dt_out: float,
                   unit: float = 1.0, denoise: bool = True, ctx: Context | None = None):
    """impulsive_gfs post-processing on the GPU (greens.jl:174-190): denoise,
    cubic B-spline resampling onto t_out0 + k dt_out with the dt-ratio scale,
    division by `unit` (gf_to_physical's C_p / C_v).  a: (nt_in, ncol)."""
    ctx = ctx or default_context()
    a = np.asfortranarray(a, np.float32)
    out = np.zeros((nt_out, a.shape[1]), np.float32, order="F")
    L.check(L.lib().adf_gf_postprocess(ctx.h, a.shape[1], a.shape[0], t_in0, dt_in, nt_out,
                                       t_out0, dt_out, _p(a), _p(out), unit, int(bool(denoise))),
            "gf_postprocess")
    return out


def gf_unit_factors(d: L.Domain, dt_save: float):
    """gf_unit_factors (greens_io.jl:180-184): (C_p, C_v) of raw FDTD GFs."""
    C_p = d.dx ** 3 * dt_save / (d.dt ** 2 * d.c0 ** 2)
    C_v = -d.r0 * d.dx ** 3 * dt_save / d.dt ** 2
    return C_p, C_v


def fp32_fma_peak(ctx: Context | None = None):
    """Measured FP32 FMA throughput (TFLOP/s) and the probe's duration (ms)."""
    ctx = ctx or default_context()
    tf, ms = C.c_double(), C.c_double()
    L.check(L.lib().adf_fp32_fma_peak(ctx.h, C.byref(tf), C.byref(ms)), "fp32_fma_peak")
    return tf.value, ms.value


def fp64_fma_peak(ctx: Context | None = None):
    """Measured FP64 FMA throughput (TFLOP/s, ms of the probe)."""
    ctx = ctx or default_context()
    tf, ms = C.c_double(), C.c_double()
    L.check(L.lib().adf_fp64_fma_peak(ctx.h, C.byref(tf), C.byref(ms)), "fp64_fma_peak")
    return tf.value, ms.value


# ---------------------------------------------------------------------------
# Impulsive Green's-function solves (src/greens.jl:48-234)
# ---------------------------------------------------------------------------
@dataclass
class GfRequest:
    """One FDTD solve of impulsive_gfs: point source + receiver shell.

    `src_direction` is [q, fx, fy, fz] ([1,0,0,0] is the :p source type,
    [0, n] the :v type, greens.jl:154-155); receivers record p and v_n along
    their outward normals.  Outputs p and vn are (nt, n_rec) Float32.
    """

    dom: L.Domain
    src_point: np.ndarray
    src_direction: np.ndarray
    src_tf: np.ndarray
    rec_points: np.ndarray
    rec_normals: np.ndarray
    npml: int = 10
    pml_rcoef: float = 1e-4
    pml_fc: float = 3e3
    scatterer: str = "none"
    scatterer_kw: dict = dc_field(default_factory=dict)
    arith: str = "promote"
    p: np.ndarray = None
    vn: np.ndarray = None

    def _c(self):
        r = L.GfRequestC()
        r.dom = self.dom
        r.npml = int(self.npml)
        r.pml_rcoef = float(self.pml_rcoef)
        r.pml_fc = float(self.pml_fc)
        r.shape = L.SHAPES[self.scatterer]
        sp = shape_params(self.scatterer, **self.scatterer_kw)
        for i in range(6):
            r.shape_params[i] = sp[i]
        for i in range(3):
            r.src_point[i] = float(self.src_point[i])
        for i in range(4):
            r.src_dir[i] = float(self.src_direction[i])
        self._tf = np.ascontiguousarray(self.src_tf, np.float64)
        self._rp = np.ascontiguousarray(self.rec_points, np.float64).reshape(-1, 3)
        self._rn = np.ascontiguousarray(self.rec_normals, np.float64).reshape(-1, 3)
        n = self._rp.shape[0]
        nt = int(self.dom.nt)
        if self.p is None:
            self.p = np.zeros((nt, n), np.float32, order="F")
        if self.vn is None:
            self.vn = np.zeros((nt, n), np.float32, order="F")
        r.src_tf = self._tf.ctypes.data
        r.n_rec = n
        r.rec_points = self._rp.ctypes.data
        r.rec_normals = self._rn.ctypes.data
        r.flags = L.ARITH[self.arith]
        r.out_p = self.p.ctypes.data
        r.out_vn = self.vn.ctypes.data
        return r


def pinned_zeros(shape, dtype=np.float32, order: str = "F") -> np.ndarray:
    """A zero-filled host array page-locked for the library's copies
    (adf_host_pin), e.g. GfRequest.p / .vn buffers reused across
    gf_solve_batch calls; it is unpinned when the array is collected.  The
    array has pages of its own (page-aligned start, whole pages), since
    page-locking works on pages and two buffers sharing one could not both
    be registered."""
    dt = np.dtype(dtype)
    n = int(np.prod(shape, dtype=np.int64)) * dt.itemsize
    page = mmap.PAGESIZE
    span = max(page, (n + page - 1) // page * page)
    raw = np.zeros(span + page, np.uint8)
    off = (-raw.ctypes.data) % page
    buf = raw[off:off + span]
    a = np.ndarray(shape, dt, buffer=buf, order=order)
    L.check(L.lib().adf_host_pin(buf.ctypes.data, span), "host_pin")
    weakref.finalize(a, L.lib().adf_host_unpin, buf.ctypes.data)
    return a


def gf_solve_batch(reqs, batched: bool = True, ctx: Context | None = None):
    """Run GF solves: batched (one launch per step for all resident solves,
    graph-captured, HBM-budget admission) or the plain one-solve-per-launch
    path.  Fills req.p / req.vn; returns (device_ms, kernel_launches)."""
    ctx = ctx or default_context()
    arr = (L.GfRequestC * len(reqs))(*[r._c() for r in reqs])
    L.check(L.lib().adf_gf_solve_batch(ctx.h, len(reqs), arr, int(bool(batched))),
            "gf_solve_batch")
    return ctx.last_timing()


def autotune(nx: int, ny: int, nz: int, npml: int = 10, n_solves: int = 4, steps: int = 32,
             ctx: Context | None = None):
    """Times the step kernel's tile shapes on synthetic GF solves of this grid
    size and stores the fastest in the tune table; returns (ty, nzc, ms)."""
    ctx = ctx or default_context()
    ty, nzc, ms = C.c_int(), C.c_int(), C.c_double()
    L.check(L.lib().adf_autotune(ctx.h, nx, ny, nz, npml, n_solves, steps, C.byref(ty),
                                 C.byref(nzc), C.byref(ms)), "autotune")
    return ty.value, nzc.value, ms.value


def impulsive_gfs(d: L.Domain, src_positions, src_normals, rec_positions, rec_normals,
                  nt_gf: int, f_3db_hz: float, npml: int, pml_rcoef: float = 1e-4,
                  pml_fc: float = 3e3, scatterer: str = "none", scatterer_kw: dict | None = None,
                  arith: str = "promote", batch: int = 8, ctx: Context | None = None) -> dict:
    """impulsive_gfs (src/greens.jl:48-234) on the GPU: for every source point
    and source type (:p, direction [1,0,0,0]; :v, direction [0, normal]) one
    FDTD solve recording p and v_n at the receivers (batched through the GF
    engine), then per solve the post-processing of greens.jl:174-190 on the
    GPU (denoise, cubic B-spline resampling from the shifted FDTD axis
    range(-timeshift, tmax-timeshift, nt) onto range(0, tmax, nt_gf) with
    the dt-ratio scale).  Returns the raw-unit tensors p_p, p_v, v_p, v_v
    (nt_gf, n_rec, n_src) Float32 (first letter: receiver channel, second:
    source type), t, src_positions, rec_positions; gf_file.save_impulsive_gfs
    writes them in physical units."""
    ctx = ctx or default_context()
    sp = np.asarray(src_positions, np.float64).reshape(-1, 3)
    sn = np.asarray(src_normals, np.float64).reshape(-1, 3)
    rp = np.asarray(rec_positions, np.float64).reshape(-1, 3)
    rn = np.asarray(rec_normals, np.float64).reshape(-1, 3)
    n_src, n_rec, nt = sp.shape[0], rp.shape[0], int(d.nt)
    tf, timeshift = impulsive_wavelet(d, f_3db_hz)
    dt_in = float(d.tmax) / (nt - 1)       # step of range(-ts, tmax - ts; length = nt)
    dt_gf = float(d.tmax) / (nt_gf - 1)    # step of range(0, tmax; length = nt_gf)
    out = {k: np.zeros((nt_gf, n_rec, n_src), np.float32, order="F")
           for k in ("p_p", "p_v", "v_p", "v_v")}
    jobs = [(i, typ) for i in range(n_src) for typ in ("p", "v")]
    for b0 in range(0, len(jobs), max(1, batch)):
        chunk = jobs[b0:b0 + max(1, batch)]
        reqs = []
        for i, typ in chunk:
            direction = [1.0, 0.0, 0.0, 0.0] if typ == "p" else [0.0, *sn[i]]
            reqs.append(GfRequest(d, sp[i], direction, tf, rp, rn, npml=npml,
                                  pml_rcoef=pml_rcoef, pml_fc=pml_fc, scatterer=scatterer,
                                  scatterer_kw=dict(scatterer_kw or {}), arith=arith))
        gf_solve_batch(reqs, batched=True, ctx=ctx)
        for (i, typ), r in zip(chunk, reqs):
            A = np.concatenate([r.p, r.vn], axis=1)  # (nt, 2 n_rec): p then v_n columns
            R = gf_postprocess(A, -timeshift, dt_in, nt_gf, 0.0, dt_gf, unit=1.0, denoise=True,
                               ctx=ctx)
            out["p_" + typ][:, :, i] = R[:, :n_rec]
            out["v_" + typ][:, :, i] = R[:, n_rec:]
    out["t"] = np.linspace(0.0, float(d.tmax), nt_gf)
    out["src_positions"] = sp
    out["rec_positions"] = rp
    return out


class Server:
    """Continuous-batching serving loop (adf_server_*)."""

    def __init__(self, hbm_budget: int = 0, max_resident: int = 0, ctx: Context | None = None,
                 work_waves: float = 0.0):
        """work_waves > 0 admits requests only while the resident solves' step
        work stays within that many waves of the GPU's resident CTAs
        (adf_server_set_work_cap); 0 = HBM budget and max_resident only."""
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        L.check(L.lib().adf_server_start(self.ctx.h, hbm_budget, max_resident, C.byref(h)),
                "server_start")
        self.h = h
        self._keep = {}
        self.work_cap = 0
        if work_waves > 0:
            self.work_cap = max(1, int(round(work_waves * self.ctx.step_resident_ctas())))
            L.check(L.lib().adf_server_set_work_cap(self.h, self.work_cap), "server_set_work_cap")

    def submit(self, req: GfRequest) -> int:
        rc = req._c()
        i = C.c_int64()
        L.check(L.lib().adf_server_submit(self.h, C.byref(rc), C.byref(i)), "server_submit")
        self._keep[i.value] = (req, rc)
        return i.value

    def poll(self, rid: int):
        st = C.c_int()
        lat = C.c_double()
        L.check(L.lib().adf_server_poll(self.h, rid, C.byref(st), C.byref(lat)), "server_poll")
        return st.value, lat.value

    def cancel(self, rid: int):
        L.check(L.lib().adf_server_cancel(self.h, rid), "server_cancel")

    def drain(self):
        L.check(L.lib().adf_server_drain(self.h), "server_drain")

    def stop(self):
        if self.h:
            rc = L.lib().adf_server_stop(self.h)
            self.h = None
            L.check(rc, "server_stop")
