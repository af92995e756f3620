"""Green's-function files and the load_gf_ref scaling chain.

Schema (the reference's impulsive/analytical GF files, written by save_h5
(src/io.jl:229-242) from scripts/greens/impulsive.jl:116-124 and read by
_read_gf_ref_h5 (src/greens_io.jl:484-510)):

  datasets  p_p, p_v, v_p, v_v   Float32 (nt_gf, n_rec, n_src), physical units
            t                    Float64 (nt_gf)
            src_positions        Float64 (n_src, 3)
            rec_positions        Float64 (n_rec, 3)
  attrs     dom_dt, dom_dx, dom_tmax, scatterer, backend, n, nPoints_outer,
            nPoints_inner, n_done, created_at, elapsed_sec,
            units_convention = "physical", ...

libhdf5 is not available to this package, so files are written in a
self-describing container with the same dataset names, shapes (Julia
order), element types and attributes:

  bytes 0-7    b"ADFGF001"
  bytes 8-15   little-endian uint64: length L of the JSON header
  bytes 16-    JSON header {"datasets": {name: {"dtype", "shape", "offset"}},
               "attrs": {...}}, then every dataset's raw little-endian bytes,
               column-major (first index fastest), at header-relative offset

`to_hdf5(src, dst)` converts a container into an HDF5 file with h5py where
h5py is installed (datasets written so that Julia's HDF5.jl reads the same
shapes); `read_gf_file` also reads such HDF5 files when h5py is present.
"""
from __future__ import annotations

import json
import math
import struct

import numpy as np

MAGIC = b"ADFGF001"
_DT = {"float32": np.float32, "float64": np.float64, "int64": np.int64}


def write_gf_file(path: str, datasets: dict, attrs: dict | None = None) -> str:
    """Writes `datasets` ({name: ndarray}, Julia shapes) and `attrs`."""
    arrs, meta, off = [], {}, 0
    for name, a in datasets.items():
        a = np.asarray(a)
        dt = {np.dtype(np.float32): "float32", np.dtype(np.float64): "float64",
              np.dtype(np.int64): "int64"}.get(a.dtype)
        if dt is None:
            raise TypeError(f"write_gf_file: unsupported dtype {a.dtype} for {name}")
        raw = np.asfortranarray(a).tobytes(order="F")
        meta[name] = {"dtype": dt, "shape": list(a.shape), "offset": off}
        arrs.append(raw)
        off += len(raw)
    hdr = json.dumps({"datasets": meta, "attrs": dict(attrs or {})}).encode()
    with open(path + ".tmp", "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<Q", len(hdr)))
        f.write(hdr)
        for raw in arrs:
            f.write(raw)
    import os

    os.replace(path + ".tmp", path)
    return path


def read_gf_file(path: str):
    """Returns (datasets, attrs) of a container (or of an HDF5 file with h5py)."""
    with open(path, "rb") as f:
        head = f.read(8)
        if head != MAGIC:
            return _read_hdf5(path)
        (n,) = struct.unpack("<Q", f.read(8))
        hdr = json.loads(f.read(n).decode())
        base = 16 + n
        out = {}
        for name, m in hdr["datasets"].items():
            dt = np.dtype(_DT[m["dtype"]])
            cnt = int(np.prod(m["shape"])) if m["shape"] else 1
            f.seek(base + m["offset"])
            a = np.frombuffer(f.read(cnt * dt.itemsize), dtype=dt)
            out[name] = a.reshape(m["shape"], order="F").copy(order="F")
    return out, hdr["attrs"]


def _read_hdf5(path):
    try:
        import h5py
    except ImportError as e:  # pragma: no cover - depends on the installation
        raise ImportError(f"{path} is not a GF container and h5py is not installed") from e
    with h5py.File(path, "r") as f:  # HDF5.jl stores Julia arrays transposed
        ds = {k: np.asfortranarray(np.asarray(f[k]).T) for k in f.keys()}
        at = {k: (v.decode() if isinstance(v, bytes) else v) for k, v in f.attrs.items()}
    return ds, at


def to_hdf5(src: str, dst: str) -> str:
    """Container -> HDF5 (needs h5py), readable by the reference's loaders."""
    import h5py

    ds, at = read_gf_file(src)
    with h5py.File(dst, "w") as f:
        for k, a in ds.items():
            f[k] = np.ascontiguousarray(a.T)
        for k, v in at.items():
            f.attrs[k] = v
    return dst


def gf_unit_factors(dx: float, dt_fdtd: float, c0: float, r0: float, dt_save: float):
    """gf_unit_factors / _scaling_factors (src/greens_io.jl:146-184):
    C_p = dx^3 dt_save / (dt_fdtd^2 c0^2),  C_v = -r0 dx^3 dt_save / dt_fdtd^2."""
    return dx ** 3 * dt_save / (dt_fdtd ** 2 * c0 ** 2), -r0 * dx ** 3 * dt_save / dt_fdtd ** 2


def save_impulsive_gfs(path: str, p_p, p_v, v_p, v_v, t, src_positions, rec_positions, dom,
                       attrs: dict | None = None) -> str:
    """scripts/greens/impulsive.jl:111-124: the four raw GF tensors
    (nt_gf, n_rec, n_src) divided by C_p / C_v (gf_to_physical,
    src/greens_io.jl:195-205) and written with units_convention="physical"."""
    t = np.asarray(t, np.float64)
    C_p, C_v = gf_unit_factors(dom.dx, dom.dt, dom.c0, dom.r0, float(t[1] - t[0]))
    cp32, cv32 = np.float32(C_p), np.float32(C_v)
    pp = np.asfortranarray(np.asarray(p_p, np.float32) / cp32)
    pv = np.asfortranarray(np.asarray(p_v, np.float32) / cv32)
    vp = np.asfortranarray(np.asarray(v_p, np.float32) / cp32)
    vv = np.asfortranarray(np.asarray(v_v, np.float32) / cv32)
    n_done = int(sum(np.any(pp[:, :, k] != 0) for k in range(pp.shape[2])))
    a = {"dom_dt": float(dom.dt), "dom_dx": float(dom.dx), "dom_tmax": float(dom.tmax),
         "n_done": n_done, "units_convention": "physical", "backend": "B200"}
    a.update(attrs or {})
    return write_gf_file(path, {"p_p": pp, "p_v": pv, "v_p": vp, "v_v": vv, "t": t,
                                "src_positions": np.asarray(src_positions, np.float64),
                                "rec_positions": np.asarray(rec_positions, np.float64)}, a)


def _read_gf_ref(path):
    ds, at = read_gf_file(path)
    t = ds["t"]
    dom_dt = float(at["dom_dt"]) if "dom_dt" in at else float(t[1] - t[0])
    dom_dx = float(at["dom_dx"]) if "dom_dx" in at else math.nan
    gf = {"p": {"p": ds["p_p"].astype(np.float32), "v": ds["p_v"].astype(np.float32)},
          "v": {"p": ds["v_p"].astype(np.float32), "v": ds["v_v"].astype(np.float32)}, "t": t}
    return gf, dom_dt, dom_dx, at.get("units_convention", "")


def fib_sphere_area(radius: float, n_points: int) -> float:
    """fib_sphere_area (src/io.jl:131)."""
    return 4.0 * math.pi * radius ** 2 / n_points


def load_gf_ref(path: str, dom, radius_inner: float, n_inner: int, radius_outer: float,
                n_outer: int, scattered: bool = False, tmax: float = 0.0,
                homogeneous_path: str | None = None, extrap_type: str = "pv_from_pin",
                resample=None):
    """load_gf_ref (src/greens_io.jl:224-477) -> (kind, tensors) of a GFMap.

    Reads a physical-units GF file, subtracts the homogeneous companion for
    scattered-only content, multiplies by C_p / C_v, resamples every tensor
    onto 0:dom.dt:t_end with the cubic B-spline (`resample(a, t_in0, dt_in,
    nt_out, t_out0, dt_out)`, the GPU gf_postprocess by default), applies the
    FDTD-injection factor e, the impedance conversions of `extrap_type`, the
    surface weights, and forms the map's tensors.  kind is "PVFromPV",
    "PVFromPin" or "PFromPin"; tensors are Float32 (the reference keeps the
    *FromPin tensors in Float64: the difference is one Float32 rounding)."""
    if extrap_type not in ("pv_from_pin", "pv_from_pv", "p_from_pin"):
        raise ValueError(f"load_gf_ref: extrap_type must be pv_from_pin, pv_from_pv or "
                         f"p_from_pin; got {extrap_type!r}")
    if scattered and homogeneous_path is None:
        raise ValueError("load_gf_ref: scattered content needs homogeneous_path")
    if resample is None:
        from .api import gf_postprocess

        def resample(a, t_in0, dt_in, nt_out, t_out0, dt_out):
            return gf_postprocess(a, t_in0, dt_in, nt_out, t_out0, dt_out, unit=1.0,
                                  denoise=False)
    s_src = fib_sphere_area(radius_inner, n_inner)
    s_rec = fib_sphere_area(radius_outer, n_outer)
    gf, dom_dt, dom_dx, units = _read_gf_ref(path)
    if units != "physical":
        raise ValueError(f"load_gf_ref: {path} has units_convention={units!r}; expected "
                         "'physical'")
    if scattered:
        hom, _, _, _ = _read_gf_ref(homogeneous_path)
        for i in "pv":
            for j in "pv":
                gf[i][j] = gf[i][j] - hom[i][j]
        gf["t"] = hom["t"]
    t_raw = gf["t"]
    dt_in = float(t_raw[1] - t_raw[0])
    dt_out = float(dom.dt)
    t_end = float(tmax) if tmax > 0 else float(t_raw[-1])
    nt_out = int(math.floor(t_end / dt_out + 1e-9)) + 1  # 0:dt_out:t_end
    if math.isnan(dom_dx):
        raise ValueError("load_gf_ref: the GF file has no dom_dx attribute")
    C_p = dom_dx ** 3 * dt_in / (dom_dt ** 2 * dom.c0 ** 2)
    C_v = -dom.r0 * dom_dx ** 3 * dt_in / dom_dt ** 2
    gf["p"]["p"] = gf["p"]["p"] * np.float32(C_p)
    gf["v"]["p"] = gf["v"]["p"] * np.float32(C_p)
    gf["p"]["v"] = gf["p"]["v"] * np.float32(C_v)
    gf["v"]["v"] = gf["v"]["v"] * np.float32(C_v)
    for i in "pv":
        for j in "pv":
            a = gf[i][j]
            nt, n2, n3 = a.shape
            r = resample(a.reshape(nt, n2 * n3, order="F"), float(t_raw[0]), dt_in, nt_out,
                         0.0, dt_out)
            gf[i][j] = np.asfortranarray(np.asarray(r, np.float32).reshape(nt_out, n2, n3,
                                                                           order="F"))
    e = (dom.c0 ** 2 * dom_dt ** 2 * dom.dt) / (C_p * dom.dx ** 3)
    s = {"p": {"p": 1.0, "v": 1.0}, "v": {"p": 1.0, "v": 1.0}}
    z0 = dom.z0
    if extrap_type == "pv_from_pv":
        for src in "pv":
            s[src]["p"] *= z0
            s[src]["v"] /= z0
        for rec in "pv":
            s["p"][rec] /= z0
            s["v"][rec] *= z0
        for src in "pv":
            for rec in "pv":
                s[src][rec] *= -1
    elif extrap_type == "pv_from_pin":
        for rec in "pv":
            s["p"][rec] /= z0
            s["v"][rec] *= z0
    for src in "pv":
        for rec in "pv":
            s[src][rec] *= s_src * s_rec * 1.0 * e
            gf[src][rec] = (gf[src][rec].astype(np.float64) * s[src][rec]).astype(np.float32)
    if extrap_type == "pv_from_pv":
        return "PVFromPV", (gf["p"]["p"], gf["p"]["v"], gf["v"]["p"], gf["v"]["v"])
    p_pin = gf["p"]["p"].astype(np.float64) - gf["p"]["v"].astype(np.float64) / z0
    v_pin = gf["v"]["p"].astype(np.float64) - gf["v"]["v"].astype(np.float64) / z0
    if extrap_type == "pv_from_pin":
        return "PVFromPin", (p_pin.astype(np.float32, order="F"), v_pin.astype(np.float32, order="F"))
    pos = (p_pin + v_pin * z0) / 2
    neg = (p_pin - v_pin * z0) / 2
    return "PFromPin", (pos.astype(np.float32, order="F"), neg.astype(np.float32, order="F"))
