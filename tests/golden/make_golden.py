"""Writes the golden fixtures of tests/test_golden.py.

The fixtures are small seeded cases computed by the CPU oracle (oracle/),
stored with their inputs so that a test can replay them without this script:

  fdtd_case.npz  20x18x16 grid, 4-cell CPML, off-centre sphere mask, one q
                 source, one f source, 8 receivers with v_n, a non-zero
                 initial pressure; 30 steps of run_fdtd! in promote and fp32
                 arithmetic (final field, all traces, CPML memory)
  kh_case.npz    24 surface points -> 6 targets, 300 samples: the two-way KH
                 pressure in FP64
  cpml_case.npz  CPML profiles (npml 10 and 12, fc 2 and 3 kHz) in Float32
  mask_case.npz  update masks of a sphere and an ellipsoid on a 21x19x17 grid

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

C0, RHO, DX = 343.0, 1.2, 0.005
DT = 0.5 * DX / C0 / np.sqrt(3.0)


def fdtd_inputs(O):
    nx, ny, nz, steps, npml = 20, 18, 16, 30, 4
    kw = dict(tmax=(steps - 0.5) * DT, xmax=(nx - 1) * DX / 2, ymax=(ny - 1) * DX / 2,
              zmax=(nz - 1) * DX / 2, nx=nx, ny=ny, nz=nz, c0=C0, r0=RHO, cf=0.5)
    d = O.domain(**kw)
    assert d.nt == steps
    rng = np.random.default_rng(20261203)
    tq = O.ricker_wavelet(d, 6000.0, injection=False)
    pts = [[0.3 * d.xmax, -0.2 * d.ymax, 0.1 * d.zmax], [-0.25 * d.xmax, 0.2 * d.ymax, -0.3 * d.zmax]]
    nv = rng.standard_normal(3)
    nv /= np.linalg.norm(nv)
    dirs = [[1.0, 0, 0, 0], [0.0, *nv]]
    tfs = [tq * 1e3, np.roll(tq, 7) * 2.0]
    rp, rn = O.fibonacci_sphere(8, 0.35 * min(d.xmax, d.ymax, d.zmax))
    for i in range(8):
        pts.append(rp[i])
        dirs.append([0.0, *rn[i]])
        tfs.append(np.zeros(steps))
    g = O.transceivers_to_grid(d, np.array(pts), np.array(dirs), np.array(tfs))
    g.vn_src[:, 1] = (np.roll(tq, 11) * 0.05).astype(np.float32)
    cp = O.CpmlState(d, npml, 1e-4, 2000.0)
    mask = O.build_update_mask(d, "sphere", radius=0.25 * d.xmax, center=(0.02 * d.xmax, 0, 0))
    field = np.zeros((nx, ny, nz, 4), np.float32, order="F")
    field[..., 0] = rng.standard_normal((nx, ny, nz)).astype(np.float32) * 1e-3
    return kw, d, g, cp, mask, field


def fdtd_case(O):
    kw, d, g, cp, mask, field = fdtd_inputs(O)
    out = dict(domain=np.array([kw[k] for k in ("tmax", "xmax", "ymax", "zmax", "nx", "ny", "nz",
                                                "c0", "r0", "cf")], np.float64),
               npml=np.int64(cp.npml), field0=field, mask=mask.astype(np.uint8),
               coef=cp.coef, dirs=g.dir, vn_src=g.vn_src)
    for c in range(4):
        out[f"idx{c}"] = g.idx[c]
        out[f"w{c}"] = g.w[c]
        out[f"src{c}"] = g.src[c]
    for mode in ("promote", "fp32"):
        f = field.copy(order="F")
        gg = g.copy()
        cc = cp.copy()
        O.run_fdtd(d, f, gg, cc, mask, start_step=1, stop_step=None, mode=mode)
        out[f"{mode}_field"] = f
        for c in range(4):
            out[f"{mode}_rec{c}"] = gg.rec[c]
        out[f"{mode}_vn_rec"] = gg.vn_rec
        for a in range(3):
            out[f"{mode}_mv{a}"] = cc.mv[a]
            out[f"{mode}_mp{a}"] = cc.mp[a]
    return out


def kh_case(O):
    rng = np.random.default_rng(7)
    ns, nr, nt, dt = 24, 6, 300, 5e-6
    i = np.arange(ns, dtype=np.float64)
    z = 1.0 - (2.0 * i + 1.0) / ns
    rxy = np.sqrt(1.0 - z * z)
    th = np.pi * (3.0 - np.sqrt(5.0)) * i
    sn = np.stack([np.cos(th) * rxy, np.sin(th) * rxy, z], axis=1)
    sp = 0.25 * sn
    u = rng.standard_normal((nr, 3))
    rp = 0.6 * u / np.linalg.norm(u, axis=1, keepdims=True)
    q = rng.standard_normal((nt, ns)).astype(np.float32)
    f = rng.standard_normal((nt, ns)).astype(np.float32)
    sigma = np.sqrt(np.log(2.0)) / (2 * np.pi * 20e3)
    dS = 4 * np.pi * 0.25 ** 2 / ns
    aq, af = -RHO * dS * dt, -dS * dt
    out = O.kh_pressure(sp, sn, rp, q, f, dt, sigma, C0, aq, af, mode=1)
    return dict(sp=sp, sn=sn, rp=rp, q=q, f=f, scal=np.array([dt, sigma, C0, RHO, aq, af]), out=out)


def cpml_case(O):
    out = {}
    for npml, fc in ((10, 2000.0), (12, 3000.0)):
        ref = O.cpml_coefficients(npml, C0, DT, 1e-4, DX * npml, fc)
        out[f"n{npml}"] = np.concatenate([r.astype(np.float32) for r in ref])
    return out


def mask_case(O):
    nx, ny, nz = 21, 19, 17
    kw = dict(tmax=1e-4, xmax=(nx - 1) * DX / 2, ymax=(ny - 1) * DX / 2, zmax=(nz - 1) * DX / 2,
              nx=nx, ny=ny, nz=nz, c0=C0, r0=RHO, cf=0.5)
    d = O.domain(**kw)
    sph = O.build_update_mask(d, "sphere", radius=0.03, center=(0.004, -0.002, 0.001))
    ell = O.build_update_mask(d, "ellipsoid", semi_axes=(0.04, 0.03, 0.02), center=(0.0, 0.005, 0.0))
    return dict(domain=np.array([kw[k] for k in ("tmax", "xmax", "ymax", "zmax", "nx", "ny", "nz",
                                                 "c0", "r0", "cf")], np.float64),
                sphere=np.packbits(sph.astype(np.uint8).ravel(order="F")),
                ellipsoid=np.packbits(ell.astype(np.uint8).ravel(order="F")))


def make_all(O):
    return {"fdtd_case": fdtd_case(O), "kh_case": kh_case(O), "cpml_case": cpml_case(O),
            "mask_case": mask_case(O)}


if __name__ == "__main__":
    import pyoracle as O

    O.build()
    for name, arrs in make_all(O).items():
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrs)
        print("wrote", name, sum(a.nbytes for a in arrs.values()), "bytes")
