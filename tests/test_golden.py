"""Golden fixtures (tests/golden/*.npz, written by tests/golden/make_golden.py).

CPU: the oracle still reproduces every fixture bit for bit, so a change to
the oracle cannot silently move the reference the GPU is compared against.
GPU: the CUDA path, fed the fixtures' stored inputs, reproduces their
outputs: CPML profiles and masks bit-exact, fields and traces within 1e-6
(promote) / 1e-5 (fp32) relative L2, KH within 1e-5 relative L2.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
sys.path.insert(0, GOLD)


def load(name):
    with np.load(os.path.join(GOLD, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / n) if n > 0 else float(np.linalg.norm(a))


def test_oracle_reproduces_golden_fixtures(oracle):
    import make_golden

    fresh = make_golden.make_all(oracle)
    for name, arrs in fresh.items():
        gold = load(name)
        assert set(gold) == set(arrs), name
        for k, v in arrs.items():
            assert np.array_equal(np.asarray(v), gold[k]), (name, k)


def _domain(adf, v):
    tmax, xmax, ymax, zmax, nx, ny, nz, c0, r0, cf = v
    return adf.Domain(tmax=tmax, xmax=xmax, ymax=ymax, zmax=zmax, nx=int(nx), ny=int(ny),
                      nz=int(nz), c0=c0, r0=r0, cf=cf)


class _Cpml:
    def __init__(self, d, npml, coef):
        import acoustic_disguising_b200._lib as L

        self._L = L
        n = int(npml)
        dims = (d.nx, d.ny, d.nz)
        self.mv, self.mp = [], []
        for a in range(3):
            sv = list(dims) + [2]
            sv[a] = n
            sp = list(sv)
            sp[a] = n + 1
            self.mv.append(np.zeros(sv, np.float32, order="F"))
            self.mp.append(np.zeros(sp, np.float32, order="F"))
        self.n = n
        self.coef = np.ascontiguousarray(coef, np.float32)

    def _c(self):
        s = self._L.CpmlC()
        s.npml = self.n
        for a in range(3):
            s.mv[a] = self.mv[a].ctypes.data
            s.mp[a] = self.mp[a].ctypes.data
        s.coef = self.coef.ctypes.data
        return s


@pytest.mark.gpu
@pytest.mark.parametrize("mode,tol", [("promote", 1e-6), ("fp32", 1e-5)])
def test_fdtd_matches_golden(adf, ctx, mode, tol):
    g = load("fdtd_case")
    d = _domain(adf, g["domain"])
    ntx = g["dirs"].shape[1]
    F = lambda a: np.array(a, np.float32, order="F")
    txs = adf.TransceiverGrid([F(g[f"idx{c}"]) for c in range(4)], [F(g[f"w{c}"]) for c in range(4)],
                              [F(g[f"src{c}"]) for c in range(4)],
                              [np.zeros((d.nt, ntx), np.float32, order="F") for _ in range(4)],
                              F(g["dirs"]), F(g["vn_src"]),
                              np.zeros((d.nt, ntx), np.float32, order="F"))
    cp = _Cpml(d, g["npml"], g["coef"])
    field = F(g["field0"])
    adf.run_fdtd(d, field, txs, cp, g["mask"].astype(bool), arith=mode)
    assert rel(field, g[f"{mode}_field"]) <= tol
    for c in range(4):
        ref = g[f"{mode}_rec{c}"]
        if np.abs(ref).max() > 0:
            assert rel(txs.rec[c], ref) <= tol, c
    assert rel(txs.vn_rec, g[f"{mode}_vn_rec"]) <= tol
    for a in range(3):
        assert rel(cp.mv[a], g[f"{mode}_mv{a}"]) <= tol
        assert rel(cp.mp[a], g[f"{mode}_mp{a}"]) <= tol


@pytest.mark.gpu
def test_kh_matches_golden(adf, ctx):
    g = load("kh_case")
    dt, sigma, c0, rho, aq, af = g["scal"]
    out = adf.kh_pressure(g["sp"], g["sn"], g["rp"], g["q"], g["f"], dt, sigma, c0, aq, af, rho=rho)
    assert rel(out, g["out"]) <= 1e-5


@pytest.mark.gpu
def test_cpml_and_masks_match_golden_bitwise(adf, ctx):
    g = load("cpml_case")
    dt = 0.5 * 0.005 / 343.0 / np.sqrt(3.0)
    for npml, fc in ((10, 2000.0), (12, 3000.0)):
        o32, _ = adf.cpml_profiles(npml, 343.0, dt, 1e-4, 0.005 * npml, fc)
        assert np.array_equal(o32, g[f"n{npml}"])
    m = load("mask_case")
    d = _domain(adf, m["domain"])
    n = d.nx * d.ny * d.nz * 4
    sph = adf.build_update_mask(d, "sphere", radius=0.03, center=(0.004, -0.002, 0.001))
    ell = adf.build_update_mask(d, "ellipsoid", semi_axes=(0.04, 0.03, 0.02), center=(0.0, 0.005, 0.0))
    assert np.array_equal(np.unpackbits(m["sphere"])[:n].astype(bool), sph.ravel(order="F"))
    assert np.array_equal(np.unpackbits(m["ellipsoid"])[:n].astype(bool), ell.ravel(order="F"))
