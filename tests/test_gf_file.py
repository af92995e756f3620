"""GF files (the schema of scripts/greens/impulsive.jl:111-124 and
src/greens_io.jl:484-510) and the load_gf_ref scaling chain
(src/greens_io.jl:224-477)."""
import numpy as np
import pytest

from acoustic_disguising_b200 import gf_file as G

C0, RHO, DX = 343.0, 1.2, 0.005


class Dom:  # the Domain fields load_gf_ref reads
    def __init__(self, dt, dx=DX, c0=C0, r0=RHO, tmax=1e-3):
        self.dt, self.dx, self.c0, self.r0, self.tmax = dt, dx, c0, r0, tmax
        self.z0 = r0 * c0


def raw_tensors(nt=120, n_rec=5, n_src=4, seed=3):
    rng = np.random.default_rng(seed)
    return [np.asfortranarray(rng.standard_normal((nt, n_rec, n_src)).astype(np.float32))
            for _ in range(4)]


def test_container_roundtrip(tmp_path):
    a = np.asfortranarray(np.arange(24, dtype=np.float32).reshape(2, 3, 4, order="F"))
    t = np.linspace(0, 1, 5)
    p = G.write_gf_file(str(tmp_path / "x.adfgf"), {"a": a, "t": t}, {"units_convention": "physical",
                                                                        "n": 7})
    ds, at = G.read_gf_file(p)
    assert np.array_equal(ds["a"], a) and ds["a"].shape == (2, 3, 4)
    assert np.array_equal(ds["t"], t)
    assert at == {"units_convention": "physical", "n": 7}


def test_save_is_physical_units(tmp_path):
    dom = Dom(dt=4.2e-6)
    pp, pv, vp, vv = raw_tensors()
    t = np.arange(pp.shape[0]) * 1e-5
    p = G.save_impulsive_gfs(str(tmp_path / "g.adfgf"), pp, pv, vp, vv, t,
                             np.zeros((4, 3)), np.zeros((5, 3)), dom)
    ds, at = G.read_gf_file(p)
    C_p, C_v = G.gf_unit_factors(DX, dom.dt, C0, RHO, 1e-5)
    assert at["units_convention"] == "physical" and at["n_done"] == 4
    assert np.array_equal(ds["p_p"], pp / np.float32(C_p))
    assert np.array_equal(ds["v_v"], vv / np.float32(C_v))


@pytest.mark.parametrize("kind", ["pv_from_pin", "pv_from_pv", "p_from_pin"])
def test_load_gf_ref_chain(tmp_path, oracle, kind):
    """Same-grid file (dt_save = dom.dt): resampling is the identity, so the
    loaded tensors are the raw ones times the chain's closed-form factors."""
    dt = 4.2e-6
    dom = Dom(dt=dt)
    pp, pv, vp, vv = raw_tensors()
    nt = pp.shape[0]
    t = np.arange(nt) * dt
    path = G.save_impulsive_gfs(str(tmp_path / "g.adfgf"), pp, pv, vp, vv, t,
                                np.zeros((4, 3)), np.zeros((5, 3)), dom)
    rs = lambda a, t0, d0, n, t1, d1: oracle.gf_postprocess(a, t0, d0, n, t1, d1, 1.0, False)
    got_kind, ts = G.load_gf_ref(path, dom, 0.1, 5, 0.2, 4, tmax=t[-1], extrap_type=kind,
                                 resample=rs)
    # expected: physical * C = raw (to Float32 rounding), then e, impedance, weights
    C_p = DX ** 3 * dt / (dt ** 2 * C0 ** 2)
    e = (C0 ** 2 * dt ** 2 * dt) / (C_p * DX ** 3)
    w = G.fib_sphere_area(0.1, 5) * G.fib_sphere_area(0.2, 4) * e
    z0 = RHO * C0
    if kind == "pv_from_pv":  # receiver- and source-side impedance, times -1
        s = {"pp": -w * z0 / z0, "pv": -w / z0 / z0, "vp": -w * z0 * z0, "vv": -w / z0 * z0}
    elif kind == "pv_from_pin":  # source-side impedance only
        s = {"pp": w / z0, "pv": w / z0, "vp": w * z0, "vv": w * z0}
    else:  # p_from_pin: no impedance conversion in the reference
        s = {"pp": w, "pv": w, "vp": w, "vv": w}
    raw = {"pp": pp, "pv": pv, "vp": vp, "vv": vv}
    sc = {k: raw[k].astype(np.float64) * s[k] for k in raw}
    if kind == "pv_from_pv":
        want = (sc["pp"], sc["pv"], sc["vp"], sc["vv"])
        assert got_kind == "PVFromPV"
    else:
        p_pin = sc["pp"] - sc["pv"] / z0
        v_pin = sc["vp"] - sc["vv"] / z0
        if kind == "pv_from_pin":
            want = (p_pin, v_pin)
            assert got_kind == "PVFromPin"
        else:
            want = ((p_pin + v_pin * z0) / 2, (p_pin - v_pin * z0) / 2)
            assert got_kind == "PFromPin"
    for g, w_ in zip(ts, want):
        assert g.shape == w_.shape
        assert np.linalg.norm(g - w_) <= 1e-6 * np.linalg.norm(w_)


def test_load_gf_ref_rejects_raw_units(tmp_path):
    p = G.write_gf_file(str(tmp_path / "r.adfgf"),
                        {"p_p": np.zeros((3, 1, 1), np.float32), "p_v": np.zeros((3, 1, 1), np.float32),
                         "v_p": np.zeros((3, 1, 1), np.float32), "v_v": np.zeros((3, 1, 1), np.float32),
                         "t": np.arange(3.0)}, {"units_convention": "raw", "dom_dx": DX})
    with pytest.raises(ValueError, match="physical"):
        G.load_gf_ref(p, Dom(dt=1.0), 0.1, 1, 0.2, 1, resample=lambda *a: None)


@pytest.mark.gpu
def test_load_gf_ref_device_resampling(tmp_path, oracle, adf, ctx):
    """Resampling a 1e-5 s file onto a 4.2e-6 s FDTD axis on the GPU agrees
    with the oracle's restatement."""
    dom = Dom(dt=4.2e-6)
    pp, pv, vp, vv = raw_tensors(nt=200)
    t = np.arange(200) * 1e-5
    path = G.save_impulsive_gfs(str(tmp_path / "g.adfgf"), pp, pv, vp, vv, t,
                                np.zeros((4, 3)), np.zeros((5, 3)), dom)
    rs = lambda a, t0, d0, n, t1, d1: oracle.gf_postprocess(a, t0, d0, n, t1, d1, 1.0, False)
    k1, a = G.load_gf_ref(path, dom, 0.1, 5, 0.2, 4, extrap_type="pv_from_pin")
    k2, b = G.load_gf_ref(path, dom, 0.1, 5, 0.2, 4, extrap_type="pv_from_pin", resample=rs)
    assert k1 == k2 == "PVFromPin"
    for x, y in zip(a, b):
        assert np.linalg.norm(x.astype(np.float64) - y) <= 1e-6 * np.linalg.norm(y)
