"""impulsive_gfs post-processing (src/greens.jl:174-190): denoise, cubic
B-spline resampling (src/resample.jl:32-76) with the dt-ratio amplitude
scale, and gf_to_physical (src/greens_io.jl:195-205).

The B-spline prefilter restates Interpolations.jl 0.16.2's published
Cubic(Line(OnGrid())) algorithm (natural ends), which is not in the
reference tree, so these checks are against the oracle restatement and
interpolation properties, not against the reference: parity unpinned.
"""
import numpy as np
import pytest


def traces(nt=700, ncol=37, seed=4):
    rng = np.random.default_rng(seed)
    t = np.arange(nt)
    a = np.zeros((nt, ncol))
    for c in range(ncol):
        t0 = rng.uniform(50, nt - 50)
        a[:, c] = np.exp(-0.5 * ((t - t0) / rng.uniform(4, 15)) ** 2) * rng.normal()
        a[:, c] += rng.normal(size=nt) * 1e-6  # residue below the denoise level
    return np.asfortranarray(a.astype(np.float32))


def test_oracle_resample_properties(oracle):
    a = traces()
    same = oracle.gf_postprocess(a, 0.0, 1.0, a.shape[0], 0.0, 1.0, denoise=False)
    assert np.abs(same - a).max() <= 1e-6 * np.abs(a).max()  # interpolating spline
    # a cubic polynomial on the interior is reproduced exactly by cubic B-splines
    t = np.linspace(0, 1, 200)
    poly = (0.3 + t - 2 * t ** 2 + 1.5 * t ** 3).astype(np.float32)[:, None]
    to = 0.31 + np.arange(50) * 0.0077
    r = oracle.gf_postprocess(poly, 0.0, t[1], 50, 0.31, 0.0077, denoise=False)
    ex = 0.3 + to - 2 * to ** 2 + 1.5 * to ** 3
    assert np.abs(r[:, 0] / (0.0077 / t[1]) - ex).max() < 1e-4
    # denoise zeroes |a| below 1e-4 of the column maximum before resampling
    b = np.zeros((40, 1), np.float32)
    b[10, 0] = 1.0
    b[30, 0] = 5e-5
    d = oracle.gf_postprocess(b, 0.0, 1.0, 40, 0.0, 1.0, denoise=True)
    assert abs(d[30, 0]) < 1e-12 and abs(d[10, 0] - 1.0) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("denoise,unit", [(True, 1.0), (False, -3.7e-9)])
def test_gf_postprocess_matches_oracle(adf, oracle, ctx, denoise, unit):
    a = traces()
    dt_in, dt_out = 4.2e-6, 1e-5
    nt_out = 300
    t_in0 = -156 * dt_in / 2  # pulse centre shifted to t = 0
    out = adf.gf_postprocess(a, t_in0, dt_in, nt_out, 0.0, dt_out, unit=unit, denoise=denoise)
    ref = oracle.gf_postprocess(a, t_in0, dt_in, nt_out, 0.0, dt_out, unit=unit, denoise=denoise)
    assert np.isfinite(out).all()
    err = np.linalg.norm(out.astype(np.float64) - ref) / np.linalg.norm(ref)
    assert err <= 1e-6, err


@pytest.mark.gpu
def test_impulsive_gfs_pipeline(adf, oracle, ctx):
    """impulsive_gfs (greens.jl:48-234) end to end on the GPU against the
    oracle's solve + post-processing for the same sources and receivers."""
    DX, C0, RHO = 0.005, 343.0, 1.2
    dt = 0.5 * DX / C0 / np.sqrt(3.0)
    n, steps, nt_gf = 40, 140, 60
    d = adf.Domain(tmax=(steps - 0.5) * dt, xmax=(n - 1) * DX / 2, nx=n, c0=C0, r0=RHO, cf=0.5)
    sp, sn = adf.fibonacci_sphere(2, 0.35 * d.xmax)
    rp, rn = adf.fibonacci_sphere(6, 0.2 * d.xmax)
    res = adf.impulsive_gfs(d, sp, sn, rp, rn, nt_gf, 4000.0, npml=5, pml_fc=2000.0,
                            scatterer="sphere", scatterer_kw=dict(radius=0.06 * d.xmax), batch=3)
    o = oracle.domain(tmax=d.tmax, xmax=d.xmax, nx=n, c0=C0, r0=RHO, cf=0.5)
    tf, ts = oracle.impulsive_wavelet(o, 4000.0)
    mask = oracle.build_update_mask(o, "sphere", radius=0.06 * d.xmax)
    for i in range(2):
        for typ in ("p", "v"):
            direction = [1.0, 0, 0, 0] if typ == "p" else [0.0, *sn[i]]
            pts = np.vstack([sp[i], rp])
            dirs = np.vstack([direction, np.hstack([np.zeros((6, 1)), rn])])
            tfs = np.vstack([tf, np.zeros((6, d.nt))])
            g = oracle.transceivers_to_grid(o, pts, dirs, tfs)
            cp = oracle.CpmlState(o, 5, 1e-4, 2000.0)
            f = np.zeros((n, n, n, 4), np.float32, order="F")
            oracle.run_fdtd(o, f, g, cp, mask)
            A = np.concatenate([g.rec[0][:, 1:], g.vn_rec[:, 1:]], axis=1)
            R = oracle.gf_postprocess(A, -ts, d.tmax / (d.nt - 1), nt_gf, 0.0,
                                      d.tmax / (nt_gf - 1), 1.0, True)
            for ch, cols in (("p", slice(0, 6)), ("v", slice(6, 12))):
                got = res[f"{ch}_{typ}"][:, :, i].astype(np.float64)
                want = R[:, cols].astype(np.float64)
                assert np.abs(want).max() > 0
                assert np.linalg.norm(got - want) <= 1e-5 * np.linalg.norm(want), (i, typ, ch)
