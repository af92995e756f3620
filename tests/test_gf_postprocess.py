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
