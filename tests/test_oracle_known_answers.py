"""Pins the CPU oracle against the reference's own known-answer tests and
against closed forms (no GPU).

Reference tests restated here (no Julia runtime exists to run them):
  * test/test_reciprocity.jl:18-69       -> test_reciprocity_reference_setup
  * test/test_extrapolation_writecount.jl:354-393
                                          -> test_extrapolation_gather_matches_fp64
"""
from fractions import Fraction

import numpy as np
import pytest


def test_reciprocity_reference_setup(oracle):
    """test_reciprocity.jl: 51^3, xmax=0.3, cf=0.5, water, tmax=4e-4, npml=0,
    impulsive_wavelet(7 kHz), q monopoles at A and B; rms/peak < 0.01."""
    d = oracle.domain(tmax=4.0e-4, xmax=0.3, nx=51, cf=0.5)
    assert d.nt == 174
    src, _ = oracle.impulsive_wavelet(d, 7000.0)
    zero = np.zeros(d.nt)
    A = [0.10, -0.05, 0.02]
    B = [-0.04, 0.07, 0.06]

    def record_at(a, b):
        g = oracle.transceivers_to_grid(d, [a, b], [[1, 0, 0, 0], [1, 0, 0, 0]], [src, zero])
        cp = oracle.CpmlState(d, 0, 1e-4, 3e3)
        f = np.zeros((51, 51, 51, 4), np.float32, order="F")
        oracle.run_fdtd(d, f, g, cp, None)
        return g.rec[0][:, 1].copy()

    ab, ba = record_at(A, B), record_at(B, A)
    rms = np.sqrt(np.mean((ab - ba) ** 2))
    peak = np.abs(ab).max()
    assert peak > 0
    assert rms / peak < 0.01


def test_fp64_run_reciprocity_and_float32_gap(oracle):
    """The oracle's FP64 run (every array in Float64) on test_reciprocity.jl's
    set-up: reciprocity holds in FP64 too, and the Float32-storage run in
    promote mode stays within Float32 rounding of it (the error the GPU
    parity tests state against this run)."""
    d = oracle.domain(tmax=4.0e-4, xmax=0.3, nx=51, cf=0.5)
    src, _ = oracle.impulsive_wavelet(d, 7000.0)
    zero = np.zeros(d.nt)
    A = [0.10, -0.05, 0.02]
    B = [-0.04, 0.07, 0.06]

    def record_at(a, b):
        args = ([a, b], [[1, 0, 0, 0], [1, 0, 0, 0]], [src, zero])
        g64 = oracle.transceivers_to_grid64(d, *args)
        f64 = np.zeros((51, 51, 51, 4), np.float64, order="F")
        oracle.run_fdtd64(d, f64, g64, oracle.CpmlState64(d, 6, 1e-4, 3e3), None)
        g = oracle.transceivers_to_grid(d, *args)
        f = np.zeros((51, 51, 51, 4), np.float32, order="F")
        oracle.run_fdtd(d, f, g, oracle.CpmlState(d, 6, 1e-4, 3e3), None)
        r64, r32 = g64.rec[0][:, 1], g.rec[0][:, 1].astype(np.float64)
        assert np.linalg.norm(r32 - r64) / np.linalg.norm(r64) < 1e-5
        assert np.abs(f - f64).max() > 0  # the runs really differ in precision
        return r64

    ab, ba = record_at(A, B), record_at(B, A)
    assert np.sqrt(np.mean((ab - ba) ** 2)) / np.abs(ab).max() < 0.01


def _random_problem(rng, n_in, n_out, k, nt):
    pin = rng.standard_normal((nt, n_in)).astype(np.float32)
    pp = rng.standard_normal((k, n_out, n_in)).astype(np.float32)
    vp = rng.standard_normal((k, n_out, n_in)).astype(np.float32)
    return np.asfortranarray(pin), np.asfortranarray(pp), np.asfortranarray(vp)


def _gather_fp64(G, s):
    K, n_out, n_in = G.shape
    nt = s.shape[0]
    u = np.zeros((nt, n_out))
    for n in range(1, nt + 1):
        for k in range(K):
            m = n - 1 - k
            if 1 <= m <= nt:
                u[n - 1] += G[k].astype(np.float64) @ s[m - 1].astype(np.float64)
    return u


@pytest.mark.parametrize("seed", [7, 3, 0xC0FFEE])
def test_extrapolation_gather_matches_fp64(oracle, seed):
    """test_extrapolation_writecount.jl:376-393: the Float32 production gather
    (extrapolate_pv_from_pin!) agrees with an FP64 gather to < 1e-3 and
    writes each output sample exactly once (rows it+1 only)."""
    rng = np.random.default_rng(seed)
    nt, n_in, n_out, K = 28, 8, 6, 11
    pin, pp, vp = _random_problem(rng, n_in, n_out, K, nt)
    p_src = np.zeros((nt, n_out), np.float32, order="F")
    v_src = np.full((nt, n_out), np.nan, np.float32, order="F")
    v_src[0] = 0
    for it in range(1, nt):
        oracle.extrapolate_pv_from_pin(pin, p_src, v_src, pp, vp, it)
    assert not np.isnan(v_src).any()  # every row 2..nt written exactly once
    u_pp, u_vp = _gather_fp64(pp, pin), _gather_fp64(vp, pin)
    rel_v = np.abs(v_src[1:] - u_pp[1:]).max() / np.abs(u_pp[1:]).max()
    rel_p = np.abs(p_src[1:] - u_vp[1:]).max() / np.abs(u_vp[1:]).max()
    assert rel_v < 1e-3 and rel_p < 1e-3


@pytest.mark.parametrize("xmax,n", [(0.2375, 96), (0.6375, 256), (1.2775, 512), (0.3, 51),
                                    (1.1, 501), (0.85, 171)])
def test_range_matches_exact_rationals(oracle, xmax, n):
    """Julia's range(-xmax; stop=xmax, length=n) with rational endpoints is
    designed to return the correctly rounded exact values; the twice-precision
    restatement must hit them bit for bit (the cell-centre coordinates behind
    masks and transceiver indices)."""
    x = oracle.julia_range(-xmax, xmax, n)
    a = Fraction(-xmax).limit_denominator(1 << 24)
    b = Fraction(xmax).limit_denominator(1 << 24)
    assert float(a) == -xmax and float(b) == xmax
    exact = [a + (b - a) * i / (n - 1) for i in range(n)]
    ref = np.array([float(v) for v in exact])
    assert np.array_equal(x, ref)
    # staggered grid x .- dx/2
    dx = 2 * xmax / (n - 1)
    xv = oracle.julia_range(-xmax, xmax, n, dx / 2)
    exact_v = np.array([float(v - Fraction(dx) / 2) for v in exact])
    # dx/2 is itself a rounded Float64, so only closeness is defined here
    assert np.max(np.abs(xv - exact_v)) <= 2.3e-16 * xmax


def test_cpml_profiles_closed_form(oracle):
    """calc_Kab_CPML (cpmlcoeffs.jl:65-126) evaluated independently in numpy."""
    npml, c0, dt, rcoef, fc, dx = 10, 343.0, 4.2081e-6, 1e-4, 2000.0, 0.005
    prof = oracle.cpml_coefficients(npml, c0, dt, rcoef, dx * npml, fc)
    d0 = -(2.0 + 1) * c0 * np.log(rcoef) / (2.0 * dx * npml)
    for half in (False, True):
        m = npml + (1 if half else 0)
        sh = 0.5 if half else 0.0
        t = np.arange(m) / max(1, m - 1)
        dist = (1 - t) * (0 - sh) + t * (m - sh - 1)
        if half:
            dist[0] = 0
        for right in (False, True):
            nd = (dist if right else dist[::-1]) / npml
            dd = d0 * nd * nd
            al = np.pi * fc * (1.0 - nd)
            b = np.exp(-(dd + al) * dt)
            a = dd * (b - 1.0) / (dd + al)
            k = (2 if half else 0) + (1 if right else 0)
            assert np.allclose(prof[k], a, rtol=1e-14, atol=0)
            assert np.allclose(prof[4 + k], b, rtol=1e-14, atol=0)


def test_update_mask_rules(oracle):
    """build_update_mask (geometry.jl:250-280): faces open iff both neighbours
    are fluid, first strip closed; `nothing` for :none."""
    d = oracle.domain(tmax=1e-4, xmax=0.1, nx=21, ny=23, nz=25, c0=343.0, r0=1.2, cf=0.5)
    assert oracle.build_update_mask(d, "none") is None
    m = oracle.build_update_mask(d, "sphere", radius=0.05)
    x = oracle.coords(d, 0, 0)
    y = oracle.coords(d, 1, 0)
    z = oracle.coords(d, 2, 0)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    s = ~(X * X + Y * Y + Z * Z > 0.05 * 0.05)
    assert np.array_equal(m[..., 0].astype(bool), ~s)
    assert not m[0, :, :, 1].any() and not m[:, 0, :, 2].any() and not m[:, :, 0, 3].any()
    assert np.array_equal(m[1:, :, :, 1].astype(bool), ~s[1:] & ~s[:-1])
    assert np.array_equal(m[:, 1:, :, 2].astype(bool), ~s[:, 1:] & ~s[:, :-1])
    assert np.array_equal(m[:, :, 1:, 3].astype(bool), ~s[:, :, 1:] & ~s[:, :, :-1])


def test_fibonacci_and_wavelets(oracle):
    pts, nrm = oracle.fibonacci_sphere(64, 0.15)
    assert np.allclose(np.linalg.norm(nrm, axis=1), 1.0, atol=1e-15)
    assert np.allclose(pts, 0.15 * nrm, rtol=0, atol=0)
    d = oracle.domain(tmax=800 * 4.208e-6, xmax=0.2375, nx=96, c0=343.0, r0=1.2, cf=0.5)
    tf, ts = oracle.impulsive_wavelet(d, 2000.0)
    assert abs(tf.sum() * d.dt - 1.0) < 1e-12
    r = oracle.ricker_wavelet(d, 2000.0, injection=False)
    tt = oracle.time_axis(d)
    i = np.argmax(r)
    assert abs(tt[i] - 1 / 2000.0) <= tt[1]


def _ref_erf(x):
    """_erf of src/kh_kernels.jl:19-25 (Abramowitz-Stegun 7.1.26), vectorised."""
    s, ax = np.sign(x), np.abs(x)
    t = 1.0 / (1.0 + 0.3275911 * ax)
    y = 1.0 - (((((1.061405429 * t - 1.453152027) * t) + 1.421413741) * t - 0.284496736) * t +
               0.254829592) * t * np.exp(-ax * ax)
    return s * y


def test_kh_velocity_pedestal_equals_full_kernel(oracle):
    """The v_v kernel does not decay (its F term tends to a constant); the
    oracle sums taps within +-12 sigma plus that constant times the running
    input sum.  Brute force: the full kernel of eval_one_kernel
    (kh_kernels.jl:106-157) at every lag, convolved directly."""
    rng = np.random.default_rng(3)
    ns, nr, nt, dt, c0, rho = 3, 2, 400, 5e-6, 343.0, 1.2
    sg = np.sqrt(np.log(2.0)) / (2 * np.pi * 20e3)
    sp = rng.standard_normal((ns, 3)) * 0.02
    sn = rng.standard_normal((ns, 3))
    sn /= np.linalg.norm(sn, axis=1, keepdims=True)
    rp = rng.standard_normal((nr, 3)) * 0.02 + np.array([0.1, 0.0, 0.0])
    rn = rng.standard_normal((nr, 3))
    rn /= np.linalg.norm(rn, axis=1, keepdims=True)
    q = rng.standard_normal((nt, ns)).astype(np.float32)
    f = rng.standard_normal((nt, ns)).astype(np.float32)
    aq, af = -0.7, 1.3
    got = oracle.kh_velocity(sp, sn, rp, rn, q, f, dt, sg, c0, rho, aq, af)
    want = np.zeros((nt, nr))
    tg = np.arange(nt) * dt
    for r in range(nr):
        for s in range(ns):
            d = rp[r] - sp[s]
            dist = np.linalg.norm(d)
            ih = d / dist
            cr, cs = rn[r] @ ih, sn[s] @ ih
            tau = tg - dist / c0
            fg = np.exp(-tau ** 2 / (2 * sg ** 2)) / (np.sqrt(2 * np.pi) * sg)
            dfg = -(tau / sg ** 2) * fg
            Fg = 0.5 * (1 + _ref_erf(tau / (sg * np.sqrt(2))))
            i1, i2, i3 = (1 / (4 * np.pi * dist ** k) for k in (1, 2, 3))
            kq = (cr / rho) * (fg * i2 + dfg * i1 / c0)
            kf = (cr * cs / rho) * (2 * Fg * i3 + 2 * fg * i2 / c0 + dfg * i1 / c0 ** 2)
            want[:, r] += aq * np.convolve(kq, q[:, s].astype(np.float64))[:nt]
            want[:, r] += af * np.convolve(kf, f[:, s].astype(np.float64))[:nt]
    assert np.abs(got).max() > 0
    assert np.linalg.norm(got - want) <= 1e-9 * np.linalg.norm(want)
