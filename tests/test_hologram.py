"""Hologram synthesis with distributed C_f / C_q injection, shell recording
and the KH extrapolation of the recorded shell in one call
(adf_run_fdtd_kh), against the oracle.

The reference flow: build_txs + inject_inner_sources! (diagnostics/
_check_inject_kh/fdtd_runners.jl:1-45: outer recording shell first, inner
injection surface after it, both with direction [0, n]; p_src = C_q vn,
vn_src = C_f p of the inner columns), C_for_N (injection_coefficients.jl:
467-472), run_fdtd!, then the two-way KH pressure of
part3_kh_extrapolation.jl:168-185 (in_q = v_n, in_f = p of the shell,
aq = -rho dS dt, af = -dS dt).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DX = 0.005
C0, RHO = 343.0, 1.2
DT = 0.5 * DX / C0 / np.sqrt(3.0)
TOL = 1e-5


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def band_noise(nt, n, seed, half=12):
    """Seeded Gaussian noise, low-passed by a Hann window of 2*half+1 samples
    (zero-padded at the ends, so the trace keeps its nt samples)."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((nt + 2 * half, n))
    w = np.hanning(2 * half + 1)
    w /= w.sum()
    y = sum(w[k] * x[k:k + nt] for k in range(2 * half + 1))
    return np.asfortranarray(y.astype(np.float32))


def hologram_case(adf, oracle, n, steps, npml, semi, r_in, r_out, n_in, n_out, seed=3):
    kw = dict(tmax=(steps - 0.5) * DT, xmax=(n - 1) * DX / 2, nx=n, c0=C0, r0=RHO, cf=0.5)
    d, o = adf.Domain(**kw), oracle.domain(**kw)
    op, on = adf.fibonacci_sphere(n_out, r_out * DX)
    ip, inn = adf.fibonacci_sphere(n_in, r_in * DX)
    pts = np.vstack([op, ip])
    dirs = np.hstack([np.zeros((n_out + n_in, 1)), np.vstack([on, inn])])
    zero = np.zeros((n_out + n_in, steps))
    g = adf.transceivers_to_grid(d, [adf.Transceiver(p, q, t) for p, q, t in zip(pts, dirs, zero)])
    go = oracle.transceivers_to_grid(o, pts, dirs, zero)
    cf_, cq_, _ = adf.injection_coefficients(d, r_in * DX, n_in)
    p_tr = band_noise(steps, n_in, seed)
    vn_tr = band_noise(steps, n_in, seed + 1)
    inner = slice(n_out, n_out + n_in)
    for grid in (g, go):  # inject_inner_sources!: vn_src = C_f p, p_src = C_q vn
        grid.vn_src[:, inner] = (cf_ * p_tr.astype(np.float64)).astype(np.float32)
        grid.src[0][:, inner] = (cq_ * vn_tr.astype(np.float64)).astype(np.float32)
    cp = adf.Cpml(d, npml, 1e-4, 2000.0)
    co = oracle.CpmlState(o, npml, 1e-4, 2000.0)
    assert np.array_equal(cp.coef, co.coef)
    sax = dict(semi_axes=tuple(a * DX for a in semi))
    m = adf.build_update_mask(d, "ellipsoid", **sax)
    mo = oracle.build_update_mask(o, "ellipsoid", **sax)
    assert np.array_equal(m, mo.astype(bool))
    return dict(d=d, o=o, g=g, go=go, cp=cp, co=co, m=m, mo=mo, pts=pts, dirs=dirs)


def run_pair(adf, oracle, c, cols, r_pts, sigma, aq, af):
    n = c["d"].nx
    f = np.zeros((n, n, n, 4), np.float32, order="F")
    fo = f.copy(order="F")
    ns = len(cols)
    sp = c["pts"][cols - 1]
    sn = c["dirs"][cols - 1, 1:]
    out = adf.run_fdtd_kh(c["d"], f, c["g"], c["cp"], c["m"], cols, sp, sn, r_pts, sigma, aq, af)
    oracle.run_fdtd(c["o"], fo, c["go"], c["co"], c["mo"])
    return f, fo, out, sp, sn


def test_hologram_128cube_injection_shell_kh(adf, oracle, ctx):
    """A reduced configuration with the full structure: 128^3, 8-cell CPML,
    rigid ellipsoid 20/15/10 cells, 512 injection points at 25 cells, a
    512-point shell at 32 cells, 260 steps, KH to 64 targets at 0.4 m (their
    delays from the shell, 165-390 samples, overlap the record)."""
    n_in = n_out = 512
    c = hologram_case(adf, oracle, 128, 260, 8, (20, 15, 10), 25, 32, n_in, n_out)
    cols = np.arange(1, n_out + 1, dtype=np.int64)
    rp, _ = adf.fibonacci_sphere(64, 0.4)
    sigma = np.sqrt(np.log(2.0)) / (2 * np.pi * 20e3)
    dS = 4 * np.pi * (32 * DX) ** 2 / n_out
    aq, af = -RHO * dS * DT, -dS * DT
    f, fo, out, sp, sn = run_pair(adf, oracle, c, cols, rp, sigma, aq, af)
    g, go = c["g"], c["go"]
    shell = slice(0, n_out)
    assert np.abs(go.rec[0][:, shell]).max() > 0
    assert rel_l2(g.rec[0][:, shell], go.rec[0][:, shell]) <= TOL
    assert rel_l2(g.vn_rec[:, shell], go.vn_rec[:, shell]) <= TOL
    assert rel_l2(f, fo) <= TOL
    # the device hand-off equals the host path on the downloaded traces, bit for bit
    host = adf.kh_pressure(sp, sn, rp, g.vn_rec[:, shell], g.rec[0][:, shell], DT, sigma, C0,
                           aq, af, rho=RHO)
    assert np.abs(host).max() > 0 and np.array_equal(out, host)
    # and the KH sum against the FP64 oracle on the oracle's own recorded traces
    ref = oracle.kh_pressure(sp, sn, rp, go.vn_rec[:, shell], go.rec[0][:, shell], DT, sigma,
                             C0, aq, af, mode=1)
    assert np.abs(ref).max() > 0
    assert rel_l2(out, ref) <= TOL


def test_hologram_512cube_16384_transceivers(adf, oracle, ctx):
    """The full hologram grid and transceiver counts: 512^3, 12-cell CPML,
    ellipsoid 80/60/40 cells, 8192 injection points at 100 cells and an
    8192-point shell at 130 cells, 24 steps (the entry lists of all 16384
    transceivers at full size), KH of the injection surface's own records to
    targets 4 cells outside it (delays from 14 samples, inside the record)."""
    n_in = n_out = 8192
    c = hologram_case(adf, oracle, 512, 24, 12, (80, 60, 40), 100, 130, n_in, n_out)
    cols = np.arange(n_out + 1, n_out + n_in + 1, dtype=np.int64)
    rp, _ = adf.fibonacci_sphere(128, 104 * DX)
    sigma = np.sqrt(np.log(2.0)) / (2 * np.pi * 20e3)
    dS = 4 * np.pi * (100 * DX) ** 2 / n_in
    f, fo, out, sp, sn = run_pair(adf, oracle, c, cols, rp, sigma, -RHO * dS * DT, -dS * DT)
    g, go = c["g"], c["go"]
    inner = slice(n_out, n_out + n_in)
    for c_ in range(4):
        assert rel_l2(g.rec[c_][:, inner], go.rec[c_][:, inner]) <= TOL
        assert rel_l2(f[..., c_], fo[..., c_]) <= TOL
    assert rel_l2(g.vn_rec[:, inner], go.vn_rec[:, inner]) <= TOL
    host = adf.kh_pressure(sp, sn, rp, g.vn_rec[:, inner], g.rec[0][:, inner], DT, sigma, C0,
                           -RHO * dS * DT, -dS * DT, rho=RHO)
    assert np.abs(host).max() > 0 and np.array_equal(out, host)
