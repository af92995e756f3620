"""KH extrapolation on the GPU against the FP64 oracle.

The oracle (or_kh_pressure) evaluates eval_one_kernel's monopole and dipole
kernels (src/kh_kernels.jl:106-157) in FP64 with a +-12 sigma window and
accumulates as direct_kh_accumulate! (src/kh_kernels.jl:256-296) does, in
FP64.  The GPU evaluates FP32 taps within +-6 sigma and accumulates in FP32
with compensation; the bar is 1e-5 relative L2 over all targets and samples.
"""
import numpy as np
import pytest

RTOL_L2 = 1e-5
C0, RHO = 343.0, 1.2


def fib(n, radius):
    i = np.arange(n, dtype=np.float64)
    z = 1.0 - (2.0 * i + 1.0) / n
    rxy = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    th = np.pi * (3.0 - np.sqrt(5.0)) * i
    nrm = np.stack([np.cos(th) * rxy, np.sin(th) * rxy, z], axis=1)
    return radius * nrm, nrm


def ricker_noise(nt, ns, dt, fc, seed):
    """Ricker-filtered Gaussian noise, unit RMS per column (float32)."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((nt, ns))
    tw = (np.arange(-int(2.0 / fc / dt), int(2.0 / fc / dt) + 1)) * dt
    w = np.pi * fc * tw
    r = (1 - 2 * w * w) * np.exp(-w * w)
    y = np.stack([np.convolve(x[:, s], r, mode="same") for s in range(ns)], axis=1)
    y /= np.sqrt((y * y).mean(axis=0, keepdims=True))
    return np.asfortranarray(y.astype(np.float32))


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def case(ns, nr, nt, dt, r_surf, r_tgt, f3db=20e3, seed=7):
    sp, sn = fib(ns, r_surf)
    rp, _ = fib(nr, r_tgt)
    sigma = np.sqrt(np.log(2.0)) / (2 * np.pi * f3db)
    q = ricker_noise(nt, ns, dt, 8e3, seed)
    f = ricker_noise(nt, ns, dt, 8e3, seed + 1)
    dS = 4 * np.pi * r_surf ** 2 / ns
    return dict(sp=sp, sn=sn, rp=rp, q=q, f=f, dt=dt, sigma=sigma, aq=-RHO * dS * dt,
                af=-dS * dt)


def run_pair(adf, oracle, c, window_sigmas=6.0):
    out = adf.kh_pressure(c["sp"], c["sn"], c["rp"], c["q"], c["f"], c["dt"], c["sigma"], C0,
                          c["aq"], c["af"], rho=RHO, window_sigmas=window_sigmas)
    ref = oracle.kh_pressure(c["sp"], c["sn"], c["rp"], c["q"], c["f"], c["dt"], c["sigma"], C0,
                             c["aq"], c["af"], mode=1)
    return out, ref


@pytest.mark.gpu
@pytest.mark.parametrize("ns,nr,nt,dt,r_surf,r_tgt", [
    (256, 96, 1024, 5e-6, 0.25, 1.0),     # far field, 16-tap window
    (45, 50, 1001, 5e-6, 0.25, 0.8),      # ragged: ns, nr, nt off every block size
    (128, 64, 900, 5e-6, 0.25, 0.30),     # targets just outside the surface (wide delay spread)
    (80, 48, 1200, 3.5e-6, 0.25, 0.7),    # 23-tap window (the 24-tap instantiation)
    (64, 40, 1500, 2.5e-6, 0.25, 0.6),    # 32-tap window
])
def test_kh_matches_fp64_oracle(adf, oracle, ctx, ns, nr, nt, dt, r_surf, r_tgt):
    c = case(ns, nr, nt, dt, r_surf, r_tgt)
    out, ref = run_pair(adf, oracle, c)
    assert np.isfinite(out).all()
    assert np.abs(ref).max() > 0
    assert rel_l2(out, ref) <= RTOL_L2


@pytest.mark.gpu
def test_kh_monopole_dipole_split(adf, oracle, ctx):
    """aq and af parts computed alone add up to the combined sum."""
    c = case(96, 40, 800, 5e-6, 0.25, 0.9)
    both, _ = run_pair(adf, oracle, c)
    cq = dict(c, af=0.0)
    cf = dict(c, aq=0.0)
    oq, rq = run_pair(adf, oracle, cq)
    of, rf = run_pair(adf, oracle, cf)
    assert rel_l2(oq, rq) <= RTOL_L2
    assert rel_l2(of, rf) <= RTOL_L2
    assert rel_l2(oq.astype(np.float64) + of, both.astype(np.float64)) <= 1e-6


@pytest.mark.gpu
def test_kh_into_caller_buffers(adf, oracle, ctx):
    """kh_pressure / kh_velocity write into a caller's page-locked output
    (reused twice, from pinned inputs) exactly what they return otherwise."""
    c = case(64, 40, 700, 5e-6, 0.25, 0.9)
    q, f = adf.pinned_zeros(c["q"].shape), adf.pinned_zeros(c["f"].shape)
    q[:], f[:] = c["q"], c["f"]
    rn = c["rp"] / np.linalg.norm(c["rp"], axis=1, keepdims=True)
    for fn, extra in ((adf.kh_pressure, ()), (adf.kh_velocity, (rn,))):
        args = (c["sp"], c["sn"], c["rp"], *extra)
        fresh = fn(*args, c["q"], c["f"], c["dt"], c["sigma"], C0, c["aq"], c["af"], rho=RHO)
        out = adf.pinned_zeros(fresh.shape)
        for _ in range(2):
            out.fill(np.nan)
            got = fn(*args, q, f, c["dt"], c["sigma"], C0, c["aq"], c["af"], rho=RHO, out=out)
            assert got is out and np.array_equal(out, fresh)
    with pytest.raises(ValueError, match="out must be"):
        adf.kh_pressure(c["sp"], c["sn"], c["rp"], q, f, c["dt"], c["sigma"], C0, c["aq"],
                        c["af"], out=np.zeros((3, 3), np.float32))


@pytest.mark.gpu
def test_kh_rejects_bad_arguments(adf, ctx):
    c = case(16, 8, 64, 5e-6, 0.25, 1.0)
    with pytest.raises(adf.AdfError, match="at most 32"):
        adf.kh_pressure(c["sp"], c["sn"], c["rp"], c["q"], c["f"], 1e-7, c["sigma"], C0,
                        c["aq"], c["af"])
    with pytest.raises(adf.AdfError, match="positive"):
        adf.kh_pressure(c["sp"], c["sn"], c["rp"], c["q"], c["f"], c["dt"], -1.0, C0,
                        c["aq"], c["af"])


@pytest.mark.gpu
def test_fp32_fma_peak_is_plausible(adf, ctx):
    tf, ms = adf.fp32_fma_peak()
    # 148 SMs x 128 FP32 lanes x 2 FLOP at 1-2 GHz
    assert 20.0 < tf < 90.0, tf
    assert ms > 0


def run_velocity(adf, oracle, c, seed=9):
    rng = np.random.default_rng(seed)
    rn = rng.standard_normal(c["rp"].shape)
    rn /= np.linalg.norm(rn, axis=1, keepdims=True)
    aq, af = -RHO * 1e-9, -1e-9  # the two-way vn form's scales, up to dS dt
    out = adf.kh_velocity(c["sp"], c["sn"], c["rp"], rn, c["q"], c["f"], c["dt"], c["sigma"], C0,
                          aq, af, rho=RHO)
    ref = oracle.kh_velocity(c["sp"], c["sn"], c["rp"], rn, c["q"], c["f"], c["dt"], c["sigma"],
                             C0, RHO, aq, af)
    return out, ref


@pytest.mark.gpu
@pytest.mark.parametrize("ns,nr,nt,dt,r_surf,r_tgt", [
    (256, 96, 1024, 5e-6, 0.25, 1.0),     # far field
    (128, 64, 900, 5e-6, 0.25, 0.30),     # near field: the 1/r^3 pedestal of v_v is large
    (45, 50, 1001, 5e-6, 0.25, 0.8),      # ragged sizes
    (80, 48, 1200, 3.5e-6, 0.25, 0.7),    # 23-tap window
    (64, 40, 1500, 2.5e-6, 0.25, 0.6),    # 32-tap window
])
def test_kh_velocity_matches_fp64_oracle(adf, oracle, ctx, ns, nr, nt, dt, r_surf, r_tgt):
    c = case(ns, nr, nt, dt, r_surf, r_tgt)
    out, ref = run_velocity(adf, oracle, c)
    assert np.isfinite(out).all()
    assert np.abs(ref).max() > 0
    assert rel_l2(out, ref) <= RTOL_L2


@pytest.mark.gpu
@pytest.mark.parametrize("skip", [0, 1])
def test_kh_bounded_wait_ends_in_an_error_code(adf, oracle, ctx, skip):
    """A staged chunk whose bytes never arrive (its copies are not issued, so
    nothing is in flight) makes every CTA's bounded wait give up: the call
    returns ADF_E_TIMEOUT instead of hanging, and the context then runs a
    normal call correctly.  skip 0 also drains the next chunk's copies, which
    were issued before the wait gave up."""
    c = case(96, 40, 700, 5e-6, 0.25, 0.9)
    adf.kh_test_fault(skip, 64, ctx=ctx)
    with pytest.raises(adf.AdfError) as ei:
        adf.kh_pressure(c["sp"], c["sn"], c["rp"], c["q"], c["f"], c["dt"], c["sigma"], C0,
                        c["aq"], c["af"], rho=RHO, ctx=ctx)
    assert ei.value.code == -6, ei.value
    out, ref = run_pair(adf, oracle, c)  # the hook is one-shot
    assert rel_l2(out, ref) <= RTOL_L2
