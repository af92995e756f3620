"""In-loop GF extrapolation: run_fdtd!(...; gf_map = PVFromPin(...)).

extrapolate!(::PVFromPin) (src/kernels/extrapolation.jl:220-235) runs after
v2vn! of every step it < nt (src/kernels/forward.jl:123-128): it forms
pin = (p_rec - z0 vn_rec)/2 over the iRec columns and sets p_src[it+1, iSrc]
and vn_src[it+1, iSrc] from extrapolate_pv_from_pin! (:139-170).  As shipped
those writes land in slice copies and are lost (discard=True reproduces
that); the documented intent is that they drive the sources (discard=False).
"""
import numpy as np
import pytest

from test_fdtd_parity import DT, _Cp, assert_parity, make_case, to_adf_grid


KINDS = {"PVFromPin": 2, "PFromPin": 2, "PVFromPV": 4}


def gf_inputs(ntx, kind="PVFromPin", nt_gf=24, seed=5, scale=2e-3):
    rng = np.random.default_rng(seed)
    i_rec = np.arange(3, 13, dtype=np.int64)   # ten shell receivers (1-based)
    i_src = np.arange(20, 24, dtype=np.int64)  # four other shell points become sources
    assert i_src.max() <= ntx
    if kind == "PVFromPin":
        shape = (nt_gf, i_src.size, i_rec.size)
    else:
        shape = (nt_gf, i_rec.size, i_src.size)
    ts = [(rng.standard_normal(shape) * scale).astype(np.float32, order="F")
          for _ in range(KINDS[kind])]
    return ts, i_src, i_rec


def test_oracle_gf_delta_kernel_copies_pin():
    """Known answer: v_pin = delta at lag 1 on the diagonal, p_pin = 0, so
    p_src[it+1, iSrc[s]] = pin[it, s] and vn_src[it+1, iSrc[s]] = 0."""
    import pyoracle as O

    adf = __import__("acoustic_disguising_b200")
    d, o, g, cp, mask, field = make_case(adf, O, 24, 22, 20, steps=30, npml=4, shape="none", seed=2)
    ntx = g.dir.shape[1]
    i_rec = np.array([3, 4, 5], np.int64)
    i_src = np.array([6, 7, 8], np.int64)
    pp = np.zeros((10, 3, 3), np.float32, order="F")
    vp = np.zeros((10, 3, 3), np.float32, order="F")
    for k in range(3):
        vp[0, k, k] = 1.0
    f = field.copy(order="F")
    O.run_fdtd_gf(o, f, g, cp, mask, "PVFromPin", (pp, vp), i_src, i_rec, o.z0)
    for k in range(3):
        pin = (g.rec[0][:, i_rec[k] - 1].astype(np.float64) -
               g.vn_rec[:, i_rec[k] - 1].astype(np.float64) * o.z0) / 2.0
        assert np.array_equal(g.src[0][1:, i_src[k] - 1], pin[:-1].astype(np.float32))
        assert not np.any(g.vn_src[1:, i_src[k] - 1])
    assert ntx > i_src.max()


def test_oracle_gf_discard_is_the_plain_run():
    import pyoracle as O

    adf = __import__("acoustic_disguising_b200")
    d, o, g, cp, mask, field = make_case(adf, O, 24, 22, 20, steps=30, npml=4, shape="sphere", seed=4)
    ts, isr, irc = gf_inputs(g.dir.shape[1])
    f1, g1, c1 = field.copy(order="F"), g.copy(), cp.copy()
    O.run_fdtd(o, f1, g1, c1, mask)
    f2, g2, c2 = field.copy(order="F"), g.copy(), cp.copy()
    O.run_fdtd_gf(o, f2, g2, c2, mask, "PVFromPin", ts, isr, irc, o.z0, discard=True)
    assert np.array_equal(f1, f2)
    assert np.array_equal(g1.rec[0], g2.rec[0])


@pytest.mark.gpu
@pytest.mark.parametrize("kind,discard,tol,steps,nt_gf", [
    ("PVFromPin", False, 1e-6, 60, 24), ("PVFromPin", True, 1e-6, 60, 24),
    ("PFromPin", False, 1e-6, 60, 24),
    # PVFromPV: the reference sums Float32 terms sequentially in Float32, the
    # GPU in Float64, so the driven sources differ by Float32 round-off
    ("PVFromPV", False, 1e-5, 60, 24),
    # graph-replayed chunks, more lags than the 32 steps of a block: the far
    # lags of each block come from the block-causal kernel
    ("PVFromPin", False, 1e-6, 100, 40), ("PFromPin", False, 1e-6, 100, 40),
])
def test_gf_map_matches_oracle(adf, oracle, ctx, kind, discard, tol, steps, nt_gf):
    case = make_case(adf, oracle, 40, 36, 32, steps=steps, npml=5, shape="sphere", seed=8,
                     n_rec=40)
    d, o, g, cp, mask, field = case
    ts, isr, irc = gf_inputs(g.dir.shape[1], kind, nt_gf=nt_gf)
    gg = to_adf_grid(adf, g)
    pc = _Cp(adf, cp)
    f_gpu = field.copy(order="F")
    adf.run_fdtd(d, f_gpu, gg, pc, mask, gf_map=adf.GfMap(kind, tuple(ts), isr, irc, discard))
    f_cpu = field.copy(order="F")
    go, co = g.copy(), cp.copy()
    oracle.run_fdtd_gf(o, f_cpu, go, co, mask, kind, ts, isr, irc, o.z0, discard=discard)
    errs = assert_parity((f_gpu, gg, pc), (f_cpu, go, co), tol)
    assert errs["rec0"] <= tol
    for k in isr - 1:  # the driven source rows
        a = gg.src[0][:, k].astype(np.float64)
        b = go.src[0][:, k].astype(np.float64)
        if not discard:
            assert np.abs(b).max() > 0
        assert np.linalg.norm(a - b) <= tol * max(np.linalg.norm(b), 1e-30)
        a = gg.vn_src[:, k].astype(np.float64)
        b = go.vn_src[:, k].astype(np.float64)
        assert np.linalg.norm(a - b) <= tol * max(np.linalg.norm(b), 1e-30)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,nt_gf", [("PVFromPin", 100), ("PFromPin", 100),
                                        ("PVFromPin", 20)])
def test_gf_map_tensor_core_contraction(adf, oracle, ctx, kind, nt_gf):
    """contraction="tf32x3": the lags older than each 32-step block summed on
    the tensor cores (TF32 split into three products).  160 sources (two
    128-source tiles, the second mostly padding), 160 receivers, 100 lags
    over 140 steps (five blocks, the later ones with far lags in every
    16-lag chunk); and a 20-lag map, shorter than a block, whose second
    16-lag chunk is mostly padding.  The driven sources, traces and fields
    stay within 1e-5 of the oracle's Float64 sums (the Float32-level bar the
    reference's own PVFromPV accumulation sets), and so does the Float64 GPU
    path."""
    case = make_case(adf, oracle, 40, 36, 32, steps=140, npml=5, shape="sphere", seed=9,
                     n_rec=320)
    d, o, g, cp, mask, field = case
    ntx = g.dir.shape[1]
    i_rec = np.arange(3, 163, dtype=np.int64)
    i_src = np.arange(163, 323, dtype=np.int64)
    assert i_src.max() <= ntx
    shape = (nt_gf, i_src.size, i_rec.size) if kind == "PVFromPin" else (nt_gf, i_rec.size,
                                                                          i_src.size)
    rng = np.random.default_rng(11)
    ts = [(rng.standard_normal(shape) * 2.5e-4).astype(np.float32, order="F") for _ in range(2)]
    runs = {}
    for contraction in ("tf32x3", "fp64"):
        gg = to_adf_grid(adf, g)
        pc = _Cp(adf, cp)
        f_gpu = field.copy(order="F")
        adf.run_fdtd(d, f_gpu, gg, pc, mask,
                     gf_map=adf.GfMap(kind, tuple(ts), i_src, i_rec, False, contraction))
        runs[contraction] = (f_gpu, gg, pc)
    f_cpu = field.copy(order="F")
    go, co = g.copy(), cp.copy()
    oracle.run_fdtd_gf(o, f_cpu, go, co, mask, kind, ts, i_src, i_rec, o.z0, discard=False)
    tol = 1e-5
    errs = assert_parity(runs["tf32x3"], (f_cpu, go, co), tol)
    assert errs["rec0"] <= tol
    tc, fp = runs["tf32x3"][1], runs["fp64"][1]
    for k in i_src - 1:
        b = go.src[0][:, k].astype(np.float64)
        assert np.abs(b[40:]).max() > 0  # the later blocks are driven
        for src in (tc.src[0][:, k], fp.src[0][:, k]):
            a = src.astype(np.float64)
            assert np.linalg.norm(a - b) <= tol * np.linalg.norm(b)
        a = tc.vn_src[:, k].astype(np.float64)
        b = go.vn_src[:, k].astype(np.float64)
        assert np.linalg.norm(a - b) <= tol * max(np.linalg.norm(b), 1e-30)


def test_gf_map_unknown_contraction(adf):
    ts, isr, irc = gf_inputs(40, "PVFromPin")
    with pytest.raises(KeyError):
        adf.GfMap("PVFromPin", tuple(ts), isr, irc, False, "bf16")._c(1.0)


def _tf32_round(x32):
    """Float32 -> TF32 as csrc/gf_tc_kernel.cu splits it (tf32_hi): half a
    TF32 unit added to the bit pattern, the low 13 mantissa bits cleared
    (nearest, ties away from zero)."""
    b = np.ascontiguousarray(x32, dtype=np.float32).view(np.uint32)
    return ((b + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32)


def _tf32_trunc(x32):
    b = np.ascontiguousarray(x32, dtype=np.float32).view(np.uint32)
    return (b & np.uint32(0xFFFFE000)).view(np.float32)


def _split_inputs(n, seed):
    """Float32 map entries and Float64 history samples over 60 binades, a
    third of the map entries with the mantissa's low 13 bits forced to the
    rounding tie (0x1000) or all ones (0x1FFF, where rounding carries into
    the exponent)."""
    rng = np.random.default_rng(seed)
    g = (rng.standard_normal(n) * np.exp2(rng.integers(-30, 30, n))).astype(np.float32)
    gb = g.view(np.uint32)
    k = n // 3
    gb[:k] = (gb[:k] & np.uint32(0xFFFFE000)) | np.uint32(0x1000)
    gb[k:2 * k] |= np.uint32(0x1FFF)
    h = rng.standard_normal(n) * np.exp2(rng.integers(-30, 30, n).astype(np.float64))
    return gb.view(np.float32), h


@pytest.mark.parametrize("tf32_read,bound", [("truncated", 5), ("rounded", 3)])
def test_tf32x3_split_product_error_bound(tf32_read, bound):
    """Precision of the tensor-core contraction per product (no GPU): a
    Float32 map entry g and a Float64 history sample h are split as the
    kernel splits them (gh = TF32 of g, gl = g - gh in Float32; hh = TF32 of
    (float)h, hl = (float)(h - hh)), and gh*hh + gh*hl + gl*hh stands for
    g*h.  gl is exact, gh and hh are TF32 values, and whether the tensor
    cores read the remainders truncated or rounded to TF32 width, the error
    stays below bound * 2^-22 of |g*h|: the dropped gl*hl is below 2^-22,
    each remainder read at TF32 width loses below 2^-21 truncated or 2^-22
    rounded (a factor 1 + 2^-9 covers the parts' own 1 + 2^-11 growth).
    The products of TF32 values are exact in Float64 here and in the tensor
    cores' FP32 products."""
    g, h = _split_inputs(1 << 20, 11)
    gh = _tf32_round(g)
    gl = (g - gh).astype(np.float32)
    assert np.array_equal(gl.astype(np.float64), g.astype(np.float64) - gh.astype(np.float64))
    assert not np.any(gh.view(np.uint32) & np.uint32(0x1FFF))
    hh = _tf32_round(h.astype(np.float32))
    hl = (h - hh.astype(np.float64)).astype(np.float32)
    read = _tf32_trunc if tf32_read == "truncated" else _tf32_round
    f = lambda v: v.astype(np.float64)  # noqa: E731
    approx = f(gh) * f(hh) + f(gh) * f(read(hl)) + f(read(gl)) * f(hh)
    exact = g.astype(np.float64) * h
    rel = np.abs(approx - exact) / np.abs(exact)
    assert rel.max() < bound * 2.0 ** -22 * (1 + 2.0 ** -9)
    # the split is needed: one TF32 product alone is about 2^-11 off
    assert (np.abs(f(gh) * f(hh) - exact) / np.abs(exact)).max() > 2.0 ** -12


def test_gf_tc_history_window_indexes():
    """Index arithmetic of the tensor-core far-lag kernel (csrc/gf_tc_kernel.cu,
    win_of and the B-operand build), restated and checked on the CPU over
    every block start, map length and chunk: each history row a far lag of
    the block reads lies in the chunk's staged window, the window is an even
    run of at most kTcWinD = 64 doubles starting on an even element (16-B
    aligned bulk copy) inside the receiver's row of the history, the chunks
    cover exactly the far lags (lag > step of the block, lag < min(it0 +
    step, ngf)), and far plus near lags (the
    per-step kernel's lag <= step) give the full causal sum."""
    L, N, WIN = 16, 32, 64
    rng = np.random.default_rng(3)
    for nt in (40, 97, 700):
        for ngf in (2, 17, 20, 33, 100, 512):
            for r in (0, 1, 5):  # receiver rows start at r * nt (odd nt: odd starts)
                g0 = r * nt
                for it0 in range(1, nt, N):
                    lag_hi = min(it0 + N - 1, ngf) - 1
                    nch = (lag_hi + L - 1) // L if lag_hi >= 1 else 0
                    covered = set()
                    for c in range(nch):
                        lo = max(0, it0 - 1 - L * (c + 1))
                        hi = min(it0 - 2, it0 + N - 3 - L * c)
                        if hi < lo:
                            gs, cnt = 0, 0
                        else:
                            gs = (g0 + lo) & ~1
                            cnt = (g0 + hi - gs + 2) & ~1
                            assert gs % 2 == 0 and cnt % 2 == 0 and 0 < cnt <= WIN
                            # the copy stays in this receiver's row of the history
                            assert g0 - 1 <= gs and gs + cnt <= (r + 1) * nt
                        for b in range(N):
                            lim = min(it0 + b, ngf)
                            for k in range(L):
                                lag = L * c + 1 + k
                                if not (b < lag < lim):
                                    continue
                                row = it0 - 1 + b - lag
                                assert 0 <= row < nt
                                w = (g0 - gs) + row
                                assert 0 <= w < cnt, (nt, ngf, it0, c, b, lag)
                                covered.add((b, lag))
                    far = {(b, lag) for b in range(N) for lag in range(b + 1, min(it0 + b, ngf))}
                    assert covered == far, (nt, ngf, it0)
    # far + near = the full causal sum, one receiver, one block
    ngf, it0, nt = 100, 65, 200
    G = rng.standard_normal(ngf)
    pin = rng.standard_normal(nt)
    for b in range(N):
        full = sum(G[lag] * pin[it0 - 1 + b - lag] for lag in range(min(it0 + b, ngf)))
        near = sum(G[lag] * pin[it0 - 1 + b - lag] for lag in range(min(b + 1, it0 + b, ngf)))
        far = sum(G[lag] * pin[it0 - 1 + b - lag] for lag in range(b + 1, min(it0 + b, ngf)))
        assert abs(full - (near + far)) <= 1e-12 * (1 + abs(full))


@pytest.mark.gpu
def test_gf_map_tensor_core_contraction_rejects_pvfrompv(adf, oracle, ctx):
    """The tensor-core contraction covers the input-history kinds only."""
    case = make_case(adf, oracle, 24, 22, 20, steps=10, npml=4, shape="none", seed=1)
    d, o, g, cp, mask, field = case
    ts, isr, irc = gf_inputs(g.dir.shape[1], "PVFromPV", nt_gf=4)
    with pytest.raises(adf.AdfError, match="tensor-core"):
        adf.run_fdtd(d, field.copy(order="F"), to_adf_grid(adf, g), _Cp(adf, cp), mask,
                     gf_map=adf.GfMap("PVFromPV", tuple(ts), isr, irc, False, "tf32x3"))


@pytest.mark.gpu
@pytest.mark.parametrize("kind,contraction,tol", [
    ("PVFromPin", "fp64", 1e-6), ("PFromPin", "fp64", 1e-6),
    ("PVFromPin", "tf32x3", 1e-5), ("PFromPin", "tf32x3", 1e-5),
])
def test_gf_map_resumed_run(adf, oracle, ctx, kind, contraction, tol):
    """A run stopped after step 45 and resumed at step 46 matches one
    uninterrupted oracle run: the resumed call starts its 32-step blocks at
    step 46 and takes the input history before it from the host traces (for
    the tensor-core far lags as well, at their Float32-level bar)."""
    case = make_case(adf, oracle, 40, 36, 32, steps=100, npml=5, shape="sphere", seed=8,
                     n_rec=40)
    d, o, g, cp, mask, field = case
    ts, isr, irc = gf_inputs(g.dir.shape[1], kind, nt_gf=40)
    gg = to_adf_grid(adf, g)
    pc = _Cp(adf, cp)
    gm = adf.GfMap(kind, tuple(ts), isr, irc, False, contraction)
    f_gpu = field.copy(order="F")
    adf.run_fdtd(d, f_gpu, gg, pc, mask, stop_step=45, gf_map=gm)
    adf.run_fdtd(d, f_gpu, gg, pc, mask, start_step=46, gf_map=gm)
    f_cpu = field.copy(order="F")
    go, co = g.copy(), cp.copy()
    oracle.run_fdtd_gf(o, f_cpu, go, co, mask, kind, ts, isr, irc, o.z0, discard=False)
    errs = assert_parity((f_gpu, gg, pc), (f_cpu, go, co), tol)
    assert errs["rec0"] <= tol
    for k in isr - 1:
        a = gg.src[0][:, k].astype(np.float64)
        b = go.src[0][:, k].astype(np.float64)
        assert np.abs(b).max() > 0
        assert np.linalg.norm(a - b) <= tol * np.linalg.norm(b)


@pytest.mark.gpu
def test_gf_map_rejects_bad_indices(adf, oracle, ctx):
    case = make_case(adf, oracle, 24, 22, 20, steps=10, npml=4, shape="none", seed=1)
    d, o, g, cp, mask, field = case
    (pp, vp), isr, irc = gf_inputs(g.dir.shape[1], nt_gf=4)
    bad = isr.copy()
    bad[0] = g.dir.shape[1] + 5
    with pytest.raises(adf.AdfError, match="iSrc"):
        adf.run_fdtd(d, field.copy(order="F"), to_adf_grid(adf, g), _Cp(adf, cp), mask,
                     gf_map=adf.PVFromPin(pp, vp, bad, irc))
    with pytest.raises(adf.AdfError, match="lengths"):
        adf.run_fdtd(d, field.copy(order="F"), to_adf_grid(adf, g), _Cp(adf, cp), mask,
                     gf_map=adf.PVFromPin(pp, vp, isr[:2], irc))


def test_oracle_pfrompin_known_answer():
    """PFromPin with pos = delta at lag 1 on the diagonal and neg = 0:
    p_src[it+1] = pin[it] and vn_src[it+1] = pin[it] / z0 (Float32)."""
    import pyoracle as O

    adf = __import__("acoustic_disguising_b200")
    d, o, g, cp, mask, field = make_case(adf, O, 24, 22, 20, steps=25, npml=4, shape="none", seed=3)
    i_rec = np.array([3, 4], np.int64)
    i_src = np.array([6, 7], np.int64)
    pos = np.zeros((6, 2, 2), np.float32, order="F")
    neg = np.zeros((6, 2, 2), np.float32, order="F")
    pos[0, 0, 0] = pos[0, 1, 1] = 1.0
    f = field.copy(order="F")
    O.run_fdtd_gf(o, f, g, cp, mask, "PFromPin", (pos, neg), i_src, i_rec, o.z0)
    for k in range(2):
        pin = ((g.rec[0][:, i_rec[k] - 1].astype(np.float64) -
                g.vn_rec[:, i_rec[k] - 1].astype(np.float64) * o.z0) / 2.0).astype(np.float32)
        assert np.array_equal(g.src[0][1:, i_src[k] - 1], pin[:-1])
        want = (pin[:-1].astype(np.float64) / o.z0).astype(np.float32)
        assert np.array_equal(g.vn_src[1:, i_src[k] - 1], want)
