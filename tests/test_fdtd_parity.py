"""GPU parity of run_fdtd! (through the C-ABI) against the CPU oracle.

Both sides get bit-identical packed inputs (TransceiverGrid, CPML
coefficients, mask); outputs compared: the field, CPML memory, every trace
buffer (rec of p/vx/vy/vz, vn_rec) and the vn2v-modified velocity sources.

Tolerances: the required bar is 1e-5 relative L2 on traces; in the
Float64-intermediate ("promote") mode the kernel repeats the reference's
operation order, so agreement is expected near 1e-7 and asserted at 1e-6.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DX = 0.005
C0, RHO = 343.0, 1.2
DT = 0.5 * DX / C0 / np.sqrt(3.0)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a))


def make_case(adf, oracle, nx, ny, nz, steps, npml=6, shape="sphere", seed=0, n_rec=40,
              vn_inject=True, overlap=False, arith="promote", extra=None):
    kw = dict(tmax=(steps - 0.5) * DT, xmax=(nx - 1) * DX / 2, ymax=(ny - 1) * DX / 2,
              zmax=(nz - 1) * DX / 2, nx=nx, ny=ny, nz=nz, c0=C0, r0=RHO, cf=0.5)
    d = adf.Domain(**kw)
    o = oracle.domain(**kw)
    assert d.nt == steps
    rng = np.random.default_rng(seed)
    tq = oracle.ricker_wavelet(o, 6000.0, injection=False)
    R = 0.35 * min(d.xmax, d.ymax, d.zmax)
    pts, dirs, tfs = [], [], []
    # q source, f source (dipole along a random direction)
    pts.append([0.31 * d.xmax, -0.2 * d.ymax, 0.11 * d.zmax])
    dirs.append([1.0, 0, 0, 0])
    tfs.append(tq * 1e3)
    nv = rng.standard_normal(3)
    nv /= np.linalg.norm(nv)
    pts.append([-0.27 * d.xmax, 0.23 * d.ymax, -0.3 * d.zmax])
    dirs.append([0.0, *nv])
    tfs.append(np.roll(tq, 7) * 2.0)
    if overlap:  # a second source and a receiver inside the first source's stencil
        pts.append([0.31 * d.xmax + 0.2 * DX, -0.2 * d.ymax + 0.1 * DX, 0.11 * d.zmax])
        dirs.append([0.5, 0.3, -0.2, 0.1])
        tfs.append(np.roll(tq, 3) * -500.0)
        pts.append([0.31 * d.xmax - 0.1 * DX, -0.2 * d.ymax, 0.11 * d.zmax + 0.3 * DX])
        dirs.append([0.0, 0.0, 0.0, 1.0])
        tfs.append(np.zeros(steps))
    if extra is not None:  # caller-placed transceivers: extra(d, tq) -> [(point, dir, tf)]
        for pt, dv, tf in extra(d, tq):
            pts.append(pt)
            dirs.append(dv)
            tfs.append(tf)
    rp, rn = oracle.fibonacci_sphere(n_rec, R)
    for i in range(n_rec):
        pts.append(rp[i])
        dirs.append([0.0, *rn[i]])
        tfs.append(np.zeros(steps))
    pts, dirs, tfs = np.array(pts), np.array(dirs), np.array(tfs)
    g = oracle.transceivers_to_grid(o, pts, dirs, tfs)
    if vn_inject:
        g.vn_src[:, 1] = (np.roll(tq, 11) * 0.05).astype(np.float32)
        g.vn_src[:, 2] = (np.roll(tq, 5) * -0.03).astype(np.float32)
    cp = oracle.CpmlState(o, npml, 1e-4, 2000.0)
    mask = None
    if shape != "none":
        size = 0.22 * min(d.xmax, d.ymax, d.zmax)
        cen = (0.02 * d.xmax, 0.0, -0.03 * d.zmax)
        kw = dict(radius=size, center=cen) if shape == "sphere" else dict(length=2 * size, center=cen)
        mask = oracle.build_update_mask(o, shape, **kw)
    field = np.zeros((nx, ny, nz, 4), np.float32, order="F")
    # a non-zero initial field exercises every update path from step 1
    field[..., 0] = rng.standard_normal((nx, ny, nz)).astype(np.float32) * 1e-3
    return d, o, g, cp, mask, field


def to_adf_grid(adf, g):
    return adf.TransceiverGrid([a.copy(order="F") for a in g.idx], [a.copy(order="F") for a in g.w],
                               [a.copy(order="F") for a in g.src], [a.copy(order="F") for a in g.rec],
                               g.dir.copy(order="F"), g.vn_src.copy(order="F"),
                               g.vn_rec.copy(order="F"))


class _Cp:
    """Product-side Cpml carrying the oracle's Float32 coefficients."""

    def __init__(self, adf, cp):
        import acoustic_disguising_b200._lib as L
        self.n = cp.npml
        self.mv = [a.copy(order="F") for a in cp.mv]
        self.mp = [a.copy(order="F") for a in cp.mp]
        self.coef = cp.coef.copy()
        self._L = L

    def _c(self):
        s = self._L.CpmlC()
        s.npml = self.n
        for a in range(3):
            s.mv[a] = self.mv[a].ctypes.data
            s.mp[a] = self.mp[a].ctypes.data
        s.coef = self.coef.ctypes.data
        return s


def run_both(adf, oracle, case, arith="promote", start=1, stop=None):
    d, o, g, cp, mask, field = case
    gg = to_adf_grid(adf, g)
    pc = _Cp(adf, cp)
    f_gpu = field.copy(order="F")
    adf.run_fdtd(d, f_gpu, gg, pc, mask, start_step=start, stop_step=stop, arith=arith)
    f_cpu = field.copy(order="F")
    go = g.copy()
    co = cp.copy()
    oracle.run_fdtd(o, f_cpu, go, co, mask, start_step=start, stop_step=stop, mode=arith)
    return (f_gpu, gg, pc), (f_cpu, go, co)


def assert_parity(gpu, cpu, tol):
    f_gpu, gg, pc = gpu
    f_cpu, go, co = cpu
    errs = {}
    for c in range(4):
        errs[f"field{c}"] = rel_l2(f_gpu[..., c], f_cpu[..., c])
        errs[f"rec{c}"] = rel_l2(gg.rec[c], go.rec[c])
    errs["vn_rec"] = rel_l2(gg.vn_rec, go.vn_rec)
    for c in range(1, 4):
        errs[f"src{c}"] = rel_l2(gg.src[c], go.src[c])
    for a in range(3):
        if co.mv[a].size and np.abs(co.mv[a]).max() > 0:
            errs[f"mv{a}"] = rel_l2(pc.mv[a], co.mv[a])
        if co.mp[a].size and np.abs(co.mp[a]).max() > 0:
            errs[f"mp{a}"] = rel_l2(pc.mp[a], co.mp[a])
    bad = {k: v for k, v in errs.items() if not (v <= tol)}
    assert not bad, f"parity failures {bad}; all {errs}"
    return errs


def test_reciprocity_gpu(adf, oracle, ctx):
    """test/test_reciprocity.jl:18-69 on the GPU, plus trace parity."""
    d = adf.Domain(tmax=4.0e-4, xmax=0.3, nx=51, cf=0.5)
    o = oracle.domain(tmax=4.0e-4, xmax=0.3, nx=51, cf=0.5)
    src, _ = adf.impulsive_wavelet(d, 7000.0)
    zero = np.zeros(d.nt)
    A, B = [0.10, -0.05, 0.02], [-0.04, 0.07, 0.06]

    def record_at(a, b):
        txs = [adf.Transceiver(a, [1.0, 0, 0, 0], src), adf.Transceiver(b, [1.0, 0, 0, 0], zero)]
        g = adf.transceivers_to_grid(d, txs)
        go = oracle.transceivers_to_grid(o, [a, b], [[1, 0, 0, 0], [1, 0, 0, 0]], [src, zero])
        f = np.zeros((51, 51, 51, 4), np.float32, order="F")
        adf.run_fdtd(d, f, g, None, None)
        fo = np.zeros((51, 51, 51, 4), np.float32, order="F")
        oracle.run_fdtd(o, fo, go, oracle.CpmlState(o, 0), None)
        assert rel_l2(g.rec[0], go.rec[0]) < 1e-6
        assert rel_l2(f, fo) < 1e-6
        return g.rec[0][:, 1].copy()

    ab, ba = record_at(A, B), record_at(B, A)
    rms = np.sqrt(np.mean((ab - ba) ** 2))
    peak = np.abs(ab).max()
    assert peak > 0 and rms / peak < 0.01


@pytest.mark.parametrize("nx,ny,nz,npml,shape", [
    (48, 44, 40, 6, "sphere"),     # CPML + mask, several y tiles and z chunks
    (51, 30, 37, 5, "none"),       # nx not a multiple of 4, no mask
    (36, 33, 34, 1, "none"),       # npml=1: p-side CPML off without a mask
    (36, 33, 34, 1, "sphere"),     # npml=1 with a mask: p-side CPML on (no guard)
    (40, 40, 40, 0, "cube"),       # masked, no CPML
    (300, 20, 18, 6, "sphere"),    # five x tiles per row, the last one partial
    (134, 24, 30, 6, "sphere"),    # x tile 1 meets only the v side of the x slab (x = 127)
    (140, 22, 34, 15, "sphere"),   # npml = 15: the widest x slab staged with the field
    (150, 24, 36, 18, "none"),     # npml = 18: x-slab memory read from global memory
])
def test_run_fdtd_parity(adf, oracle, ctx, nx, ny, nz, npml, shape):
    case = make_case(adf, oracle, nx, ny, nz, steps=60, npml=npml, shape=shape, seed=nx + npml)
    gpu, cpu = run_both(adf, oracle, case)
    errs = assert_parity(gpu, cpu, 1e-6)
    assert errs["rec0"] <= 1e-5


@pytest.mark.parametrize("tile", ["8,16", "12,16", "2,8", "5,32"])
def test_tile_shapes(adf, oracle, ctx, monkeypatch, tile):
    """Every tile height / z-chunk depth gives the same result: heights above
    the kernel's 7 rows (clamped to 7), 2-row tiles with short z chunks and
    5-row tiles with 32-plane chunks."""
    monkeypatch.setenv("ADF_TILE", tile)
    case = make_case(adf, oracle, 48, 44, 40, steps=50, npml=6, shape="sphere", seed=17)
    gpu, cpu = run_both(adf, oracle, case)
    errs = assert_parity(gpu, cpu, 1e-6)
    assert errs["rec0"] <= 1e-5


def test_overlapping_stencils_sequential_order(adf, oracle, ctx):
    """Overlapping source/receiver stencils: the reference's threaded loop is
    racy there; both implementations use ascending transceiver order."""
    case = make_case(adf, oracle, 40, 36, 32, steps=40, npml=4, shape="none", seed=3, overlap=True)
    gpu, cpu = run_both(adf, oracle, case)
    assert_parity(gpu, cpu, 1e-6)


def test_entries_on_tile_edges(adf, oracle, ctx):
    """Sources and receivers whose trilinear stencils straddle the step
    kernel's tile edges: x = 63|64 and 127|128 (64-cell x tiles: the halo
    column), y = 6|7 and 13|14 (7-row tiles: the halo row), z = 15|16 and
    31|32 (16-plane chunks: the prologue plane).  Their injection must reach
    the neighbouring tile's recomputed halo and every recording must be
    written once; the result must match the oracle."""
    def edges(d, tq):
        def at(i, j, k):  # fractional P-grid cell coordinates (0-based) -> position
            return [-d.xmax + i * DX, -d.ymax + j * DX, -d.zmax + k * DX]
        n = len(tq)
        return [
            (at(63.5, 6.5, 15.5), [1.0, 0, 0, 0], tq * 700.0),            # q source on three edges
            (at(127.6, 13.4, 31.5), [0.0, 0.6, -0.48, 0.64], tq * 1.5),   # f dipole on three edges
            (at(64.2, 7.3, 16.1), [0.0, 0.0, 0.6, 0.8], np.zeros(n)),     # receivers just across
            (at(63.0, 6.0, 15.0), [0.0, 1.0, 0.0, 0.0], np.zeros(n)),     # on a P node at the edges
            (at(128.4, 20.5, 31.9), [0.0, 0.0, 0.0, 1.0], np.zeros(n)),
            (at(0.6, 27.5, 47.5), [0.0, 1.0, 0.0, 0.0], np.zeros(n)),     # inside the x slab
        ]
    case = make_case(adf, oracle, 140, 30, 50, steps=40, npml=6, shape="sphere", seed=4,
                     n_rec=24, extra=edges)
    gpu, cpu = run_both(adf, oracle, case)
    assert_parity(gpu, cpu, 1e-6)


def test_fp32_mode(adf, oracle, ctx):
    case = make_case(adf, oracle, 44, 40, 36, steps=50, npml=6, shape="sphere", seed=9)
    gpu, cpu = run_both(adf, oracle, case, arith="fp32")
    errs = assert_parity(gpu, cpu, 1e-5)
    assert errs["rec0"] <= 1e-5


def test_partial_step_ranges(adf, oracle, ctx):
    """start_step > 1 (resume) and stop_step < nt, composed = one run."""
    case = make_case(adf, oracle, 40, 36, 40, steps=70, npml=5, shape="sphere", seed=11)
    d, o, g, cp, mask, field = case
    gpu1, cpu1 = run_both(adf, oracle, case, start=1, stop=25)
    case2 = (d, o, cpu1[1], cpu1[2], mask, cpu1[0])
    gpu2, cpu2 = run_both(adf, oracle, case2, start=26, stop=70)
    assert_parity(gpu2, cpu2, 1e-6)


def test_on_step_callback(adf, oracle, ctx):
    case = make_case(adf, oracle, 32, 32, 32, steps=12, npml=3, shape="none", seed=2)
    d, o, g, cp, mask, field = case
    seen = []

    def on_step(it, read):
        seen.append((it, float(np.abs(read(0)).sum())))

    gg = to_adf_grid(adf, g)
    f_gpu = field.copy(order="F")
    adf.run_fdtd(d, f_gpu, gg, _Cp(adf, cp), mask, on_step=on_step)
    assert [s[0] for s in seen] == list(range(1, 13))
    # the last callback saw the returned field
    assert abs(seen[-1][1] - float(np.abs(f_gpu[..., 0]).sum())) <= 1e-6 * seen[-1][1]


def test_cpml_profiles_bit_exact(adf, oracle, ctx):
    for npml, dt, fc in [(10, DT, 2000.0), (12, DT, 2000.0), (1, DT, 3000.0), (0, DT, 3000.0),
                         (7, 2.309e-6, 10e3)]:
        o32, o64 = adf.cpml_profiles(npml, C0, dt, 1e-4, DX * npml if npml else 0.0, fc)
        ref = oracle.cpml_coefficients(npml, C0, dt, 1e-4, DX * npml if npml else 0.0, fc)
        ref32 = np.concatenate([r.astype(np.float32) for r in ref])
        assert np.array_equal(o32, ref32), npml
        # FP64 values agree to a few ulps (device exp vs libm); b-1 cancellation amplifies a
        assert np.allclose(o64, np.concatenate(ref), rtol=1e-12, atol=1e-300)


@pytest.mark.parametrize("shape,kw", [
    ("sphere", dict(radius=24 * DX)),
    ("sphere", dict(radius=0.05, center=(0.011, -0.02, 0.004))),
    ("cube", dict(length=0.1)),
    ("cross", dict(length=0.15)),
    ("ellipsoid", dict(semi_axes=(0.08, 0.06, 0.04), center=(0.0, 0.01, 0.0))),
])
def test_update_mask_bit_exact(adf, oracle, ctx, shape, kw):
    for nx, ny, nz in [(96, 96, 96), (51, 60, 45)]:
        d = adf.Domain(tmax=1e-4, xmax=(nx - 1) * DX / 2, ymax=(ny - 1) * DX / 2,
                       zmax=(nz - 1) * DX / 2, nx=nx, ny=ny, nz=nz, c0=C0, r0=RHO, cf=0.5)
        o = oracle.domain(tmax=1e-4, xmax=(nx - 1) * DX / 2, ymax=(ny - 1) * DX / 2,
                          zmax=(nz - 1) * DX / 2, nx=nx, ny=ny, nz=nz, c0=C0, r0=RHO, cf=0.5)
        m = adf.build_update_mask(d, shape, **kw)
        mo = oracle.build_update_mask(o, shape, **kw).astype(bool)
        assert np.array_equal(m, mo)
        assert m[..., 0].sum() < m[..., 0].size  # a scatterer was carved


def test_injection_coefficients(adf, ctx):
    d = adf.Domain(tmax=1e-3, xmax=0.3, nx=121, c0=C0, r0=RHO, cf=0.5)
    cf, cq, ds = adf.injection_coefficients(d, 0.2, 300)
    ds_ref = 4 * np.pi * 0.2 ** 2 / 300
    cf_ref = ds_ref * d.dt / (RHO * d.dx ** 3)
    assert ds == pytest.approx(ds_ref, rel=1e-15)
    assert cf == pytest.approx(cf_ref, rel=1e-15)
    assert cq == pytest.approx(cf_ref * d.z0 ** 2, rel=1e-15)
