"""Impulsive GF solves through the batched engine, the plain path and the
serving loop, against the oracle; each result must be the same alone and in
the mix (impulsive_gfs, src/greens.jl:143-199)."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DX = 0.005
C0, RHO = 343.0, 1.2
DT = 0.5 * DX / C0 / np.sqrt(3.0)


def domain(adf, n, steps):
    return adf.Domain(tmax=(steps - 0.5) * DT, xmax=(n - 1) * DX / 2, nx=n, c0=C0, r0=RHO, cf=0.5)


def make_req(adf, n, steps, scatterer, seed, n_rec=64):
    d = domain(adf, n, steps)
    rng = np.random.default_rng(seed)
    tf, _ = adf.impulsive_wavelet(d, 2000.0 + 500 * (seed % 3))
    rp, rn = adf.fibonacci_sphere(n_rec, 0.3 * d.xmax)
    sp, sn = adf.fibonacci_sphere(16, 0.4 * d.xmax)
    k = seed % 16
    kw = {}
    if scatterer == "sphere":
        kw = dict(radius=0.12 * d.xmax, center=tuple(rng.uniform(-0.02, 0.02, 3) * d.xmax))
    elif scatterer == "cube":
        kw = dict(length=0.2 * d.xmax)
    elif scatterer == "ellipsoid":
        kw = dict(semi_axes=(0.15 * d.xmax, 0.1 * d.xmax, 0.08 * d.xmax))
    direction = [1.0, 0, 0, 0] if seed % 2 == 0 else [0.0, *sn[k]]
    return adf.GfRequest(d, sp[k], direction, tf, rp, rn, npml=6, pml_fc=2000.0,
                         scatterer=scatterer, scatterer_kw=kw)


def oracle_gf(adf, oracle, req):
    d = req.dom
    o = oracle.domain(tmax=d.tmax, xmax=d.xmax, nx=d.nx, c0=C0, r0=RHO, cf=0.5)
    n = req.rec_points.shape[0]
    pts = np.vstack([req.src_point, req.rec_points])
    dirs = np.vstack([req.src_direction, np.hstack([np.zeros((n, 1)), req.rec_normals])])
    tfs = np.vstack([req.src_tf, np.zeros((n, d.nt))])
    g = oracle.transceivers_to_grid(o, pts, dirs, tfs)
    cp = oracle.CpmlState(o, req.npml, req.pml_rcoef, req.pml_fc)
    mask = None
    if req.scatterer != "none":
        mask = oracle.build_update_mask(o, req.scatterer, **req.scatterer_kw)
    f = np.zeros((d.nx, d.ny, d.nz, 4), np.float32, order="F")
    oracle.run_fdtd(o, f, g, cp, mask)
    return g.rec[0][:, 1:], g.vn_rec[:, 1:]


def rel(a, b):
    return float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b))


def test_gf_batched_matches_oracle_and_plain(adf, oracle, ctx):
    specs = [(40, 50, "sphere", 0), (48, 64, "none", 1), (36, 40, "cube", 2),
             (44, 70, "ellipsoid", 3)]
    reqs = [make_req(adf, *s) for s in specs]
    adf.gf_solve_batch(reqs, batched=True)
    plain = [make_req(adf, *s) for s in specs]
    adf.gf_solve_batch(plain, batched=False)
    for r, q in zip(reqs, plain):
        # same kernel, same per-cell arithmetic: alone == in the mix, bit for bit
        assert np.array_equal(r.p, q.p) and np.array_equal(r.vn, q.vn)
    for r in reqs:
        po, vo = oracle_gf(adf, oracle, r)
        assert rel(r.p, po) < 1e-6
        assert rel(r.vn, vo) < 1e-6


def test_gf_batches_reuse_memory_without_carry_over(adf, ctx):
    """Solve memory is recycled between batches by the context's pool: a
    batch, a larger one (longer traces, bigger grid), then the first batch
    again gives the first batch's results bit for bit."""
    small = [(36, 40, "sphere", 0), (40, 30, "none", 1)]
    first = [make_req(adf, *s) for s in small]
    adf.gf_solve_batch(first, batched=True)
    big = [make_req(adf, 48, 90, "cube", 2), make_req(adf, 44, 70, "ellipsoid", 3)]
    adf.gf_solve_batch(big, batched=True)
    again = [make_req(adf, *s) for s in small]
    adf.gf_solve_batch(again, batched=True)
    for a, b in zip(first, again):
        assert np.array_equal(a.p, b.p) and np.array_equal(a.vn, b.vn)


def test_gf_pinned_result_buffers(adf, ctx):
    """Result traces written into caller-owned page-locked buffers
    (pinned_zeros, reused by a second batch) equal those of fresh arrays."""
    specs = [(36, 40, "sphere", 0), (40, 30, "none", 1)]
    fresh = [make_req(adf, *s) for s in specs]
    adf.gf_solve_batch(fresh, batched=True)
    bufs = [(adf.pinned_zeros((r.dom.nt, 64)), adf.pinned_zeros((r.dom.nt, 64))) for r in fresh]
    for _ in range(2):
        reqs = [make_req(adf, *s) for s in specs]
        for r, (p, vn) in zip(reqs, bufs):
            p.fill(np.nan)
            vn.fill(np.nan)
            r.p, r.vn = p, vn
        adf.gf_solve_batch(reqs, batched=True)
        for a, r in zip(fresh, reqs):
            assert r.p is not None and np.array_equal(a.p, r.p) and np.array_equal(a.vn, r.vn)


def test_gf_budget_admission(adf, ctx):
    """A budget that fits about two solves forces waves of admission; results
    equal the unconstrained batch."""
    specs = [(40, 40, "none", s) for s in range(5)]
    free = [make_req(adf, *s) for s in specs]
    adf.gf_solve_batch(free, batched=True)
    srv = adf.Server(hbm_budget=int(2.5 * 40 ** 3 * 4 * 4 * 2 * 1.3) + (8 << 20))
    reqs = [make_req(adf, *s) for s in specs]
    ids = [srv.submit(r) for r in reqs]
    srv.drain()
    for i in ids:
        st, lat = srv.poll(i)
        assert st == 1 and lat > 0
    srv.stop()
    for a, b in zip(free, reqs):
        assert np.array_equal(a.p, b.p) and np.array_equal(a.vn, b.vn)


def test_server_continuous_batching(adf, ctx):
    """Requests arriving while others run are admitted and finish with the
    same result they give alone."""
    specs = [(36, 120, "none", 0), (44, 60, "sphere", 1), (40, 80, "none", 2),
             (48, 50, "cube", 3), (36, 90, "sphere", 4), (40, 40, "none", 5)]
    alone = []
    for s in specs:
        r = make_req(adf, *s)
        adf.gf_solve_batch([r], batched=False)
        alone.append(r)
    srv = adf.Server(max_resident=3)
    reqs = [make_req(adf, *s) for s in specs]
    ids = []
    for r in reqs:
        ids.append(srv.submit(r))
        time.sleep(0.01)
    srv.drain()
    for i in ids:
        assert srv.poll(i)[0] == 1
    srv.stop()
    for a, b in zip(alone, reqs):
        assert np.array_equal(a.p, b.p) and np.array_equal(a.vn, b.vn)


def test_server_work_cap_admission(adf, ctx):
    """Admission by work (a cap of a fraction of one wave of step CTAs): the
    solves still all complete, each with the result it gives alone; a solve
    bigger than the cap is admitted on its own."""
    specs = [(36, 60, "none", 0), (64, 50, "sphere", 1), (40, 70, "none", 2),
             (36, 40, "cube", 3), (44, 30, "sphere", 4)]
    alone = []
    for s in specs:
        r = make_req(adf, *s)
        adf.gf_solve_batch([r], batched=False)
        alone.append(r)
    waves = 64 / ctx.step_resident_ctas()  # 64 work items: a few small solves at a time
    srv = adf.Server(work_waves=waves)
    assert srv.work_cap == 64
    reqs = [make_req(adf, *s) for s in specs]
    ids = [srv.submit(r) for r in reqs]
    srv.drain()
    for i in ids:
        assert srv.poll(i)[0] == 1
    srv.stop()
    for a, b in zip(alone, reqs):
        assert np.array_equal(a.p, b.p) and np.array_equal(a.vn, b.vn)


def test_server_cancel_and_bad_request(adf, ctx):
    srv = adf.Server(max_resident=1)
    r1 = make_req(adf, 40, 400, "none", 0)
    r2 = make_req(adf, 40, 400, "none", 1)
    i1, i2 = srv.submit(r1), srv.submit(r2)
    srv.cancel(i2)
    bad = make_req(adf, 40, 40, "none", 2)
    bad.rec_points = bad.rec_points * 100.0  # receivers far outside the grid
    i3 = srv.submit(bad)
    srv.drain()
    assert srv.poll(i1)[0] == 1
    assert srv.poll(i2)[0] < 0
    assert srv.poll(i3)[0] < 0
    srv.stop()


def test_kernel_timing_in_graphs(adf, ctx):
    """Per-launch step-kernel timing works inside captured graphs."""
    ctx.set_kernel_timing(True)
    ctx.kernel_timing(reset=True)
    reqs = [make_req(adf, 40, 70, "none", s) for s in range(2)]
    adf.gf_solve_batch(reqs, batched=True)
    ms, n = ctx.kernel_timing(reset=True)
    ctx.set_kernel_timing(False)
    assert n == 70 and ms > 0


@pytest.mark.gpu
def test_autotune_stores_a_shape_that_later_solves_use(adf, ctx, tmp_path, monkeypatch):
    table = tmp_path / "tune_table.json"
    monkeypatch.setenv("ADF_TUNE_TABLE", str(table))
    monkeypatch.delenv("ADF_TILE", raising=False)
    ty, nzc, ms = adf.autotune(72, 64, 60, npml=6, n_solves=2, steps=12, ctx=ctx)
    assert ty in (3, 5, 7) and nzc in (8, 16, 32) and ms > 0
    txt = table.read_text()
    assert f'"72,64,60": [{ty}, {nzc}]' in txt
