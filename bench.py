#!/usr/bin/env python
"""Benchmark: impulsive Green's-function solves/s on the 256^3 GF-retrieval
workload (rigid sphere scatterer, 10-cell CPML, 2048-point shell, 2000
steps per solve), batched through the C-ABI on B200.

One bench step = one call of adf_gf_solve_batch over `--batch` complete
solves (B sources of the 512-point Fibonacci source sphere): set-up, 2000
time steps for all B solves advanced together (one step-kernel launch per
time step over all of their tiles, graph-captured), and the p / v_n traces copied back.

  value : GF solves/s from device time (CUDA events on the library's
          stream around the stepping of each batch; inputs resident)
  e2e   : GF solves/s from the wall clock around the C-ABI call with host
          buffers (set-up uploads and trace downloads inside; the result
          traces land in page-locked buffers the caller reuses every step)
  roofline : the fused step kernel's algorithmic HBM bytes per launch over
          its mean launch time (per-launch CUDA events), against the
          measured copy bandwidth
  kh    : Kirchhoff-Helmholtz extrapolation of 4096 surface points (Ricker-
          filtered noise traces, 2048 samples at 5 us) to 16384 targets on a
          2 m sphere: TFLOP/s of the KH kernel against the FP32 FMA peak
          measured in the same run, the C-ABI call's wall time, and the
          relative L2 error of a sample of targets against the FP64 oracle
  gf_map : in-loop GF extrapolation (run_fdtd! on 128^3 with a PVFromPin
          map of 256 lags x 256 sources x 256 receivers): device time per
          step of the map's work (the run minus the same run with the map
          discarded)
  gf_map_tensor_core : the same with a 512-lag x 1024 x 1024 map on 96^3:
          the Float64 far-lag kernel against the tensor-core contraction
          (tcgen05 TF32 split), their per-step cost, speedup and agreement,
          and the map bytes per second against the HBM peak
  step512 : one 512^3 solve (12-cell CPML, rigid ellipsoid): the step
          kernel's roofline on the largest single-solve grid
  serving : 100 GF solves of mixed grid sizes (96..256^3), step counts
          (500..3000) and scatterers, Poisson arrivals offered at 4x the plain
          path's capacity, served in real time by the continuous-batching
          server and by the plain one-solve-at-a-time path: p50/p99 latency
          and solves/s of both
  hologram512 : the 512^3 hologram run (12-cell CPML, ellipsoid, C_f/C_q
          injection at 8192 points, 8192-point shell, 4000 steps) and the KH
          pressure of its shell to 16384 targets, through adf_run_fdtd_kh
  parity : the first solve of the workload over its first 200 steps against
          the oracle in the same arithmetic and against the oracle's FP64 run
          (relative L2 of the p and v_n traces), outside the timed region

`--impl reference` times the CPU restatement of the reference's Threads
path (oracle/) on this host's cores on a bounded sample of the same solve.
Multi-GPU (torchrun): each rank runs its own disjoint sources (weak
scaling, no collective in the data path); times are the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 256
DX = 0.005
C0, RHO = 343.0, 1.2
NT = 2000
NPML = 10
N_SRC, R_SRC = 512, 60 * DX
N_REC, R_REC = 2048, 45 * DX
R_SPHERE = 24 * DX
F3DB = 2000.0
PML_FC = 2000.0
METRIC = "GF solves/s"


def dt_of():
    return 0.5 * DX / C0 / math.sqrt(3.0)


def tmax_of(nt):
    return (nt - 0.5) * dt_of()


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=8, help="solves per bench step and rank")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--arith", default="promote", choices=["promote", "fp32"])
    ap.add_argument("--cpu-steps", type=int, default=40,
                    help="time steps of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nt", type=int, default=NT,
                    help="steps per solve (profiling runs only; the metric uses 2000)")
    ap.add_argument("--no-kh", action="store_true", help="skip the KH section")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving section")
    ap.add_argument("--no-step512", action="store_true", help="skip the 512^3 step section")
    ap.add_argument("--no-gf", action="store_true", help="skip the in-loop GF section")
    ap.add_argument("--no-parity", action="store_true", help="skip the parity section")
    ap.add_argument("--no-hologram", action="store_true", help="skip the 512^3 hologram section")
    ap.add_argument("--no-tune", action="store_true",
                    help="use the tune table / default tile shape (profiling runs)")
    ap.add_argument("--hologram-only", action="store_true",
                    help="run only the 512^3 hologram section and print it (profiling runs)")
    ap.add_argument("--hologram-nt", type=int, default=H_NT)
    ap.add_argument("--serving-requests", type=int, default=100)
    ap.add_argument("--serving-resident", type=int, default=0,
                    help="server slot limit (0: HBM budget and work cap only)")
    ap.add_argument("--serving-waves", type=float, default=2.0,
                    help="server work cap in waves of resident step CTAs (0: none)")
    ap.add_argument("--serving-only", action="store_true",
                    help="run only the serving section and print it")
    ap.add_argument("--kh-only", action="store_true",
                    help="run only the KH section and print it (profiling runs)")
    ap.add_argument("--gf-only", action="store_true",
                    help="run only the in-loop GF section and print it (profiling runs)")
    ap.add_argument("--gf-tc-only", action="store_true",
                    help="run only the tensor-core GF section once, no warm-up (profiling runs)")
    ap.add_argument("--gf-tc-io", type=int, default=1024, help="sources = receivers of that map")
    ap.add_argument("--gf-tc-lags", type=int, default=512, help="lags of that map")
    ap.add_argument("--gf-tc-nt", type=int, default=700, help="steps of that run")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.th.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                smax = float(f[1])
            except ValueError:
                continue
            for name, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        load = [s for s in sm if smax and s > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def workload_config(batch, n_gpus):
    return {"workload": "impulsive GF retrieval, 256^3 grid (dx=5 mm, air c0=343 rho=1.2, "
                        "CFL 0.5), rigid sphere r=24 cells, 10-cell CPML (fc 2 kHz, R=1e-4), "
                        "q point sources on a 512-point Fibonacci sphere r=60 cells, p+vn "
                        "recorded on a 2048-point shell r=45 cells, 2000 steps per solve",
            "grid": [N, N, N], "steps_per_solve": NT, "solves_per_step": batch,
            "solves_per_step_all_ranks": batch * n_gpus, "source_wavelet":
                "impulsive_wavelet f_3db=2 kHz", "l2": "fields 268 MB/solve > 126 MB L2",
            "parallelism": f"independent solves sharded over {n_gpus} GPU(s)"}


def make_requests(A, first_source, batch, arith, nt=NT):
    d = A.Domain(tmax=tmax_of(nt), xmax=(N - 1) * DX / 2, nx=N, c0=C0, r0=RHO, cf=0.5)
    assert d.nt == nt
    tf, _ = A.impulsive_wavelet(d, F3DB)
    sp, _ = A.fibonacci_sphere(N_SRC, R_SRC)
    rp, rn = A.fibonacci_sphere(N_REC, R_REC)
    reqs = []
    for b in range(batch):
        k = (first_source + b) % N_SRC
        reqs.append(A.GfRequest(d, sp[k], [1.0, 0.0, 0.0, 0.0], tf, rp, rn, npml=NPML,
                                pml_rcoef=1e-4, pml_fc=PML_FC, scatterer="sphere",
                                scatterer_kw=dict(radius=R_SPHERE), arith=arith))
    return d, reqs


def algorithmic_bytes_per_solve_step(n=N, npml=NPML):
    cells = n ** 3
    field = 32.0 * cells + 0.5 * cells  # 4 fields read + written, 4-bit mask
    psi = 8.0 * 6 * npml * n * n + 8.0 * 6 * (npml + 1) * n * n  # p- and v-side slabs, r+w
    return field + psi


def read_traffic():
    """dram bytes per cell-step of the step kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "fdtd_step_256cube.md")
    if not os.path.exists(p):
        return None
    for ln in open(p):
        if ln.startswith("traffic_bytes_per_cell_step:"):
            try:
                return float(ln.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------------------
# CPU restatement of the reference (oracle/) on this host
# ---------------------------------------------------------------------------
def cpu_sample(steps, threads):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O

    O.build()
    d = O.domain(tmax=tmax_of(NT), xmax=(N - 1) * DX / 2, nx=N, c0=C0, r0=RHO, cf=0.5)
    tf, _ = O.impulsive_wavelet(d, F3DB)
    sp, _ = O.fibonacci_sphere(N_SRC, R_SRC)
    rp, rn = O.fibonacci_sphere(N_REC, R_REC)
    pts = np.vstack([sp[0], rp])
    dirs = np.vstack([[1.0, 0, 0, 0], np.hstack([np.zeros((N_REC, 1)), rn])])
    tfs = np.vstack([tf, np.zeros((N_REC, d.nt))])
    g = O.transceivers_to_grid(d, pts, dirs, tfs)
    cp = O.CpmlState(d, NPML, 1e-4, PML_FC)
    m = O.build_update_mask(d, "sphere", radius=R_SPHERE)
    f = np.zeros((N, N, N, 4), np.float32, order="F")
    O.run_fdtd(d, f, g, cp, m, start_step=1, stop_step=1, nthreads=threads)  # warm
    t0 = time.perf_counter()
    O.run_fdtd(d, f, g, cp, m, start_step=2, stop_step=1 + steps, nthreads=threads)
    sec = time.perf_counter() - t0
    return sec / steps


def parity_section(A, ctx, steps=200, arith="promote"):
    """The headline workload's first solve (256^3, sphere, 2048-point shell)
    over its first `steps` steps through the C-ABI, against the oracle in the
    same arithmetic (the 1e-5 bar) and against the oracle's FP64 run (the
    stated error).  Runs outside the timed region."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O

    O.build()
    _, reqs = make_requests(A, 0, 1, arith, steps)
    req = reqs[0]
    A.gf_solve_batch([req], batched=True, ctx=ctx)
    d = O.domain(tmax=tmax_of(steps), xmax=(N - 1) * DX / 2, nx=N, c0=C0, r0=RHO, cf=0.5)
    pts = np.vstack([req.src_point, req.rec_points])
    dirs = np.vstack([[1.0, 0, 0, 0], np.hstack([np.zeros((N_REC, 1)), req.rec_normals])])
    tfs = np.vstack([req.src_tf, np.zeros((N_REC, steps))])
    m = O.build_update_mask(d, "sphere", radius=R_SPHERE)
    rel = lambda a, b: float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))
    g = O.transceivers_to_grid(d, pts, dirs, tfs)
    f = np.zeros((N, N, N, 4), np.float32, order="F")
    O.run_fdtd(d, f, g, O.CpmlState(d, NPML, 1e-4, PML_FC), m, mode=arith)
    del f
    same = {"p": rel(req.p, g.rec[0][:, 1:]), "vn": rel(req.vn, g.vn_rec[:, 1:])}
    g64 = O.transceivers_to_grid64(d, pts, dirs, tfs)
    f64 = np.zeros((N, N, N, 4), np.float64, order="F")
    O.run_fdtd64(d, f64, g64, O.CpmlState64(d, NPML, 1e-4, PML_FC), m)
    del f64
    fp64 = {"p": rel(req.p, g64.rec[0][:, 1:]), "vn": rel(req.vn, g64.vn_rec[:, 1:])}
    ref64 = {"p": rel(g.rec[0][:, 1:], g64.rec[0][:, 1:]),
             "vn": rel(g.vn_rec[:, 1:], g64.vn_rec[:, 1:])}
    return {"workload": f"source 0 of the headline workload, first {steps} of its {NT} steps, "
                        "p and v_n traces of the 2048-point shell",
            f"rel_l2_vs_{arith}_oracle": same, "rel_l2_vs_fp64_oracle": fp64,
            f"{arith}_oracle_rel_l2_vs_fp64_oracle": ref64,
            "tolerance": 1e-5, "pass": max(same.values()) <= 1e-5}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    per = []
    t_all = time.perf_counter()
    sample = max(2, args.cpu_steps // 10)  # time steps of one solve per bench step
    for i in range(args.warmup + args.steps):
        s = cpu_sample(sample, threads)
        if i >= args.warmup:
            per.append(s)
    sec_per_step = statistics.mean(per)  # per FDTD time step
    sps = 1.0 / (NT * sec_per_step)      # solve-equivalents of 2000 steps per second
    line = {
        "impl": "reference", "metric": METRIC, "value": sps, "unit": "solves/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        # one bench step = the timed sample (`sample` time steps), as measured
        "ms_per_step": sec_per_step * 1e3 * sample, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 intermediates, f32 storage", "data": "synthetic",
        "config": workload_config(1, 1),
        "cpu_baseline": {"value": sps, "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": f"{sample} time steps of one solve per bench step (the "
                                   "bench step); solves/s = its rate over a 2000-step solve"},
        "e2e": {"value": sps, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "CPU restatement (oracle/) of the reference's Threads path; the reference is "
                "Julia and no Julia runtime is available",
        "wall_s": time.perf_counter() - t_all,
    }
    print(json.dumps(line), flush=True)
    return 0



# ---------------------------------------------------------------------------
# Kirchhoff-Helmholtz extrapolation: 4096 surface points -> 16384 targets
# ---------------------------------------------------------------------------
KH_NS, KH_NR, KH_NT, KH_DT = 4096, 16384, 2048, 5e-6
KH_R_SURF, KH_R_TGT, KH_F3DB, KH_SEED = 0.25, 2.0, 20e3, 20261203


def ricker_noise(rng, nt, ns, dt, fc):
    """Ricker-filtered Gaussian noise (nt, ns), unit RMS per column, float32."""
    x = rng.standard_normal((nt, ns))
    half = int(2.0 / fc / dt)
    tw = np.arange(-half, half + 1) * dt
    w = np.pi * fc * tw
    r = (1 - 2 * w * w) * np.exp(-w * w)
    nfft = 1 << int(math.ceil(math.log2(nt + len(r))))
    y = np.fft.irfft(np.fft.rfft(x, nfft, axis=0) * np.fft.rfft(r, nfft)[:, None], nfft,
                     axis=0)[half:half + nt]
    y /= np.sqrt((y * y).mean(axis=0, keepdims=True))
    return np.asfortranarray(y.astype(np.float32))


def kh_section(A, ctx, steps, warmup):
    sp, sn = A.fibonacci_sphere(KH_NS, KH_R_SURF)
    rp, _ = A.fibonacci_sphere(KH_NR, KH_R_TGT)
    rng = np.random.default_rng(KH_SEED)
    p_tr = ricker_noise(rng, KH_NT, KH_NS, KH_DT, 8e3)
    vn_tr = ricker_noise(rng, KH_NT, KH_NS, KH_DT, 8e3)
    sigma = math.sqrt(math.log(2.0)) / (2 * math.pi * KH_F3DB)
    dS = 4 * math.pi * KH_R_SURF ** 2 / KH_NS
    aq, af = -RHO * dS * KH_DT, -dS * KH_DT  # part3_kh_extrapolation.jl:168-185 scales
    peak_tf, _ = A.fp32_fma_peak(ctx)
    # the caller's trace and result buffers, page-locked once and reused
    q_in = A.pinned_zeros((KH_NT, KH_NS))
    f_in = A.pinned_zeros((KH_NT, KH_NS))
    q_in[:] = vn_tr
    f_in[:] = p_tr
    out = A.pinned_zeros((KH_NT, KH_NR))
    kms, walls = [], []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        A.kh_pressure(sp, sn, rp, q_in, f_in, KH_DT, sigma, C0, aq, af, rho=RHO, ctx=ctx, out=out)
        w = time.perf_counter() - t0
        ms, _ = ctx.last_timing()
        if i >= warmup:
            kms.append(ms)
            walls.append(w)
    h2d, d2h = ctx.last_io_bytes()
    flop = 64.0 * KH_NS * KH_NR * KH_NT  # 2 channels x 16 taps x 2 FLOP per pair-sample
    k_ms = statistics.mean(kms)
    achieved = flop / (k_ms / 1e3) / 1e12
    # parity sample: the first 16 targets against the FP64 oracle
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O

    O.build()
    nchk = 16
    ref = O.kh_pressure(sp, sn, rp, vn_tr, p_tr, KH_DT, sigma, C0, aq, af, r_begin=0,
                        r_end=nchk, mode=1)
    rel = float(np.linalg.norm(out[:, :nchk] - ref) / np.linalg.norm(ref))
    return {
        "workload": "KH pressure, 4096 Fibonacci surface points r=0.25 m with normals -> "
                    "16384 targets on a 2 m sphere, 2048 samples at dt=5 us, Gaussian kernel "
                    "f_3db=20 kHz (+-6 sigma, 16 taps), Ricker-filtered noise traces (seeded)",
        "value": flop / (k_ms / 1e3) / 1e12, "unit": "TFLOP/s", "kernel_ms": k_ms,
        "e2e": {"value": flop / statistics.mean(walls) / 1e12, "unit": "TFLOP/s",
                "wall_ms": statistics.mean(walls) * 1e3, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "fp32 fma", "achieved": achieved, "peak": peak_tf,
                     "unit": "TFLOP/s", "frac": achieved / peak_tf,
                     "peak_source": "measured in this run (adf_fp32_fma_peak)",
                     "flop_per_launch": flop, "traffic": None},
        "rel_l2_vs_fp64_oracle": rel, "parity_sample": f"targets 0..{nchk - 1}, all samples",
        "tolerance": 1e-5, "steps": steps, "warmup": warmup,
    }


def kh_sharded_section(A, ctx, dist, device):
    """The KH workload with its targets split across the ranks: rank 0 holds
    the surface traces and broadcasts them once; each rank sums its block of
    targets on its GPU; the blocks are all-gathered.  TFLOP/s from the
    slowest rank's kernel time (max over ranks)."""
    from acoustic_disguising_b200.shard import kh_sharded, target_block

    rank, world = dist.get_rank(), dist.get_world_size()
    sp, sn = A.fibonacci_sphere(KH_NS, KH_R_SURF)
    rp, _ = A.fibonacci_sphere(KH_NR, KH_R_TGT)
    q_in = f_in = None
    if rank == 0:
        rng = np.random.default_rng(KH_SEED)
        f_in = ricker_noise(rng, KH_NT, KH_NS, KH_DT, 8e3)  # p traces
        q_in = ricker_noise(rng, KH_NT, KH_NS, KH_DT, 8e3)  # v_n traces
    sigma = math.sqrt(math.log(2.0)) / (2 * math.pi * KH_F3DB)
    dS = 4 * math.pi * KH_R_SURF ** 2 / KH_NS
    aq, af = -RHO * dS * KH_DT, -dS * KH_DT
    kms = []

    def compute(sp_, sn_, q, f, rp_, _rn):
        out = A.kh_pressure(sp_, sn_, rp_, q, f, KH_DT, sigma, C0, aq, af, rho=RHO, ctx=ctx)
        kms.append(ctx.last_timing()[0])
        return out

    full = None
    for _ in range(2):  # warm-up, then the timed call
        kms.clear()
        full = kh_sharded(compute, sp if rank == 0 else None, sn if rank == 0 else None,
                          q_in, f_in, rp, dist=dist, device=device)
    k_ms = reduce_max(kms[-1], dist, device)
    flop = 64.0 * KH_NS * KH_NR * KH_NT
    b, e = target_block(KH_NR, rank, world)
    return {"workload": "the KH section's workload, targets split across ranks (rank 0 "
                        "broadcasts the surface traces once, blocks all-gathered)",
            "value": flop / (k_ms / 1e3) / 1e12, "unit": "TFLOP/s", "kernel_ms_max": k_ms,
            "targets_per_rank": e - b, "result_shape": list(full.shape)}


# ---------------------------------------------------------------------------
# Serving: Poisson stream of mixed GF solves, batched server vs plain path
# ---------------------------------------------------------------------------
SERVE_SIZES = (96, 128, 160, 192, 256)
SERVE_BUDGET = 120 * 10 ** 9


def serving_requests(A, n_req, seed, sizes=SERVE_SIZES, steps_range=(500, 3001)):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_req):
        n = int(rng.choice(sizes))
        steps = int(rng.integers(*steps_range))
        xmax = (n - 1) * DX / 2
        d = A.Domain(tmax=tmax_of(steps), xmax=xmax, nx=n, c0=C0, r0=RHO, cf=0.5)
        tf, _ = A.impulsive_wavelet(d, F3DB)
        shape = str(rng.choice(["none", "sphere", "cube", "ellipsoid"]))
        size = rng.uniform(0.1, 0.3) * 2 * xmax  # at most 30 % of the domain
        centre = rng.uniform(-0.2, 0.2, 3) * xmax
        kw = {}
        if shape == "sphere":
            kw = dict(radius=size / 2, center=tuple(centre))
        elif shape == "cube":
            kw = dict(length=size, center=tuple(centre))
        elif shape == "ellipsoid":
            kw = dict(semi_axes=tuple(size / 2 * rng.uniform(0.5, 1.0, 3)), center=tuple(centre))
        u = rng.standard_normal(3)
        src = 0.75 * xmax * u / np.linalg.norm(u)
        rp, rn = A.fibonacci_sphere(256, 0.6 * xmax)
        out.append(A.GfRequest(d, src, [1.0, 0.0, 0.0, 0.0], tf, rp, rn, npml=NPML,
                               pml_rcoef=1e-4, pml_fc=PML_FC, scatterer=shape, scatterer_kw=kw))
    return out


def serve_stream(A, ctx, n_req, make, max_resident=0, waves=2.0, load=4.0, seed=20261203):
    """One request stream served twice in real time on the same Poisson
    arrivals, offered at `load` times the plain path's capacity (estimated
    from 8 calibration requests of another seed, then measured): the plain
    path runs one solve at a time (FIFO, one launch sequence per solve); the
    continuous-batching server admits by HBM budget and by work (resident
    step work within `waves` waves of the GPU's resident CTAs).  Latency =
    completion - arrival; solves/s = requests / (last completion - first
    arrival).  `make(n, seed)` builds n requests."""
    svc = []
    for r in make(8, seed + 7):  # calibration (and warm-up)
        t0 = time.perf_counter()
        A.gf_solve_batch([r], batched=False, ctx=ctx)
        svc.append(time.perf_counter() - t0)
    lam = load * len(svc) / sum(svc)
    arr = np.cumsum(np.random.default_rng(seed + 1).exponential(1.0 / lam, n_req))
    arr -= arr[0]
    # plain arm: one solve at a time, in real time on the arrivals
    reqs = make(n_req, seed)
    done, busy = [], 0.0
    t0 = time.perf_counter()
    for a, r in zip(arr, reqs):
        dly = t0 + a - time.perf_counter()
        if dly > 0:
            time.sleep(dly)
        s0 = time.perf_counter()
        A.gf_solve_batch([r], batched=False, ctx=ctx)
        busy += time.perf_counter() - s0
        done.append(time.perf_counter() - t0)
    plain_lat = np.array(done) - arr
    plain_sps = n_req / (done[-1] - arr[0])
    plain_cap = n_req / busy
    # batched arm: the server fed the same arrivals in real time
    reqs = make(n_req, seed)
    srv = A.Server(hbm_budget=SERVE_BUDGET, max_resident=max_resident, ctx=ctx, work_waves=waves)
    ids = []
    t0 = time.perf_counter()
    for a, r in zip(arr, reqs):
        dly = t0 + a - time.perf_counter()
        if dly > 0:
            time.sleep(dly)
        ids.append(srv.submit(r))
    lat, done_at = {}, {}
    while len(lat) < n_req:
        for i in ids:
            if i in lat:
                continue
            st, ms = srv.poll(i)
            if st == 1:
                lat[i] = ms / 1e3
                done_at[i] = time.perf_counter() - t0
            elif st < 0:
                raise RuntimeError(f"serving request {i} failed: {st}")
        time.sleep(0.002)
    cap_items = srv.work_cap
    srv.stop()
    b_lat = np.array([lat[i] for i in ids])
    b_sps = n_req / (max(done_at.values()) - arr[0])
    pct = lambda x, q: float(np.percentile(x, q))
    return {
        "batched": {"solves_per_s": b_sps, "p50_ms": pct(b_lat, 50) * 1e3,
                    "p99_ms": pct(b_lat, 99) * 1e3,
                    "admission": f"HBM budget + work cap {cap_items} step work items "
                                 f"({waves:g} waves of resident CTAs)"
                                 + (f", at most {max_resident} resident" if max_resident else "")},
        "plain": {"solves_per_s": plain_sps, "p50_ms": pct(plain_lat, 50) * 1e3,
                  "p99_ms": pct(plain_lat, 99) * 1e3, "capacity_per_s": plain_cap,
                  "note": "one solve per launch sequence, served in real time (FIFO)"},
        "speedup_solves_per_s": b_sps / plain_sps, "offered_per_s": lam,
        "offered_over_plain_capacity": lam / plain_cap, "requests": n_req,
    }


def serving_section(A, ctx, n_req, max_resident=0, waves=2.0, load=4.0):
    """The mixed stream of the serving workload, and the same stream drawn
    from its two smallest grids (where one solve fills a fraction of the GPU
    and batching pays most)."""
    out = serve_stream(A, ctx, n_req, lambda n, sd: serving_requests(A, n, sd), max_resident,
                       waves, load)
    out["workload"] = (f"{n_req} impulsive GF solves, grids {{96,128,160,192,256}}^3 drawn "
                       "uniformly, 500-3000 steps, scatterer none/sphere/cube/ellipsoid (random "
                       "centre, size <= 30% of the domain), 10-cell CPML, 256-point shell; "
                       f"Poisson arrivals offered at {load:g}x the plain path's estimated "
                       "capacity; 120 GB HBM budget; both arms served in real time")
    small = serve_stream(A, ctx, 64, lambda n, sd: serving_requests(A, n, sd, sizes=(96, 128)),
                         max_resident, waves, load, seed=20261205)
    small["workload"] = ("64 requests of the same stream restricted to 96^3 and 128^3 grids "
                         "(one solve fills 23-41 % of the GPU's resident CTAs)")
    out["small_grids"] = small
    return out

# ---------------------------------------------------------------------------
# The 512^3 step: 12-cell CPML, rigid ellipsoid (semi-axes 80/60/40 cells)
# ---------------------------------------------------------------------------
def step512_section(A, ctx, nt=48, tune=True):
    n, npml = 512, 12
    d = A.Domain(tmax=tmax_of(nt), xmax=(n - 1) * DX / 2, nx=n, c0=C0, r0=RHO, cf=0.5)
    tf, _ = A.impulsive_wavelet(d, F3DB)
    rp, rn = A.fibonacci_sphere(256, 130 * DX)
    req = A.GfRequest(d, [100 * DX, 0.0, 0.0], [1.0, 0.0, 0.0, 0.0], tf, rp, rn, npml=npml,
                      pml_rcoef=1e-4, pml_fc=PML_FC, scatterer="ellipsoid",
                      scatterer_kw=dict(semi_axes=(80 * DX, 60 * DX, 40 * DX)))
    tuned = None
    if tune:
        tuned = A.autotune(n, n, n, npml=npml, n_solves=1, steps=16, ctx=ctx)
    ctx.set_kernel_timing(True)
    ctx.kernel_timing(reset=True)
    A.gf_solve_batch([req], batched=True, ctx=ctx)
    k_ms, k_n = ctx.kernel_timing(reset=True)
    ctx.set_kernel_timing(False)
    per = k_ms / max(k_n, 1)
    byt = algorithmic_bytes_per_solve_step(n, npml)
    peak = hbm_peak()[0]
    gbs = byt / (per / 1e3) / 1e9
    return {"workload": "one 512^3 solve (dx=5 mm air), 12-cell CPML, rigid ellipsoid 80/60/40 "
                        f"cells, point source, 256-point shell, {nt} steps",
            "mean_launch_ms": per, "launches": k_n, "gcell_upd_per_s": n ** 3 / (per / 1e3) / 1e9,
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                         "frac": gbs / peak, "frac_of_nominal_8000": gbs / 8000.0,
                         "bytes_per_launch": byt},
            "tile": {"ty": tuned[0], "nzc": tuned[1]} if tuned else "table/default"}


# ---------------------------------------------------------------------------
# Hologram synthesis at 512^3: distributed C_f/C_q injection at 8192 points,
# an 8192-point recording shell, 4000 steps, then KH to 16384 targets
# ---------------------------------------------------------------------------
H_N, H_NPML, H_NT = 512, 12, 4000
H_NIN, H_RIN, H_NOUT, H_ROUT = 8192, 100 * DX, 8192, 130 * DX
H_SEMI = (80 * DX, 60 * DX, 40 * DX)
H_NR, H_RT, H_F3DB, H_SEED = 16384, 2.0, 20e3, 20261204


def hologram_section(A, ctx, nt=H_NT):
    """build_hologram's run at the large size, end to end through the C-ABI:
    transceivers packed as build_txs does (shell first, then the injection
    surface, directions [0, n]), inner sources p_src = C_q vn and vn_src =
    C_f p (inject_inner_sources!) from seeded band-limited noise traces,
    run_fdtd! over `nt` steps, then the two-way KH pressure of the recorded
    shell to 16384 targets on a 2 m sphere, the traces handed over in HBM."""
    d = A.Domain(tmax=tmax_of(nt), xmax=(H_N - 1) * DX / 2, nx=H_N, c0=C0, r0=RHO, cf=0.5)
    op, on = A.fibonacci_sphere(H_NOUT, H_ROUT)
    ip, inn = A.fibonacci_sphere(H_NIN, H_RIN)
    zero = np.zeros(d.nt)
    txs = [A.Transceiver(op[k], np.r_[0.0, on[k]], zero) for k in range(H_NOUT)]
    txs += [A.Transceiver(ip[k], np.r_[0.0, inn[k]], zero) for k in range(H_NIN)]
    g = A.transceivers_to_grid(d, txs)
    cf_, cq_, _ = A.injection_coefficients(d, H_RIN, H_NIN, ctx=ctx)
    rng = np.random.default_rng(H_SEED)
    p_tr = ricker_noise(rng, nt, H_NIN, d.dt, 2000.0)   # stand-ins for GF-convolved signals
    vn_tr = ricker_noise(rng, nt, H_NIN, d.dt, 2000.0) / (RHO * C0)
    inner = slice(H_NOUT, H_NOUT + H_NIN)
    g.vn_src[:, inner] = cf_ * p_tr
    g.src[0][:, inner] = cq_ * vn_tr
    cp = A.Cpml(d, H_NPML, 1e-4, PML_FC, ctx=ctx)
    m = A.build_update_mask(d, "ellipsoid", ctx=ctx, semi_axes=H_SEMI)
    f = np.zeros((H_N, H_N, H_N, 4), np.float32, order="F")
    rp, _ = A.fibonacci_sphere(H_NR, H_RT)
    sigma = math.sqrt(math.log(2.0)) / (2 * math.pi * H_F3DB)
    dS = 4 * math.pi * H_ROUT ** 2 / H_NOUT
    cols = np.arange(1, H_NOUT + 1, dtype=np.int64)
    ctx.set_kernel_timing(True)
    ctx.kernel_timing(reset=True)
    t0 = time.perf_counter()
    out = A.run_fdtd_kh(d, f, g, cp, m, cols, op, on, rp, sigma, -RHO * dS * d.dt, -dS * d.dt,
                        ctx=ctx)
    wall = time.perf_counter() - t0
    k_ms, k_n = ctx.kernel_timing(reset=True)
    ctx.set_kernel_timing(False)
    run_ms, _ = ctx.last_timing()
    kh_ms = ctx.last_kh_ms()
    per = k_ms / max(k_n, 1)
    byt = algorithmic_bytes_per_solve_step(H_N, H_NPML)
    peak = hbm_peak()[0]
    taps = math.ceil(12 * sigma / d.dt)
    flop = 4.0 * taps * H_NOUT * H_NR * nt  # 2 channels x taps x 2 FLOP per pair-sample
    gbs = byt / (per / 1e3) / 1e9
    return {"workload": f"512^3 (dx=5 mm air), 12-cell CPML, rigid ellipsoid 80/60/40 cells; "
                        f"C_f/C_q injection at {H_NIN} Fibonacci points r=100 cells (seeded "
                        f"band-limited noise traces), {H_NOUT}-point shell r=130 cells, {nt} "
                        f"steps; KH pressure of the shell to {H_NR} targets on a 2 m sphere "
                        f"(f_3db 20 kHz, {taps} taps)",
            "wall_s": wall, "run_ms": run_ms, "gcell_upd_per_s": H_N ** 3 * nt / run_ms / 1e6,
            "step_kernel": {"mean_launch_ms": per, "launches": k_n,
                            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak,
                                         "unit": "GB/s", "frac": gbs / peak,
                                         "frac_of_nominal_8000": gbs / 8000.0,
                                         "bytes_per_launch": byt}},
            "kh": {"kernel_ms": kh_ms, "tflops": flop / (kh_ms / 1e3) / 1e12,
                   "flop": flop, "traces": "recorded shell, handed over in HBM"},
            "shell_p_rms": float(np.sqrt(np.mean(g.rec[0][:, :H_NOUT].astype(np.float64) ** 2))),
            "kh_out_rms": float(np.sqrt(np.mean(out.astype(np.float64) ** 2)))}


def fp32_section(A, ctx, batch, nt=96):
    """The headline launch (batch x 256^3 GF solves) with Float32 arithmetic
    instead of the reference's Float64 promotion: what the promotion costs.
    Not the headline: the reference computes in Float64."""
    _, reqs = make_requests(A, 0, batch, "fp32", nt)
    A.gf_solve_batch(reqs, batched=True, ctx=ctx)  # warm
    ctx.set_kernel_timing(True)
    ctx.kernel_timing(reset=True)
    _, reqs = make_requests(A, 0, batch, "fp32", nt)
    A.gf_solve_batch(reqs, batched=True, ctx=ctx)
    k_ms, k_n = ctx.kernel_timing(reset=True)
    ctx.set_kernel_timing(False)
    per = k_ms / max(k_n, 1)
    return {"workload": f"{batch} x 256^3 GF solves as the headline, {nt} steps, Float32 "
                        "arithmetic (all updates in Float32, as ParallelStencil would compute "
                        "them if it narrowed the Float64 Domain scalars)",
            "mean_launch_ms": per,
            "achieved_gbs": batch * algorithmic_bytes_per_solve_step() / (per / 1e3) / 1e9}


# ---------------------------------------------------------------------------
# In-loop GF extrapolation (run_fdtd! gf_map = PVFromPin) on a 128^3 run
# ---------------------------------------------------------------------------
def gf_section(A, ctx, n=128, nt=300, nt_gf=256, n_io=256, contraction="fp64"):
    d = A.Domain(tmax=tmax_of(nt), xmax=(n - 1) * DX / 2, nx=n, c0=C0, r0=RHO, cf=0.5)
    tf = A.ricker_wavelet(d, 2000.0, injection=False)
    rp, rn = A.fibonacci_sphere(n_io, 40 * DX)   # recording shell (iRec)
    ip, inn = A.fibonacci_sphere(n_io, 30 * DX)  # injection surface (iSrc)
    txs = [A.Transceiver(np.zeros(3), np.array([1.0, 0, 0, 0]), tf * 1e3)]
    txs += [A.Transceiver(rp[k], np.r_[0.0, rn[k]], np.zeros(d.nt)) for k in range(n_io)]
    txs += [A.Transceiver(ip[k], np.r_[0.0, inn[k]], np.zeros(d.nt)) for k in range(n_io)]
    i_rec = np.arange(2, 2 + n_io, dtype=np.int64)
    i_src = np.arange(2 + n_io, 2 + 2 * n_io, dtype=np.int64)
    rng = np.random.default_rng(11)
    shape = (nt_gf, n_io, n_io)
    pp = (rng.standard_normal(shape) * 1e-4).astype(np.float32, order="F")
    vp = (rng.standard_normal(shape) * 1e-4).astype(np.float32, order="F")
    times = {}
    for discard in (True, False):
        g = A.transceivers_to_grid(d, txs)
        cp = A.Cpml(d, NPML, 1e-4, PML_FC)
        f = np.zeros((n, n, n, 4), np.float32, order="F")
        A.run_fdtd(d, f, g, cp, ctx=ctx,
                   gf_map=A.PVFromPin(pp, vp, i_src, i_rec, discard, contraction))
        times[discard] = ctx.last_timing()[0]
    gf_ms = times[False] - times[True]
    lags = sum(min(it, nt_gf) for it in range(1, nt))
    byts = 2.0 * 4 * n_io * n_io * lags  # both tensors' lag slices, read once per step
    flop = 2.0 * 2 * n_io * n_io * lags  # 2 tensors x sources x receivers x lags, FMA = 2
    peak64, _ = A.fp64_fma_peak(ctx)
    achieved = flop / (gf_ms / 1e3) / 1e12 if gf_ms > 0 else None
    return {"workload": f"{n}^3 run_fdtd!, {nt} steps, PVFromPin map {nt_gf} lags x {n_io} "
                        f"sources x {n_io} receivers",
            "run_ms_without_map": times[True], "run_ms_with_map": times[False],
            "gf_ms_per_step": gf_ms / (nt - 1),
            "gf_tensor_gbs": byts / (gf_ms / 1e3) / 1e9 if gf_ms > 0 else None,
            "roofline": {"bound": "fp64 fma (Float64 accumulation, as the reference's)",
                         "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                         "frac": achieved / peak64 if achieved else None,
                         "peak_source": "measured in this run (adf_fp64_fma_peak)",
                         "flop": flop, "time": "run with the map minus the run with it "
                                               "discarded (every GF kernel, per step and "
                                               "per block)"}}


def hbm_peak():
    """The HBM roofline denominator: MEASURED_PEAKS.json's measured copy
    bandwidth when the file is present, else the pool's earlier measurement."""
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs")
    except (OSError, ValueError):
        peak = None
    if peak:
        return float(peak), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6650"


def gf_tc_section(A, ctx, n=96, nt=700, nt_gf=512, n_io=1024):
    """In-loop GF extrapolation with a map whose older lags dominate (512 lags
    x 1024 sources x 1024 receivers, 4.3 GB): the Float64 far-lag kernel
    against the tensor-core contraction (TF32 split into three products).
    GF cost = run with the map minus the run with it discarded; the map bytes
    are the algorithmic reads of both tensors (the far lags once per 32-step
    block, the near lags every step)."""
    d = A.Domain(tmax=tmax_of(nt), xmax=(n - 1) * DX / 2, nx=n, c0=C0, r0=RHO, cf=0.5)
    tf = A.ricker_wavelet(d, 2000.0, injection=False)
    rp, rn = A.fibonacci_sphere(n_io, 30 * DX)
    ip, inn = A.fibonacci_sphere(n_io, 22 * DX)
    txs = [A.Transceiver(np.zeros(3), np.array([1.0, 0, 0, 0]), tf * 1e3)]
    txs += [A.Transceiver(rp[k], np.r_[0.0, rn[k]], np.zeros(d.nt)) for k in range(n_io)]
    txs += [A.Transceiver(ip[k], np.r_[0.0, inn[k]], np.zeros(d.nt)) for k in range(n_io)]
    i_rec = np.arange(2, 2 + n_io, dtype=np.int64)
    i_src = np.arange(2 + n_io, 2 + 2 * n_io, dtype=np.int64)
    rng = np.random.default_rng(12)
    shape = (nt_gf, n_io, n_io)
    pp = np.asfortranarray(rng.standard_normal(shape, dtype=np.float32) * np.float32(1e-6))
    vp = np.asfortranarray(rng.standard_normal(shape, dtype=np.float32) * np.float32(1e-6))
    times, srcs = {}, {}
    for mode in ("discard", "fp64", "tf32x3"):
        g = A.transceivers_to_grid(d, txs)
        cp = A.Cpml(d, NPML, 1e-4, PML_FC)
        f = np.zeros((n, n, n, 4), np.float32, order="F")
        gm = A.PVFromPin(pp, vp, i_src, i_rec, mode == "discard",
                         "fp64" if mode == "discard" else mode)
        A.run_fdtd(d, f, g, cp, ctx=ctx, gf_map=gm)
        times[mode] = ctx.last_timing()[0]
        srcs[mode] = np.array(g.src[0][:, i_src - 1], np.float64)
    del pp, vp
    gf = {m: times[m] - times["discard"] for m in ("fp64", "tf32x3")}
    B = 32
    far = sum(min(it0 + B - 1, nt_gf) - 1 for it0 in range(1, nt, B))  # lags per block
    near = sum(min(min(it, nt_gf), (it - 1) % B + 1) for it in range(1, nt))
    byts = 2.0 * 4 * n_io * n_io * (far + near)
    err = float(np.linalg.norm(srcs["tf32x3"] - srcs["fp64"]) / np.linalg.norm(srcs["fp64"]))
    peak = hbm_peak()
    gbs = byts / (gf["tf32x3"] / 1e3) / 1e9 if gf["tf32x3"] > 0 else None
    return {"workload": f"{n}^3 run_fdtd!, {nt} steps, PVFromPin map {nt_gf} lags x {n_io} "
                        f"sources x {n_io} receivers (seeded)",
            "run_ms": times, "gf_ms_per_step": {m: gf[m] / (nt - 1) for m in gf},
            "speedup_tensor_core": gf["fp64"] / gf["tf32x3"] if gf["tf32x3"] > 0 else None,
            "rel_l2_driven_sources_tf32x3_vs_fp64": err,
            "roofline_tf32x3": {"bound": "hbm (map tensors)", "achieved": gbs,
                                "peak": peak[0], "unit": "GB/s",
                                "frac": gbs / peak[0] if gbs else None,
                                "peak_source": peak[1], "map_bytes": byts,
                                "time": "run with the map minus the run with it discarded "
                                        "(every GF kernel: near lags per step, far lags per "
                                        "block on the tensor cores)"}}


# ---------------------------------------------------------------------------
# multi-rank plumbing (one process per GPU)
# ---------------------------------------------------------------------------
def rank_first_source(step_ix, world, rank, batch):
    """First source index of this rank's batch in bench step `step_ix`: the
    ranks take disjoint, consecutive blocks of `batch` sources (weak scaling)."""
    return (step_ix * world + rank) * batch


def reduce_max(x, dist=None, device=None):
    """Maximum of x over all ranks (x itself without a process group)."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def b200_arm(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import acoustic_disguising_b200 as A

    if not os.path.exists(A.LIB_PATH):
        A.build()
    ctx = A.Context(local)
    ctx.set_kernel_timing(True)

    def barrier():
        if dist is not None:
            dist.barrier()

    B = args.batch
    # the product's tuner picks this grid's tile shape (stored in the tune
    # table beside the library, which every later solve of the size reads)
    tuned = (A.autotune(N, N, N, npml=NPML, n_solves=B, steps=32, ctx=ctx) if not args.no_tune
             else ("table/default", "table/default"))
    step_ix = 0
    # the caller's result buffers (p and v_n traces of every solve), page-locked
    # once and reused by every step, as a serving caller keeps its buffers
    outs = [(A.pinned_zeros((args.nt, N_REC)), A.pinned_zeros((args.nt, N_REC)))
            for _ in range(B)]

    def one_step():
        nonlocal step_ix
        first = rank_first_source(step_ix, world, rank, B)
        step_ix += 1
        _, reqs = make_requests(A, first, B, args.arith, args.nt)
        for r, (p, vn) in zip(reqs, outs):
            r.p, r.vn = p, vn
        t0 = time.perf_counter()
        A.gf_solve_batch(reqs, batched=True, ctx=ctx)
        wall = time.perf_counter() - t0
        dev_ms, launches = ctx.last_timing()
        h2d, d2h = ctx.last_io_bytes()
        return wall, dev_ms, launches, h2d, d2h

    for _ in range(args.warmup):
        one_step()
    ctx.kernel_timing(reset=True)
    clocks = Clocks(local)
    barrier()
    clocks.start()
    t_region = time.perf_counter()
    walls, devs, launches, h2ds, d2hs = [], [], 0, [], []
    for _ in range(args.steps):
        w, dm, ln, h2d, d2h = one_step()
        walls.append(w)
        devs.append(dm)
        launches += ln + 4 * B  # + per-solve set-up/extract kernels (cpml, mask, 2 extracts)
        h2ds.append(h2d)
        d2hs.append(d2h)
    barrier()
    region = time.perf_counter() - t_region
    clk = clocks.stop()
    k_ms, k_n = ctx.kernel_timing(reset=True)
    ctx.set_kernel_timing(False)
    extra = {}
    if world == 1 and not args.no_kh:
        extra["kh"] = kh_section(A, ctx, steps=3, warmup=1)
    if world > 1 and not args.no_kh:  # every rank takes part in the collectives
        extra["kh_sharded"] = kh_sharded_section(A, ctx, dist, f"cuda:{local}")
    if world == 1 and not args.no_gf:
        gf_section(A, ctx, nt=40)  # warm-up: graphs, pool blocks
        extra["gf_map"] = gf_section(A, ctx)
        gf_tc_section(A, ctx, nt=80, nt_gf=64, n_io=256)  # warm-up of both contractions
        extra["gf_map_tensor_core"] = gf_tc_section(A, ctx)
    if world == 1 and not args.no_step512:
        extra["step512"] = step512_section(A, ctx)
    if world == 1 and args.arith == "promote":
        extra["arith_fp32"] = fp32_section(A, ctx, B)
    if world == 1 and not args.no_hologram:
        extra["hologram512"] = hologram_section(A, ctx)
    if world == 1 and not args.no_serving:
        extra["serving"] = serving_section(A, ctx, args.serving_requests,
                                           args.serving_resident, args.serving_waves)
    if world == 1 and not args.no_parity:
        extra["parity"] = parity_section(A, ctx, arith=args.arith)
    dev_total = reduce_max(sum(devs), dist, f"cuda:{local}")
    wall_total = reduce_max(sum(walls), dist, f"cuda:{local}")
    k_avg_ms = reduce_max(k_ms / max(k_n, 1), dist, f"cuda:{local}")
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return 0

    solves = world * B * args.steps * args.nt / NT  # solve-equivalents of 2000 steps
    value = solves / (dev_total / 1e3)
    e2e = solves / wall_total
    bytes_launch = B * algorithmic_bytes_per_solve_step()
    achieved = bytes_launch / (k_avg_ms / 1e3) / 1e9
    peak, peak_note = hbm_peak()
    tpc = read_traffic()
    cells = N ** 3
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 intermediates, f32 storage" if args.arith == "promote" else "f32",
        "data": "synthetic (seeded geometry, reference wavelets; no dataset)",
        "config": workload_config(B, world),
        "e2e": {"value": e2e, "unit": "solves/s",
                "h2d_bytes_per_step": int(statistics.mean(h2ds)),
                "d2h_bytes_per_step": int(statistics.mean(d2hs)),
                "wall_ms_per_step": [round(w * 1e3, 1) for w in walls],
                "device_ms_per_step": [round(d, 1) for d in devs]},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_note,
                     "frac_of_nominal_8000": achieved / 8000.0,
                     "traffic": (tpc * cells * B) if tpc else None,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per "
                                       "cell-step of a one-launch capture of this kernel "
                                       "(profiles/fdtd_step_256cube.md), scaled to this "
                                       "launch's cells" if tpc else None,
                     "kernel": "adf_fdtd_step_kernel", "bytes_per_launch": bytes_launch,
                     "mean_launch_ms": k_avg_ms, "launches_timed": k_n},
        "gcell_upd_per_s": cells * NT * solves / (dev_total / 1e3) / 1e9,
        "clocks": clk,
        "region_wall_s": region,
        "tile": {"ty": tuned[0], "nzc": tuned[1], "chosen_by": "adf_autotune"},
    }
    line.update(extra)
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sec = cpu_sample(args.cpu_steps, threads)
        line["cpu_baseline"] = {
            "value": 1.0 / (NT * sec), "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": f"{args.cpu_steps} time steps of one solve of this workload on the CPU "
                      "restatement of the reference (oracle/), extrapolated to 2000 steps"}
    print(json.dumps(line), flush=True)
    return 0


def kh_only(args):
    import acoustic_disguising_b200 as A

    if not os.path.exists(A.LIB_PATH):
        A.build()
    ctx = A.Context(0)
    print(json.dumps({"kh": kh_section(A, ctx, steps=args.steps, warmup=args.warmup)}), flush=True)
    ctx.close()
    return 0


def serving_only(args):
    import acoustic_disguising_b200 as A

    if not os.path.exists(A.LIB_PATH):
        A.build()
    ctx = A.Context(0)
    print(json.dumps({"serving": serving_section(A, ctx, args.serving_requests,
                                                 args.serving_resident, args.serving_waves)}),
          flush=True)
    ctx.close()
    return 0


def hologram_only(args):
    import acoustic_disguising_b200 as A

    if not os.path.exists(A.LIB_PATH):
        A.build()
    ctx = A.Context(0)
    print(json.dumps({"hologram512": hologram_section(A, ctx, nt=args.hologram_nt)}), flush=True)
    ctx.close()
    return 0


def gf_only(args):
    import acoustic_disguising_b200 as A

    if not os.path.exists(A.LIB_PATH):
        A.build()
    ctx = A.Context(0)
    gf_section(A, ctx, nt=40)
    print(json.dumps({"gf_map": gf_section(A, ctx)}), flush=True)
    ctx.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    if args.kh_only:
        return kh_only(args)
    if args.gf_only:
        return gf_only(args)
    if args.gf_tc_only:
        import acoustic_disguising_b200 as A

        ctx = A.Context(0)
        out = gf_tc_section(A, ctx, nt=args.gf_tc_nt, nt_gf=args.gf_tc_lags, n_io=args.gf_tc_io)
        print(json.dumps({"gf_map_tensor_core": out}), flush=True)
        ctx.close()
        return 0
    if args.hologram_only:
        return hologram_only(args)
    if args.serving_only:
        return serving_only(args)
    return b200_arm(args)


if __name__ == "__main__":
    sys.exit(main())
