"""Target sharding of the Kirchhoff-Helmholtz sum across ranks.

The KH sum of the reference is a loop over targets with the surface sum
inside (src/kh_kernels.jl:272, `Threads.@threads` over targets): targets are
independent.  Across GPUs, one process per GPU, the surface traces are
broadcast once from the rank that holds them, each rank sums a contiguous
block of targets, and the blocks are gathered.  The broadcast and the gather
are the only collectives; torch.distributed carries them (NCCL between GPUs,
gloo on the host).
"""
from __future__ import annotations

import numpy as np


def target_block(n_targets: int, rank: int, world: int) -> tuple[int, int]:
    """[begin, end) of this rank's targets: contiguous blocks whose sizes
    differ by at most one, covering every target exactly once."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    base, extra = divmod(int(n_targets), world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def _broadcast(a: np.ndarray | None, shape, dtype, dist, src: int, device) -> np.ndarray:
    import torch

    t = (torch.from_numpy(np.ascontiguousarray(a)).to(device) if a is not None
         else torch.empty(shape, dtype=getattr(torch, np.dtype(dtype).name), device=device))
    dist.broadcast(t, src=src)
    return t.cpu().numpy()


def kh_sharded(compute, s_pts, s_nrm, in_q, in_f, r_pts, dist=None, src: int = 0,
               device="cpu", r_nrm=None):
    """Runs `compute(s_pts, s_nrm, in_q, in_f, r_pts_block, r_nrm_block)` on
    this rank's block of targets and returns the full (nt, nr) result on
    every rank.

    Without a process group the call is `compute` on all targets.  With one,
    the surface arrays (s_pts, s_nrm (ns, 3) float64; in_q, in_f (nt, ns)
    float32) need only be valid on rank `src`: their shapes and contents are
    broadcast from there, once.  Targets r_pts (and r_nrm, for the normal
    velocity) are known on every rank.  Output blocks are padded to the
    largest block for the all-gather and trimmed afterwards."""
    r_pts = np.asarray(r_pts, np.float64)
    nr = r_pts.shape[0]
    if dist is None:
        return compute(s_pts, s_nrm, in_q, in_f, r_pts, r_nrm)
    import torch

    rank, world = dist.get_rank(), dist.get_world_size()
    # shapes first (ns, nt), then the arrays themselves
    dims = torch.tensor(list(np.shape(in_q)) if rank == src else [0, 0], dtype=torch.int64,
                        device=device)
    dist.broadcast(dims, src=src)
    nt, ns = (int(x) for x in dims.cpu().tolist())
    mine = rank == src
    s_pts = _broadcast(np.asarray(s_pts, np.float64) if mine else None, (ns, 3), np.float64,
                       dist, src, device)
    s_nrm = _broadcast(np.asarray(s_nrm, np.float64) if mine else None, (ns, 3), np.float64,
                       dist, src, device)
    # (nt, ns) Fortran arrays travel as their (ns, nt) C-order transposes
    in_q = _broadcast(np.asarray(in_q, np.float32).T if mine else None, (ns, nt), np.float32,
                      dist, src, device).T
    in_f = _broadcast(np.asarray(in_f, np.float32).T if mine else None, (ns, nt), np.float32,
                      dist, src, device).T
    b, e = target_block(nr, rank, world)
    out = compute(s_pts, s_nrm, np.asfortranarray(in_q), np.asfortranarray(in_f), r_pts[b:e],
                  None if r_nrm is None else np.asarray(r_nrm, np.float64)[b:e])
    width = -(-nr // world)
    blk = np.zeros((width, nt), np.float32)  # this rank's targets, target-major
    blk[:e - b] = np.asarray(out, np.float32).T
    parts = [torch.empty((width, nt), dtype=torch.float32, device=device) for _ in range(world)]
    dist.all_gather(parts, torch.from_numpy(blk).to(device))
    full = np.empty((nt, nr), np.float32, order="F")
    for r, t in enumerate(parts):
        rb, re = target_block(nr, r, world)
        full[:, rb:re] = t.cpu().numpy()[:re - rb].T
    return full
