"""Multi-process (one GPU per rank) host logic of the (q, omega) loop.

The path shards by compound (q, omega) points with no exchange inside the
loop.  Like the reference's MPI runtime, each rank takes one contiguous block
of points (``mpi_distribute``, src/mpi_org.F90:65-98); after the loop the
per-rank accumulators are summed (``MPI_reduce`` of Sigma and of the local
susceptibilities, src/main.F90:845-850, 912-927) and the per-point outputs are
gathered in block order (``MPI_gatherv``, src/main.F90:979, 1052, 1129).

``torch.distributed`` provides the collectives: NCCL between GPUs, gloo for
the CPU tests.  Complex arrays travel as real views.
"""
from __future__ import annotations

from typing import Dict, Tuple

import numpy as np

# accumulators that are summed over ranks, and per-point outputs gathered in order
SUMMED = ("bubble_loc", "chi_loc_dens", "chi_loc_magn", "sigma_nl", "sigma_dmft", "sigma_hf")
GATHERED = ("chi_qw_dens", "chi_qw_magn", "bubble_nl")


def distribute(nqw: int, world: int, rank: int) -> Tuple[int, int]:
    """1-based (qwstart, qwstop) of ``rank``: rct(i) = (nqw - disp(i)) / (world + 1 - i)
    for the first world-1 ranks, the remainder for the last (src/mpi_org.F90:70-79)."""
    disp = [0] * (world + 1)
    rct = [0] * world
    for i in range(world - 1):
        rct[i] = (nqw - disp[i]) // (world - i)
        disp[i + 1] = disp[i] + rct[i]
    rct[world - 1] = nqw - disp[world - 1]
    return disp[rank] + 1, disp[rank] + rct[rank]


def counts(nqw: int, world: int):
    return [distribute(nqw, world, r)[1] - distribute(nqw, world, r)[0] + 1 for r in range(world)]


def _as_real_tensor(a):
    import torch
    return torch.view_as_real(torch.from_numpy(np.ascontiguousarray(a)))


def reduce_outputs(out: Dict[str, np.ndarray], nqw: int, group=None, device=None) -> Dict[str, np.ndarray]:
    """Sum the accumulators and gather the per-point outputs of every rank.

    ``out`` holds this rank's arrays with the point axis last (Fortran order
    as returned by ``Ladder.get_outputs``).  Every rank receives the full
    result (all-reduce / all-gather), so any rank can assemble it.
    """
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    res = {}
    for k in SUMMED:
        if k not in out:
            continue
        t = _as_real_tensor(out[k])
        if device is not None:
            t = t.to(device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        res[k] = torch.view_as_complex(t.cpu()).numpy().reshape(out[k].shape)
    cnt = counts(nqw, world)
    mx = max(cnt)
    for k in GATHERED:
        if k not in out:
            continue
        a = np.moveaxis(np.asarray(out[k]), -1, 0)                 # [point, ...]
        pad = np.zeros((mx,) + a.shape[1:], dtype=a.dtype)
        pad[: a.shape[0]] = a
        t = _as_real_tensor(pad)
        if device is not None:
            t = t.to(device)
        parts = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(parts, t, group=group)
        full = np.concatenate([torch.view_as_complex(p.cpu()).numpy()[: c] for p, c in zip(parts, cnt)])
        res[k] = np.asfortranarray(np.moveaxis(full, 0, -1))
    return res


def run_ladder_distributed(prob, precision="fp64", group=None):
    """Each rank runs its block of the full loop on its GPU, then the results
    are combined; returns the assembled outputs on every rank."""
    import torch.distributed as dist
    from .ladder import Ladder
    s = prob.spec
    nqw = s.nqp * (2 * s.iwb + 1)
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    qs, qe = distribute(nqw, world, rank)
    lad = Ladder.from_problem(prob)
    try:
        for iwb in sorted({-s.iwb + (i - 1) // s.nqp for i in range(qs, qe + 1)}):
            lad.set_vertex(iwb, *prob.vertex(iwb))
        status, stats = lad.ladder_run(qs, qe, precision)
        out = lad.get_outputs()
    finally:
        lad.close()
    full = reduce_outputs(out, nqw, group)
    return full, status, stats
