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

import os
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


def rank_device(group=None):
    """The device the collectives of this rank use: under NCCL the rank's own
    GPU (LOCAL_RANK, else rank modulo the visible GPUs), made current for the
    calling thread so that the library's handle lives there too; None (host
    tensors) under gloo."""
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) != "nccl":
        return None
    ngpu = torch.cuda.device_count()
    local = int(os.environ.get("LOCAL_RANK", dist.get_rank(group) % max(ngpu, 1)))
    torch.cuda.set_device(local)
    return torch.device("cuda", local)


def run_ladder_distributed(prob, precision="fp64", group=None, ladder_factory=None):
    """Each rank runs its block of the full loop on its GPU, then the results
    are combined; returns (assembled outputs, status, stats) on every rank.

    ladder_factory(prob) makes the rank's ladder (default
    ``Ladder.from_problem``); it is called after the rank's GPU is made
    current."""
    import torch.distributed as dist
    s = prob.spec
    nqw = s.nqp * (2 * s.iwb + 1)
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    qs, qe = distribute(nqw, world, rank)
    device = rank_device(group)
    if ladder_factory is None:
        from .ladder import Ladder
        ladder_factory = Ladder.from_problem
    lad = ladder_factory(prob)
    try:
        for iwb in sorted({-s.iwb + (i - 1) // s.nqp for i in range(qs, qe + 1)}):
            lad.set_vertex(iwb, *prob.vertex(iwb))
        status, stats = lad.ladder_run(qs, qe, precision)
        out = lad.get_outputs()
    finally:
        lad.close()
    full = reduce_outputs(out, nqw, group, device=device)
    full.update(assemble_outputs(full, prob, nqw))
    return full, status, stats


def assemble_outputs(full, prob, nqw):
    """chi(q, w) = chi_nl + bubble_nl + chi_loc(w) (chi_loc += bubble_loc) and
    Sigma = Sigma_nl + siw on the diagonal for the whole loop
    (src/main.F90:935-936,1050-1063,1127-1140; add_siw_dmft,
    src/eom_module.f90:237-251)."""
    s = prob.spec
    widx = np.arange(nqw) // s.nqp
    cld = full["chi_loc_dens"] + full["bubble_loc"]
    clm = full["chi_loc_magn"] + full["bubble_loc"]
    res = {"chi_dens": full["chi_qw_dens"] + full["bubble_nl"] + cld[:, :, widx],
           "chi_magn": full["chi_qw_magn"] + full["bubble_nl"] + clm[:, :, widx]}
    sig = full["sigma_nl"].copy(order="F")
    nu = np.arange(-s.iwf, s.iwf) + prob.iwmax
    for b in range(s.ndim):
        sig[b, b] += np.asarray(prob.siw)[nu, b][:, None]
    res["sigma"] = sig
    return res
