"""Multi-rank host logic on CPU (gloo, world size 2): the mpi_distribute block
split and the reduction/gather of the per-rank outputs reproduce a
single-process run, both through reduce_outputs directly and through
run_ladder_distributed (each rank's GPU ladder replaced by an oracle-backed
stand-in with the same methods).  Each rank computes its block with the FP64
oracle, so no GPU is involved."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from adga_b200 import dist as D


def test_distribute_matches_reference_block_split():
    # rct(i) = (n - disp(i)) / (size + 1 - i), last rank takes the rest
    for n, w in [(21000, 8), (10, 3), (7, 7), (5, 1), (100, 6)]:
        blocks = [D.distribute(n, w, r) for r in range(w)]
        assert blocks[0][0] == 1 and blocks[-1][1] == n
        for (a, b), (c, d) in zip(blocks, blocks[1:]):
            assert c == b + 1
        sizes = D.counts(n, w)
        assert max(sizes) - min(sizes) <= 1 and sum(sizes) == n


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    from tests.helpers import oracle_run, problem
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = problem("t3")
        s = p.spec
        nqw = s.nqp * (2 * s.iwb + 1)
        qs, qe = D.distribute(nqw, world, rank)
        out = oracle_run(p, qwstart=qs, qwstop=qe)
        full = D.reduce_outputs({k: out[k] for k in D.SUMMED + D.GATHERED}, nqw)
        if rank == 0:
            q.put({k: v for k, v in full.items()})
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_reduction_matches_single_process():
    from tests.helpers import oracle_run, problem
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    got = q.get(timeout=240)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    want = oracle_run(problem("t3"))
    for k in D.SUMMED + D.GATHERED:
        a, b = got[k], want[k]
        assert a.shape == b.shape, k
        err = np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)
        assert err < 1e-13, (k, err)


class OracleLadder:
    """Stand-in for adga_b200.Ladder in CPU tests: the same calls
    (set_vertex, ladder_run, get_outputs, close), computed by the oracle."""

    def __init__(self, prob):
        self.p = prob
        self.out = None

    def set_vertex(self, iwb, d, m):
        pass

    def ladder_run(self, qs, qe, precision):
        from oracle.adga_oracle import Oracle
        from tests.helpers import qw_points, to_inputs
        # raw accumulators, as Ladder.get_outputs returns them (no assembly)
        self.out = Oracle(to_inputs(self.p)).run(qw_points(self.p, qs, qe))
        return self.out["status"], {"points": qe - qs + 1}

    def get_outputs(self):
        return {k: self.out[k] for k in D.SUMMED + D.GATHERED}

    def close(self):
        pass


def _worker_run(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    from tests.helpers import problem
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        assert D.rank_device() is None           # gloo: host tensors
        full, status, stats = D.run_ladder_distributed(problem("t3"), "fp64", ladder_factory=OracleLadder)
        if rank == 0:
            q.put({k: full[k] for k in ("chi_dens", "chi_magn", "sigma") + D.SUMMED + D.GATHERED})
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_run_ladder_distributed_matches_single_process():
    from oracle.adga_oracle import Oracle
    from tests.helpers import oracle_run, problem, to_inputs
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_run, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    got = q.get(timeout=240)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    want = oracle_run(problem("t3"))
    raw = Oracle(to_inputs(problem("t3"))).run()
    for k in ("chi_dens", "chi_magn", "sigma") + D.SUMMED + D.GATHERED:
        a, b = got[k], (want if k in ("chi_dens", "chi_magn", "sigma") else raw)[k]
        assert a.shape == b.shape, k
        err = np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)
        assert err < 1e-13, (k, err)
