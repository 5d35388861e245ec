#!/usr/bin/env python
"""Benchmark of the ladder hot path: BSE q.omega points/s, by default on the
SrVO3-like t2g workload (3 orbitals, 20^3 k, 10^3 q, 2x60 fermionic and 21
bosonic frequencies, BSE matrices 1080 x 1080 complex, 21,000 points);
--workload c0 (single orbital, N = 40) and c3 (two-orbital e_g, N = 320,
with the gradient arm) run the other single-problem workloads the same way.

One step = one bosonic slice: the full (q, omega) loop body for all 1000 q
points of one omega (chi0 bubble, both BSE channels, chi sums, EOM).
`value` is the mixed-precision path (FP32 LU with BF16x3 tensor-core updates
and FP64 refinement); the plain FP64 GPU path is timed on the same steps and
reported beside it, with the relative error between the two, and both are
checked against the FP64 oracle over the whole omega = 0 slice (chi_d/m(q, w)
of every point and Sigma(k, nu) accumulated over the slice), the oracle
running on the host cores.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank drives one GPU on its own omega slices (weak
scaling, no data-path collective); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "BSE q·ω pts/s at 1e-8 rel err vs FP64 oracle: mixed-prec vs plain FP64 on B200"
# DRAM bytes / algorithmic bytes of the k_tc_persist launches of one group of three
# steps (two narrow K = 64 regions, two narrow K = 128 regions, one wide K = 192
# region) measured with ncu on the 160-point t2g case, 320 matrices
TRAFFIC_OVER_ALG = 1.06
UNIT = "qw_points/s"
WORKLOAD = "c1"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 arm")
    ap.add_argument("--no-grad", action="store_true",
                    help="skip the gradient arm (ladder + tangents in U, J, t, mixed and FP64)")
    ap.add_argument("--cpu-points", type=int, default=0, help="CPU baseline sample (0 = one per core)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default kernel choices instead of tuning them on the first slice")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the oracle run over the whole omega = 0 slice (errors of both GPU arms "
                         "against the FP64 oracle for chi_d/m(q, omega) and Sigma(k, nu))")
    ap.add_argument("--full-grid", action="store_true",
                    help="also run every omega slice (the whole q x omega grid) in both precisions and "
                         "report the errors of chi_d/m(q, omega) and of the accumulated Sigma(k, nu)")
    ap.add_argument("--compare-library-lu", action="store_true",
                    help="also time the library batched LU (torch.linalg.lu_factor) on matrices of the "
                         "workload's size, FP64 and FP32, for comparison with this library's LU")
    ap.add_argument("--points", type=int, default=0,
                    help="q points per step (0 = the whole slice); smaller cases are for profiling")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# CPU baseline: the FP64 oracle on host cores, one (q, omega) point per worker
# ---------------------------------------------------------------------------
_W = {}


def _cpu_init(workload, iwb):
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    os.environ["OMP_NUM_THREADS"] = "1"
    from adga_b200 import synth
    from oracle.adga_oracle import LadderInputs, Oracle
    p = synth.make_problem(workload)
    s = p.spec
    inp = LadderInputs(ndim=s.ndim, nk=s.nk, nq=s.nq, iwmax=p.iwmax, iwfmax_small=s.iwf,
                       iwbmax_small=s.iwb, beta=p.beta, mu=p.mu, hk=p.hk, siw=p.siw, giw=p.giw,
                       dc=p.dc, u=p.u, u_tilde=p.u_tilde, n_dmft=p.n_dmft, vertex=p.vertex,
                       iw_data=p.iw_data)
    o = Oracle(inp)
    import numpy as np
    scratch = {k: np.zeros((p.ndim2, p.ndim2, 2 * s.iwb + 1), complex)
               for k in ("bubble_loc", "chi_loc_dens", "chi_loc_magn")}
    _W.update(o=o, loc=o.local_block(iwb, 1, scratch), iwb=iwb, p=p)


def _cpu_point(iq):
    """One point of the reference loop body: chi0, BSE build, two zgetrf+zgetri
    inversions, eta, chi sums and the EOM contribution."""
    import numpy as np
    o, loc, iwb, p = _W["o"], _W["loc"], _W["iwb"], _W["p"]
    t = time.perf_counter()
    res = o.point(iq, iwb, loc)
    sig = np.zeros((p.ndim, p.ndim, 2 * p.spec.iwf, p.spec.nkp), complex, order="F")
    o.calc_eom_dynamic(res["etaqd"], res["etaqm"], res["gammaqd"], iwb, iq, sig)
    return time.perf_counter() - t, res["chi_qw_dens"], res["chi_qw_magn"]


# raw accumulators of the reference loop that the parity check compares
ORACLE_KEYS = ("chi_qw_dens", "chi_qw_magn", "bubble_nl", "bubble_loc", "chi_loc_dens", "chi_loc_magn",
               "sigma_nl", "sigma_dmft", "sigma_hf")


def _cpu_block(rng_iq):
    """The reference loop (src/main.F90:486-799) over the contiguous q block
    [a, b) of the worker's omega slice, local terms included where the block
    holds iq = 0: its raw accumulators."""
    o, iwb = _W["o"], _W["iwb"]
    a, b = rng_iq
    out = o.run([(iwb, iq) for iq in range(a, b)])
    return a, b, {k: out[k] for k in ORACLE_KEYS}


class CpuPool:
    def __init__(self, workload, iwb, nproc):
        import multiprocessing as mp
        self.n = nproc
        self.pool = mp.get_context("spawn").Pool(nproc, initializer=_cpu_init, initargs=(workload, iwb))
        self.pool.map(_cpu_point, [0] * nproc)          # warm every worker once

    def step(self, iqs):
        t = time.perf_counter()
        res = self.pool.map(_cpu_point, iqs, chunksize=1)
        return time.perf_counter() - t, res

    def slice_async(self, npts):
        """Start the oracle over q = 0..npts-1 of the slice, one contiguous block
        per worker; returns the async iterator of the blocks."""
        cuts = [round(i * npts / self.n) for i in range(self.n + 1)]
        blocks = [(a, b) for a, b in zip(cuts, cuts[1:]) if b > a]
        return self.pool.imap_unordered(_cpu_block, blocks)

    @staticmethod
    def gather_slice(it, npts):
        """Sum the blocks' accumulators and place their per-point outputs."""
        import numpy as np
        tot = None
        for a, b, out in it:
            if tot is None:
                tot = {k: (np.zeros(v.shape[:-1] + (npts,), complex, order="F")
                           if k in ("chi_qw_dens", "chi_qw_magn", "bubble_nl") else np.zeros_like(v))
                       for k, v in out.items()}
            for k, v in out.items():
                if k in ("chi_qw_dens", "chi_qw_magn", "bubble_nl"):
                    tot[k][..., a:b] = v
                else:
                    tot[k] += v
        return tot

    def close(self):
        self.pool.terminate()


# ---------------------------------------------------------------------------
# Config 4, the uneven-size parameter sweep: the oracle on one (q, omega = 0)
# point of every distinct (ndim, N), in spawned workers on the host cores
# ---------------------------------------------------------------------------
def _c4_cpu_point(spec):
    """Seconds of the FP64 oracle (zgetrf + zgetri inversions, on-the-fly G,
    EOM) for point iq = 1 (0-based) of the omega = 0 slice, single-threaded,
    and its chi_qw_dens / chi_qw_magn."""
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    os.environ["OMP_NUM_THREADS"] = "1"
    import numpy as np
    from adga_b200 import synth
    from oracle.adga_oracle import LadderInputs, Oracle
    p = synth.make_problem(spec)
    s = p.spec
    inp = LadderInputs(ndim=s.ndim, nk=s.nk, nq=s.nq, iwmax=p.iwmax, iwfmax_small=s.iwf, iwbmax_small=s.iwb,
                       beta=p.beta, mu=p.mu, hk=p.hk, siw=p.siw, giw=p.giw, dc=p.dc, u=p.u, u_tilde=p.u_tilde,
                       n_dmft=p.n_dmft, vertex=p.vertex, iw_data=p.iw_data)
    o = Oracle(inp)
    scratch = {k: np.zeros((p.ndim2, p.ndim2, 2 * s.iwb + 1), complex)
               for k in ("bubble_loc", "chi_loc_dens", "chi_loc_magn")}
    loc = o.local_block(0, 1, scratch)
    o.point(0, 0, loc)                                # warm the G caches
    t = time.perf_counter()
    res = o.point(1, 0, loc)
    sig = np.zeros((p.ndim, p.ndim, 2 * s.iwf, s.nkp), complex, order="F")
    o.calc_eom_dynamic(res["etaqd"], res["etaqm"], res["gammaqd"], 0, 1, sig)
    return time.perf_counter() - t, res["chi_qw_dens"], res["chi_qw_magn"]


def run_c4(args):
    """The 64 seeded parameter points (ndim 1/3/5, BSE 40..4000) over all 11
    bosonic frequencies, mixed ladder with the gradients in U and J per point,
    then the FP64 pass (adga_b200.sweep); per-size CPU baseline and oracle probes."""
    import multiprocessing as mp
    import numpy as np
    from adga_b200 import synth
    specs = synth.sweep_specs(64)
    sizes = {}
    for sp in specs:
        sizes.setdefault((sp.ndim, sp.ndim ** 2 * 2 * sp.iwf), []).append(sp)
    keys = sorted(sizes)
    reps = [sizes[k][0] for k in keys]
    cores = os.cpu_count() or 1
    pool = mp.get_context("spawn").Pool(min(len(reps), cores))   # before any GPU call
    job = pool.map_async(_c4_cpu_point, reps, chunksize=1)
    from adga_b200 import sweep
    probes = {sp.name: (0 + sp.iwb) * sp.nqp + 2 for sp in reps}  # omega = 0, iq = 1 (0-based)
    res = sweep.run_sweep(specs, None, check_fp64=True, autotune=True, probes=probes)
    cpu = job.get()
    pool.close()
    summ, recs = res["summary"], {r["name"]: r for r in res["points"]}
    rel = lambda a, b: float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
    per_size, core_s = {}, 0.0
    for k, sp, (sec, cd, cm) in zip(keys, reps, cpu):
        pts = sum(x.nqp * (2 * x.iwb + 1) for x in sizes[k])
        core_s += pts * sec
        pr = recs[sp.name]["probe"]
        per_size[f"ndim{k[0]}_N{k[1]}"] = {
            "parameter_points": len(sizes[k]), "qw_points": pts, "cpu_s_per_point": sec,
            "tune": recs[sp.name]["tune"],
            "mixed_vs_oracle_probe": max(rel(pr["chi_qw_dens"], cd), rel(pr["chi_qw_magn"], cm)),
            "mixed_pts_per_s": sum(recs[x.name]["points"] for x in sizes[k]) /
                               (1e-3 * sum(recs[x.name]["ms_mixed"] for x in sizes[k])),
            "fp64_over_mixed": sum(recs[x.name]["ms_fp64"] for x in sizes[k]) /
                               sum(recs[x.name]["ms_mixed"] for x in sizes[k])}
    cpu_v = summ["qw_points"] / core_s * cores
    line = {"metric": METRIC, "value": summ["pts_per_s_device"], "unit": UNIT, "n_gpus": 1, "steps": 1,
            "warmup": 0, "ms_per_step": summ["ms_mixed"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "mixed: c64 LU (bf16x3 tensor-core updates) + c128 refinement, "
                                          "tangents of U and J in the same pass",
            "data": "synthetic (64 seeded parameter points)",
            "config": {"workload": "c4: uneven-size sweep, 64 parameter points, ndim 1/3/5, BSE N 40..4000, "
                                   "12^3 k, 6^3 q, 11 bosonic frequencies, gradients in U and J per point",
                       "step": "the whole sweep once (each size's kernel choices tuned first, untimed)"},
            "fp64_ms": summ.get("ms_fp64"), "mixed_over_fp64": summ.get("mixed_over_fp64"),
            "max_err_vs_fp64": summ.get("max_err_vs_fp64"), "per_size": per_size,
            "sweep_wall_s": summ["wall_s"], "autotune_wall_s": summ["autotune_wall_s"],
            "cpu_baseline": {"value": cpu_v, "unit": UNIT, "cores": cores, "kind": "port", "cpu_model": cpu_model(),
                             "sample": "one (q, omega=0) point per distinct (ndim, N), FP64 oracle port single-"
                                       "threaded, weighted by each size's share of the points, scaled to all cores"}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, gpu_index=0):
        self.samples, self.proc, self.gpu = [], None, gpu_index

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=5)

    def summary(self):
        import statistics
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text()), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


# ---------------------------------------------------------------------------
def run_reference(args, rank):
    if rank != 0:
        return
    import numpy as np
    from adga_b200 import synth
    spec = synth.SPECS[args.workload]
    cores = os.cpu_count() or 1
    pool = CpuPool(args.workload, 0, cores)
    rng = np.random.default_rng(0)
    times = []
    npts = cores
    for it in range(args.warmup + args.steps):
        iqs = [int(x) for x in rng.integers(0, spec.nqp, npts)]
        dt, _ = pool.step(iqs)
        if it >= args.warmup:
            times.append(dt)
    pool.close()
    v = npts * len(times) / sum(times)
    sample = (f"{npts} (q, omega=0) points per step of the {args.workload} slice, one per process "
              f"on {cores} host cores, FP64 oracle port (zgetrf+zgetri via OpenBLAS, 1 thread each)")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128 (f64)",
            "data": "synthetic",
            "config": config(args, spec),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
                             "cpu_model": cpu_model()},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


MODELS = {"sc": "single-orbital simple cubic", "t2g": "SrVO3-like t2g", "eg": "two-orbital e_g",
          "d5": "five-orbital d shell"}


def config(args, spec, npts=None):
    n = npts or spec.nqp
    gb = 2 * n * spec.maxdim * (spec.maxdim + spec.ndim2) * 8 / 1e9     # FP32 BSE matrices of a step
    return {"workload": f"{args.workload}: {MODELS.get(spec.model, spec.model)}, ndim={spec.ndim}, "
                        f"k={spec.nk}, q={spec.nq}, 2x{spec.iwf} fermionic x {2 * spec.iwb + 1} bosonic, "
                        f"BSE N={spec.maxdim} complex",
            "points_per_step": n, "step": "one omega slice (all q at one bosonic frequency)",
            "l2": (f"inputs larger than L2 (BSE matrices of one slice: ~{gb:.1f} GB FP32 / ~{2 * gb:.1f} GB FP64)"
                   if gb > 0.126 else f"L2 flushed (512 MB write) before every timed step: the {gb * 1e3:.0f} MB "
                                      f"of FP32 BSE matrices of one slice fit in L2"),
            "parallelism": f"replicas x{args.gpus} (independent omega slices per GPU)"}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        # one GPU per process: the library's runtime and torch both see device 0
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local)
    if args.workload == "c4" and args.impl == "ours":
        if rank == 0:
            run_c4(args)
        return
    if args.impl == "reference":
        if world > 1:
            import torch.distributed as dist
            dist.init_process_group("gloo", init_method="env://")
        run_reference(args, rank)
        if world > 1:
            dist.destroy_process_group()
        return

    import numpy as np
    from adga_b200 import synth
    spec = synth.SPECS[args.workload]
    cores = os.cpu_count() or 1
    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = CpuPool(args.workload, 0, args.cpu_points or cores)   # spawned before any GPU call

    import torch
    import torch.distributed as dist
    from adga_b200 import Ladder
    if world > 1:
        torch.cuda.set_device(0)
        dist.init_process_group("nccl", init_method="env://")

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def allmax(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    p = synth.make_problem(args.workload)
    npts = min(args.points, spec.nqp) if args.points > 0 else spec.nqp
    nw = 2 * spec.iwb + 1
    nsteps = args.warmup + args.steps
    omegas = [(-spec.iwb + (rank * nsteps + s) % nw) for s in range(nsteps)]
    # pinned host copies of the vertices (the e2e inputs)
    pinned = {}
    for iwb in sorted(set(omegas) | {0}):     # omega = 0 is also the CPU-sample slice
        d, m = p.vertex(iwb)
        pd = torch.empty(d.size, dtype=torch.complex128).pin_memory().numpy().reshape(d.shape, order="F")
        pm = torch.empty(m.size, dtype=torch.complex128).pin_memory().numpy().reshape(m.shape, order="F")
        pd[...] = d
        pm[...] = m
        pinned[iwb] = (pd, pm)
    p.clear_vertex_cache()
    lad = Ladder.from_problem(p)
    for iwb, (d, m) in pinned.items():
        lad.set_vertex(iwb, d, m)

    def slice_range(iwb):
        q0 = (iwb + spec.iwb) * spec.nqp + 1
        return q0, q0 + npts - 1

    # a slice whose BSE matrices fit in L2 gets an L2 flush (a 512 MB write,
    # outside the library's timed region) before every timed step
    small = 2 * npts * spec.maxdim * (spec.maxdim + spec.ndim2) * 8 <= 126e6
    flush = torch.empty(64 * 2 ** 20, dtype=torch.float64, device="cuda") if small else None

    def l2_flush():
        if flush is not None:
            flush.add_(1.0)
            torch.cuda.synchronize()

    def timed(prec):
        for s in range(args.warmup):
            lad.ladder_run(*slice_range(omegas[s]), prec)
        barrier()
        ms, stats = 0.0, []
        with ClockSampler() as clk:
            for s in range(args.warmup, nsteps):
                l2_flush()
                _, st = lad.ladder_run(*slice_range(omegas[s]), prec)
                ms += st["ms_total"]
                stats.append(st)
            barrier()
        return allmax(ms), stats, clk.summary()

    # kernel choices of the mixed path, measured on the first warm-up slice (set-up, untimed)
    tuned = None
    if not args.no_autotune:
        t0 = time.perf_counter()
        best, trials = lad.autotune(*slice_range(omegas[0]))
        tuned = {"choice": best, "trials": trials, "sample": "the first warm-up omega slice",
                 "wall_s": time.perf_counter() - t0}
    ms_mixed, st_mixed, clk = timed("mixed")
    v_mixed = world * npts * args.steps / (ms_mixed * 1e-3)
    res = {}
    if not args.no_fp64:
        ms64, st64, clk64 = timed("fp64")
        res["fp64"] = world * npts * args.steps / (ms64 * 1e-3)

    # gradient arm: the ladder with the tangents of (U, J, t) in the same pass
    # (everything the backward of adga_b200.grad needs), mixed and FP64, on the same steps
    grad = None
    if not args.no_grad:
        for d, par in enumerate(synth.PARAMS):
            dhk, du, dut, dvertex = synth.tangent_inputs(p, par)
            lad.set_tangent(dhk, du, dut, direction=d)
            if dvertex is not None:
                for iwb in sorted(set(omegas)):
                    lad.set_vertex_tangent(iwb, *dvertex(iwb), direction=d)
        p.clear_vertex_cache()

        def timed_grad(prec):
            for s in range(args.warmup):
                lad.ladder_run_tangent(*slice_range(omegas[s]), prec)
            barrier()
            ms = 0.0
            for s in range(args.warmup, nsteps):
                l2_flush()
                ms += lad.ladder_run_tangent(*slice_range(omegas[s]), prec)[1]["ms_total"]
            barrier()
            return allmax(ms)

        ms_gm = timed_grad("mixed")
        ms_g64 = timed_grad("fp64")
        lad.clear_tangents()
        # the mixed-precision gradient against the mixed forward, the FP64 one against FP64
        grad = {"directions": list(synth.PARAMS), "precision": "mixed",
                "value": world * npts * args.steps / (ms_gm * 1e-3), "unit": UNIT,
                "ms_per_step": ms_gm / args.steps, "over_mixed_forward": ms_gm / ms_mixed,
                "fp64": {"value": world * npts * args.steps / (ms_g64 * 1e-3), "ms_per_step": ms_g64 / args.steps,
                         "over_fp64_forward": (ms_g64 / ms64) if not args.no_fp64 else None}}

    # whole grid: every omega slice in both precisions, Sigma accumulated over all of them
    full_grid = None
    if args.full_grid:
        for iwb in range(-spec.iwb, spec.iwb + 1):
            if iwb not in pinned:
                lad.set_vertex(iwb, *p.vertex(iwb))
        p.clear_vertex_cache()
        nqw = spec.nqp * nw
        grid_out, grid_ms = {}, {}
        for prec in ("fp64", "mixed"):
            lad.reset_outputs()
            _, stg = lad.ladder_run(1, nqw, prec)
            grid_ms[prec] = stg["ms_total"]
            grid_out[prec] = lad.assemble(lad.get_outputs(), p.siw)
        full_grid = {"qw_points": nqw, "ms_fp64": grid_ms["fp64"], "ms_mixed": grid_ms["mixed"],
                     "mixed_over_fp64": grid_ms["fp64"] / grid_ms["mixed"],
                     "mixed_vs_fp64": {k: float(np.max(np.abs(grid_out["mixed"][k] - grid_out["fp64"][k]))
                                               / np.max(np.abs(grid_out["fp64"][k])))
                                       for k in ("chi_dens", "chi_magn", "sigma")}}
        del grid_out

    # comparison only: a library batched LU on matrices of the same size (not this library's path)
    library_lu = None
    if args.compare_library_lu:
        library_lu = {}
        gen = torch.Generator(device="cuda").manual_seed(0)
        nbse = spec.ndim ** 2 * 2 * spec.iwf
        for name, dt in (("complex128", torch.complex128), ("complex64", torch.complex64)):
            nb = 128
            A = torch.eye(nbse, dtype=dt, device="cuda").expand(nb, nbse, nbse).clone()
            A += 0.02 * torch.randn(nb, nbse, nbse, dtype=dt, device="cuda", generator=gen)
            torch.linalg.lu_factor(A.clone())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            X = A.clone()
            torch.cuda.synchronize()
            e0.record(); torch.linalg.lu_factor(X); e1.record(); torch.cuda.synchronize()
            library_lu[name] = {"ms_per_matrix": e0.elapsed_time(e1) / nb, "batch": nb}
            del A, X
        torch.cuda.empty_cache()

    # accuracy: mixed vs FP64 on the same slice, and vs the oracle on sampled points
    iwb_chk = omegas[-1]
    acc = {}
    lad.reset_outputs()
    lad.ladder_run(*slice_range(iwb_chk), "fp64")
    o64 = lad.get_outputs()
    lad.reset_outputs()
    lad.ladder_run(*slice_range(iwb_chk), "mixed")
    omx = lad.get_outputs()

    def rel(a, b):
        return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))

    a64 = lad.assemble(o64, p.siw)
    amx = lad.assemble(omx, p.siw)
    acc["mixed_vs_fp64"] = {k: rel(amx[k], a64[k]) for k in ("chi_dens", "chi_magn", "sigma")}

    # e2e: through the C ABI with host buffers (pinned h2d of the slice's
    # vertex, the run, d2h of every accumulator) on the device already set up
    e2e_t, h2d, d2h = 0.0, 0, 0
    # pinned host buffers for the accumulators, allocated once like the inputs
    pinned_out = {}
    for k, sh in lad.output_shapes(npts).items():
        n = int(np.prod(sh))
        pinned_out[k] = torch.empty(n, dtype=torch.complex128).pin_memory().numpy().reshape(sh, order="F")
    barrier()
    for s in range(args.warmup, nsteps):
        iwb = omegas[s]
        l2_flush()
        t = time.perf_counter()
        lad.set_vertex(iwb, *pinned[iwb])
        lad.ladder_run(*slice_range(iwb), "mixed")
        out = lad.get_outputs(out=pinned_out)
        e2e_t += time.perf_counter() - t
        h2d = sum(x.nbytes for x in pinned[iwb])
        d2h = sum(v.nbytes for v in out.values())
    e2e_t = allmax(e2e_t)
    e2e = {"value": world * npts * args.steps / e2e_t, "unit": UNIT,
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}

    # CPU baseline (rank 0): the oracle timed on one random point per host core
    cpu_line = None
    if cpu is not None:
        rng = np.random.default_rng(1)
        iqs = [int(x) for x in rng.integers(0, npts, cpu.n)]
        dt, _ = cpu.step(iqs)
        cpu_line = {"value": len(iqs) / dt, "unit": UNIT, "cores": cpu.n, "kind": "port",
                    "cpu_model": cpu_model(),
                    "sample": f"{len(iqs)} random q points of the {args.workload} omega=0 slice, one per "
                              f"process (single-threaded OpenBLAS), FP64 oracle port"}

    # parity at the workload's size (rank 0): the oracle over the whole omega = 0
    # slice on the host cores, against both GPU arms on the same slice -- chi_d/m(q, w)
    # of every point and Sigma(k, nu) accumulated over the slice
    if cpu is not None and not args.no_parity:
        t_or = time.perf_counter()
        job = cpu.slice_async(npts)
        gpu_out = {}
        for prec in ("fp64", "mixed"):
            lad.reset_outputs()
            _, stp = lad.ladder_run(*slice_range(0), prec)
            o = lad.get_outputs()
            gpu_out[prec] = (o, lad.assemble(o, p.siw), stp)
        ref = CpuPool.gather_slice(job, npts)
        t_or = time.perf_counter() - t_or
        from oracle.adga_oracle import LadderInputs, assemble as oracle_assemble
        inp = LadderInputs(ndim=spec.ndim, nk=spec.nk, nq=spec.nq, iwmax=p.iwmax, iwfmax_small=spec.iwf,
                           iwbmax_small=spec.iwb, beta=p.beta, mu=p.mu, hk=p.hk, siw=p.siw, giw=p.giw,
                           dc=p.dc, u=p.u, u_tilde=p.u_tilde, n_dmft=p.n_dmft, vertex=p.vertex,
                           iw_data=p.iw_data)
        ref["qw"] = np.array([(0, iq) for iq in range(npts)], dtype=np.int64)
        want = oracle_assemble(inp, ref)
        want.update({k: ref[k] for k in ("chi_qw_dens", "chi_qw_magn", "sigma_nl", "sigma_dmft")})
        keys = ("chi_dens", "chi_magn", "chi_qw_dens", "chi_qw_magn", "sigma", "sigma_nl", "sigma_dmft")
        for prec, (o, a, stp) in gpu_out.items():
            got = dict(a)
            got.update({k: o[k] for k in ("chi_qw_dens", "chi_qw_magn", "sigma_nl", "sigma_dmft")})
            acc[f"{prec}_vs_oracle"] = {k: rel(got[k], want[k]) for k in keys}
            acc[f"{prec}_vs_oracle"]["fallbacks"] = stp["mixed_fallbacks"]
        acc["oracle_slice"] = {"points": npts, "omega": 0, "oracle_s": t_or, "workers": cpu.n,
                               "what": "normwise max relative error against the FP64 oracle over the "
                                       "whole slice; sigma = Sigma_nl + siw, sigma_nl the non-local "
                                       "part accumulated over the slice's points"}
        p.clear_vertex_cache()
    if cpu is not None:
        cpu.close()

    # roofline of the dominant kernel: the LU trailing update (tensor cores).
    # Its C read-modify-write makes it HBM-bound, so it is reported against
    # the measured copy bandwidth with algorithmic bytes (C read + write, L21
    # and U12 read once per launch region); `traffic` scales them by the DRAM /
    # algorithmic ratio ncu measured on the launches of one group of three steps:
    # TRAFFIC_OVER_ALG.
    pk, pk_kind = peaks()
    gflop = sum(s["trail_gflop"] for s in st_mixed)
    gbytes = sum(s["trail_gbytes"] for s in st_mixed)
    mst = sum(s["ms_trail"] for s in st_mixed)
    nlaunch = max(sum(s["trail_launches"] for s in st_mixed), 1)
    achieved = gbytes / mst * 1e3 if mst else 0.0          # GB/s
    peak = pk.get("hbm_gbs")
    bf16_tf = 3 * gflop / mst if mst else 0.0
    roof = {"kernel": "k_tc_persist: tensor-core LU trailing updates of the mixed path (per group of "
                      "three steps: the narrow K=64 and K=128 updates of the next step's strips, two "
                      "launches each, and the wide K=192 update, one launch; GEMMs only)",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if peak else None,
            "traffic": TRAFFIC_OVER_ALG * gbytes * 1e9 / nlaunch,
            "peak_kind": f"hbm copy bandwidth, {pk_kind}",
            "alg_bytes_per_update": gbytes * 1e9 / nlaunch, "avg_update_ms": mst / nlaunch,
            "updates": nlaunch, "complex_tflops": gflop / mst if mst else 0.0,
            "bf16_tensor_tflops": bf16_tf,
            "tensor_frac": bf16_tf / pk["bf16_tflops_sustained"] if pk.get("bf16_tflops_sustained") else None,
            "tensor_peak_kind": f"bf16 sustained, {pk_kind}"}
    stage_keys = ("ms_chi0", "ms_bse", "ms_lu", "ms_trail", "ms_post", "ms_eom", "ms_total")
    stage = {k: sum(s[k] for s in st_mixed) / args.steps for k in stage_keys}
    stage64 = {k: sum(s[k] for s in st64) / args.steps for k in stage_keys} if not args.no_fp64 else None
    line = {"metric": METRIC, "value": v_mixed, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_mixed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "mixed: c64 LU (bf16x3 tensor-core updates, f32 accumulate) + c128 refinement; "
                     "chi0/EOM c128",
            "data": f"synthetic (seeded {MODELS.get(spec.model, spec.model)} model, "
                    "chi_loc = (chi0_loc^-1 + Gamma)^-1)",
            "config": config(args, spec, npts), "fp64_value": res.get("fp64"),
            "mixed_over_fp64": (v_mixed / res["fp64"]) if res.get("fp64") else None,
            "accuracy": acc, "stage_ms_per_step": stage, "fp64_stage_ms_per_step": stage64,
            "refine": {"max_iters": max(s["max_refine_iters"] for s in st_mixed),
                       "fallbacks": sum(s["mixed_fallbacks"] for s in st_mixed)},
            "gradient": grad, "library_lu": library_lu, "full_grid": full_grid, "autotune": tuned,
            "roofline": roof, "cpu_baseline": cpu_line, "e2e": e2e,
            "gpu_launches": int(sum(s["kernel_launches"] for s in st_mixed)),
            "clocks": {k: clk[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")}}
    lad.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
