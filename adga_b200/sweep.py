"""Uneven-size parameter sweep: many model parameter points (mixed orbital
counts and frequency boxes, so BSE dimensions from 40 to 4000) through the
ladder, each with its gradient in U and J.

Every parameter point is one resident problem (`Ladder`, its own G table,
vertex store and batch buffers sized for its BSE dimension); points run
largest dimension first, each as full-GPU batches of its (q, omega) points,
while a host thread builds the next point's inputs (H(k), G, the local
vertex).  Per point: the mixed-precision ladder with the tangents of U and J
in the same pass (`adga_ladder_run_tangent`), then, on the same handle, the
FP64 ladder with the same tangents, which gives the per-point error of the
mixed outputs and gradients.  Throughput counts mixed device time only.  The
mixed path's kernel choices come from the autotuner, measured once per
(orbital count, BSE size) on the first point of that size and reused.  A
point whose tangent refinement does not converge (the library's
ADGA_ENOCONV) runs its pass again in FP64, recorded as 'fp64_pass'.

    python -m adga_b200.sweep [--points 64] [--omegas all|0] [--no-fp64] [--json FILE]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import time
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import synth
from ._lib import ADGA_ENOCONV
from .ladder import AdgaError, Ladder

GRAD_PARAMS = ("U", "J")


def _rel(a, b):
    den = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b)) / den) if den > 0 else float(np.max(np.abs(a)))


def _prepare(spec, omegas):
    """Host-side inputs of one parameter point: the problem, its vertices and
    the tangent inputs of U and J on the requested bosonic frequencies."""
    prob = synth.make_problem(spec)
    verts = {iwb: prob.vertex(iwb) for iwb in omegas}
    tans = []
    for par in GRAD_PARAMS:
        dhk, du, dut, dvertex = synth.tangent_inputs(prob, par)
        tans.append((dhk, du, dut, {iwb: dvertex(iwb) for iwb in omegas} if dvertex else None))
    return prob, verts, tans


def _ranges(nqp, iwbmax, omegas):
    """1-based compound ranges (qwstart, qwstop) covering the omega slices."""
    return [((iwb + iwbmax) * nqp + 1, (iwb + iwbmax + 1) * nqp) for iwb in sorted(omegas)]


def _run_pass(lad, prob, ranges, precision, probe=None):
    """One pass over the ranges; probe: a 1-based compound point whose raw
    chi_qw_dens / chi_qw_magn are returned as well (in the result's 'probe')."""
    lad.reset_outputs()
    ms, iters, fallbacks, outs, touts, got = 0.0, 0, 0, [], [], None
    for qs, qe in ranges:
        _, st = lad.ladder_run_tangent(qs, qe, precision)
        ms += st["ms_total"]
        iters = max(iters, st["max_refine_iters"])
        fallbacks += st["mixed_fallbacks"]
        raw = lad.get_outputs()
        if probe is not None and qs <= probe <= qe:
            got = {k: raw[k][:, :, probe - qs].copy() for k in ("chi_qw_dens", "chi_qw_magn")}
        outs.append(lad.assemble(raw, prob.siw))
        touts.append([lad.assemble_tangent(lad.get_tangent_outputs(d)) for d in range(len(GRAD_PARAMS))])
    # chi per point of every range, Sigma after the last range (it accumulates)
    chi = {k: np.concatenate([o[k] for o in outs], axis=-1) for k in ("chi_dens", "chi_magn")}
    dchi = [np.concatenate([t[d]["chi_magn"] for t in touts], axis=-1) for d in range(len(GRAD_PARAMS))]
    res = dict(chi_dens=chi["chi_dens"], chi_magn=chi["chi_magn"], sigma=outs[-1]["sigma"],
               dchi_magn=dchi, dsigma=[touts[-1][d]["sigma"] for d in range(len(GRAD_PARAMS))], probe=got)
    return ms, iters, fallbacks, res


def run_point(prepared, omegas, check_fp64=True, keep=False, tune_cache=None, probe=None) -> Dict:
    """One parameter point: mixed ladder + tangents of U and J on the omega
    slices `omegas`, then (check_fp64) the FP64 pass; keep: also return the
    mixed outputs (chi_dens, chi_magn per point, sigma, dchi_magn, dsigma).
    tune_cache: dict of the mixed path's kernel choices per (ndim, N); a
    missing entry is measured with the autotuner on the first omega slice."""
    prob, verts, tans = prepared
    s = prob.spec
    N = s.ndim ** 2 * 2 * s.iwf
    ranges = _ranges(s.nqp, s.iwb, omegas)
    npts = s.nqp * len(omegas)
    tuned = None
    with Ladder.from_problem(prob) as lad:
        for iwb, (d, m) in verts.items():
            lad.set_vertex(iwb, d, m)
        if tune_cache is not None:
            key = (s.ndim, N)
            if key not in tune_cache:
                t0 = time.perf_counter()
                best, trials = lad.autotune(*ranges[0])
                tune_cache[key] = best
                tuned = dict(choice=best, trials=trials, wall_s=time.perf_counter() - t0)
            lad.tune = tune_cache[key]
        for dr, (dhk, du, dut, dv) in enumerate(tans):
            lad.set_tangent(dhk, du, dut, direction=dr)
            if dv:
                for iwb, (a, b) in dv.items():
                    lad.set_vertex_tangent(iwb, a, b, direction=dr)
        fell_back = None
        try:
            ms, iters, fb, mx = _run_pass(lad, prob, ranges, "mixed", probe)
        except AdgaError as e:
            # a tangent refinement that does not converge: the point's pass again in FP64
            # (its accumulators restart from zero), timed as this point's mixed time
            if e.code != ADGA_ENOCONV:
                raise
            fell_back = str(e)
            ms, iters, fb, mx = _run_pass(lad, prob, ranges, "fp64", probe)
        rec = dict(name=s.name, ndim=s.ndim, iwf=s.iwf, beta=s.beta, U=s.U, J=s.J, N=N, points=npts,
                   ms_mixed=ms, pts_per_s=npts / (ms * 1e-3), max_refine_iters=iters, mixed_fallbacks=fb,
                   tune=lad.tune)
        if fell_back:
            rec["fp64_pass"] = fell_back
        if tuned:
            rec["autotune"] = tuned
        if mx["probe"] is not None:
            rec["probe"] = mx["probe"]
        if check_fp64:
            ms64, _, _, f64 = _run_pass(lad, prob, ranges, "fp64")
            rec["ms_fp64"] = ms64
            err = {k: _rel(mx[k], f64[k]) for k in ("chi_dens", "chi_magn", "sigma")}
            for d, par in enumerate(GRAD_PARAMS):
                err[f"dchi_magn/d{par}"] = _rel(mx["dchi_magn"][d], f64["dchi_magn"][d])
                err[f"dsigma/d{par}"] = _rel(mx["dsigma"][d], f64["dsigma"][d])
            rec["err_vs_fp64"] = err
        if keep:
            rec["mixed"] = mx
    return rec


def run_sweep(specs: Sequence, omegas: Optional[Sequence[int]] = None, check_fp64: bool = True,
              log=None, autotune: bool = True, probes: Optional[Dict[str, int]] = None) -> Dict:
    """Run every parameter point (largest BSE dimension first); the next
    point's host inputs are prepared while the current one runs.  autotune:
    the mixed path's kernel choices are measured once per (ndim, N) and
    reused by every point of that size.  probes: {point name: 1-based compound
    point} whose raw chi_qw the records keep ('probe')."""
    order = sorted(specs, key=lambda sp: -(sp.ndim ** 2 * 2 * sp.iwf))
    om = lambda sp: list(range(-sp.iwb, sp.iwb + 1)) if omegas is None else list(omegas)
    recs: List[Dict] = []
    tune_cache = {} if autotune else None
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=1) as pool:
        nxt = pool.submit(_prepare, order[0], om(order[0])) if order else None
        for i, sp in enumerate(order):
            prepared = nxt.result()
            nxt = pool.submit(_prepare, order[i + 1], om(order[i + 1])) if i + 1 < len(order) else None
            rec = run_point(prepared, om(sp), check_fp64, tune_cache=tune_cache,
                            probe=(probes or {}).get(sp.name))
            recs.append(rec)
            if log:
                log(rec)
    wall = time.perf_counter() - t0
    pts = sum(r["points"] for r in recs)
    ms = sum(r["ms_mixed"] for r in recs)
    summary = dict(parameter_points=len(recs), qw_points=pts, ms_mixed=ms,
                   pts_per_s_device=pts / (ms * 1e-3) if ms else None, wall_s=wall,
                   gradient=list(GRAD_PARAMS), precision="mixed",
                   tune={f"ndim{k[0]}_N{k[1]}": v for k, v in (tune_cache or {}).items()},
                   autotune_wall_s=sum(r["autotune"]["wall_s"] for r in recs if "autotune" in r))
    if check_fp64 and recs:
        ms64 = sum(r["ms_fp64"] for r in recs)
        summary["ms_fp64"] = ms64
        summary["mixed_over_fp64"] = ms64 / ms if ms else None
    if check_fp64 and recs:
        keys = recs[0]["err_vs_fp64"].keys()
        summary["max_err_vs_fp64"] = {k: max(r["err_vs_fp64"][k] for r in recs) for k in keys}
    return dict(summary=summary, points=recs)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--points", type=int, default=64, help="parameter points (seeded)")
    ap.add_argument("--seed", type=int, default=4321)
    ap.add_argument("--omegas", default="all", help="'all' or comma-separated bosonic indices, e.g. 0")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 check pass")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default kernel choices")
    ap.add_argument("--json", default=None, help="write the full record to this file")
    args = ap.parse_args(argv)
    specs = synth.sweep_specs(args.points, args.seed)
    omegas = None if args.omegas == "all" else [int(x) for x in args.omegas.split(",")]
    res = run_sweep(specs, omegas, not args.no_fp64,
                    log=lambda r: print(json.dumps({k: v for k, v in r.items() if k != "err_vs_fp64"}),
                                        flush=True), autotune=not args.no_autotune)
    print(json.dumps(res["summary"]), flush=True)
    if args.json:
        with open(args.json, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
