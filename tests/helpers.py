"""Shared helpers of the test-suite: problem cache, oracle adapters, errors."""
import contextlib
import os
from functools import lru_cache

import numpy as np

from adga_b200 import synth
from oracle.adga_oracle import LadderInputs, Oracle, assemble


@lru_cache(maxsize=None)
def problem(name):
    return synth.make_problem(name)


def to_inputs(p, do_chi=True, do_eom=True, bubble_big_box=False, vertex=None):
    s = p.spec
    return LadderInputs(ndim=s.ndim, nk=s.nk, nq=s.nq, iwmax=p.iwmax, iwfmax_small=s.iwf,
                        iwbmax_small=s.iwb, beta=p.beta, mu=p.mu, hk=p.hk, siw=p.siw, giw=p.giw,
                        dc=p.dc, u=p.u, u_tilde=p.u_tilde, n_dmft=p.n_dmft,
                        vertex=vertex or p.vertex, do_chi=do_chi, do_eom=do_eom,
                        bubble_big_box=bubble_big_box, iw_data=p.iw_data)


def qw_points(p, qwstart, qwstop):
    s = p.spec
    return [(-s.iwb + (i - 1) // s.nqp, (i - 1) % s.nqp) for i in range(qwstart, qwstop + 1)]


def oracle_run(p, qwstart=1, qwstop=None, **kw):
    s = p.spec
    qwstop = s.nqp * (2 * s.iwb + 1) if qwstop is None else qwstop
    inp = to_inputs(p, **kw)
    out = Oracle(inp).run(qw_points(p, qwstart, qwstop))
    out.update(assemble(inp, out))
    return out


def rel_err(a, b):
    """normwise max-abs relative error of a against reference b"""
    a = np.asarray(a); b = np.asarray(b)
    den = np.max(np.abs(b))
    if den == 0:
        return float(np.max(np.abs(a)))
    return float(np.max(np.abs(a - b)) / den)


LIBRARY_ENV = ("ADGA_DFT_MIN_POINTS", "ADGA_BUBBLE", "ADGA_MIXED_PIVOT", "ADGA_MAX_REFINE",
               "ADGA_REFINE_EXACT", "ADGA_NO_PAIRS", "ADGA_TRI_TILE", "ADGA_BATCH", "ADGA_RESID_FP64",
               "ADGA_TRSV_STREAM")


@contextlib.contextmanager
def library_env(settings):
    """The library's ADGA_* switches (read when a handle is created) set to
    `settings` and every other one unset, restored afterwards."""
    old = {k: os.environ.get(k) for k in LIBRARY_ENV}
    for k in old:
        os.environ.pop(k, None)
    os.environ.update(settings)
    try:
        yield
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
