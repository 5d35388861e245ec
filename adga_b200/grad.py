"""Gradients of the ladder outputs with respect to model parameters.

The derivative machinery is the library's forward-mode tangent ladder
(``adga_ladder_run_tangent``): the hand-written derivative of every stage,
d(A^-1) = -A^-1 dA A^-1 through the BSE with the forward LU factors, the
tangent chi0 and EOM contractions.  A tangent direction is defined by its
input tangents -- dH(k), du, du~ and dchi_loc^{dens,magn}(omega) -- with the
DMFT one-particle inputs (siw, giw, mu, dc, n_dmft) held fixed.  One pass runs
the forward ladder together with up to four directions; more parameters take
more passes.  The backward of the torch.autograd.Function contracts the
incoming gradients with the tangents (PyTorch's convention for a real input
theta and complex outputs y: theta_bar = Re sum conj(y_bar) dy/dtheta).

Two entry points:

* ``ladder_outputs(theta, model)``: any caller model.  ``model.problem(theta)``
  returns the ladder inputs at theta (an object with the fields
  ``Ladder.from_problem`` reads and ``vertex(iwb)``), ``model.tangents(theta,
  i)`` the input tangents of parameter i as (dhk, du, du_tilde, dvertex) --
  each optional, dvertex(iwb) -> (dchi_loc_dens, dchi_loc_magn).  Returns
  chi_d(q, omega), chi_m(q, omega) of every point and Sigma(k, nu).
* ``ladder_chi_sigma(params, base)``: the synthetic model's (U, J, t) --
  Kanamori couplings (V = U - 2J) and hopping scale -- through
  ``SynthModel``; returns chi_m(q, omega = 0) and Sigma(k, nu).

Not covered: tangents together with the non-local interaction V(q) (the
library rejects them), derivatives with respect to the DMFT one-particle
inputs themselves.
"""
from __future__ import annotations

from typing import Callable, List, Sequence, Tuple

import numpy as np
import torch

from . import synth
from .ladder import Ladder
from ._lib import ADGA_FP64  # noqa: F401  (precision names below mirror the C constants)

MAX_DIRECTIONS = 4          # ADGA_MAX_TANGENTS: directions per pass


class SynthModel:
    """The synthetic model as a differentiable model of (U, J, t) at the DMFT
    one-particle inputs of ``base``."""

    names = synth.PARAMS

    def __init__(self, base):
        self.base = base

    def theta0(self):
        s = self.base.spec
        return np.array([s.U, s.J, s.hop["t"]], dtype=float)

    def problem(self, theta):
        U, J, t = (float(x) for x in theta)
        s = self.base.spec
        return synth.perturbed_problem(self.base, dU=U - s.U, dJ=J - s.J, dt=t - s.hop["t"])

    def tangents(self, theta, i):
        return synth.tangent_inputs(self.problem(theta), self.names[i])


def _omegas(prob):
    s = prob.spec
    return range(-s.iwb, s.iwb + 1)


def run_with_tangents(prob, tangent_inputs: Sequence, precision: str = "fp64"):
    """The full ladder of ``prob`` with the given input tangents (a list of
    (dhk, du, du_tilde, dvertex) per direction, any length: passes of up to
    four).  Returns (assembled outputs, [assembled tangent outputs per
    direction])."""
    fwd, tans = None, []
    dirs = list(tangent_inputs)
    passes = [dirs[i:i + MAX_DIRECTIONS] for i in range(0, len(dirs), MAX_DIRECTIONS)] or [[]]
    with Ladder.from_problem(prob) as lad:
        for iwb in _omegas(prob):
            lad.set_vertex(iwb, *prob.vertex(iwb))
        for chunk in passes:
            lad.clear_tangents()
            lad.reset_outputs()
            for d, (dhk, du, dut, dvertex) in enumerate(chunk):
                lad.set_tangent(dhk, du, dut, direction=d)
                if dvertex is not None:
                    for iwb in _omegas(prob):
                        lad.set_vertex_tangent(iwb, *dvertex(iwb), direction=d)
            if chunk:
                lad.ladder_run_tangent(precision=precision)
            else:
                lad.ladder_run(1, None, precision)
            if fwd is None:
                fwd = lad.assemble(lad.get_outputs(), prob.siw)
            tans += [lad.assemble_tangent(lad.get_tangent_outputs(d)) for d in range(len(chunk))]
    return fwd, tans


class _ModelFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, model, pick, want_tangents, precision):
        th = theta.detach().cpu().numpy().astype(float)
        prob = model.problem(th)
        tin = [model.tangents(th, i) for i in range(len(th))] if want_tangents else []
        fwd, tans = run_with_tangents(prob, tin, precision)
        ctx.tans = [pick(t, prob) for t in tans]
        return tuple(torch.from_numpy(x) for x in pick(fwd, prob))

    @staticmethod
    def backward(ctx, *grads):
        out = []
        for tan in ctx.tans:
            v = torch.zeros((), dtype=torch.float64)
            for g, dy in zip(grads, tan):
                if g is not None:
                    v = v + (torch.conj(g) * torch.from_numpy(dy)).real.sum()
            out.append(v)
        return torch.stack(out), None, None, None, None


def _check(theta, precision):
    if theta.ndim != 1 or theta.dtype != torch.float64:
        raise ValueError("theta must be a 1-d float64 tensor")
    if precision not in ("fp64", "mixed"):
        raise ValueError("precision must be 'fp64' or 'mixed'")


def _all_outputs(o, prob):
    return (np.ascontiguousarray(o["chi_dens"]), np.ascontiguousarray(o["chi_magn"]),
            np.ascontiguousarray(o["sigma"]))


def ladder_outputs(theta: torch.Tensor, model, precision: str = "fp64"):
    """(chi_d (ndim2, ndim2, nqp*(2 iwb+1)), chi_m (same), Sigma (ndim, ndim, 2 iwf, nkp_eom)),
    complex128, differentiable in the float64 parameter vector theta of a
    caller model (``model.problem(theta)``, ``model.tangents(theta, i)``)."""
    _check(theta, precision)
    grad = torch.is_grad_enabled() and theta.requires_grad
    return _ModelFn.apply(theta, model, _all_outputs, grad, precision)


def _chi_m_omega0_sigma(o, prob):
    s = prob.spec
    w0 = s.iwb * s.nqp + np.arange(s.nqp)            # the points of omega = 0
    return np.ascontiguousarray(o["chi_magn"][:, :, w0]), np.ascontiguousarray(o["sigma"])


def ladder_chi_sigma(params: torch.Tensor, base, precision: str = "fp64"):
    """(chi_m(q, omega=0) (ndim2, ndim2, nqp), Sigma (ndim, ndim, 2 iwf, nkp)), complex128,
    differentiable in params = tensor([U, J, t], dtype=float64) of the synthetic
    model at the DMFT inputs of ``base``.  precision "fp64" (FP64 LU) or "mixed"
    (FP32 LU with FP64 refinement of the outputs and of their tangents,
    agreeing with FP64 to ~1e-12)."""
    if params.shape != (3,) or params.dtype != torch.float64:
        raise ValueError("params must be a float64 tensor [U, J, t]")
    _check(params, precision)
    grad = torch.is_grad_enabled() and params.requires_grad
    return _ModelFn.apply(params, SynthModel(base), _chi_m_omega0_sigma, grad, precision)
