"""Gradients of the ladder outputs with respect to model parameters.

``ladder_chi_sigma(params, base)`` returns chi_m(q, omega = 0) and the DGA
self-energy Sigma(k, nu) of the FP64 GPU ladder as complex torch tensors and
is differentiable in ``params = (U, J, t)``: the Kanamori couplings (V = U - 2J)
and the hopping scale t of the synthetic model, at the DMFT one-particle
inputs of ``base`` (siw, giw, mu held fixed).

The forward pass runs the ladder (FP64 or mixed precision) once with the three tangent directions of
(U, J, t) (``adga_ladder_run_tangent``: the hand-written forward-mode
derivative of every stage, d(A^-1) = -A^-1 dA A^-1 through the BSE with the
forward LU factors, and the tangent chi0 and EOM contractions); the backward
pass only contracts the incoming gradients with those tangents.  PyTorch's
convention for a real input theta and complex outputs y is
theta_bar = Re sum conj(y_bar) dy/dtheta.

The model's input tangents (dH/dt, du/dU, du/dJ and dchi_loc = -chi_loc
dGamma chi_loc) come from ``synth.tangent_inputs``; a caller with its own
model supplies them the same way through ``Ladder.set_tangent`` /
``Ladder.set_vertex_tangent``.
"""
from __future__ import annotations

import numpy as np
import torch

from . import synth
from .ladder import Ladder


def _run(prob, tangents: bool, precision: str):
    s = prob.spec
    with Ladder.from_problem(prob) as lad:
        for iwb in range(-s.iwb, s.iwb + 1):
            lad.set_vertex(iwb, *prob.vertex(iwb))
        if tangents:
            for d, par in enumerate(synth.PARAMS):
                dhk, du, dut, dvertex = synth.tangent_inputs(prob, par)
                lad.set_tangent(dhk, du, dut, direction=d)
                if dvertex is not None:
                    for iwb in range(-s.iwb, s.iwb + 1):
                        lad.set_vertex_tangent(iwb, *dvertex(iwb), direction=d)
            lad.ladder_run_tangent(precision=precision)
        else:
            lad.ladder_run(1, None, precision)
        fwd = lad.assemble(lad.get_outputs(), prob.siw)
        tans = [lad.assemble_tangent(lad.get_tangent_outputs(d)) for d in range(len(synth.PARAMS))] \
            if tangents else []
    w0 = s.iwb * s.nqp + np.arange(s.nqp)            # the points of omega = 0
    pick = lambda o: (np.ascontiguousarray(o["chi_magn"][:, :, w0]), np.ascontiguousarray(o["sigma"]))
    return pick(fwd), [pick(t) for t in tans]


class _LadderFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, base, tangents, precision):
        U, J, t = (float(x) for x in params.detach().cpu().numpy())
        s = base.spec
        prob = synth.perturbed_problem(base, dU=U - s.U, dJ=J - s.J, dt=t - s.hop["t"])
        (chi_m, sig), tans = _run(prob, tangents, precision)
        ctx.tans = tans
        return torch.from_numpy(chi_m), torch.from_numpy(sig)

    @staticmethod
    def backward(ctx, g_chi, g_sig):
        out = []
        for dchi, dsig in ctx.tans:
            v = torch.zeros((), dtype=torch.float64)
            if g_chi is not None:
                v = v + (torch.conj(g_chi) * torch.from_numpy(dchi)).real.sum()
            if g_sig is not None:
                v = v + (torch.conj(g_sig) * torch.from_numpy(dsig)).real.sum()
            out.append(v)
        return torch.stack(out), None, None, None


def ladder_chi_sigma(params: torch.Tensor, base, precision: str = "fp64"):
    """(chi_m(q, omega=0) (ndim2, ndim2, nqp), Sigma (ndim, ndim, 2 iwf, nkp)), complex128,
    differentiable in params = tensor([U, J, t], dtype=float64).  precision "fp64"
    (FP64 LU) or "mixed" (FP32 LU with FP64 refinement of the outputs and of
    their tangents, agreeing with FP64 to ~1e-12)."""
    if params.shape != (3,) or params.dtype != torch.float64:
        raise ValueError("params must be a float64 tensor [U, J, t]")
    if precision not in ("fp64", "mixed"):
        raise ValueError("precision must be 'fp64' or 'mixed'")
    return _LadderFn.apply(params, base, torch.is_grad_enabled() and params.requires_grad, precision)
