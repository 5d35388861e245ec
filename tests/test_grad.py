"""Gradients of chi_m(q, omega = 0) and Sigma(k, nu) in (U, J, t) through the
torch.autograd.Function of adga_b200.grad:
  * torch.autograd.gradcheck (central differences of the GPU FP64 ladder
    against the vector-Jacobian products of backward, every output),
  * the gradient of a scalar loss against central differences of the loss,
  * the vector-Jacobian product against the dense Jacobian of the FP64 oracle
    (central differences of every output of the small grid).
"""
import numpy as np
import pytest
import torch

from adga_b200 import synth
from adga_b200.grad import ladder_chi_sigma
from oracle import adga_oracle as O
from tests.helpers import problem, qw_points, rel_err, to_inputs

pytestmark = pytest.mark.gpu
H = 1e-5


def params_of(p, grad=True):
    s = p.spec
    return torch.tensor([s.U, s.J, s.hop["t"]], dtype=torch.float64, requires_grad=grad)


def test_gradcheck_chi_m_and_sigma():
    p = problem("t2")
    x = params_of(p)
    assert torch.autograd.gradcheck(lambda y: ladder_chi_sigma(y, p), (x,), eps=H, atol=1e-7, rtol=1e-5)


@pytest.mark.parametrize("name,precision", [("t2", "fp64"), ("t3", "fp64"), ("t2", "mixed"), ("t3", "mixed")])
def test_loss_gradient_matches_finite_differences(name, precision):
    """The mixed forward leaves a ~1e-12 relative refinement remainder, so its
    difference quotients carry ~1e-7 relative noise: 1e-5 for mixed."""
    p = problem(name)
    rng = np.random.default_rng(7)
    x = params_of(p)
    chi, sig = ladder_chi_sigma(x, p, precision)
    wc = torch.from_numpy(rng.standard_normal(chi.shape) + 1j * rng.standard_normal(chi.shape))
    ws = torch.from_numpy(rng.standard_normal(sig.shape) + 1j * rng.standard_normal(sig.shape))

    def loss(c, s):
        return (c.abs() ** 2).sum() + (wc * c).real.sum() + (ws * s).imag.sum() + (s.abs() ** 2).sum()

    loss(chi, sig).backward()
    want = []
    with torch.no_grad():
        for i in range(3):
            e = torch.zeros(3, dtype=torch.float64)
            e[i] = H
            lp = loss(*ladder_chi_sigma(x.detach() + e, p, precision))
            lm = loss(*ladder_chi_sigma(x.detach() - e, p, precision))
            want.append(float((lp - lm) / (2 * H)))
    got = x.grad.numpy()
    tol = 1e-6 if precision == "fp64" else 1e-5
    assert np.max(np.abs(got - want)) < tol * max(1.0, np.max(np.abs(want))), (got, want)


def oracle_chi_sigma(p):
    s = p.spec
    inp = to_inputs(p)
    out = O.Oracle(inp).run(qw_points(p, 1, s.nqp * (2 * s.iwb + 1)))
    out.update(O.assemble(inp, out))
    w0 = s.iwb * s.nqp + np.arange(s.nqp)
    return out["chi_magn"][:, :, w0], out["sigma"]


def test_vjp_matches_oracle_dense_jacobian():
    p = problem("t2")
    s = p.spec
    cols = []
    for kw in ("dU", "dJ", "dt"):                  # dense Jacobian, one column per parameter
        cp, sp = oracle_chi_sigma(synth.perturbed_problem(p, **{kw: H}))
        cm, sm = oracle_chi_sigma(synth.perturbed_problem(p, **{kw: -H}))
        cols.append(np.concatenate([((cp - cm) / (2 * H)).ravel(), ((sp - sm) / (2 * H)).ravel()]))
    jac = np.stack(cols, axis=1)                   # (outputs, 3), complex
    x = params_of(p)
    chi, sig = ladder_chi_sigma(x, p)
    rng = np.random.default_rng(3)
    for _ in range(3):
        vc = rng.standard_normal(chi.shape) + 1j * rng.standard_normal(chi.shape)
        vs = rng.standard_normal(sig.shape) + 1j * rng.standard_normal(sig.shape)
        g = torch.autograd.grad((chi, sig), x, (torch.from_numpy(vc), torch.from_numpy(vs)), retain_graph=True)[0]
        v = np.concatenate([vc.ravel(), vs.ravel()])
        want = np.real(np.conj(v) @ jac)
        assert rel_err(g.numpy(), want) < 1e-6, (g.numpy(), want)


class SplitModel:
    """A caller model: the synthetic couplings (U, J), the hopping scale t and
    on-site shifts d_a of the first orbitals (H_aa(k) += d_a).  Its input
    tangents: the synthetic model's for U, J, t; dH/dd_a = E_aa for the shifts."""

    def __init__(self, base, nshift):
        self.base, self.nshift = base, nshift

    def problem(self, theta):
        import dataclasses
        s = self.base.spec
        p = synth.perturbed_problem(self.base, dU=theta[0] - s.U, dJ=theta[1] - s.J, dt=theta[2] - s.hop["t"])
        hk = p.hk.copy(order="F")
        for a in range(self.nshift):
            hk[a, a, :] += theta[3 + a]
        return dataclasses.replace(p, hk=hk, _vcache={})

    def tangents(self, theta, i):
        if i < 3:
            return synth.tangent_inputs(self.problem(theta), synth.PARAMS[i])
        p = self.base
        dhk = np.zeros_like(p.hk, order="F")
        dhk[i - 3, i - 3, :] = 1.0
        return dhk, None, None, None


@pytest.mark.parametrize("nshift", [1, 2])
def test_caller_model_gradient_matches_finite_differences(nshift):
    """ladder_outputs with a caller's model and its own input tangents: 4 or 5
    parameters (the latter in two tangent passes), every output of the full
    grid in a scalar loss, against central differences of the loss."""
    from adga_b200.grad import ladder_outputs
    p = problem("t2")
    model = SplitModel(p, nshift)
    s = p.spec
    theta = torch.tensor([s.U, s.J, s.hop["t"]] + [0.01 * (a + 1) for a in range(nshift)],
                         dtype=torch.float64, requires_grad=True)
    rng = np.random.default_rng(3)
    chi_d, chi_m, sig = ladder_outputs(theta, model)
    w = [torch.from_numpy(rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape))
         for x in (chi_d, chi_m, sig)]

    def loss(*ys):
        return sum((wi * y).real.sum() + (y.abs() ** 2).sum() for wi, y in zip(w, ys))

    loss(chi_d, chi_m, sig).backward()
    want = []
    with torch.no_grad():
        for i in range(len(theta)):
            e = torch.zeros(len(theta), dtype=torch.float64)
            e[i] = H
            lp = loss(*ladder_outputs(theta.detach() + e, model))
            lm = loss(*ladder_outputs(theta.detach() - e, model))
            want.append(float((lp - lm) / (2 * H)))
    got = theta.grad.numpy()
    assert np.max(np.abs(got - want)) < 1e-6 * max(1.0, np.max(np.abs(want))), (got, want)
