"""The torch.autograd front end of the reverse-time stepper, host side (no GPU): with the oracle
standing in for the forward and the autograd checker for the B200 gradient, a loss composed of the
torch map from material parameters to coefficients and :func:`autograd.responses` gets, by torch's
chain rule, the gradient that :meth:`AdjointFit.chain` gives from the coefficients' gradient."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import adjoint_reference
from acoustic_spaces_b200 import autograd, fit
from oracle.oracle import OracleSolver


class _Stepper:
    def __init__(self, layout, precision="fp32"):
        self.layout, self.precision = dict(layout), precision

    def run(self, signal):
        return OracleSolver(self.layout, self.precision).run(signal)

    def gradient(self, signal, dloss_dy, segment=250):
        return adjoint_reference.gradient(self.layout, signal, dloss_dy)

    def close(self):
        pass


def test_responses_compose_with_the_material_map(monkeypatch):
    monkeypatch.setattr(autograd, "B200WaveSolver", _Stepper)
    monkeypatch.setattr(fit, "B200WaveSolver", _Stepper)
    problem = fit.patched_room(4, size=(2.4, 2.0, 1.4), cell=0.1, steps=300, precision="fp64")
    f, params = problem.fit, problem.start
    conductance = torch.tensor(params.conductance, requires_grad=True)
    corner = torch.tensor(params.corner_hz, requires_grad=True)
    coefs = f.coefficient_tensors(conductance, corner)
    y = autograd.responses(f.built.layout, f.signal, precision="fp64", **coefs)
    loss = torch.sum((y - torch.as_tensor(f.target)) ** 2)
    loss.backward()
    ours = np.concatenate([conductance.grad.numpy(), corner.grad.numpy()])
    lay = f.layout(params)
    reference = OracleSolver(lay, "fp64").run(f.signal)
    np.testing.assert_allclose(y.detach().numpy(), reference, rtol=0, atol=1e-13 * np.abs(reference).max())
    G = adjoint_reference.gradient(lay, f.signal, 2.0 * (reference - f.target))
    expected = f.chain(params, lay, G)
    np.testing.assert_allclose(ours, expected, rtol=1e-9, atol=1e-12 * np.abs(expected).max())


def test_responses_checks_the_coefficient_shapes():
    problem_layout = {"coef_b": np.zeros(3), "coef_inv": np.zeros(3), "branch_now": np.zeros(1),
                      "branch_before": np.zeros(1), "branch_gain": np.zeros(1)}  # fmt: skip
    with pytest.raises(ValueError, match="coef_inv"):
        autograd.responses(problem_layout, np.zeros(4), coef_b=torch.zeros(3), coef_inv=torch.zeros(2),
                           branch_now=torch.zeros(1), branch_before=torch.zeros(1), branch_gain=torch.zeros(1))  # fmt: skip
