"""The reverse-time stepper's gradient against the autograd checker (needs a B200).

L = sum over probes and steps of (y - t)^2 for a target t; dL/dy = 2 (y - t). The B200 adjoint
gives dL/d of every special row's coef_b, coef_inv and every branch state's now, before, gain.
The checker differentiates a float64 torch restatement of the forward step by autograd
(tests/adjoint_reference.py, itself pinned against the oracle and against exactly symmetric
central differences on the CPU). FP64 on the B200 must equal it to 1e-9 of each array's largest
value; FP32 must match its directional derivative along a random direction to 1e-3.
"""

from __future__ import annotations

import numpy as np
import pytest
from conftest import load_golden

import adjoint_reference
from acoustic_spaces_b200 import B200WaveSolver, fit, layouts

pytestmark = pytest.mark.gpu

_FAMILIES = (("coef_b", "coef_b"), ("coef_inv", "coef_inv"), ("branch_now", "now"),
             ("branch_before", "before"), ("branch_gain", "gain"))  # fmt: skip


def _problem(layout, signal, seed=0):
    rng = np.random.default_rng(seed)
    base = B200WaveSolver(layout, precision="fp64").run(signal)
    target = 0.8 * base + 0.01 * np.abs(base).max() * rng.standard_normal(base.shape)
    return target, adjoint_reference.gradient(layout, signal, 2.0 * (base - target))


def _gradient(layout, signal, target, precision, segment=0):
    solver = B200WaveSolver(layout, precision=precision)
    y = solver.run(signal)
    solver.reset()
    return solver.gradient(signal, 2.0 * (y - target), segment=segment)


def _directional(grad, layout, seed=1):
    rng = np.random.default_rng(seed)
    branch = np.asarray(layout["state_branch"], np.int64)
    total = 0.0
    for name, key in _FAMILIES:
        coef = np.asarray(layout[name], np.float64)
        delta = coef * rng.uniform(-1.0, 1.0, len(coef))
        total += float(np.sum(grad[key] * (delta[branch] if name.startswith("branch") else delta)))
    return total


def _assert_equal_gradients(ours, checker, rtol):
    for key in ("coef_b", "coef_inv", "now", "before", "gain"):
        scale = np.max(np.abs(checker[key])) if checker[key].size else 0.0
        np.testing.assert_allclose(ours[key], checker[key], rtol=0, atol=rtol * scale, err_msg=key)


# (the grids with a speed field or the 19-point stencil: tests/test_wide_and_scaled_gradient.py)
_GRIDS = ["resonant7", "drive7", "fitted_closed"]


@pytest.mark.parametrize("name", _GRIDS)
def test_fp64_gradient_is_the_autograd_gradient(name):
    layout, signal, _ = load_golden(name)
    signal = signal[:300]
    target, checker = _problem(layout, signal)
    _assert_equal_gradients(_gradient(layout, signal, target, "fp64"), checker, 1e-9)


@pytest.mark.parametrize("name", _GRIDS)
def test_fp32_gradient_matches_the_autograd_gradient(name):
    layout, signal, _ = load_golden(name)
    signal = signal[:300]
    target, checker = _problem(layout, signal)
    ours = _gradient(layout, signal, target, "fp32")
    predicted, exact = _directional(ours, layout), _directional(checker, layout)
    assert abs(predicted - exact) <= 1e-3 * abs(exact), (predicted, exact)


def test_checkpointed_segments_give_the_same_gradient():
    layout, signal, _ = load_golden("resonant7")
    signal = signal[:300]
    y = B200WaveSolver(layout, precision="fp64").run(signal)
    dloss = 2.0 * (y - 0.5 * y)
    whole = B200WaveSolver(layout, precision="fp64").gradient(signal, dloss, segment=0)
    pieces = B200WaveSolver(layout, precision="fp64").gradient(signal, dloss, segment=37)
    for key in whole:
        np.testing.assert_allclose(pieces[key], whole[key], rtol=1e-10, atol=1e-14 * np.abs(whole[key]).max())


# (grids with a matched layer: tests/test_layer_gradient.py)


def test_gradient_of_a_builder_room_is_the_autograd_gradient():
    b = layouts.batched_rooms(5, rooms=1, sources=1, cell=0.1, dims=(2.0, 3.0), steps=250)
    target, checker = _problem(b.layouts[0], b.signal)
    _assert_equal_gradients(_gradient(b.layouts[0], b.signal, target, "fp64", segment=60), checker, 1e-9)


# ---- material parameters: the adjoint fit --------------------------------------------------------


def test_material_gradient_matches_the_checker_and_central_differences():
    # A patched room (8 materials, a relaxation branch each: 16 parameters), misfit to its responses
    # at other parameters. The B200 gradient with respect to the coefficients equals the checker's;
    # along every parameter's tangent it matches central differences of L with exactly symmetric
    # float32 steps (relative step 1e-4) to 1e-4.
    problem = fit.patched_room(1, size=(3.0, 2.4, 1.6), cell=0.1, steps=600, precision="fp64", segment=100)
    f, params = problem.fit, problem.start
    _, grad, G = f.loss_and_gradient(params, "fp64", coefficients=True)
    lay = f.layout(params)
    y = B200WaveSolver(lay, precision="fp64").run(f.signal)
    checker = adjoint_reference.gradient(lay, f.signal, 2.0 * (y - f.target))
    _assert_equal_gradients(G, checker, 1e-9)
    np.testing.assert_allclose(grad, f.chain(params, lay, checker), rtol=1e-9, atol=1e-12 * np.abs(grad).max())
    for index in range(len(params.vector())):
        predicted, measured = f.central_difference(params, index, G)
        assert abs(predicted - measured) <= 1e-4 * abs(measured), (index, predicted, measured)


def test_fp32_material_gradient_is_the_fp64_one():
    problem = fit.patched_room(2, size=(3.0, 2.4, 1.6), cell=0.1, steps=600, segment=100)
    _, g32 = problem.fit.loss_and_gradient(problem.start, "fp32")
    _, g64 = problem.fit.loss_and_gradient(problem.start, "fp64")
    assert np.max(np.abs(g32 - g64)) <= 1e-3 * np.max(np.abs(g64))


def test_adam_recovers_the_parameters():
    # 8 patch materials (16 parameters) from +-30 %, to 1 %: 64 iterations when measured.
    problem = fit.patched_room(3, size=(3.0, 2.4, 1.6), cell=0.1, steps=800, segment=200)
    result = fit.adam(problem, iterations=400, rate=0.05)
    assert result["converged"], result["worst_relative_error"]


def test_lbfgs_recovers_the_parameters():
    problem = fit.patched_room(3, size=(3.0, 2.4, 1.6), cell=0.1, steps=800, segment=200)
    result = fit.lbfgs(problem, iterations=150)
    assert result["converged"], result["worst_relative_error"]


def test_the_autograd_function_gives_the_material_gradient():
    # The torch map from parameters to coefficients composed with autograd.responses: torch's chain
    # rule through the B200 reverse-time stepper equals AdjointFit's gradient.
    import torch

    from acoustic_spaces_b200 import autograd

    problem = fit.patched_room(5, size=(3.0, 2.4, 1.6), cell=0.1, steps=500, precision="fp64", segment=100)
    f, params = problem.fit, problem.start
    conductance = torch.tensor(params.conductance, requires_grad=True)
    corner = torch.tensor(params.corner_hz, requires_grad=True)
    y = autograd.responses(f.built.layout, f.signal, precision="fp64", segment=100,
                           **f.coefficient_tensors(conductance, corner))  # fmt: skip
    loss = torch.sum((y - torch.as_tensor(f.target)) ** 2)
    loss.backward()
    ours = np.concatenate([conductance.grad.numpy(), corner.grad.numpy()])
    expected_loss, expected = f.loss_and_gradient(params, "fp64")
    assert abs(float(loss.detach()) - expected_loss) <= 1e-12 * expected_loss
    np.testing.assert_allclose(ours, expected, rtol=1e-9, atol=1e-12 * np.abs(expected).max())


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("budget", [None, 0], ids=["trajectory", "checkpoints"])
def test_a_taped_run_gives_the_gradient_to_the_bit(budget, precision):
    # fdtd_set_tape: the run keeps the special rows' whole trajectory (within the budget; the
    # gradient then recomputes nothing) or its checkpoints (the gradient recomputes each segment
    # from them); either way the gradient equals an untaped one's to the bit, and a gradient of
    # another drive does not use the tape.
    layout, signal, _ = load_golden("resonant7")
    signal = np.ascontiguousarray(signal[:300])
    y = B200WaveSolver(layout, precision=precision).run(signal)
    dloss = 2.0 * (y - 0.5 * y)
    plain = B200WaveSolver(layout, precision=precision).gradient(signal, dloss, segment=37)
    taped = B200WaveSolver(layout, precision=precision)
    taped.set_tape_budget(budget)
    taped.set_tape(37)
    np.testing.assert_array_equal(taped.run(signal), y)
    taped.reset()
    got = taped.gradient(signal, dloss, segment=37)
    for key in plain:
        np.testing.assert_array_equal(got[key], plain[key], err_msg=key)
    other = signal * 0.5
    y2 = B200WaveSolver(layout, precision=precision).run(other)
    expected = B200WaveSolver(layout, precision=precision).gradient(other, 2.0 * y2, segment=37)
    got = taped.gradient(other, 2.0 * y2, segment=37)
    for key in expected:
        np.testing.assert_array_equal(got[key], expected[key], err_msg=key)


def test_new_coefficients_step_and_differentiate_as_a_new_solver():
    # fdtd_set_coefficients after a gradient (the adjoint's tables set up): the run and the
    # gradient equal those of a solver built with the new coefficients, to the bit.
    problem = fit.patched_room(1, size=(3.0, 2.4, 1.6), cell=0.1, steps=300, precision="fp64", segment=100)
    f = problem.fit
    first, second = f.layout(problem.start), f.layout(problem.truth)
    kept = B200WaveSolver(first, precision="fp64")
    y = kept.run(f.signal)
    kept.reset()
    kept.gradient(f.signal, 2.0 * y, segment=100)
    kept.set_coefficients(*(second[k] for k in ("coef_b", "coef_inv", "branch_now", "branch_before", "branch_gain")))
    fresh = B200WaveSolver(second, precision="fp64")
    y2 = fresh.run(f.signal)
    np.testing.assert_array_equal(kept.run(f.signal), y2)
    kept.reset()
    fresh.reset()
    got = kept.gradient(f.signal, 2.0 * y2, segment=100)
    expected = fresh.gradient(f.signal, 2.0 * y2, segment=100)
    for key in expected:
        np.testing.assert_array_equal(got[key], expected[key], err_msg=key)
