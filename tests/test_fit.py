"""The adjoint fit's host side: coefficients rebuilt from material parameters, and the chain rule
from the coefficients' gradient to the parameters, against finite differences of a loss defined
directly on the coefficients (no GPU)."""

from __future__ import annotations

import math

import numpy as np

from acoustic_spaces_b200 import fit, layouts


def _small_problem():
    rng = np.random.default_rng(4)
    size = np.array([2.0, 1.6, 1.2])
    cell = 0.1
    rate = 343.0 / (layouts.COURANT * cell)
    m = 4
    truth = fit.Relaxation(np.full(m, 0.02), rng.uniform(0.05, 0.5, m), rng.uniform(50, 500, m))
    mats = [layouts.Material(0.02, fit.relaxation_branch(truth.conductance[k], truth.corner_hz[k], rate)) for k in range(m)]
    room = layouts.shoebox(size, [layouts.Material(0.0)] * 6)
    room.patches = lambda planes, points: np.asarray(planes) % m
    room.patch_materials = mats
    points = layouts.inside_points(rng, room, size, 3, 0.35, apart=0.4)
    built = layouts.cell_face_layout(room, layouts.room_grid(size, cell), points[0], points[1:], rate=rate)
    problem = fit.AdjointFit(built, np.zeros(10, np.float32), np.zeros((2, 10)), rate, truth.beta)
    return problem, truth, built


def test_coefficients_from_the_truth_equal_the_builders():
    problem, truth, built = _small_problem()
    lay = problem.layout(truth)
    for name in ("branch_now", "branch_before", "branch_gain"):
        assert np.array_equal(lay[name], built.layout[name]), name
    # g is summed in another order than the builder's: to a float's rounding
    np.testing.assert_allclose(lay["coef_b"], built.layout["coef_b"], rtol=2e-7)
    np.testing.assert_allclose(lay["coef_inv"], built.layout["coef_inv"], rtol=2e-7)


def test_the_chain_rule_matches_finite_differences():
    problem, truth, built = _small_problem()
    rng = np.random.default_rng(9)
    lay0 = problem.layout(truth)
    K, S = len(lay0["coef_b"]), len(lay0["state_branch"])
    weights = {"coef_b": rng.standard_normal(K), "coef_inv": rng.standard_normal(K), "now": rng.standard_normal(S),
               "before": rng.standard_normal(S), "gain": rng.standard_normal(S)}  # fmt: skip
    branch = np.asarray(lay0["state_branch"], np.int64)

    def synthetic(params):  # a linear loss of the coefficients, in double
        mrq = problem._branches(params)
        a = mrq[:, 0] + 0.5 * mrq[:, 1] + 0.5 * mrq[:, 2]
        g = problem._g(params, mrq)
        B = problem.sens["boundary_rows"]
        cb = 1.0 - g
        ci = 1.0 / (1.0 + g)
        now, before, gain = 2 * mrq[:, 0] / a, (2 * mrq[:, 0] + mrq[:, 2]) / a, 0.5 / a
        return (np.dot(weights["coef_b"][:B], cb) + np.dot(weights["coef_inv"][:B], ci)
                + np.dot(weights["now"], now[branch]) + np.dot(weights["before"], before[branch])
                + np.dot(weights["gain"], gain[branch]))  # fmt: skip

    grad = problem.chain(truth, lay0, weights)
    v = truth.vector()
    for i in range(len(v)):
        h = 1e-6 * v[i]
        up, down = v.copy(), v.copy()
        up[i] += h
        down[i] -= h
        fd = (synthetic(fit.Relaxation.from_vector(truth.beta, up)) - synthetic(fit.Relaxation.from_vector(truth.beta, down))) / (2 * h)
        assert math.isclose(grad[i], fd, rel_tol=1e-6, abs_tol=1e-9 * abs(fd) + 1e-12), (i, grad[i], fd)
