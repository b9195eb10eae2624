"""The adjoint fit's host side: coefficients rebuilt from material parameters, and the chain rule
from the coefficients' gradient to the parameters, against finite differences of a loss defined
directly on the coefficients (no GPU)."""

from __future__ import annotations

import math

import numpy as np
import pytest

from acoustic_spaces_b200 import fit, layouts
from oracle.oracle import OracleSolver


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


def test_the_fit_room_is_laid_out_as_the_reference_lays_it(monkeypatch):
    # The adjoint fit's room (a box, the floor and the ceiling each cut in two patches, 8 materials
    # of one relaxation branch each) handed to the reference as triangles with a material each: the
    # reference's own layout, array for array, and its run equal to the oracle's to the bit.
    from oracle.oracle import reference_native

    native = reference_native()
    if native is None:
        pytest.skip("the reference sources are not here")

    class _Oracle:
        def __init__(self, layout, precision="fp32"):
            self._solver = OracleSolver(layout, precision)

        def run(self, signal):
            return self._solver.run(signal)

        def close(self):
            pass

    monkeypatch.setattr(fit, "B200WaveSolver", _Oracle)
    X, Y, Z = 3.0, 2.4, 1.6
    problem = fit.patched_room(1, size=(X, Y, Z), cell=0.1, steps=150)
    sc = problem.scene
    xc, yc, order = sc["x_cut"], sc["y_cut"], sc["order"]

    def rect(normal, corners):  # corners ordered round their centroid, as layouts.room_mesh orders them
        pts = np.array(corners, float)
        c = pts.mean(0)
        e1 = (pts[0] - c) / np.linalg.norm(pts[0] - c)
        e2 = np.cross(normal, e1)
        return pts[np.argsort(np.arctan2((pts - c) @ e2, (pts - c) @ e1))]

    walls = [
        (rect([-1, 0, 0], [[0, 0, 0], [0, Y, 0], [0, Y, Z], [0, 0, Z]]), order[4]),
        (rect([1, 0, 0], [[X, 0, 0], [X, Y, 0], [X, Y, Z], [X, 0, Z]]), order[5]),
        (rect([0, -1, 0], [[0, 0, 0], [X, 0, 0], [X, 0, Z], [0, 0, Z]]), order[6]),
        (rect([0, 1, 0], [[0, Y, 0], [X, Y, 0], [X, Y, Z], [0, Y, Z]]), order[7]),
        (rect([0, 0, -1], [[0, 0, 0], [xc, 0, 0], [xc, Y, 0], [0, Y, 0]]), order[0]),
        (rect([0, 0, -1], [[xc, 0, 0], [X, 0, 0], [X, Y, 0], [xc, Y, 0]]), order[1]),
        (rect([0, 0, 1], [[0, 0, Z], [X, 0, Z], [X, yc, Z], [0, yc, Z]]), order[2]),
        (rect([0, 0, 1], [[0, yc, Z], [X, yc, Z], [X, Y, Z], [0, Y, Z]]), order[3]),
    ]
    vertices, triangles, owner = [], [], []
    for pts, material in walls:
        base = len(vertices)
        vertices.extend(pts)
        triangles += [(base, base + k, base + k + 1) for k in range(1, len(pts) - 1)]
        owner += [int(material)] * (len(pts) - 2)
    mats = sc["materials"]
    rows = [np.asarray(m.branches, float).reshape(-1, 3) for m in mats]
    grid = sc["grid"]
    solver = native.WaveSolver(
        native.Bvh(np.array(vertices), np.array(triangles, np.int64)), np.array(owner, np.int64),
        np.array([m.beta for m in mats]), np.ascontiguousarray(np.vstack(rows)),
        np.concatenate([np.full(len(r), k, np.int64) for k, r in enumerate(rows)]), grid.origin, grid.cell,
        *grid.shape, sc["source"], sc["receivers"], layer=0, layer_damping=0.0, threads=2,
    )  # fmt: skip
    ref, lay = solver.layout(), problem.fit.built.layout
    for name, value in lay.items():
        assert np.array_equal(np.asarray(value), np.asarray(ref[name])), name
    assert np.array_equal(solver.run(problem.fit.signal), OracleSolver(lay).run(problem.fit.signal))
