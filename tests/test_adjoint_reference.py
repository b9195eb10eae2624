"""The autograd checker of the reverse-time stepper, pinned on the CPU (no GPU).

Its forward equals the FP64 oracle's, and its gradient equals central differences of the loss taken
with exactly symmetric float32 steps of the coefficients (a coefficient of the layout is a float32,
so a step is a whole number of units in the last place: c + d and c - d are then both exact, and
the central difference keeps no second-order term). The material fit's ``central_difference``
is checked the same way, with the oracle standing in for the B200 stepper.
"""

from __future__ import annotations

import numpy as np
import pytest
from conftest import load_golden

import adjoint_reference
from acoustic_spaces_b200 import fit
from oracle.oracle import OracleSolver

_FAMILIES = (("coef_b", "coef_b"), ("coef_inv", "coef_inv"), ("branch_now", "now"),
             ("branch_before", "before"), ("branch_gain", "gain"))  # fmt: skip


def _misfit(layout, signal, seed=0):
    rng = np.random.default_rng(seed)
    base = OracleSolver(layout, "fp64").run(signal)
    target = 0.8 * base + 0.01 * np.abs(base).max() * rng.standard_normal(base.shape)
    return base, target


_PLAIN_KINDS = ["resonant7", "drive7", "fitted_closed", "resonant19", "speed7", "speed19", "uniform099"]


@pytest.mark.parametrize("name", _PLAIN_KINDS)
def test_the_autograd_stepper_steps_as_the_oracle(name):
    layout, signal, _ = load_golden(name)
    ours = adjoint_reference.series(layout, signal[:200])
    oracle = OracleSolver(layout, "fp64").run(signal[:200])
    assert np.max(np.abs(ours - oracle)) <= 1e-12 * np.max(np.abs(oracle))


@pytest.mark.parametrize("name", ["resonant7", "drive7", "fitted_closed", "resonant19", "speed7", "speed19"])
def test_the_autograd_gradient_matches_symmetric_central_differences(name):
    layout, signal, _ = load_golden(name)
    signal = signal[:300]
    y, target = _misfit(layout, signal)
    grad = adjoint_reference.gradient(layout, signal, 2.0 * (y - target))
    rng = np.random.default_rng(1)
    branch = np.asarray(layout["state_branch"], np.int64)
    plus, minus = dict(layout), dict(layout)
    predicted = 0.0
    for name_, key in _FAMILIES:
        c0 = np.asarray(layout[name_], np.float32)
        unit = np.spacing(np.abs(c0)).astype(np.float64)
        d = np.round(1e-6 * c0.astype(np.float64) * rng.uniform(-1, 1, len(c0)) / unit) * unit
        plus[name_] = (c0.astype(np.float64) + d).astype(np.float32)
        minus[name_] = (c0.astype(np.float64) - d).astype(np.float32)
        assert np.array_equal(plus[name_].astype(np.float64) - c0, d)
        assert np.array_equal(c0 - minus[name_].astype(np.float64), d)
        predicted += float(np.sum(grad[key] * (d[branch] if name_.startswith("branch") else d)))
    loss = lambda lay: float(np.sum((OracleSolver(lay, "fp64").run(signal) - target) ** 2))  # noqa: E731
    measured = 0.5 * (loss(plus) - loss(minus))
    assert abs(predicted - measured) <= 1e-4 * abs(measured), (predicted, measured)


class _OracleStepper:
    """The oracle behind the B200 stepper's forward interface, for host-side tests."""

    def __init__(self, layout, precision="fp32"):
        self._solver = OracleSolver(layout, precision)

    def run(self, signal):
        return self._solver.run(signal)

    def close(self):
        pass


def test_central_difference_of_the_material_parameters(monkeypatch):
    monkeypatch.setattr(fit, "B200WaveSolver", _OracleStepper)
    problem = fit.patched_room(1, size=(3.0, 2.4, 1.6), cell=0.1, steps=400, precision="fp64", segment=100)
    f, params = problem.fit, problem.start
    lay = f.layout(params)
    y = OracleSolver(lay, "fp64").run(f.signal)
    G = adjoint_reference.gradient(lay, f.signal, 2.0 * (y - f.target))
    for index in (0, 3, 9, 14):  # conductances and corner frequencies of several materials
        predicted, measured = f.central_difference(params, index, G)
        assert abs(predicted - measured) <= 1e-4 * abs(measured), (index, predicted, measured)
    # the chain rule: dL/dparameter = G . (the coefficients' tangent), the tangent in float64
    grad = f.chain(params, lay, G)
    v = params.vector()
    branch = np.asarray(lay["state_branch"], np.int64)
    B = f.sens["boundary_rows"]
    for index in range(len(v)):
        h = 1e-6 * v[index]
        up, down = v.copy(), v.copy()
        up[index] += h
        down[index] -= h
        cu = f.coefficients(fit.Relaxation.from_vector(params.beta, up))
        cd = f.coefficients(fit.Relaxation.from_vector(params.beta, down))
        tangent = 0.0
        for name, key in _FAMILIES:
            t = (cu[name] - cd[name]) / (2 * h)
            tangent += float(np.sum(G[key][:B] * t) if name.startswith("coef") else np.sum(G[key] * t[branch]))
        assert abs(grad[index] - tangent) <= 1e-5 * np.max(np.abs(grad)), (index, grad[index], tangent)


# ---- the matched layer's parameters --------------------------------------------------------------

_TABLES = adjoint_reference.KEEP + adjoint_reference.PUSH


@pytest.mark.parametrize("name", ["open_layer", "fitted_open", "open_layer_speed"])
def test_the_autograd_stepper_steps_a_matched_layer_as_the_oracle(name):
    layout, signal, _ = load_golden(name)
    ours = adjoint_reference.series(layout, signal[:200])
    oracle = OracleSolver(layout, "fp64").run(signal[:200])
    assert np.max(np.abs(ours - oracle)) <= 1e-12 * np.max(np.abs(oracle))


@pytest.mark.parametrize("name", ["open_layer", "open_layer_speed"])
def test_the_layer_tables_gradient_matches_symmetric_central_differences(name):
    # Every entry of the twelve tables stepped by a whole number of float32 units at once: the
    # directional derivative from the gradient against the loss's central difference.
    layout, signal, _ = load_golden(name)
    signal = signal[:150]
    y, target = _misfit(layout, signal)
    grad = adjoint_reference.gradient(layout, signal, 2.0 * (y - target))
    rng = np.random.default_rng(2)
    plus, minus, predicted = dict(layout), dict(layout), 0.0
    for name in _TABLES:
        c0 = np.asarray(layout[name], np.float32)
        unit = np.spacing(np.abs(c0)).astype(np.float64)
        d = np.round(1e-5 * np.abs(c0.astype(np.float64)) * rng.uniform(-1, 1, len(c0)) / unit) * unit
        plus[name] = (c0.astype(np.float64) + d).astype(np.float32)
        minus[name] = (c0.astype(np.float64) - d).astype(np.float32)
        assert np.array_equal(plus[name].astype(np.float64) - c0, d)
        predicted += float(np.sum(grad[name] * d))
    loss = lambda lay: float(np.sum((OracleSolver(lay, "fp64").run(signal) - target) ** 2))  # noqa: E731
    measured = 0.5 * (loss(plus) - loss(minus))
    assert abs(measured) > 0.0
    assert abs(predicted - measured) <= 1e-4 * abs(measured), (predicted, measured)


def test_the_layer_damping_gradient_by_the_chain_rule():
    # dL/d(layer damping) = the tables' gradient times their tangent in the damping
    # (layouts.layer_tables_tangent), against a central difference of the loss in the damping with
    # the room laid out again at damping -+ h: a 4 x 3 x 2.4 m convex room at 10 cm, open through
    # one face into a 4-cell matched layer.
    from acoustic_spaces_b200 import layouts as L

    cell, box, layer, damping = 0.1, (4.0, 3.0, 2.4), 4, 0.5
    rng = np.random.default_rng(3)
    rate = 343.0 / (L.COURANT * cell)
    room = L.convex_room(rng, box, faces=14, margin=cell * (layer + 3), open_face=1,
                         material=lambda r: L.Material(float(r.uniform(0.02, 0.1))))  # fmt: skip
    points = L.inside_points(rng, room, box, 5, 0.35, apart=0.35)
    grid = L.Grid(-L.OFFSET * cell, cell, tuple(int(round(b / cell)) for b in box))
    signal = L.gaussian_drive(rate, 150)

    def built(value):
        return L.cell_face_layout(room, grid, points[0], points[1:], layer=layer, layer_damping=value).layout

    lay = built(damping)
    y, target = _misfit(lay, signal)
    grad = adjoint_reference.gradient(lay, signal, 2.0 * (y - target))
    courant = float(np.sqrt(np.float64(np.asarray(lay["weights"], np.float32)[0])))
    predicted = 0.0
    for a, axis in enumerate("xyz"):
        t = L.layer_tables_tangent(int(grid.shape[a]), layer, damping, courant)
        for table, kind in ((f"keep_{axis}", "keep"), (f"push_{axis}", "push"), (f"keep_face_{axis}", "keep_face"),
                            (f"push_face_{axis}", "push_face")):  # fmt: skip
            predicted += float(np.sum(grad[table] * t[kind]))
    h = 0.01 * damping
    loss = lambda value: float(np.sum((OracleSolver(built(value), "fp64").run(signal) - target) ** 2))  # noqa: E731
    measured = (loss(damping + h) - loss(damping - h)) / (2.0 * h)
    assert abs(measured) > 0.0
    assert abs(predicted - measured) <= 2e-3 * abs(measured), (predicted, measured)


def test_the_layer_reverse_step_formulas():
    # The reverse step of one matched-layer update, as the GPU adjoint of the layer is to form it
    # (per axis: Q += P; H~ = H - p Q, L~ = L + p Q; the old q takes k Q, the old faces kf H~ and
    # kf L~; the pressures b_(i+s), b_(i-s), b_i take -pf H~, pf L~, pf H~ - pf L~; the tables
    # dk += Q q, dp -= Q (hi' - lo'), dkf += H~ hi, dpf -= H~ (b_(i+s) - b_i), and the same for the
    # - face), against autograd's vector-Jacobian product through the forward update.
    import torch

    rng = np.random.default_rng(4)
    n = 50  # cells along each axis of one line, the layer's cells at 1 .. n-2
    cells = np.arange(1, n - 1)
    tabs = {k: torch.tensor(rng.uniform(0.2, 1.0, n + 1), dtype=torch.float64, requires_grad=True)
            for k in ("k", "p", "kf", "pf")}  # fmt: skip
    b = torch.tensor(rng.standard_normal(n), dtype=torch.float64, requires_grad=True)
    lo, hi, q = (torch.tensor(rng.standard_normal(len(cells)), dtype=torch.float64, requires_grad=True) for _ in range(3))
    x = torch.as_tensor(cells)
    lo1 = tabs["kf"][x] * lo - tabs["pf"][x] * (b[x] - b[x - 1])
    hi1 = tabs["kf"][x + 1] * hi - tabs["pf"][x + 1] * (b[x + 1] - b[x])
    q1 = tabs["k"][x] * q - tabs["p"][x] * (hi1 - lo1)
    P, L, H, Q = (rng.standard_normal(len(cells)) for _ in range(4))  # adjoints of p', lo', hi', q'
    (q1 * torch.as_tensor(P + Q) + lo1 * torch.as_tensor(L) + hi1 * torch.as_tensor(H)).sum().backward()
    # the formulas, in numpy
    k, p, kf, pf = (tabs[name].detach().numpy() for name in ("k", "p", "kf", "pf"))
    bn, lon, hin, qn = (v.detach().numpy() for v in (b, lo, hi, q))
    lo1n, hi1n = lo1.detach().numpy(), hi1.detach().numpy()
    Qt = Q + P
    Ht = H - p[cells] * Qt
    Lt = L + p[cells] * Qt
    gb = np.zeros(n)
    np.add.at(gb, cells + 1, -pf[cells + 1] * Ht)
    np.add.at(gb, cells - 1, pf[cells] * Lt)
    np.add.at(gb, cells, pf[cells + 1] * Ht - pf[cells] * Lt)
    gk, gp, gkf, gpf = (np.zeros(n + 1) for _ in range(4))
    np.add.at(gk, cells, Qt * qn)
    np.add.at(gp, cells, -Qt * (hi1n - lo1n))
    np.add.at(gkf, cells + 1, Ht * hin)
    np.add.at(gpf, cells + 1, -Ht * (bn[cells + 1] - bn[cells]))
    np.add.at(gkf, cells, Lt * lon)
    np.add.at(gpf, cells, -Lt * (bn[cells] - bn[cells - 1]))
    close = lambda a, b_: np.testing.assert_allclose(a, b_, rtol=1e-12, atol=1e-12)  # noqa: E731
    close(q.grad.numpy(), k[cells] * Qt)
    close(hi.grad.numpy(), kf[cells + 1] * Ht)
    close(lo.grad.numpy(), kf[cells] * Lt)
    close(b.grad.numpy(), gb)
    for name, g in (("k", gk), ("p", gp), ("kf", gkf), ("pf", gpf)):
        close(tabs[name].grad.numpy(), g)


@pytest.mark.parametrize("stencil", [7, 19])
def test_a_speed_fields_reverse_step_is_its_forward_sweep_on_scaled_adjoints(stencil):
    # With a speed field the interior update is u' = (2 - t s_i) u_i + s_i (a sum_faces u_j + d
    # sum_edges u_j) - u-: each row scaled by its own cell's factor s_i, so the operator is no
    # longer symmetric, and its transpose takes s_j of every reader j. Carried as v = s lam, the
    # adjoint of the pressure times its cell's factor, the reverse step is then the forward sweep
    # itself: v_i = (2 - t s_i) V_i + s_i (a sum V_j + d sum V_j) - v+_i with V = s Lam, the
    # adjoints of the level after. So the GPU adjoint of a speed field can step v with the forward
    # scaled kernel. Checked against autograd's vector-Jacobian product through one update, on an
    # 8^3 box of interior cells inside a solid border.
    import itertools

    import torch

    rng = np.random.default_rng(5)
    n = 10
    interior = np.zeros((n, n, n), bool)
    interior[1:-1, 1:-1, 1:-1] = True
    a, d = (0.25, 0.125) if stencil == 19 else (1.0 / 3.0, 0.0)
    t = 6 * a + 12 * d
    scale = np.where(interior, rng.uniform(0.5, 1.0, (n, n, n)), 0.0)
    faces = [o for o in itertools.product((-1, 0, 1), repeat=3) if sum(map(abs, o)) == 1]
    edges = [o for o in itertools.product((-1, 0, 1), repeat=3) if sum(map(abs, o)) == 2]

    def neighbours(field, offsets):
        # the sum over the offsets, a cell outside the interior holding 0 (solid)
        field = np.where(interior, field, 0.0) if isinstance(field, np.ndarray) else field * torch.as_tensor(interior)
        roll = np.roll if isinstance(field, np.ndarray) else (lambda f, o, axis: torch.roll(f, o, axis))
        return sum(roll(field, tuple(-np.asarray(o)), (0, 1, 2)) for o in offsets)

    def update(u, s):
        return (2.0 - t * s) * u + s * (a * neighbours(u, faces) + d * neighbours(u, edges))

    u = torch.tensor(rng.standard_normal((n, n, n)) * interior, dtype=torch.float64, requires_grad=True)
    s = torch.as_tensor(scale)
    Lam = rng.standard_normal((n, n, n)) * interior  # the adjoints of the level after
    (update(u, s) * torch.as_tensor(interior) * torch.as_tensor(Lam)).sum().backward()
    lam = u.grad.numpy() * interior
    v = scale * lam
    swept = update(scale * Lam, scale) * interior
    np.testing.assert_allclose(v, swept, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize(
    "name", ["resonant7", "drive7", "fitted_closed", "speed19", "uniform099", "open_layer", "fitted_open",
             "open_layer_speed"],
)  # fmt: skip
def test_the_adjoint_decomposition_gives_the_autograd_gradient(name):
    # The CUDA adjoint's decomposition by kind of cell (tests/adjoint_decomposition.py: the sweep,
    # corrected cells, special rows, and the matched layer's part to come) against autograd, which
    # differentiates the forward scheme whole.
    import adjoint_decomposition

    layout, signal, _ = load_golden(name)
    signal = signal[:150]
    y, target = _misfit(layout, signal)
    ours = adjoint_decomposition.gradient(layout, signal, 2.0 * (y - target))
    checker = adjoint_reference.gradient(layout, signal, 2.0 * (y - target))
    for key, value in ours.items():
        scale = np.abs(checker[key]).max() if checker[key].size else 0.0
        np.testing.assert_allclose(value, checker[key], rtol=0, atol=1e-12 * scale, err_msg=key)


@pytest.mark.parametrize("name", ["fitted_open", "open_layer_speed"])
def test_the_adjoint_decomposition_gives_the_layer_tables_gradient(name):
    # The twelve tables' gradient from the layer's adjoints of each step's new states and the
    # states before and after it, against autograd (with a speed field, each cell's push scaled).
    import adjoint_decomposition

    layout, signal, _ = load_golden(name)
    signal = signal[:60]
    y, target = _misfit(layout, signal)
    ours = adjoint_decomposition.gradient(layout, signal, 2.0 * (y - target), tables=True)
    checker = adjoint_reference.gradient(layout, signal, 2.0 * (y - target))
    assert set(_TABLES) <= set(ours)
    for key in _TABLES:
        scale = np.abs(checker[key]).max()
        np.testing.assert_allclose(ours[key], checker[key], rtol=0, atol=1e-12 * scale, err_msg=key)
