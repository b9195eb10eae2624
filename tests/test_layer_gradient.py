"""The reverse-time stepper through a matched layer against the autograd checker (needs a B200).

On grids with a matched layer the B200 gradient carries the layer's own adjoint (its split-field
states' adjoints, carried from step to step, and their terms on the pressures the states read)
and gives, beside the rows' and branch states' coefficients, dL/d of the layer's twelve tables
(keep and push of the centres and the faces per axis, fdtd.hpp:2219-2238). The checker steps the
layer as the reference does (each cell its own copy of both faces) in float64 torch and
differentiates it by autograd (tests/adjoint_reference.py, pinned on the CPU to the oracle and to
exactly symmetric central differences). FP64 must equal it to 1e-9 of each array's largest value;
FP32 its directional derivative to 1e-3. The damping's gradient, by the chain rule through the
tables, must match a central difference of the loss with the room laid out again.
"""

from __future__ import annotations

import numpy as np
import pytest
from conftest import load_golden

import adjoint_reference
from acoustic_spaces_b200 import B200WaveSolver
from acoustic_spaces_b200 import layouts as L
from oracle.oracle import OracleSolver

pytestmark = pytest.mark.gpu

_TABLES = adjoint_reference.KEEP + adjoint_reference.PUSH
_LAYER_GRIDS = ["open_layer", "fitted_open", "open_layer_speed"]


def _problem(layout, signal, seed=0):
    rng = np.random.default_rng(seed)
    base = B200WaveSolver(layout, precision="fp64").run(signal)
    target = 0.8 * base + 0.01 * np.abs(base).max() * rng.standard_normal(base.shape)
    return target, adjoint_reference.gradient(layout, signal, 2.0 * (base - target))


def _gradient(layout, signal, target, precision, segment=0, tape=0):
    solver = B200WaveSolver(layout, precision=precision)
    if tape:
        solver.set_tape(tape)
    y = solver.run(signal)
    if not tape:
        solver.reset()
    return solver.gradient(signal, 2.0 * (y - target), segment=segment)


def _keys(checker):
    return [k for k in ("coef_b", "coef_inv", "now", "before", "gain", *_TABLES) if k in checker]


@pytest.mark.parametrize("name", _LAYER_GRIDS)
def test_fp64_layer_gradient_is_the_autograd_gradient(name):
    layout, signal, _ = load_golden(name)
    signal = signal[:240]
    target, checker = _problem(layout, signal)
    ours = _gradient(layout, signal, target, "fp64")
    assert set(_TABLES) <= set(ours)
    for key in _keys(checker):
        scale = np.max(np.abs(checker[key])) if checker[key].size else 0.0
        np.testing.assert_allclose(ours[key], checker[key], rtol=0, atol=1e-9 * scale, err_msg=key)


@pytest.mark.parametrize("name", _LAYER_GRIDS)
def test_fp32_layer_gradient_matches_the_autograd_gradient(name):
    layout, signal, _ = load_golden(name)
    signal = signal[:240]
    target, checker = _problem(layout, signal)
    ours = _gradient(layout, signal, target, "fp32")
    rng = np.random.default_rng(7)
    predicted = exact = 0.0
    for key in _keys(checker):
        direction = rng.uniform(-1.0, 1.0, len(checker[key]))
        predicted += float(np.sum(ours[key] * direction))
        exact += float(np.sum(checker[key] * direction))
    assert abs(predicted - exact) <= 1e-3 * abs(exact), (predicted, exact)


def test_layer_gradient_in_segments_and_from_a_tape_is_one_segments():
    layout, signal, _ = load_golden("fitted_open")
    signal = signal[:200]
    target, _ = _problem(layout, signal)
    whole = _gradient(layout, signal, target, "fp64", segment=0)
    pieces = _gradient(layout, signal, target, "fp64", segment=37)
    taped = _gradient(layout, signal, target, "fp64", segment=37, tape=37)
    for key in whole:
        scale = np.abs(whole[key]).max() if whole[key].size else 0.0
        np.testing.assert_allclose(pieces[key], whole[key], rtol=1e-10, atol=1e-14 * scale, err_msg=key)
        np.testing.assert_array_equal(taped[key], pieces[key], err_msg=key)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_the_walls_gradient_without_the_tables_is_the_same(precision):
    # Without the tables no layer factor is recorded: the walls' gradient is the same to the bit,
    # and a second gradient with the tables gives them again, summed in the same fixed order.
    layout, signal, _ = load_golden("fitted_open")
    signal = signal[:150]
    target, _ = _problem(layout, signal)
    solver = B200WaveSolver(layout, precision=precision)
    y = solver.run(signal)
    solver.reset()
    dloss = 2.0 * (y - target)
    with_tables = solver.gradient(signal, dloss, segment=40)
    walls = solver.gradient(signal, dloss, segment=40, layer_tables=False)
    again = solver.gradient(signal, dloss, segment=40)
    assert set(walls) | set(_TABLES) == set(with_tables) and not set(walls) & set(_TABLES)
    for key in walls:
        np.testing.assert_array_equal(walls[key], with_tables[key], err_msg=key)
    for key in with_tables:
        np.testing.assert_array_equal(again[key], with_tables[key], err_msg=key)


def test_a_walls_only_tape_keeps_the_trajectory_and_gives_the_same_gradient():
    # Taped without the tables, a grid with a matched layer keeps the rows' trajectory (no
    # checkpoints, nothing recomputed); its walls' gradient equals the untaped one to the bit. A
    # gradient that asks for the tables after such a tape runs the forward pass again and gives
    # the untaped tables too.
    layout, signal, _ = load_golden("open_layer")
    signal = signal[:120]
    target, _ = _problem(layout, signal)
    solver = B200WaveSolver(layout, precision="fp64")
    y = solver.run(signal)
    solver.reset()
    dloss = 2.0 * (y - target)
    plain = solver.gradient(signal, dloss, segment=30, layer_tables=False)
    full = solver.gradient(signal, dloss, segment=30)
    solver.set_tape(30, layer_tables=False)
    solver.run(signal)
    taped = solver.gradient(signal, dloss, segment=30, layer_tables=False)
    for key in plain:
        np.testing.assert_array_equal(taped[key], plain[key], err_msg=key)
    solver.run(signal)
    retaped = solver.gradient(signal, dloss, segment=30)
    for key in full:
        np.testing.assert_array_equal(retaped[key], full[key], err_msg=key)


def test_the_layer_damping_gradient_on_the_gpu_matches_central_differences():
    # dL/d(layer damping) = the B200's tables' gradient times the tables' tangent in the damping
    # (layouts.layer_tables_tangent), against a central difference of the loss (the FP64 oracle)
    # with the room laid out again at damping -+ h: a 4 x 3 x 2.4 m convex room at 10 cm, open
    # through one face into a 4-cell matched layer.
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
    y = OracleSolver(lay, "fp64").run(signal)
    target = 0.7 * y
    solver = B200WaveSolver(lay, precision="fp64")
    grad = solver.gradient(signal, 2.0 * (y - target), segment=50)
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
    # the same along the damping's tangent on the device (fdtd_set_layer_tangent)
    solver.set_layer_tangent(L.damping_tangent(lay, layer, damping))
    along = solver.gradient(signal, 2.0 * (y - target), segment=50)["layer_tangent"]
    assert abs(along - predicted) <= 1e-9 * abs(predicted), (along, predicted)


def test_the_reverse_steps_launch_caps_leave_the_gradient_unchanged():
    # Bounded grids for the reverse step's rows launches (each block taking blocks' worth of rows
    # in turn) give the same gradient to the bit, tables included.
    layout, signal, _ = load_golden("fitted_open")
    signal = signal[:100]
    target, _ = _problem(layout, signal)
    solver = B200WaveSolver(layout, precision="fp32")
    y = solver.run(signal)
    solver.reset()
    dloss = 2.0 * (y - target)
    plain = solver.gradient(signal, dloss, segment=30)
    for far, near in [(1, 1), (2, 8), (4, 16)]:
        solver.set_adjoint_launch(far, near)
        capped = solver.gradient(signal, dloss, segment=30)
        for key in plain:
            np.testing.assert_array_equal(capped[key], plain[key], err_msg=f"{key} {far} {near}")
    with pytest.raises(ValueError, match="0 to 32"):
        solver.set_adjoint_launch(-1, 4)


def _tables_along(grads, tangent):
    return sum(float(np.sum(grads[name] * tangent[name])) for name in _TABLES)


def _random_tangent(solver, seed):
    # Every entry moved: the factors of every layer cell along every axis.
    rng = np.random.default_rng(seed)
    nx, ny, nz = solver.shape
    lengths = dict(zip(_TABLES, [nx + 1, nx + 1, ny + 1, ny + 1, nz + 1, nz + 1] * 2))
    return {name: rng.standard_normal(n) for name, n in lengths.items()}


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", _LAYER_GRIDS)
def test_the_gradient_along_a_tangent_is_the_tables_gradient_along_it(name, precision):
    # dL/dθ along a tangent of the tables (the layer's damping, and a random one moving every entry)
    # equals the twelve tables' gradient summed with the tangent; the walls' gradient is the same
    # to the bit, with checkpoints across segments (the products of a segment's last step wait for
    # its recomputation) and in one segment.
    layout, signal, _ = load_golden(name)
    signal = signal[:160]
    target, _ = _problem(layout, signal)
    solver = B200WaveSolver(layout, precision=precision)
    y = solver.run(signal)
    solver.reset()
    dloss = 2.0 * (y - target)
    tangents = [_random_tangent(solver, 7), L.damping_tangent(layout, 4, 0.5)]
    for segment in (0, 45):
        solver.set_layer_tangent(None)
        tables = solver.gradient(signal, dloss, segment=segment)
        for tangent in tangents:
            solver.set_layer_tangent(tangent)
            along = solver.gradient(signal, dloss, segment=segment)
            assert set(_TABLES).isdisjoint(along)
            for key in ("coef_b", "coef_inv", "now", "before", "gain"):
                np.testing.assert_array_equal(along[key], tables[key], err_msg=key)
            expected = _tables_along(tables, tangent)
            scale = sum(float(np.sum(np.abs(tables[n] * tangent[n]))) for n in _TABLES)
            tolerance = 1e-11 if precision == "fp64" else 1e-5
            assert abs(along["layer_tangent"] - expected) <= tolerance * scale, (segment, along["layer_tangent"], expected)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_a_taped_run_keeps_the_tangents_factors_and_the_gradient_recomputes_nothing(precision):
    # A taped run from rest with a tangent set keeps the rows' trajectory and the tangent's factors
    # of every step: the gradient that follows equals the one that recomputes the forward pass, to
    # the bit, in one segment and across segments.
    layout, signal, _ = load_golden("fitted_open")
    signal = signal[:150]
    target, _ = _problem(layout, signal)
    solver = B200WaveSolver(layout, precision=precision)
    tangent = L.damping_tangent(layout, 4, 0.5)
    solver.set_layer_tangent(tangent)
    y = solver.run(signal)
    solver.reset()
    dloss = 2.0 * (y - target)
    for segment in (0, 40):
        plain = solver.gradient(signal, dloss, segment=segment)
        solver.set_tape(segment if segment else len(signal))
        solver.run(signal)
        taped = solver.gradient(signal, dloss, segment=segment)
        solver.set_tape(0)
        for key in plain:
            np.testing.assert_array_equal(taped[key], plain[key], err_msg=f"{key} {segment}")
    solver.set_layer_tangent(None)
    assert set(_TABLES) <= set(solver.gradient(signal, dloss, segment=40))
    with pytest.raises(ValueError, match="keep_x has 3 values"):
        solver.set_layer_tangent({"keep_x": np.zeros(3)})
    bad = dict(tangent, push_z=np.full_like(tangent["push_z"], np.nan))
    with pytest.raises(ValueError, match="not finite"):
        solver.set_layer_tangent(bad)
    plain_layout, _, _ = load_golden("resonant7")
    without = B200WaveSolver(plain_layout)
    with pytest.raises(ValueError, match="no matched layer"):
        without.set_layer_tangent({})
