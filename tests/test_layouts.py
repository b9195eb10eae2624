"""The host layout builder (acoustic_spaces_b200.layouts) against the reference's own layouts.

A convex room handed to the reference's WaveSolver as a triangle mesh (walls on cell faces, the
7-point stencil) and built here from its planes must give the same layout, array for array
(cpp/include/acoustic_spaces/fdtd.hpp:452-690 against layouts.cell_face_layout). Without the
reference sources, the builder's invariants are checked instead.
"""

from __future__ import annotations

import numpy as np
import pytest

import cases
from acoustic_spaces_b200 import layouts as L
from oracle.oracle import OracleSolver

H = 0.1
BOX = (4.0, 3.0, 2.4)
RATE = 343.0 / (L.COURANT * H)


def _material(rng):
    return L.Material(
        float(rng.uniform(0.02, 0.1)),
        L.resonant_branch(rng.uniform(0.005, 0.5), rng.uniform(0.5, 10.0), rng.uniform(30.0, 300.0), RATE),
    )


def _room(seed: int, open_face: int | None, layer: int, faces: int = 14, speed=None):
    rng = np.random.default_rng(seed)
    room = L.convex_room(rng, BOX, faces=faces, margin=H * (layer + 3), open_face=open_face, material=_material)
    points = L.inside_points(rng, room, BOX, 5, 0.35, apart=0.35)
    grid = L.Grid(-L.OFFSET * H, H, tuple(int(round(b / H)) for b in BOX))
    built = L.cell_face_layout(
        room, grid, points[0], points[1:], layer=layer, layer_damping=0.5 if layer else 0.0, speed=speed
    )
    return room, grid, points, built


def _reference_layout(room, grid, points, layer, speed=None):
    native = cases.reference_native()
    vertices, faces, owner = L.room_mesh(room)
    beta = np.array([0.0 if m is None else m.beta for m in room.materials])
    rows, owners = [np.zeros((0, 3))], [np.zeros(0, np.int64)]
    for k, m in enumerate(room.materials):
        if m is not None:
            rows.append(m.branches)
            owners.append(np.full(len(m.branches), k, np.int64))
    speeds = None if speed is None else np.full(grid.n, speed, np.float32)
    solver = native.WaveSolver(
        native.Bvh(vertices, faces), owner, beta, np.ascontiguousarray(np.vstack(rows)), np.concatenate(owners),
        grid.origin, grid.cell, *grid.shape, points[0], points[1:], layer=layer,
        layer_damping=0.5 if layer else 0.0, threads=2, speed=speeds,
    )  # fmt: skip
    return solver, solver.layout()


ROOMS = [(3, 1, 4, None), (4, None, 0, None), (5, 1, 4, 0.93), (6, None, 0, 0.99)]


@pytest.mark.parametrize("seed, open_face, layer, speed", ROOMS)
def test_the_builder_lays_a_room_out_as_the_reference_does(seed, open_face, layer, speed):
    if not cases.available():
        pytest.skip("the reference sources are not here")
    room, grid, points, built = _room(seed, open_face, layer, speed=speed)
    solver, ref = _reference_layout(room, grid, points, layer, speed)
    assert solver.air_cells == built.air_cells
    assert solver.boundary_cells == built.boundary_cells
    for name, value in built.layout.items():
        mine, theirs = np.asarray(value), np.asarray(ref[name])
        assert mine.dtype == theirs.dtype, name
        assert np.array_equal(mine, theirs), name


@pytest.mark.parametrize("seed, open_face, layer, speed", ROOMS)
def test_the_builders_layout_is_consistent(seed, open_face, layer, speed):
    _, grid, _, built = _room(seed, open_face, layer, speed=speed)
    lay = built.layout
    types = lay["types"]
    assert np.all(types[lay["special"]] == 2)
    assert np.all(types[lay["layer_cells"]] == 3)
    assert len(lay["special"]) == np.count_nonzero(types == 2)
    assert len(lay["layer_cells"]) == np.count_nonzero(types == 3)
    assert built.air_cells == np.count_nonzero(types)
    assert np.all(np.diff(lay["link_start"].astype(np.int64)) >= 0)
    assert abs(float(np.sum(lay["source"])) - (1.0 if speed is None else np.float32(speed * speed))) < 1e-5
    # every interior cell's six neighbours are air
    nx, ny, _ = grid.shape
    interior = np.flatnonzero(types == 1)
    for off in (1, -1, nx, -nx, nx * ny, -nx * ny):
        assert np.all(types[interior + off] != 0)


def test_the_builders_room_steps_stably_in_the_oracle():
    _, _, _, built = _room(3, 1, 4)
    signal = L.gaussian_drive(RATE, 300)
    out = OracleSolver(built.layout).run(signal)
    assert np.all(np.isfinite(out)) and np.abs(out).max() > 0.0


def test_the_builder_refuses_a_probe_next_to_the_source():
    rng = np.random.default_rng(1)
    room = L.convex_room(rng, BOX, faces=8, margin=0.3, open_face=None, material=_material)
    points = L.inside_points(rng, room, BOX, 1, 0.35)
    grid = L.Grid(-L.OFFSET * H, H, tuple(int(round(b / H)) for b in BOX))
    with pytest.raises(ValueError, match="three cells"):
        L.cell_face_layout(room, grid, points[0], points[:1] + 0.05)


def test_the_plain_shoebox_is_laid_out_as_the_reference_lays_it():
    # The plain box at 10 cm: six real walls, no branches, speed 0.99 in every cell; the reference's
    # own layout array for array, and its FP32 run equal to the oracle's to the bit.
    if not cases.available():
        pytest.skip("the reference sources are not here")
    w = L.shoebox_room(2, cell=0.1, steps=150)
    native = cases.reference_native()
    vertices, faces, owner = L.room_mesh(w.room)
    beta = np.array([m.beta for m in w.room.materials])
    assert np.all((beta > 0.0) & (beta < 1.0))
    solver = native.WaveSolver(
        native.Bvh(vertices, faces), owner, beta, np.zeros((0, 3)), np.zeros(0, np.int64), w.built.grid.origin,
        w.built.grid.cell, *w.built.grid.shape, w.source, w.receivers, layer=0, layer_damping=0.0, threads=2,
        speed=np.full(w.built.grid.n, 0.99, np.float32),
    )  # fmt: skip
    ref = solver.layout()
    for name, value in w.built.layout.items():
        assert np.array_equal(np.asarray(value), np.asarray(ref[name])), name
    assert np.array_equal(solver.run(w.signal), OracleSolver(w.built.layout).run(w.signal))


def test_the_batched_solves_are_laid_out_as_the_reference_lays_them():
    # Each (room, source) of the batch, from its scene, laid out by the reference: array for array.
    if not cases.available():
        pytest.skip("the reference sources are not here")
    b = L.batched_rooms(2, rooms=2, sources=2, cell=0.1, dims=(2.0, 4.0), steps=10)
    native = cases.reference_native()
    for lay, (room, grid, source, receivers) in zip(b.layouts, b.scenes):
        vertices, faces, owner = L.room_mesh(room)
        beta = np.array([m.beta for m in room.materials])
        solver = native.WaveSolver(
            native.Bvh(vertices, faces), owner, beta, np.zeros((0, 3)), np.zeros(0, np.int64), grid.origin,
            grid.cell, *grid.shape, source, receivers, layer=0, layer_damping=0.0, threads=2,
        )  # fmt: skip
        ref = solver.layout()
        for name, value in lay.items():
            assert np.array_equal(np.asarray(value), np.asarray(ref[name])), name
        assert np.array_equal(solver.run(b.signal), OracleSolver(lay).run(b.signal))


def test_the_polyhedral_workload_is_seeded():
    a = L.polyhedral_room(0, cell=0.2, steps=10)
    b = L.polyhedral_room(0, cell=0.2, steps=10)
    assert a.description == b.description
    for name in a.built.layout:
        assert np.array_equal(a.built.layout[name], b.built.layout[name])
    assert 12 <= int(a.description["room"].split(",")[1].split()[0]) <= 20


# ---- many grids stacked into one ---------------------------------------------------------------


def test_paris_admittance_inverts_paris_absorption():
    alpha = np.array([0.02, 0.1, 0.3, 0.5, 0.9])
    beta = L.paris_admittance(alpha)
    assert np.allclose(L.paris_absorption(1.0 / beta), alpha, rtol=1e-9)
    assert np.all(np.diff(beta) > 0)


def test_a_stack_steps_each_grid_as_it_steps_alone():
    # Two rooms with two sources each, stacked: every solve's probes equal its own run's, to the
    # bit, in the oracle (float) — the stack changes no row's coefficients or neighbours.
    b = L.batched_rooms(1, rooms=2, sources=2, cell=0.1, dims=(2.0, 4.0), steps=120)
    stacked = OracleSolver(b.stacked.layout).run(b.signal)
    for lay, (p0, p1, air, _) in zip(b.layouts, b.stacked.parts):
        assert np.array_equal(OracleSolver(lay).run(b.signal), stacked[p0:p1])
        assert air == np.count_nonzero(lay["types"])


@pytest.mark.parametrize("across", [1, 2, 3])
def test_golden_grids_stack_with_their_own_runs(across):
    # (across > 1: grids of different shapes side by side along x in one group of planes)
    from conftest import load_golden, still_names

    names = [n for n in still_names() if len(load_golden(n)[0]["layer_cells"]) == 0 and load_golden(n)[0]["scaled"][0] == 0]
    layouts = [load_golden(n)[0] for n in names]
    sevens = [lay for lay in layouts if int(lay["stencil"][0]) == 7]
    stacked = L.stack(sevens, across=across)
    signal = np.random.default_rng(2).standard_normal(150).astype(np.float32)
    together = OracleSolver(stacked.layout).run(signal)
    for lay, (p0, p1, _, _) in zip(sevens, stacked.parts):
        assert np.array_equal(OracleSolver(lay).run(signal), together[p0:p1])


def test_stacking_refuses_a_matched_layer():
    from conftest import load_golden

    with pytest.raises(ValueError, match="matched layer"):
        L.stack([load_golden("resonant7")[0], load_golden("open_layer")[0]])


def test_the_batched_solves_partition_across_ranks():
    # Each rank builds its own rooms (balanced by cells); together they are every room, once.
    import numpy as np

    from acoustic_spaces_b200 import layouts as L

    parts = L.partition([5, 3, 8, 1, 9, 2, 7], 3)
    assert sorted(k for p in parts for k in p) == list(range(7))
    loads = [sum([5, 3, 8, 1, 9, 2, 7][k] for k in p) for p in parts]
    assert max(loads) - min(loads) <= 9
    whole = L.batched_rooms(3, rooms=4, sources=1, cell=0.2, steps=10)
    halves = [L.batched_rooms(3, rooms=4, sources=1, cell=0.2, steps=10, part=(r, 2)) for r in range(2)]
    assert sum(h.description["air_cells"] for h in halves) == whole.description["air_cells"]
    mine = [L.partition([int(np.prod(L.room_grid(np.random.default_rng([3, k]).uniform(3.0, 12.0, 3), 0.2).shape))
                         for k in range(4)], 2)[r] for r in range(2)]  # fmt: skip
    assert sorted(mine[0] + mine[1]) == [0, 1, 2, 3]


def test_inside_points_refuses_a_room_too_small_for_the_clearance():
    room = L.shoebox(np.array([1.0, 1.0, 0.5]), [L.Material(0.1)] * 6)
    with pytest.raises(ValueError, match="too small"):
        L.inside_points(np.random.default_rng(0), room, (1.0, 1.0, 0.5), 2, 0.3)
