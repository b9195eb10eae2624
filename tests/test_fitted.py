"""Fitted (cut-cell) walls on the CPU: the rows' rules against the reference's own fitted layouts.

* ``fitted.set_up_fitted`` restates the reference's second stage (fdtd.hpp:970-1264): fed the
  reference's own fit (its CutFit: rows, air volumes, open and wall areas, slivers, kinds, widths)
  and the reference's own source and probe cells, it must give the reference's fitted layout array
  for array — on a convex polyhedral room open to a matched layer and on the reference's L-room
  with two free plates.
* ``fitted.lattice_widths`` must give the reference's cell widths on its lattice, to the bit.
* ``fitted.fit_from_cut`` (the owner rule and the rows' sums of this library's fit) is checked on
  an axis-aligned box open through one face, whose cut this test works out exactly by hand (the
  overlaps of intervals): against the reference's fit of the same box, every cell's kind, the rows
  and the air volumes, open areas, wall areas and slivers of the rows.
(The GPU cut of a general convex room: tests/test_gpu_fitted.py.)
"""

from __future__ import annotations

import numpy as np
import pytest

from acoustic_spaces_b200 import fitted
from acoustic_spaces_b200 import layouts as L
from oracle import oracle

native = oracle.reference_native()
needs_reference = pytest.mark.skipif(native is None, reason="the reference's compiled solver (oracle/_ref) is absent")

#: Moving-air arrays of the reference's layout, empty in still air (not stepped here).
_STILL = ("flow_x", "flow_y", "wind_x", "wind_y", "wind_z", "loop_x", "loop_y", "loop_z")


def _reference_solver(room, grid, source, probes, layer, damping):
    vertices, faces, owner = L.room_mesh(room)
    beta = np.array([0.0 if m is None else m.beta for m in room.materials])
    rows, owners = [np.zeros((0, 3))], [np.zeros(0, np.int64)]
    for k, m in enumerate(room.materials):
        if m is not None:
            rows.append(m.branches)
            owners.append(np.full(len(m.branches), k, np.int64))
    solver = native.WaveSolver(
        native.Bvh(vertices, faces), owner, beta, np.ascontiguousarray(np.vstack(rows)), np.concatenate(owners),
        grid.origin, grid.cell, *grid.shape, np.asarray(source, float), np.asarray(probes, float), layer=layer,
        layer_damping=damping, threads=4, fitted_walls=True, vertices=np.ascontiguousarray(vertices),
        faces=np.ascontiguousarray(faces),
    )  # fmt: skip
    fit = native.CutFit(vertices, faces, owner, len(room.materials), grid.origin, grid.cell, *grid.shape,
                        np.asarray(source, float), layer=layer, threads=4)  # fmt: skip
    return solver, fit


def _as_fit(cut_fit) -> fitted.Fit:
    c = cut_fit.cut_cells()
    return fitted.Fit(c["cell"], c["air_volume"], c["open_area"], c["wall_area"], c["sliver"],
                      np.asarray(cut_fit.cut_air()), tuple(np.asarray(w) for w in cut_fit.cut_widths()))  # fmt: skip


def _assert_layouts_equal(ours, reference):
    for key, value in reference.items():
        if key in _STILL:
            assert len(np.asarray(value)) == 0, key
            continue
        expected = np.asarray(value)
        got = np.asarray(ours[key])
        assert got.shape == expected.shape, key
        np.testing.assert_array_equal(got.astype(expected.dtype), expected, err_msg=key)


def _polyhedral():
    w = L.polyhedral_room(0, box=(4.0, 3.0, 2.0), cell=0.04, steps=10)
    return w.room, w.built.grid, w.source, w.receivers


@needs_reference
def test_set_up_fitted_on_the_references_fit_is_the_references_layout():
    room, grid, source, probes = _polyhedral()
    solver, cut_fit = _reference_solver(room, grid, source, probes, 8, 0.5)
    points = cut_fit.cut_points(np.asarray(source).reshape(1, 3), np.asarray(probes), 1)
    ours = fitted.set_up_fitted(_as_fit(cut_fit), grid, room.materials, points["source"], points["probes"], layer=8,
                                layer_damping=0.5)  # fmt: skip
    _assert_layouts_equal(ours, solver.layout())


@needs_reference
def test_set_up_fitted_on_the_l_room_is_the_references_layout():
    # The reference's L-room (tests/test_fitted_walls.py:280-300): a closed, non-convex room with
    # two turned free plates of a second and third material, resonant walls.
    import cases

    v, f, mat, h, origin, shape, src = cases.l_room()
    probes = cases.l_room_points()
    wall = L.Material(0.05, np.array([[0.3, 0.02, 0.1]]))
    materials = [wall, L.Material(0.3), wall]
    beta = np.array([m.beta for m in materials])
    solver = native.WaveSolver(
        native.Bvh(v, f), mat, beta, np.vstack([wall.branches, wall.branches]), np.array([0, 2], np.int64),
        origin, h, *(int(n) for n in shape), src, probes, threads=2, fitted_walls=True,
        vertices=np.ascontiguousarray(v), faces=np.ascontiguousarray(f),
    )  # fmt: skip
    cut_fit = native.CutFit(v, f, mat, 3, origin, h, *(int(n) for n in shape), src, threads=2)
    points = cut_fit.cut_points(np.asarray(src).reshape(1, 3), probes, 1)
    grid = L.Grid(np.asarray(origin, float), h, tuple(int(n) for n in shape))
    ours = fitted.set_up_fitted(_as_fit(cut_fit), grid, materials, points["source"], points["probes"])
    _assert_layouts_equal(ours, solver.layout())


@needs_reference
def test_lattice_widths_are_the_references():
    room, grid, source, probes = _polyhedral()
    _, cut_fit = _reference_solver(room, grid, source, probes, 8, 0.5)
    for ours, theirs in zip(fitted.lattice_widths(room, grid), cut_fit.cut_widths()):
        np.testing.assert_array_equal(ours, np.asarray(theirs))


@needs_reference
def test_the_fitted_cubic_stencil_is_the_references_to_rounding():
    room, grid, source, probes = _polyhedral()
    _, cut_fit = _reference_solver(room, grid, source, probes, 8, 0.5)
    points = cut_fit.cut_points(np.asarray(source).reshape(1, 3), np.asarray(probes), 1)
    for point, expected in zip([source, *probes], [points["source"], *points["probes"]]):
        ours = fitted.fitted_cubic(grid, point)
        assert [i for i, _ in ours] == [int(i) for i, _ in expected]
        np.testing.assert_allclose([w for _, w in ours], [w for _, w in expected], rtol=0, atol=1e-14)


# ---- the owner rule and the sums, on a box cut by hand ------------------------------------------


def _box(open_face=1):
    """A 1.47 x 1.13 x 0.91 m box of three materials (one a resonant branch) off the grid's planes,
    open through its +x face (``open_face``), on 4 cm cells with a 4-cell layer beyond a 3-cell
    margin."""
    cell, layer = 0.04, 4
    lo = np.array([0.3011, 0.2897, 0.3103])
    hi = lo + np.array([1.47, 1.13, 0.91])
    normals, offsets = [], []
    for a in range(3):
        for sign in (-1.0, 1.0):
            n = np.zeros(3)
            n[a] = sign
            normals.append(n)
            offsets.append(sign * (hi[a] if sign > 0 else lo[a]))
    rate = 343.0 / (L.COURANT * cell)
    branch = L.resonant_branch(0.2, 2.0, 120.0, rate)
    mats = [L.Material(0.05, branch), None, L.Material(0.08), L.Material(0.03, branch), L.Material(0.08),
            L.Material(0.05, branch)]  # fmt: skip
    if open_face != 1:
        mats[1], mats[open_face] = mats[open_face], None
    room = L.Room(np.array(normals), np.array(offsets), mats)
    margin = cell * (layer + 3)
    origin = lo - margin - L.OFFSET * cell
    shape = tuple(int(np.ceil((hi[a] + margin - origin[a]) / cell)) + 1 for a in range(3))
    return room, L.Grid(origin, cell, shape), layer, lo, hi


def _box_cut(room, grid, lo, hi) -> fitted.Cut:
    """The cut of an axis-aligned box's walls by the grid, exactly as fdtd_cut_convex defines it:
    per axis the overlap of each cell with the walls' interval (a face left open does not bound the
    air's regions, and bounds the walls' faces), the products of those overlaps."""
    nx, ny, nz = grid.shape
    open_ = [m is None for m in room.materials]
    units = [(np.array([lo[a], hi[a]]) - grid.origin[a]) / grid.cell for a in range(3)]
    per_axis = []
    for a, n in enumerate((nx, ny, nz)):
        c0 = np.arange(n, dtype=np.float64)
        low, high = units[a]
        wall_low, wall_high = not open_[2 * a], not open_[2 * a + 1]
        # the regions' interval on this axis: the walls' planes only
        r_lo = low if wall_low else -np.inf
        r_hi = high if wall_high else np.inf
        region = np.clip(np.minimum(c0 + 1, r_hi) - np.maximum(c0, r_lo), 0.0, 1.0)
        # the walls' faces' interval: every plane
        face = np.clip(np.minimum(c0 + 1, high) - np.maximum(c0, low), 0.0, 1.0)
        face_lo = (c0 <= r_lo) & (r_lo <= c0 + 1) if np.isfinite(r_lo) else np.zeros(n, bool)
        crosses = [(c0 < p) & (p < c0 + 1) if np.isfinite(p) else np.zeros(n, bool) for p in (r_lo, r_hi)]
        # each cell face's position inside the regions' interval (-: at c0, +: at c0 + 1)
        inside_lo = (c0 >= r_lo) & (c0 <= r_hi)
        inside_hi = (c0 + 1 >= r_lo) & (c0 + 1 <= r_hi)
        per_axis.append(dict(region=region, face=face, crosses=crosses, inside=(inside_lo, inside_hi)))
        del face_lo
    X, Y, Z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    X, Y, Z = X.transpose(2, 1, 0).reshape(-1), Y.transpose(2, 1, 0).reshape(-1), Z.transpose(2, 1, 0).reshape(-1)
    at = (X, Y, Z)
    cut_any = np.zeros(nx * ny * nz, bool)
    outside = np.zeros(nx * ny * nz, bool)
    for a in range(3):
        p = per_axis[a]
        for side in (0, 1):
            if not open_[2 * a + side]:
                cut_any |= p["crosses"][side][at[a]]
        outside |= p["region"][at[a]] <= 0.0
    cells = np.flatnonzero(cut_any & ~outside)
    C = len(cells)
    xyz = [c[cells] for c in at]
    region = [per_axis[a]["region"][xyz[a]] for a in range(3)]
    face = [per_axis[a]["face"][xyz[a]] for a in range(3)]
    volume = region[0] * region[1] * region[2]
    face_area = np.zeros((C, 6))
    for a in range(3):
        b, c = (a + 1) % 3, (a + 2) % 3
        for side in (0, 1):
            face_area[:, 2 * a + side] = np.where(per_axis[a]["inside"][side][xyz[a]], region[b] * region[c], 0.0)
    cap = np.zeros((C, 6))
    bare = np.zeros(C)
    for f in range(6):
        a, side = f // 2, f % 2
        if open_[f]:
            continue
        b, c = (a + 1) % 3, (a + 2) % 3
        crosses = per_axis[a]["crosses"][side][xyz[a]]
        cap[:, f] = np.where(crosses, face[b] * face[c], 0.0)
        bare += np.where(crosses, region[b] * region[c] - cap[:, f], 0.0)
    return fitted.Cut(cells.astype(np.int64), volume, face_area, cap, bare)


@needs_reference
@pytest.mark.parametrize("open_face", [1, 4])
def test_the_owner_rule_and_sums_on_a_box_are_the_references(open_face):
    room, grid, layer, lo, hi = _box(open_face)
    source = 0.5 * (lo + hi)
    probes = source + np.array([[0.2, 0.1, 0.05]])
    _, cut_fit = _reference_solver(room, grid, source, probes, layer, 0.5)
    ref = _as_fit(cut_fit)
    ours = fitted.fit_from_cut(_box_cut(room, grid, lo, hi), room, grid, layer=layer)
    np.testing.assert_array_equal(ours.air, ref.air)
    np.testing.assert_array_equal(ours.cell, ref.cell)
    for key in ("air_volume", "open_area", "wall_area", "sliver"):
        np.testing.assert_allclose(getattr(ours, key), getattr(ref, key), rtol=0, atol=1e-9, err_msg=key)


def test_accumulate_sums_a_tables_columns_as_the_whole_table_does():
    # target[index] += values with repeated indices: by column over a table's rows (a short index
    # into a large table) the entries gain exactly what one bincount over the whole table gives.
    rng = np.random.default_rng(5)
    rows, cols = 5000, 18
    base = rng.standard_normal((rows, cols))
    index = rng.integers(0, rows * cols, 900) // 3 * 3  # repeats, a few columns
    values = rng.standard_normal(900)
    by_column = base.copy()
    fitted._accumulate(by_column, index, values)
    whole = base.copy().reshape(-1)
    whole += np.bincount(index, values, minlength=whole.size)
    np.testing.assert_array_equal(by_column.reshape(-1), whole)
    scalar = base.copy()
    fitted._accumulate(scalar, index, 0.5)
    whole = base.copy().reshape(-1)
    whole += np.bincount(index, np.full(900, 0.5), minlength=whole.size)
    np.testing.assert_array_equal(scalar.reshape(-1), whole)
