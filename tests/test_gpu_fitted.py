"""Fitted (cut-cell) walls on the B200: this library's FP64 fit of a convex room, and stepping it.

* The cut on the GPU (fdtd_cut_convex) and the rows from it (``fitted.fit_from_cut``) against the
  reference's own fit of the same room (its CutFit, exact lattice arithmetic on the host): every
  cell's kind equal, the rows a subset of the reference's, and the rows' air volumes, open areas,
  wall areas and slivers within 1e-9 on all but a few rows (measured: 11 of 35,747 differ, at the
  room's edges).
* The grid laid out from this fit, stepped by the oracle, against the reference's own fitted grid
  stepped by the reference: the probes' series within 1e-4 (relative L2; measured 8e-6).
* The B200 steps the fitted grid (its 18-link rows) as the oracle does, to the bit, in FP32 and
  FP64, run in pieces; the full-size room (500 x 375 x 250 cells of 4 cm) run in pieces equals one
  run, and its FP32 responses stay within 1e-4 of FP64.
"""

from __future__ import annotations

import numpy as np
import pytest

from acoustic_spaces_b200 import B200WaveSolver, fitted
from acoustic_spaces_b200 import layouts as L
from oracle import oracle
from oracle.oracle import OracleSolver

pytestmark = pytest.mark.gpu
native = oracle.reference_native()
needs_reference = pytest.mark.skipif(native is None, reason="the reference's compiled solver (oracle/_ref) is absent")


def _room(steps=1500):
    return L.polyhedral_room(0, box=(4.0, 3.0, 2.0), cell=0.04, steps=steps, walls="fitted")


def _reference(w):
    room, grid = w.room, w.built.grid
    vertices, faces, owner = L.room_mesh(room)
    beta = np.array([0.0 if m is None else m.beta for m in room.materials])
    rows, owners = [np.zeros((0, 3))], [np.zeros(0, np.int64)]
    for k, m in enumerate(room.materials):
        if m is not None:
            rows.append(m.branches)
            owners.append(np.full(len(m.branches), k, np.int64))
    solver = native.WaveSolver(
        native.Bvh(vertices, faces), owner, beta, np.ascontiguousarray(np.vstack(rows)), np.concatenate(owners),
        grid.origin, grid.cell, *grid.shape, w.source, w.receivers, layer=8, layer_damping=0.5, threads=8,
        fitted_walls=True, vertices=np.ascontiguousarray(vertices), faces=np.ascontiguousarray(faces),
    )  # fmt: skip
    cut_fit = native.CutFit(vertices, faces, owner, len(room.materials), grid.origin, grid.cell, *grid.shape,
                            w.source, layer=8, threads=8)  # fmt: skip
    return solver, cut_fit


@needs_reference
def test_the_gpu_fit_is_the_references_fit_away_from_a_few_edge_cells():
    w = _room(10)
    ours = fitted.convex_fit(w.room, w.built.grid, layer=8)
    _, cut_fit = _reference(w)
    ref = cut_fit.cut_cells()
    np.testing.assert_array_equal(ours.air, np.asarray(cut_fit.cut_air()))
    common, ia, ib = np.intersect1d(ours.cell, ref["cell"], return_indices=True)
    assert len(common) == len(ours.cell)
    assert len(common) >= 0.999 * len(ref["cell"])
    for key in ("air_volume", "open_area", "wall_area", "sliver"):
        d = np.abs(getattr(ours, key)[ia] - ref[key][ib]).reshape(len(common), -1).max(axis=1)
        assert np.count_nonzero(d > 1e-9) <= 0.001 * len(common), key


@needs_reference
def test_the_fitted_grid_responds_as_the_references_fitted_grid():
    w = _room()
    solver, _ = _reference(w)
    theirs = solver.run(w.signal)
    ours = OracleSolver(w.built.layout).run(w.signal)
    rel = np.linalg.norm(ours - theirs, axis=1) / np.linalg.norm(theirs, axis=1)
    assert rel.max() <= 1e-4, rel.max()


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_gpu_steps_the_fitted_grid_as_the_oracle(precision):
    w = _room(600)
    layout = w.built.layout
    assert int(np.diff(layout["link_start"]).max()) > 6  # rows with edge-diagonal links
    gpu = B200WaveSolver(layout, precision=precision, autotune=False)
    got = np.concatenate([gpu.run(w.signal[a:b]) for a, b in [(0, 199), (199, 200), (200, 600)]], axis=1)
    oracle_ = OracleSolver(layout, precision)
    assert np.array_equal(got, oracle_.run(w.signal))
    sa, sb = gpu.state(), oracle_.state()
    for key in sa:
        assert np.array_equal(sa[key], sb[key]), key


def test_gpu_full_size_fitted_room_in_pieces_is_one_run():
    # The full polyhedral room (500 x 375 x 250 cells of 4 cm) with fitted walls, fitted on the GPU.
    w = L.polyhedral_room(0, steps=600, walls="fitted")
    layout = w.built.layout
    one = B200WaveSolver(layout).run(w.signal)
    pieces = B200WaveSolver(layout)
    got = np.concatenate([pieces.run(w.signal[a:b]) for a, b in [(0, 77), (77, 300), (300, 600)]], axis=1)
    assert np.array_equal(got, one)
    p64 = B200WaveSolver(layout, precision="fp64").run(w.signal)
    # (over the receivers the sound has reached in these 600 steps)
    energy = np.linalg.norm(p64, axis=1)
    reached = energy > 1e-3 * energy.max()
    assert reached.sum() >= 4
    rel = np.linalg.norm(one - p64, axis=1)[reached] / energy[reached]
    assert rel.max() <= 1e-4, rel.max()
