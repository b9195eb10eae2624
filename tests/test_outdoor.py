"""The outdoor half-space (porous ground into a five-sided matched layer, a thin rigid barrier):
its layout on the CPU, and the B200 stepping it bit for bit as the oracle does (gpu)."""

from __future__ import annotations

import numpy as np
import pytest

from acoustic_spaces_b200 import B200WaveSolver, layouts
from oracle.oracle import OracleSolver

SMALL = dict(shape=(128, 64, 48), layer=8, receivers=8, steps=300)
STEPS = ((-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1))


def _cells(lay, index):
    nx, ny, _ = (int(v) for v in lay["shape"])
    return index % nx, (index // nx) % ny, index // (nx * ny)


def test_no_open_link_crosses_the_barrier():
    w = layouts.outdoor_halfspace(0, **SMALL)
    lay, grid = w.built.layout, w.built.grid
    screen = w.room.screens[0]
    special = np.asarray(lay["special"], np.int64)
    start = np.asarray(lay["link_start"], np.int64)
    direction = np.asarray(lay["link_direction"], np.int64)
    x, y, z = _cells(lay, special)
    crossings = 0
    for k in range(len(special)):
        for d in direction[start[k]:start[k + 1]]:
            if STEPS[d][0] == 0:
                continue
            here = grid.centres(0)[x[k]]
            there = here + STEPS[d][0] * grid.cell
            yc, zc = grid.centres(1)[y[k]], grid.centres(2)[z[k]]
            within = screen.lo[0] <= yc <= screen.hi[0] and screen.lo[1] <= zc <= screen.hi[1]
            crossings += within and (here - screen.position) * (there - screen.position) < 0
    assert crossings == 0
    # and the cells on either side of it are special rows (their link across is cut)
    free = layouts.outdoor_halfspace(0, barrier=False, **SMALL)
    assert len(lay["special"]) > len(free.built.layout["special"])


def test_the_layer_has_no_floor_and_the_ground_runs_into_it():
    w = layouts.outdoor_halfspace(0, **SMALL)
    lay = w.built.layout
    nx, ny, nz = (int(v) for v in lay["shape"])
    types = np.asarray(lay["types"]).reshape(nz, ny, nx)
    assert not np.any(types[:2])  # below the ground
    first = types[2]
    assert np.count_nonzero(first == 2) > 0 and np.count_nonzero(first == 3) > 0  # ground rows, layer
    layer = np.asarray(lay["layer_cells"], np.int64)
    x, y, z = _cells(lay, layer)
    near_side = (x <= 8) | (x >= nx - 9) | (y <= 8) | (y >= ny - 9) | (z >= nz - 9)
    assert np.all(near_side)
    kz = np.asarray(lay["keep_z"])
    assert kz[3] == kz[nz // 2]  # no damping toward the floor
    assert kz[nz - 2] < kz[nz // 2]


def test_the_reference_lays_the_outdoor_pieces_out_alike_where_they_stop_short_of_the_layer():
    # The reference refuses the half-space itself (its ground runs into the matched layer), so its
    # pieces are checked on a grid it accepts: a floating porous ground panel (Miki's admittance,
    # three relaxation branches) and the rigid barrier, both short of a 4-cell layer on all six
    # sides, air all round. Handed to the reference as four triangles, the same scene gives the
    # same layout, array for array, and the reference's run equals the oracle's to the bit.
    from oracle.oracle import reference_native

    native = reference_native()
    if native is None:
        pytest.skip("the reference sources are not here")
    cell, layer, shape = 0.1, 4, (80, 40, 40)
    rate = 343.0 / (layouts.COURANT * cell)
    grid = layouts.Grid(-layouts.OFFSET * cell, cell, shape)
    ground_z = grid.origin[2] + 12.37 * cell
    ground = layouts.porous_ground(200e3, rate)
    lo = (grid.origin[0] + (layer + 4) * cell, grid.origin[1] + (layer + 4.21) * cell)
    hi = (grid.origin[0] + (shape[0] - layer - 4) * cell, grid.origin[1] + (shape[1] - layer - 3.79) * cell)
    barrier_x = grid.origin[0] + 40.37 * cell
    room = layouts.Room(np.zeros((0, 3)), np.zeros(0), [])
    room.screens.append(layouts.Screen(2, ground_z, lo, hi, ground))
    room.screens.append(layouts.Screen(0, barrier_x, (lo[1], ground_z), (hi[1], ground_z + 1.0), layouts.Material(0.0)))
    y = 0.5 * (lo[1] + hi[1])
    source = np.array([barrier_x - 1.0, y, ground_z + 0.5])
    probes = np.array([[barrier_x + 1.0, y, ground_z + 1.0], [barrier_x + 2.0, y + 0.3, ground_z + 1.2]])
    built = layouts.cell_face_layout(room, grid, source, probes, layer=layer, layer_damping=0.5, rate=rate,
                                     layer_meets_walls=False)  # fmt: skip
    vertices, faces, owner = [], [], []
    for k, screen in enumerate(room.screens):
        others = [b for b in range(3) if b != screen.axis]
        for u, v in ((screen.lo[0], screen.lo[1]), (screen.hi[0], screen.lo[1]), (screen.hi[0], screen.hi[1]),
                     (screen.lo[0], screen.hi[1])):  # fmt: skip
            p = np.zeros(3)
            p[screen.axis], p[others[0]], p[others[1]] = screen.position, u, v
            vertices.append(p)
        faces += [[4 * k, 4 * k + 1, 4 * k + 2], [4 * k, 4 * k + 2, 4 * k + 3]]
        owner += [k, k]
    branches = np.ascontiguousarray(np.asarray(ground.branches, float).reshape(-1, 3))
    solver = native.WaveSolver(
        native.Bvh(np.array(vertices), np.array(faces, np.int64)), np.array(owner, np.int64),
        np.array([ground.beta, 0.0]), branches, np.zeros(len(branches), np.int64), grid.origin, grid.cell, *grid.shape,
        source, probes, layer=layer, layer_damping=0.5, threads=2,
    )  # fmt: skip
    ref = solver.layout()
    assert len(built.layout["state_branch"]) > 0 and len(built.layout["layer_cells"]) > 0
    for name, value in built.layout.items():
        assert np.array_equal(np.asarray(value), np.asarray(ref[name])), name
    signal = layouts.gaussian_drive(rate, 200)
    assert np.array_equal(solver.run(signal), OracleSolver(built.layout).run(signal))


def test_the_oracle_steps_it():
    w = layouts.outdoor_halfspace(0, **SMALL)
    y = OracleSolver(w.built.layout, "fp32").run(w.signal)
    assert np.all(np.isfinite(y)) and np.abs(y).max() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("barrier", [True, False])
def test_gpu_steps_the_half_space_as_the_oracle(barrier):
    w = layouts.outdoor_halfspace(0, barrier=barrier, **SMALL)
    for precision in ("fp32", "fp64"):
        ours = B200WaveSolver(w.built.layout, precision=precision).run(w.signal)
        oracle = OracleSolver(w.built.layout, precision).run(w.signal)
        np.testing.assert_array_equal(ours, oracle, err_msg=precision)


@pytest.mark.parametrize("sigma", [50e3, 1e6, 20e6])
def test_the_ground_fit_follows_mikis_admittance(sigma):
    # A real beta and up to three relaxation branches (g jw / (jw + 2 pi fc), fc log-spaced over the
    # band, non-negative least squares: passive) against Miki's admittance, 20-600 Hz: within 15 %
    # rms and 30 % at worst over the flow resistivities of the half-space (the fit's bound, not the
    # model's: its corners are fixed).
    import math

    rate = 343.0 / (layouts.COURANT * 0.1)
    ground = layouts.porous_ground(sigma, rate)
    assert ground.beta >= 0.0 and np.all(np.asarray(ground.branches) >= 0.0)
    f = np.geomspace(20.0, 600.0, 400)
    jw = 2j * math.pi * f
    fitted = ground.beta + sum((1.0 / r) * jw / (jw + q * rate / r) for _, r, q in np.asarray(ground.branches))
    miki = layouts.miki_admittance(f, sigma)
    rel = np.abs(fitted - miki) / np.abs(miki)
    assert np.sqrt(np.mean(rel**2)) < 0.15 and rel.max() < 0.30, (np.sqrt(np.mean(rel**2)), rel.max())
