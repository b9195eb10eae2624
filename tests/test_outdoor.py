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
