"""Moving air on the GPU (fdtd_flow.cuh) against the oracle's carry.

The reference's own wind grids (the plain form and the form round the solids, tests/golden/
wind_*.npz) are stepped by the golden-grid tests of test_gpu_parity.py, to the bit against the
reference's series. Here the carry runs on a larger room with synthetic moving air of both forms,
laid out by the reference's rules (fdtd.hpp:1680-1735 for the plain form's neighbour bits; the
round form's mask 1 inside the moving air and 2 on its border), against the oracle in FP32 and FP64,
in pieces that flip the levels' roles; and what steps still air only refuses moving air.
"""

from __future__ import annotations

import numpy as np
import pytest

from acoustic_spaces_b200 import B200WaveSolver, layouts
from oracle.oracle import OracleSolver

pytestmark = pytest.mark.gpu


def _grid(layout):
    nx, ny, nz = (int(v) for v in layout["shape"])
    return np.asarray(layout["types"]).reshape(nz, ny, nx)


def _step(a, axis, k):
    """a shifted so that entry i holds a's value k cells along `axis` (axis 0 = x), solid outside."""
    ax = 2 - axis
    out = np.zeros_like(a)
    src = [slice(None)] * 3
    dst = [slice(None)] * 3
    n = a.shape[ax]
    if k > 0:
        src[ax], dst[ax] = slice(k, n), slice(0, n - k)
    else:
        src[ax], dst[ax] = slice(0, n + k), slice(-k, n)
    out[tuple(dst)] = a[tuple(src)]
    return out


def _plain_flow(layout, shift=(0.2, 0.07)):
    # The air moves every interior and special cell by `shift`; each cell's bits say which of its
    # row's neighbours, one and two cells along x and y, are air that moves too.
    types = _grid(layout)
    moving = (types == 1) | (types == 2)
    mask = np.zeros(types.shape, np.uint8)
    for axis in (0, 1):
        below, above = _step(moving, axis, -1) & moving, _step(moving, axis, 1) & moving
        below2 = below & _step(moving, axis, -2)
        above2 = above & _step(moving, axis, 2)
        bits = below * 1 + above * 2 + below2 * 4 + above2 * 8
        mask |= (bits << (4 * axis)).astype(np.uint8)
    fx = np.where(moving, shift[0], 0.0).astype(np.float32)
    fy = np.where(moving, shift[1], 0.0).astype(np.float32)
    return {"flow_x": fx.reshape(-1), "flow_y": fy.reshape(-1), "flow_mask": mask.reshape(-1)}


def _round_flow(layout, seed=3):
    # Face winds and loop terms drawn at random; the interior and special cells two cells or more
    # from the grid's edges move (1), those with a still axial neighbour on the border (2).
    types = _grid(layout)
    nz, ny, nx = types.shape
    moving = (types == 1) | (types == 2)
    inner = np.zeros_like(moving)
    inner[2 : nz - 2, 2 : ny - 2, 2 : nx - 2] = True
    moving &= inner
    border = np.zeros_like(moving)
    for axis in range(3):
        for k in (-1, 1):
            border |= moving & ~_step(moving, axis, k)
    mask = np.where(border, 2, np.where(moving, 1, 0)).astype(np.uint8)
    rng = np.random.default_rng(seed)
    out = {"flow_mask": mask.reshape(-1)}
    for a in "xyz":
        out[f"wind_{a}"] = rng.uniform(-0.2, 0.2, types.size).astype(np.float32)
        out[f"loop_{a}"] = rng.uniform(-0.01, 0.01, types.size).astype(np.float32)
    return out


@pytest.fixture(scope="module")
def room():
    return layouts.polyhedral_room(0, box=(4.0, 3.0, 2.0), cell=0.04, steps=60)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("form", ["plain", "round"])
def test_gpu_carries_moving_air_as_the_oracle_does(room, form, precision):
    layout = dict(room.built.layout)
    layout.update(_plain_flow(layout) if form == "plain" else _round_flow(layout))
    gpu = B200WaveSolver(layout, precision=precision, autotune=False)
    oracle = OracleSolver(layout, precision)
    cuts = [0, 1, 30, 60]
    got = np.concatenate([gpu.run(room.signal[a:b]) for a, b in zip(cuts[:-1], cuts[1:])], axis=1)
    want = oracle.run(room.signal[:60])
    assert np.all(np.isfinite(want)) and np.abs(want).max() > 0
    assert np.array_equal(got, want), np.abs(got - want).max()
    sa, sb = gpu.state(), oracle.state()
    for key in sa:
        assert np.array_equal(sa[key], sb[key]), key
    # the air's motion changes the field: the same room with still air differs
    still = OracleSolver(room.built.layout, precision).run(room.signal[:60])
    assert not np.array_equal(still, want)


def test_gpu_moving_air_refuses_what_steps_still_air_only():
    from conftest import load_golden

    layout, signal, _ = load_golden("wind_plain")
    with pytest.raises(ValueError, match="still air only"):
        B200WaveSolver(layout, precision="fp32c")
    gpu = B200WaveSolver(layout)
    with pytest.raises(ValueError, match="still air only"):
        gpu.gradient(signal[:20], np.ones((gpu.probes, 20)))
    # the handle steps on as before
    _, _, reference = load_golden("wind_plain")
    assert np.array_equal(gpu.run(signal), reference)
