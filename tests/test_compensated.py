"""Compensated single precision (FDTD_FP32_COMPENSATED): the same scheme stepped in float on each
cell's pressure and its increment p_n - p_(n-1), with the matched layer's pressure carried on from
its own.

It has no counterpart in the reference, so its bar is accuracy: against the FP64 oracle it must
stay far closer than the reference's FP32 arithmetic where that drifts (a closed room with a net
mass, an open room draining one into the matched layer), and no worse where it does not. Its own
oracle instantiation (ORACLE_FP32C) is the GPU's checker: the GPU steps every golden grid — both
stencils, speed fields, branches, fitted walls, the matched layer — equal to it to the bit.
"""

from __future__ import annotations

import numpy as np
import pytest
from conftest import load_golden, still_names

from acoustic_spaces_b200 import layouts as L
from oracle.oracle import OracleSolver


def _rel(a: np.ndarray, b: np.ndarray) -> float:
    """The worst receiver's relative L2 distance of a from b, over receivers the sound reached."""
    energy = np.linalg.norm(b, axis=1)
    reached = energy > 1e-3 * energy.max()
    return float((np.linalg.norm(a - b, axis=1)[reached] / energy[reached]).max())


def _open_room(steps: int):
    # The polyhedral room at 20 cm (100 x 75 x 50): 19 planes with resonant walls, the +x face open
    # into an 8-cell matched layer; the Gaussian drive leaves a net mass that drains into the layer.
    return L.polyhedral_room(0, cell=0.2, steps=steps)


@pytest.fixture(scope="module")
def open_room_runs():
    w = _open_room(1500)
    return {p: OracleSolver(w.built.layout, p).run(w.signal) for p in ("fp64", "fp32", "fp32c")}


def test_compensated_stays_with_fp64_where_fp32_drifts_in_an_open_room(open_room_runs):
    r = open_room_runs
    e32, e32c = _rel(r["fp32"], r["fp64"]), _rel(r["fp32c"], r["fp64"])
    assert e32 > 5e-6, e32  # the split layer's rounding (its parts grow far beyond the pressure)
    assert e32c < 2e-6, e32c
    assert e32c < e32 / 5


def test_compensated_holds_a_closed_rooms_net_mass():
    # The plain box at 10 cm with the Gaussian drive: a constant mode that the real walls do not
    # damp, in which fp32's rounding accumulates step after step; the increments do not feed it.
    w = L.shoebox_room(0, cell=0.1, steps=2000)
    r = {p: OracleSolver(w.built.layout, p).run(w.signal) for p in ("fp64", "fp32", "fp32c")}
    e32, e32c = _rel(r["fp32"], r["fp64"]), _rel(r["fp32c"], r["fp64"])
    assert e32 > 1e-2, e32
    assert e32c < 1e-5, e32c


@pytest.mark.parametrize("name", still_names())
def test_compensated_is_no_worse_than_fp32_on_the_golden_grids(name):
    layout, signal, reference = load_golden(name)
    p64 = OracleSolver(layout, "fp64").run(signal)
    p32c = OracleSolver(layout, "fp32c").run(signal)
    assert np.all(np.isfinite(p32c))
    # the reference's own FP32 series against the FP64 oracle: the compensated form within it
    # (and within single precision's reach where both are at rounding level)
    assert _rel(p32c, p64) <= max(2.0 * _rel(reference, p64), 1e-5), (_rel(p32c, p64), _rel(reference, p64))


def test_compensated_state_reads_the_level_before_as_pressure_less_increment():
    layout, signal, _ = load_golden("open_layer")
    a = OracleSolver(layout, "fp32c")
    a.run(signal[:101])
    st = a.state()
    b = OracleSolver(layout, "fp32c")
    b.run(signal[:100])
    before = b.state()["current"]
    # the pressure a step before, to within the increment's rounding
    scale = np.abs(before).max()
    assert np.abs(st["previous"] - before).max() <= 1e-6 * scale


def test_compensated_reset_and_pieces_repeat_the_run():
    layout, signal, _ = load_golden("resonant19")
    a = OracleSolver(layout, "fp32c")
    whole = a.run(signal)
    a.reset()
    pieces = np.concatenate([a.run(signal[:77]), a.run(signal[77:])], axis=1)
    assert np.array_equal(whole, pieces)


# ---- the GPU against its checker -------------------------------------------------------------


@pytest.mark.gpu
@pytest.mark.parametrize("name", still_names())
def test_gpu_compensated_equals_its_oracle_on_the_golden_grids(name):
    from acoustic_spaces_b200 import B200WaveSolver

    layout, signal, _ = load_golden(name)
    gpu = B200WaveSolver(layout, precision="fp32c")
    oracle = OracleSolver(layout, "fp32c")
    cuts = [0, 177, 178, len(signal)]
    got = np.concatenate([gpu.run(signal[a:b]) for a, b in zip(cuts[:-1], cuts[1:])], axis=1)
    assert np.array_equal(got, oracle.run(signal))
    sa, sb = gpu.state(), oracle.state()
    for key in sa:
        assert np.array_equal(sa[key], sb[key]), key


@pytest.mark.gpu
def test_gpu_compensated_steps_the_open_room_as_its_oracle_does():
    from acoustic_spaces_b200 import B200WaveSolver

    w = _open_room(400)
    gpu = B200WaveSolver(w.built.layout, precision="fp32c")
    assert np.array_equal(gpu.run(w.signal), OracleSolver(w.built.layout, "fp32c").run(w.signal))


@pytest.mark.gpu
def test_gpu_compensated_refuses_the_gradient():
    from acoustic_spaces_b200 import B200WaveSolver

    layout, signal, _ = load_golden("resonant7")
    gpu = B200WaveSolver(layout, precision="fp32c")
    with pytest.raises(ValueError, match="compensated"):
        gpu.gradient(signal[:50], np.zeros((gpu.probes, 50)))
