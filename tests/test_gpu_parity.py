"""Parity of the B200 stepper with the reference, through the C ABI (needs a B200).

FP32 is the reference's arithmetic operation for operation, so the bar is equality to the bit:
- the probes' series against the golden fixtures (the reference's own run() on its own layouts),
  run from rest in pieces of odd and even lengths;
- the whole state (both pressure levels, both branch-velocity sets, the matched layer's nine
  values per cell) against the oracle's after the same run;
FP64 against the oracle's FP64 instantiation: the same IEEE operations in the same order, so
equal to the bit as well.
"""

from __future__ import annotations

import numpy as np
import pytest
from conftest import golden_names, load_golden

from acoustic_spaces_b200 import B200WaveSolver
from oracle.oracle import OracleSolver

pytestmark = pytest.mark.gpu
NAMES = golden_names()


def _pieces(solver, signal, cuts):
    return np.concatenate([solver.run(signal[a:b]) for a, b in zip(cuts[:-1], cuts[1:])], axis=1)


@pytest.mark.parametrize("name", NAMES)
def test_gpu_steps_every_golden_grid_as_the_reference_does(name):
    layout, signal, reference = load_golden(name)
    gpu = B200WaveSolver(layout)
    got = _pieces(gpu, signal, [0, 177, 178, len(signal)])
    assert np.array_equal(got, reference), np.abs(got - reference).max()


@pytest.mark.parametrize("name", NAMES)
def test_gpu_state_equals_the_oracles(name):
    layout, signal, _ = load_golden(name)
    gpu = B200WaveSolver(layout)
    oracle = OracleSolver(layout)
    cuts = [0, 101, len(signal)]
    a = _pieces(gpu, signal, cuts)
    b = _pieces(oracle, signal, cuts)
    assert np.array_equal(a, b)
    sa, sb = gpu.state(), oracle.state()
    for key in sa:
        assert np.array_equal(sa[key], sb[key]), key


@pytest.mark.parametrize("name", NAMES)
def test_gpu_fp64_equals_the_fp64_oracle(name):
    layout, signal, reference = load_golden(name)
    gpu = B200WaveSolver(layout, precision="fp64")
    oracle = OracleSolver(layout, "fp64")
    a = _pieces(gpu, signal, [0, 77, len(signal)])
    b = oracle.run(signal)
    assert np.array_equal(a, b), np.abs(a - b).max() / np.abs(b).max()
    sa, sb = gpu.state(), oracle.state()
    for key in sa:
        assert np.array_equal(sa[key], sb[key]), key


@pytest.mark.parametrize("name", ["resonant7", "open_layer", "fitted_open"])
def test_gpu_reset_silences_the_grid(name):
    layout, signal, reference = load_golden(name)
    gpu = B200WaveSolver(layout)
    gpu.run(signal[:123])
    gpu.reset()
    assert gpu.info().steps_done == 0
    assert np.array_equal(gpu.run(signal), reference)


def test_gpu_two_solvers_are_independent():
    layout_a, signal_a, reference_a = load_golden("resonant19")
    layout_b, signal_b, reference_b = load_golden("open_layer_speed")
    a, b = B200WaveSolver(layout_a), B200WaveSolver(layout_b)
    got_a, got_b = [], []
    for lo, hi in [(0, 200), (200, 400)]:
        got_a.append(a.run(signal_a[lo:hi]))
        got_b.append(b.run(signal_b[lo:hi]))
    got_b.append(b.run(signal_b[400:]))
    assert np.array_equal(np.concatenate(got_a, axis=1), reference_a)
    assert np.array_equal(np.concatenate(got_b, axis=1), reference_b)


def test_gpu_info_counts_the_layout():
    layout, _, _ = load_golden("fitted_open")
    gpu = B200WaveSolver(layout)
    info = gpu.info()
    types = layout["types"]
    assert info.air_cells == int(np.count_nonzero(types))
    assert info.interior_cells == int(np.count_nonzero(types == 1))
    assert info.special_cells == len(layout["special"])
    assert info.layer_cells == len(layout["layer_cells"])
    assert info.probes == gpu.probes == len(layout["probe_start"]) - 1
