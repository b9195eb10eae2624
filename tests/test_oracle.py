"""The oracle pinned: the C restatement of WaveSolver::run against the reference's own numbers.

- against the golden fixtures (the reference's run() on its own layouts, stored by
  tests/golden/make_golden.py): bit for bit, also when run in pieces;
- against the reference compiled from its unmodified headers, live, on drives the fixtures do not
  hold (where the reference sources are present);
- its FP64 instantiation close to FP32, as rounding alone allows.
"""

from __future__ import annotations

import hashlib
import json

import numpy as np
import pytest
from conftest import GOLDEN, golden_names, load_golden

from oracle.oracle import OracleSolver

NAMES = golden_names()


@pytest.mark.parametrize("name", NAMES)
def test_golden_fixture_is_the_manifests(name):
    layout, signal, reference = load_golden(name)
    entry = json.loads((GOLDEN / "manifest.json").read_text())[name]
    assert hashlib.sha256(reference.tobytes()).hexdigest() == entry["reference_sha256"]
    assert reference.shape == (entry["probes"], entry["steps"]) == (len(layout["probe_start"]) - 1, len(signal))
    assert np.abs(reference).max() > 0.0


@pytest.mark.parametrize("name", NAMES)
def test_oracle_steps_every_golden_grid_as_the_reference_does(name):
    layout, signal, reference = load_golden(name)
    oracle = OracleSolver(layout)
    assert np.array_equal(oracle.run(signal), reference)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_runs_in_pieces_as_one_run(name):
    # Pieces of odd and even lengths, so the levels swap both ways between runs
    # (tests/test_gpu.py:45-54 of the reference).
    layout, signal, reference = load_golden(name)
    oracle = OracleSolver(layout)
    cuts = [0, 1, 78, 177, len(signal)]
    pieces = [oracle.run(signal[a:b]) for a, b in zip(cuts[:-1], cuts[1:])]
    assert np.array_equal(np.concatenate(pieces, axis=1), reference)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reset_silences_the_grid(name):
    layout, signal, reference = load_golden(name)
    oracle = OracleSolver(layout)
    oracle.run(signal[:50])
    oracle.reset()
    assert np.array_equal(oracle.run(signal), reference)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_fp64_differs_from_fp32_by_rounding_only(name):
    layout, signal, reference = load_golden(name)
    # Closed boxes with a speed field stray most: their uniform pressure's eigenvalue is not 0
    # in single precision (2 - total s and s axial each rounded to a float, fdtd.hpp:198-202):
    # 1.0e-3 of the peak after 400 steps at a uniform 0.99 (no branches to damp it), 5e-5 with the
    # graded fields; the others stay within 6e-6.
    fp64 = OracleSolver(layout, "fp64").run(signal)
    bound = {"uniform099": 2e-3, "speed7": 1e-4, "speed19": 1e-4}.get(name, 2e-5)
    assert np.abs(fp64 - reference).max() <= bound * np.abs(reference).max()


def test_an_empty_run_changes_nothing():
    layout, signal, reference = load_golden("resonant7")
    oracle = OracleSolver(layout)
    assert oracle.run(signal[:0]).shape == (len(layout["probe_start"]) - 1, 0)
    assert np.array_equal(oracle.run(signal), reference)


def test_the_oracle_refuses_moving_air():
    layout, _, _ = load_golden("resonant7")
    layout = dict(layout, flow_mask=np.ones(3, np.uint8))
    with pytest.raises(ValueError, match="moving air"):
        OracleSolver(layout)


# ---- live against the reference (development container only) --------------------------------

cases = pytest.importorskip("cases")


def _live(name: str, seed: int):
    if not cases.available():
        pytest.skip("the reference sources are not here")
    solver, signal = cases.build_case(name)
    signal = np.random.default_rng(seed).standard_normal(len(signal)).astype(np.float32) * 0.5
    return solver, signal


@pytest.mark.parametrize("name", ["resonant7", "resonant19", "speed19", "open_layer_speed", "fitted_closed", "fitted_open"])
def test_oracle_matches_the_reference_live_on_new_drives(name):
    solver, signal = _live(name, seed=1234)
    layout = solver.layout()
    oracle = OracleSolver(layout)
    reference = np.concatenate([solver.run(signal[:101]), solver.run(signal[101:])], axis=1)
    assert np.array_equal(oracle.run(signal), reference)


@pytest.mark.parametrize("precision", ["fp32", "fp64", "fp32c"])
def test_the_oracle_steps_alike_on_one_thread_and_on_many(precision, monkeypatch):
    # Large grids split their cells, rows and layer cells across host threads with one barrier a
    # step: the probes and the whole state equal a single thread's, bit for bit.
    from acoustic_spaces_b200 import layouts as L

    w = L.polyhedral_room(0, cell=0.2, steps=150)
    runs = {}
    for threads in ("1", "5"):
        monkeypatch.setenv("ORACLE_THREADS", threads)
        solver = OracleSolver(w.built.layout, precision)
        runs[threads] = (solver.run(w.signal[:77]), solver.run(w.signal[77:]), solver.state())
    one, many = runs["1"], runs["5"]
    assert np.array_equal(one[0], many[0]) and np.array_equal(one[1], many[1])
    for key in one[2]:
        assert np.array_equal(one[2][key], many[2][key]), key
