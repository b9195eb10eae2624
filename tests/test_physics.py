"""Known answers of the scheme itself, independent of the reference's code: a rigid box rings at
its room modes (the reference's tests/test_wave.py:263-284 checks its own solver the same way), and
the matched layer takes a pulse's energy out of an open grid far better than the grid's edge alone.

On the oracle (CPU) and on the B200 (gpu): both step the builder's layouts, so the answers pin the
layouts as well as the stepping.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from acoustic_spaces_b200 import layouts as L
from oracle.oracle import OracleSolver

C = 343.0
SIZE = (2.0, 1.5, 1.0)
MODES = ((1, 0, 0), (0, 1, 0), (1, 1, 0))


def _rigid_box(cell: float = 0.1):
    rate = C / (L.COURANT * cell)
    room = L.shoebox(np.asarray(SIZE), [L.Material(0.0)] * 6)
    built = L.cell_face_layout(room, L.room_grid(np.asarray(SIZE), cell), (0.33, 0.27, 0.33), [(1.67, 1.21, 0.67)],
                               rate=rate)  # fmt: skip
    return built, rate


def _mode_peaks(pressure: np.ndarray, rate: float) -> list[tuple[float, float]]:
    n_fft = 1 << 18
    spectrum = np.abs(np.fft.rfft(pressure, n_fft))
    f = np.fft.rfftfreq(n_fft, 1.0 / rate)
    out = []
    for mode in MODES:
        expected = C / 2 * math.hypot(*(m / s for m, s in zip(mode, SIZE)))
        near = (f > expected - 4) & (f < expected + 4)
        out.append((float(f[near][np.argmax(spectrum[near])]), expected))
    return out


def _check(run):
    built, rate = _rigid_box()
    assert built.air_cells == 20 * 15 * 10
    steps = int(4 * rate)
    pressure = run(built.layout, L.ricker_drive(rate, steps))[0]
    for peak, expected in _mode_peaks(pressure, rate):
        assert peak == pytest.approx(expected, abs=0.6), (peak, expected)


def test_a_rigid_box_rings_at_its_modes():
    _check(lambda layout, signal: OracleSolver(layout).run(signal))


def _open_pulse_energy(run, layer: int = 8) -> tuple[float, float]:
    # An open grid of air (no walls) with a matched layer of ``layer`` cells on every side (0: the
    # grid's edge alone, an admittance of 1): a pulse's pressure at a probe, its energy while the
    # pulse passes against what is left long after.
    cell = 0.1
    rate = C / (L.COURANT * cell)
    box = (3.0, 3.0, 3.0)
    room = L.Room(np.zeros((0, 3)), np.zeros(0), [])
    grid = L.Grid(-L.OFFSET * cell, cell, tuple(int(round(b / cell)) for b in box))
    built = L.cell_face_layout(room, grid, (1.5, 1.5, 1.5), [(1.9, 1.6, 1.4)], layer=layer,
                               layer_damping=0.5 if layer else 0.0, rate=rate)  # fmt: skip
    steps = 2000
    p = run(built.layout, L.ricker_drive(rate, steps))[0]
    return float(np.sum(p[:300] ** 2)), float(np.sum(p[1000:] ** 2))


def _layer_against_edge(run):
    # The layer leaves a hundred times less of the pulse than the grid's edge alone does.
    passing, left = _open_pulse_energy(run)
    bare_passing, bare_left = _open_pulse_energy(run, layer=0)
    assert passing > 0.0 and bare_passing > 0.0
    assert left / passing < 1e-2 * (bare_left / bare_passing), (left / passing, bare_left / bare_passing)


def test_the_matched_layer_absorbs_a_pulse():
    _layer_against_edge(lambda layout, signal: OracleSolver(layout).run(signal))


@pytest.mark.gpu
def test_gpu_a_rigid_box_rings_at_its_modes():
    from acoustic_spaces_b200 import B200WaveSolver

    _check(lambda layout, signal: B200WaveSolver(layout).run(signal))


@pytest.mark.gpu
def test_gpu_the_matched_layer_absorbs_a_pulse():
    from acoustic_spaces_b200 import B200WaveSolver

    _layer_against_edge(lambda layout, signal: B200WaveSolver(layout).run(signal))
