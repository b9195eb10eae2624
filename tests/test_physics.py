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


def _speed_runs(run):
    # An open convex room with resonant walls and a 4-cell matched layer, laid out with a speed
    # ratio of exactly 1 in every cell and with none.
    rng = np.random.default_rng(7)
    cell, box = 0.1, (4.0, 3.0, 2.4)
    rate = C / (L.COURANT * cell)

    def material(r):
        return L.Material(float(r.uniform(0.02, 0.1)),
                          L.resonant_branch(r.uniform(0.005, 0.5), r.uniform(0.5, 10.0), r.uniform(30.0, 300.0), rate))  # fmt: skip

    room = L.convex_room(rng, box, faces=12, margin=cell * (4 + 3), open_face=1, material=material)
    points = L.inside_points(rng, room, box, 3, 0.35, apart=0.35)
    grid = L.Grid(-L.OFFSET * cell, cell, tuple(int(round(b / cell)) for b in box))
    signal = L.gaussian_drive(rate, 400)
    out = []
    for speed in (1.0, None):
        built = L.cell_face_layout(room, grid, points[0], points[1:], layer=4, layer_damping=0.5, speed=speed, rate=rate)
        out.append(run(built.layout, signal))
    return out


def test_one_speed_everywhere_changes_nothing():
    # As the reference's tests/test_wave.py:2545 checks its own solver: the scaled update with every
    # cell at the grid's speed is the unscaled one, to the bit, walls and layer included.
    scaled, plain = _speed_runs(lambda layout, signal: OracleSolver(layout).run(signal))
    assert np.array_equal(scaled, plain)


@pytest.mark.gpu
def test_gpu_one_speed_everywhere_changes_nothing():
    from acoustic_spaces_b200 import B200WaveSolver

    scaled, plain = _speed_runs(lambda layout, signal: B200WaveSolver(layout).run(signal))
    assert np.array_equal(scaled, plain)


@pytest.mark.parametrize("stencil", [7, 19])
def test_the_update_keeps_its_highest_modes_inside_the_stability_limit(stencil):
    # The layout's constants (the reference's tests/test_wave.py:400-439): on a mode alternating
    # along some axes (signs c = +-1) the update is p+ = A p - p-; the weights are the exact ones
    # lowered by 2^-18, so that A stays 2^-16 inside -2, and in single precision a kicked
    # checkerboard swings within about 1 / (2 sqrt(2^-18)) = 256 times its kick rather than growing.
    import itertools

    from conftest import load_golden

    if stencil == 7:
        layout = _rigid_box()[0].layout
    else:
        layout = load_golden("resonant19")[0]
    axial = float(np.asarray(layout["weights"])[0])
    diagonal = float(np.asarray(layout["weights"])[6]) if stencil == 19 else 0.0
    centre = float(np.asarray(layout["centre"])[0])
    margin = 2.0**-18
    exact = (1 / 3, 0.0) if stencil == 7 else (0.25, 0.125)
    np.testing.assert_allclose([axial, diagonal], np.multiply(exact, 1 - margin), rtol=2**-22)
    c = np.array(list(itertools.product([1.0, -1.0], repeat=3)))
    pairs = c[:, 0] * c[:, 1] + c[:, 0] * c[:, 2] + c[:, 1] * c[:, 2]
    factors = centre + 2 * axial * c.sum(axis=1) + 4 * diagonal * pairs
    assert factors[0] == 2.0 and factors.min() >= -2 + 4 * margin
    f32 = np.float32
    kicks = np.random.default_rng(1).uniform(0.5, 2.0, 32).astype(f32)
    previous, current, peak = np.zeros_like(kicks), kicks.copy(), np.zeros_like(kicks)
    a, d, centre32 = f32(axial), f32(diagonal), f32(centre)
    for _ in range(20_000):
        p, q = current, -current
        if stencil == 7:
            following = centre32 * p + a * (q + q + q + q + q + q) - previous
        else:
            edges = q + q + q + q + q + q + q + q + p + p + p + p
            following = centre32 * p + a * (p + p + q + q + q + q) + d * edges - previous
        previous, current = current, following
        np.maximum(peak, np.abs(current), out=peak)
    assert np.max(peak / kicks) < 1.1 * 256


@pytest.mark.parametrize("beta", [0.0, 0.1, 0.5, 1.0])
def test_a_duct_end_reflects_as_its_admittance_says(beta):
    # As the reference's tests/test_wave.py:538-568: a plane wave down an 80 m duct whose near end
    # absorbs (admittance 1) reflects off the far end, of admittance beta, by (1 - beta) / (1 + beta)
    # at normal incidence — the incident and reflected waves, 40-200 Hz, gated by Hann windows.
    size = np.array([80.0, 0.6, 0.6])
    cell = 0.1
    rate = C / (L.COURANT * cell)
    betas = [1.0, beta, 0.0, 0.0, 0.0, 0.0]  # -x (near), +x (far), then the duct's sides
    room = L.shoebox(size, [L.Material(b) for b in betas])
    built = L.cell_face_layout(room, L.room_grid(size, cell), (10.0, 0.3, 0.3), [(30.0, 0.3, 0.3)], rate=rate)
    steps = int(0.45 * rate)
    pressure = OracleSolver(built.layout, "fp64").run(L.gaussian_drive(rate, steps))[0]
    delay = 6 * 0.5e-3 * rate  # the pulse's centre
    n_fft = 1 << 14
    f = np.fft.rfftfreq(n_fft, 1.0 / rate)
    gain = np.clip((f - 40) / 20, 0, 1) * np.clip((200 - f) / 50, 0, 1)
    pressure = np.fft.irfft(np.fft.rfft(pressure, n_fft) * gain, n_fft)[:steps]
    t = (np.arange(steps) - delay) / rate

    def gated(path: float) -> float:
        x = t - path / C
        window = np.where(np.abs(x) < 0.04, 0.5 + 0.5 * np.cos(np.pi * x / 0.04), 0.0)
        return float(np.sum((pressure * window) ** 2))

    reflection = math.sqrt(gated(120.0) / gated(20.0))
    assert reflection == pytest.approx((1 - beta) / (1 + beta), abs=0.005 if beta < 1 else 0.05)


def test_a_tubes_modes_sit_at_the_schemes_own_frequencies():
    # The axial modes of a rigid 6 m tube at 10 cm (cross-section 0.4 m, its first cross mode at
    # 429 Hz, above those tested) at 20, 16 and 12 cells per wavelength: each at the frequency the
    # 7-point leapfrog gives a plane wave along an axis, sin(w dt / 2) = sqrt(a) sin(k h / 2) with a
    # the layout's (lowered) axial weight, to 2e-5 (the reference's tests/test_wave.py:287-317 measures
    # its solver's dispersion the same way), and below the tube's own by that much.
    size, h = np.array([6.0, 0.4, 0.4]), 0.1
    rate = C / (L.COURANT * h)
    room = L.shoebox(size, [L.Material(0.0)] * 6)
    built = L.cell_face_layout(room, L.room_grid(size, h), (0.27, 0.2, 0.2), [(5.73, 0.2, 0.2)], rate=rate)
    a = float(np.asarray(built.layout["weights"], np.float32)[0])
    steps = int(3 * rate)
    pressure = OracleSolver(built.layout, "fp64").run(L.ricker_drive(rate, steps, sigma_s=0.25e-3))[0]
    n_fft = 1 << 20
    spectrum = np.abs(np.fft.rfft(pressure * np.hanning(len(pressure)), n_fft))
    f = np.fft.rfftfreq(n_fft, 1.0 / rate)
    spacing = C / (2 * size[0])
    for per_wavelength in (20, 16, 12):
        m = round(2 * size[0] / (per_wavelength * h))
        k = math.pi * m / size[0]
        scheme = rate / math.pi * math.asin(math.sqrt(a) * math.sin(k * h / 2))
        near = np.abs(f - scheme) < 0.4 * spacing
        peak = f[near][np.argmax(spectrum[near])]
        assert peak == pytest.approx(scheme, rel=2e-5), (per_wavelength, peak, scheme)
        assert scheme < m * spacing
