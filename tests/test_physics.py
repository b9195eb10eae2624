"""Known answers of the scheme itself, independent of the reference's code: room modes, the
scheme's own dispersion (both stencils), a wall's reflection, the stability margin of the update's constants, what
the matched layer takes out of a pulse, and a speed field of ones.

On the oracle (CPU) and, where marked, on the B200: both step the builder's layouts, so the answers
pin the layouts as well as the stepping.
"""

from __future__ import annotations

import itertools
import math

import numpy as np
import pytest

from acoustic_spaces_b200 import layouts as L
from oracle.oracle import OracleSolver

C = 343.0


def _peak(series: np.ndarray, rate: float, around: float, half_width: float) -> float:
    """The frequency of the strongest spectral line of ``series`` within ``half_width`` Hz of
    ``around``: a Blackman-windowed, zero-padded transform, its largest bin there refined by the
    parabola through the log magnitudes of that bin and its two neighbours."""
    n = 1 << max(18, int(math.ceil(math.log2(len(series)))) + 3)
    spectrum = np.abs(np.fft.rfft(series * np.blackman(len(series)), n))
    step = rate / n
    lo, hi = int((around - half_width) / step), int((around + half_width) / step) + 1
    k = lo + int(np.argmax(spectrum[lo:hi]))
    a, b, c = np.log(spectrum[k - 1 : k + 2] + 1e-300)
    return (k + 0.5 * (a - c) / (a - 2 * b + c)) * step


# ---- a rigid box's modes ---------------------------------------------------------------------

BOX = (2.0, 1.5, 1.0)


def _rigid_box(cell: float = 0.1):
    rate = C / (L.COURANT * cell)
    room = L.shoebox(np.asarray(BOX), [L.Material(0.0)] * 6)
    built = L.cell_face_layout(room, L.room_grid(np.asarray(BOX), cell), (0.33, 0.27, 0.33), [(1.67, 1.21, 0.67)],
                               rate=rate)  # fmt: skip
    return built, rate


def _lowest_modes(count: int) -> list[tuple[tuple[int, int, int], float]]:
    """The box's lowest ``count`` modes above 0 Hz: C/2 sqrt((l/X)^2 + (m/Y)^2 + (n/Z)^2)."""
    modes = [(lmn, C / 2 * math.sqrt(sum((q / s) ** 2 for q, s in zip(lmn, BOX))))
             for lmn in itertools.product(range(4), repeat=3) if any(lmn)]  # fmt: skip
    return sorted(modes, key=lambda m: m[1])[:count]


def _check_modes(run):
    built, rate = _rigid_box()
    assert built.air_cells == 20 * 15 * 10
    response = run(built.layout, L.ricker_drive(rate, int(4 * rate)))[0]
    modes = _lowest_modes(3)
    assert [m[0] for m in modes] == [(1, 0, 0), (0, 1, 0), (1, 1, 0)]
    for lmn, expected in modes:
        # (the 10 cm grid's dispersion puts them a tenth of a hertz low)
        assert abs(_peak(response, rate, expected, 3.0) - expected) < 0.5, lmn


def test_a_rigid_box_rings_at_its_modes():
    _check_modes(lambda layout, signal: OracleSolver(layout).run(signal))


@pytest.mark.gpu
def test_gpu_a_rigid_box_rings_at_its_modes():
    from acoustic_spaces_b200 import B200WaveSolver

    _check_modes(lambda layout, signal: B200WaveSolver(layout).run(signal))


# ---- the scheme's own dispersion -------------------------------------------------------------


def test_a_tubes_modes_sit_at_the_schemes_own_frequencies():
    # The axial modes of a rigid 6 m tube at 10 cm (cross-section 0.4 m, its first cross mode at
    # 429 Hz, above those tested) at 20, 16 and 12 cells per wavelength: each where the 7-point
    # leapfrog puts a plane wave along an axis, sin(w dt / 2) = sqrt(a) sin(k h / 2) with a the
    # layout's (lowered) axial weight, to 1e-6; below the tube's continuous mode by 0.3-0.8 %.
    size, h = np.array([6.0, 0.4, 0.4]), 0.1
    rate = C / (L.COURANT * h)
    room = L.shoebox(size, [L.Material(0.0)] * 6)
    built = L.cell_face_layout(room, L.room_grid(size, h), (0.27, 0.2, 0.2), [(5.73, 0.2, 0.2)], rate=rate)
    a = float(np.asarray(built.layout["weights"], np.float32)[0])
    response = OracleSolver(built.layout, "fp64").run(L.ricker_drive(rate, int(3 * rate), sigma_s=0.25e-3))[0]
    spacing = C / (2 * size[0])
    for per_wavelength in (20, 16, 12):
        m = round(2 * size[0] / (per_wavelength * h))
        scheme = rate / math.pi * math.asin(math.sqrt(a) * math.sin(math.pi * m * h / (2 * size[0])))
        assert _peak(response, rate, scheme, 0.3 * spacing) == pytest.approx(scheme, rel=1e-6), per_wavelength
        assert 0.002 < 1 - scheme / (m * spacing) < 0.01


def test_a_slower_speed_of_sound_moves_the_tubes_modes_as_the_scheme_says():
    # The rigid tube with a speed ratio of 0.9 and of 0.6 in every cell (each interior cell's update
    # scaled by s, the ratio squared): its axial modes sit at sin(w dt / 2) = sqrt(s a) sin(k h / 2)
    # to 1e-5 (measured: 4e-7 to 1.6e-6), in cycles a step, 10 % and 40 % below the plain tube's.
    size, h = np.array([6.0, 0.4, 0.4]), 0.1
    room = L.shoebox(size, [L.Material(0.0)] * 6)
    for speed in (0.9, 0.6):
        built = L.cell_face_layout(room, L.room_grid(size, h), (0.27, 0.2, 0.2), [(5.73, 0.2, 0.2)], speed=speed)
        layout = built.layout
        a = float(np.asarray(layout["weights"], np.float64)[0])
        s = float(np.asarray(layout["scale"], np.float64)[np.asarray(layout["types"]) == 1][0])
        assert s == pytest.approx(speed**2, rel=1e-6)
        response = OracleSolver(layout, "fp64").run(L.ricker_drive(1.0, 20000, sigma_s=1.2))[0]
        for per_wavelength in (20, 16, 12):
            m = round(2 * size[0] / (per_wavelength * h))
            scheme = math.asin(math.sqrt(s * a) * math.sin(math.pi * m * h / (2 * size[0]))) / math.pi
            got = _peak(response, 1.0, scheme, 0.3 * scheme / m)
            assert got == pytest.approx(scheme, rel=1e-5), (speed, per_wavelength)


def test_the_19_point_stencils_tube_modes_sit_at_its_own_frequencies():
    # The same rigid 6 m tube laid out by the reference itself (a box of twelve triangles) with the
    # 19-point stencil, stepped by the FP64 oracle: a plane wave along an axis sees
    # sin(w dt / 2) = sqrt(a + 4 d) sin(k h / 2), a and d the layout's face and edge weights (the
    # faces across the wave add 4 a and its edges 8 d cos(k h) + 4 d), so each axial mode sits there
    # to 1e-6 (measured: 3e-9), in cycles a step; the 7-point layout of the same tube, likewise
    # with d = 0.
    from oracle.oracle import reference_native

    native = reference_native()
    if native is None:
        pytest.skip("the reference's solver is not built")
    size, h = np.array([6.0, 0.4, 0.4]), 0.1
    grid = L.room_grid(size, h)
    corners = np.array([[x, y, z] for z in (0, size[2]) for y in (0, size[1]) for x in (0, size[0])], float)
    quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    triangles = np.array([t for a, b, c, d in quads for t in ([a, b, c], [a, c, d])], np.int64)
    for stencil in (7, 19):
        solver = native.WaveSolver(
            native.Bvh(corners, triangles), np.zeros(12, np.int64), np.array([0.0]), np.zeros((0, 3)),
            np.zeros(0, np.int64), grid.origin, grid.cell, *grid.shape, np.array([0.27, 0.2, 0.2]),
            np.array([[5.73, 0.2, 0.2]]), threads=2, stencil=stencil,
        )  # fmt: skip
        layout = solver.layout()
        w = np.asarray(layout["weights"], np.float64)
        a, d = float(w[0]), (float(w[6]) if stencil == 19 else 0.0)
        response = OracleSolver(layout, "fp64").run(L.ricker_drive(1.0, 20000, sigma_s=1.2))[0]
        for per_wavelength in (20, 16, 12):
            m = round(2 * size[0] / (per_wavelength * h))
            scheme = math.asin(math.sqrt(a + 4 * d) * math.sin(math.pi * m * h / (2 * size[0]))) / math.pi
            got = _peak(response, 1.0, scheme, 0.3 * scheme / m)
            assert got == pytest.approx(scheme, rel=1e-6), (stencil, per_wavelength)


# ---- a wall's reflection -----------------------------------------------------------------------


@pytest.mark.parametrize("beta", [0.0, 0.1, 0.3, 0.5, 1.0])
def test_a_duct_end_reflects_as_its_admittance_says(beta):
    # A plane wave down an 80 m duct whose near end absorbs (admittance 1): the pulse that comes
    # back from the far end, of admittance beta, against the one that passed, each cut out of the
    # response by a Tukey gate round its arrival. Below the duct's cross modes the ratio of their
    # spectra is the grid's reflection factor: (1 - beta) / (1 + beta), normal incidence on a
    # locally reacting wall, plus a discretisation term that grows with frequency (at 10 cm, 0.08
    # at 180 Hz for an absorbing end). A quadratic through the ratio over 40-200 Hz meets the
    # continuous factor at 0 Hz to 1e-3; a rigid end reflects all of it at every frequency (to 1e-4,
    # what the gates leave).
    from scipy.signal.windows import tukey

    size, cell = np.array([80.0, 0.6, 0.6]), 0.1
    rate = C / (L.COURANT * cell)
    room = L.shoebox(size, [L.Material(b) for b in (1.0, beta, 0.0, 0.0, 0.0, 0.0)])  # -x near, +x far
    source, receiver = (10.0, 0.3, 0.3), (30.0, 0.3, 0.3)
    built = L.cell_face_layout(room, L.room_grid(size, cell), source, [receiver], rate=rate)
    steps, sigma = int(0.45 * rate), 1.5e-3
    # (a Ricker drive: a Gaussian's pressure would leave a plateau behind the passing front that
    # the reflected pulse's gate cuts into)
    response = OracleSolver(built.layout, "fp64").run(L.ricker_drive(rate, steps, sigma_s=sigma))[0]
    n = 1 << 14
    f = np.fft.rfftfreq(n, 1.0 / rate)
    band = (f >= 40.0) & (f <= 200.0)

    def spectrum(path: float) -> np.ndarray:
        centre = int(round((6 * sigma + path / C) * rate))
        width = int(0.06 * rate)
        gate = np.zeros(steps)
        gate[centre - width // 2 : centre - width // 2 + width] = tukey(width, 0.5)
        return np.abs(np.fft.rfft(response * gate, n))[band]

    ratio = spectrum((size[0] - source[0]) + (size[0] - receiver[0])) / spectrum(receiver[0] - source[0])
    expected = (1 - beta) / (1 + beta)
    assert np.polyfit(f[band], ratio, 2)[-1] == pytest.approx(expected, abs=1e-3)
    assert np.all(np.abs(ratio - expected) < (1e-4 if beta == 0 else 0.1))


# ---- the update's stability margin -------------------------------------------------------------


@pytest.mark.parametrize("stencil", [7, 19])
def test_the_update_keeps_its_highest_modes_inside_the_stability_limit(stencil):
    # On a mode that alternates in sign along some axes (s_a = -1) and is constant along the rest
    # (s_a = 1), the update is the two-step recurrence p+ = A p - p-, A = centre + 2 axial sum_a s_a
    # + 4 diagonal sum_{a<b} s_a s_b, whose roots stay on the unit circle while |A| <= 2. The
    # layout's weights are the exact ones times (1 - 2^-18): A is 2 for a constant pressure and at
    # least -2 + 2^-16 elsewhere. Stepped in single precision, a kicked mode then swings within
    # 1 / sin(acos(A / 2)) of its kick (256 at the margin) instead of growing.
    from conftest import load_golden

    layout = _rigid_box()[0].layout if stencil == 7 else load_golden("resonant19")[0]
    w = np.asarray(layout["weights"], np.float64)
    axial, diagonal = float(w[0]), (float(w[6]) if stencil == 19 else 0.0)
    centre = float(np.asarray(layout["centre"])[0])
    exact = (1.0 / 3.0, 0.0) if stencil == 7 else (0.25, 0.125)
    assert axial == pytest.approx(exact[0] * (1 - 2.0**-18), rel=2**-22)
    assert diagonal == pytest.approx(exact[1] * (1 - 2.0**-18), rel=2**-22)
    patterns = np.array(list(itertools.product((1.0, -1.0), repeat=3)))
    pair_sum = np.array([s[0] * s[1] + s[0] * s[2] + s[1] * s[2] for s in patterns])
    A = centre + 2 * axial * patterns.sum(axis=1) + 4 * diagonal * pair_sum
    assert A.max() == 2.0 and A.min() >= -2 + 2.0**-16
    # the kicked recurrence in float32, every sign pattern at once: six face neighbours, twelve
    # edge neighbours
    f32 = np.float32
    c32, a32, d32 = f32(centre), f32(axial), f32(diagonal)
    kick = np.random.default_rng(3).uniform(0.5, 2.0, len(patterns)).astype(f32)
    s = patterns.astype(f32)
    before, now = np.zeros_like(kick), kick.copy()
    worst = np.zeros_like(kick)
    for _ in range(20_000):
        axial_sum = np.zeros_like(now)
        for sign in (s[:, 0], s[:, 0], s[:, 1], s[:, 1], s[:, 2], s[:, 2]):
            axial_sum = axial_sum + sign * now
        edge_sum = np.zeros_like(now)
        for sign in [s[:, 0] * s[:, 1]] * 4 + [s[:, 0] * s[:, 2]] * 4 + [s[:, 1] * s[:, 2]] * 4:
            edge_sum = edge_sum + sign * now
        before, now = now, c32 * now + a32 * axial_sum + d32 * edge_sum - before
        np.maximum(worst, np.abs(now), out=worst)
    bound = 1.0 / np.sqrt(np.maximum(1e-12, 1.0 - (np.clip(A, -2, 2) / 2) ** 2))
    oscillating = np.abs(A) < 2.0
    assert np.all(worst[oscillating] / kick[oscillating] <= 1.1 * bound[oscillating])


# ---- the matched layer, and a speed field of ones ---------------------------------------------


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
