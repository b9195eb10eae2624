"""Small grids laid out by the reference's own C++ solver, for parity checks.

Each builder follows a construction of the reference's tests (file:line below) and returns a fresh
``acoustic_spaces._native.WaveSolver`` (the reference, compiled from its unmodified headers by
``oracle/Makefile``) and a drive signal. They need the reference's Python sources, so they run in
the development container only; ``tests/golden/make_golden.py`` stores their layouts and the
reference's outputs as fixtures for machines without them.
"""

from __future__ import annotations

import math

import numpy as np

from oracle.oracle import REFERENCE, reference_native, reference_python

C = 343.0
OFFSET = np.array([0.0137, 0.0219, 0.0291])  # tests/test_fitted_walls.py:41


def available() -> bool:
    return reference_python() is not None


def _modules():
    reference_python()
    from acoustic_spaces.engine import impedance, wave
    from acoustic_spaces.geometry import box_mesh

    return reference_native(), impedance, wave, box_mesh


def _courant(stencil: int) -> float:
    _, _, wave, _ = _modules()
    return wave.COURANT if stencil == 7 else wave.ISOTROPIC_COURANT


def drive(rate: float, cell: float, steps: int, stencil: int = 7) -> np.ndarray:
    """The source's term per step as wave_responses gives it (tests/test_wave.py:140-146)."""
    _, _, wave, _ = _modules()
    signal, _ = wave.source_signal(rate, cell, _courant(stencil))
    out = np.zeros(steps, np.float32)
    out[: len(signal)] = signal[:steps]
    return out


def noise(steps: int, seed: int) -> np.ndarray:
    """A seeded white drive: every step's source term different."""
    return np.random.default_rng(seed).standard_normal(steps).astype(np.float32)


def spread_points(low, high, count: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).uniform(low, high, (count, 3))


def box_solver(size, cell, stencil, *, branches=True, speed=None, probes=24, beta=0.02, seed=5):
    """A box room from the origin to ``size`` on the grid of tests/test_wave.py:59-107 (origin
    2 cells and a fraction off, shape 2 cells beyond), three faces resonant (the branches of
    fit_admittance([0.1, 0.3, 0.6], 8, rate), tests/test_wave.py:515-535), ``probes`` points
    spread through it; ``speed(centres)`` gives each cell's speed ratio."""
    native, impedance, _, box_mesh = _modules()
    mesh = box_mesh(size)
    bvh = native.Bvh(mesh.vertices, mesh.faces)
    origin = -cell * (2.0 + OFFSET)
    shape = np.ceil((np.array(size) - origin) / cell).astype(int) + 2
    rate = C / (_courant(stencil) * cell)
    beta_arr = np.full(len(mesh.faces), beta)
    rows, owners = [np.zeros((0, 3))], [np.zeros(0, np.int64)]
    if branches:
        fit = impedance.fit_admittance([0.1, 0.3, 0.6], 8, rate)
        for face in (0, 3, 5):
            beta_arr[face] += fit.beta
            rows.append(fit.branches(rate))
            owners.append(np.full(len(fit.conductance), face, np.int64))
    speeds = None
    if speed is not None:
        x, y, z = (origin[a] + (np.arange(shape[a]) + 0.5) * cell for a in range(3))
        zz, yy, xx = np.meshgrid(z, y, x, indexing="ij")
        centres = np.column_stack([xx.reshape(-1), yy.reshape(-1), zz.reshape(-1)])
        speeds = np.ascontiguousarray(speed(centres), dtype=np.float32)
    size = np.asarray(size, float)
    points = spread_points(0.1 * size, 0.9 * size, probes, seed)
    source = np.array([0.31, 0.43, 0.27]) * size
    solver = native.WaveSolver(
        bvh,
        np.arange(len(mesh.faces), dtype=np.int64),
        beta_arr,
        np.ascontiguousarray(np.vstack(rows)),
        np.concatenate(owners),
        origin,
        cell,
        *map(int, shape),
        source,
        points,
        threads=1,
        stencil=stencil,
        speed=speeds,
    )
    return solver, rate


def open_ground(h=0.3, speed=None, probes=6, flow=None, screen=False):
    """A 5 m x 4 m ground in the open, its grid ringed by the matched layer (8 cells, damping
    0.5): tests/test_gpu.py:87-110. ``flow(centres)`` gives the air's motion (cells per step along
    x and y, tests/test_wave.py:123-133); ``screen`` stands a 1.5 m wall across y at x = 2.6 m on
    the ground, which the wind must go round."""
    native, _, wave, _ = _modules()
    vertices = np.array([[0, 0, 0], [5, 0, 0], [5, 4, 0], [0, 4, 0]], float)
    faces = np.array([[0, 1, 2], [0, 2, 3]], np.int64)
    if screen:
        wall = np.array([[2.6, 1.0, 0.0], [2.6, 3.0, 0.0], [2.6, 3.0, 1.5], [2.6, 1.0, 1.5]], float)
        faces = np.vstack([faces, np.array([[4, 5, 6], [4, 6, 7]], np.int64)])
        vertices = np.vstack([vertices, wall])
    bvh = native.Bvh(vertices, faces)
    source = np.array([2.0, 2.0, 1.5])
    listeners = np.vstack(
        [np.array([[4.0, 3.0, 1.2], [1.0, 1.0, 0.6]]), spread_points([0.5, 0.5, 0.3], [4.5, 3.5, 2.0], probes - 2, 11)]
    )
    points = np.vstack([source, listeners])
    low = np.minimum(vertices.min(0), points.min(0) - 2 * h) - h * (2.0 + wave.LAYER_CELLS)
    high = np.maximum(vertices.max(0), points.max(0) + 2 * h)
    shape = np.ceil((high - low) / h).astype(int) + 2 + wave.LAYER_CELLS
    origin = low + OFFSET * h
    speeds = None
    if speed is not None:
        x, y, z = (origin[a] + (np.arange(shape[a]) + 0.5) * h for a in range(3))
        zz, yy, xx = np.meshgrid(z, y, x, indexing="ij")
        centres = np.column_stack([xx.reshape(-1), yy.reshape(-1), zz.reshape(-1)])
        speeds = np.ascontiguousarray(speed(centres), dtype=np.float32)
    flows = {}
    if flow is not None:
        x, y, z = (origin[a] + (np.arange(shape[a]) + 0.5) * h for a in range(3))
        zz, yy, xx = np.meshgrid(z, y, x, indexing="ij")
        fx, fy = flow(np.column_stack([xx.reshape(-1), yy.reshape(-1), zz.reshape(-1)]))
        flows = {"flow_x": np.ascontiguousarray(fx, np.float32), "flow_y": np.ascontiguousarray(fy, np.float32)}
    solver = native.WaveSolver(
        bvh,
        np.zeros(len(faces), np.int64),
        np.array([0.05]),
        np.zeros((0, 3)),
        np.zeros(0, np.int64),
        origin,
        h,
        *map(int, shape),
        source,
        listeners,
        layer=wave.LAYER_CELLS,
        layer_damping=wave.LAYER_DAMPING,
        threads=1,
        speed=speeds,
        **flows,
    )
    return solver, C / (wave.COURANT * h)


def _wind(centres):
    """A wind along +x and a little along -y, stronger with height: 0.12 + 0.04 z cells a step along x,
    -0.03 along y (each below half a cell a step)."""
    z = np.maximum(centres[:, 2], 0.0)
    return 0.12 + 0.04 * np.minimum(z, 2.0), np.full(len(centres), -0.03)


def _uniform_wind(centres):
    return np.full(len(centres), 0.2), np.full(len(centres), 0.07)


# ---- the L-room of tests/test_fitted_walls.py:280-300, with fitted walls ----------------------


def _turned(v, degrees, axis=2):
    about = v.mean(axis=0)
    t = math.radians(degrees)
    c, s = math.cos(t), math.sin(t)
    a, b = (axis + 1) % 3, (axis + 2) % 3
    out = v - about
    x, y = out[:, a].copy(), out[:, b].copy()
    out[:, a], out[:, b] = c * x - s * y, s * x + c * y
    return out + about


def l_room():
    """An L-shaped room 1.2 x 0.9 m in plan and 0.6 m high with two turned free plates, on a grid
    of h = 0.1 m (tests/test_fitted_walls.py:280-300)."""
    h = 0.1
    plan = np.array([(0, 0), (1.2, 0), (1.2, 0.5), (0.6, 0.5), (0.6, 0.9), (0, 0.9)])
    n = len(plan)
    v = np.array([(x, y, z) for z in (0.0, 0.6) for x, y in plan])
    f = [(0, k + 1, k) for k in range(1, n - 1)]
    f += [(n, n + k, n + k + 1) for k in range(1, n - 1)]
    for k in range(n):
        a, b = k, (k + 1) % n
        f += [(a, b, n + b), (a, n + b, n + a)]
    room_v, room_f = v, np.array(f, np.int64)
    quad = np.array([[0, 1, 2], [0, 2, 3]], np.int64)
    p1 = np.array([(0.2, 0.2, 0.15), (0.5, 0.2, 0.15), (0.5, 0.2, 0.45), (0.2, 0.2, 0.45)], float)
    p2 = np.array([(0.8, 0.1, 0.1), (1.05, 0.1, 0.1), (1.05, 0.1, 0.4), (0.8, 0.1, 0.4)], float)
    p1 = _turned(_turned(p1, 22.5), 11, axis=0)
    p2 = _turned(_turned(p2, 11), 22.5, axis=0)
    verts = np.vstack([room_v, p1, p2])
    faces = np.vstack([room_f, quad + len(room_v), quad + len(room_v) + 4])
    mat = np.r_[np.zeros(len(room_f)), [1, 1, 2, 2]].astype(np.int64)
    origin = room_v.min(axis=0) - h * (2 + OFFSET)
    shape = np.ceil((room_v.max(axis=0) - origin) / h).astype(int) + 2
    return verts, faces, mat, h, origin, shape, np.array([0.31, 0.62, 0.33])


def l_room_points(count=24, seed=3):
    """Points spread through the L-room's air (tests/test_fitted_walls.py:1806-1810)."""
    rng = np.random.default_rng(seed)
    points = rng.uniform([0.05, 0.05, 0.05], [1.15, 0.85, 0.55], (4 * count, 3))
    return points[~((points[:, 0] > 0.6) & (points[:, 1] > 0.5))][:count]


def _fitted(v, f, h, origin, shape, src, probes, mat, beta, branches=(), layer=0, damping=0.0):
    native, _, _, _ = _modules()
    rows = [np.zeros((0, 3))] + [np.asarray(r, float) for _, r in branches]
    owners = [np.zeros(0, np.int64)] + [np.full(len(r), m, np.int64) for m, r in branches]
    v = np.ascontiguousarray(v, float)
    f = np.ascontiguousarray(f, np.int64)
    return native.WaveSolver(
        native.Bvh(v, f),
        np.asarray(mat, np.int64),
        np.asarray(beta, float),
        np.ascontiguousarray(np.vstack(rows)),
        np.concatenate(owners),
        np.asarray(origin, float),
        float(h),
        *(int(n) for n in shape),
        np.asarray(src, float),
        np.asarray(probes, float).reshape(-1, 3),
        edge_admittance=1.0,
        layer=layer,
        layer_damping=damping,
        threads=1,
        fitted_walls=True,
        vertices=v,
        faces=f,
    )


def fitted_closed():
    """The L-room closed, its walls and one plate resonant (tests/test_gpu.py:420-441)."""
    _, impedance, wave, _ = _modules()
    v, f, mat, h, origin, shape, src = l_room()
    rate = C / (wave.COURANT * h)
    wall = impedance.Admittance(0.05, np.array([0.6, 0.3]), np.array([2.0, 1.5]), np.array([100.0, 250.0]))
    branches = [(0, wall.branches(rate)), (2, wall.branches(rate))]
    solver = _fitted(v, f, h, origin, shape, src, l_room_points(), mat, (wall.beta, 0.3, wall.beta), branches)
    return solver, rate


def fitted_open():
    """The L-room open through its missing ceiling to a 4-cell matched layer
    (tests/test_fitted_walls.py:1822-1839)."""
    _, _, wave, _ = _modules()
    v, f, mat, h, origin, shape, src = l_room()
    keep = np.r_[0:4, 8 : len(f)]
    room_v = v[:12]
    origin = room_v.min(axis=0) - h * (6.0 + OFFSET)
    shape = np.ceil((room_v.max(axis=0) - origin) / h).astype(int) + 6
    solver = _fitted(v, f[keep], h, origin, shape, src, l_room_points(), mat[keep], (0.0, 0.0, 0.0), layer=4, damping=0.5)
    return solver, C / (wave.COURANT * h)


def _gradient(centres):
    """A speed ratio falling with height and varying along x: every cell's scale different."""
    z = centres[:, 2]
    x = centres[:, 0]
    return np.clip(1.0 - 0.03 * np.maximum(z, 0.0) - 0.01 * np.sin(x), 0.5, 1.0)


#: name -> (builder of (solver, rate), steps, drive kind)
CASES = {
    "resonant7": (lambda: box_solver((1.2, 0.9, 0.7), 0.1, 7), 400, "noise"),
    "resonant19": (lambda: box_solver((1.2, 0.9, 0.7), 0.1, 19), 400, "noise"),
    "drive7": (lambda: box_solver((2.0, 1.5, 1.1), 0.1, 7, probes=8), 600, "drive"),
    "speed7": (lambda: box_solver((1.2, 0.9, 0.7), 0.1, 7, speed=_gradient), 400, "noise"),
    "speed19": (lambda: box_solver((1.2, 0.9, 0.7), 0.1, 19, speed=_gradient), 400, "noise"),
    "uniform099": (lambda: box_solver((1.2, 0.9, 0.7), 0.1, 7, branches=False, speed=lambda c: np.full(len(c), 0.99)), 400, "drive"),
    "open_layer": (lambda: open_ground(), 600, "drive"),
    "open_layer_speed": (lambda: open_ground(speed=_gradient), 500, "noise"),
    "fitted_closed": (fitted_closed, 400, "drive"),
    "fitted_open": (fitted_open, 400, "noise"),
    "wind_plain": (lambda: open_ground(flow=_uniform_wind), 400, "drive"),
    "wind_round": (lambda: open_ground(flow=_wind, screen=True), 400, "noise"),
}


def build_case(name: str):
    """(solver, signal) of the named case: a fresh reference solver and its drive."""
    make, steps, kind = CASES[name]
    solver, rate = make()
    layout = solver.layout()
    cell = None
    if kind == "drive":
        # the cell size back from the layout's grid: rate = c / (L h)
        stencil = int(layout["stencil"][0])
        cell = C / (_courant(stencil) * rate)
        signal = drive(rate, cell, steps, stencil)
    else:
        signal = noise(steps, seed=len(name))
    return solver, signal
