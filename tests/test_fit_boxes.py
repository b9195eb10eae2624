"""This library's fit on the convex cases of the reference's own golden fit fixtures.

The reference pins its exact fit by the bytes of every field of eleven small cases
(tests/test_fit_golden.py:1-120 of the reference; their inputs and expected hashes for the three
convex rooms, `room`, `fold` and `far`, are copied into tests/golden/fit_boxes.npz by
tests/golden/make_fit_boxes.py). Here:

* the reference's fit compiled here (oracle/_ref, its CutFit) gives those fields with the bytes the
  reference's fixtures expect: the checker is the reference's own fit, bit for bit;
* the walls of each mesh (``fitted.mesh_walls``) are its box's six planes, each cut into the two
  triangles of its face, with the triangles' own materials;
* on the GPU, this library's fit (``fdtd_cut_convex`` with the walls in pieces, then
  ``fitted.fit_from_cut``) equals the reference's: the same air, the same rows, and each row's air
  volume, open areas, wall area per material and slivers (in cells' volumes and faces) within what
  the meshes themselves allow. The fit takes each face of a box as one plane, while the reference
  clips by each triangle exactly, and no face is quite flat: `room`'s faces are flat to 2.5e-9 of a
  cell (measured error 3e-9, tolerance 1e-8); one face of `fold` is folded by 5e-7 of a cell
  (measured 8e-7, tolerance 1e-6); `far`, cells of 4 cm a thousand million metres from the origin,
  has its vertices rounded to the doubles there (steps of 1.2e-7 m), its faces flat to 4e-6 of a
  cell and its cells' faces at origin + i h rounded alike (measured 1.1e-5 on a row's wall area,
  the sum of several cells', tolerance 3e-5).
"""

from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from acoustic_spaces_b200 import fitted
from acoustic_spaces_b200 import layouts as L
from oracle import oracle

BOXES = Path(__file__).resolve().parent / "golden" / "fit_boxes.npz"
NAMES = ["room", "fold", "far"]
native = oracle.reference_native()
needs_reference = pytest.mark.skipif(native is None, reason="the reference's compiled fit (oracle/_ref) is absent")


def _case(name):
    with np.load(BOXES) as data:
        case = {k: data[f"{name}/{k}"] for k in ("vertices", "faces", "materials", "grid", "shape")}
        expected = json.loads(str(data["expected"]))[name]
    return case, expected


def _digest(value) -> str:
    """The reference fixtures' hash of an array: SHA-256 of its float64 (or int64) bytes and its
    shape, the first 24 hex digits."""
    a = np.asarray(value)
    a = a.astype(np.float64 if a.dtype.kind == "f" else np.int64)
    return hashlib.sha256(np.ascontiguousarray(a).tobytes() + str(a.shape).encode()).hexdigest()[:24]


def _reference(case):
    g = case["grid"]
    nx, ny, nz, materials = (int(x) for x in case["shape"])
    return native.CutFit(case["vertices"], case["faces"], case["materials"], materials, g[0:3], float(g[3]),
                         nx, ny, nz, g[4:7], layer=0, threads=2)  # fmt: skip


def _grid(case):
    g = case["grid"]
    return L.Grid(np.asarray(g[0:3], np.float64), float(g[3]), tuple(int(x) for x in case["shape"][:3]))


@needs_reference
@pytest.mark.parametrize("name", NAMES)
def test_the_checker_is_the_references_fit_to_the_byte(name):
    case, expected = _case(name)
    cut = _reference(case)
    got = {"air": _digest(cut.cut_air())}
    for key, value in cut.cut_cells().items():
        got[f"cells/{key}"] = _digest(value)
    for a, w in enumerate(cut.cut_widths()):
        got[f"widths/{a}"] = _digest(w)
    assert {k: got[k] for k in expected} == expected


@pytest.mark.parametrize("name", NAMES)
def test_the_walls_of_each_box_are_six_planes_of_two_triangles(name):
    case, _ = _case(name)
    walls = fitted.mesh_walls(case["vertices"], case["faces"], case["materials"], int(case["shape"][3]))
    # (`fold` has one face folded by 1e-7 m, taken as flat: a fit of half-spaces cannot follow
    # a fold into the room)
    assert len(walls.offsets) == 6 and not walls.open
    assert len(walls.piece_plane) == len(case["faces"]) == 12
    assert np.all(np.bincount(walls.piece_plane, minlength=6) == 2)
    assert np.array_equal(walls.column_material, case["materials"])
    # every vertex of a triangle inside its piece's edges, and the room inside every plane
    v = case["vertices"] - walls.anchor  # (the planes are taken from the anchor)
    edges = walls.piece_edges.reshape(-1, 4)
    for k, tri in enumerate(case["faces"]):
        for e in edges[walls.piece_start[k] : walls.piece_start[k + 1]]:
            assert np.all(v[tri] @ e[:3] - e[3] <= 1e-9 * max(1.0, np.abs(v).max()))
    # (within the fold of `fold`, and the rounding of `far`'s vertices to the doubles near 1e9 m)
    flat = 2e-6 if name == "far" else 1e-7
    assert np.all(v @ walls.normals.T - walls.offsets <= flat * max(1.0, np.abs(v).max()))


def test_a_mesh_that_is_not_convex_is_refused():
    # an L of two boxes: a triangle of the inner corner lies on no face of the hull
    case, _ = _case("room")
    v = np.array([(0, 0, 0), (2, 0, 0), (2, 1, 0), (1, 1, 0), (1, 2, 0), (0, 2, 0)], float)
    top = v + np.array([0, 0, 1.0])
    verts = np.vstack([v, top])
    faces = [(0, 2, 1), (0, 3, 2), (0, 5, 3), (3, 5, 4), (6, 7, 8), (6, 8, 9), (6, 9, 11), (9, 10, 11)]
    for a in range(6):
        b = (a + 1) % 6
        faces += [(a, b, b + 6), (a, b + 6, a + 6)]
    with pytest.raises(ValueError, match="not convex"):  # fmt: skip
        fitted.mesh_walls(verts, np.array(faces), np.zeros(len(faces), np.int64), 1)


@pytest.mark.gpu
@needs_reference
@pytest.mark.parametrize("name", NAMES)
def test_gpu_fit_of_the_golden_boxes_is_the_references(name):
    case, _ = _case(name)
    grid = _grid(case)
    walls = fitted.mesh_walls(case["vertices"], case["faces"], case["materials"], int(case["shape"][3]))
    ours = fitted.convex_fit(walls, grid)
    ref = _reference(case)
    cells = ref.cut_cells()
    assert np.array_equal(ours.air != fitted.SOLID, np.asarray(ref.cut_air()) != 0)
    assert np.array_equal(ours.cell, np.asarray(cells["cell"]))
    tol = {"room": 1e-8, "fold": 1e-6, "far": 3e-5}[name]
    for key in ("air_volume", "open_area", "wall_area", "sliver"):
        mine, theirs = getattr(ours, key), np.asarray(cells[key])
        assert mine.shape == theirs.shape, key
        np.testing.assert_allclose(mine, theirs, rtol=0, atol=tol, err_msg=key)
