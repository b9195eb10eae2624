"""Fitted (cut-cell) walls: the fit of a convex room on the GPU, and the grid's layout from a fit.

The reference lays fitted walls out in two stages (cpp/include/acoustic_spaces/fdtd.hpp:929-1264
of naelolaiz/acoustic-spaces): the fit (cut_cells.hpp, CutCells) measures, for every row — an air
cell that owns cut air — its air volume V, its open area towards each of its 18 neighbours A_k,
its wall area per material W_m and the thickness of the slivers of air it owns through each face;
then set_up_fitted turns those into special rows: link weights lowered(g A_k / V), the wall term
(L/2) sum_m W_m (beta_m + sum_j 1 / (2 a_j)) / V with one branch state per branch, the sliver rule
that scales the link opposite a sliver by w(1 + f) = 3 l / ((l + 1/2)(l + 1)), l = 1 + f, and the
clamp V >= (g/2) sum_k A_k.

* :func:`set_up_fitted` restates the second stage over any fit: fed the reference's own fit (its
  CutFit) it gives the reference's layout array for array (tests/test_fitted.py).
* :func:`convex_fit` is this library's first stage for convex rooms of planar walls, one face of
  which may be open: the cut of every cell by the walls in double precision on the GPU
  (``fdtd_cut_convex``), then on the host each cut cell's air on each side of the walls as a
  region, the reference's owner rule (a region holding an air cell's centre is that cell's; each
  other region, round by round, goes to the air cell whose regions it shares the most open area
  with, ties to the lowest cell) and the rows' sums. Its regions are the cell's air inside and
  outside the room — where the reference's exact fit splits a cell at a room's edge along each
  wall plane into further convex pieces, this fit keeps the air outside the room as one region —
  so its rows agree with the reference's away from the room's edges and corners, and differ in
  those cells (the measured agreement: tests/test_fitted.py).
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import layouts as L

#: The directions of fdtd.hpp:924-927: six axial, then the twelve edge neighbours.
STEPS = np.array(
    [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1), (-1, -1, 0), (1, -1, 0), (-1, 1, 0),
     (1, 1, 0), (-1, 0, -1), (1, 0, -1), (-1, 0, 1), (1, 0, 1), (0, -1, -1), (0, 1, -1), (0, -1, 1), (0, 1, 1)],
    np.int64,
)  # fmt: skip
#: The fit's kinds of cell (cut_cells.hpp:1042).
SOLID, AIR, LAYER = 0, 1, 2


def _edge(grid: L.Grid) -> np.ndarray:
    """Whether each cell lies on the grid's edge (x fastest)."""
    nx, ny, nz = grid.shape
    e = [np.zeros(m, bool) for m in (nx, ny, nz)]
    for a in e:
        a[0] = a[-1] = True
    return (e[2][:, None, None] | e[1][None, :, None] | e[0][None, None, :]).reshape(-1)


def _accumulate(target: np.ndarray, index: np.ndarray, values) -> None:
    """target[index] += values for repeated indices (a flat view of target), by bincount: each
    entry gains the sum of its values in their order. A table of rows (2-D target) sums column by
    column over its rows, not over the whole table."""
    flat = target.reshape(-1)
    index = np.asarray(index, np.int64).reshape(-1)
    values = np.broadcast_to(values, index.shape)
    if target.ndim != 2 or target.shape[1] == 1 or len(index) * 16 > flat.size:
        flat += np.bincount(index, values, minlength=flat.size)
        return
    if not len(index):
        return
    cols = target.shape[1]
    row, col = np.divmod(index, cols)
    if col.min() == col.max():
        target[:, col[0]] += np.bincount(row, values, minlength=target.shape[0])
        return
    # (grouped by column, each group in the values' order)
    order = np.argsort(col, kind="stable")
    row, col, values = row[order], col[order], np.asarray(values)[order]
    starts = np.flatnonzero(np.concatenate([[True], col[1:] != col[:-1]]))
    ends = np.concatenate([starts[1:], [len(col)]])
    for a, b in zip(starts, ends):
        target[:, col[a]] += np.bincount(row[a:b], values[a:b], minlength=target.shape[0])


def opposite(k: int) -> int:
    """The direction opposite k (fdtd.hpp:929)."""
    return k ^ 1 if k < 6 else 6 + 4 * ((k - 6) // 4) + 3 - (k - 6) % 4


def sliver_factor(f):
    """The sliver rule's factor for a sliver f cells thick (fdtd.hpp:950-954)."""
    lam = 1.0 + np.asarray(f, np.float64)
    return 3.0 * lam / ((lam + 0.5) * (lam + 1.0))


@dataclass
class Fit:
    """What a fit gives, as the reference's CutFit names it: the rows (ascending cells), each
    row's ``air_volume`` (cells^3), ``open_area`` (rows, 18), ``wall_area`` (rows, materials + 1;
    the last column the grid's edge) and ``sliver`` (rows, 6); every cell's kind ``air``
    (SOLID, AIR, LAYER); and each cell's ``widths`` per axis on the fit's lattice (cells)."""

    cell: np.ndarray
    air_volume: np.ndarray
    open_area: np.ndarray
    wall_area: np.ndarray
    sliver: np.ndarray
    air: np.ndarray
    widths: tuple[np.ndarray, np.ndarray, np.ndarray]


def set_up_fitted(
    fit: Fit,
    grid: L.Grid,
    materials: list[L.Material | None],
    source_cells: list[tuple[int, float]],
    probe_cells: list[list[tuple[int, float]]],
    *,
    layer: int = 0,
    layer_damping: float = 0.0,
    edge_admittance: float = 1.0,
) -> dict[str, np.ndarray]:
    """The layout of the grid from ``fit`` with the reference's rules for fitted walls
    (set_up_fitted, fdtd.hpp:970-1217; add_special_fitted, fdtd.hpp:1219-1264), the 7-point
    stencil and no speed field (as the reference's fitted walls take them): ``materials`` in the
    fit's columns (None: a material of no admittance), the source's and the probes' cells with
    their weights. Vectorised over the rows."""
    nx, ny, nz = grid.shape
    n = nx * ny * nz
    sy, sz = nx, nx * ny
    offsets = STEPS[:, 0] + STEPS[:, 1] * sy + STEPS[:, 2] * sz

    # The cells' kinds (fdtd.hpp:976-995).
    types = np.zeros(n, np.uint8)
    types[fit.air == AIR] = 1
    types[fit.air == LAYER] = 3
    layer_cells = np.flatnonzero(types == 3).astype(np.int64)
    edge = _edge(grid)

    # The stencil (set_up_stencil, fdtd.hpp:1649-1670).
    exact = 1.0 / 3.0
    plane = exact / (2.0 * math.sqrt(exact))  # L/2: a whole cell face's boundary weight
    half_g = exact / 2.0
    weight_plain = np.float32(L.lowered(exact))
    total_plain = 0.0
    for _ in range(6):
        total_plain += float(weight_plain)
    centre = np.float32(2.0 - total_plain)

    # Materials and branches (fdtd.hpp:392-411).
    M = fit.wall_area.shape[1] - 1
    betas = np.zeros(M)
    branch_rows, branch_owner = [], []
    for m in range(M):
        mat = materials[m] if m < len(materials) else None
        if mat is None:
            continue
        betas[m] = mat.beta
        for row in np.asarray(mat.branches, float).reshape(-1, 3):
            branch_rows.append(row)
            branch_owner.append(m)
    branch_rows = np.array(branch_rows, np.float64).reshape(-1, 3)
    branch_owner = np.array(branch_owner, np.int64)
    branch_a = branch_rows[:, 0] + 0.5 * branch_rows[:, 1] + 0.5 * branch_rows[:, 2]
    if len(branch_a) and not np.all((branch_rows >= 0) & (branch_a[:, None] > 0)):
        raise ValueError("a branch needs mass, resistance and stiffness >= 0")
    material_branches = [np.flatnonzero(branch_owner == m) for m in range(M)]

    rows = np.asarray(fit.cell, np.int64)
    R = len(rows)

    def row_of(cells):
        cells = np.asarray(cells, np.int64)
        at = np.searchsorted(rows, cells)
        at_c = np.minimum(at, max(R - 1, 0))
        hit = (at < R) & (rows[at_c] == cells) if R else np.zeros(len(cells), bool)
        return np.where(hit, at_c, -1)

    wx, wy, wz = (np.asarray(w, np.float64) for w in fit.widths)

    def width(cells, a):
        return (wx[cells % nx], wy[(cells // nx) % ny], wz[cells // sz])[a]

    def cell_volume(cells):
        return width(cells, 0) * width(cells, 1) * width(cells, 2)

    def face_area(cells, a):
        return width(cells, (a + 1) % 3) * width(cells, (a + 2) % 3)

    # The sliver rule (fdtd.hpp:1019-1075): per row o and face k with a sliver of f > 0, the link
    # between o and its neighbour m across the opposite face, scaled on both sides; where both
    # cells' rules touch a link, the product of their factors (in ascending order of factor).
    keys, facs = [], []
    for k in range(6):
        f = fit.sliver[:, k]
        has = f > 0.0
        o = rows[has]
        m = o + offsets[opposite(k)]
        ok = ~edge[m] & (types[m] != 0) & (types[m] != 3)
        o, m, fk = o[ok], m[ok], f[has][ok]
        keys.append(3 * np.minimum(o, m) + k // 2)
        facs.append(sliver_factor(fk))
    keys = np.concatenate(keys) if keys else np.zeros(0, np.int64)
    facs = np.concatenate(facs) if facs else np.zeros(0)
    order = np.lexsort((facs, keys))
    keys, facs = keys[order], facs[order]
    factor_keys, first = np.unique(keys, return_index=True)
    factor_values = np.ones(len(factor_keys))
    # products in sorted order, one factor at a time (each key has a handful)
    counts = np.diff(np.concatenate([first, [len(keys)]]))
    for step in range(int(counts.max()) if len(counts) else 0):
        has = counts > step
        factor_values[has] = factor_values[has] * facs[first[has] + step]
    lower = factor_keys // 3
    upper = lower + np.array([1, sy, sz], np.int64)[factor_keys % 3]
    far = np.unique(np.concatenate([lower, upper]))
    far = far[row_of(far) < 0]

    def factor_of(i, j, axis):
        key = 3 * np.minimum(i, j) + axis
        at = np.searchsorted(factor_keys, key)
        at_c = np.minimum(at, max(len(factor_keys) - 1, 0))
        hit = (at < len(factor_keys)) & (factor_keys[at_c] == key) if len(factor_keys) else np.zeros(len(key), bool)
        return np.where(hit, factor_values[at_c] if len(factor_keys) else 1.0, 1.0)

    # The candidates in ascending order: the rows and the plain cells the sliver rule reaches.
    cand = np.union1d(rows, far).astype(np.int64)
    r_of = row_of(cand)
    is_row = r_of >= 0
    rc = np.maximum(r_of, 0)
    room = (types == 1) | (types == 2)

    # Each candidate's open area towards each direction (area_towards, fdtd.hpp:1087-1100): a
    # row's own; along the axes also a plain cell's whole face, and the sliver rule's factors.
    area = fit.open_area[rc] if R else np.zeros((len(cand), 18))
    area[~is_row] = 0.0
    for k in range(6):
        j = cand + offsets[k]
        a = area[:, k]
        plain = ~is_row & (types[cand] != 0) & ~edge[j] & (types[j] != 0)
        a = np.where(plain, face_area(cand, k // 2), a)
        touched = (a > 0.0) & room[cand] & room[j]
        area[:, k] = np.where(touched, a * factor_of(cand, j, k // 2), a)
    air_volume = np.where(is_row, fit.air_volume[rc] if R else 0.0, cell_volume(cand))

    # The wall term and the branch states (fdtd.hpp:1106-1128), in material order.
    wall = np.zeros(len(cand))
    st_cand, st_branch, st_weight = [], [], []
    for m in range(M):
        W = np.where(is_row, fit.wall_area[rc, m] if R else 0.0, 0.0)
        has = W > 0.0
        weight = plane * W
        wall = np.where(has, wall + weight * betas[m], wall)
        for j in material_branches[m]:
            wall = np.where(has, wall + weight * (0.5 / branch_a[j]), wall)
            st_cand.append(np.flatnonzero(has))
            st_branch.append(np.full(int(has.sum()), j, np.int64))
            st_weight.append(weight[has])
    edge_wall = np.where(is_row, fit.wall_area[rc, M] if R else 0.0, 0.0)
    wall = np.where(edge_wall > 0.0, wall + plane * edge_wall * edge_admittance, wall)
    total = np.zeros(len(cand))
    for k in range(18):
        total = total + area[:, k]
    volume = np.maximum(air_volume, half_g * total)

    # add_special_fitted (fdtd.hpp:1219-1264), s = 1, r = 1 / V.
    r = 1.0 / volume
    lw = np.zeros((len(cand), 18), np.float32)
    linked = area > 0.0
    lw[linked] = L.lowered(exact * area[linked] / np.broadcast_to(volume[:, None], area.shape)[linked])
    link_total = np.zeros(len(cand))
    for k in range(18):
        link_total = link_total + lw[:, k].astype(np.float64)
    centre_d = 2.0 - link_total
    coef_a = centre_d.astype(np.float32)
    over = coef_a.astype(np.float64) > centre_d
    coef_a = np.where(over, np.nextafter(coef_a, np.float32(-np.inf)), coef_a).astype(np.float32)
    coef_b = (1.0 - r * wall).astype(np.float32)
    coef_inv = (1.0 / (1.0 + r * wall)).astype(np.float32)
    n_states = np.zeros(len(cand), np.int64)
    for c in st_cand:
        n_states += np.bincount(c, minlength=len(cand))
    plain_links = np.all(lw[:, :6] == weight_plain, axis=1) & np.all(lw[:, 6:] == 0.0, axis=1)
    spared = (n_states == 0) & (coef_a == centre) & (coef_b == 1.0) & (coef_inv == 1.0) & plain_links
    kept = ~spared

    special = cand[kept]
    K = len(special)
    volumes = volume[kept]
    has_link = area[kept] > 0.0
    link_direction = np.broadcast_to(np.arange(18, dtype=np.uint8), (K, 18))[has_link]
    link_weight = lw[kept][has_link]
    link_counts = has_link.sum(axis=1)
    # Branch states in row order, each row's in material then branch order.
    if st_cand:
        sc = np.concatenate(st_cand)
        order = np.argsort(sc, kind="stable")
        sc = sc[order]
        sb = np.concatenate(st_branch)[order]
        sw = np.concatenate(st_weight)[order]
        keep_state = kept[sc]
        sc, sb, sw = sc[keep_state], sb[keep_state], sw[keep_state]
        state_weight = (r[sc] * sw).astype(np.float32)
        per_row = np.bincount(np.searchsorted(np.flatnonzero(kept), sc), minlength=K)
    else:
        sb = np.zeros(0, np.int64)
        state_weight = np.zeros(0, np.float32)
        per_row = np.zeros(K, np.int64)
    state_start = np.concatenate([[0], np.cumsum(per_row)]).astype(np.uint64)
    types[special] = 2

    # The source's cells (fdtd.hpp:1141-1163): a cell not yet special becomes special (a row that
    # stayed plain with its own coefficients, any other cell with the interior's), each fed w / V.
    # (The rows' arrays stay arrays; the few cells the source adds follow them.)
    coef_a_k, coef_b_k, coef_inv_k = coef_a[kept], coef_b[kept], coef_inv[kept]
    source_k = np.zeros(K, np.float32)
    extra_cell, extra_a, extra_b, extra_inv, extra_volume, extra_source = [], [], [], [], [], []
    extra_dir, extra_w, extra_count = [], [], []
    added: dict[int, int] = {}
    for i, w in source_cells:
        i = int(i)
        k = int(np.searchsorted(special, i))
        if not (k < K and special[k] == i):
            k = added.get(i, -1)
        if k < 0:
            at = int(np.searchsorted(cand, i))
            if at < len(cand) and cand[at] == i and is_row[at]:
                # a row that stayed plain: its own coefficients (add_special_fitted, no spare)
                hl = area[at] > 0.0
                extra_dir.append(np.arange(18, dtype=np.uint8)[hl])
                extra_w.append(lw[at][hl])
                extra_count.append(int(hl.sum()))
                extra_a.append(coef_a[at]), extra_b.append(coef_b[at]), extra_inv.append(coef_inv[at])
                extra_volume.append(volume[at])
            else:
                # add_special(i, exact, 0): the interior's links and coefficients
                extra_dir.append(np.arange(6, dtype=np.uint8))
                extra_w.append(np.full(6, weight_plain, np.float32))
                extra_count.append(6)
                tot = 0.0
                for _ in range(6):
                    tot += exact
                extra_a.append(np.float32(2.0 - tot * (1.0 - L.MARGIN)))
                extra_b.append(np.float32(1.0)), extra_inv.append(np.float32(1.0))
                extra_volume.append(float(cell_volume(np.array([i]))[0]))
            types[i] = 2
            k = K + len(extra_cell)
            extra_cell.append(i)
            extra_source.append(np.float32(0.0))
            added[i] = k
        if k < K:
            source_k[k] = np.float32(source_k[k] + np.float32(w / volumes[k]))
        else:
            e = k - K
            extra_source[e] = np.float32(extra_source[e] + np.float32(w / extra_volume[e]))
    E = len(extra_cell)
    state_start = np.concatenate([state_start, np.full(E, state_start[-1], np.uint64)])
    link_start = np.concatenate([[0], np.cumsum(np.concatenate([link_counts, np.array(extra_count, np.int64)]))])
    link_start = link_start.astype(np.uint64)

    layout: dict[str, np.ndarray] = {}
    layout["shape"] = np.array(grid.shape, np.uint64)
    layout["stencil"] = np.array([7], np.uint64)
    layout["weights"] = np.full(6, weight_plain, np.float32)
    layout["centre"] = np.array([centre], np.float32)
    layout["total"] = np.array([total_plain], np.float32)
    layout["scaled"] = np.array([0], np.uint64)
    layout["scale"] = np.zeros(0, np.float32)
    layout["layer_scale"] = np.zeros(0, np.float32)
    layout["types"] = types
    layout["special"] = np.concatenate([special, np.array(extra_cell, np.int64)]).astype(np.int64)
    layout["link_start"] = link_start
    layout["link_direction"] = np.concatenate([link_direction, *extra_dir]).astype(np.uint8)
    layout["link_weight"] = np.concatenate([link_weight, *extra_w]).astype(np.float32)
    layout["coef_a"] = np.concatenate([coef_a_k, np.array(extra_a, np.float32)]).astype(np.float32)
    layout["coef_b"] = np.concatenate([coef_b_k, np.array(extra_b, np.float32)]).astype(np.float32)
    layout["coef_inv"] = np.concatenate([coef_inv_k, np.array(extra_inv, np.float32)]).astype(np.float32)
    layout["source"] = np.concatenate([source_k, np.array(extra_source, np.float32)]).astype(np.float32)
    layout["state_start"] = state_start
    layout["state_branch"] = sb.astype(np.int32)
    layout["state_weight"] = state_weight
    layout["branch_now"] = (2.0 * branch_rows[:, 0] / branch_a).astype(np.float32)
    layout["branch_before"] = ((2.0 * branch_rows[:, 0] + branch_rows[:, 2]) / branch_a).astype(np.float32)
    layout["branch_gain"] = (0.5 / branch_a).astype(np.float32)
    layout["layer_cells"] = layer_cells
    courant = math.sqrt(float(weight_plain))
    for a, name in enumerate("xyz"):
        if len(layer_cells):
            ck, cp, fk, fp = L._layer_tables(grid.shape[a], layer, layer_damping, courant)
        else:
            ck = cp = fk = fp = np.zeros(0, np.float32)
        layout[f"keep_{name}"], layout[f"push_{name}"] = ck, cp
        layout[f"keep_face_{name}"], layout[f"push_face_{name}"] = fk, fp
    starts, cells, weights = [0], [], []
    for probe in probe_cells:
        for i, w in probe:
            cells.append(int(i))
            weights.append(float(w))
        starts.append(len(cells))
    layout["probe_start"] = np.array(starts, np.uint64)
    layout["probe_cells"] = np.array(cells, np.uint64)
    layout["probe_weights"] = np.array(weights, np.float64)
    layout["flow_mask"] = np.zeros(0, np.uint8)
    return layout


# ---- this library's fit of a convex room --------------------------------------------------------


@dataclass
class Cut:
    """The cells the walls' planes cut (fdtd_cut_convex), ascending: each cell's air inside the
    walls (cells^3), its faces' areas on that side (cells, 6), each plane's wall area in it, and
    the area of the walls' planes between its two sides that no wall covers."""

    cell: np.ndarray
    volume: np.ndarray
    face_area: np.ndarray
    cap: np.ndarray
    bare: np.ndarray


@dataclass
class Walls:
    """A convex room's walls as the fit takes them: its planes (unit normals out of the room,
    offsets, and which are open: no wall), the count of materials, and the columns of the cut's
    wall areas with the material of each (one a plane, the plane's own index; or one a piece of
    wall, the walls cut into pieces of their own materials as a mesh's triangles carry them), and
    the walls as triangles (the fit's lattice frame takes their extent). Offsets (and the pieces'
    edges' offsets) are taken from ``anchor``."""

    normals: np.ndarray
    offsets: np.ndarray
    open_: np.ndarray
    materials: int
    column_material: np.ndarray
    vertices: np.ndarray
    faces: np.ndarray
    piece_plane: np.ndarray | None = None
    piece_start: np.ndarray | None = None
    piece_edges: np.ndarray | None = None
    # The point the offsets are taken from (planes n . (x - anchor) <= offset).
    anchor: np.ndarray = field(default_factory=lambda: np.zeros(3))

    @property
    def open(self) -> bool:
        return bool(np.any(self.open_))

    @property
    def wall_planes(self) -> np.ndarray:
        return np.flatnonzero(self.open_ == 0)


def walls_of(room) -> Walls:
    """The walls of a :class:`layouts.Room` (each plane its own material index), or ``room``
    itself when it is a :class:`Walls` already."""
    if isinstance(room, Walls):
        return room
    normals = np.ascontiguousarray(room.normals, np.float64)
    offsets = np.ascontiguousarray(room.offsets, np.float64)
    open_ = np.array([m is None for m in room.materials], np.uint8)
    vertices, faces, _ = L.room_mesh(room)
    return Walls(normals, offsets, open_, len(room.materials), np.arange(len(offsets), dtype=np.int64),
                 np.asarray(vertices, np.float64), np.asarray(faces, np.int64))  # fmt: skip


def mesh_walls(vertices, faces, materials, count: int, *, tolerance: float = 1e-7, convexity: float = 1e-7) -> Walls:
    """The walls of a convex room given as a triangle mesh, each triangle with its material (as
    the reference's WaveSolver and CutFit take a room, native_module.cpp:1465-1559): the planes of
    its triangles (coplanar ones merged), each triangle a piece of wall on its plane bounded by
    its three edges, and the faces of the vertices' convex hull on which no triangle lies left
    open. Triangles within ``tolerance`` (of the room's size) of one plane share it (the first's):
    a face folded by less, either way, is taken as flat, since a fit of the walls' half-spaces
    cannot follow a fold into the room. The planes are taken relative to the first vertex (``anchor``), so
    that a room far from the origin keeps its digits. Raises ValueError where vertices lie farther
    on both sides of a triangle's plane (the room is not convex)."""
    from scipy.spatial import ConvexHull

    v = np.asarray(vertices, np.float64)
    f = np.asarray(faces, np.int64)
    mat = np.asarray(materials, np.int64)
    anchor = v[0].copy()
    w = v - anchor  # (exact where the coordinates are alike, as a room's are)
    size = max(float(np.abs(w).max()), 1e-300)
    # (a room far from the origin has its vertices rounded to the doubles there: its faces are
    # planar to a few of their steps only)
    rounding = 8.0 * float(np.spacing(np.abs(v).max())) / size
    tolerance, convexity = max(tolerance, rounding), max(convexity, rounding)
    planes: list[tuple[np.ndarray, float]] = []

    def plane_of(n, d, tol):
        for k, (m, e) in enumerate(planes):
            if np.abs(n - m).max() < tol and abs(d - e) < tol * size:
                return k
        return -1

    piece_plane, piece_start, edges = [], [0], []
    for tri in f:
        a, b, c = w[tri]
        n = np.cross(b - a, c - a)
        if np.linalg.norm(n) == 0.0:
            raise ValueError("a triangle of the room has no area")
        n /= np.linalg.norm(n)
        d = float(n @ a)
        side = w @ n - d
        if side.max() > convexity * size:  # (the triangle faces into the room: turn it out)
            if side.min() < -convexity * size:
                raise ValueError("vertices lie on both sides of a triangle's plane: the room is not convex")
            n, d = -n, -d
        k = plane_of(n, d, tolerance)
        if k < 0:
            planes.append((n, d))
            k = len(planes) - 1
        m = planes[k][0]
        for p, q, r in ((a, b, c), (b, c, a), (c, a, b)):
            h = np.cross(q - p, m)
            h /= np.linalg.norm(h)
            if h @ (r - p) > 0.0:
                h = -h
            edges.append((*h, float(h @ p)))
        piece_plane.append(k)
        piece_start.append(len(edges))
    walls = len(planes)
    # the hull's faces that no triangle covers: open (no wall, the air goes through)
    for eq in ConvexHull(w).equations:  # n . x + c <= 0 inside
        norm = np.linalg.norm(eq[:3])
        n, d = eq[:3] / norm, float(-eq[3] / norm)
        if plane_of(n, d, 1e-6) < 0:
            planes.append((n, d))
    normals = np.array([n for n, _ in planes], np.float64)
    offsets = np.array([d for _, d in planes], np.float64)
    open_ = np.r_[np.zeros(walls, np.uint8), np.ones(len(planes) - walls, np.uint8)]
    # piece edges relative to the anchor too (their offsets were taken in its frame)
    return Walls(normals, offsets, open_, int(count), mat.copy(), v, f,
                 np.array(piece_plane, np.uint32), np.array(piece_start, np.uint32),
                 np.ascontiguousarray(np.array(edges, np.float64).reshape(-1)), anchor)  # fmt: skip


def cut_room(room, grid: L.Grid) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """The room's planes as the fit takes them: unit normals, offsets, and which are open."""
    w = walls_of(room)
    return w.normals, w.offsets, w.open_


def cut_convex(room, grid: L.Grid, device: int = 0) -> Cut:
    """The FP64 cut of ``room``'s walls (a :class:`layouts.Room` or :class:`Walls`) by ``grid``'s
    cells on the GPU (fdtd_cut_convex)."""
    from . import _abi

    lib = _abi.load_library()
    w = walls_of(room)
    normals, offsets, open_ = w.normals, w.offsets, w.open_
    r = _abi.FdtdCutRoom()
    r.normals = normals.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    r.offsets = offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    r.open = open_.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
    r.planes = len(offsets)
    if w.piece_plane is not None:
        r.pieces = len(w.piece_plane)
        r.piece_plane = w.piece_plane.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        r.piece_start = w.piece_start.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        r.piece_edges = w.piece_edges.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    for a in range(3):
        r.origin[a] = float(grid.origin[a] - w.anchor[a])
    r.cell = float(grid.cell)
    r.nx, r.ny, r.nz = (int(v) for v in grid.shape)
    out = _abi.FdtdCutCells()
    status = lib.fdtd_cut_convex(ctypes.byref(r), int(device), ctypes.byref(out))
    if status != _abi.FDTD_OK:
        message = lib.fdtd_cut_error().decode()
        if status == _abi.FDTD_EINVAL:
            raise ValueError(message)
        raise RuntimeError(message)
    try:
        return cut_from(out)
    finally:
        lib.fdtd_cut_free(ctypes.byref(out))


def cut_from(out) -> Cut:
    """A Cut from a filled ``fdtd_cut_cells`` (copied; ascending cells)."""
    n, P = int(out.cells), int(out.planes)
    cell = np.ctypeslib.as_array(out.cell, (max(n, 1),))[:n].copy()
    volume = np.ctypeslib.as_array(out.volume, (max(n, 1),))[:n].copy()
    face = np.ctypeslib.as_array(out.face_area, (max(n, 1) * 6,))[: 6 * n].reshape(n, 6).copy()
    cap = np.ctypeslib.as_array(out.cap, (max(n, 1) * P,))[: P * n].reshape(n, P).copy()
    bare = np.ctypeslib.as_array(out.bare, (max(n, 1),))[:n].copy()
    order = np.argsort(cell, kind="stable")
    return Cut(cell[order].astype(np.int64), volume[order], face[order], cap[order], bare[order])


#: A cell's wall counts as cut where its area there exceeds this (in cell faces), a region as air
#: where its volume does (in cells^3): FP64 noise lies far below both.
TINY = 1e-12


def _direction_table():
    table = np.full(27, -1, np.int64)
    for k, (dx, dy, dz) in enumerate(STEPS):
        table[(dx + 1) + 3 * (dy + 1) + 9 * (dz + 1)] = k
    return table


_DIRECTION = _direction_table()


def _direction(grid: L.Grid, a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """The direction k of the step from cell a to cell b (-1 unless one of the 18 neighbours)."""
    nx, ny, _ = grid.shape
    sz = nx * ny
    d = [(b % nx) - (a % nx), ((b // nx) % ny) - ((a // nx) % ny), (b // sz) - (a // sz)]
    near = (np.abs(d[0]) <= 1) & (np.abs(d[1]) <= 1) & (np.abs(d[2]) <= 1)
    key = np.where(near, (d[0] + 1) + 3 * (d[1] + 1) + 9 * (d[2] + 1), 13)
    return np.where(near, _DIRECTION[key], -1)


def lattice_widths(room, grid: L.Grid) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Each cell's width per axis (cells) as the reference's fit measures it on its lattice
    (cut_cells.hpp:2031-2122): the frame E is the largest half-extent of the room's triangles that
    reach the grid's box grown by 2h and of the grid's box, grown by 2h; p = the exponent of E plus
    one, s = 61 - p; the middle X0 per axis rounded to a multiple of 2^(p - 2); a face's double x
    becomes round(x 2^s) - X0 2^s (ties to even); a cell's width is the difference of its faces'
    quanta over h 2^s. Uncut cells hold these widths' product of air (1 within about 1e-15)."""
    w = walls_of(room)
    vertices, faces = w.vertices, w.faces
    h = float(grid.cell)
    face_at = [grid.origin[a] + np.arange(grid.shape[a] + 1, dtype=np.float64) * h for a in range(3)]
    glo = [float(face_at[a][0]) - 2.0 * h for a in range(3)]
    ghi = [float(face_at[a][-1]) + 2.0 * h for a in range(3)]
    lo, hi = [1e300] * 3, [-1e300] * 3
    tri = vertices[faces]  # (T, 3 corners, 3)
    mn, mx = tri.min(axis=1), tri.max(axis=1)
    meets = np.all((mx >= np.array(glo)) & (mn <= np.array(ghi)), axis=1)
    for a in range(3):
        if np.any(meets):
            lo[a] = min(lo[a], float(mn[meets, a].min()))
            hi[a] = max(hi[a], float(mx[meets, a].max()))
        lo[a] = min(lo[a], float(face_at[a][0]))
        hi[a] = max(hi[a], float(face_at[a][-1]))
    E = max((hi[a] - lo[a]) / 2.0 for a in range(3)) + 2.0 * h
    m, e = math.frexp(E)
    p = (e if m > 0.5 else e - 1) + 1
    shift = 61 - p
    S = math.ldexp(h, shift)
    widths = []
    for a in range(3):
        x0 = math.ldexp(float(np.rint(math.ldexp((lo[a] + hi[a]) / 2.0, -(p - 2)))), p - 2)
        q0 = int(math.ldexp(x0, shift))

        def quantize(x: float) -> int:
            y = math.ldexp(float(x), shift)  # exact
            fl = math.floor(y)
            fr = y - fl
            t = int(fl) - q0
            if fr > 0.5 or (fr == 0.5 and t & 1):
                t += 1
            return t

        g = [quantize(v) for v in face_at[a]]
        widths.append(np.array([float(g[i + 1] - g[i]) / S for i in range(grid.shape[a])]))
    return tuple(widths)


def fit_from_cut(cut: Cut, room, grid: L.Grid, *, layer: int = 0) -> Fit:
    """The rows of a convex room from its cut (:func:`cut_convex`), by the reference's rules for
    what a row owns and sums (cut_cells.hpp: the owner rule, sum_up): each cut cell holds up to
    two regions, its air inside the walls' planes and outside them; a region holding an air cell's
    centre is that cell's, and the uncut cells next to a cut one own themselves; then, round by
    round, each region without an owner goes to the air cell (not of the matched layer) whose
    regions it shares the most open area with across the squares between cells, within 1e-12 the
    lowest cell. A row's air volume, walls, open areas towards its 18 neighbours (between regions
    of two owners, by the direction from one owner to the other) and slivers (the volume it owns in
    a face neighbour's cell over the open area through which it owns it) are the sums of what it
    owns."""
    nx, ny, nz = grid.shape
    n = nx * ny * nz
    sy, sz = nx, nx * ny
    edge = _edge(grid)
    ax_depth = [np.minimum(np.arange(m), m - 1 - np.arange(m)).astype(np.int32) for m in (nx, ny, nz)]
    depth = np.minimum(np.minimum(ax_depth[2][:, None, None], ax_depth[1][None, :, None]),
                       ax_depth[0][None, None, :]).reshape(-1)  # fmt: skip
    room = walls_of(room)
    normals, offsets = room.normals, room.offsets
    walls = room.wall_planes
    # The cut's columns of wall area, each with its material's column of the rows' sums.
    columns = [(c, int(m)) for c, m in enumerate(room.column_material) if m >= 0 and c < cut.cap.shape[1]]
    # The air: with an open face every cell but the grid's edge; closed, the cells whose centre
    # lies inside the walls. Cells within `layer` of the edge form the matched layer.
    if room.open:
        air_mask = ~edge
    else:
        inside = np.ones((nz, ny, nx), bool)
        cz, cy, cx_ = (grid.centres(a) - room.anchor[a] for a in (2, 1, 0))
        for f in walls:
            nf = normals[f]
            inside &= (nf[0] * cx_[None, None, :] + nf[1] * cy[None, :, None] + nf[2] * cz[:, None, None]) - offsets[f] < 0.0
        air_mask = ~edge & inside.reshape(-1)
    air = np.where(air_mask, AIR, SOLID).astype(np.uint8)
    if layer > 0:
        air[air_mask & (depth <= layer)] = LAYER

    # The cut cells: those a wall reaches with positive area.
    is_cut = np.any(cut.cap > TINY, axis=1) if len(walls) else np.zeros(len(cut.cell), bool)
    cc = cut.cell[is_cut]
    C = len(cc)
    wx, wy, wz = lattice_widths(room, grid)

    def cell_volume(cells):
        return wx[cells % nx] * wy[(cells // nx) % ny] * wz[cells // sz]

    def face_area(cells, a):
        """The area of each cell's face across axis a (a scalar or one axis per cell)."""
        w3 = np.stack([wx[cells % nx], wy[(cells // nx) % ny], wz[cells // sz]])
        a = np.broadcast_to(np.asarray(a), np.shape(cells))
        cols = np.arange(np.size(cells))
        return w3[(a + 1) % 3, cols] * w3[(a + 2) % 3, cols]

    v_in = np.clip(cut.volume[is_cut], 0.0, 1.0)
    v_out = np.maximum(cell_volume(cc) - v_in, 0.0)
    # Where the walls' planes leave part of the boundary between the two sides bare (past a face
    # left open), the sides meet: one region, as the reference joins leaves across a bare facet.
    joined = cut.bare[is_cut] > TINY
    v_in = np.where(joined, cell_volume(cc), v_in)
    v_out = np.where(joined, 0.0, v_out)
    faces = cut.face_area[is_cut]
    caps = cut.cap[is_cut]
    # Which side holds each cut cell's centre: inside every wall plane that cuts it (a joined
    # cell's one region holds it).
    cx = np.stack([grid.centres(0)[cc % nx], grid.centres(1)[(cc // nx) % ny], grid.centres(2)[cc // sz]], axis=1)
    cx = cx - room.anchor
    centre_in = np.all(cx @ normals[walls].T - offsets[walls] < 0.0, axis=1) | joined

    # Regions: 2c the inside of cut cell c, 2c + 1 its outside; whole cells after them.
    has_in = v_in > TINY
    has_out = v_out > TINY
    cut_index = np.full(n, -1, np.int64)
    cut_index[cc] = np.arange(C)
    offsets6 = np.array([-1, 1, -sy, sy, -sz, sz], np.int64)
    neigh = cc[:, None] + offsets6[None, :]
    whole = np.unique(neigh[(cut_index[neigh] < 0) & ~edge[neigh]])
    W = len(whole)
    whole_index = np.full(n, -1, np.int64)
    whole_index[whole] = 2 * C + np.arange(W)
    G = 2 * C + W
    reg_cell = np.concatenate([np.repeat(cc, 2), whole])
    reg_volume = np.concatenate([np.stack([v_in, v_out], axis=1).reshape(-1), cell_volume(whole)])
    reg_valid = np.concatenate([np.stack([has_in, has_out], axis=1).reshape(-1), np.ones(W, bool)])
    in_air = reg_valid & (air[reg_cell] != SOLID)
    # A cut cell's air inside the walls is the room's whether or not the cell's centre is: where
    # the centre lies outside, the owner rule gives that region to a neighbour.
    in_air[0 : 2 * C : 2] |= reg_valid[0 : 2 * C : 2] & ~edge[cc]
    if not room.open:  # the air outside a closed room's walls is not the source's
        in_air[1 : 2 * C : 2] = False

    # The squares of the cut cells: (lower cell, axis), each once; each gives an inside piece and
    # an outside piece, joining the regions on its two sides.
    lower = np.concatenate([cc[:, None] + np.zeros(3, np.int64)[None, :], neigh[:, [0, 2, 4]]], axis=0).reshape(-1)
    axis = np.concatenate([np.tile(np.arange(3), (C, 1)), np.tile(np.arange(3), (C, 1))], axis=0).reshape(-1)
    key = np.unique(3 * lower + axis)
    lower, axis = key // 3, key % 3
    upper = lower + np.array([1, sy, sz], np.int64)[axis]
    ok = ~edge[lower] & ~edge[upper]
    lower, upper, axis = lower[ok], upper[ok], axis[ok]
    la, ua = cut_index[lower], cut_index[upper]
    # The inside part of the square: from the lower cell's + face where it is cut, else the upper's - face.
    a_in = np.where(la >= 0, faces[np.maximum(la, 0), 2 * axis + 1], faces[np.maximum(ua, 0), 2 * axis])
    a_in = np.clip(a_in, 0.0, 1.0)

    def region(cell_cut, cell, side):
        # (a joined cell's pieces on both sides meet its one region)
        side = np.where(joined[np.maximum(cell_cut, 0)], 0, side)
        return np.where(cell_cut >= 0, 2 * np.maximum(cell_cut, 0) + side, whole_index[cell])

    p_low = np.concatenate([region(la, lower, 0), region(la, lower, 1)])
    p_high = np.concatenate([region(ua, upper, 0), region(ua, upper, 1)])
    p_area = np.concatenate([a_in, np.maximum(face_area(lower, axis) - a_in, 0.0)])
    keep = (p_area > TINY) & (p_low >= 0) & (p_high >= 0)
    keep[keep] &= reg_valid[p_low[keep]] & reg_valid[p_high[keep]]
    p_low, p_high, p_area = p_low[keep], p_high[keep], p_area[keep]

    # Owners (cut_cells.hpp:4641-4711).
    owner = np.full(G, -1, np.int64)
    centre_region = 2 * np.arange(C) + np.where(centre_in, 0, 1)
    own_centre = air[cc] == AIR
    owner[centre_region[own_centre]] = cc[own_centre]
    owner[2 * C :] = np.where(air[whole] != SOLID, whole, -1)
    owner[~reg_valid] = -2  # no region
    for _ in range(64):
        offer_r, offer_o, offer_a = [], [], []
        for to, by in ((p_low, p_high), (p_high, p_low)):
            ob = owner[by]
            ok = (owner[to] == -1) & in_air[to] & (ob >= 0)
            ok[ok] &= air[ob[ok]] == AIR
            offer_r.append(to[ok]), offer_o.append(ob[ok]), offer_a.append(np.maximum(p_area[ok], 0.0))
        r_ = np.concatenate(offer_r)
        if len(r_) == 0:
            break
        o_, a_ = np.concatenate(offer_o), np.concatenate(offer_a)
        order = np.lexsort((o_, r_))
        r_, o_, a_ = r_[order], o_[order], a_[order]
        pair = np.flatnonzero(np.r_[True, (r_[1:] != r_[:-1]) | (o_[1:] != o_[:-1])])
        sums = np.add.reduceat(a_, pair)
        pr, po = r_[pair], o_[pair]
        start = np.flatnonzero(np.r_[True, pr[1:] != pr[:-1]])
        count = np.diff(np.r_[start, len(pr)])
        best, most = po[start].copy(), sums[start].copy()
        for step in range(1, int(count.max())):
            has = count > step
            cand_a = sums[start[has] + step]
            better = cand_a > most[has] + 1e-12
            sel = np.flatnonzero(has)[better]
            best[sel] = po[start[sel] + step]
            most[sel] = cand_a[better]
        owner[pr[start]] = best
    owner[owner == -2] = -1

    # The rows and their sums (sum_up, cut_cells.hpp:4846-4960).
    is_row_cell = np.zeros(n, bool)
    owned = owner >= 0
    is_row_cell[owner[owned]] = air[owner[owned]] == AIR
    rows = np.flatnonzero(is_row_cell)
    row_index = np.full(n, -1, np.int64)
    row_index[rows] = np.arange(len(rows))
    R = len(rows)
    M = room.materials
    air_volume = np.zeros(R)
    open_area = np.zeros((R, 18))
    wall_area = np.zeros((R, M + 1))
    sliver = np.zeros((R, 6))
    sliver_area = np.zeros((R, 6))
    g_ok = owned & np.zeros(G, bool)
    g_ok[owned] = is_row_cell[owner[owned]]
    gr = np.flatnonzero(g_ok)
    ro = row_index[owner[gr]]
    _accumulate(air_volume, ro, reg_volume[gr])
    # walls: both sides of a wall see it (a cut cell's inside and outside regions)
    cut_g = gr[gr < 2 * C]
    both_sides = np.where(joined[cut_g // 2], 2.0, 1.0)  # a joined region sees each wall's two sides
    for col, mat in columns:
        _accumulate(wall_area, row_index[owner[cut_g]] * (M + 1) + mat, both_sides * caps[cut_g // 2, col])
    k = _direction(grid, owner[gr], reg_cell[gr])
    ax = (k >= 0) & (k < 6)
    _accumulate(sliver, ro[ax] * 6 + k[ax], reg_volume[gr][ax])
    oa, ob = owner[p_low], owner[p_high]
    rowa = (oa >= 0) & is_row_cell[np.maximum(oa, 0)]
    rowb = (ob >= 0) & is_row_cell[np.maximum(ob, 0)]
    same = (oa == ob) & (oa >= 0)
    ca, cb = reg_cell[p_low], reg_cell[p_high]
    sl = same & rowa & ((ca == oa) != (cb == oa))
    other = np.where(ca == oa, cb, ca)
    ks = _direction(grid, oa, other)
    sl &= (ks >= 0) & (ks < 6)
    _accumulate(sliver_area, row_index[oa[sl]] * 6 + ks[sl], p_area[sl])
    diff = ~same & (oa >= 0) & (ob >= 0)
    kd = _direction(grid, oa, ob)
    both = rowa & rowb
    link = diff & (kd >= 0) & ((kd < 6) | both)
    ka = link & rowa
    _accumulate(open_area, row_index[oa[ka]] * 18 + kd[ka], p_area[ka])
    kb = link & rowb
    opp = np.array([opposite(k) for k in range(18)], np.int64)
    _accumulate(open_area, row_index[ob[kb]] * 18 + opp[kd[kb]], p_area[kb])
    # A row's faces that no square was cut for: whole (its cell and the one across both uncut).
    uncut_rows = rows[cut_index[rows] < 0]
    for k6 in range(6):
        j = uncut_rows + offsets6[k6]
        whole_face = cut_index[j] < 0
        to_edge = whole_face & edge[j]
        to_air = whole_face & ~edge[j] & (air[j] != SOLID)
        _accumulate(wall_area, row_index[uncut_rows[to_edge]] * (M + 1) + M, face_area(uncut_rows[to_edge], k6 // 2))
        _accumulate(open_area, row_index[uncut_rows[to_air]] * 18 + k6, face_area(uncut_rows[to_air], k6 // 2))
    sliver = np.where(sliver_area > 1e-9, sliver / np.where(sliver_area > 1e-9, sliver_area, 1.0), 0.0)

    # The conduit rule (thin_conduits, cut_cells.hpp:5190-5360): a region of the air outside its
    # owner's cube (round a convex edge of the walls whose faces lie just inside the grid's
    # planes, a thin L of air) has its open area to an edge-diagonal neighbour n of its owner o
    # scaled by phi = 2 V / (A_s A_p) (V its volume, A_s its open area to o's own cube, A_p its
    # open area through the link) where that is below 1 - 1e-12, and a share
    # (1 - phi) A_p / (A_s + the sum of its A_p) of its walls moves from o's row to n's.
    diag = ~same & rowa & rowb & (kd >= 6)
    if np.any(diag):
        pl, ph, pa_, da, db_, kk = p_low[diag], p_high[diag], p_area[diag], oa[diag], ob[diag], kd[diag]
        ca_, cb_ = reg_cell[pl] != da, reg_cell[ph] != db_
        link_g = np.concatenate([pl[ca_], ph[cb_]])
        link_k = np.concatenate([kk[ca_], opp[kk[cb_]]])
        link_a = np.concatenate([pa_[ca_], pa_[cb_]])
        lkey = link_g * 18 + link_k
        keys_u, inv = np.unique(lkey, return_inverse=True)
        through = np.zeros(len(keys_u))
        np.add.at(through, inv, link_a)
        lg, lk = keys_u // 18, keys_u % 18
        conduits = np.unique(lg)
        # A_s: each conduit's open area to the regions of its owner's own cube.
        contact = np.zeros(len(conduits))
        sm = same & (oa >= 0)
        ia_, ib_ = reg_cell[p_low] == oa, reg_cell[p_high] == oa
        one = sm & (ia_ != ib_)
        gg = np.where(ia_, p_high, p_low)[one]
        at = np.searchsorted(conduits, gg)
        hit = (at < len(conduits)) & (conduits[np.minimum(at, len(conduits) - 1)] == gg)
        np.add.at(contact, at[hit], p_area[one][hit])
        ci_ = np.searchsorted(conduits, lg)
        a_s = contact[ci_]
        kc = _direction(grid, owner[lg], reg_cell[lg])
        ok_link = (kc >= 0) & (kc < 6) & (a_s > 0.0) & (through > 0.0)
        ratio = np.where(ok_link, 2.0 * reg_volume[lg] / np.where(ok_link, a_s * through, 1.0), 1.0)
        phi = np.where(ok_link & (ratio < 1.0 - 1e-12), ratio, 1.0)
        if np.any(phi < 1.0):
            def phi_of(g, k):
                key_ = g * 18 + k
                at_ = np.searchsorted(keys_u, key_)
                return phi[np.minimum(at_, len(keys_u) - 1)]

            f = np.ones(len(pl))
            f = np.where(ca_, f * phi_of(pl, kk), f)
            f = np.where(cb_, f * phi_of(ph, opp[kk]), f)
            ra, rb = row_index[da], row_index[db_]
            marked = np.zeros((R, 18), bool)
            marked[ra[f < 1.0], kk[f < 1.0]] = True
            marked[rb[f < 1.0], opp[kk[f < 1.0]]] = True
            plain = np.zeros((R, 18))
            scaled = np.zeros((R, 18))
            for rr, kq in ((ra, kk), (rb, opp[kk])):
                m_ = marked[rr, kq]
                np.add.at(plain, (rr[m_], kq[m_]), pa_[m_])
                np.add.at(scaled, (rr[m_], kq[m_]), pa_[m_] * f[m_])
            open_area = np.where(marked, scaled, open_area)
            # The walls: each link's share of its conduit's walls, to the diagonal neighbour's row.
            spans = contact.copy()
            np.add.at(spans, ci_, through)
            share = (1.0 - phi) * through / spans[ci_]
            o_ = owner[lg]
            across = o_ + np.array([int(d[0] + d[1] * sy + d[2] * sz) for d in STEPS], np.int64)[lk]
            # (in the order of the links, conduit by conduit; a whole cell has no walls)
            moving = np.flatnonzero((share > 0.0) & is_row_cell[across] & (lg < 2 * C))
            ro_, rn_ = row_index[o_[moving]], row_index[across[moving]]
            gl = lg[moving] // 2
            sides = np.where(joined[gl], 2.0, 1.0)
            for col, mat in columns:
                a_ = sides * caps[gl, col]
                has = a_ > 0.0
                np.subtract.at(wall_area[:, mat], ro_[has], share[moving][has] * a_[has])
                np.add.at(wall_area[:, mat], rn_[has], share[moving][has] * a_[has])
    return Fit(rows.astype(np.int64), air_volume, open_area, wall_area, sliver, air, (wx, wy, wz))


def fitted_cubic(grid: L.Grid, point) -> list[tuple[int, float]]:
    """The 4 x 4 x 4 cells round ``point`` with the fitted path's cubic weights, z then y then x
    (reading_cells_fitted, fdtd.hpp:1518-1605, for a point whose cells are all air in sight of
    it): along each axis, with lo the point's place between the centres below and above it, the
    weight of cell k of the four is prod over m != k of (lo - (m - 1)) / (k - m)."""
    nx, ny, _ = grid.shape
    start, weight = [], []
    for a in range(3):
        centres = grid.centres(a)
        p = float(np.asarray(point, float)[a])
        j = int(np.searchsorted(centres, p, side="right")) - 1
        if not (1 <= j < grid.shape[a] - 3):
            raise ValueError("the point is too near the grid's edge for its cubic stencil")
        lo = (p - centres[j]) / (centres[j + 1] - centres[j])
        ws = []
        for k in range(4):
            w = 1.0
            for m in range(4):
                if m != k:
                    w *= (lo - float(m - 1)) / float(k - m)
            ws.append(w)
        start.append(j - 1)
        weight.append(ws)
    out = []
    for z in range(4):
        for y in range(4):
            for x in range(4):
                w = weight[0][x] * weight[1][y] * weight[2][z]
                if w != 0.0:
                    out.append((int(start[0] + x + (start[1] + y) * nx + (start[2] + z) * nx * ny), w))
    return out


def convex_fit(room, grid: L.Grid, *, layer: int = 0, device: int = 0) -> Fit:
    """This library's fit of a convex room (a :class:`layouts.Room` or :class:`Walls`): the cut
    on the GPU, then the rows on the host."""
    return fit_from_cut(cut_convex(room, grid, device), room, grid, layer=layer)


def fitted_layout(room: L.Room, grid: L.Grid, source, probes, *, layer: int = 0, layer_damping: float = 0.0,
                  edge_admittance: float = 1.0, device: int = 0, fit: Fit | None = None) -> dict[str, np.ndarray]:
    """The layout of ``room`` with fitted walls: this library's fit (or ``fit``), then the
    reference's rules for its rows, with the source and the probes on the fitted cubic stencil
    (each must lie where its 64 cells are air clear of every wall)."""
    if fit is None:
        fit = convex_fit(room, grid, layer=layer, device=device)
    source_cells = fitted_cubic(grid, source)
    probe_cells = [fitted_cubic(grid, p) for p in np.asarray(probes, float).reshape(-1, 3)]
    rows = set(int(i) for i in fit.cell)
    for cells in [source_cells, *probe_cells]:
        for i, _ in cells:
            if fit.air[i] != AIR:
                raise ValueError("a point's cubic stencil reaches a cell outside the air or in the matched layer")
    for cells in probe_cells:
        if any(int(i) in rows for i, _ in cells):
            raise ValueError("a probe's cubic stencil reaches a cut cell: keep the probes clear of the walls")
    return set_up_fitted(fit, grid, room.materials, source_cells, probe_cells, layer=layer,
                         layer_damping=layer_damping, edge_admittance=edge_admittance)  # fmt: skip
