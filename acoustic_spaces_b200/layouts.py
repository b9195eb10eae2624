"""Grid layouts of synthetic rooms, built on the host with the reference's rules.

The reference lays out a grid in its ``WaveSolver`` constructor (cpp/include/acoustic_spaces/
fdtd.hpp:360-690 of naelolaiz/acoustic-spaces) from a triangle mesh, by casting rays along every
link near a face. For rooms whose walls are planes — convex polyhedra, boxes — the same layout
follows from the planes directly, and this module builds it with NumPy for grids of tens of
millions of cells, with the reference's rules for walls on cell faces and the 7-point stencil:

- a link between two cell centres is cut when its segment leaves the room through a wall (the
  face it crosses nearest the cell: for a convex room, the plane it exits through), not through
  an open face (fdtd.hpp:452-497);
- the air is what the source reaches (fdtd.hpp:499-519): the room's inside, and with an open face
  every cell but the grid's edge;
- air cells within ``layer`` cells of the grid's edge form the matched layer (fdtd.hpp:521-542),
  with the coefficients of layer_coefficients (fdtd.hpp:2219-2238);
- an air cell with a cut link, or one to the grid's edge, is a boundary row (fdtd.hpp:544-625):
  links 1/3 where open, the cut links' boundary weight 1/(2 L) · 1/3 times each wall's admittance
  beta and its branches' 1/(2 a), one set of branch states per material met, coefficients as
  add_special (fdtd.hpp:3499-3517), with a speed field's s and r;
- the source and the probes read the 4 x 4 x 4 cells round them with cubic weights
  (reading_cells, fdtd.hpp:2361-2472, away from surfaces), the source's cells made special
  (fdtd.hpp:627-638).

Every array has the name and dtype of ``WaveSolver.layout()`` (fdtd.hpp:727-782), and the tests
check that a room built here equals the reference's own layout of it, array for array.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

#: fdtd.hpp:920: the stability margin each link weight is lowered by.
MARGIN = 1.0 / 262144.0
AXIAL = 1.0 / 3.0
COURANT = 1.0 / math.sqrt(3.0)
#: The boundary weight of one cut axial link of the 7-point stencil: g / (2 L).
BOUNDARY = AXIAL / (2.0 * math.sqrt(AXIAL))
#: The axial steps in the reference's order of directions (fdtd.hpp:924-925).
AXIAL_STEPS = ((-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1))
LAYER_CELLS = 8
LAYER_DAMPING = 0.5


def down(w: np.ndarray | float) -> np.ndarray:
    """The largest float32 not above each double w (fdtd.hpp:2127-2131)."""
    w = np.asarray(w, np.float64)
    f = w.astype(np.float32)
    over = f.astype(np.float64) > w
    return np.where(over, np.nextafter(f, np.float32(0)), f).astype(np.float32)


def lowered(w) -> np.ndarray:
    """A link's weight as the update takes it (fdtd.hpp:2133-2135)."""
    return down(np.asarray(w, np.float64) * (1.0 - MARGIN))


@dataclass
class Material:
    """A wall's specific admittance: ``beta`` and mass-resistance-stiffness branches (m, r, q),
    each as the solver takes it (mass over the time step, resistance, stiffness times the time
    step; engine/impedance.py:199-211)."""

    beta: float
    branches: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))


def resonant_branch(conductance: float, quality: float, frequency_hz: float, rate: float) -> np.ndarray:
    """One resonant branch (m, r, q) of admittance ``conductance`` at resonance, quality
    ``quality`` and resonance ``frequency_hz`` at ``rate`` steps a second: M = Q R / w0,
    S = Q R w0, R = 1 / conductance (engine/impedance.py:199-211)."""
    t = 1.0 / rate
    r = 1.0 / conductance
    w0 = 2.0 * math.pi * frequency_hz
    return np.array([[quality * r / (w0 * t), r, quality * r * w0 * t]])


@dataclass
class Grid:
    """``shape`` cells of ``cell`` metres, cell 0's corner at ``origin``, x fastest."""

    origin: np.ndarray
    cell: float
    shape: tuple[int, int, int]

    @property
    def n(self) -> int:
        return int(np.prod(self.shape))

    def centres(self, axis: int) -> np.ndarray:
        return self.origin[axis] + (np.arange(self.shape[axis]) + 0.5) * self.cell


@dataclass
class Screen:
    """A thin planar wall (a barrier) across axis ``axis`` at ``position`` metres, spanning
    ``lo`` to ``hi`` along the other two axes (in their order), of ``material``: the links of the
    cells whose centres it separates, within its span, are cut."""

    axis: int
    position: float
    lo: tuple[float, float]
    hi: tuple[float, float]
    material: Material


@dataclass
class Room:
    """A convex room: the cells with n_f . x < d_f for every plane f. ``materials[f]`` is plane
    f's wall, or None for an open face (no wall: the air goes through). With ``patches``, the walls
    are cut into patches: ``patches(planes, points)`` gives the index into ``patch_materials`` of
    the wall at each crossing point of a plane (arrays). ``screens`` are thin walls inside."""

    normals: np.ndarray  # (F, 3), unit
    offsets: np.ndarray  # (F,)
    materials: list[Material | None]
    patches: object = None
    patch_materials: list[Material] | None = None
    screens: list[Screen] = field(default_factory=list)

    def wall_materials(self) -> list[Material | None]:
        walls = list(self.patch_materials) if self.patches is not None else list(self.materials)
        return walls + [screen.material for screen in self.screens]

    @property
    def open(self) -> bool:
        return any(m is None for m in self.materials)


@dataclass
class Built:
    """A layout and what was set up with it."""

    layout: dict[str, np.ndarray]
    grid: Grid
    air_cells: int
    boundary_cells: int
    source_cells: int
    rate: float
    sensitivity: dict | None = None


def _inside(room: Room, grid: Grid) -> tuple[np.ndarray, np.ndarray]:
    """Each cell's centre inside the room, and within a cell's reach of it (every plane's
    signed distance below one cell), as (nz, ny, nx) masks.

    The signed distance of a cell's centre (x, y, z) to plane f is worked out in double as
    (n_z z + n_y y) + n_x x - d_f; along a row of fixed y and z it never decreases in x where n_x > 0 (the
    float sums are monotone) and never increases where n_x < 0, so the cells on the inner side of
    the plane are a prefix or a suffix of the row. Its end is found by bisection on that same
    expression, row by row, and each mask is the intersection of the planes' intervals."""
    nx, ny, nz = grid.shape
    xs, ys, zs = grid.centres(0), grid.centres(1), grid.centres(2)
    limits = {"inside": 0.0, "near": 1.01 * grid.cell}
    spans = {key: (np.zeros((nz, ny), np.int64), np.full((nz, ny), nx, np.int64)) for key in limits}
    for f in range(len(room.offsets)):
        nrm, d = room.normals[f], room.offsets[f]
        x = nrm[0] * xs
        zy = (nrm[2] * zs)[:, None] + (nrm[1] * ys)[None, :]
        for key, limit in limits.items():
            lo, hi = spans[key]
            if nrm[0] == 0.0:
                lo[~(((zy + x[0]) - d) < limit)] = nx  # the whole row on one side
                continue
            # a: the count of leading cells on the inner side (n_x > 0), or of leading cells on
            # the outer side, the first inner one (n_x < 0)
            a, b = np.zeros((nz, ny), np.int64), np.full((nz, ny), nx, np.int64)
            while np.any(a < b):
                mid = (a + b) // 2
                value = (zy + x[np.minimum(mid, nx - 1)]) - d
                goes = (value < limit) if nrm[0] > 0 else ~(value < limit)
                open_ = a < b
                a = np.where(open_ & goes, mid + 1, a)
                b = np.where(open_ & ~goes, mid, b)
            if nrm[0] > 0:
                np.minimum(hi, a, out=hi)
            else:
                np.maximum(lo, a, out=lo)
    column = np.arange(nx)[None, None, :]
    masks = [(column >= lo[:, :, None]) & (column < hi[:, :, None]) for lo, hi in spans.values()]
    return masks[0], masks[1]


def _first_wall(room: Room, grid: Grid, start: np.ndarray, end: np.ndarray) -> np.ndarray:
    """For the links from cells ``start`` to cells ``end`` (flat indices), the wall each crosses
    nearest its start, or -1 where it crosses none. The segment's part inside the (convex) room
    is clipped by every plane: it enters through the plane of the largest entry parameter and
    leaves through that of the smallest exit one; a cut is either where it is a wall (not an
    open face), the entry first."""
    nx, ny, _ = grid.shape

    def centres(i):
        return np.stack(
            [grid.centres(0)[i % nx], grid.centres(1)[(i // nx) % ny], grid.centres(2)[i // (nx * ny)]], 1
        )

    ca, cb = centres(start), centres(end)
    m = len(start)
    t_in, t_out = np.zeros(m), np.ones(m)
    enter, leave = np.full(m, -1, np.int64), np.full(m, -1, np.int64)
    empty = np.zeros(m, bool)
    for f in range(len(room.offsets)):
        sa = ca @ room.normals[f] - room.offsets[f]
        sb = cb @ room.normals[f] - room.offsets[f]
        empty |= (sa >= 0.0) & (sb >= 0.0)
        outgoing = (sa < 0.0) & (sb >= 0.0)
        incoming = (sa >= 0.0) & (sb < 0.0)
        denom = np.where(outgoing | incoming, sa - sb, 1.0)
        t = sa / denom
        later_in = incoming & (t > t_in)
        t_in = np.where(later_in, t, t_in)
        enter = np.where(later_in, f, enter)
        sooner_out = outgoing & (t < t_out)
        t_out = np.where(sooner_out, t, t_out)
        leave = np.where(sooner_out, f, leave)
    crosses = ~empty & (t_in < t_out)
    walls = np.array([mat is not None for mat in room.materials] + [False])
    enter_wall = crosses & (enter >= 0) & walls[enter]
    leave_wall = crosses & (leave >= 0) & walls[leave]
    face = np.where(enter_wall, enter, np.where(leave_wall, leave, -1))
    if room.patches is None:
        return face
    # The patch of the wall where the link crosses it.
    hit = face >= 0
    t = np.where(enter_wall, t_in, t_out)
    points = ca + t[:, None] * (cb - ca)
    out = np.full(len(face), -1, np.int64)
    if np.any(hit):
        out[hit] = np.asarray(room.patches(face[hit], points[hit]), np.int64)
    return out


def cubic_cells(grid: Grid, point) -> list[tuple[int, float]]:
    """The 4 x 4 x 4 cells round ``point`` and their cubic weights, z then y then x
    (reading_cells, fdtd.hpp:2361-2472, for a point away from every surface)."""
    nx, ny, _ = grid.shape
    q = (np.asarray(point, float) - grid.origin) / grid.cell - 0.5
    start, weight = [], []
    for a in range(3):
        below = math.floor(q[a])
        if not (q[a] >= 1.0 and q[a] < grid.shape[a] - 3.0 and below >= 1):
            raise ValueError("the point is too near the grid's edge for its cubic stencil")
        s = below - 1
        x = q[a] - s
        ws = []
        for j in range(4):
            w = 1.0
            for m in range(4):
                if m != j:
                    w *= (x - m) / float(j - m)
            ws.append(w)
        start.append(s)
        weight.append(ws)
    out = []
    for z in range(4):
        for y in range(4):
            for x in range(4):
                w = weight[0][x] * weight[1][y] * weight[2][z]
                if w != 0.0:
                    out.append((int(start[0] + x + (start[1] + y) * nx + (start[2] + z) * nx * ny), w))
    return out


def _layer_tables(size: int, layer: int, damping: float, courant: float, ends=(True, True)):
    """keep and push of the centres and the faces along an axis (fdtd.hpp:2219-2238), damped
    toward the ends of the axis that have the layer."""

    def damp(from_edge: float) -> float:
        into = max(0.0, layer + 0.5 - from_edge) / layer
        return damping * into * into

    ck, cp, fk, fp = [], [], [], []
    last = float(size - 1)
    far = float("inf")
    for x in range(size + 1):
        c = float(x)
        dc = damp(min(c if ends[0] else far, last - c if ends[1] else far))
        df = damp(min(c - 0.5 if ends[0] else far, last - c + 0.5 if ends[1] else far))
        ck.append((1.0 - dc) / (1.0 + dc))
        cp.append(courant / (1.0 + dc))
        fk.append((1.0 - df) / (1.0 + df))
        fp.append(courant / (1.0 + df))
    f32 = lambda v: np.array(v, np.float64).astype(np.float32)  # noqa: E731
    return f32(ck), f32(cp), f32(fk), f32(fp)


def layer_tables_tangent(size: int, layer: int, damping: float, courant: float, ends=(True, True)):
    """The derivatives in ``damping`` of :func:`_layer_tables`'s keep and push of the centres and
    the faces (float64): with d = damping * into^2 (into the layer's depth fraction),
    keep = (1 - d) / (1 + d) and push = courant / (1 + d) give d keep = -2 into^2 / (1 + d)^2 and
    d push = -courant into^2 / (1 + d)^2 — the chain from a gradient in the tables to one in the
    layer's damping."""

    def into2(from_edge: float) -> float:
        into = max(0.0, layer + 0.5 - from_edge) / layer
        return into * into

    last, far = float(size - 1), float("inf")
    out = {"keep": [], "push": [], "keep_face": [], "push_face": []}
    for x in range(size + 1):
        c = float(x)
        for kind, edge in (("", min(c if ends[0] else far, last - c if ends[1] else far)),
                           ("_face", min(c - 0.5 if ends[0] else far, last - c + 0.5 if ends[1] else far))):  # fmt: skip
            i2 = into2(edge)
            d = damping * i2
            out["keep" + kind].append(-2.0 * i2 / (1.0 + d) ** 2)
            out["push" + kind].append(-courant * i2 / (1.0 + d) ** 2)
    return {k: np.array(v, np.float64) for k, v in out.items()}


def damping_tangent(layout, layer: int, damping: float, layer_sides=(True,) * 6) -> dict[str, np.ndarray]:
    """The derivatives in the layer's damping of ``layout``'s twelve tables (by their names, as
    :meth:`B200WaveSolver.set_layer_tangent` takes them): :func:`layer_tables_tangent` along each
    axis with the layout's own Courant number (the square root of its axial weight) and the axis'
    ends that have the layer."""
    shape = [int(v) for v in np.asarray(layout["shape"]).reshape(-1)]
    courant = math.sqrt(float(np.asarray(layout["weights"], np.float32)[0]))
    out = {}
    for a, name in enumerate("xyz"):
        t = layer_tables_tangent(shape[a], layer, damping, courant, (layer_sides[2 * a], layer_sides[2 * a + 1]))
        for kind in ("keep", "push", "keep_face", "push_face"):
            out[f"{kind}_{name}"] = t[kind]
    return out


def cell_face_layout(room: Room, grid: Grid, source, probes, **options) -> Built:
    """The reference's layout of ``room`` on ``grid`` with walls on cell faces, the 7-point
    stencil, a uniform speed ratio ``speed`` (None: the grid's), the source at ``source`` and
    the probes at ``probes`` (each at least two cells from every wall and from the layer)."""
    return cell_face_layouts(room, grid, [source], probes, **options)[0]


def cell_face_layouts(
    room: Room,
    grid: Grid,
    sources,
    probes,
    *,
    layer: int = 0,
    layer_damping: float = 0.0,
    edge_admittance: float = 1.0,
    speed: float | None = None,
    rate: float | None = None,
    layer_sides=(True,) * 6,
    layer_meets_walls: bool = False,
) -> list[Built]:
    """The layouts of one room with each of ``sources`` in turn (the same probes): the room's
    rows are worked out once. ``layer_sides``: which faces of the grid (x-, x+, y-, y+, z-, z+)
    have the matched layer. ``layer_meets_walls``: let walls reach the layer's cells, which then
    take their plain layer update (a solid neighbour's pressure is zero); the reference refuses
    such a model, and by default so does this builder."""
    nx, ny, nz = grid.shape
    n = grid.n
    sy, sz = nx, nx * ny
    inside, near = _inside(room, grid)
    inside, near = inside.reshape(-1), near.reshape(-1)
    # The grid's edge, and each cell's depth into it.
    def axis_depth(size, low, high):
        i = np.arange(size)
        big = np.full(size, np.iinfo(np.int64).max // 4)
        return np.minimum(np.where(low, i, big), np.where(high, size - 1 - i, big))

    def edge_depth(size):
        i = np.arange(size)
        return np.minimum(i, size - 1 - i)

    dx, dy, dz = (axis_depth(size, layer_sides[2 * a], layer_sides[2 * a + 1]) for a, size in enumerate((nx, ny, nz)))
    depth = np.minimum(np.minimum(dz[:, None, None], dy[None, :, None]), dx[None, None, :]).reshape(-1)
    ex, ey, ez = edge_depth(nx), edge_depth(ny), edge_depth(nz)
    edge = (np.minimum(np.minimum(ez[:, None, None], ey[None, :, None]), ex[None, None, :]) == 0).reshape(-1)

    # Air: the inside, and with an open face all but the edge (fdtd.hpp:499-519).
    air = (~edge) if room.open else (inside & ~edge)
    types = np.where(air, 1, 0).astype(np.uint8)
    layer_cells = np.zeros(0, np.int64)
    if layer > 0:
        in_layer = air & (depth <= layer)
        types[in_layer] = 3
        layer_cells = np.flatnonzero(in_layer).astype(np.int64)

    # Cut links: between inside and outside cells, leaving through a wall (not the open face).
    offsets = [s[0] + s[1] * sy + s[2] * sz for s in AXIAL_STEPS]
    blocked = np.zeros((6, n), bool)
    if len(room.wall_materials()) >= np.iinfo(np.int16).max:
        raise ValueError("a room of 32,767 materials or more")
    material = np.full((6, n), -1, np.int16)  # a wall, screen or patch index; -1 none, -2 the edge
    is_candidate = air & (types == 1)
    candidates = np.flatnonzero(is_candidate)

    def ahead(mask: np.ndarray, off: int) -> np.ndarray:
        """mask[i + off] at every cell i (False where that leaves the grid: never a candidate's)."""
        out = np.zeros_like(mask)
        if off > 0:
            out[:-off] = mask[off:]
        else:
            out[-off:] = mask[:off]
        return out

    for k, off in enumerate(offsets):
        edge_ahead = ahead(edge, off)
        edge_link = is_candidate & edge_ahead
        blocked[k, edge_link] = True
        material[k, edge_link] = -2  # the grid's edge
        # Links that may meet a wall: an end inside and one out, or both within a cell's reach
        # of the room (a link can clip an edge or corner of it).
        maybe = is_candidate & ~edge_ahead & near & ahead(near, off) & ~(inside & ahead(inside, off))
        if not np.any(maybe):
            continue
        c = np.flatnonzero(maybe)
        jj = c + off
        face = _first_wall(room, grid, c, jj)
        walled = face >= 0
        blocked[k, c[walled]] = True
        material[k, c[walled]] = face[walled]
    # Screens: the links along a screen's axis between cells on its two sides, within its span.
    walls = len(room.wall_materials()) - len(room.screens)

    def screened(screen: Screen, cells: np.ndarray, k: int) -> np.ndarray:
        a = screen.axis
        step = AXIAL_STEPS[k][a]
        if step == 0:
            return np.zeros(len(cells), bool)
        index = (cells % nx, (cells // nx) % ny, cells // (nx * ny))
        here = grid.centres(a)[index[a]]
        there = here + step * grid.cell
        others = [b for b in range(3) if b != a]
        inside_span = np.ones(len(cells), bool)
        for m, b in enumerate(others):
            centre = grid.centres(b)[index[b]]
            inside_span &= (centre >= screen.lo[m]) & (centre <= screen.hi[m])
        return inside_span & ((here - screen.position) * (there - screen.position) < 0.0)

    for si, screen in enumerate(room.screens):
        for k in range(6):
            hit = screened(screen, candidates, k) & ~blocked[k, candidates]
            blocked[k, candidates[hit]] = True
            material[k, candidates[hit]] = walls + si
    boundary = np.flatnonzero(blocked.any(axis=0) & (types == 1))
    # The matched layer's air must meet no face (fdtd.hpp:521-528).
    if not layer_meets_walls:
        for k, off in enumerate(offsets):
            j = layer_cells + off
            maybe = near[layer_cells] & near[j] & ~edge[j]
            if np.any(_first_wall(room, grid, layer_cells[maybe], j[maybe]) >= 0) or any(
                np.any(screened(screen, layer_cells, k)) for screen in room.screens
            ):
                raise ValueError("the model reaches into the matched layer")

    # Materials: beta and branches.
    mats = room.wall_materials()
    betas = np.array([0.0 if m is None else m.beta for m in mats])
    branch_rows, branch_owner = [], []
    for f, m in enumerate(mats):
        if m is None:
            continue
        for row in np.asarray(m.branches, float).reshape(-1, 3):
            branch_rows.append(row)
            branch_owner.append(f)
    branch_rows = np.array(branch_rows).reshape(-1, 3)
    branch_owner = np.array(branch_owner, np.int64)
    a_of = branch_rows[:, 0] + 0.5 * branch_rows[:, 1] + 0.5 * branch_rows[:, 2]
    if len(a_of) and not np.all((branch_rows >= 0) & (a_of[:, None] > 0)):
        raise ValueError("a branch needs mass, resistance and stiffness >= 0")
    branch_now = (2.0 * branch_rows[:, 0] / a_of).astype(np.float32)
    branch_before = ((2.0 * branch_rows[:, 0] + branch_rows[:, 2]) / a_of).astype(np.float32)
    branch_gain = (0.5 / a_of).astype(np.float32)

    # Each cell's scale is its speed ratio (a float) squared, rounded to a float (fdtd.hpp:415-425);
    # its boundary terms take the square root of that scale.
    if speed is None:
        s = 1.0
    else:
        ratio = float(np.float32(speed))
        s = float(np.float32(ratio * ratio))
    r = math.sqrt(s)

    # Boundary rows (fdtd.hpp:560-623), vectorised over the rows, in the reference's order of
    # directions and materials.
    B = len(boundary)
    blk = blocked[:, boundary]  # (6, B)
    mat = material[:, boundary]
    open_link = ~blk
    beta_sum = np.zeros(B)
    padded = np.concatenate([betas, [0.0]])  # (a room of no walls: only the grid's edge is met)
    for k in range(6):
        term = np.where(mat[k] == -2, BOUNDARY * edge_admittance, BOUNDARY * padded[np.maximum(mat[k], 0)])
        beta_sum = beta_sum + np.where(blk[k], term, 0.0)
    # The materials met, in order of first meeting, and the weight of each one's cut links.
    kinds = np.full((6, B), -1, np.int64)
    kind_weight = np.zeros((6, B))
    count = np.zeros(B, np.int64)
    for k in range(6):
        m = np.where(blk[k] & (mat[k] >= 0), mat[k], -1)
        seen = np.zeros(B, bool)
        for slot in range(6):
            hit = (kinds[slot] == m) & (m >= 0)
            kind_weight[slot] = np.where(hit, kind_weight[slot] + BOUNDARY, kind_weight[slot])
            seen |= hit
        new = (m >= 0) & ~seen
        rows = np.flatnonzero(new)
        kinds[count[rows], rows] = m[rows]
        kind_weight[count[rows], rows] = BOUNDARY
        count[rows] += 1
    g = beta_sum.copy()
    state_rows, state_branch, state_weight = [], [], []
    by_material = {f: np.flatnonzero(branch_owner == f) for f in range(len(mats))}
    for slot in range(6):
        has = kinds[slot] >= 0
        if not np.any(has):
            break
        for f in np.unique(kinds[slot][has]):
            rows = np.flatnonzero(kinds[slot] == f)
            for j in by_material[int(f)]:
                g[rows] = g[rows] + kind_weight[slot, rows] * (0.5 / a_of[j])
                state_rows.append(np.repeat(rows, 1))
                state_branch.append(np.full(len(rows), j, np.int32))
                state_weight.append((r * kind_weight[slot, rows]).astype(np.float32))
    # Each row's states in slot order then branch order: sort by (row, insertion order).
    if state_rows:
        rows_all = np.concatenate(state_rows)
        order = np.argsort(rows_all, kind="stable")
        rows_all = rows_all[order]
        st_branch = np.concatenate(state_branch)[order]
        st_weight = np.concatenate(state_weight)[order]
    else:
        rows_all = np.zeros(0, np.int64)
        st_branch = np.zeros(0, np.int32)
        st_weight = np.zeros(0, np.float32)
    states_per_row = np.bincount(rows_all, minlength=B)

    link_w = lowered(s * AXIAL)
    total = np.zeros(B)
    for k in range(6):
        total = total + np.where(open_link[k], AXIAL, 0.0)
    coef_a = (2.0 - s * total * (1.0 - MARGIN)).astype(np.float32)
    coef_b = (1.0 - r * g).astype(np.float32)
    coef_inv = (1.0 / (1.0 + r * g)).astype(np.float32)
    links_per_row = open_link.sum(axis=0)
    link_direction = np.tile(np.arange(6, dtype=np.uint8), (B, 1))[open_link.T]
    types[boundary] = 2

    special = list(boundary.astype(np.int64))
    link_start = np.concatenate([[0], np.cumsum(links_per_row)]).astype(np.uint64)
    state_start = np.concatenate([[0], np.cumsum(states_per_row)]).astype(np.uint64)
    base_types = types

    def place(source) -> Built:
        types = base_types.copy()
        special = list(base_special)
        source_values = np.zeros(B, np.float32)

        # The source's cells (fdtd.hpp:627-638): made special with the stencil's own weights, each
        # source term summed in float as the reference's source_[k] += float(s w).
        extra_link_dir: list[np.ndarray] = []
        accumulated: dict[int, np.float32] = {}
        made: dict[int, int] = {}
        for ci, w in cubic_cells(grid, source):
            t = types[ci]
            if t == 3:
                raise ValueError("the source is in the matched layer")
            if t == 0:
                raise ValueError("the source sees no cell of the wave grid")
            if t == 2:
                k = made.get(ci)
                if k is None:
                    k = int(np.searchsorted(boundary, ci))
                    if k >= B or boundary[k] != ci:
                        raise ValueError("a source cell is special but not a boundary row")
            else:
                types[ci] = 2
                k = len(special)
                special.append(ci)
                made[ci] = k
                extra_link_dir.append(np.arange(6, dtype=np.uint8))
            accumulated[k] = np.float32(accumulated.get(k, np.float32(0.0)) + np.float32(s * w))
        E = len(made)
        extra_source = np.zeros(E, np.float32)
        for k, value in accumulated.items():
            if k < B:
                source_values[k] = value
            else:
                extra_source[k - B] = value
        exact_total = 0.0
        for _ in range(6):
            exact_total += AXIAL
        extra_coef_a = np.full(E, np.float32(2.0 - s * exact_total * (1.0 - MARGIN)), np.float32)

        layout: dict[str, np.ndarray] = {}
        weights = np.full(6, lowered(AXIAL), np.float32)
        tot = 0.0
        for w in weights:
            tot += float(w)
        layout["shape"] = np.array(grid.shape, np.uint64)
        layout["stencil"] = np.array([7], np.uint64)
        layout["weights"] = weights
        layout["centre"] = np.array([2.0 - tot], np.float32)
        layout["total"] = np.array([tot], np.float32)
        layout["scaled"] = np.array([0 if speed is None else 1], np.uint64)
        layout["scale"] = np.full(n, np.float32(s), np.float32) if speed is not None else np.zeros(0, np.float32)
        layout["layer_scale"] = (
            np.full(len(layer_cells), np.float32(s), np.float32) if speed is not None else np.zeros(0, np.float32)
        )
        layout["types"] = types
        layout["special"] = np.array(special, np.int64)
        layout["link_start"] = np.concatenate([link_start, link_start[-1] + 6 * np.arange(1, E + 1, dtype=np.uint64)])
        layout["link_direction"] = np.concatenate([link_direction] + extra_link_dir).astype(np.uint8)
        layout["link_weight"] = np.full(len(layout["link_direction"]), link_w, np.float32)
        layout["coef_a"] = np.concatenate([coef_a, extra_coef_a])
        layout["coef_b"] = np.concatenate([coef_b, np.ones(E, np.float32)])
        layout["coef_inv"] = np.concatenate([coef_inv, np.ones(E, np.float32)])
        layout["source"] = np.concatenate([source_values, extra_source])
        layout["state_start"] = np.concatenate([state_start, np.full(E, state_start[-1], np.uint64)])
        layout["state_branch"] = st_branch.astype(np.int32)
        layout["state_weight"] = st_weight.astype(np.float32)
        layout["branch_now"] = branch_now
        layout["branch_before"] = branch_before
        layout["branch_gain"] = branch_gain
        layout["layer_cells"] = layer_cells
        courant = math.sqrt(float(weights[0]))
        for a, name in enumerate("xyz"):
            if len(layer_cells):
                ends = (layer_sides[2 * a], layer_sides[2 * a + 1])
                ck, cp, fk, fp = _layer_tables(grid.shape[a], layer, layer_damping, courant, ends)
            else:
                ck = cp = fk = fp = np.zeros(0, np.float32)
            layout[f"keep_{name}"], layout[f"push_{name}"] = ck, cp
            layout[f"keep_face_{name}"], layout[f"push_face_{name}"] = fk, fp
        starts, cells, pweights = [0], [], []
        for p in np.asarray(probes, float).reshape(-1, 3):
            if np.linalg.norm(p - np.asarray(source, float)) < (3.0 - 1e-9) * grid.cell:
                # the reference reads such a probe from the eight cells round it (fdtd.hpp:645-646)
                raise ValueError("a probe lies within three cells of the source")
            for ci, w in cubic_cells(grid, p):
                if types[ci] not in (1, 2):
                    raise ValueError("a probe reads a cell outside the air")
                cells.append(ci)
                pweights.append(w)
            starts.append(len(cells))
        layout["probe_start"] = np.array(starts, np.uint64)
        layout["probe_cells"] = np.array(cells, np.uint64)
        layout["probe_weights"] = np.array(pweights, np.float64)
        layout["flow_mask"] = np.zeros(0, np.uint8)
        air_cells = int(np.count_nonzero(types))
        return Built(layout, grid, air_cells, B, E, rate or 0.0)

    base_special = special
    # How each boundary row's coefficients depend on the materials (for gradients): per row, each
    # material's weight of cut links (the kinds above) and the weight of its links to the grid's
    # edge; each branch's material and (m, r, q).
    rows_, mats_, weights_ = [], [], []
    for slot in range(6):
        has = kinds[slot] >= 0
        rows_.append(np.flatnonzero(has))
        mats_.append(kinds[slot][has])
        weights_.append(kind_weight[slot][has])
    edge_weight = np.zeros(B)
    for k in range(6):
        edge_weight = edge_weight + np.where(blk[k] & (mat[k] == -2), BOUNDARY, 0.0)
    sensitivity = {
        "row": np.concatenate(rows_) if rows_ else np.zeros(0, np.int64),
        "material": np.concatenate(mats_) if mats_ else np.zeros(0, np.int64),
        "weight": np.concatenate(weights_) if weights_ else np.zeros(0),
        "edge_weight": edge_weight,
        "edge_admittance": edge_admittance,
        "boundary_rows": B,
        "r": r,
        "branch_material": branch_owner,
        "branch_mrq": branch_rows,
        "materials": len(mats),
    }
    built = [place(source) for source in sources]
    for b in built:
        b.sensitivity = sensitivity
    return built


# ---- seeded synthetic rooms ------------------------------------------------------------------

OFFSET = np.array([0.0137, 0.0219, 0.0291])  # cell centres off round numbers


def convex_room(
    rng: np.random.Generator,
    box,
    *,
    faces: int,
    margin: float,
    open_face: int | None,
    material,
) -> Room:
    """A seeded convex room with ``faces`` planes inside the box [0, box] shrunk by ``margin``
    on every side: the shrunk box's six faces (-x, +x, -y, +y, -z, +z) and ``faces - 6`` planes
    tangent to the ellipsoid inscribed in it at random points, each cutting off part of the box.
    ``material(rng)`` gives each wall's Material; plane ``open_face`` (an index of the six box
    faces) is open."""
    box = np.asarray(box, float)
    low, high = np.full(3, margin), box - margin
    normals, offsets = [], []
    for a in range(3):
        for sign in (-1.0, 1.0):
            nrm = np.zeros(3)
            nrm[a] = sign
            normals.append(nrm)
            offsets.append(sign * (high[a] if sign > 0 else low[a]))
    centre, semi = 0.5 * (low + high), 0.5 * (high - low)
    for _ in range(max(0, faces - 6)):
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        point = centre + semi * u
        nrm = u / semi
        nrm /= np.linalg.norm(nrm)
        normals.append(nrm)
        offsets.append(float(nrm @ point))
    mats = [material(rng) for _ in normals]
    if open_face is not None:
        mats[open_face] = None
    return Room(np.array(normals), np.array(offsets), mats)


def inside_points(
    rng: np.random.Generator, room: Room, box, count: int, clearance: float, apart: float = 0.0
) -> np.ndarray:
    """``count`` seeded points inside ``room`` at least ``clearance`` from each of its planes,
    the others at least ``apart`` from the first (a source and its receivers). Raises ValueError
    when 200,000 draws find none (a room too small for the clearance)."""
    box = np.asarray(box, float)
    out: list[np.ndarray] = []
    draws = 0
    while len(out) < count:
        draws += 1
        if draws > 200_000:
            raise ValueError(f"no point {clearance} m inside every wall of the room: is it too small?")
        p = rng.uniform(0.0, box)
        if not np.all(room.normals @ p - room.offsets < -clearance):
            continue
        if out and np.linalg.norm(p - out[0]) < apart:
            continue
        out.append(p)
    return np.array(out)


def room_mesh(room: Room) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """The walls of ``room`` as triangles: vertices (V, 3), faces (T, 3) and each triangle's plane
    (the open face has none). For handing the same room to the reference's mesh-based solver."""
    from scipy.spatial import HalfspaceIntersection

    halfspaces = np.column_stack([room.normals, -room.offsets])
    interior = None
    # a point well inside: the centre of the box the first six planes bound
    lo = np.array([room.offsets[1 - 1] * -1, -room.offsets[2], -room.offsets[4]])
    hi = np.array([room.offsets[1], room.offsets[3], room.offsets[5]])
    interior = 0.5 * (lo + hi)
    corners = HalfspaceIntersection(halfspaces, interior).intersections
    verts, tris, owner = [], [], []
    for f in range(len(room.offsets)):
        if room.materials[f] is None:
            continue
        on = np.abs(corners @ room.normals[f] - room.offsets[f]) < 1e-9
        pts = corners[on]
        if len(pts) < 3:
            continue
        # distinct points, ordered round their centroid in the plane
        pts = np.unique(np.round(pts, 12), axis=0)
        c = pts.mean(axis=0)
        nrm = room.normals[f]
        e1 = pts[0] - c
        e1 /= np.linalg.norm(e1)
        e2 = np.cross(nrm, e1)
        angle = np.arctan2((pts - c) @ e2, (pts - c) @ e1)
        pts = pts[np.argsort(angle)]
        base = len(verts)
        verts.extend(pts)
        for k in range(1, len(pts) - 1):
            tris.append((base, base + k, base + k + 1))
            owner.append(f)
    return np.array(verts), np.array(tris, np.int64), np.array(owner, np.int64)


def gaussian_drive(rate: float, steps: int, sigma_s: float = 0.5e-3) -> np.ndarray:
    """A Gaussian pulse of ``sigma_s`` seconds sampled at ``rate``, centred at 6 sigma, peak 1."""
    t = (np.arange(steps) - 6.0 * sigma_s * rate) / (sigma_s * rate)
    return np.exp(-0.5 * t * t).astype(np.float32)


def ricker_drive(rate: float, steps: int, sigma_s: float = 0.5e-3) -> np.ndarray:
    """The second derivative of a Gaussian of ``sigma_s`` seconds (a Ricker wavelet), sampled at
    ``rate``, centred at 6 sigma, peak 1: a drive that adds no net mass to a closed room (zero mean
    and zero first moment, as the reference's twice high-passed drive, engine/wave.py:135-139), so
    that a closed room's pressure does not drift."""
    t = (np.arange(steps) - 6.0 * sigma_s * rate) / (sigma_s * rate)
    return ((1.0 - t * t) * np.exp(-0.5 * t * t)).astype(np.float32)


@dataclass
class Workload:
    """A seeded room ready to step: its room, grid, layout, drive and description."""

    name: str
    room: Room
    built: Built
    source: np.ndarray
    receivers: np.ndarray
    signal: np.ndarray
    description: dict


def polyhedral_room(
    seed: int = 0,
    *,
    box=(20.0, 15.0, 10.0),
    cell: float = 0.04,
    layer: int = LAYER_CELLS,
    receivers: int = 16,
    steps: int = 12000,
    speed_of_sound: float = 343.0,
    walls: str = "faces",
    device: int = 0,
) -> Workload:
    """A seeded convex polyhedral room of 12 to 20 planar faces inscribed in ``box`` metres, open
    through its +x face into the air round it, on a grid of ``cell`` metres spanning the box with
    a ``layer``-cell matched layer inside its edge (damping 0.5). Each wall has a 2-pole
    admittance: a real beta in [0.02, 0.1] and one passive resonant branch of seeded resonance
    (30 to 300 Hz), quality (0.5 to 10) and conductance (0.005 to 0.5). One source and
    ``receivers`` receivers at seeded points at least 0.5 m from every plane; the drive a 0.5 ms
    Gaussian pulse. 7-point stencil at its Courant limit. ``walls``: "faces" for walls on cell
    faces (the reference's default path), "fitted" for fitted (cut-cell) walls by this library's
    FP64 fit on the GPU (``fitted.fitted_layout``; ``device`` runs it)."""
    if walls not in ("faces", "fitted"):
        raise ValueError("walls are 'faces' or 'fitted'")
    rng = np.random.default_rng(seed)
    rate = speed_of_sound / (COURANT * cell)
    faces = int(rng.integers(12, 21))

    def material(r):
        return Material(
            float(r.uniform(0.02, 0.1)),
            resonant_branch(r.uniform(0.005, 0.5), r.uniform(0.5, 10.0), r.uniform(30.0, 300.0), rate),
        )

    margin = cell * (layer + 3)
    room = convex_room(rng, box, faces=faces, margin=margin, open_face=1, material=material)
    points = inside_points(rng, room, box, 1 + receivers, max(0.5, 3 * cell), apart=max(0.5, 4 * cell))
    grid = Grid(-OFFSET * cell, cell, tuple(int(round(b / cell)) for b in box))
    if walls == "fitted":
        from . import fitted

        lay = fitted.fitted_layout(room, grid, points[0], points[1:], layer=layer, layer_damping=LAYER_DAMPING,
                                   device=device)  # fmt: skip
        built = Built(lay, grid, int(np.count_nonzero(lay["types"])), len(lay["special"]), 0, rate)
    else:
        built = cell_face_layout(room, grid, points[0], points[1:], layer=layer, layer_damping=LAYER_DAMPING,
                                 rate=rate)  # fmt: skip
    lay = built.layout
    description = {
        "room": f"convex polyhedron, {faces} planes in {box[0]:g}x{box[1]:g}x{box[2]:g} m, +x face open",
        "grid": "x".join(str(v) for v in grid.shape),
        "cell_m": cell,
        "cells": grid.n,
        "air_cells": built.air_cells,
        "interior_cells": int(np.count_nonzero(lay["types"] == 1)),
        "special_rows": len(lay["special"]),
        "links": len(lay["link_direction"]),
        "branch_states": len(lay["state_branch"]),
        "layer_cells": len(lay["layer_cells"]),
        "probes": receivers,
        "steps": steps,
        "rate_hz": rate,
        "walls": ("fitted cut cells (this library's FP64 GPU fit of the convex room), 2-pole admittance per wall"
                  if walls == "fitted" else "cell faces, 2-pole admittance per wall"),  # fmt: skip
        "stencil": 7,
        "seed": seed,
    }
    return Workload("polyhedral_room", room, built, points[0], points[1:], gaussian_drive(rate, steps), description)


def miki_admittance(frequency_hz, flow_resistivity):
    """Normalised surface admittance of a semi-infinite porous ground of flow resistivity
    ``flow_resistivity`` (Pa s/m^2) by Miki's model (Miki 1990, a revision of Delany and
    Bazley's): Z = 1 + 5.50 X^-0.632 - j 8.43 X^-0.632, X = 1000 f / sigma, time dependence
    e^{j w t}; the reference fits its ground materials to the same model (materials/ground.py)."""
    x = 1000.0 * np.asarray(frequency_hz, float) / flow_resistivity
    z = 1.0 + 5.50 * x**-0.632 - 1j * 8.43 * x**-0.632
    return 1.0 / z


def porous_ground(flow_resistivity: float, rate: float, *, poles: int = 3, band=(20.0, 600.0)) -> Material:
    """A ground material: Miki's admittance fitted over ``band`` Hz by a real beta and ``poles``
    relaxation branches (conductance g_j, corner frequency f_j: Y = beta + sum g_j jw / (jw +
    2 pi f_j)), corner frequencies log-spaced over the band and the conductances and beta by
    non-negative least squares, so that the fit is passive."""
    from scipy.optimize import nnls

    f = np.geomspace(band[0], band[1], 200)
    target = miki_admittance(f, flow_resistivity)
    corners = np.geomspace(band[0], band[1], poles)
    jw = 2j * math.pi * f
    columns = [np.ones_like(jw)] + [jw / (jw + 2.0 * math.pi * fc) for fc in corners]
    a = np.vstack([np.concatenate([c.real, c.imag]) for c in columns]).T
    b = np.concatenate([target.real, target.imag])
    coef, _ = nnls(a, b)
    branches = [np.array([[0.0, 1.0 / g, (1.0 / g) * 2.0 * math.pi * fc / rate]])
                for g, fc in zip(coef[1:], corners) if g > 0.0]  # fmt: skip
    return Material(float(coef[0]), np.vstack(branches) if branches else np.zeros((0, 3)))


def shoebox_room(
    seed: int = 0,
    *,
    size=(6.0, 4.0, 3.0),
    cell: float = 0.05,
    speed: float = 0.99,
    absorption=(0.05, 0.3),
    steps: int = 4000,
    speed_of_sound: float = 343.0,
) -> Workload:
    """A closed box of ``size`` metres on cells of ``cell`` metres, laid out as the reference's
    tests lay a box out (two cells of margin); its six walls each a real admittance from an
    absorption uniform in ``absorption`` (Paris's formula); a uniform speed ratio ``speed`` (the
    Courant number speed / sqrt(3)), the grid's rate such that the sound travels at
    ``speed_of_sound``; one source and one receiver at seeded points 0.5 m from every wall; a 0.5 ms
    Gaussian drive."""
    rng = np.random.default_rng(seed)
    rate = speed_of_sound / (speed * COURANT * cell)
    betas = paris_admittance(rng.uniform(absorption[0], absorption[1], 6))
    room = shoebox(np.asarray(size, float), [Material(float(b)) for b in betas])
    points = inside_points(rng, room, np.asarray(size, float), 2, 0.5, apart=4 * cell)
    grid = room_grid(np.asarray(size, float), cell)
    built = cell_face_layout(room, grid, points[0], points[1:], speed=speed, rate=rate)
    lay = built.layout
    description = {
        "room": f"box {size[0]:g}x{size[1]:g}x{size[2]:g} m, real admittance per wall from absorption U[%g, %g]"
        % absorption,
        "grid": "x".join(str(v) for v in grid.shape),
        "cell_m": cell,
        "cells": grid.n,
        "air_cells": built.air_cells,
        "interior_cells": int(np.count_nonzero(lay["types"] == 1)),
        "special_rows": len(lay["special"]),
        "links": len(lay["link_direction"]),
        "branch_states": len(lay["state_branch"]),
        "layer_cells": 0,
        "probes": 1,
        "steps": steps,
        "rate_hz": rate,
        "speed_ratio": speed,
        "walls": "cell faces, real admittance",
        "stencil": 7,
        "seed": seed,
    }
    return Workload("shoebox_room", room, built, points[0], points[1:], gaussian_drive(rate, steps), description)


def outdoor_halfspace(
    seed: int = 0,
    *,
    shape=(1024, 256, 256),
    cell: float = 0.1,
    layer: int = 12,
    receivers: int = 64,
    steps: int = 8000,
    barrier: bool = True,
    barrier_height: float = 3.0,
    speed_of_sound: float = 343.0,
) -> Workload:
    """An outdoor half-space on a grid of ``shape`` cells of ``cell`` metres: porous ground two
    cells above the grid's floor (Miki's admittance of a flow resistivity log-uniform in 50 to
    20,000 kPa s/m^2, fitted by three relaxation branches), air above it, a ``layer``-cell matched
    layer (damping 0.5) on the five open sides, the ground running into it (this project's own
    layout: the reference refuses a model that reaches its matched layer). A rigid thin barrier
    ``barrier_height`` m high at a seeded x across y (short of the layer); the source 0.5 m above
    the ground 5 to 15 m before the barrier (less on small grids); ``receivers`` receivers 1.5 m above the ground on a
    line along x behind it; a 0.5 ms Gaussian drive."""
    rng = np.random.default_rng(seed)
    rate = speed_of_sound / (COURANT * cell)
    nx, ny, nz = shape
    grid = Grid(-OFFSET * cell, cell, tuple(shape))
    ground_z = grid.origin[2] + 2.0 * cell
    sigma = math.exp(rng.uniform(math.log(50.0), math.log(20000.0))) * 1000.0
    ground = porous_ground(sigma, rate)
    room = Room(np.array([[0.0, 0.0, -1.0]]), np.array([-ground_z]), [ground])
    lo_x = grid.origin[0] + (layer + 4) * cell
    hi_x = grid.origin[0] + (nx - layer - 4) * cell
    lo_y = grid.origin[1] + (layer + 4) * cell
    hi_y = grid.origin[1] + (ny - layer - 4) * cell
    barrier_x = float(rng.uniform(0.35, 0.5) * (hi_x - lo_x) + lo_x) + 0.5 * cell * 0.37
    y_mid = 0.5 * (lo_y + hi_y) + float(rng.uniform(-1.0, 1.0))
    before = min(float(rng.uniform(5.0, 15.0)), 0.8 * (barrier_x - lo_x))  # (small grids: what there is)
    source = np.array([barrier_x - before, y_mid, ground_z + 0.5])
    xs = np.linspace(barrier_x + 2.0, hi_x - 1.0, receivers)
    probes = np.stack([xs, np.full(receivers, y_mid), np.full(receivers, ground_z + 1.5)], 1)
    if barrier:
        room.screens.append(Screen(0, barrier_x, (lo_y, ground_z), (hi_y, ground_z + barrier_height), Material(0.0)))
    built = cell_face_layout(room, grid, source, probes, layer=layer, layer_damping=LAYER_DAMPING, rate=rate,
                             layer_sides=(True, True, True, True, False, True), layer_meets_walls=True)  # fmt: skip
    lay = built.layout
    description = {
        "room": f"outdoor half-space, porous ground (Miki, sigma {sigma / 1000:.0f} kPa s/m^2, 3 relaxation branches)"
        + (f", rigid barrier {barrier_height:g} m high at x {barrier_x:.2f} m" if barrier else ", no barrier"),
        "grid": "x".join(str(v) for v in grid.shape),
        "cell_m": cell,
        "cells": grid.n,
        "air_cells": built.air_cells,
        "interior_cells": int(np.count_nonzero(lay["types"] == 1)),
        "special_rows": len(lay["special"]),
        "links": len(lay["link_direction"]),
        "branch_states": len(lay["state_branch"]),
        "layer_cells": len(lay["layer_cells"]),
        "probes": receivers,
        "steps": steps,
        "rate_hz": rate,
        "walls": "cell faces; the ground runs into the matched layer",
        "stencil": 7,
        "seed": seed,
    }
    return Workload("outdoor_halfspace", room, built, source, probes, gaussian_drive(rate, steps), description)


# ---- many rooms in one grid ------------------------------------------------------------------


def paris_absorption(impedance):
    """Random-incidence absorption of a locally reacting surface of real normalised impedance z,
    Paris's formula for a diffuse field: 8/z (1 + 1/(1+z) - 2/z ln(1+z))
    (engine/impedance.py:52-56 of the reference states the same formula)."""
    z = np.asarray(impedance, float)
    return 8.0 / z * (1.0 + 1.0 / (1.0 + z) - 2.0 / z * np.log1p(z))


def paris_admittance(absorption):
    """The real admittance 1/z whose random-incidence absorption is ``absorption``, on the side of
    hard surfaces (z above the impedance of the most absorbing real surface, about 1.5672): the
    inverse of :func:`paris_absorption` by bisection in log z."""
    alpha = np.clip(np.asarray(absorption, float), 0.0, 1.0)
    low = np.full(alpha.shape, math.log(1.5672))
    high = np.full(alpha.shape, math.log(1e9))
    for _ in range(60):
        mid = 0.5 * (low + high)
        above = paris_absorption(np.exp(mid)) > alpha
        low = np.where(above, mid, low)
        high = np.where(above, high, mid)
    return np.where(alpha <= 0.0, 0.0, np.exp(-0.5 * (low + high)))


def shoebox(size, materials) -> Room:
    """A closed box room from the origin to ``size``: its six walls -x, +x, -y, +y, -z, +z with
    ``materials``."""
    normals, offsets = [], []
    for a in range(3):
        for sign in (-1.0, 1.0):
            nrm = np.zeros(3)
            nrm[a] = sign
            normals.append(nrm)
            offsets.append(size[a] if sign > 0 else 0.0)
    return Room(np.array(normals), np.array(offsets), list(materials))


def room_grid(size, cell: float) -> Grid:
    """The grid of a box room as the reference's tests lay it out (tests/test_wave.py:80-82): the
    origin two cells and a fraction of a cell below the room, two cells beyond it."""
    origin = -cell * (2.0 + OFFSET)
    shape = tuple(int(v) for v in np.ceil((np.asarray(size, float) - origin) / cell).astype(int) + 2)
    return Grid(origin, cell, shape)


@dataclass
class Stacked:
    """Layouts of several grids stepped as one: ``layout`` the combined grid; ``parts[k]`` the k-th
    input's (first probe, last probe + 1, air cells, first plane)."""

    layout: dict[str, np.ndarray]
    parts: list[tuple[int, int, int, int]]

    @property
    def air_cells(self) -> int:
        return sum(part[2] for part in self.parts)


def stack(layouts: list[dict[str, np.ndarray]], across: int = 1) -> Stacked:
    """One layout of many grids without matched layers. The grids go in groups of ``across``
    consecutive ones: a group's grids side by side along x (each after the one before), the group
    at y = 0 of a plane as wide as the widest group and as deep as the deepest grid, its planes
    after the group before's (as many as its tallest grid has). Grids of one room with several
    sources, side by side, fill the interior sweep's tiles where one alone would leave most of a
    tile empty. Each grid's outermost layer of cells is never air, so no link joins two grids, and
    each grid is stepped exactly as on its own: every row keeps its coefficients, every link its
    neighbour."""
    first = layouts[0]
    for lay in layouts:
        if int(lay["stencil"][0]) != int(first["stencil"][0]) or not np.array_equal(lay["weights"], first["weights"]):
            raise ValueError("the grids to stack have different stencils")
        if not (np.array_equal(lay["centre"], first["centre"]) and np.array_equal(lay["total"], first["total"])):
            raise ValueError("the grids to stack have different centres")
        if int(lay["scaled"][0]) != int(first["scaled"][0]):
            raise ValueError("the grids to stack are not all scaled or all unscaled")
        if len(lay["layer_cells"]):
            raise ValueError("grids with a matched layer cannot be stacked (its tables are the grid's own)")
        if len(lay.get("flow_mask", [])):
            raise ValueError("moving air cannot be stacked")
    if across < 1:
        raise ValueError("at least one grid a group")
    shapes = [tuple(int(v) for v in lay["shape"]) for lay in layouts]
    groups = [list(range(g, min(g + across, len(shapes)))) for g in range(0, len(shapes), across)]
    # Each grid's offset: x after the grids before it in its group, z after the groups before.
    x_at, z_at, z = [0] * len(shapes), [0] * len(shapes), 0
    for group in groups:
        x = 0
        for k in group:
            x_at[k], z_at[k] = x, z
            x += shapes[k][0]
        z += max(shapes[k][2] for k in group)
    NX = max(sum(shapes[k][0] for k in group) for group in groups)
    NY = max(s[1] for s in shapes)
    NZ = z
    scaled = int(first["scaled"][0]) == 1
    types = np.zeros((NZ, NY, NX), np.uint8)
    scale = np.ones((NZ, NY, NX), np.float32) if scaled else None
    out = {k: [] for k in ("special", "link_direction", "link_weight", "coef_a", "coef_b", "coef_inv", "source",
                           "state_branch", "state_weight", "branch_now", "branch_before", "branch_gain",
                           "probe_cells", "probe_weights")}  # fmt: skip
    link_start, state_start, probe_start = [np.zeros(1, np.uint64)], [np.zeros(1, np.uint64)], [np.zeros(1, np.uint64)]
    links = states = branches = probes = reads = 0
    parts = []

    def mapped(index, shape, x_first, z_first):
        nx, ny, _ = shape
        i = np.asarray(index, np.int64)
        return (i % nx + x_first) + NX * ((i // nx) % ny + NY * (i // (nx * ny) + z_first))

    for k, (lay, shape) in enumerate(zip(layouts, shapes)):
        nx, ny, nz = shape
        x0, z0 = x_at[k], z_at[k]
        t = np.asarray(lay["types"]).reshape(nz, ny, nx)
        types[z0 : z0 + nz, :ny, x0 : x0 + nx] = t
        if scaled:
            scale[z0 : z0 + nz, :ny, x0 : x0 + nx] = np.asarray(lay["scale"]).reshape(nz, ny, nx)
        out["special"].append(mapped(lay["special"], shape, x0, z0))
        for name in ("link_direction", "link_weight", "coef_a", "coef_b", "coef_inv", "source", "state_weight",
                     "branch_now", "branch_before", "branch_gain", "probe_weights"):  # fmt: skip
            out[name].append(np.asarray(lay[name]))
        out["state_branch"].append(np.asarray(lay["state_branch"], np.int64) + branches)
        out["probe_cells"].append(mapped(lay["probe_cells"], shape, x0, z0).astype(np.uint64))
        link_start.append(np.asarray(lay["link_start"], np.uint64)[1:] + np.uint64(links))
        state_start.append(np.asarray(lay["state_start"], np.uint64)[1:] + np.uint64(states))
        probe_start.append(np.asarray(lay["probe_start"], np.uint64)[1:] + np.uint64(reads))
        p = len(lay["probe_start"]) - 1
        parts.append((probes, probes + p, int(np.count_nonzero(t)), z0))
        links += len(lay["link_direction"])
        states += len(lay["state_branch"])
        branches += len(lay["branch_now"])
        probes += p
        reads += len(lay["probe_cells"])
    layout = {
        "shape": np.array([NX, NY, NZ], np.uint64),
        "stencil": np.asarray(first["stencil"]).copy(),
        "weights": np.asarray(first["weights"]).copy(),
        "centre": np.asarray(first["centre"]).copy(),
        "total": np.asarray(first["total"]).copy(),
        "scaled": np.asarray(first["scaled"]).copy(),
        "scale": scale.reshape(-1) if scaled else np.zeros(0, np.float32),
        "layer_scale": np.zeros(0, np.float32),
        "types": types.reshape(-1),
        "link_start": np.concatenate(link_start),
        "state_start": np.concatenate(state_start),
        "probe_start": np.concatenate(probe_start),
        "layer_cells": np.zeros(0, np.int64),
        "flow_mask": np.zeros(0, np.uint8),
        **{k: np.zeros(0, np.float32) for k in ("keep_x", "keep_face_x", "keep_y", "keep_face_y", "keep_z",
                                                 "keep_face_z", "push_x", "push_face_x", "push_y", "push_face_y",
                                                 "push_z", "push_face_z")},  # fmt: skip
    }
    dtypes = {"special": np.int64, "link_direction": np.uint8, "state_branch": np.int32, "probe_cells": np.uint64,
              "probe_weights": np.float64}  # fmt: skip
    for name, pieces in out.items():
        layout[name] = np.concatenate(pieces).astype(dtypes.get(name, np.float32))
    return Stacked(layout, parts)


@dataclass
class Batch:
    """Many rooms with several sources each, stacked into one grid."""

    stacked: Stacked
    layouts: list[dict[str, np.ndarray]]  # each solve's own layout (room, source)
    signal: np.ndarray
    rate: float
    description: dict
    # each solve's scene: (room, grid, source, receivers), for the reference to lay out alike
    scenes: list = field(default_factory=list)


def partition(cells: list[int], world: int) -> list[list[int]]:
    """Items of sizes ``cells`` dealt to ``world`` parts, largest first, each to the part with the
    fewest cells so far (ties to the lower part): each part's list in increasing order."""
    parts: list[list[int]] = [[] for _ in range(world)]
    load = [0] * world
    for k in sorted(range(len(cells)), key=lambda k: (-cells[k], k)):
        r = min(range(world), key=lambda r: (load[r], r))
        parts[r].append(k)
        load[r] += cells[k]
    return [sorted(p) for p in parts]


def batched_rooms(
    seed: int = 0,
    *,
    rooms: int = 64,
    sources: int = 4,
    cell: float = 0.05,
    dims=(3.0, 12.0),
    absorption=(0.02, 0.5),
    receivers: int = 4,
    steps: int = 6000,
    speed_of_sound: float = 343.0,
    part: tuple[int, int] = (0, 1),
) -> Batch:
    """``rooms`` seeded shoebox rooms of dims uniform in ``dims`` metres per axis on cells of
    ``cell`` metres, each wall's absorption uniform in ``absorption`` (a real admittance by Paris's
    formula), each room with ``sources`` seeded source positions (separate solves) and
    ``receivers`` receivers, all at least 0.5 m from the walls; one 0.5 ms Gaussian drive. Every
    (room, source) is a solve of its own, and all are stacked into one grid. Room k is drawn from
    its own generator (seed, k). With ``part`` = (rank, world), only the rooms of
    :func:`partition` for that rank are built (the solves shard across GPUs with no exchange)."""
    rate = speed_of_sound / (COURANT * cell)
    sizes = [np.random.default_rng([seed, k]).uniform(dims[0], dims[1], 3) for k in range(rooms)]
    mine = partition([int(np.prod(room_grid(size, cell).shape)) for size in sizes], part[1])[part[0]]
    layouts, cells, scenes = [], [], []
    for k in mine:
        rng = np.random.default_rng([seed, k])
        size = rng.uniform(dims[0], dims[1], 3)
        betas = paris_admittance(rng.uniform(absorption[0], absorption[1], 6))
        room = shoebox(size, [Material(float(b)) for b in betas])
        points = inside_points(rng, room, size, sources + receivers, 0.5, apart=0.0)
        src, rec = points[:sources], points[sources:]
        # every receiver three cells at least from every source (the reference's cubic reading)
        for k in range(len(rec)):
            while np.min(np.linalg.norm(src - rec[k], axis=1)) < 4 * cell:
                rec[k] = inside_points(rng, room, size, 1, 0.5)[0]
        grid = room_grid(size, cell)
        for j, built in enumerate(cell_face_layouts(room, grid, list(src), rec, rate=rate)):
            layouts.append(built.layout)
            cells.append(built.air_cells)
            scenes.append((room, grid, src[j], rec))
    stacked = stack(layouts, across=sources)  # a room's solves side by side
    description = {
        "rooms": rooms,
        "rooms_here": len(mine),
        "sources_per_room": sources,
        "solves": len(layouts),
        "cell_m": cell,
        "air_cells": int(sum(cells)),
        "smallest_solve_cells": int(min(cells)),
        "largest_solve_cells": int(max(cells)),
        "stacked_grid": "x".join(str(int(v)) for v in stacked.layout["shape"]),
        "receivers_per_room": receivers,
        "steps": steps,
        "rate_hz": rate,
        "walls": "cell faces, real admittance per wall from absorption U[%g, %g]" % absorption,
        "seed": seed,
    }
    return Batch(stacked, layouts, gaussian_drive(rate, steps), rate, description, scenes)
