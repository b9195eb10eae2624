"""One grid stepped by several ranks: a decomposition into slabs of z-planes.

The stepping of WaveSolver::run (cpp/include/acoustic_spaces/fdtd.hpp:786-904 of
naelolaiz/acoustic-spaces) reaches one plane along z each step: the 7- and 19-point stencils, the
special rows' links (every direction of fdtd.hpp:924-927 has |dz| <= 1) and the matched layer's
faces (fdtd.hpp:2242-2264) all read the planes z-1, z and z+1 only. So rank r steps the planes
[z0, z1) of the grid on a grid of its own holding them and one ghost plane on each side that has a
neighbour: the ghost cells are solid to it (nothing of its own updates them), and after every step
each rank's first and last planes of the new pressure go to its neighbours' ghost planes. That is
one plane per neighbour per step; nothing else crosses ranks.

Every row, layer cell and probe belongs to the rank whose planes hold its cell; the boundaries
between ranks are put where no probe's cells (up to 4 planes, cubic weights) straddle them, so that
each probe's weighted sum is formed by one rank, in the layout's order. A matched-layer cell on a
rank's first plane works out the velocity on its face towards the ghost plane itself, from its
own copy — the reference keeps that face twice, once per cell (fdtd.hpp:2245), and both copies
take the same operations on the same values, so the split changes nothing. With the ghost planes
filled exactly, every rank's cells step as the whole grid's do: bit for bit.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Mapping, Sequence

import numpy as np

# Work of a step per unit of each kind, for balancing (bytes moved, as the kernels move them).
_WORK = {1: 12, 2: 40, 3: 60}


def _planes(layout: Mapping[str, np.ndarray]) -> tuple[int, int, int]:
    nx, ny, nz = (int(v) for v in np.asarray(layout["shape"]).reshape(-1))
    return nx, ny, nz


def _probe_spans(layout) -> list[tuple[int, int]]:
    """Each probe's lowest and highest plane."""
    nx, ny, _ = _planes(layout)
    start = np.asarray(layout["probe_start"], np.int64).reshape(-1)
    cells = np.asarray(layout["probe_cells"], np.int64).reshape(-1)
    spans = []
    for p in range(max(0, len(start) - 1)):
        z = cells[start[p] : start[p + 1]] // (nx * ny)
        spans.append((int(z.min()), int(z.max())) if len(z) else (0, 0))
    return spans


def partition_planes(layout: Mapping[str, np.ndarray], world: int) -> list[tuple[int, int]]:
    """The planes [z0, z1) of each of ``world`` ranks: contiguous, balanced by each plane's work,
    with no boundary inside a probe's span. Raises ValueError where that cannot be done."""
    nx, ny, nz = _planes(layout)
    if world < 1:
        raise ValueError("at least one rank")
    if world == 1:
        return [(0, nz)]
    types = np.asarray(layout["types"], np.uint8).reshape(nz, ny * nx)
    work = np.zeros(nz)
    for kind, weight in _WORK.items():
        work += weight * np.count_nonzero(types == kind, axis=1)
    cumulative = np.concatenate([[0.0], np.cumsum(work)])
    # A boundary b splits planes b-1 | b: it needs a plane below and one above on each side for
    # the ghosts, and must not cut a probe (zmin < b <= zmax).
    allowed = np.ones(nz + 1, bool)
    allowed[:2] = allowed[nz - 1 :] = False
    for lo, hi in _probe_spans(layout):
        allowed[lo + 1 : hi + 1] = False
    bounds = [0]
    for r in range(1, world):
        target = cumulative[-1] * r / world
        candidates = np.flatnonzero(allowed)
        candidates = candidates[candidates > bounds[-1] + 1]
        if len(candidates) == 0:
            raise ValueError(f"the grid's {nz} planes do not split into {world} slabs")
        b = int(candidates[np.argmin(np.abs(cumulative[candidates] - target))])
        bounds.append(b)
    bounds.append(nz)
    if any(b1 - b0 < 1 for b0, b1 in zip(bounds[:-1], bounds[1:])):
        raise ValueError(f"the grid's {nz} planes do not split into {world} slabs")
    return list(zip(bounds[:-1], bounds[1:]))


@dataclass
class Slab:
    """Rank ``rank``'s part: its planes [z0, z1) of the whole grid, held with the ghost planes
    as the planes [lo, hi) of ``layout`` (its own grid's plane q is the whole grid's lo + q), and
    the whole grid's probes it records, in order."""

    rank: int
    z0: int
    z1: int
    lo: int
    hi: int
    layout: dict
    probes: list[int]

    @property
    def below(self) -> bool:
        """Whether a rank lies below (a ghost plane at the slab's plane 0)."""
        return self.lo < self.z0

    @property
    def above(self) -> bool:
        return self.hi > self.z1


def slab(layout: Mapping[str, np.ndarray], bounds: Sequence[tuple[int, int]], rank: int) -> Slab:
    """Rank ``rank``'s grid of ``bounds`` (from :func:`partition_planes`)."""
    nx, ny, nz = _planes(layout)
    plane = nx * ny
    z0, z1 = bounds[rank]
    lo, hi = (z0 - 1 if z0 > 0 else 0), (z1 + 1 if z1 < nz else nz)
    sub: dict = {}
    for name in ("stencil", "weights", "centre", "total", "scaled", "branch_now", "branch_before", "branch_gain",
                 "keep_x", "keep_face_x", "keep_y", "keep_face_y", "push_x", "push_face_x", "push_y",
                 "push_face_y"):  # fmt: skip
        if name in layout:
            sub[name] = np.asarray(layout[name]).copy()
    sub["shape"] = np.array([nx, ny, hi - lo], np.uint64)
    for name in ("keep_z", "keep_face_z", "push_z", "push_face_z"):
        if name in layout and len(np.asarray(layout[name])):
            sub[name] = np.asarray(layout[name])[lo : hi + 1].copy()
    types = np.asarray(layout["types"], np.uint8)[lo * plane : hi * plane].copy()
    types[: (z0 - lo) * plane] = 0  # the ghost planes: solid to this rank
    types[(z1 - lo) * plane :] = 0
    sub["types"] = types
    scaled = bool(np.asarray(layout.get("scaled", [0])).reshape(-1)[0])
    scale = np.asarray(layout.get("scale", np.zeros(0, np.float32)), np.float32)
    sub["scale"] = scale[lo * plane : hi * plane].copy() if scaled else np.zeros(0, np.float32)
    base = lo * plane

    def mine(cells: np.ndarray) -> np.ndarray:
        z = cells // plane
        return (z >= z0) & (z < z1)

    # Special rows, their links and branch states.
    special = np.asarray(layout["special"], np.int64)
    link_start = np.asarray(layout["link_start"], np.int64)
    state_start = np.asarray(layout["state_start"], np.int64)
    rows = np.flatnonzero(mine(special))
    sub["special"] = special[rows] - base
    for name in ("coef_a", "coef_b", "coef_inv", "source"):
        sub[name] = np.asarray(layout[name], np.float32)[rows].copy()

    def gather(starts: np.ndarray, arrays: Sequence[str]) -> np.ndarray:
        counts = starts[rows + 1] - starts[rows]
        idx = np.concatenate([np.arange(starts[k], starts[k + 1]) for k in rows]) if len(rows) else np.zeros(0, np.int64)
        for name in arrays:
            sub[name] = np.asarray(layout[name])[idx.astype(np.int64)].copy()
        return np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)

    sub["link_start"] = gather(link_start, ("link_direction", "link_weight"))
    sub["state_start"] = gather(state_start, ("state_branch", "state_weight"))
    # Matched-layer cells.
    layer = np.asarray(layout["layer_cells"], np.int64)
    keep = mine(layer)
    sub["layer_cells"] = layer[keep] - base
    layer_scale = np.asarray(layout.get("layer_scale", np.zeros(0, np.float32)), np.float32)
    sub["layer_scale"] = layer_scale[keep].copy() if scaled else np.zeros(0, np.float32)
    # Probes whose cells all lie in the slab.
    start = np.asarray(layout["probe_start"], np.int64)
    cells = np.asarray(layout["probe_cells"], np.int64)
    weights = np.asarray(layout["probe_weights"], np.float64)
    owned, new_start, new_cells, new_weights = [], [0], [], []
    for p in range(len(start) - 1):
        c = cells[start[p] : start[p + 1]]
        if len(c) and mine(c).all():
            owned.append(p)
            new_cells.append(c - base)
            new_weights.append(weights[start[p] : start[p + 1]])
            new_start.append(new_start[-1] + len(c))
    sub["probe_start"] = np.array(new_start, np.uint64)
    sub["probe_cells"] = (np.concatenate(new_cells) if new_cells else np.zeros(0, np.int64)).astype(np.uint64)
    sub["probe_weights"] = np.concatenate(new_weights) if new_weights else np.zeros(0, np.float64)
    return Slab(rank, z0, z1, lo, hi, sub, owned)


# ---- stepping the slabs -------------------------------------------------------------------------


class Planes:
    """Access to a stepper's current pressure level, plane by plane: ``get(q)`` gives plane q of
    the slab's grid as an array (numpy for the oracle, a torch tensor on the device for the GPU),
    ``put(q, values)`` writes it."""

    def get(self, q: int):  # pragma: no cover - interface
        raise NotImplementedError

    def put(self, q: int, values) -> None:  # pragma: no cover - interface
        raise NotImplementedError


class DevicePlanes(Planes):
    """The current level of a :class:`~acoustic_spaces_b200.solver.B200WaveSolver` on its device
    (fdtd_level_plane): a plane is pitch x ny elements, contiguous."""

    def __init__(self, solver) -> None:
        import torch

        self.solver, self.torch = solver, torch

    def _view(self, q: int):
        ptr, nbytes = self.solver.level_plane(q)

        class _Array:
            __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3}

        return self.torch.as_tensor(_Array(), device=f"cuda:{self.solver.device}")

    def get(self, q: int):
        return self._view(q).clone()

    def put(self, q: int, values) -> None:
        self._view(q).copy_(values)


def step_slabs(steppers: Sequence, planes: Sequence[Planes], slabs: Sequence[Slab], signal: np.ndarray,
               step: Callable[[object, np.ndarray], np.ndarray], sync: Callable[[], None] = lambda: None) -> list[np.ndarray]:  # fmt: skip
    """Steps every slab of one grid in this process, one step at a time, filling the ghost planes
    after each step; ``step(stepper, signal_piece)`` runs a piece and returns its probes' records.
    Returns each slab's records (its probes, steps)."""
    records = [[] for _ in slabs]
    for k in range(len(signal)):
        for r, stepper in enumerate(steppers):
            records[r].append(step(stepper, signal[k : k + 1]))
        sync()
        fill_ghosts(planes, slabs, sync)
    return [np.concatenate(rec, axis=1) if rec else np.zeros((len(s.probes), 0)) for rec, s in zip(records, slabs)]


def fill_ghosts(planes: Sequence[Planes], slabs: Sequence[Slab], sync: Callable[[], None] = lambda: None) -> None:
    """Each slab's first and last planes of the current pressure into its neighbours' ghost
    planes (all slabs in this process)."""
    for r in range(len(slabs) - 1):
        lower, upper = slabs[r], slabs[r + 1]
        # lower's last plane -> upper's ghost plane 0; upper's first plane -> lower's last (ghost) plane
        planes[r + 1].put(0, planes[r].get(lower.z1 - 1 - lower.lo))
        planes[r].put(lower.hi - 1 - lower.lo, planes[r + 1].get(upper.z0 - upper.lo))
    sync()


def exchange_ghosts(planes: Planes, slab: Slab, rank: int, world: int, dist) -> None:
    """Across processes (torch.distributed: gloo with host arrays, NCCL with device tensors):
    this rank's first and last planes to its neighbours, theirs into its ghost planes. Every rank
    sends before it receives on a non-blocking pair, so that no two ranks wait on each other."""
    ops, received = [], []
    if slab.above:
        mine = planes.get(slab.z1 - 1 - slab.lo)
        other = _like(mine)
        ops += [dist.P2POp(dist.isend, _tensor(mine), rank + 1), dist.P2POp(dist.irecv, _tensor(other), rank + 1)]
        received.append((slab.hi - 1 - slab.lo, other))
    if slab.below:
        mine = planes.get(slab.z0 - slab.lo)
        other = _like(mine)
        ops += [dist.P2POp(dist.isend, _tensor(mine), rank - 1), dist.P2POp(dist.irecv, _tensor(other), rank - 1)]
        received.append((0, other))
    if ops:
        for request in dist.batch_isend_irecv(ops):
            request.wait()
    for q, values in received:
        planes.put(q, values)


def _like(values):
    return values.copy() if isinstance(values, np.ndarray) else values.clone()


def _tensor(values):
    import torch

    return values if isinstance(values, torch.Tensor) else torch.from_numpy(values)


def gather_records(slabs: Sequence[Slab], records: Sequence[np.ndarray], probes: int, steps: int) -> np.ndarray:
    """The whole grid's probe records (probes, steps) from each slab's."""
    out = np.full((probes, steps), np.nan)
    for s, rec in zip(slabs, records):
        for j, p in enumerate(s.probes):
            out[p] = rec[j]
    return out


def links(slabs: Sequence[Slab]) -> list[tuple[int, int, int, int]]:
    """The plane copies after each step, (from slab, to slab, its plane, their plane): each slab's
    first and last planes into its neighbours' ghost planes."""
    out = []
    for r in range(len(slabs) - 1):
        lower, upper = slabs[r], slabs[r + 1]
        out.append((r, r + 1, lower.z1 - 1 - lower.lo, 0))
        out.append((r + 1, r, upper.z0 - upper.lo, lower.hi - 1 - lower.lo))
    return out


def run_linked(solvers: Sequence, slabs: Sequence[Slab], signal: np.ndarray, *, device_buffers=None) -> list[np.ndarray]:
    """Steps every slab of one grid together in the library (fdtd_run_linked): the ghost planes
    are filled on the devices after each step, the host enqueues the whole run and waits once.
    Returns each slab's probe records (its probes, steps). ``device_buffers``: optional
    ``(signals, outs, stride)`` already on the devices (each solver's drive and records), for
    timing without host copies."""
    import ctypes

    import torch

    from . import _abi

    lib = _abi.load_library()
    steps = len(signal)
    if device_buffers is None:
        signals = [torch.from_numpy(np.ascontiguousarray(signal, np.float32)).to(f"cuda:{s.device}") for s in solvers]
        outs = [torch.zeros((max(1, s.probes), max(1, steps)), dtype=torch.float64, device=f"cuda:{s.device}")
                for s in solvers]  # fmt: skip
        stride = max(1, steps)
    else:
        signals, outs, stride = device_buffers
    joined = links(slabs)
    link_array = (_abi.FdtdPlaneLink * max(1, len(joined)))()
    for k, (a, b, pa, pb) in enumerate(joined):
        link_array[k].from_, link_array[k].to, link_array[k].from_plane, link_array[k].to_plane = a, b, pa, pb
    handles = (ctypes.c_void_p * len(solvers))(*[s._handle for s in solvers])
    sig_ptrs = (ctypes.c_void_p * len(solvers))(*[t.data_ptr() for t in signals])
    out_ptrs = (ctypes.c_void_p * len(solvers))(*[t.data_ptr() for t in outs])
    status = lib.fdtd_run_linked(handles, len(solvers), link_array, len(joined), sig_ptrs, steps, out_ptrs, stride)
    if status != _abi.FDTD_OK:
        message = (lib.fdtd_last_error(solvers[0]._handle) or lib.fdtd_global_error()).decode()
        raise RuntimeError(message or f"fdtd_run_linked failed ({status})")
    for s in solvers:
        s.synchronize()
    return [o[: s.probes, :steps].cpu().numpy() for o, s in zip(outs, solvers)]
