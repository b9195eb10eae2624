"""Test infrastructure: the gradient of a loss of the probe series with respect to the special rows'
coefficients, by PyTorch autograd through a float64 restatement of the forward step.

This is the checker of the CUDA reverse-time stepper. It differentiates the forward scheme as the
reference steps it (special rows fdtd.hpp:860-881, interior cells fdtd.hpp:242-288, probes
fdtd.hpp:3525-3533), written here with whole-array torch operations, and shares no derivation with
the hand-written transposed operator of the CUDA library. Both stencils (7 and 19 points), with
or without a speed field (each interior cell's update scaled by its speed of sound over the
grid's, squared, as fdtd.hpp:250-262 scales it). With a matched layer it also steps the layer as
the reference does (fdtd.hpp:2242-2264: each cell its own copy of both faces on every axis; with a
speed field each cell's push scaled by its own factor) and gives the gradient in the layer's
twelve coefficient tables (keep and push of the centres and the faces per axis,
fdtd.hpp:2219-2238). The CUDA adjoint covers grids without a matched layer so far; the layer's
part of this checker is the bar for what comes next.
"""

from __future__ import annotations

import numpy as np
import torch

#: The layer's tables: per axis the centres' keep, the faces' keep (and the same for push).
KEEP = ("keep_x", "keep_face_x", "keep_y", "keep_face_y", "keep_z", "keep_face_z")
PUSH = ("push_x", "push_face_x", "push_y", "push_face_y", "push_z", "push_face_z")

# The link directions of fdtd.hpp:924-927: six axial, then the twelve edge neighbours.
_DIRECTIONS = (
    (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1),
    (-1, -1, 0), (1, -1, 0), (-1, 1, 0), (1, 1, 0), (-1, 0, -1), (1, 0, -1),
    (-1, 0, 1), (1, 0, 1), (0, -1, -1), (0, 1, -1), (0, -1, 1), (0, 1, 1),
)  # fmt: skip


class AutogradStepper:
    """The forward scheme of one layout in float64 torch, differentiable in the special rows'
    coef_b, coef_inv and the branch states' now, before, gain (one leaf per state, as the CUDA
    gradient reports them), and with a matched layer in its twelve tables (KEEP, PUSH)."""

    def __init__(self, layout) -> None:
        nx, ny, nz = (int(v) for v in layout["shape"])
        stencil = int(np.asarray(layout["stencil"]).reshape(-1)[0])
        if stencil not in (7, 19):
            raise ValueError("the stencil has 7 or 19 points")
        sy, sz = nx, nx * ny
        self.n = nx * ny * nz
        offsets = torch.tensor([x + y * sy + z * sz for x, y, z in _DIRECTIONS], dtype=torch.int64)
        d = torch.float64
        types = torch.as_tensor(np.asarray(layout["types"]))
        self.interior = torch.nonzero(types == 1).flatten()
        self.neighbours = self.interior[:, None] + offsets[None, :6]
        self.edges = self.interior[:, None] + offsets[None, 6:] if stencil == 19 else None
        weights = np.asarray(layout["weights"], np.float64)
        self.centre = float(np.asarray(layout["centre"])[0])
        self.total = float(np.asarray(layout["total"])[0])
        self.axial = float(weights[0])
        self.diagonal = float(weights[6]) if stencil == 19 else 0.0
        # A speed field: each interior cell's factor, and each layer cell's (its push's).
        scale = np.asarray(layout.get("scale", ()), np.float64)
        self.scale = torch.as_tensor(scale[self.interior.numpy()]) if len(scale) else None
        self.layer_scale = torch.as_tensor(np.asarray(layout["layer_scale"], np.float64)) if len(scale) else None
        self.special = torch.as_tensor(np.asarray(layout["special"], np.int64))
        link_start = np.asarray(layout["link_start"], np.int64)
        state_start = np.asarray(layout["state_start"], np.int64)
        specials = len(self.special)
        self.link_row = torch.as_tensor(np.repeat(np.arange(specials), np.diff(link_start)))
        direction = torch.as_tensor(np.asarray(layout["link_direction"], np.int64))
        self.link_cell = self.special[self.link_row] + offsets[direction]
        self.link_weight = torch.as_tensor(np.asarray(layout["link_weight"], np.float64))
        self.state_row = torch.as_tensor(np.repeat(np.arange(specials), np.diff(state_start)))
        self.state_weight = torch.as_tensor(np.asarray(layout["state_weight"], np.float64))
        self.coef_a = torch.as_tensor(np.asarray(layout["coef_a"], np.float64))
        self.source = torch.as_tensor(np.asarray(layout["source"], np.float64))
        branch = np.asarray(layout["state_branch"], np.int64)
        self.params = {
            "coef_b": torch.tensor(np.asarray(layout["coef_b"], np.float64), dtype=d, requires_grad=True),
            "coef_inv": torch.tensor(np.asarray(layout["coef_inv"], np.float64), dtype=d, requires_grad=True),
            "now": torch.tensor(np.asarray(layout["branch_now"], np.float64)[branch], dtype=d, requires_grad=True),
            "before": torch.tensor(np.asarray(layout["branch_before"], np.float64)[branch], dtype=d, requires_grad=True),
            "gain": torch.tensor(np.asarray(layout["branch_gain"], np.float64)[branch], dtype=d, requires_grad=True),
        }
        # The matched layer: its cells, their coordinates and strides per axis, and the tables.
        self.layer = torch.as_tensor(np.asarray(layout.get("layer_cells", np.zeros(0)), np.int64))
        self.strides = (1, sy, sz)
        if len(self.layer):
            cells = self.layer
            self.coords = (cells % nx, (cells // sy) % ny, cells // sz)
            for name in KEEP + PUSH:
                self.params[name] = torch.tensor(np.asarray(layout[name], np.float64), dtype=d, requires_grad=True)
        probe_start = np.asarray(layout["probe_start"], np.int64)
        self.probes = len(probe_start) - 1
        self.probe_row = torch.as_tensor(np.repeat(np.arange(self.probes), np.diff(probe_start)))
        self.probe_cells = torch.as_tensor(np.asarray(layout["probe_cells"], np.int64))
        self.probe_weights = torch.as_tensor(np.asarray(layout["probe_weights"], np.float64))

    def run(self, signal) -> torch.Tensor:
        p = self.params
        specials = len(self.special)
        states = len(self.state_row)
        a = torch.zeros(self.n, dtype=torch.float64)
        b = torch.zeros(self.n, dtype=torch.float64)
        wa = torch.zeros(states, dtype=torch.float64)
        wb = torch.zeros(states, dtype=torch.float64)
        cells = len(self.layer)
        # The layer's nine values per cell: the parts, and per axis the - face and the + face.
        parts = [torch.zeros(cells, dtype=torch.float64) for _ in range(3)]
        below = [torch.zeros(cells, dtype=torch.float64) for _ in range(3)]
        above = [torch.zeros(cells, dtype=torch.float64) for _ in range(3)]
        # Each layer cell's coefficients, gathered from the tables once (one gather node each,
        # whose gradient the steps accumulate).
        coef = []
        for axis in range(3) if cells else ():
            x = self.coords[axis]
            keep, keep_face = p[KEEP[2 * axis]], p[KEEP[2 * axis + 1]]
            push, push_face = p[PUSH[2 * axis]], p[PUSH[2 * axis + 1]]
            pushed = push[x] if self.layer_scale is None else push[x] * self.layer_scale
            coef.append((keep[x], pushed, keep_face[x], push_face[x], keep_face[x + 1], push_face[x + 1]))
        series = []
        for s in np.asarray(signal, np.float64):
            series.append(torch.zeros(self.probes, dtype=torch.float64).index_add(
                0, self.probe_row, self.probe_weights * b[self.probe_cells]))
            here, sums = b[self.interior], b[self.neighbours].sum(1)
            if self.scale is None:
                interior = self.centre * here + self.axial * sums - a[self.interior]
                if self.edges is not None:
                    interior = interior + self.diagonal * b[self.edges].sum(1)
            else:
                sc = self.scale
                interior = (2.0 - self.total * sc) * here + (sc * self.axial) * sums - a[self.interior]
                if self.edges is not None:
                    interior = interior + (sc * self.diagonal) * b[self.edges].sum(1)
            links = torch.zeros(specials, dtype=torch.float64).index_add(
                0, self.link_row, self.link_weight * b[self.link_cell])
            own = p["now"] * wb - p["before"] * wa
            flow = torch.zeros(specials, dtype=torch.float64).index_add(0, self.state_row, self.state_weight * own)
            previous = a[self.special]
            rows = (self.coef_a * b[self.special] + links - p["coef_b"] * previous - flow + self.source * s) * p["coef_inv"]
            w_next = wa + (rows - previous)[self.state_row] * p["gain"] + own
            new = a.index_put((self.interior,), interior).index_put((self.special,), rows)
            if cells:
                here = b[self.layer]
                total = torch.zeros(cells, dtype=torch.float64)
                for axis in range(3):
                    st = self.strides[axis]
                    keep, push, keep_lo, push_lo, keep_hi, push_hi = coef[axis]
                    below[axis] = keep_lo * below[axis] - push_lo * (here - b[self.layer - st])
                    above[axis] = keep_hi * above[axis] - push_hi * (b[self.layer + st] - here)
                    parts[axis] = keep * parts[axis] - push * (above[axis] - below[axis])
                    total = total + parts[axis]
                new = new.index_put((self.layer,), total)
            a, b, wa, wb = b, new, wb, w_next
        return torch.stack(series, 1)


class _Flushed:
    """Subnormal results flush to zero while the checker runs, forward and backward: values below
    1e-308 (ahead of the wavefront, where the stencil's reach leaves vanishing values) would slow
    the CPU's arithmetic a hundredfold; the FP64 oracle keeps them, which changes nothing at the
    checks' tolerances."""

    def __enter__(self):
        # (The flag is the calling thread's: torch's operations run on that thread alone meanwhile.)
        self.threads = torch.get_num_threads()
        torch.set_num_threads(1)
        self.set = torch.set_flush_denormal(True)

    def __exit__(self, *exc):
        if self.set:
            torch.set_flush_denormal(False)
        torch.set_num_threads(self.threads)


def gradient(layout, signal, dloss_dy) -> dict[str, np.ndarray]:
    """dL/d(coef_b, coef_inv per special row; now, before, gain per branch state; with a matched
    layer, every entry of its twelve tables) for a loss whose derivative by the probe series is
    dloss_dy (probes, steps): the vector-Jacobian product."""
    with torch.enable_grad(), _Flushed():  # also when called from inside another backward pass
        stepper = AutogradStepper(layout)
        y = stepper.run(signal)
        y.backward(torch.as_tensor(np.asarray(dloss_dy, np.float64)))
    return {k: v.grad.numpy().copy() for k, v in stepper.params.items()}


def series(layout, signal) -> np.ndarray:
    with torch.no_grad(), _Flushed():
        return AutogradStepper(layout).run(signal).numpy()
