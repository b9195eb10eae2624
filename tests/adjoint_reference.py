"""Test infrastructure: the gradient of a loss of the probe series with respect to the special rows'
coefficients, by PyTorch autograd through a float64 restatement of the forward step.

This is the checker of the CUDA reverse-time stepper. It differentiates the forward scheme as the
reference steps it (special rows fdtd.hpp:860-881, interior cells fdtd.hpp:242-288 for the
7-point stencil, probes fdtd.hpp:3525-3533), written here with whole-array torch operations, and
shares no derivation with the hand-written transposed operator of the CUDA library. Grids of the
7-point stencil without a matched layer or a speed field only, the case the CUDA adjoint covers.
"""

from __future__ import annotations

import numpy as np
import torch

# The link directions of fdtd.hpp:924-927: six axial, then the twelve edge neighbours.
_DIRECTIONS = (
    (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1),
    (-1, -1, 0), (1, -1, 0), (-1, 1, 0), (1, 1, 0), (-1, 0, -1), (1, 0, -1),
    (-1, 0, 1), (1, 0, 1), (0, -1, -1), (0, 1, -1), (0, -1, 1), (0, 1, 1),
)  # fmt: skip


class AutogradStepper:
    """The forward scheme of one layout in float64 torch, differentiable in the special rows'
    coef_b, coef_inv and the branch states' now, before, gain (one leaf per state, as the CUDA
    gradient reports them)."""

    def __init__(self, layout) -> None:
        nx, ny, nz = (int(v) for v in layout["shape"])
        if len(layout.get("layer_cells", ())) or len(np.asarray(layout.get("scale", ()))):
            raise ValueError("the autograd stepper covers grids without a matched layer or speed field")
        if int(np.asarray(layout["stencil"]).reshape(-1)[0]) != 7:
            raise ValueError("the autograd stepper covers the 7-point stencil")
        sy, sz = nx, nx * ny
        self.n = nx * ny * nz
        offsets = torch.tensor([x + y * sy + z * sz for x, y, z in _DIRECTIONS], dtype=torch.int64)
        d = torch.float64
        types = torch.as_tensor(np.asarray(layout["types"]))
        self.interior = torch.nonzero(types == 1).flatten()
        self.neighbours = self.interior[:, None] + offsets[None, :6]
        self.centre = float(np.asarray(layout["centre"])[0])
        self.axial = float(np.asarray(layout["weights"])[0])
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
        probe_start = np.asarray(layout["probe_start"], np.int64)
        self.probes = len(probe_start) - 1
        self.probe_row = torch.as_tensor(np.repeat(np.arange(self.probes), np.diff(probe_start)))
        self.probe_cells = torch.as_tensor(np.asarray(layout["probe_cells"], np.int64))
        self.probe_weights = torch.as_tensor(np.asarray(layout["probe_weights"], np.float64))

    def run(self, signal) -> torch.Tensor:
        """The probe series (probes, steps) from a zero state, differentiable in the parameters."""
        p = self.params
        specials = len(self.special)
        states = len(self.state_row)
        a = torch.zeros(self.n, dtype=torch.float64)
        b = torch.zeros(self.n, dtype=torch.float64)
        wa = torch.zeros(states, dtype=torch.float64)
        wb = torch.zeros(states, dtype=torch.float64)
        series = []
        for s in np.asarray(signal, np.float64):
            series.append(torch.zeros(self.probes, dtype=torch.float64).index_add(
                0, self.probe_row, self.probe_weights * b[self.probe_cells]))
            interior = self.centre * b[self.interior] + self.axial * b[self.neighbours].sum(1) - a[self.interior]
            links = torch.zeros(specials, dtype=torch.float64).index_add(
                0, self.link_row, self.link_weight * b[self.link_cell])
            own = p["now"] * wb - p["before"] * wa
            flow = torch.zeros(specials, dtype=torch.float64).index_add(0, self.state_row, self.state_weight * own)
            previous = a[self.special]
            rows = (self.coef_a * b[self.special] + links - p["coef_b"] * previous - flow + self.source * s) * p["coef_inv"]
            w_next = wa + (rows - previous)[self.state_row] * p["gain"] + own
            new = a.index_put((self.interior,), interior).index_put((self.special,), rows)
            a, b, wa, wb = b, new, wb, w_next
        return torch.stack(series, 1)


def gradient(layout, signal, dloss_dy) -> dict[str, np.ndarray]:
    """dL/d(coef_b, coef_inv per special row; now, before, gain per branch state) for a loss whose
    derivative by the probe series is dloss_dy (probes, steps): the vector-Jacobian product."""
    with torch.enable_grad():  # also when called from inside another backward pass
        stepper = AutogradStepper(layout)
        y = stepper.run(signal)
        y.backward(torch.as_tensor(np.asarray(dloss_dy, np.float64)))
    return {k: v.grad.numpy().copy() for k, v in stepper.params.items()}


def series(layout, signal) -> np.ndarray:
    with torch.no_grad():
        return AutogradStepper(layout).run(signal).numpy()
