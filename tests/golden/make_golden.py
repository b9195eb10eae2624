"""Writes the golden fixtures of the wave solver's time stepping: ``python tests/golden/make_golden.py
[case ...]`` (every case when none is named).

For each case of ``tests/cases.py`` (small grids laid out by the reference's own C++ solver,
naelolaiz/acoustic-spaces cpp/include/acoustic_spaces/fdtd.hpp, compiled unmodified by
``oracle/Makefile``), it stores in ``<case>.npz``:

- the grid's layout, as ``WaveSolver.layout()`` gives it (fdtd.hpp:727-782), under ``layout/<name>``;
- ``signal``: the drive, one float32 per step;
- ``reference``: the reference's ``WaveSolver.run(signal)`` from rest — each probe's pressure before
  each step, float64 (probes, steps), computed by the reference's own code in this container.

The reference sources exist only where the fixtures are made; the fixtures travel with the tests,
so that machines without the reference check parity against the reference's own numbers.
"""

from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE.parent))

import cases  # noqa: E402

#: The layout arrays the stepper reads (moving-air arrays are empty in still air and left out).
KEEP = (
    "shape", "stencil", "weights", "centre", "total", "scaled", "scale", "layer_scale", "types",
    "special", "link_start", "link_direction", "link_weight", "coef_a", "coef_b", "coef_inv",
    "source", "state_start", "state_branch", "state_weight", "branch_now", "branch_before",
    "branch_gain", "layer_cells", "keep_x", "keep_face_x", "keep_y", "keep_face_y", "keep_z",
    "keep_face_z", "push_x", "push_face_x", "push_y", "push_face_y", "push_z", "push_face_z",
    "probe_start", "probe_cells", "probe_weights", "flow_mask", "flow_x", "flow_y", "wind_x", "wind_y", "wind_z",
    "loop_x", "loop_y", "loop_z",
)  # fmt: skip


def main(names: list[str]) -> None:
    """Writes the fixtures of ``names`` (every case when empty), keeping the others' entries."""
    if not cases.available():
        raise SystemExit("the reference sources are needed to make the golden fixtures")
    path = HERE / "manifest.json"
    manifest = json.loads(path.read_text()) if path.exists() else {}
    for name in names or cases.CASES:
        solver, signal = cases.build_case(name)
        layout = solver.layout()
        reference = solver.run(signal)
        arrays = {f"layout/{k}": np.asarray(layout[k]) for k in KEEP if k in layout}
        arrays["signal"] = signal
        arrays["reference"] = reference
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        manifest[name] = {
            "shape": [int(v) for v in layout["shape"]],
            "stencil": int(layout["stencil"][0]),
            "steps": len(signal),
            "specials": len(layout["special"]),
            "branch_states": len(layout["state_branch"]),
            "layer_cells": len(layout["layer_cells"]),
            "probes": len(layout["probe_start"]) - 1,
            "scaled": int(layout["scaled"][0]),
            "fitted_walls": bool(solver.fitted_walls),
            "air_cells": int(solver.air_cells),
            "reference_sha256": hashlib.sha256(reference.tobytes()).hexdigest(),
        }
        print(name, manifest[name]["shape"], manifest[name]["reference_sha256"][:12])
    manifest = {name: manifest[name] for name in cases.CASES if name in manifest}
    path.write_text(json.dumps(manifest, indent=1) + "\n")


if __name__ == "__main__":
    main(sys.argv[1:])
