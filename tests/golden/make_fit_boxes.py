"""Writes tests/golden/fit_boxes.npz: the convex cases of the reference's golden fit fixtures.

The reference pins its exact fit (cut_cells.hpp, CutCells, bound as CutFit,
cpp/bindings/native_module.cpp:1465-1559) by hashing every field of eleven small cases
(tests/reference/fit_golden.npz and fit_golden.json, checked by tests/test_fit_golden.py:1-120).
Three of them are convex rooms this library's GPU fit takes: `room` (a turned box, 68 x 58 x 53
cells of 4 cm), `fold` (a box of four materials on 19.8 cm cells) and `far` (a box a thousand
million metres from the origin). This script copies their inputs and the reference's expected
hashes of the fields that the reference's compiled fit here (oracle/_ref) exposes; the tests
recompute those fields with oracle/_ref, check that they hash as the reference says, and compare
this library's fit with them.

    python tests/golden/make_fit_boxes.py [path of the reference's repository]
"""

from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

NAMES = ["room", "fold", "far"]
FIELDS = ["air", "cells/air_volume", "cells/cell", "cells/open_area", "cells/sliver", "cells/wall_area",
          "widths/0", "widths/1", "widths/2"]  # fmt: skip


def main() -> None:
    root = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ACOUSTIC_SPACES_REFERENCE", "../reference"))
    data = np.load(root / "tests" / "reference" / "fit_golden.npz")
    expected = json.loads((root / "tests" / "reference" / "fit_golden.json").read_text())
    out = {}
    for name in NAMES:
        for key in ("vertices", "faces", "materials", "grid", "shape"):
            out[f"{name}/{key}"] = data[f"{name}/{key}"]
    hashes = {name: {field: expected[name][field] for field in FIELDS} for name in NAMES}
    out["expected"] = np.array(json.dumps(hashes, sort_keys=True))
    target = Path(__file__).resolve().parent / "fit_boxes.npz"
    np.savez_compressed(target, **out)
    print(f"wrote {target}")


if __name__ == "__main__":
    main()
