"""Builds ``libfdtd_b200.so`` in-tree with nvcc for sm_100a.

``python -m acoustic_spaces_b200.build`` (or :func:`build`) compiles ``csrc/*.cu`` into one shared
library beside this file. Flags: ``--fmad=false`` so that no multiply-add is fused where the
reference's -ffp-contract=off build has none, ``-ftz=true`` so that subnormal single-precision
results flush to zero as the reference's MXCSR flush does (fdtd.hpp:316-336), and the CUDA runtime
linked statically.
"""

from __future__ import annotations

import hashlib
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
SOURCES = sorted((HERE / "csrc").glob("*.cu"))
OUTPUT = HERE / "libfdtd_b200.so"
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--fmad=false", "-ftz=true", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC,-O2", "-shared", "-cudart", "static",
]  # fmt: skip


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc not found: the B200 wave stepper is built with the CUDA toolkit")
    return found


def dependencies() -> list[Path]:
    """Every file the library is compiled from."""
    csrc = HERE / "csrc"
    return sorted([*csrc.glob("*.cu"), *csrc.glob("*.cuh"), *csrc.glob("*.h"), *(ROOT / "include").glob("*.h")])


def source_id() -> str:
    """A digest of the sources' names and contents and of the flags: the library carries the one
    it was built from (fdtd_build_id), so that a library built from other sources is refused."""
    digest = hashlib.sha256(" ".join(FLAGS).encode())
    for path in dependencies():
        digest.update(path.name.encode() + b"\0" + path.read_bytes())
    return digest.hexdigest()[:32]


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compiles the library unless it is newer than its sources; returns its path."""
    deps = dependencies() + [Path(__file__)]
    if not force and OUTPUT.exists():
        built = OUTPUT.stat().st_mtime
        if all(p.stat().st_mtime <= built for p in deps):
            return OUTPUT
    cmd = [nvcc(), *FLAGS, f'-DFDTD_BUILD_ID="{source_id()}"', f"-I{ROOT / 'include'}", "-o", str(OUTPUT),
           *map(str, SOURCES)]  # fmt: skip
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return OUTPUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
