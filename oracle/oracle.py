"""ORACLE / TEST INFRASTRUCTURE ONLY — the checker, never the product.

Only ``tests/``, ``__graft_entry__.smoke()`` and the benchmark's CPU-baseline leg
(``bench.py --impl reference`` and its ``cpu_baseline`` key) import this module.

Two CPU checkers of the wave solver's time stepping (cpp/include/acoustic_spaces/fdtd.hpp:786-904
of naelolaiz/acoustic-spaces):

- :func:`reference_native` — the reference's own, unmodified C++ solver (its headers compiled by
  ``oracle/Makefile`` into ``oracle/_ref/``, bound by ``ref_native.cpp``), with the reference's
  Python constructor: ``WaveSolver(bvh, face_material, beta, branches, ...)``, ``run``,
  ``reset``, ``layout``. :func:`reference_python` also makes the reference's Python package
  (``acoustic_spaces``) importable with it, where the reference sources are present (the
  development container only).
- :class:`OracleSolver` — the project's C restatement (``fdtd_oracle.c``) over a layout dict, in
  float (bit-exact with the reference) or double (the FP64 oracle).

Parity of the restatement is pinned by ``tests/test_oracle.py``: against the reference's run() on
the reference's own layouts, and against the golden fixtures of ``tests/golden/``.
"""

from __future__ import annotations

import ctypes
import importlib.util
import os
import subprocess
import sys
import sysconfig
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
#: The reference's sources: ACOUSTIC_SPACES_REFERENCE, else a checkout named "reference" beside
#: this repository.
REFERENCE = Path(os.environ.get("ACOUSTIC_SPACES_REFERENCE", HERE.parent.parent / "reference")).resolve()
REF_SO = HERE / "_ref" / f"_native{sysconfig.get_config_var('EXT_SUFFIX')}"
ORACLE_SO = HERE / "libfdtd_oracle.so"

ORACLE_FP32 = 0
ORACLE_FP64 = 1
ORACLE_FP32C = 2
#: Grids of this many cells or more step on oracle_threads() host threads (ORACLE_PARALLEL_CELLS).
PARALLEL_CELLS = 1 << 16
PRECISIONS = {"fp32": ORACLE_FP32, "fp64": ORACLE_FP64, "fp32c": ORACLE_FP32C}


def build(reference: bool = True) -> None:
    """Compiles the C restatement, and the reference's solver where its sources are present."""
    targets = ["oracle"]
    if reference and (REFERENCE / "cpp" / "include").is_dir():
        targets.append("ref")
    subprocess.run(
        ["make", "-s", "-C", str(HERE), f"REFERENCE={REFERENCE}", f"PYTHON={sys.executable}", *targets],
        check=True,
    )


_oracle_lib: ctypes.CDLL | None = None


def load_oracle() -> ctypes.CDLL:
    global _oracle_lib
    if _oracle_lib is None:
        if not ORACLE_SO.exists():
            build(reference=False)
        lib = ctypes.CDLL(str(ORACLE_SO))
        lib.oracle_create.restype = ctypes.c_int
        lib.oracle_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        lib.oracle_run.restype = ctypes.c_int
        lib.oracle_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
        lib.oracle_reset.restype = ctypes.c_int
        lib.oracle_reset.argtypes = [ctypes.c_void_p]
        lib.oracle_destroy.restype = None
        lib.oracle_destroy.argtypes = [ctypes.c_void_p]
        lib.oracle_threads.restype = ctypes.c_int
        lib.oracle_threads.argtypes = []
        lib.oracle_level.restype = ctypes.c_void_p
        lib.oracle_level.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.oracle_read_state.restype = ctypes.c_int
        lib.oracle_read_state.argtypes = [ctypes.c_void_p] * 6
        lib.oracle_error.restype = ctypes.c_char_p
        lib.oracle_error.argtypes = []
        _oracle_lib = lib
    return _oracle_lib


class OracleSolver:
    """The C restatement of WaveSolver::run over a layout dict: ``run(signal)`` returns the probes'
    pressures before each step (probes, steps), the state persisting across calls."""

    def __init__(self, layout, precision: str = "fp32") -> None:
        from acoustic_spaces_b200._abi import pack_layout  # the layout struct of include/fdtd_b200.h

        self._lib = lib = load_oracle()
        self.precision = precision
        packed, arrays = pack_layout(layout)
        handle = ctypes.c_void_p()
        status = lib.oracle_create(
            ctypes.byref(packed), PRECISIONS[precision], ctypes.byref(handle)
        )
        del arrays
        if status != 0:
            raise ValueError(lib.oracle_error().decode())
        self._handle = handle
        self.probes = len(layout["probe_start"]) - 1
        self.cells = int(np.prod(np.asarray(layout["shape"], np.int64)))
        self.states = len(layout["state_branch"])
        self.layers = len(layout["layer_cells"])

    def run(self, signal) -> np.ndarray:
        signal = np.ascontiguousarray(signal, np.float32).reshape(-1)
        out = np.empty((self.probes, len(signal)), np.float64)
        if len(signal):
            self._lib.oracle_run(self._handle, signal.ctypes.data, len(signal), out.ctypes.data)
        return out

    def reset(self) -> None:
        self._lib.oracle_reset(self._handle)

    def level_pointer(self, which: int = 0) -> int:
        """The address of the current (0) or previous (1) pressure level, between runs."""
        return int(self._lib.oracle_level(self._handle, which))

    def state(self) -> dict[str, np.ndarray]:
        dtype = np.float64 if self.precision == "fp64" else np.float32
        arrays = {
            "current": np.empty(self.cells, dtype),
            "previous": np.empty(self.cells, dtype),
            "branch_current": np.empty(self.states, dtype),
            "branch_previous": np.empty(self.states, dtype),
            "layer": np.empty((self.layers, 9), dtype),
        }
        self._lib.oracle_read_state(self._handle, *(a.ctypes.data for a in arrays.values()))
        return arrays

    def __del__(self) -> None:
        handle = getattr(self, "_handle", None)
        if handle:
            self._lib.oracle_destroy(handle)
            self._handle = None


_native = None


def reference_native():
    """The reference's own solver module (``oracle/_ref/_native``), built on first use where the
    reference sources are present; None where it cannot be had."""
    global _native
    if _native is not None:
        return _native
    if not REF_SO.exists():
        if not (REFERENCE / "cpp" / "include").is_dir():
            return None
        build(reference=True)
    spec = importlib.util.spec_from_file_location("_native", REF_SO)
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    _native = module
    return module


def reference_python():
    """The reference's Python package ``acoustic_spaces`` with its ``_native`` core taken from
    :func:`reference_native`, or None where the reference sources are absent."""
    src = REFERENCE / "src"
    native = reference_native()
    if native is None or not (src / "acoustic_spaces").is_dir():
        return None
    if str(src) not in sys.path:
        sys.path.insert(0, str(src))
    sys.modules["acoustic_spaces._native"] = native
    import acoustic_spaces

    acoustic_spaces._native = native
    return acoustic_spaces
