"""ctypes view of the C ABI in ``include/fdtd_b200.h`` and the packing of a layout.

A layout is the dict of named NumPy arrays that the reference's
``acoustic_spaces._native.WaveSolver.layout()`` returns (cpp/include/acoustic_spaces/
fdtd.hpp:727-782 of naelolaiz/acoustic-spaces; bound at cpp/bindings/native_module.cpp:1306-1313),
or one that :mod:`acoustic_spaces_b200.layouts` builds with the same names and meanings.
:func:`pack_layout` turns it into the ``fdtd_layout`` struct the library reads, keeping the
contiguous arrays alive for as long as the struct is used.
"""

from __future__ import annotations

import ctypes
import os
from collections.abc import Mapping
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIBRARY = _HERE / "libfdtd_b200.so"

FDTD_OK = 0
FDTD_EINVAL = -1
FDTD_ECUDA = -2
FDTD_ENOMEM = -3
FDTD_ENODEV = -4
FDTD_ENONFINITE = -5
FDTD_FP32 = 0
FDTD_FP64 = 1
FDTD_FP32_COMPENSATED = 2

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)


class FdtdLayout(ctypes.Structure):
    """``struct fdtd_layout`` (include/fdtd_b200.h), field for field."""

    _fields_ = [
        ("nx", ctypes.c_uint64),
        ("ny", ctypes.c_uint64),
        ("nz", ctypes.c_uint64),
        ("stencil", ctypes.c_uint32),
        ("weight_count", ctypes.c_uint32),
        ("weights", _f32p),
        ("centre", ctypes.c_float),
        ("total", ctypes.c_float),
        ("scaled", ctypes.c_uint32),
        ("scale", _f32p),
        ("layer_scale", _f32p),
        ("types", _u8p),
        ("special_count", ctypes.c_uint64),
        ("special", _i64p),
        ("link_start", _u64p),
        ("link_count", ctypes.c_uint64),
        ("link_direction", _u8p),
        ("link_weight", _f32p),
        ("coef_a", _f32p),
        ("coef_b", _f32p),
        ("coef_inv", _f32p),
        ("source", _f32p),
        ("state_start", _u64p),
        ("state_count", ctypes.c_uint64),
        ("state_branch", _i32p),
        ("state_weight", _f32p),
        ("branch_count", ctypes.c_uint64),
        ("branch_now", _f32p),
        ("branch_before", _f32p),
        ("branch_gain", _f32p),
        ("layer_count", ctypes.c_uint64),
        ("layer_cells", _i64p),
        ("keep", _f32p * 6),
        ("push", _f32p * 6),
        ("probe_count", ctypes.c_uint64),
        ("probe_start", _u64p),
        ("probe_cells", _u64p),
        ("probe_weights", _f64p),
        ("flow_count", ctypes.c_uint64),
        ("flow_x", _f32p),
        ("flow_y", _f32p),
        ("flow_mask", _u8p),
        ("wind", _f32p * 3),
        ("loop", _f32p * 3),
    ]


class FdtdInfo(ctypes.Structure):
    """``struct fdtd_info`` (include/fdtd_b200.h)."""

    _fields_ = [
        ("cells", ctypes.c_uint64),
        ("air_cells", ctypes.c_uint64),
        ("interior_cells", ctypes.c_uint64),
        ("special_cells", ctypes.c_uint64),
        ("links", ctypes.c_uint64),
        ("branch_states", ctypes.c_uint64),
        ("layer_cells", ctypes.c_uint64),
        ("probes", ctypes.c_uint64),
        ("steps_done", ctypes.c_uint64),
        ("device_bytes", ctypes.c_uint64),
        ("precision", ctypes.c_int32),
        ("device", ctypes.c_int32),
    ]


class FdtdTiles(ctypes.Structure):
    """``struct fdtd_tiles`` (include/fdtd_b200.h)."""

    _fields_ = [
        ("shape", ctypes.c_int32),
        ("tile_x", ctypes.c_int32),
        ("tile_y", ctypes.c_int32),
        ("stages", ctypes.c_int32),
        ("planes", ctypes.c_uint64),
        ("tiles", ctypes.c_uint32),
        ("blocks_per_sm", ctypes.c_int32),
        ("concurrent", ctypes.c_int32),
        ("threads", ctypes.c_int32),
        ("cols", ctypes.c_int32),
    ]


class FdtdCutRoom(ctypes.Structure):
    """``struct fdtd_cut_room`` (include/fdtd_b200.h)."""

    _fields_ = [
        ("normals", _f64p),
        ("offsets", _f64p),
        ("open", _u8p),
        ("planes", ctypes.c_uint32),
        ("origin", ctypes.c_double * 3),
        ("cell", ctypes.c_double),
        ("nx", ctypes.c_uint64),
        ("ny", ctypes.c_uint64),
        ("nz", ctypes.c_uint64),
        ("pieces", ctypes.c_uint32),
        ("piece_plane", _u32p),
        ("piece_start", _u32p),
        ("piece_edges", _f64p),
    ]


class FdtdCutCells(ctypes.Structure):
    """``struct fdtd_cut_cells`` (include/fdtd_b200.h)."""

    _fields_ = [
        ("cells", ctypes.c_uint64),
        ("planes", ctypes.c_uint32),
        ("cell", _u64p),
        ("volume", _f64p),
        ("face_area", _f64p),
        ("cap", _f64p),
        ("bare", _f64p),
    ]


class FdtdPlaneLink(ctypes.Structure):
    """``struct fdtd_plane_link`` (include/fdtd_b200.h)."""

    _fields_ = [
        ("from_", ctypes.c_uint32),
        ("to", ctypes.c_uint32),
        ("from_plane", ctypes.c_uint64),
        ("to_plane", ctypes.c_uint64),
    ]


#: The axis tables of the matched layer, in the order of fdtd_layout.keep / .push.
KEEP = ("keep_x", "keep_face_x", "keep_y", "keep_face_y", "keep_z", "keep_face_z")
PUSH = ("push_x", "push_face_x", "push_y", "push_face_y", "push_z", "push_face_z")

#: The arrays of a layout this library reads, with their dtypes.
ARRAYS = {
    "weights": np.float32,
    "scale": np.float32,
    "layer_scale": np.float32,
    "types": np.uint8,
    "special": np.int64,
    "link_start": np.uint64,
    "link_direction": np.uint8,
    "link_weight": np.float32,
    "coef_a": np.float32,
    "coef_b": np.float32,
    "coef_inv": np.float32,
    "source": np.float32,
    "state_start": np.uint64,
    "state_branch": np.int32,
    "state_weight": np.float32,
    "branch_now": np.float32,
    "branch_before": np.float32,
    "branch_gain": np.float32,
    "layer_cells": np.int64,
    "probe_start": np.uint64,
    "probe_cells": np.uint64,
    "probe_weights": np.float64,
    **{name: np.float32 for name in KEEP + PUSH},
    "flow_x": np.float32,
    "flow_y": np.float32,
    "flow_mask": np.uint8,
    **{f"{kind}_{axis}": np.float32 for kind in ("wind", "loop") for axis in "xyz"},
}


def _ptr(array: np.ndarray | None, kind):
    if array is None or array.size == 0:
        return ctypes.cast(None, kind)
    return array.ctypes.data_as(kind)


def pack_layout(layout: Mapping[str, np.ndarray]) -> tuple[FdtdLayout, dict[str, np.ndarray]]:
    """The ``fdtd_layout`` of ``layout`` and the contiguous arrays it points into (keep the
    second alive while the first is in use)."""
    keep: dict[str, np.ndarray] = {}
    for name, dtype in ARRAYS.items():
        value = layout.get(name)
        keep[name] = np.ascontiguousarray(
            np.zeros(0, dtype) if value is None else np.asarray(value), dtype=dtype
        ).reshape(-1)
    shape = [int(v) for v in np.asarray(layout["shape"]).reshape(-1)]
    if len(shape) != 3:
        raise ValueError("the layout's shape has three sizes")
    specials = len(keep["special"])
    if specials == 0 and len(keep["link_start"]) == 0:
        keep["link_start"] = np.zeros(1, np.uint64)
        keep["state_start"] = np.zeros(1, np.uint64)
    if len(keep["link_start"]) != specials + 1 or len(keep["state_start"]) != specials + 1:
        raise ValueError("link_start and state_start have one entry more than special")
    if len(keep["probe_start"]) == 0:
        keep["probe_start"] = np.zeros(1, np.uint64)
    s = FdtdLayout()
    s.nx, s.ny, s.nz = shape
    s.stencil = int(np.asarray(layout["stencil"]).reshape(-1)[0])
    s.weight_count = len(keep["weights"])
    s.weights = _ptr(keep["weights"], _f32p)
    s.centre = float(np.asarray(layout["centre"], np.float32).reshape(-1)[0])
    s.total = float(np.asarray(layout["total"], np.float32).reshape(-1)[0])
    scaled = layout.get("scaled")
    s.scaled = int(np.asarray(scaled).reshape(-1)[0]) if scaled is not None and len(scaled) else 0
    s.scale = _ptr(keep["scale"], _f32p)
    s.layer_scale = _ptr(keep["layer_scale"], _f32p)
    s.types = _ptr(keep["types"], _u8p)
    s.special_count = specials
    s.special = _ptr(keep["special"], _i64p)
    s.link_start = _ptr(keep["link_start"], _u64p)
    s.link_count = len(keep["link_direction"])
    s.link_direction = _ptr(keep["link_direction"], _u8p)
    s.link_weight = _ptr(keep["link_weight"], _f32p)
    s.coef_a = _ptr(keep["coef_a"], _f32p)
    s.coef_b = _ptr(keep["coef_b"], _f32p)
    s.coef_inv = _ptr(keep["coef_inv"], _f32p)
    s.source = _ptr(keep["source"], _f32p)
    s.state_start = _ptr(keep["state_start"], _u64p)
    s.state_count = len(keep["state_branch"])
    s.state_branch = _ptr(keep["state_branch"], _i32p)
    s.state_weight = _ptr(keep["state_weight"], _f32p)
    s.branch_count = len(keep["branch_now"])
    s.branch_now = _ptr(keep["branch_now"], _f32p)
    s.branch_before = _ptr(keep["branch_before"], _f32p)
    s.branch_gain = _ptr(keep["branch_gain"], _f32p)
    s.layer_count = len(keep["layer_cells"])
    s.layer_cells = _ptr(keep["layer_cells"], _i64p)
    for k, name in enumerate(KEEP):
        s.keep[k] = _ptr(keep[name], _f32p)
    for k, name in enumerate(PUSH):
        s.push[k] = _ptr(keep[name], _f32p)
    s.probe_count = len(keep["probe_start"]) - 1
    s.probe_start = _ptr(keep["probe_start"], _u64p)
    s.probe_cells = _ptr(keep["probe_cells"], _u64p)
    s.probe_weights = _ptr(keep["probe_weights"], _f64p)
    s.flow_count = len(keep["flow_mask"])
    s.flow_x = _ptr(keep["flow_x"], _f32p)
    s.flow_y = _ptr(keep["flow_y"], _f32p)
    s.flow_mask = _ptr(keep["flow_mask"], _u8p)
    for a, axis in enumerate("xyz"):
        s.wind[a] = _ptr(keep[f"wind_{axis}"], _f32p)
        s.loop[a] = _ptr(keep[f"loop_{axis}"], _f32p)
    return s, keep


#: Every symbol include/fdtd_b200.h declares, with (restype, argtypes).
SIGNATURES = {
    "fdtd_abi_version": (ctypes.c_int, []),
    "fdtd_build_id": (ctypes.c_char_p, []),
    "fdtd_global_error": (ctypes.c_char_p, []),
    "fdtd_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "fdtd_device_count": (ctypes.c_int, []),
    "fdtd_device_name": (ctypes.c_int, [ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]),
    "fdtd_create": (
        ctypes.c_int,
        [ctypes.POINTER(FdtdLayout), ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
    ),
    "fdtd_run": (ctypes.c_int, [ctypes.c_void_p, _f32p, ctypes.c_uint64, _f64p]),
    "fdtd_run_device": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64],
    ),
    "fdtd_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "fdtd_stream": (ctypes.c_void_p, [ctypes.c_void_p]),
    "fdtd_set_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "fdtd_gradient": (
        ctypes.c_int,
        [ctypes.c_void_p, _f32p, ctypes.c_uint64, _f64p, ctypes.c_uint64, _f64p, _f64p, _f64p, _f64p, _f64p],
    ),
    "fdtd_gradient_noalloc": (
        ctypes.c_int,
        [ctypes.c_void_p, _f32p, ctypes.c_uint64, _f64p, ctypes.c_uint64, _f64p, _f64p, _f64p, _f64p, _f64p],
    ),
    "fdtd_layer_gradient": (ctypes.c_int, [ctypes.c_void_p, _f64p]),
    "fdtd_set_gradient_tables": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "fdtd_set_adjoint_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "fdtd_set_tape_budget": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "fdtd_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int)]),
    "fdtd_set_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "fdtd_run_linked": (
        ctypes.c_int,
        [ctypes.POINTER(ctypes.c_void_p), ctypes.c_uint32, ctypes.POINTER(FdtdPlaneLink), ctypes.c_uint32,
         ctypes.POINTER(ctypes.c_void_p), ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p), ctypes.c_uint64],
    ),
    "fdtd_set_tiles": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64]),
    "fdtd_get_tiles": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(FdtdTiles)]),
    "fdtd_set_streams": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "fdtd_set_layer_tangent": (ctypes.c_int, [ctypes.c_void_p, _f64p, ctypes.c_uint64]),
    "fdtd_layer_tangent_gradient": (ctypes.c_int, [ctypes.c_void_p, _f64p]),
    "fdtd_level_plane": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_uint64)]),
    "fdtd_test_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32]),
    "fdtd_set_tape": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "fdtd_set_coefficients": (ctypes.c_int, [ctypes.c_void_p, _f32p, _f32p, _f32p, _f32p, _f32p]),
    "fdtd_get_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint64)]),
    "fdtd_cut_convex": (ctypes.c_int, [ctypes.POINTER(FdtdCutRoom), ctypes.c_int, ctypes.POINTER(FdtdCutCells)]),
    "fdtd_cut_free": (None, [ctypes.POINTER(FdtdCutCells)]),
    "fdtd_cut_error": (ctypes.c_char_p, []),
    "fdtd_reset": (ctypes.c_int, [ctypes.c_void_p]),
    "fdtd_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "fdtd_get_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(FdtdInfo)]),
    "fdtd_read_state": (
        ctypes.c_int,
        [ctypes.c_void_p] + [ctypes.c_void_p] * 5,
    ),
}

_lib: ctypes.CDLL | None = None


def load_library(path: str | os.PathLike | None = None) -> ctypes.CDLL:
    """The built library (``libfdtd_b200.so`` beside this file), its prototypes set. Raises
    RuntimeError when it is missing: there is no other path to step the grid on."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    where = Path(path) if path is not None else LIBRARY
    if not where.exists():
        raise RuntimeError(
            f"the B200 wave stepper's CUDA library is not built ({where}): run "
            "`python -m acoustic_spaces_b200.build` (nvcc for sm_100a)"
        )
    lib = ctypes.CDLL(str(where))
    for name, (restype, argtypes) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    if lib.fdtd_abi_version() != 3:
        raise RuntimeError("the B200 wave stepper's library has another ABI version")
    if path is None:
        from acoustic_spaces_b200 import build

        if lib.fdtd_build_id().decode() != build.source_id():
            raise RuntimeError(
                f"{where} was built from other sources than those beside it: rebuild it with "
                "`python -m acoustic_spaces_b200.build`"
            )
    if path is None:
        _lib = lib
    return lib
