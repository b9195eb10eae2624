"""The C ABI without a GPU: the library loads, exports every function include/fdtd_b200.h
declares, and refuses bad layouts on the host (before any device is touched) with the reference's
wording; the Python wrapper maps the statuses to the reference's exceptions."""

from __future__ import annotations

import ctypes
import re

import numpy as np
import pytest
from conftest import ROOT, load_golden

from acoustic_spaces_b200 import B200WaveSolver, _abi

HEADER = (ROOT / "include" / "fdtd_b200.h").read_text()
DECLARED = sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(fdtd_\w+)\s*\(", HEADER, re.M)))


def test_the_header_declares_the_boundary():
    assert {"fdtd_create", "fdtd_run", "fdtd_reset", "fdtd_destroy", "fdtd_last_error"} <= set(DECLARED)


@pytest.mark.parametrize("name", DECLARED)
def test_the_library_exports_every_declared_function(name):
    lib = ctypes.CDLL(str(_abi.LIBRARY))
    assert hasattr(lib, name)
    assert name in _abi.SIGNATURES


def test_the_abi_version():
    assert _abi.load_library().fdtd_abi_version() == 3


def _create(layout, precision=_abi.FDTD_FP32):
    lib = _abi.load_library()
    packed, keep = _abi.pack_layout(layout)
    handle = ctypes.c_void_p()
    status = lib.fdtd_create(ctypes.byref(packed), precision, 0, ctypes.byref(handle))
    if status == _abi.FDTD_OK:
        lib.fdtd_destroy(handle)
    return status, lib.fdtd_global_error().decode()


def _bad(**changes):
    layout, _, _ = load_golden("resonant7")
    layout = dict(layout)
    layout.update(changes)
    return layout


@pytest.mark.parametrize(
    "changes, message",
    [
        ({"stencil": np.array([9], np.uint64)}, "the stencil has 7 or 19 points"),
        ({"flow_mask": np.ones(4, np.uint8)}, "one mask per cell"),
        ({"shape": np.array([2, 14, 12], np.uint64)}, "the grid is too small"),
        ({"shape": np.array([70000, 70000, 12], np.uint64)}, "32-bit indices"),
    ],
)
def test_the_library_refuses_what_the_reference_refuses(changes, message):
    status, error = _create(_bad(**changes))
    assert status == _abi.FDTD_EINVAL
    assert message in error


def test_an_out_of_grid_special_cell_is_refused():
    layout = _bad()
    special = layout["special"].copy()
    special[3] = 10**9
    status, error = _create(dict(layout, special=special))
    assert status == _abi.FDTD_EINVAL and "outside the grid" in error


def test_a_link_off_the_grid_is_refused():
    layout = _bad()
    special = layout["special"].copy()
    special[0] = 0  # a corner cell: its -x link leaves the grid
    types = layout["types"].copy()
    types[layout["special"][0]] = 0
    types[0] = 2
    direction = layout["link_direction"].copy()
    direction[: int(layout["link_start"][1])] = 0
    status, error = _create(dict(layout, special=special, link_direction=direction, types=types))
    assert status == _abi.FDTD_EINVAL and "links outside the grid" in error


def test_an_unknown_link_direction_is_refused():
    layout = _bad()
    direction = layout["link_direction"].copy()
    direction[5] = 18
    status, error = _create(dict(layout, link_direction=direction))
    assert status == _abi.FDTD_EINVAL and "direction" in error


def test_an_interior_cell_on_the_edge_is_refused():
    layout = _bad()
    types = layout["types"].copy()
    types[0] = 1
    status, error = _create(dict(layout, types=types))
    assert status == _abi.FDTD_EINVAL and "edge" in error


def test_a_special_cell_of_another_type_is_refused():
    layout = _bad()
    types = layout["types"].copy()
    types[layout["special"][7]] = 1
    status, error = _create(dict(layout, types=types))
    assert status == _abi.FDTD_EINVAL and "type is not special" in error


def test_a_special_cell_listed_twice_is_refused():
    layout = _bad()
    special = layout["special"].copy()
    special[1] = special[0]
    status, error = _create(dict(layout, special=special))
    assert status == _abi.FDTD_EINVAL and "twice" in error


def test_a_probe_off_the_grid_is_refused():
    layout = _bad()
    cells = layout["probe_cells"].copy()
    cells[0] = 10**9
    status, error = _create(dict(layout, probe_cells=cells))
    assert status == _abi.FDTD_EINVAL and "probe" in error


def test_a_branch_state_without_a_branch_is_refused():
    layout = _bad()
    branch = layout["state_branch"].copy()
    branch[0] = 99
    status, error = _create(dict(layout, state_branch=branch))
    assert status == _abi.FDTD_EINVAL and "branch" in error


def test_a_layer_cell_on_the_edge_is_refused():
    layout, _, _ = load_golden("open_layer")
    cells = layout["layer_cells"].copy()
    cells[0] = 0
    status, error = _create(dict(layout, layer_cells=cells))
    assert status == _abi.FDTD_EINVAL and "matched-layer" in error


def test_a_bad_precision_is_refused():
    layout, _, _ = load_golden("resonant7")
    status, error = _create(layout, precision=7)
    assert status == _abi.FDTD_EINVAL and "precision" in error


def test_the_wrapper_raises_value_error_on_refusals():
    with pytest.raises(ValueError, match="7 or 19"):
        B200WaveSolver(_bad(stencil=np.array([5], np.uint64)))


def test_pack_layout_keeps_counts():
    layout, _, _ = load_golden("fitted_open")
    packed, keep = _abi.pack_layout(layout)
    assert packed.special_count == len(layout["special"])
    assert packed.link_count == len(layout["link_direction"])
    assert packed.layer_count == len(layout["layer_cells"])
    assert packed.probe_count == len(layout["probe_start"]) - 1
    assert (packed.nx, packed.ny, packed.nz) == tuple(int(v) for v in layout["shape"])
    assert packed.keep[1][0] == layout["keep_face_x"][0]


@pytest.mark.skipif(_abi.load_library().fdtd_device_count() > 0, reason="a GPU is present")
def test_without_a_device_creation_says_so():
    layout, _, _ = load_golden("resonant7")
    status, error = _create(layout)
    assert status == _abi.FDTD_ENODEV and "no CUDA device" in error
    with pytest.raises(RuntimeError, match="CUDA device"):
        B200WaveSolver(layout)


def test_the_loader_refuses_a_library_built_from_other_sources(monkeypatch):
    # The library carries the digest of the sources it was built from; a stale build is refused
    # rather than run.
    from acoustic_spaces_b200 import build

    assert _abi.load_library().fdtd_build_id().decode() == build.source_id()
    monkeypatch.setattr(_abi, "_lib", None)
    monkeypatch.setattr(build, "source_id", lambda: "not-these-sources")
    with pytest.raises(RuntimeError, match="built from other sources"):
        _abi.load_library()


@pytest.mark.parametrize("bad", [0.0, 1.5, float("nan")])
def test_a_speed_outside_its_range_is_refused(bad):
    # A cell's scale is its speed ratio squared, the ratio in (0, 1] (fdtd.hpp:415-425).
    layout, _, _ = load_golden("speed7")
    scale = np.asarray(layout["scale"], np.float32).copy()
    scale[len(scale) // 2] = bad
    status, error = _create(dict(layout, scale=scale))
    assert status == _abi.FDTD_EINVAL and "lies in (0, 1]" in error
    assert _create(layout)[0] != _abi.FDTD_EINVAL  # the golden layout itself passes the check


@pytest.mark.parametrize("name", ["wind_plain", "wind_round"])
def test_moving_air_is_checked_before_the_device(name):
    # The reference's wind grids pass; the compensated form refuses moving air; a moving cell
    # whose carry would read beyond the grid's edge is refused (the round form reads two cells
    # either side along every axis).
    layout, _, _ = load_golden(name)
    assert _create(layout)[0] != _abi.FDTD_EINVAL
    status, error = _create(layout, _abi.FDTD_FP32_COMPENSATED)
    assert status == _abi.FDTD_EINVAL and "still air only" in error
    nx, ny, _ = (int(v) for v in layout["shape"])
    types = np.asarray(layout["types"])
    edge = [i for i in np.flatnonzero(types) if i % nx == 1][0]
    mask = np.asarray(layout["flow_mask"]).copy()
    changed = dict(layout, flow_mask=mask)
    if name == "wind_round":
        mask[edge] = 1
    else:
        mask[edge] = 15  # x's four bits: two cells either side along x
        fx = np.asarray(layout["flow_x"], np.float32).copy()
        fx[edge] = 0.1
        changed["flow_x"] = fx
    status, error = _create(changed)
    assert status == _abi.FDTD_EINVAL and "reads outside the grid" in error
