"""The wave solver's time steps on a B200, behind the reference's own stepping interface.

:class:`B200WaveSolver` is a drop-in for ``acoustic_spaces.engine.gpu.GpuWaveSolver``
(src/acoustic_spaces/engine/gpu.py:445-612 of naelolaiz/acoustic-spaces): it takes a grid that the
C++ solver (``acoustic_spaces._native.WaveSolver``) has laid out, reads its ``layout()`` once, and
:meth:`B200WaveSolver.run` does what the solver's ``run`` does — it advances one step per sample
of the drive and returns each probe's pressure before each step, probes x steps in float64 — from
the GPU's own state, which persists across calls. Stepping is done by hand-written sm_100a
kernels through the C ABI of ``include/fdtd_b200.h``; there is no other path, and a missing
library or device raises.

:func:`gpu_name`, :func:`hardware_gpu` and :func:`use_gpu` mirror the module functions of
engine/gpu.py:302-346 for this device.
"""

from __future__ import annotations

import ctypes
from collections.abc import Mapping
from typing import Literal

import numpy as np

from acoustic_spaces_b200 import _abi

Device = Literal["cpu", "gpu", "auto"]
Precision = Literal["fp32", "fp64", "fp32c"]
_PRECISIONS = {"fp32": _abi.FDTD_FP32, "fp64": _abi.FDTD_FP64, "fp32c": _abi.FDTD_FP32_COMPENSATED}


def _error(lib, handle=None) -> str:
    raw = lib.fdtd_last_error(handle) if handle else lib.fdtd_global_error()
    return (raw or b"").decode("utf-8", "replace")


def _raise(lib, status: int, handle=None) -> None:
    message = _error(lib, handle)
    if status == _abi.FDTD_EINVAL:
        raise ValueError(message)
    if status == _abi.FDTD_ENOMEM:
        raise MemoryError(message)
    raise RuntimeError(message or f"the B200 wave stepper failed ({status})")


def gpu_name(device: int = 0) -> str | None:
    """The GPU the wave solver would run on, as ``"<name> (CUDA sm_100, <memory> GiB)"``, or
    None without one (engine/gpu.py:302-311)."""
    try:
        lib = _abi.load_library()
    except (RuntimeError, OSError):
        return None
    if lib.fdtd_device_count() <= device:
        return None
    buf = ctypes.create_string_buffer(256)
    if lib.fdtd_device_name(device, buf, len(buf)) != _abi.FDTD_OK:
        return None
    return buf.value.decode()


def hardware_gpu() -> bool:
    """Whether a B200 is there to step on (engine/gpu.py:314-317)."""
    return gpu_name() is not None


def use_gpu(device: Device, steps: int | None = None) -> bool:
    """Whether the wave solver runs on the GPU for the setting ``device`` (engine/gpu.py:318-346):
    ``cpu`` never, ``gpu`` always (a ValueError without a B200), ``auto`` when there is one."""
    del steps  # a B200 steps any grid the wave stage makes faster than the host
    if device == "cpu":
        return False
    if device == "gpu":
        if not hardware_gpu():
            raise ValueError(
                "simulation.wave.device is gpu, but no B200 (CUDA sm_100) is visible: set it to "
                "cpu or auto"
            )
        return True
    if device == "auto":
        return hardware_gpu()
    raise ValueError(f"the wave solver's device must be cpu, gpu or auto, not {device!r}")


class B200WaveSolver:
    """Steps the grid of ``solver`` (a fresh or reset ``acoustic_spaces._native.WaveSolver``, or
    a layout dict with the names of its ``layout()``) on the GPU: :meth:`run` does what the
    solver's ``run`` does, from the GPU's own state.

    ``precision`` ``"fp32"`` is the reference's arithmetic, bit for bit; ``"fp64"`` steps the same
    layout in double; ``"fp32c"`` steps it in compensated single precision (each cell's pressure
    and its increment, 16 bytes of traffic per interior cell against fp64's 24), which stays
    close to fp64 over long runs where fp32's rounding drifts.

    ``autotune`` chooses the matched-layer and special-row kernels' launch shapes by timing a few
    steps of each (:meth:`autotune`); by default on grids of ``AUTOTUNE_CELLS`` cells or more,
    where a step is long enough to time. The results do not depend on it."""

    AUTOTUNE_CELLS = 1 << 22

    def __init__(self, solver, *, precision: Precision = "fp32", device: int = 0, autotune: bool | None = None) -> None:
        self._lib = lib = _abi.load_library()
        layout = solver if isinstance(solver, Mapping) else solver.layout()
        if precision not in _PRECISIONS:
            raise ValueError("precision is fp32, fp64 or fp32c")
        self.precision = precision
        packed, self._arrays = _abi.pack_layout(layout)
        handle = ctypes.c_void_p()
        status = lib.fdtd_create(
            ctypes.byref(packed),
            _PRECISIONS[precision],
            int(device),
            ctypes.byref(handle),
        )
        self._arrays = None  # borrowed only during fdtd_create
        if status != _abi.FDTD_OK:
            _raise(lib, status)
        self._handle = handle
        self.device = int(device)
        info = self.info()
        self._probes = int(info.probes)
        self.shape = tuple(int(v) for v in np.asarray(layout["shape"]).reshape(-1))
        self._branches = len(np.asarray(layout["branch_now"]).reshape(-1))
        self.launch: dict[str, int] | None = None
        if autotune or (autotune is None and int(np.prod(self.shape)) >= self.AUTOTUNE_CELLS):
            self.launch = self.autotune()

    @property
    def probes(self) -> int:
        return self._probes

    def info(self) -> _abi.FdtdInfo:
        """The solver's counts (air cells, special rows, branch states, layer cells, ...)."""
        info = _abi.FdtdInfo()
        status = self._lib.fdtd_get_info(self._handle, ctypes.byref(info))
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)
        return info

    @property
    def air_cells(self) -> int:
        return int(self.info().air_cells)

    def run(self, signal: np.ndarray) -> np.ndarray:
        """Advances one step per sample of ``signal`` (added at the source) and returns the
        pressure at every probe before each step (probes, steps). A run that does not stay finite
        returns its non-finite values, as the reference's does; the wave stage refuses it."""
        signal = np.ascontiguousarray(signal, dtype=np.float32).reshape(-1)
        steps = len(signal)
        out = np.empty((self._probes, steps), np.float64)
        if steps == 0:
            return out
        status = self._lib.fdtd_run(
            self._handle,
            signal.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
            steps,
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        )
        if status not in (_abi.FDTD_OK, _abi.FDTD_ENONFINITE):
            _raise(self._lib, status, self._handle)
        return out

    def run_device(self, signal_ptr: int, steps: int, out_ptr: int, out_stride: int) -> None:
        """Queues ``steps`` steps on device buffers (addresses): the drive at ``signal_ptr``
        (float32) and the probes' records at ``out_ptr`` (float64, probe p's step k at
        ``p * out_stride + k``). Asynchronous; :meth:`synchronize` waits."""
        status = self._lib.fdtd_run_device(self._handle, signal_ptr, steps, out_ptr, out_stride)
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)

    @property
    def stream(self) -> int:
        """The address of the solver's CUDA stream (for events and ordering)."""
        return int(self._lib.fdtd_stream(self._handle) or 0)

    def gradient(self, signal: np.ndarray, dloss_dy: np.ndarray, segment: int = 250,
                 layer_tables: bool = True) -> dict[str, np.ndarray]:  # fmt: skip
        """The gradient of a loss L of the probes' series with respect to the layout's
        coefficients, by the reverse-time stepper: the run from rest on ``signal`` gives the
        series y (probes, steps); ``dloss_dy`` is dL/dy. Returns dL/d ``coef_b``, ``coef_inv``
        (one per special row) and dL/d ``now``, ``before``, ``gain`` (one per branch state); on a
        grid with a matched layer also dL/d of its twelve tables (``keep_x``, ``keep_face_x``, ...,
        ``push_face_z``, the layout's names, fdtd.hpp:2219-2238), unless ``layer_tables`` is False
        (then the walls' gradient alone, without recording the layer's factors). The forward pass
        is recomputed in segments of ``segment`` steps from checkpoints. The solver is left at
        rest."""
        signal = np.ascontiguousarray(signal, np.float32).reshape(-1)
        steps = len(signal)
        dloss = np.ascontiguousarray(dloss_dy, np.float64).reshape(self._probes, steps)
        info = self.info()
        out = {
            "coef_b": np.zeros(int(info.special_cells)),
            "coef_inv": np.zeros(int(info.special_cells)),
            "now": np.zeros(int(info.branch_states)),
            "before": np.zeros(int(info.branch_states)),
            "gain": np.zeros(int(info.branch_states)),
        }
        f64 = ctypes.POINTER(ctypes.c_double)
        if int(info.layer_cells):
            self._lib.fdtd_set_gradient_tables(self._handle, int(bool(layer_tables)))
        status = self._lib.fdtd_gradient(
            self._handle,
            signal.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
            steps,
            dloss.ctypes.data_as(f64),
            int(segment),
            *(a.ctypes.data_as(f64) for a in out.values()),
        )
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)
        if int(info.layer_cells) and getattr(self, "_tangent", False):
            value = ctypes.c_double()
            status = self._lib.fdtd_layer_tangent_gradient(self._handle, ctypes.byref(value))
            if status != _abi.FDTD_OK:
                _raise(self._lib, status, self._handle)
            out["layer_tangent"] = float(value.value)
        elif int(info.layer_cells) and layer_tables:
            out.update(self.layer_gradient())
        return out

    def set_layer_tangent(self, tangent: Mapping[str, np.ndarray] | None) -> None:
        """A tangent of the matched layer's twelve tables: d(entry)/dθ for one parameter θ (the
        layer's damping, say: :func:`layouts.damping_tangent`), by the tables' names (``keep_x``,
        ``keep_face_x``, ..., ``push_face_z``; a missing table is 0). While it is set, :meth:`gradient`
        gives ``layer_tangent`` = dL/dθ in place of the tables' gradient, and a taped run keeps the
        few factors that needs beside the rows' trajectory, so that the gradient recomputes
        nothing. None clears it. The walls' gradient is the same."""
        if tangent is None:
            status = self._lib.fdtd_set_layer_tangent(self._handle, None, 0)
            if status != _abi.FDTD_OK:
                _raise(self._lib, status, self._handle)
            self._tangent = False
            return
        nx, ny, nz = self.shape
        lengths = [nx + 1, nx + 1, ny + 1, ny + 1, nz + 1, nz + 1]
        unknown = set(tangent) - set(_abi.KEEP + _abi.PUSH)
        if unknown:
            raise ValueError(f"no such table of the matched layer: {sorted(unknown)}")
        parts = []
        for name, n in zip(_abi.KEEP + _abi.PUSH, lengths + lengths):
            value = np.asarray(tangent.get(name, np.zeros(n)), np.float64).reshape(-1)
            if len(value) != n:
                raise ValueError(f"{name} has {len(value)} values, the grid's table has {n}")
            parts.append(value)
        flat = np.ascontiguousarray(np.concatenate(parts))
        status = self._lib.fdtd_set_layer_tangent(self._handle, flat.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                  len(flat))  # fmt: skip
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)
        self._tangent = True

    def layer_gradient(self) -> dict[str, np.ndarray]:
        """The last gradient's part in the matched layer's twelve tables, by the layout's names."""
        nx, ny, nz = self.shape
        lengths = [nx + 1, nx + 1, ny + 1, ny + 1, nz + 1, nz + 1]
        flat = np.zeros(2 * sum(lengths))
        status = self._lib.fdtd_layer_gradient(self._handle, flat.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)
        out, at = {}, 0
        for name, n in zip(_abi.KEEP + _abi.PUSH, lengths + lengths):
            out[name] = flat[at : at + n].copy()
            at += n
        return out

    def set_coefficients(self, coef_b=None, coef_inv=None, branch_now=None, branch_before=None,
                         branch_gain=None) -> None:  # fmt: skip
        """Replaces the layout's material coefficients (any of them; float32, one per special row
        for coef_b/coef_inv, one per branch for the branch terms), keeping the grid, the state and
        the adjoint's tables: the next steps and gradients are those of a solver built with them."""
        info = self.info()
        lengths = {"coef_b": info.special_cells, "coef_inv": info.special_cells}
        given = {"coef_b": coef_b, "coef_inv": coef_inv, "branch_now": branch_now,
                 "branch_before": branch_before, "branch_gain": branch_gain}  # fmt: skip
        arrays, pointers = [], []
        for name, value in given.items():
            if value is None:
                pointers.append(None)
                continue
            value = np.ascontiguousarray(value, np.float32).reshape(-1)
            if name in lengths and len(value) != int(lengths[name]):
                raise ValueError(f"{name} has {len(value)} values, the grid has {int(lengths[name])} special rows")
            if name.startswith("branch") and len(value) != self._branches:
                raise ValueError(f"{name} has {len(value)} values, the grid has {self._branches} branches")
            arrays.append(value)
            pointers.append(value.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        status = self._lib.fdtd_set_coefficients(self._handle, *pointers)
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)

    def set_tape(self, segment: int, layer_tables: bool = True) -> None:
        """With ``segment`` > 0, each :meth:`run` from rest keeps what a following
        :meth:`gradient` of that drive with that ``segment`` needs, so that the gradient does not
        run the forward pass again: the whole trajectory of the special rows and branch
        velocities where it fits the tape's budget (:meth:`set_tape_budget`; the gradient then
        recomputes nothing), else the state every ``segment`` steps (the gradient recomputes each
        segment from it). 0 turns it off. On a grid with a matched layer the trajectory serves
        only gradients without the layer's tables (``layer_tables`` False, as the following
        :meth:`gradient` must then be asked); with them the tape keeps checkpoints."""
        self._lib.fdtd_set_gradient_tables(self._handle, int(bool(layer_tables)))
        status = self._lib.fdtd_set_tape(self._handle, int(segment))
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)

    def autotune(self, trial_steps: int = 12) -> dict[str, int]:
        """Chooses the launch shapes for this grid by timing a few steps of each candidate (from
        rest; the state is reset after): the interior sweep's tile shape and planes a tile, then
        the matched-layer and special-row kernels' blocks per multiprocessor. Returns the choice
        (blocks 0: one thread a cell; the tiles as :meth:`tiles` gives them)."""
        layer, special = ctypes.c_int(), ctypes.c_int()
        status = self._lib.fdtd_autotune(self._handle, int(trial_steps), ctypes.byref(layer), ctypes.byref(special))
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)
        return {"layer_blocks_per_sm": layer.value, "special_blocks_per_sm": special.value, **self.tiles()}

    def tiles(self) -> dict[str, int]:
        """The interior sweep's tiles: shape index, cells a tile along x and y, ring stages,
        planes a tile, tiles, resident blocks a multiprocessor and threads a block."""
        t = _abi.FdtdTiles()
        status = self._lib.fdtd_get_tiles(self._handle, ctypes.byref(t))
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)
        return {"tile_shape": t.shape, "tile_x": t.tile_x, "tile_y": t.tile_y, "tile_stages": t.stages,
                "tile_planes": int(t.planes), "tiles": int(t.tiles), "tile_blocks_per_sm": t.blocks_per_sm,
                "tile_threads": t.threads, "tile_cols": t.cols, "concurrent": t.concurrent}  # fmt: skip

    def set_adjoint_launch(self, far_blocks_per_sm: int, near_blocks_per_sm: int) -> None:
        """Blocks an SM of the gradient's reverse-step launches (0: one a 128 items); results are
        the same to the bit."""
        status = self._lib.fdtd_set_adjoint_launch(self._handle, int(far_blocks_per_sm), int(near_blocks_per_sm))
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)

    def set_streams(self, concurrent: int) -> None:
        """How a step's kernels share the streams, as :meth:`autotune` may choose (1 or True: each
        kind on its own; 2: the layer and then the special rows beside the sweep; 3: the special rows
        after the sweep, the layer beside them; 0 or False: all in turn; 4 and 5: as 1 and 2 with the
        special rows at the highest stream priority); results are the same to the bit."""
        status = self._lib.fdtd_set_streams(self._handle, int(concurrent))
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)
        self.launch = {**(getattr(self, "launch", None) or {}), **self.tiles()}

    def set_tiles(self, shape: int, planes: int) -> None:
        """Sets the interior sweep's tile shape (0: 64 x 16, 1: 128 x 16, 2: 64 x 32, 3: 32 x 32)
        and planes a tile, as :meth:`autotune` would; results are the same to the bit."""
        status = self._lib.fdtd_set_tiles(self._handle, int(shape), int(planes))
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)
        self.launch = {**(getattr(self, "launch", None) or {}), **self.tiles()}

    def level_plane(self, z: int, previous: bool = False) -> tuple[int, int]:
        """The device address and byte size of plane ``z`` of the current (or previous) pressure
        level between runs: pitch x ny elements, the rows padded to 16 cells."""
        ptr, nbytes = ctypes.c_void_p(), ctypes.c_uint64()
        status = self._lib.fdtd_level_plane(self._handle, int(z), int(bool(previous)), ctypes.byref(ptr),
                                            ctypes.byref(nbytes))  # fmt: skip
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)
        return int(ptr.value or 0), int(nbytes.value)

    def test_wait(self, spins: int = 1 << 16) -> None:
        """Runs the kernels' bounded-wait failure path on its own (a wait on a flag nothing sets);
        raises RuntimeError with the status's message, as an expired wait in a step would."""
        status = self._lib.fdtd_test_wait(self._handle, int(spins))
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)

    def set_launch(self, layer_blocks_per_sm: int, special_blocks_per_sm: int) -> None:
        """Sets the matched-layer and special-row kernels' blocks per multiprocessor (0: one
        thread a cell), as :meth:`autotune` would."""
        status = self._lib.fdtd_set_launch(self._handle, int(layer_blocks_per_sm), int(special_blocks_per_sm))
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)
        self.launch = {"layer_blocks_per_sm": int(layer_blocks_per_sm), "special_blocks_per_sm": int(special_blocks_per_sm)}

    def set_tape_budget(self, nbytes: int | None) -> None:
        """The device memory the tape's trajectory may take: None for half the device memory free
        at the run, 0 for checkpoints always."""
        value = (1 << 64) - 1 if nbytes is None else int(nbytes)
        status = self._lib.fdtd_set_tape_budget(self._handle, value)
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)

    def set_timing(self, enable: bool) -> None:
        """Brackets each kernel of the following run_device steps with CUDA events."""
        status = self._lib.fdtd_set_timing(self._handle, int(bool(enable)))
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)

    def timing(self) -> dict[str, float]:
        """Milliseconds per kind of kernel summed over the steps timed since the last call, and
        the steps: {"bulk", "layer", "special", "probe", "steps"}."""
        ms = (ctypes.c_double * 4)()
        steps = ctypes.c_uint64()
        status = self._lib.fdtd_get_timing(self._handle, ms, ctypes.byref(steps))
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)
        return {"bulk": ms[0], "layer": ms[1], "special": ms[2], "probe": ms[3], "steps": int(steps.value)}

    def synchronize(self) -> None:
        status = self._lib.fdtd_synchronize(self._handle)
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)

    def reset(self) -> None:
        """Silences the grid (WaveSolver::reset, fdtd.hpp:906-915)."""
        status = self._lib.fdtd_reset(self._handle)
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)

    def state(self) -> dict[str, np.ndarray]:
        """The whole state on the host: ``current`` and ``previous`` pressures (cells), the
        ``branch_current`` and ``branch_previous`` velocities, and ``layer`` (layer cells, 9)."""
        info = self.info()
        dtype = np.float64 if self.precision == "fp64" else np.float32
        arrays = {
            "current": np.empty(int(info.cells), dtype),
            "previous": np.empty(int(info.cells), dtype),
            "branch_current": np.empty(int(info.branch_states), dtype),
            "branch_previous": np.empty(int(info.branch_states), dtype),
            "layer": np.empty((int(info.layer_cells), 9), dtype),
        }
        status = self._lib.fdtd_read_state(
            self._handle, *(a.ctypes.data_as(ctypes.c_void_p) for a in arrays.values())
        )
        if status != _abi.FDTD_OK:
            _raise(self._lib, status, self._handle)
        return arrays

    def close(self) -> None:
        handle, self._handle = getattr(self, "_handle", None), None
        if handle:
            self._lib.fdtd_destroy(handle)

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass

    def __enter__(self) -> B200WaveSolver:
        return self

    def __exit__(self, *exc) -> None:
        self.close()


__all__ = ["B200WaveSolver", "Device", "gpu_name", "hardware_gpu", "use_gpu"]
