"""Registers the B200 stepper as the wave stage's GPU device, without editing the reference.

The wave stage picks its stepper in ``wave_responses`` (src/acoustic_spaces/engine/wave.py:1159-1178
of naelolaiz/acoustic-spaces): ``GpuWaveSolver(solver) if use_gpu(device, steps) and not
solver.flowing else solver``, with the names imported from ``acoustic_spaces.engine.gpu``
(wave.py:105). :func:`install` points those names, in both modules, at
:class:`~acoustic_spaces_b200.solver.B200WaveSolver`, :func:`~acoustic_spaces_b200.solver.use_gpu`
and :func:`~acoustic_spaces_b200.solver.gpu_name`, so that ``simulation.wave.device: gpu`` (or
``auto``) steps on the B200; :func:`uninstall` puts the originals back.
"""

from __future__ import annotations

import importlib

from acoustic_spaces_b200 import solver as _solver

_NAMES = ("GpuWaveSolver", "use_gpu", "gpu_name", "hardware_gpu")
_saved: dict[tuple[str, str], object] = {}


def _replacements() -> dict[str, object]:
    return {
        "GpuWaveSolver": _solver.B200WaveSolver,
        "use_gpu": _solver.use_gpu,
        "gpu_name": _solver.gpu_name,
        "hardware_gpu": _solver.hardware_gpu,
    }


def install() -> None:
    """Makes the reference's wave stage step on the B200 (idempotent)."""
    new = _replacements()
    for module_name in ("acoustic_spaces.engine.gpu", "acoustic_spaces.engine.wave"):
        module = importlib.import_module(module_name)
        for name in _NAMES:
            if not hasattr(module, name):
                continue
            key = (module_name, name)
            if key not in _saved:
                _saved[key] = getattr(module, name)
            setattr(module, name, new[name])


def uninstall() -> None:
    """Puts the reference's own GPU names back."""
    for (module_name, name), value in list(_saved.items()):
        setattr(importlib.import_module(module_name), name, value)
    _saved.clear()


def installed() -> bool:
    return bool(_saved)
