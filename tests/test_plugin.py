"""The drop-in: the plugin registers the B200 stepper under the reference's wave stage.

`wave_responses` (src/acoustic_spaces/engine/wave.py:1159-1178 of the reference) picks
`GpuWaveSolver(solver) if use_gpu(device, steps) and not solver.flowing else solver`, with the
names imported from engine/gpu.py (wave.py:105). These tests need the reference's Python sources
(the development container); without a GPU the stepper is stood in for by the oracle, through the
same layout contract, to check the plumbing end to end.
"""

from __future__ import annotations

import numpy as np
import pytest

import cases
from acoustic_spaces_b200 import plugin, solver
from oracle.oracle import OracleSolver

pytestmark = pytest.mark.skipif(not cases.available(), reason="the reference sources are not here")


@pytest.fixture
def installed():
    plugin.install()
    yield
    plugin.uninstall()


def test_install_points_the_wave_stage_at_the_b200_stepper(installed):
    from acoustic_spaces.engine import gpu, wave

    assert gpu.GpuWaveSolver is solver.B200WaveSolver
    assert wave.GpuWaveSolver is solver.B200WaveSolver
    assert wave.use_gpu is solver.use_gpu and wave.gpu_name is solver.gpu_name
    assert plugin.installed()


def test_uninstall_puts_the_reference_back():
    from acoustic_spaces.engine import gpu, wave

    before = (gpu.GpuWaveSolver, wave.GpuWaveSolver, wave.use_gpu)
    plugin.install()
    plugin.install()  # idempotent
    plugin.uninstall()
    assert (gpu.GpuWaveSolver, wave.GpuWaveSolver, wave.use_gpu) == before
    assert not plugin.installed()


def test_the_device_setting_without_a_b200(installed, monkeypatch):
    monkeypatch.setattr(solver, "gpu_name", lambda device=0: None)
    assert not solver.use_gpu("cpu")
    assert not solver.use_gpu("auto")
    with pytest.raises(ValueError, match="cpu, gpu or auto"):
        solver.use_gpu("tpu")
    with pytest.raises(ValueError, match="simulation.wave.device is gpu"):
        solver.use_gpu("gpu")


class _LayoutStepper:
    """Stands in for B200WaveSolver on a machine without a GPU: the same constructor contract
    (reads solver.layout() once) and run(), stepped by the oracle."""

    made = 0

    def __init__(self, native_solver):
        _LayoutStepper.made += 1
        self._oracle = OracleSolver(native_solver.layout())
        self.probes = self._oracle.probes

    def run(self, signal):
        return self._oracle.run(signal)


def test_wave_responses_step_through_the_registered_stepper(installed, monkeypatch):
    from acoustic_spaces import Room
    from acoustic_spaces.engine import wave
    from acoustic_spaces.engine.model import TraceModel

    shoebox = cases.REFERENCE / "examples" / "shoebox" / "scene.yaml"
    room = Room.from_yaml(shoebox)
    model = TraceModel.from_room(room)
    source = np.array(room.scene.sources[0].position)
    listener = np.array(room.scene.listeners[0].position)
    common = {"max_band_hz": 63, "length_s": 0.2, "sample_rate": 48_000, "speed_of_sound": 343.0}
    cpu, _ = wave.wave_responses(model, source, [listener], ["l"], **common)
    monkeypatch.setattr(wave, "GpuWaveSolver", _LayoutStepper)
    monkeypatch.setattr(wave, "use_gpu", lambda device, steps=None: device == "gpu")
    monkeypatch.setattr(wave, "gpu_name", lambda: "stand-in")
    _LayoutStepper.made = 0
    said = []
    on_gpu, info = wave.wave_responses(model, source, [listener], ["l"], device="gpu", say=said.append, **common)
    assert _LayoutStepper.made == 1
    assert info["wave_gpu"] == 1.0 and "stand-in" in said[0]
    # The layout stepped in float32 by the reference's operations: the responses to the bit.
    assert np.array_equal(cpu[0].signals, on_gpu[0].signals)
