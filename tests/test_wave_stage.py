"""The reference's wave stage, stored: the drop-in's slot stepped without the reference's sources.

tests/golden/make_wave_stage.py runs the reference's `wave_responses` (engine/wave.py:1159-1178)
on its shoebox example with a recording stepper in the `GpuWaveSolver` slot, and stores the layout
the stage handed over, the drive it ran and the series the reference's solver returned. Here the
oracle (CPU) and B200WaveSolver (the class `plugin.install()` puts in that slot, built the way the
stage builds it: from an object whose `layout()` gives the layout) must return that series to the
bit, so that the stage's post-processing receives what it receives from the reference.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import OracleSolver

STAGE = Path(__file__).resolve().parent / "golden" / "wave_stage.npz"


def _stage():
    with np.load(STAGE) as data:
        layout = {k.split("/", 1)[1]: data[k] for k in data.files if k.startswith("layout/")}
        runs = sorted(int(k.split("/")[1]) for k in data.files if k.startswith("signal/"))
        return layout, [(data[f"signal/{k}"], data[f"series/{k}"]) for k in runs]


class _Laid:
    """What the stage hands the slot: a solver whose layout() gives its arrays."""

    def __init__(self, layout):
        self._layout = layout

    def layout(self):
        return self._layout


def test_the_oracle_steps_the_stages_layout_as_the_reference_did():
    layout, runs = _stage()
    oracle = OracleSolver(layout)
    for signal, series in runs:
        assert np.array_equal(oracle.run(signal), series)


@pytest.mark.gpu
def test_gpu_the_plugins_stepper_returns_the_stages_series():
    from acoustic_spaces_b200 import solver

    assert solver.use_gpu("gpu") and solver.gpu_name() is not None
    layout, runs = _stage()
    gpu = solver.B200WaveSolver(_Laid(layout))
    assert gpu.probes == runs[0][1].shape[0]
    for signal, series in runs:
        assert np.array_equal(gpu.run(signal), series)
