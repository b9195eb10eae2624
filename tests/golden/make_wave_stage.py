"""Writes tests/golden/wave_stage.npz: the wave stage of the reference's own pipeline, stored.

The reference's `wave_responses` (src/acoustic_spaces/engine/wave.py:1159-1178) lays a scene out
with its WaveSolver and, on the GPU path, hands the solver to `GpuWaveSolver(solver)` and calls
`run` on it. This script runs `wave_responses` on the reference's shoebox example with a recording
stepper in that slot: it keeps the layout the stepper was given, every drive it was asked to run,
and what the reference's own solver returns for each (its CPU `run`, the series the stage goes on
to post-process), and the stage's final WaveResponse signals. The GPU test steps the stored layout
through B200WaveSolver, as the plugin's registered class, and must return the stored series to the
bit, without the reference's sources on the machine.

    python tests/golden/make_wave_stage.py
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import cases  # noqa: E402


class _Recorder:
    """The GpuWaveSolver slot's contract (read solver.layout() once; run(signal) -> (probes,
    steps) float64), stepped by the reference's own solver, keeping what passed through it."""

    seen: list = []

    def __init__(self, native_solver):
        self._solver = native_solver
        self.probes = native_solver.probes
        _Recorder.seen.append({"layout": native_solver.layout(), "runs": []})

    def run(self, signal):
        out = self._solver.run(signal)
        _Recorder.seen[-1]["runs"].append((np.asarray(signal, np.float32).copy(), np.asarray(out).copy()))
        return out


def main() -> None:
    if not cases.available():
        raise SystemExit("the reference's sources and its compiled solver (oracle/_ref) are needed")
    from acoustic_spaces import Room
    from acoustic_spaces.engine import wave
    from acoustic_spaces.engine.model import TraceModel

    room = Room.from_yaml(cases.REFERENCE / "examples" / "shoebox" / "scene.yaml")
    model = TraceModel.from_room(room)
    source = np.array(room.scene.sources[0].position)
    listener = np.array(room.scene.listeners[0].position)
    common = {"max_band_hz": 63, "length_s": 0.2, "sample_rate": 48_000, "speed_of_sound": 343.0}
    wave.GpuWaveSolver = _Recorder
    wave.use_gpu = lambda device, steps=None: device == "gpu"
    wave.gpu_name = lambda: "recorder"
    responses, _ = wave.wave_responses(model, source, [listener], ["l"], device="gpu", say=lambda _: None, **common)
    (seen,) = _Recorder.seen
    out = {f"layout/{k}": np.asarray(v) for k, v in seen["layout"].items()}
    for k, (signal, series) in enumerate(seen["runs"]):
        out[f"signal/{k}"] = signal
        out[f"series/{k}"] = series
    out["response"] = np.asarray(responses[0].signals)
    target = Path(__file__).resolve().parent / "wave_stage.npz"
    np.savez_compressed(target, **out)
    print(f"wrote {target}: {len(seen['runs'])} run(s), series {[s.shape for _, s in seen['runs']]}")


if __name__ == "__main__":
    main()
