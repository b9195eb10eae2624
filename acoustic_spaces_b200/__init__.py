"""acoustic_spaces_b200: the time stepping of acoustic-spaces' low-frequency wave solver on a
B200 (sm_100a), as a drop-in for the wave stage's GPU stepper.

- :class:`B200WaveSolver` — ``GpuWaveSolver``'s interface over the C ABI of include/fdtd_b200.h.
- :func:`gpu_name`, :func:`hardware_gpu`, :func:`use_gpu` — engine/gpu.py's device functions.
- :mod:`acoustic_spaces_b200.plugin` — ``install()`` registers the stepper with the reference's
  wave stage.
- :mod:`acoustic_spaces_b200.layouts` — grid layouts of synthetic rooms, built on the host.
- :mod:`acoustic_spaces_b200.build` — the nvcc build of the library.
"""

from acoustic_spaces_b200.solver import B200WaveSolver, gpu_name, hardware_gpu, use_gpu

__all__ = ["B200WaveSolver", "gpu_name", "hardware_gpu", "use_gpu"]
