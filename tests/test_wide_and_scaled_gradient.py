"""The reverse-time stepper on grids with a speed field or the 19-point stencil, against the
autograd checker (needs a B200), as tests/test_gpu_adjoint.py checks the plain grids.

With a speed field each interior row of the update is scaled by its own cell's factor s, and the
adjoint carries an interior cell's value as s lam, which the forward scaled sweep steps; the
19-point operator is symmetric, and the wide forward sweep steps its adjoint as it is. FP64 must
equal the checker to 1e-9 of each array's largest value; FP32 must match its directional
derivative along a random direction to 1e-3.
"""

from __future__ import annotations

import pytest
from conftest import load_golden
from test_gpu_adjoint import _assert_equal_gradients, _directional, _gradient, _problem

pytestmark = pytest.mark.gpu

# speed7, uniform099 (no branch states): a speed field; resonant19: 19 points; speed19: both
_GRIDS = ["speed7", "uniform099", "resonant19", "speed19"]


@pytest.mark.parametrize("name", _GRIDS)
def test_fp64_gradient_is_the_autograd_gradient(name):
    layout, signal, _ = load_golden(name)
    signal = signal[:300]
    target, checker = _problem(layout, signal)
    _assert_equal_gradients(_gradient(layout, signal, target, "fp64"), checker, 1e-9)


# (Not uniform099: a closed box driven by a Gaussian, its FP32 forward already 6e-4 off FP64 after
# 300 steps, so the FP32 loss's own gradient is 2e-3 off the FP64 one, the adjoint aside.)
@pytest.mark.parametrize("name", ["speed7", "resonant19", "speed19"])
def test_fp32_gradient_matches_the_autograd_gradient(name):
    layout, signal, _ = load_golden(name)
    signal = signal[:300]
    target, checker = _problem(layout, signal)
    ours = _gradient(layout, signal, target, "fp32")
    predicted, exact = _directional(ours, layout), _directional(checker, layout)
    assert abs(predicted - exact) <= 1e-3 * abs(exact), (predicted, exact)


def test_a_segmented_gradient_of_a_19_point_speed_field_is_the_whole_runs():
    # Checkpoints every 70 steps (recomputation through the wide, scaled forward kernels) against
    # one segment.
    import numpy as np

    from acoustic_spaces_b200 import B200WaveSolver

    layout, signal, _ = load_golden("speed19")
    signal = signal[:300]
    y = B200WaveSolver(layout, precision="fp64").run(signal)
    dloss = 2.0 * (y - 0.5 * y)
    whole = B200WaveSolver(layout, precision="fp64").gradient(signal, dloss, segment=0)
    pieces = B200WaveSolver(layout, precision="fp64").gradient(signal, dloss, segment=70)
    for key in whole:
        np.testing.assert_allclose(pieces[key], whole[key], rtol=1e-10, atol=1e-14 * np.abs(whole[key]).max())
