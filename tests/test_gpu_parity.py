"""Parity of the B200 stepper with the reference, through the C ABI (needs a B200).

FP32 is the reference's arithmetic operation for operation, so the bar is equality to the bit:
- the probes' series against the golden fixtures (the reference's own run() on its own layouts),
  run from rest in pieces of odd and even lengths;
- the whole state (both pressure levels, both branch-velocity sets, the matched layer's nine
  values per cell) against the oracle's after the same run;
FP64 against the oracle's FP64 instantiation: the same IEEE operations in the same order, so
equal to the bit as well.
"""

from __future__ import annotations

import numpy as np
import pytest
from conftest import golden_names, load_golden

from acoustic_spaces_b200 import B200WaveSolver
from oracle.oracle import OracleSolver

pytestmark = pytest.mark.gpu
NAMES = golden_names()


def _pieces(solver, signal, cuts):
    return np.concatenate([solver.run(signal[a:b]) for a, b in zip(cuts[:-1], cuts[1:])], axis=1)


@pytest.mark.parametrize("name", NAMES)
def test_gpu_steps_every_golden_grid_as_the_reference_does(name):
    layout, signal, reference = load_golden(name)
    gpu = B200WaveSolver(layout)
    got = _pieces(gpu, signal, [0, 177, 178, len(signal)])
    assert np.array_equal(got, reference), np.abs(got - reference).max()


@pytest.mark.parametrize("name", NAMES)
def test_gpu_state_equals_the_oracles(name):
    layout, signal, _ = load_golden(name)
    gpu = B200WaveSolver(layout)
    oracle = OracleSolver(layout)
    cuts = [0, 101, len(signal)]
    a = _pieces(gpu, signal, cuts)
    b = _pieces(oracle, signal, cuts)
    assert np.array_equal(a, b)
    sa, sb = gpu.state(), oracle.state()
    for key in sa:
        assert np.array_equal(sa[key], sb[key]), key


@pytest.mark.parametrize("name", NAMES)
def test_gpu_fp64_equals_the_fp64_oracle(name):
    layout, signal, reference = load_golden(name)
    gpu = B200WaveSolver(layout, precision="fp64")
    oracle = OracleSolver(layout, "fp64")
    a = _pieces(gpu, signal, [0, 77, len(signal)])
    b = oracle.run(signal)
    assert np.array_equal(a, b), np.abs(a - b).max() / np.abs(b).max()
    sa, sb = gpu.state(), oracle.state()
    for key in sa:
        assert np.array_equal(sa[key], sb[key]), key


@pytest.mark.parametrize("name", ["resonant7", "open_layer", "fitted_open"])
def test_gpu_reset_silences_the_grid(name):
    layout, signal, reference = load_golden(name)
    gpu = B200WaveSolver(layout)
    gpu.run(signal[:123])
    gpu.reset()
    assert gpu.info().steps_done == 0
    assert np.array_equal(gpu.run(signal), reference)


def test_gpu_two_solvers_are_independent():
    layout_a, signal_a, reference_a = load_golden("resonant19")
    layout_b, signal_b, reference_b = load_golden("open_layer_speed")
    a, b = B200WaveSolver(layout_a), B200WaveSolver(layout_b)
    got_a, got_b = [], []
    for lo, hi in [(0, 200), (200, 400)]:
        got_a.append(a.run(signal_a[lo:hi]))
        got_b.append(b.run(signal_b[lo:hi]))
    got_b.append(b.run(signal_b[400:]))
    assert np.array_equal(np.concatenate(got_a, axis=1), reference_a)
    assert np.array_equal(np.concatenate(got_b, axis=1), reference_b)


def test_gpu_info_counts_the_layout():
    layout, _, _ = load_golden("fitted_open")
    gpu = B200WaveSolver(layout)
    info = gpu.info()
    types = layout["types"]
    assert info.air_cells == int(np.count_nonzero(types))
    assert info.interior_cells == int(np.count_nonzero(types == 1))
    assert info.special_cells == len(layout["special"])
    assert info.layer_cells == len(layout["layer_cells"])
    assert info.probes == gpu.probes == len(layout["probe_start"]) - 1


@pytest.mark.parametrize("name", ["resonant7", "open_layer_speed", "fitted_open"])
def test_gpu_runs_in_pieces_that_flip_the_levels(name):
    # Chunks of the captured graph (64 steps) and remainders of odd lengths, so that the levels'
    # roles flip between the graph's captures.
    layout, signal, reference = load_golden(name)
    gpu = B200WaveSolver(layout)
    cuts = [0, 1, 66, 130, 131, 259, 323, len(signal)]
    assert np.array_equal(_pieces(gpu, signal, cuts), reference)


def test_gpu_run_device_equals_run():
    import torch

    layout, signal, reference = load_golden("resonant19")
    gpu = B200WaveSolver(layout)
    sig = torch.from_numpy(signal).cuda()
    out = torch.zeros((gpu.probes, len(signal)), dtype=torch.float64, device="cuda")
    gpu.run_device(sig.data_ptr(), 200, out.data_ptr(), len(signal))
    gpu.run_device(sig.data_ptr() + 4 * 200, len(signal) - 200, out.data_ptr() + 8 * 200, len(signal))
    gpu.synchronize()
    assert np.array_equal(out.cpu().numpy(), reference)


# ---- the benchmark's room, laid out by the host builder --------------------------------------

from acoustic_spaces_b200 import layouts  # noqa: E402


def test_gpu_steps_a_polyhedral_room_as_the_oracle_does():
    # The benchmark's workload at 20 cm cells (100 x 75 x 50): 19 planes, an open face, an 8-cell
    # matched layer, resonant walls; the whole state equal to the oracle's after 300 steps.
    w = layouts.polyhedral_room(0, cell=0.2, steps=300)
    gpu = B200WaveSolver(w.built.layout)
    oracle = OracleSolver(w.built.layout)
    a = _pieces(gpu, w.signal, [0, 129, 300])
    b = oracle.run(w.signal)
    assert np.array_equal(a, b)
    sa, sb = gpu.state(), oracle.state()
    for key in sa:
        assert np.array_equal(sa[key], sb[key]), key


def test_gpu_steps_a_larger_room_as_the_oracle_does():
    # The benchmark's workload at 7 cm cells (286 x 214 x 143, 8.7M cells, its levels and types
    # well beyond a small grid's, in hundreds of tiles): the probes and the whole state equal to
    # the oracle's.
    w = layouts.polyhedral_room(0, cell=0.07, steps=120)
    gpu = B200WaveSolver(w.built.layout)
    oracle = OracleSolver(w.built.layout)
    assert np.array_equal(_pieces(gpu, w.signal, [0, 57, 120]), oracle.run(w.signal))
    sa, sb = gpu.state(), oracle.state()
    for key in sa:
        assert np.array_equal(sa[key], sb[key]), key


@pytest.fixture(scope="module")
def full_room():
    return layouts.polyhedral_room(0, steps=600)


def test_gpu_full_size_run_in_pieces_equals_one_run(full_room):
    # At the benchmark's full size (500 x 375 x 250): a run cut into pieces is the run, to the bit,
    # and a reset run repeats it.
    w = full_room
    gpu = B200WaveSolver(w.built.layout)
    whole = gpu.run(w.signal)
    gpu.reset()
    pieces = _pieces(gpu, w.signal, [0, 77, 300, 301, 600])
    assert np.array_equal(whole, pieces)
    assert np.all(np.isfinite(whole)) and np.abs(whole).max() > 0.0


def test_gpu_full_size_fp32_stays_within_1e4_of_fp64(full_room):
    # The accuracy bar on the full grid: FP32 against FP64 stepping of the same
    # layout, relative L2 of every receiver's response within 1e-4.
    w = full_room
    p32 = B200WaveSolver(w.built.layout).run(w.signal)
    p64 = B200WaveSolver(w.built.layout, precision="fp64").run(w.signal)
    # (Receivers the sound has reached in 600 steps, 14 m at its speed: the others hold only the
    # grid's numerical precursor, which single precision flushes to zero.)
    energy = np.linalg.norm(p64, axis=1)
    reached = energy > 1e-3 * energy.max()
    assert reached.sum() >= 4
    rel = np.linalg.norm(p32 - p64, axis=1)[reached] / energy[reached]
    assert rel.max() < 1e-4, rel.max()


def test_gpu_steps_a_stack_of_rooms_as_each_alone():
    # Many rooms with several sources each, stacked into one grid and stepped by one launch per
    # kind: each solve equals the oracle's run of its own layout, to the bit.
    b = layouts.batched_rooms(3, rooms=3, sources=3, cell=0.1, dims=(2.0, 5.0), steps=200)
    gpu = B200WaveSolver(b.stacked.layout)
    together = _pieces(gpu, b.signal, [0, 64, 65, 200])
    for lay, (p0, p1, _, _) in zip(b.layouts, b.stacked.parts):
        assert np.array_equal(OracleSolver(lay).run(b.signal), together[p0:p1])


def test_gpu_fp64_steps_the_plain_shoebox_as_the_fp64_oracle_does():
    # The plain box the reference runs on its CPU (6 x 4 x 3 m at 5 cm, six real walls, Courant
    # 0.99/sqrt(3)), all 4000 steps: FP64 equal to the FP64 oracle to the bit, FP32 to the oracle's
    # FP32 (the reference's arithmetic). (FP32 and FP64 part in this box's constant mode: the
    # Gaussian drive leaves net mass in a closed room, a mode the real walls do not damp, and in
    # which single precision's rounding accumulates step after step.)
    w = layouts.shoebox_room(0)
    p64 = B200WaveSolver(w.built.layout, precision="fp64").run(w.signal)
    assert np.array_equal(p64, OracleSolver(w.built.layout, "fp64").run(w.signal))
    p32 = B200WaveSolver(w.built.layout).run(w.signal)
    assert np.array_equal(p32, OracleSolver(w.built.layout).run(w.signal))


def test_gpu_autotuned_launch_shapes_step_as_the_oracle_does():
    # fdtd_autotune picks the layer and special kernels' blocks per SM by timing; every choice
    # steps each cell with the same operations, so the run still equals the oracle's to the bit.
    w = layouts.polyhedral_room(0, cell=0.2, steps=200)
    gpu = B200WaveSolver(w.built.layout, autotune=True)
    assert {"layer_blocks_per_sm", "special_blocks_per_sm", "tile_shape", "tile_planes"} <= set(gpu.launch)
    assert np.array_equal(_pieces(gpu, w.signal, [0, 64, 128, 200]), OracleSolver(w.built.layout).run(w.signal))
    with pytest.raises(ValueError, match="from rest"):
        gpu.autotune()


@pytest.mark.parametrize("precision", ["fp32", "fp64", "fp32c"])
def test_gpu_every_tile_shape_steps_as_the_oracle_does(precision):
    # The sweep's four tile shapes, each with a few planes a tile, on a room large enough for
    # tiles whose cells are all interior (they load and check no cell types): every choice equals
    # the oracle to the bit, whole state included, also when the shape changes between runs.
    w = layouts.polyhedral_room(0, box=(4.0, 3.0, 2.0), cell=0.04, steps=90)
    oracle = OracleSolver(w.built.layout, precision)
    expected = oracle.run(w.signal)
    state = oracle.state()
    for shape, planes in [(0, 8), (1, 16), (2, 32), (3, 5), (1, 64), (4, 16), (5, 8), (6, 24), (7, 16), (8, 9), (9, 32)]:
        gpu = B200WaveSolver(w.built.layout, precision=precision, autotune=False)
        gpu.set_tiles(shape, planes)
        t = gpu.tiles()
        assert (t["tile_shape"], t["tile_planes"]) == (shape, planes)
        assert t["tile_blocks_per_sm"] >= 1
        got = np.concatenate([gpu.run(w.signal[:31]), gpu.run(w.signal[31:])], axis=1)
        assert np.array_equal(got, expected), (shape, planes)
        got_state = gpu.state()
        for key in state:
            assert np.array_equal(got_state[key], state[key]), (shape, planes, key)
        gpu.close()
    # changed mid-run, between pieces of odd length
    gpu = B200WaveSolver(w.built.layout, precision=precision, autotune=False)
    pieces = []
    for (a, b), shape in zip([(0, 17), (17, 50), (50, 90)], [7, 4, 9]):
        gpu.set_tiles(shape, 12)
        pieces.append(gpu.run(w.signal[a:b]))
    assert np.array_equal(np.concatenate(pieces, axis=1), expected)
    with pytest.raises(ValueError, match="tile shape"):
        gpu.set_tiles(10, 8)


def test_gpu_an_expired_wait_is_a_status_and_the_handle_stays_usable():
    # Failure detection without a fault: a bounded wait on a flag that nothing sets gives up, the
    # error flag carries it to the host as a status, and the handle steps on as before.
    layout, signal, reference = load_golden("resonant7")
    gpu = B200WaveSolver(layout)
    with pytest.raises(RuntimeError, match="bounded wait gave up"):
        gpu.test_wait(1 << 12)
    assert np.array_equal(gpu.run(signal), reference)


def test_gpu_an_empty_run_changes_nothing():
    # A drive of no steps records nothing and leaves the state as it was: the run that follows is
    # the reference's run from rest.
    layout, signal, reference = load_golden("resonant7")
    gpu = B200WaveSolver(layout)
    assert gpu.run(signal[:0]).shape == (gpu.probes, 0)
    assert np.array_equal(gpu.run(signal), reference)


def test_gpu_steps_a_layout_without_probes_as_the_oracle_does():
    # No probes at all: nothing is recorded, and the whole state equals the oracle's.
    layout, signal, _ = load_golden("open_layer")
    layout = dict(layout)
    layout.update(probe_start=np.zeros(1, np.uint64), probe_cells=np.zeros(0, np.uint64),
                  probe_weights=np.zeros(0, np.float64))  # fmt: skip
    gpu, oracle = B200WaveSolver(layout), OracleSolver(layout)
    assert gpu.probes == 0
    assert gpu.run(signal).shape == (0, len(signal))
    oracle.run(signal)
    sa, sb = gpu.state(), oracle.state()
    for key in sa:
        assert np.array_equal(sa[key], sb[key]), key


@pytest.mark.parametrize("name", ["fitted_open", "open_layer_speed"])
def test_gpu_every_stream_arrangement_steps_as_the_reference_does(name):
    # The step's kernels on three streams, on two (the layer then the special rows beside the
    # sweep; or the special rows after the sweep, the layer beside them), on one, and on three or
    # two with the special rows at the highest priority: each gives the reference's series to the
    # bit, also when the arrangement changes between runs.
    layout, signal, reference = load_golden(name)
    for mode in (0, 1, 2, 3, 4, 5):
        gpu = B200WaveSolver(layout)
        gpu.set_streams(mode)
        assert gpu.tiles()["concurrent"] == mode
        assert np.array_equal(_pieces(gpu, signal, [0, 65, 130, len(signal)]), reference), mode
    gpu = B200WaveSolver(layout)
    pieces = []
    for (a, b), mode in zip([(0, 99), (99, 230), (230, len(signal))], [2, 4, 5]):
        gpu.set_streams(mode)
        pieces.append(gpu.run(signal[a:b]))
    assert np.array_equal(np.concatenate(pieces, axis=1), reference)
    with pytest.raises(ValueError, match="0 to 5"):
        gpu.set_streams(6)
