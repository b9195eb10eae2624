"""The benchmark's accuracy figures (bench.py): decay times and IR errors on synthetic responses."""

from __future__ import annotations

import numpy as np

import bench


def _decaying_noise(t60: float, rate: float, seconds: float, seed: int = 0) -> np.ndarray:
    # white noise under an envelope whose energy falls 60 dB in t60 seconds
    t = np.arange(int(seconds * rate)) / rate
    return np.random.default_rng(seed).standard_normal(len(t)) * np.exp(-3.0 * np.log(10.0) * t / t60)


def test_decay_times_read_a_known_reverberation_time():
    rate = 8000.0
    p = _decaying_noise(0.6, rate, 2.0)
    edt, t30 = bench.decay_times(p, rate)
    assert abs(t30 - 0.6) < 0.03 and abs(edt - 0.6) < 0.08, (edt, t30)


def test_decay_times_are_nan_where_the_curve_does_not_fall_far_enough():
    rate = 8000.0
    p = _decaying_noise(20.0, rate, 0.5)  # falls ~1.5 dB over the response
    edt, t30 = bench.decay_times(p, rate)
    assert np.isnan(edt) and np.isnan(t30)


def test_ir_errors_report_each_figure():
    rate = 8000.0
    p64 = np.stack([_decaying_noise(0.5, rate, 1.5, seed) for seed in range(3)])
    p32 = p64 * (1.0 + 1e-5) + 1e-6  # a small gain error and an offset
    e = bench.ir_errors(p32, p64, rate)
    assert e["receivers"] == 3 and 0.0 < e["ir_rel_l2_max"] < 1e-3
    # removing each receiver's mean takes the offset away, leaving the gain error
    assert e["ir_rel_l2_demeaned_max"] < e["ir_rel_l2_max"]
    assert abs(e["ir_rel_l2_demeaned_max"] - 1e-5) < 2e-6
    assert e["t30_rel_max"] < 1e-3 and e["t30_receivers"] == 3


def test_kind_bytes_count_the_compensated_increment():
    d = {"interior_cells": 10, "special_rows": 2, "links": 6, "branch_states": 3, "layer_cells": 4}
    plain, comp = bench.kind_bytes(d), bench.kind_bytes(d, "fp32c")
    assert plain["bulk"] == 120 and comp["bulk"] == 160
    assert comp["layer"] - plain["layer"] == 16 and comp["special"] - plain["special"] == 8
    assert bench.algorithmic_bytes(d) == sum(plain.values())


def test_the_reference_arm_prints_the_contracts_line():
    # bench.py --impl reference: the reference's own CPU solver on the benchmark's room (here at
    # 20 cm cells), one JSON line with the metric, a cpu_baseline describing the run and a zero-copy
    # e2e, after at least 3 warm-up steps.
    import json
    import subprocess
    import sys

    from conftest import ROOT
    from oracle.oracle import reference_native

    if reference_native() is None:
        import pytest

        pytest.skip("the reference's solver is not built")
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--cell", "0.2", "--steps", "2",
                          "--warmup", "3"], capture_output=True, text=True, timeout=600, check=True).stdout  # fmt: skip
    line = json.loads(out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == bench.UNIT and line["metric"] == bench.METRIC
    assert line["value"] > 0 and line["warmup"] >= 3 and line["higher_is_better"] is True
    cpu = line["cpu_baseline"]
    assert cpu["kind"] == "reference" and cpu["cores"] >= 1 and cpu["value"] == line["value"] and cpu["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_the_reference_arm_leaves_the_other_ranks_idle():
    # Under torchrun every rank but 0 exits at once, with nothing printed and no process group.
    import os
    import subprocess
    import sys

    from conftest import ROOT

    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT="1")
    done = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2"],
                          capture_output=True, text=True, timeout=120, env=env)  # fmt: skip
    assert done.returncode == 0 and done.stdout.strip() == ""
