#!/usr/bin/env python
"""Benchmark of the B200 wave stepper: FDTD Gcell-updates/s on the polyhedral-room workload.

Workload (the FP32 forward configuration with walls and a matched layer): a seeded convex
polyhedral room of 12 to 20 planar faces inscribed in 20 x 15 x 10 m, open through one face into
the air round it, on a 500 x 375 x 250 grid of 4 cm cells (46.9M cells) with an 8-cell matched
layer inside the grid's edge; every wall a 2-pole admittance (beta and one resonant branch);
1 source, 16 receivers; built on the host by acoustic_spaces_b200.layouts with the reference's
rules for walls on cell faces (the tests check it against the reference's own layouts).

A step is one time step of the whole grid (WaveSolver::run's loop body, fdtd.hpp:838-886): probe
records, interior air, special rows with their branch states, and the matched layer.

``python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]`` prints one JSON
line. ``value`` is air cells x steps / device time of K steps with every input resident in HBM
(CUDA events on the solver's own stream; max over ranks); ``e2e`` is the same metric through the
public API (``B200WaveSolver.run`` on a host drive, its probe series back on the host);
``roofline`` relates the step kernel's algorithmic bytes per launch to the measured HBM peak;
``cpu_baseline`` is the reference's own CPU solver (oracle/_ref, the reference's unmodified C++)
timed on the host's cores on a bounded sample of the same workload. Under torchrun each rank steps
its own replica of the room (weak scaling); ``--slabs`` splits the one grid into z-slabs across the
ranks instead, one plane swapped with each neighbour per step (strong scaling), and the batched
rooms shard their solves by cell count. ``--impl reference`` times the reference's CPU solver alone
and prints its line. ``--workload`` picks the other configurations (the plain FP64 box, the outdoor
half-space, the batched rooms, the adjoint fit).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "FDTD Gcell-updates/s (+HBM roofline %) at stated IR error vs FP64; adjoint/fwd"
UNIT = "Gcell-updates/s"

# Algorithmic bytes of one step per unit of each kind (FP32): what a step must move at least.
BYTES_INTERIOR = 12  # read p, read p-, write p+
BYTES_SPECIAL = 40  # read p, read/write p-, coef_a/b/inv/source, its index and two table starts
BYTES_LINK = 5  # direction and weight
BYTES_STATE = 28  # read/write w-, read w, its four coefficients
# A layer cell keeps three pressure parts and, on the cell below each face, one velocity per
# face (the reference's nine values per cell hold every face twice, 84 B):
BYTES_LAYER = 60  # read p, write p+, read/write three parts, read/write three faces, its index


# Compensated single precision moves each cell's increment besides its pressure: an interior cell
# reads p and its increment and writes both (16 B); a special row reads and writes the increment
# in place of reading and writing p- and writes p+ (+4 B); a layer cell writes its increment (+4 B).
EXTRA_COMPENSATED = {"interior": 4, "special": 4, "layer": 4}


def kind_bytes(d: dict, precision: str = "fp32") -> dict:
    """Each step kernel's algorithmic bytes per launch."""
    extra = EXTRA_COMPENSATED if precision == "fp32c" else {"interior": 0, "special": 0, "layer": 0}
    return {
        "bulk": (BYTES_INTERIOR + extra["interior"]) * d["interior_cells"],
        "layer": (BYTES_LAYER + extra["layer"]) * d["layer_cells"],
        "special": (BYTES_SPECIAL + extra["special"]) * d["special_rows"]
        + BYTES_LINK * d["links"]
        + BYTES_STATE * d["branch_states"],
    }


def algorithmic_bytes(d: dict, precision: str = "fp32") -> int:
    return sum(kind_bytes(d, precision).values())


def decay_times(p: np.ndarray, rate: float) -> tuple[float, float]:
    """EDT and T30 (s) of one receiver's broadband response: the backward-integrated (Schroeder)
    decay of p^2 in dB, a least-squares line from its first sample at or below 0 dB (EDT) or -5 dB
    (T30) to its first at or below -10 or -35 dB, -60 dB over its slope (the ranges of ISO 3382,
    as src/acoustic_spaces/parameters.py:55 and :266-296 of the reference fit them, here without
    its estimate of the energy past the response's end). NaN where the curve does not fall so far
    within the first 80 % of the response: without that estimate every curve plunges at the end,
    which is the response's truncation, not its decay (parameters.py:454-462 refuses such curves)."""
    e = np.cumsum((p * p)[::-1])[::-1]
    if e[0] <= 0:
        return float("nan"), float("nan")
    with np.errstate(divide="ignore"):
        level = 10.0 * np.log10(np.maximum(e, 0.0) / e[0])
    t = np.arange(len(p)) / rate
    out = []
    for top, bottom in ((0.0, -10.0), (-5.0, -35.0)):
        below = level <= bottom
        if not below.any() or not np.isfinite(level[int(np.argmax(below))]):
            out.append(float("nan"))
            continue
        start, stop = int(np.argmax(level <= top)), int(np.argmax(below))
        if stop - start < 2 or stop >= 0.8 * len(p):
            out.append(float("nan"))
            continue
        slope = np.polyfit(t[start : stop + 1], level[start : stop + 1], 1)[0]
        out.append(float(-60.0 / slope) if slope < 0 else float("nan"))
    return out[0], out[1]


def apply_launch(solver, launch) -> None:
    """Gives `solver` the launch choice `launch` (an autotuned solver's `launch` of the same grid)."""
    if not launch:
        return
    if "tile_shape" in launch:
        solver.set_tiles(launch["tile_shape"], launch["tile_planes"])
    solver.set_launch(launch["layer_blocks_per_sm"], launch["special_blocks_per_sm"])
    if "concurrent" in launch:
        solver.set_streams(int(launch["concurrent"]))


def ir_errors(p32: np.ndarray, p64: np.ndarray, rate: float) -> dict:
    """FP32 against FP64 impulse responses (probes, steps): the relative L2 error of each receiver,
    and of its energy-decay curve (Schroeder's backward integral) the largest difference in dB
    down to 60 dB below its start."""
    energy = np.linalg.norm(p64, axis=1)
    reached = energy > 1e-3 * energy.max()  # receivers the sound has reached
    if not np.any(reached):  # (a run too short for the sound to reach any receiver)
        return {"ir_rel_l2_max": None, "ir_rel_l2_median": None, "ir_rel_l2_demeaned_max": None, "edt_rel_max": None,
                "t30_rel_max": None, "t30_receivers": 0, "edc_db_max_abs": None}  # fmt: skip
    rel = np.linalg.norm(p32 - p64, axis=1)[reached] / energy[reached]
    # The same after removing each receiver's mean (a Gaussian drive's net mass shows as one).
    d = p32 - p64
    d = d - d.mean(axis=1, keepdims=True)
    q = p64 - p64.mean(axis=1, keepdims=True)
    rel_demeaned = np.linalg.norm(d, axis=1)[reached] / np.linalg.norm(q, axis=1)[reached]
    edt_err, t30_err = [], []
    for a, b in zip(p32[reached], p64[reached]):
        (ea, ta), (eb, tb) = decay_times(a, rate), decay_times(b, rate)
        if np.isfinite(ea) and np.isfinite(eb):
            edt_err.append(abs(ea - eb) / eb)
        if np.isfinite(ta) and np.isfinite(tb):
            t30_err.append(abs(ta - tb) / tb)
    worst_db = 0.0
    for a, b in zip(p32[reached], p64[reached]):
        ea = np.cumsum((a * a)[::-1])[::-1]
        eb = np.cumsum((b * b)[::-1])[::-1]
        keep = eb > eb[0] * 1e-6
        if np.any(keep) and eb[0] > 0:
            da = 10 * np.log10(np.maximum(ea[keep], 1e-300) / ea[0])
            db = 10 * np.log10(eb[keep] / eb[0])
            worst_db = max(worst_db, float(np.max(np.abs(da - db))))
    return {
        "ir_rel_l2_max": float(rel.max()),
        "ir_rel_l2_median": float(np.median(rel)),
        "ir_rel_l2_demeaned_max": float(rel_demeaned.max()),
        "edt_rel_max": float(max(edt_err)) if edt_err else None,
        "t30_rel_max": float(max(t30_err)) if t30_err else None,
        "t30_receivers": len(t30_err),
        "edc_db_max_abs": worst_db,
        "seconds": float(p64.shape[1] / rate),
        "receivers": int(reached.sum()),
    }


def measured_peaks() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        return float(json.loads(path.read_text())["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s"


class Clocks:
    """The SM clock and throttle reasons sampled through NVML while the timed region runs: a thread
    polls as fast as NVML answers (about every half millisecond), since the timed region can be
    a few milliseconds, shorter than nvidia-smi's sampling period. Nothing is set, only read."""

    # NVML's clocks-event reason bits (nvml.h): the four the timing rules name.
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, device: int):
        self.device = device
        self.samples: list[tuple[float, int]] = []
        self.max_mhz = None
        self._stop = threading.Event()
        self._thread = None
        self._nvml = None

    def _handle(self, nvml):
        try:
            import torch

            props = torch.cuda.get_device_properties(self.device)
            bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
            return nvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return nvml.nvmlDeviceGetHandleByIndex(self.device)

    def _poll(self, nvml, handle):
        while not self._stop.is_set():
            try:
                mhz = nvml.nvmlDeviceGetClockInfo(handle, nvml.NVML_CLOCK_SM)
                reasons = nvml.nvmlDeviceGetCurrentClocksEventReasons(handle)
            except Exception:
                return
            self.samples.append((float(mhz), int(reasons)))
            time.sleep(0.0002)

    def __enter__(self):
        try:
            import pynvml as nvml

            nvml.nvmlInit()
            self._nvml = nvml
            handle = self._handle(nvml)
            self.max_mhz = float(nvml.nvmlDeviceGetMaxClockInfo(handle, nvml.NVML_CLOCK_SM))
            self._thread = threading.Thread(target=self._poll, args=(nvml, handle), daemon=True)
            self._thread.start()
        except Exception:
            self._thread = None
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread is not None:
            self._thread.join(timeout=5)
        if self._nvml is not None:
            try:
                self._nvml.nvmlShutdown()
            except Exception:
                pass

    def summary(self) -> dict:
        sm = [mhz for mhz, _ in self.samples]
        reasons = sorted(name for name, bit in self.REASONS.items() if any(r & bit for _, r in self.samples))
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": self.max_mhz,
            "reasons": reasons,
            "samples": len(sm),
            "source": "NVML, polled through the timed region",
        }


def build_workload(args, barrier: bool = True):
    from acoustic_spaces_b200 import layouts

    if args.workload == "outdoor_halfspace":
        return layouts.outdoor_halfspace(args.seed, steps=max(args.steps, args.ir_steps), barrier=barrier)
    return layouts.polyhedral_room(args.seed, cell=args.cell, steps=max(args.steps, args.ir_steps, 1), walls=args.walls,
                                   device=int(os.environ.get("LOCAL_RANK", "0")))  # fmt: skip


def insertion_loss(free: np.ndarray, screened: np.ndarray, rate: float, band=(20.0, 300.0)) -> tuple[np.ndarray, np.ndarray]:
    """Each receiver's insertion loss 20 log10 |P_free(f)| / |P_screened(f)| in dB over ``band``
    Hz, from the spectra of the whole responses (probes, steps), and a mask of the bins where the
    free field is within 40 dB of its receiver's peak in the band."""
    f = np.fft.rfftfreq(free.shape[1], 1.0 / rate)
    sel = (f >= band[0]) & (f <= band[1])
    pf = np.abs(np.fft.rfft(free, axis=1))[:, sel]
    ps = np.abs(np.fft.rfft(screened, axis=1))[:, sel]
    tiny = 1e-300
    il = 20.0 * np.log10((pf + tiny) / (ps + tiny))
    valid = pf >= 1e-2 * pf.max(axis=1, keepdims=True)
    return il, valid


def outdoor_insertion_loss(args, workload, local: int) -> dict:
    """The half-space's insertion-loss spectra (the barrier's; free field = the same ground without
    it) from FP32 runs against those from FP64 runs on the same layouts, over the config's steps."""
    from acoustic_spaces_b200 import B200WaveSolver

    free = build_workload(args, barrier=False)
    steps = min(len(workload.signal), args.ir_steps)
    runs = {}
    for name, w in (("screened", workload), ("free", free)):
        for precision in ("fp32", "fp64"):
            solver = B200WaveSolver(w.built.layout, precision=precision, device=local)
            runs[name, precision] = solver.run(w.signal[:steps])
            solver.close()
    il32, valid = insertion_loss(runs["free", "fp32"], runs["screened", "fp32"], workload.built.rate)
    il64, _ = insertion_loss(runs["free", "fp64"], runs["screened", "fp64"], workload.built.rate)
    diff = np.abs(il32 - il64)[valid]
    return {
        "il_db_max_abs_diff": float(diff.max()),
        "il_db_median_abs_diff": float(np.median(diff)),
        "il_db_mean_fp64": float(np.mean(il64[valid])),
        "band_hz": [20.0, 300.0],
        "bins": int(valid.sum()),
        "receivers": int(il32.shape[0]),
        "steps": steps,
        "vs": "the same two layouts (with and without the barrier) stepped in FP64 on the GPU",
    }


def oracle_cores(layout) -> int:
    """The host threads the oracle's C port steps a grid of this layout on."""
    from oracle import oracle

    cells = int(np.prod(np.asarray(layout["shape"], np.int64)))
    return int(oracle.load_oracle().oracle_threads()) if cells >= oracle.PARALLEL_CELLS else 1


def cpu_reference_rate(workload, sample_steps: int, warmup: int = 3, fitted_walls: bool = False) -> dict:
    """The reference's own CPU solver (its unmodified C++, oracle/_ref) on the same room, timed
    over ``sample_steps`` steps with every host thread; else the oracle's C port, on every host
    thread too where the grid is large."""
    from acoustic_spaces_b200 import layouts
    from oracle import oracle

    threads = os.cpu_count() or 1
    # (The reference lays out rooms that keep clear of the matched layer only; for the others, the
    # oracle's C port of its stepping runs on the same layout.)
    native = oracle.reference_native() if workload.name == "polyhedral_room" else None
    air = workload.built.air_cells
    signal = workload.signal[:sample_steps]
    if native is not None:
        room, grid = workload.room, workload.built.grid
        vertices, faces, owner = layouts.room_mesh(room)
        beta = np.array([0.0 if m is None else m.beta for m in room.materials])
        rows, owners = [np.zeros((0, 3))], [np.zeros(0, np.int64)]
        for k, m in enumerate(room.materials):
            if m is not None:
                rows.append(m.branches)
                owners.append(np.full(len(m.branches), k, np.int64))
        t0 = time.perf_counter()
        solver = native.WaveSolver(
            native.Bvh(vertices, faces), owner, beta, np.ascontiguousarray(np.vstack(rows)),
            np.concatenate(owners), grid.origin, grid.cell, *grid.shape, workload.source,
            workload.receivers, layer=8, layer_damping=0.5, threads=threads, fitted_walls=fitted_walls,
            vertices=np.ascontiguousarray(vertices), faces=np.ascontiguousarray(faces),
        )  # fmt: skip
        setup = time.perf_counter() - t0
        solver.run(workload.signal[:warmup])  # its threads spun up, untimed
        solver.reset()
        t0 = time.perf_counter()
        solver.run(signal)
        seconds = time.perf_counter() - t0
        kind, cores, ref_air = "reference", int(solver.threads), int(solver.air_cells)
        if ref_air != air:
            raise RuntimeError(f"the reference lays the room out with {ref_air} air cells, the builder {air}")
        extra = {"setup_s": round(setup, 2), "walls": "the reference's own fitted walls (its exact fit) of the same room"
                 if fitted_walls else "cell faces"}  # fmt: skip
    else:
        ported = oracle.OracleSolver(workload.built.layout)
        ported.run(workload.signal[:warmup])
        ported.reset()
        t0 = time.perf_counter()
        ported.run(signal)
        seconds = time.perf_counter() - t0
        kind, cores, extra = "port", oracle_cores(workload.built.layout), {}
    value = air * len(signal) / seconds / 1e9
    return {
        "value": round(value, 4),
        "unit": UNIT,
        "cores": cores,
        "kind": kind,
        "sample": f"{len(signal)} steps of the full {workload.description['grid']} grid "
        f"({air} air cells), after {warmup} warm-up steps",
        **extra,
    }


def run_reference(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    # The room as the host lays it out (no GPU on this arm): the reference builds its own layout of
    # it, with its own fitted walls where those are asked for, and is checked to hold the same air.
    fitted_walls = args.walls == "fitted" and args.workload == "polyhedral_room"
    walls = args.walls
    args.walls = "faces"
    workload = build_workload(args)
    args.walls = walls
    if fitted_walls:
        workload.description["walls"] = "fitted cut cells (the reference's own exact fit), 2-pole admittance per wall"
        for key in ("special_rows", "links", "branch_states", "interior_cells"):
            workload.description.pop(key, None)
    steps = max(1, min(args.steps, args.reference_steps))
    warmup = max(3, args.warmup)
    times = []
    base = None
    for _ in range(max(1, args.reference_repeats)):
        base = cpu_reference_rate(workload, steps, warmup, fitted_walls)
        times.append(base["value"])
    value = statistics.median(times)
    base["value"] = round(value, 4)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 4),
        "unit": UNIT,
        "n_gpus": world,
        "steps": steps,
        "warmup": warmup,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "polyhedral_room", **workload.description, "sample_steps": steps},
        "cpu_baseline": base,
        "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def batch_reference_rate(batch, sample, sample_steps: int) -> dict:
    """The reference's own solver (oracle/_ref) on two solves of ``sample``, each laid out by the
    reference from its scene (a box with real walls, one source), every host thread, timed over
    ``sample_steps`` steps each: cell updates per second, the rate the whole batch would run at."""
    from acoustic_spaces_b200 import layouts
    from oracle import oracle

    native = oracle.reference_native()
    if native is None:
        raise RuntimeError("the reference's solver is not built")
    threads = os.cpu_count() or 1
    cells, seconds, used = 0, 0.0, []
    for k in list(sample)[:2]:
        room, grid, source, receivers = batch.scenes[k]
        vertices, faces, owner = layouts.room_mesh(room)
        beta = np.array([m.beta for m in room.materials])
        solver = native.WaveSolver(
            native.Bvh(vertices, faces), owner, beta, np.zeros((0, 3)), np.zeros(0, np.int64), grid.origin,
            grid.cell, *grid.shape, source, receivers, layer=0, layer_damping=0.0, threads=threads,
        )  # fmt: skip
        air = int(solver.air_cells)
        if air != int(np.count_nonzero(batch.layouts[k]["types"])):
            raise RuntimeError("the reference lays a solve out otherwise than the builder")
        solver.run(batch.signal[:2])
        t0 = time.perf_counter()
        solver.run(batch.signal[:sample_steps])
        seconds += time.perf_counter() - t0
        cells += air * sample_steps
        used.append(k)
        threads = int(solver.threads)
    return {"value": round(cells / seconds / 1e9, 4), "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"solves {used} of the batch, {sample_steps} steps each, scaled as cell updates per second"}  # fmt: skip


def run_batched(args, world: int, rank: int, local: int) -> None:
    """The batched configuration: many shoebox rooms with several sources each, every (room,
    source) a solve of its own, stacked into one grid and stepped by one launch per kind per step
    (64 rooms of 3-12 m at 5 cm cells, 4 sources each: 256 solves). Beside it, a sample of the same solves stepped one after another through
    the same public API, and each solve's FP32 error against FP64."""
    import torch
    import torch.distributed as dist

    from acoustic_spaces_b200 import B200WaveSolver, layouts

    # With N ranks, the solves shard by cell count (no exchange): each rank steps its own rooms.
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=900), device_id=torch.device("cuda", local))
    batch = layouts.batched_rooms(args.seed, rooms=args.rooms, sources=args.sources, steps=args.steps + args.warmup,
                                  part=(rank, world))  # fmt: skip
    desc = batch.description
    solver = B200WaveSolver(batch.stacked.layout, precision=args.precision, device=local)
    if args.streams >= 0:
        solver.set_streams(args.streams)
    air = batch.stacked.air_cells
    steps, warmup = args.steps, args.warmup
    sig = torch.from_numpy(np.ascontiguousarray(batch.signal)).to(f"cuda:{local}")
    out = torch.zeros((solver.probes, steps + warmup), dtype=torch.float64, device=f"cuda:{local}")
    stream = torch.cuda.ExternalStream(solver.stream, device=f"cuda:{local}")
    solver.run_device(sig.data_ptr(), warmup, out.data_ptr(), steps + warmup)
    solver.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clocks:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        start.record(stream)
        solver.run_device(sig.data_ptr() + 4 * warmup, steps, out.data_ptr() + 8 * warmup, steps + warmup)
        end.record(stream)
        solver.synchronize()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    ms = start.elapsed_time(end)
    # Each kernel's own duration: the step's kernels one after another, CUDA events around each.
    solver.set_timing(True)
    solver.run_device(sig.data_ptr(), min(steps, 10), out.data_ptr(), steps + warmup)
    solver.synchronize()
    solver.set_timing(False)
    timed = solver.timing()
    kernel_us = {k: round(1e3 * v / max(1, timed["steps"]), 2) for k, v in timed.items() if k != "steps" and v}
    total_air = air
    if world > 1:
        t = torch.tensor([ms, float(air)], dtype=torch.float64, device=f"cuda:{local}")
        mx = t[:1].clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        sm = t[1:].clone()
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        ms, total_air = float(mx.item()), int(sm.item())
    value = total_air * steps / (ms / 1e3) / 1e9
    # End to end, the whole batch through the public API (the slowest rank's time).
    solver.reset()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    solver.run(batch.signal[:steps])
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    # A sample of the solves one after another (each its own grid), through the same API.
    rng = np.random.default_rng(1)
    sample = sorted(rng.choice(len(batch.layouts), size=min(args.sequential_sample, len(batch.layouts)), replace=False))
    seq_cells, seq_s = 0, 0.0
    for k in sample:
        one = B200WaveSolver(batch.layouts[k], precision=args.precision, device=local)
        one.run(batch.signal[: max(warmup, 130)])  # both of its step graphs captured before timing
        one.reset()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        one.run(batch.signal[:steps])
        seq_s += time.perf_counter() - t0
        seq_cells += one.air_cells * steps
        one.close()
    sequential = seq_cells / seq_s / 1e9
    # The reference's own CPU solver on two of the solves (seeded), every host thread, over a
    # bounded sample of steps; scaled as cell updates per second.
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            cpu = batch_reference_rate(batch, sample, args.cpu_steps)
        except Exception as error:  # the baseline is reported, not required
            cpu = {"value": None, "unit": UNIT, "error": str(error)[:200]}
    # Each solve's FP32 response against FP64 (the stacked grid in both).
    m = min(args.ir_steps, steps)
    solver.reset()
    p32 = solver.run(batch.signal[:m])
    fp64 = B200WaveSolver(batch.stacked.layout, precision="fp64", device=local)
    p64 = fp64.run(batch.signal[:m])
    fp64.close()
    worst = []
    for p0, p1, _, _ in batch.stacked.parts:
        err = ir_errors(p32[p0:p1], p64[p0:p1], batch.rate)["ir_rel_l2_max"]
        if err is not None:
            worst.append(err)
    line = {
        "metric": METRIC,
        "value": round(value, 4),
        "unit": UNIT,
        "n_gpus": world,
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": round(ms / steps, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "batched_rooms", **desc, "air_cells_all_ranks": total_air,
                   "parallelism": f"solves sharded over {world} GPUs by cell count" if world > 1 else "single GPU",
                   "precision": "FP32, bit-exact with the reference" if args.precision == "fp32"
                   else "FP32 compensated: each cell's pressure and its increment",
                   "launch": solver.launch},
        "kernel_mean_us_serialised": kernel_us,
        "e2e": {"value": round(total_air * steps / e2e_s / 1e9, 4), "unit": UNIT, "h2d_bytes_per_step": 4,
                "d2h_bytes_per_step": 8 * solver.probes},  # fmt: skip
        "sequential_solves": {"value": round(sequential, 4), "unit": UNIT, "solves_timed": len(sample),
                              "api": "B200WaveSolver.run, one solve after another, on one GPU"},  # fmt: skip
        "batched_over_sequential": round(value / world / sequential, 3),
        "per_solve_ir_rel_l2_vs_fp64": {"max": float(max(worst)) if worst else None,
                                        "median": float(np.median(worst)) if worst else None, "steps": m,
                                        "solves_reached": len(worst)},  # fmt: skip
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
        "gpu_launches": 3 * steps,  # the sweep, the special rows, the probes
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_shoebox(args, world: int, rank: int, local: int) -> None:
    """The plain FP64 box (6 x 4 x 3 m at 5 cm, Courant 0.99/sqrt(3), six real walls, one source
    and one receiver, 4000 steps): the configuration the reference runs on its CPU. The B200 steps
    it in FP64 (device time, and end to end through the API) and must equal the FP64 oracle (its C
    port, one core, timed) to the bit; beside them the reference's own FP32 solver on all host
    threads."""
    import torch

    from acoustic_spaces_b200 import B200WaveSolver, layouts
    from oracle import oracle

    w = layouts.shoebox_room(args.seed, steps=args.shoebox_steps)
    steps = len(w.signal)
    air = w.built.air_cells
    solver = B200WaveSolver(w.built.layout, precision="fp64", device=local)
    sig = torch.from_numpy(np.ascontiguousarray(w.signal)).to(f"cuda:{local}")
    out = torch.zeros((solver.probes, steps), dtype=torch.float64, device=f"cuda:{local}")
    stream = torch.cuda.ExternalStream(solver.stream, device=f"cuda:{local}")
    solver.run_device(sig.data_ptr(), args.warmup, out.data_ptr(), steps)
    solver.synchronize()
    solver.reset()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clocks:
        torch.cuda.synchronize()
        start.record(stream)
        solver.run_device(sig.data_ptr(), steps, out.data_ptr(), steps)
        end.record(stream)
        solver.synchronize()
    ms = start.elapsed_time(end)
    solver.reset()
    t0 = time.perf_counter()
    ours = solver.run(w.signal)
    e2e_s = time.perf_counter() - t0
    ported = oracle.OracleSolver(w.built.layout, "fp64")
    t0 = time.perf_counter()
    theirs = ported.run(w.signal)
    port_s = time.perf_counter() - t0
    reference = None
    native = oracle.reference_native()
    if native is not None:
        vertices, faces, owner = layouts.room_mesh(w.room)
        beta = np.array([m.beta for m in w.room.materials])
        threads = os.cpu_count() or 1
        ref = native.WaveSolver(
            native.Bvh(vertices, faces), owner, beta, np.zeros((0, 3)), np.zeros(0, np.int64), w.built.grid.origin,
            w.built.grid.cell, *w.built.grid.shape, w.source, w.receivers, layer=0, layer_damping=0.0,
            threads=threads, speed=np.full(w.built.grid.n, w.description["speed_ratio"], np.float32),
        )  # fmt: skip
        t0 = time.perf_counter()
        ref_series = ref.run(w.signal)
        ref_s = time.perf_counter() - t0
        reference = {"value": round(air * steps / ref_s / 1e9, 4), "unit": UNIT, "cores": int(ref.threads),
                     "kind": "reference", "precision": "FP32 (the reference's)",
                     "sample": f"all {steps} steps", "rel_l2_vs_fp64": float(np.linalg.norm(ref_series - theirs)
                                                                             / np.linalg.norm(theirs))}  # fmt: skip
    line = {
        "metric": METRIC,
        "value": round(air * steps / (ms / 1e3) / 1e9, 4),
        "unit": UNIT,
        "n_gpus": world,
        "steps": steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms / steps, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "shoebox_room", **w.description, "precision": "FP64 (bit-exact with the FP64 oracle)"},
        "e2e": {"value": round(air * steps / e2e_s / 1e9, 4), "unit": UNIT, "h2d_bytes_per_step": 4,
                "d2h_bytes_per_step": 8 * solver.probes},  # fmt: skip
        "bit_exact_vs_fp64_oracle": bool(np.array_equal(ours, theirs)),
        "cpu_baseline": {"value": round(air * steps / port_s / 1e9, 4), "unit": UNIT,
                         "cores": oracle_cores(w.built.layout), "kind": "port",
                         "precision": "FP64", "sample": f"all {steps} steps"},  # fmt: skip
        "reference_cpu": reference,
        "clocks": clocks.summary(),
        "gpu_launches": 3 * steps,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_slabs(args, world: int, rank: int, local: int) -> None:
    """The polyhedral room as one grid split into slabs of z-planes (strong scaling), one plane per
    neighbour exchanged after every step. Across ranks (one GPU each): each rank steps its slab and
    swaps its boundary planes with its neighbours over NCCL, everything enqueued on the solver's
    stream (torch's NCCL streams wait for it and it for them) so the host never waits between
    steps. In one process (``--slab-count`` S > 1 on one GPU): the S slabs stepped together inside
    the library (fdtd_run_linked), the planes copied on the device. Reports the whole grid's cell
    updates over the slowest rank's device time."""
    import torch
    import torch.distributed as dist

    from acoustic_spaces_b200 import B200WaveSolver, slabs

    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    workload = build_workload(args)
    layout = workload.built.layout
    count = args.slab_count if (world == 1 and args.slab_count > 1) else world
    bounds = slabs.partition_planes(layout, count)
    steps, warmup = args.steps, args.warmup
    signal = np.ascontiguousarray(np.resize(workload.signal, steps + warmup), np.float32)
    sig = torch.from_numpy(signal).to(f"cuda:{local}")
    if world == 1 and count > 1:
        parts = [slabs.slab(layout, bounds, r) for r in range(count)]
        solvers = [B200WaveSolver(p.layout, device=local) for p in parts]
        outs = [torch.zeros((max(1, s.probes), steps + warmup), dtype=torch.float64, device=f"cuda:{local}")
                for s in solvers]  # fmt: skip
        slabs.run_linked(solvers, parts, signal[:warmup], device_buffers=([sig] * count, outs, steps + warmup))
        torch.cuda.synchronize(local)
        stream = torch.cuda.ExternalStream(solvers[0].stream, device=f"cuda:{local}")
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(local) as clocks:
            start.record(stream)
            shifted = [torch.narrow(sig, 0, warmup, steps)] * count
            outs_k = [o[:, warmup:] for o in outs]
            slabs.run_linked(solvers, parts, signal[warmup:], device_buffers=(shifted, outs_k, steps + warmup))
            end.record(stream)
            torch.cuda.synchronize(local)
        ms = start.elapsed_time(end)
        exchange = "one plane per neighbour per step, copied on the device inside the library (fdtd_run_linked)"
    else:
        part = slabs.slab(layout, bounds, rank)
        solver = B200WaveSolver(part.layout, device=local)
        planes = slabs.DevicePlanes(solver)
        out = torch.zeros((max(1, len(part.probes)), steps + warmup), dtype=torch.float64, device=f"cuda:{local}")
        stream = torch.cuda.ExternalStream(solver.stream, device=f"cuda:{local}")

        def step(k: int) -> None:
            solver.run_device(sig.data_ptr() + 4 * k, 1, out.data_ptr() + 8 * k, steps + warmup)
            if world > 1:
                with torch.cuda.stream(stream):
                    slabs.exchange_ghosts(planes, part, rank, world, dist)

        for k in range(warmup):
            step(k)
        torch.cuda.synchronize(local)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(local)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(local) as clocks:
            start.record(stream)
            for k in range(warmup, warmup + steps):
                step(k)
            end.record(stream)
            torch.cuda.synchronize(local)
        ms = start.elapsed_time(end)
        exchange = "one plane per neighbour per step over NCCL, enqueued on the solver's stream (no host wait between steps)"
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
        dist.destroy_process_group()
    air = workload.built.air_cells
    if rank == 0:
        line = {
            "metric": METRIC,
            "value": round(air * steps / (ms / 1e3) / 1e9, 4),
            "unit": UNIT,
            "n_gpus": world,
            "steps": steps,
            "warmup": warmup,
            "ms_per_step": round(ms / steps, 5),
            "higher_is_better": True,
            "scaling": "strong",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": workload.name, **workload.description, "parallelism": f"z-slabs x{count}",
                       "slabs": [list(b) for b in bounds], "exchange": exchange},  # fmt: skip
            "clocks": clocks.summary(),
            "gpu_launches": 4 * steps * count // max(1, world),
        }
        print(json.dumps(line), flush=True)


def run_adjoint(args, world: int, rank: int, local: int) -> None:
    """The adjoint fit: a 10 x 8 x 4 m room at 5 cm cells with 8
    materials on seeded patches, a 1-pole admittance each (16 parameters); the misfit of the
    responses at 4 receivers over 3000 steps to those at seeded true parameters, from parameters
    off by up to 30 %; checkpoints every 250 steps. Reports the forward and forward + adjoint
    times, the gradient against central differences (relative step 1e-4, taken in the layout's
    float32 coefficients along each parameter's tangent) and the FP32 gradient against the FP64
    one, the peak device memory, and the Adam iterations to recover every parameter to 1 %."""
    import torch

    from acoustic_spaces_b200 import fit

    problem = fit.patched_room(args.seed, steps=args.adjoint_steps, segment=250)
    f = problem.fit
    params = problem.start
    f.loss_and_gradient(params, "fp32")  # warm-up: the fit's solver, its graphs and its tables
    times = []
    for _ in range(3):
        # A plain forward run on the fit's own solver (its graphs captured, no tape) ...
        solver = f._solver(f.layout(params), "fp32")
        solver.set_tape(0)
        solver.reset()
        t0 = time.perf_counter()
        solver.run(f.signal)
        plain_s = time.perf_counter() - t0
        # ... and an iteration of the fit: the taped forward run, then the gradient.
        f.loss_and_gradient(params, "fp32")
        times.append((plain_s, f.forward_s, f.gradient_s))
    forward_s = min(t[0] for t in times)
    taped_s = min(t[1] for t in times)
    gradient_s = min(t[2] for t in times)
    # The same with the tape held to checkpoints (budget 0): the gradient recomputes each segment.
    solver = f._solver(f.layout(params), "fp32")
    solver.set_tape_budget(0)
    f.loss_and_gradient(params, "fp32")  # warm-up: the recomputation's graphs
    checkpointed = []
    for _ in range(2):
        f.loss_and_gradient(params, "fp32")
        checkpointed.append((f.forward_s, f.gradient_s))
    solver.set_tape_budget(None)
    ck_taped_s = min(t[0] for t in checkpointed)
    ck_gradient_s = min(t[1] for t in checkpointed)
    # Peak device memory of a gradient: free memory sampled while it runs.
    free_min = [torch.cuda.mem_get_info(local)[0]]
    stop = threading.Event()

    def watch():
        while not stop.is_set():
            free_min[0] = min(free_min[0], torch.cuda.mem_get_info(local)[0])
            time.sleep(0.002)

    total = torch.cuda.mem_get_info(local)[1]
    watcher = threading.Thread(target=watch, daemon=True)
    watcher.start()
    _, g32 = f.loss_and_gradient(params, "fp32")
    stop.set()
    watcher.join()
    _, g64, G64 = f.loss_and_gradient(params, "fp64", coefficients=True)
    _, _, G32 = f.loss_and_gradient(params, "fp32", coefficients=True)
    # Central differences of L in the coefficients along each parameter's tangent (relative step
    # 1e-4, exactly symmetric float32 steps), against the FP64 and the FP32 adjoint.
    triples = []
    for i in range(len(params.vector())):
        p64, measured = f.central_difference(params, i, G64)
        p32, _ = f.central_difference(params, i, G32)
        triples.append((p64, p32, measured))
    # (Relative to each parameter's own difference; a parameter whose walls the sound has not yet
    # reached, whose difference is 0 beside the largest, is left out.)
    largest = max(abs(m) for _, _, m in triples)
    kept = [(a, b, m) for a, b, m in triples if abs(m) > 1e-12 * largest]
    cd64 = [abs(a - m) / abs(m) for a, _, m in kept]
    cd32 = [abs(b - m) / abs(m) for _, b, m in kept]
    rel = lambda a, b: float(np.max(np.abs(a - b)) / np.max(np.abs(b)))  # noqa: E731
    result = fit.adam(problem, iterations=args.adam_iterations, rate=0.05)
    t0 = time.perf_counter()
    quasi = fit.lbfgs(problem, iterations=args.adam_iterations)
    quasi["seconds"] = round(time.perf_counter() - t0, 2)
    line = {
        "metric": METRIC,
        "value": round(f.built.air_cells * len(f.signal) / forward_s / 1e9, 4),
        "unit": UNIT,
        "n_gpus": world,
        "steps": len(f.signal),
        "warmup": 1,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "adjoint_fit", **problem.description},
        "adjoint_over_forward": round((taped_s + gradient_s) / forward_s, 3),
        "forward_s": round(forward_s, 4),
        "taped_forward_s": round(taped_s, 4),
        "gradient_s": round(gradient_s, 4),
        "adjoint_over_forward_means": "(the taped forward run + the gradient) / a plain forward run, host buffers both; "
        "the tape holds the special rows' and branch states' trajectory, so the gradient is the reverse steps alone",
        "with_checkpoints": {
            "adjoint_over_forward": round((ck_taped_s + ck_gradient_s) / forward_s, 3),
            "taped_forward_s": round(ck_taped_s, 4), "gradient_s": round(ck_gradient_s, 4),
            "means": "the tape held to checkpoints every 250 steps (budget 0): the gradient recomputes each segment",
        },  # fmt: skip
        "gradient_vs_central_differences": {
            "max_rel": max(cd64), "h": 1e-4, "precision": "fp64",
            "difference": "L(c + d) - L(c - d) over 2, d the coefficients' change along each parameter, exact float32 steps",
        },
        "fp32_gradient_vs_central_differences": {"max_rel": max(cd32)},
        "fp32_gradient_vs_fp64": {"max_rel": rel(g32, g64)},
        "peak_device_bytes": int(total - free_min[0]),
        "adam": {k: result[k] for k in ("iterations", "converged", "worst_relative_error")},
        "lbfgs": {k: quasi[k] for k in ("iterations", "evaluations", "converged", "worst_relative_error", "seconds")},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=2000)
    parser.add_argument("--warmup", type=int, default=20)
    parser.add_argument("--impl", choices=["b200", "reference"], default="b200")
    parser.add_argument("--seed", type=int, default=0)
    parser.add_argument("--cell", type=float, default=0.04, help="cell size in metres (0.04: the full workload)")
    parser.add_argument("--walls", choices=["fitted", "faces"], default="fitted",
                        help="the polyhedral room's walls: fitted cut cells (the configuration's) or on cell faces")  # fmt: skip
    parser.add_argument("--no-compensated", action="store_true", help="skip the compensated-precision leg")
    parser.add_argument("--gradient-steps", type=int, default=200,
                        help="steps of the forward + adjoint timing on the polyhedral room (0: skip)")  # fmt: skip
    parser.add_argument("--gradient-segment", type=int, default=50)
    parser.add_argument("--no-fp64-rate", action="store_true", help="skip timing the FP64 stepper alike")
    parser.add_argument("--launch", default="", help="layer,special blocks per SM (skips the autotuner)")
    parser.add_argument("--streams", type=int, default=-1,
                        help="the step's stream arrangement (0 to 5), set after the autotuner's choice")
    parser.add_argument("--tiles", default="", help="with --launch: the sweep's tile shape,planes a tile")
    parser.add_argument("--slab-count", type=int, default=0,
                        help="with --slabs on one GPU: this many slabs stepped together in one process")  # fmt: skip
    parser.add_argument("--slabs", action="store_true",
                        help="one grid split into z-slabs across the ranks, boundary planes swapped each step")  # fmt: skip
    parser.add_argument("--precision", choices=["fp32", "fp32c"], default="fp32",
                        help="fp32: the reference's arithmetic; fp32c: compensated single precision")  # fmt: skip
    parser.add_argument("--cpu-steps", type=int, default=10, help="steps of the CPU-baseline sample")
    parser.add_argument("--reference-steps", type=int, default=10)
    parser.add_argument("--reference-repeats", type=int, default=3)
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--no-e2e", action="store_true")
    parser.add_argument("--workload", choices=["polyhedral_room", "outdoor_halfspace", "batched_rooms", "adjoint_fit",
                                               "shoebox_room"], default="polyhedral_room")  # fmt: skip
    parser.add_argument("--shoebox-steps", type=int, default=4000)
    parser.add_argument("--adjoint-steps", type=int, default=3000)
    parser.add_argument("--adam-iterations", type=int, default=300)
    parser.add_argument("--rooms", type=int, default=64)
    parser.add_argument("--sources", type=int, default=4)
    parser.add_argument("--sequential-sample", type=int, default=16)
    parser.add_argument("--no-ir-error", action="store_true")
    parser.add_argument("--kernel-steps", type=int, default=200, help="steps of the per-kernel timing pass")
    parser.add_argument("--ir-steps", type=int, default=12000,
                        help="steps of the FP32-vs-FP64 comparison (12000: the configuration's full length)")  # fmt: skip
    args = parser.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist

    from acoustic_spaces_b200 import B200WaveSolver

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device (the B200 stepper has no CPU path)")
    torch.cuda.set_device(local)
    if args.workload == "batched_rooms":
        run_batched(args, world, rank, local)
        return
    if args.workload == "adjoint_fit":
        run_adjoint(args, world, rank, local)
        return
    if args.workload == "shoebox_room":
        run_shoebox(args, world, rank, local)
        return
    if args.slabs:
        run_slabs(args, world, rank, local)
        return
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    # Set-up, outside the metric and reported apart: the layout on the host, then the handle (its
    # uploads, and the autotuner's trial steps).
    t_setup = time.perf_counter()
    workload = build_workload(args)
    layout_s = time.perf_counter() - t_setup
    desc = workload.description
    t_setup = time.perf_counter()
    if args.launch:
        solver = B200WaveSolver(workload.built.layout, precision=args.precision, device=local, autotune=False)
        solver.set_launch(*(int(v) for v in args.launch.split(",")))
        if args.tiles:
            solver.set_tiles(*(int(v) for v in args.tiles.split(",")))
        solver.launch = {**solver.tiles(), "layer_blocks_per_sm": int(args.launch.split(",")[0]),
                         "special_blocks_per_sm": int(args.launch.split(",")[1])}  # fmt: skip
    else:
        solver = B200WaveSolver(workload.built.layout, precision=args.precision, device=local)
    if args.streams >= 0:
        solver.set_streams(args.streams)
    handle_s = time.perf_counter() - t_setup
    air = solver.air_cells
    probes = solver.probes
    steps, warmup = args.steps, args.warmup
    if warmup < 3:
        raise SystemExit("at least 3 warm-up steps")

    signal = workload.signal
    sig_dev = torch.from_numpy(np.ascontiguousarray(np.resize(signal, steps + warmup))).to(f"cuda:{local}")
    out_dev = torch.zeros((probes, steps + warmup), dtype=torch.float64, device=f"cuda:{local}")
    stream = torch.cuda.ExternalStream(solver.stream, device=f"cuda:{local}")
    # Warm-up.
    solver.run_device(sig_dev.data_ptr(), warmup, out_dev.data_ptr(), steps + warmup)
    solver.synchronize()

    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clocks:
        barrier()
        torch.cuda.synchronize()
        solver.synchronize()
        with torch.cuda.stream(stream):
            start.record(stream)
        solver.run_device(sig_dev.data_ptr() + 4 * warmup, steps, out_dev.data_ptr() + 8 * warmup, steps + warmup)
        with torch.cuda.stream(stream):
            end.record(stream)
        solver.synchronize()
        torch.cuda.synchronize()
        barrier()
    ms = start.elapsed_time(end)
    # Each kernel's own duration: a second timed pass with CUDA events around every launch, the
    # step's kernels one after another on the solver's stream.
    timed = max(3, min(steps, args.kernel_steps))
    solver.set_timing(True)
    solver.run_device(sig_dev.data_ptr(), timed, out_dev.data_ptr(), steps + warmup)
    solver.synchronize()
    solver.set_timing(False)
    kernel_ms = solver.timing()
    if world > 1:
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * air * steps / (ms / 1e3) / 1e9

    finite = bool(torch.isfinite(out_dev).all().item())

    # End to end through the public API: a host drive in, the probes' series out.
    e2e = None
    if not args.no_e2e:
        host_signal = np.ascontiguousarray(np.resize(signal, steps), dtype=np.float32)
        solver.reset()
        solver.run(host_signal[:warmup])
        solver.reset()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        recorded = solver.run(host_signal)
        seconds = time.perf_counter() - t0
        if world > 1:
            t = torch.tensor([seconds], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            seconds = float(t.item())
        finite = finite and bool(np.isfinite(recorded).all())
        e2e = {
            "value": round(world * air * steps / seconds / 1e9, 4),
            "unit": UNIT,
            "h2d_bytes_per_step": 4,
            "d2h_bytes_per_step": 8 * probes,
            "api": "B200WaveSolver.run(host float32 drive) -> host float64 (probes, steps)",
        }

    # The plain FP64 stepper on the same GPU and grid, timed alike: the accurate mode to beat.
    fp64_rate = None
    if not args.no_fp64_rate:
        fp64 = B200WaveSolver(workload.built.layout, precision="fp64", device=local)
        fp64.run_device(sig_dev.data_ptr(), warmup, out_dev.data_ptr(), steps + warmup)
        fp64.synchronize()
        s64 = torch.cuda.ExternalStream(fp64.stream, device=f"cuda:{local}")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s64)
        fp64.run_device(sig_dev.data_ptr() + 4 * warmup, steps, out_dev.data_ptr() + 8 * warmup, steps + warmup)
        e1.record(s64)
        fp64.synchronize()
        fp64.close()
        fp64_rate = {"value": round(air * steps / (e0.elapsed_time(e1) / 1e3) / 1e9, 4), "unit": UNIT,
                     "what": "the same grid stepped in FP64 on the same GPU, device-timed alike"}  # fmt: skip

    # The IR error against FP64 on the same grid: both run from rest over the same drive.
    ir_error = None
    p64 = None
    if not args.no_ir_error:
        fp64 = B200WaveSolver(workload.built.layout, precision="fp64", device=local)
        m = min(args.ir_steps, len(signal))
        solver.reset()
        p32 = solver.run(signal[:m])
        p64 = fp64.run(signal[:m])
        fp64.close()
        ir_error = ir_errors(p32, p64, workload.built.rate)
        ir_error["steps"] = m
        ir_error["vs"] = "the same layout stepped in FP64 on the GPU (bit-exact with the FP64 oracle on the golden grids)"

    # The compensated single precision on the same grid, device-timed alike, with its IR error
    # over the same steps: the mode that meets the 1e-4 bar over the configuration's full length.
    compensated = None
    if args.precision == "fp32" and not args.no_compensated:
        comp = B200WaveSolver(workload.built.layout, precision="fp32c", device=local)
        comp.run_device(sig_dev.data_ptr(), warmup, out_dev.data_ptr(), steps + warmup)
        comp.synchronize()
        sc = torch.cuda.ExternalStream(comp.stream, device=f"cuda:{local}")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(sc)
        comp.run_device(sig_dev.data_ptr() + 4 * warmup, steps, out_dev.data_ptr() + 8 * warmup, steps + warmup)
        e1.record(sc)
        comp.synchronize()
        comp_ms = e0.elapsed_time(e1)
        compensated = {
            "value": round(air * steps / (comp_ms / 1e3) / 1e9, 4),
            "unit": UNIT,
            "ms_per_step": round(comp_ms / steps, 5),
            "what": "the same grid in compensated FP32 (each cell's pressure and its increment), device-timed alike",
        }
        if p64 is not None:
            comp.reset()
            pc = comp.run(signal[: p64.shape[1]])
            compensated["ir_error_vs_fp64"] = {**ir_errors(pc, p64, workload.built.rate), "steps": int(p64.shape[1])}
        comp.close()

    # Forward + adjoint against forward on the same grid (the gradient in the walls' coefficients
    # and, with a matched layer, its tables), checkpoints every `gradient_segment` steps: a taped
    # forward run keeps them, the gradient recomputes each segment from them and steps back.
    adjoint = None
    if args.gradient_steps > 0 and workload.name == "polyhedral_room":
        try:
            g_steps = min(args.gradient_steps, len(signal))
            grad_solver = B200WaveSolver(workload.built.layout, device=local, autotune=False)
            apply_launch(grad_solver, solver.launch)
            head = np.ascontiguousarray(signal[:g_steps])
            y = grad_solver.run(head)
            dloss = 2.0 * (y - 0.9 * y)
            grad_solver.reset()
            for tables in (True, False):  # set-up of the adjoint, untimed
                grad_solver.gradient(head, dloss, segment=args.gradient_segment, layer_tables=tables)
                grad_solver.reset()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            grad_solver.run(head)
            forward_s = time.perf_counter() - t0
            grad_solver.reset()

            def taped_gradient(tables, tangent=None):
                # (a fit's iterations keep the tape and the gradient's workspace: one untimed pass
                # takes them, as the first iteration would)
                grad_solver.set_layer_tangent(tangent)
                grad_solver.set_tape(args.gradient_segment, layer_tables=tables)
                grad_solver.run(head)
                grad_solver.gradient(head, dloss, segment=args.gradient_segment, layer_tables=tables)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                grad_solver.run(head)
                t1 = time.perf_counter()
                grads = grad_solver.gradient(head, dloss, segment=args.gradient_segment, layer_tables=tables)
                return time.perf_counter() - t0, t1 - t0, grads

            both_s, taped_s, grads = taped_gradient(False)
            tables_s, _, with_tables = taped_gradient(True)
            # The gradient in the layer's damping: along the tables' tangent in it, on the device.
            from acoustic_spaces_b200.layouts import LAYER_CELLS, LAYER_DAMPING, damping_tangent

            tangent = damping_tangent(workload.built.layout, LAYER_CELLS, LAYER_DAMPING)
            damping_s, damping_taped_s, with_damping = taped_gradient(False, tangent)
            grad_solver.set_layer_tangent(None)
            tables_along = sum(float(np.sum(with_tables[k] * tangent[k])) for k in tangent)
            adjoint = {
                "ratio": round(both_s / forward_s, 3),
                "steps": g_steps,
                "segment": args.gradient_segment,
                "forward_s": round(forward_s, 4),
                "forward_and_adjoint_s": round(both_s, 4),
                "taped_forward_s": round(taped_s, 4),
                "finite": bool(all(np.isfinite(v).all() for v in grads.values())),
                "gradient_in": "the walls' coefficients and branch states (the matched layer's tables fixed)",
                "with_layer_tables": {
                    "ratio": round(tables_s / forward_s, 3),
                    "forward_and_adjoint_s": round(tables_s, 4),
                    "finite": bool(all(np.isfinite(v).all() for v in with_tables.values())),
                    "walls_equal": bool(all(np.array_equal(grads[k], with_tables[k]) for k in grads)),
                },
                "with_layer_damping": {
                    "ratio": round(damping_s / forward_s, 3),
                    "forward_and_adjoint_s": round(damping_s, 4),
                    "taped_forward_s": round(damping_taped_s, 4),
                    "dloss_ddamping": with_damping["layer_tangent"],
                    "tables_gradient_along_the_tangent": tables_along,
                    "walls_equal": bool(all(np.array_equal(grads[k], with_damping[k]) for k in grads)),
                    "what": "dL/d(layer damping) on the device along the tables' tangent in the damping "
                            "(fdtd_set_layer_tangent): the taped run keeps three factors a layer cell and "
                            "damped axis a step beside the rows' trajectory, and the gradient recomputes nothing; "
                            "both values are 0 while the window is too short for sound to reach the layer and "
                            "come back to a receiver (the gradient's values are checked by the GPU tests)",
                },
                "what": "taped forward + gradient over the same steps, against a plain forward run; wall clock through "
                        "B200WaveSolver, the tape and workspace kept from an untimed first pass as a fit keeps them; "
                        "walls only: the rows' trajectory tape (nothing recomputed); with the layer's tables: "
                        "checkpoints every `segment` steps, each segment recomputed with the layer's factors",
            }  # fmt: skip
            grad_solver.close()
        except Exception as error:  # reported, not required
            adjoint = {"ratio": None, "error": str(error)[:300]}
    insertion = None
    if args.workload == "outdoor_halfspace" and not args.no_ir_error:
        insertion = outdoor_insertion_loss(args, workload, local)

    bytes_per_step = algorithmic_bytes(desc, args.precision)
    peak, peak_source = measured_peaks()
    achieved = bytes_per_step / (ms / 1e3 / steps) / 1e9
    # Each kernel's algorithmic bytes per launch and its average launch time, live.
    per_kernel_bytes = kind_bytes(desc, args.precision)
    traffic_table = {}
    suffix = "" if args.precision == "fp32" else f"_{args.precision}"
    traffic_file = ROOT / "profiles" / f"kernel_traffic_{args.workload}{suffix}.json"
    if traffic_file.exists() and (args.cell == 0.04 or args.workload != "polyhedral_room"):
        traffic_table = json.loads(traffic_file.read_text()).get("dram_bytes_per_launch", {})
    kernels = {}
    for kind, nbytes in per_kernel_bytes.items():
        launch_s = kernel_ms[kind] / 1e3 / max(1, kernel_ms["steps"])
        got = nbytes / launch_s / 1e9 if launch_s > 0 else None
        kernels[kind] = {
            "algorithmic_bytes_per_launch": nbytes,
            "mean_launch_us": round(launch_s * 1e6, 2),
            "achieved": round(got, 1) if got else None,
            "frac": round(got / peak, 4) if got else None,
            "traffic": traffic_table.get(kind),
        }
    kernels["probe"] = {"mean_launch_us": round(kernel_ms["probe"] / max(1, kernel_ms["steps"]) * 1e3, 2)}
    dominant = max(per_kernel_bytes, key=lambda k: kernel_ms[k])
    # Launches a step: the interior sweep, the matched layer, the special rows, the probes (each
    # when the grid has such cells).
    launches_per_step = sum(int(desc[k] > 0) for k in ("interior_cells", "layer_cells", "special_rows")) + int(solver.probes > 0)

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                cpu = cpu_reference_rate(workload, args.cpu_steps, fitted_walls=args.walls == "fitted")
            except Exception as error:  # the baseline is reported, not required
                cpu = {"value": None, "unit": UNIT, "error": str(error)[:200]}
        line = {
            "metric": METRIC,
            "value": round(value, 4),
            "unit": UNIT,
            "n_gpus": world,
            "steps": steps,
            "warmup": warmup,
            "ms_per_step": round(ms / steps, 5),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {
                "workload": workload.name,
                **desc,
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                "l2": "inputs larger than L2 (two pressure levels alone are "
                f"{2 * 4 * desc['cells'] / 1e6:.0f} MB vs 126 MB L2), no flush",
                "launch": solver.launch,
                "setup_s": {"layout_on_host": round(layout_s, 2), "create_and_autotune": round(handle_s, 2)},
                "precision": "FP32, bit-exact with the reference (no FMA, subnormals flushed)"
                if args.precision == "fp32"
                else "FP32 compensated: each cell's pressure and its increment (not bit-equal to the reference)",
            },
            "e2e": e2e,
            "gpu_launches": launches_per_step * steps,
            "roofline": {
                "bound": "hbm",
                "kernel": f"{dominant}_kernel (the longest of the step's kernels, by CUDA events)",
                "achieved": kernels[dominant]["achieved"],
                "peak": peak,
                "unit": "GB/s",
                "frac": kernels[dominant]["frac"],
                "traffic": kernels[dominant]["traffic"],
                "algorithmic_bytes_per_launch": per_kernel_bytes[dominant],
                "peak_source": peak_source,
                "kernels": kernels,
                "step": {
                    "algorithmic_bytes": bytes_per_step,
                    "achieved": round(achieved, 1),
                    "frac": round(achieved / peak, 4),
                    "bulk_12B_per_air_cell_frac": round(12 * air / (ms / 1e3 / steps) / 1e9 / peak, 4),
                },
            },
            "cpu_baseline": cpu,
            "ir_error_vs_fp64": ir_error,
            "fp64_same_gpu": fp64_rate,
            "insertion_loss_vs_fp64": insertion,
            "adjoint_over_forward": adjoint,
            "compensated": compensated,
            "clocks": clocks.summary(),
            "finite": finite,
        }
        print(json.dumps(line), flush=True)
    del solver
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
