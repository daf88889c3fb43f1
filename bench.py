"""Throughput of the CUDA leapfrog on the large plain-method room, in Gcell-updates/s.

Workload (one bench step = one full impulse-response run): 384^3 cells at dx = c/(10*4 kHz),
float32, per-wall absorption drawn U(0.05, 0.5) (seeded), a 16-cell sponge on the two x faces,
ISO 9613-1 air at 20 C / 50 % RH (three relaxation states: O2, N2, classical), a Gaussian pulse
to 4 kHz at a seeded interior cell and four seeded receivers, 4000 leapfrog steps. The fields
(2.5 GB) are far larger than L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

``value`` is device-timed (CUDA events on the launching stream, inputs resident in HBM); ``e2e``
goes through the public API with host buffers: upload the full state from pinned host memory,
run, read back the recordings and the final pressure. The reference arm times the reference's
own compiled C backend (``oracle/_ref``) on the host cores over a bounded sample of the same
workload. Multi-GPU runs are independent replicas of the room (one per rank, weak scaling);
``--slabs`` cuts the one room into an x slab per rank instead (strong scaling, one line with
``value`` and clocks only).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Gcell-updates/s"
N_RECEIVERS = 4


def workload(size: int, seed: int = 2, walls_only: bool = False):
    """The headline room; ``walls_only`` keeps its walls, source and receivers and drops the
    sponge and the air (the room the pressure-only scheme can run)."""
    from ac_fdtd_b200.workloads import plain_room_large

    grid, objects, source, receivers = plain_room_large(size, seed, N_RECEIVERS)
    if walls_only:
        objects = dict(walls=objects["walls"])
    return grid, objects, [source, *receivers]


def config_dict(args, grid) -> dict:
    physics = ("" if getattr(args, "walls_only", False) else
               "16-cell sponge on 2 x faces, ISO air 20C/50%RH (3 relaxation states), ")
    return {
        "workload": f"plain-method room {grid.nx}^3 fp32, 6 walls alpha~U(0.05,0.5), {physics}"
                    f"gaussian pulse 4 kHz, {N_RECEIVERS} receivers, {args.time_steps} steps "
                    f"per bench step",
        "cells": grid.n_cells,
        "time_steps_per_bench_step": args.time_steps,
        "relaxation_states": 0 if getattr(args, "walls_only", False) else 3,
        "dtype": "float32",
        "l2": "inputs larger than L2 (fields 2.5 GB at 384^3); no flush",
        "parallelism": f"replicas x{args.gpus}",
    }


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: str):
        self.device = device
        self.rows: list[list[str]] = []
        self._stop = threading.Event()
        self._thread = threading.Thread(target=self._loop, daemon=True)

    def _loop(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._thread.join(timeout=10)

    def summary(self) -> dict:
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        sm_max = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower().startswith("active")})
        loaded = [s for s in sm if s > 0] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(sm_max) if sm_max else None, "reasons": reasons,
                "samples": len(self.rows)}


def measured_peak_hbm() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        try:
            return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def ncu_traffic_per_cell(kernel: str) -> float | None:
    """DRAM bytes per cell of one launch of ``kernel``, from the committed ncu summary
    (``profiles/dram_traffic.json``: one ncu capture on a 256^3 case, scaled per cell)."""
    path = ROOT / "profiles" / "dram_traffic.json"
    if not path.exists():
        return None
    try:
        return float(json.loads(path.read_text())[kernel]["dram_bytes_per_cell"])
    except Exception:
        return None


def launch_dict(geometry) -> dict:
    if geometry[0] == "staged":
        return {"scheme": "staged", "rows_per_cta": geometry[1], "stages": geometry[2] or "auto",
                "planes_per_cta": geometry[3], "z_elements_per_thread": geometry[4]}
    return {"scheme": geometry[0], "block_threads": geometry[1], "planes_per_block": geometry[2]}


# --------------------------------------------------------------------------- CPU baseline
def cpu_baseline(size: int, budget_s: float = 12.0) -> dict:
    """The reference C backend on this host's cores, on a bounded sample of the workload."""
    from oracle import ref_c

    grid, objects, points = workload(size)
    if ref_c.available() or ref_c.build():
        from ac_fdtd_b200 import AIR

        solver = ref_c.RefCSolver(grid, AIR, dtype=np.float32, threads=0, **objects)
        kind = "reference"
        cores = solver.threads
    else:
        from ac_fdtd_b200 import AIR
        from oracle.leapfrog import OracleFDTD

        solver = OracleFDTD(grid, AIR, dtype=np.float32, **objects)
        kind = "port"
        cores = 1
    from ac_fdtd_b200 import gaussian_pulse

    solver.add_volume_source(points[0], gaussian_pulse(4000, solver.dt, 4000.0))
    for point in points[1:]:
        solver.add_pressure_receiver(point)
    solver.run(2)  # warm-up: first touch of the 1.6 GB of host fields
    start = time.perf_counter()
    solver.run(2)
    per_step = (time.perf_counter() - start) / 2
    steps = int(max(2, min(400, budget_s / max(per_step, 1e-6))))
    start = time.perf_counter()
    solver.run(steps)
    elapsed = time.perf_counter() - start
    value = grid.n_cells * steps / elapsed / 1e9
    return {"value": value, "unit": METRIC, "cores": int(cores), "kind": kind,
            "host_cpus": os.cpu_count(), "cpu_model": cpu_model(),
            "sample": f"{size}^3 fp32 same room, {steps} leapfrog steps after 4 warm-up steps, "
                      f"{elapsed:.1f} s",
            "sample_leapfrog_steps": steps, "sample_ms": elapsed * 1e3}


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    values, sample_ms, leapfrog_steps = [], [], []
    last = None
    for _ in range(args.warmup):
        cpu_baseline(args.size, budget_s=2.0)
    for _ in range(args.steps):
        last = cpu_baseline(args.size, budget_s=args.cpu_budget)
        values.append(last["value"])
        sample_ms.append(last["sample_ms"])
        leapfrog_steps.append(last["sample_leapfrog_steps"])
    from ac_fdtd_b200 import Grid

    grid = Grid(dx=343.2 / 40000.0, nx=args.size, ny=args.size, nz=args.size)
    value = float(statistics.median(values))
    # One bench step of this arm is one bounded sample of the workload: `sample_leapfrog_steps`
    # leapfrog steps of the 384^3 room, timed in full; ms_per_step is that sample's time, so
    # steps x ms_per_step is the work that actually ran. The rate extrapolates to the full
    # 4000-step run only through `value`.
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": float(statistics.mean(sample_ms)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {**config_dict(args, grid),
                   "bench_step": "one bounded sample of the room: sample_leapfrog_steps leapfrog "
                                 "steps from a fresh solver (CPU time budget per sample)",
                   "sample_leapfrog_steps": leapfrog_steps},
        "cpu_baseline": {**last, "value": value},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- our arm
def physical_gpu(local: int) -> str:
    """The GPU (index or UUID, as CUDA_VISIBLE_DEVICES names it) that local rank `local` runs on."""
    visible = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    return visible[local] if local < len(visible) else str(local)


def run_slab_mode(args) -> None:
    """``--slabs``: the headline room cut into one x slab per rank, a ghost p plane exchanged
    each way per cut and step (``DistributedSlabRoom``; one batched isend/irecv over NCCL), for
    strong scaling of one room. The default mode (replicas) gives the headline line."""
    import datetime
    import socket

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    gpu = physical_gpu(int(os.environ.get("LOCAL_RANK", "0")))
    os.environ["CUDA_VISIBLE_DEVICES"] = gpu
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(0)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", 0))
    else:       # a one-rank group, so the same class runs
        with socket.socket() as sock:
            sock.bind(("127.0.0.1", 0))
            port = sock.getsockname()[1]
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0,
                                world_size=1)
    from ac_fdtd_b200 import gaussian_pulse
    from ac_fdtd_b200.slabs import DistributedSlabRoom

    grid, objects, points = workload(args.size)
    room = DistributedSlabRoom(grid, dtype=np.float32, device=0, **objects)
    T = args.time_steps
    room.add_volume_source(points[0], gaussian_pulse(T, room.dt, 4000.0))
    for point in points[1:]:
        room.add_pressure_receiver(point)

    def one_run():
        room.slab.solver.step_index = 0
        room.run(T)

    for _ in range(args.warmup):
        one_run()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu) as clocks:
        dist.barrier()
        torch.cuda.synchronize()
        start.record()
        for _ in range(args.steps):
            one_run()
        end.record()
        torch.cuda.synchronize()
        dist.barrier()
    elapsed = torch.tensor([start.elapsed_time(end)], dtype=torch.float64,
                           device="cuda" if world > 1 else "cpu")
    dist.all_reduce(elapsed, op=dist.ReduceOp.MAX)
    elapsed_ms = float(elapsed.item())
    room.close()
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": grid.n_cells * T * args.steps / (elapsed_ms * 1e-3) / 1e9,
            "unit": METRIC, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {**config_dict(args, grid), "parallelism": f"x slabs x{world}",
                       "exchange": "ghost p planes, one batched isend/irecv per rank and step"},
            "clocks": clocks.summary(),
        }), flush=True)


def run_ours(args) -> None:
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    gpu = physical_gpu(local)
    # One visible GPU per process, before CUDA starts: device 0 is then the same GPU for torch
    # (NCCL, events) and for the CUDA library's own runtime, whatever device either would pick.
    os.environ["CUDA_VISIBLE_DEVICES"] = gpu
    import torch

    torch.cuda.set_device(0)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", 0))

    from ac_fdtd_b200 import CudaAcousticFDTD, gaussian_pulse, pinned_array

    from ac_fdtd_b200.autotune import _apply as apply_geometry
    from ac_fdtd_b200.autotune import apply_tuned

    grid, objects, points = workload(args.size, walls_only=args.walls_only)
    solver = CudaAcousticFDTD(grid, dtype=np.float32, **objects)
    if args.launch:
        parts = args.launch.split(",")
        geometry = (parts[0], *map(int, parts[1:]))
        apply_geometry(solver, geometry)
    else:
        geometry = apply_tuned(solver)
    solver.add_volume_source(points[0], gaussian_pulse(args.time_steps, solver.dt, 4000.0))
    for point in points[1:]:
        solver.add_pressure_receiver(point)
    T = args.time_steps

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def one_run():
        solver.step_index = 0
        solver.run(T)

    # ---- device-resident timing of the runs as the API runs them (CUDA graphs), CUDA events
    # around the timed region; then one more run with CUDA events around every launch, for the
    # per-sweep times of the two-sweep scheme and as a cross-check of the others
    for _ in range(args.warmup):
        one_run()
    launches0 = solver.launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu) as clocks:
        barrier()
        start.record()
        for _ in range(args.steps):
            one_run()
        end.record()
        barrier()
    region_ms = start.elapsed_time(end)
    elapsed_ms = max_over_ranks(region_ms)
    launches = solver.launch_count() - launches0
    solver.profile(True)
    one_run()
    vel_ms, pres_ms, timed_steps = solver.profile_read()
    solver.profile(False)
    cell_updates = grid.n_cells * T * args.steps * world
    value = cell_updates / (elapsed_ms * 1e-3) / 1e9

    # ---- roofline of the dominant kernel: the fused step, the pressure-only step, or the
    # pressure sweep
    R = 0 if args.walls_only else 3
    itemsize = 4
    layer = "nolayer" if args.walls_only else "layer"
    peak, peak_kind = measured_peak_hbm()
    peak_source = (f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                   else "fallback 6650 GB/s")
    vel_avg = vel_ms / max(timed_steps, 1)
    pres_avg = pres_ms / max(timed_steps, 1)
    # One kernel per step (fused, staged, pressure-only): its average launch over the timed
    # region is the region's event time over its launches (one per leapfrog step; the graphs'
    # step-counter bumps, one per 64 steps, are counted in it).
    region_avg = region_ms / max(T * args.steps, 1)
    if geometry[0] == "pressure_only":
        step_bytes = grid.n_cells * 3 * itemsize
        step_avg = region_avg
        achieved = step_bytes / (step_avg * 1e-3) / 1e9
        traffic_per_cell = ncu_traffic_per_cell("pressure_only_sweep")
        roofline = {
            "bound": "hbm", "kernel": "pressure_only_sweep<float,walls>",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": peak_source, "algorithmic_bytes_per_launch": step_bytes,
            "bytes_per_cell": 3 * itemsize, "avg_launch_ms": step_avg,
            "avg_launch_ms_source": "timed region / launches",
            "avg_launch_ms_per_launch_events": vel_avg + pres_avg,
            "traffic": None if traffic_per_cell is None else traffic_per_cell * grid.n_cells,
        }
    elif geometry[0] in ("fused", "staged"):
        if geometry[0] == "staged":
            kernel, label = "fused_staged_sweep", f"fused_staged_sweep<float,{layer},walls,{R}>"
        else:                      # single precision: the lean column
            kernel = "lean_sweep"
            label = (f"lean_sweep<{layer},walls,{R}>" if grid.nz % 4 == 0
                     else f"lean_sweep_padded<{layer},walls,{R}>")
        step_bytes = grid.n_cells * (8 + 2 * R) * itemsize
        step_avg = region_avg
        achieved = step_bytes / (step_avg * 1e-3) / 1e9
        traffic_per_cell = ncu_traffic_per_cell(kernel)
        roofline = {
            "bound": "hbm", "kernel": label,
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": peak_source, "algorithmic_bytes_per_launch": step_bytes,
            "bytes_per_cell": (8 + 2 * R) * itemsize, "avg_launch_ms": step_avg,
            "avg_launch_ms_source": "timed region / launches",
            "avg_launch_ms_per_launch_events": vel_avg + pres_avg,
            "traffic": None if traffic_per_cell is None else traffic_per_cell * grid.n_cells,
            "two_sweep_equivalent": {"bytes_per_cell": (12 + 2 * R) * itemsize,
                                     "effective_GBps": grid.n_cells * (12 + 2 * R) * itemsize
                                     / (step_avg * 1e-3) / 1e9},
        }
    else:
        pressure_bytes = grid.n_cells * (5 + 2 * R) * itemsize
        velocity_bytes = grid.n_cells * 7 * itemsize
        achieved = pressure_bytes / (pres_avg * 1e-3) / 1e9
        traffic_per_cell = ncu_traffic_per_cell("pressure_sweep")
        roofline = {
            "bound": "hbm", "kernel": "pressure_sweep<float,layer,walls,3>",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": peak_source, "algorithmic_bytes_per_launch": pressure_bytes,
            "bytes_per_cell": (5 + 2 * R) * itemsize, "avg_launch_ms": pres_avg,
            "traffic": None if traffic_per_cell is None else traffic_per_cell * grid.n_cells,
            "velocity_sweep": {"avg_launch_ms": vel_avg, "bytes_per_cell": 7 * itemsize,
                               "achieved": velocity_bytes / (vel_avg * 1e-3) / 1e9},
            "step": {"bytes_per_cell": (12 + 2 * R) * itemsize,
                     "achieved": (pressure_bytes + velocity_bytes) / ((pres_avg + vel_avg) * 1e-3) / 1e9,
                     "frac": (pressure_bytes + velocity_bytes) / ((pres_avg + vel_avg) * 1e-3) / 1e9 / peak},
        }

    # ---- end to end through the public API with pinned host buffers
    p0 = pinned_array(grid.shape, np.float32)
    v0 = [pinned_array(grid.velocity_shape(a), np.float32) for a in range(3)]
    psi0 = [pinned_array(grid.shape, np.float32) for _ in range(R)]
    p_out = pinned_array(grid.shape, np.float32)
    p0[...] = np.random.default_rng(rank).standard_normal(grid.shape).astype(np.float32) * 1e-3

    phase_ms = {"h2d_ms": 0.0, "run_ms": 0.0, "d2h_ms": 0.0}
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(4)]

    def e2e_step(timed: bool):
        # Each phase is bracketed by CUDA events on the solver's stream (the legacy default
        # stream, torch's current one); set_state and get_state return after their copies.
        solver.step_index = 0
        marks[0].record()
        if geometry[0] == "pressure_only":
            solver.reset_state()          # its velocities are only taken before the first step
        h2d = solver.set_state(p=p0, velocity=v0, relaxation=psi0)
        marks[1].record()
        solver.run(T)
        marks[2].record()
        recorded = solver.recorded_pressure
        d2h = solver.get_state(p=p_out) + recorded.nbytes
        marks[3].record()
        if timed:
            marks[3].synchronize()
            for key, (a, b) in zip(phase_ms, ((0, 1), (1, 2), (2, 3))):
                phase_ms[key] += marks[a].elapsed_time(marks[b])
        return h2d, d2h

    for _ in range(min(args.warmup, 1)):
        e2e_step(False)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        h2d, d2h = e2e_step(True)
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = cell_updates / e2e_s / 1e9
    phases = {k: v / args.steps for k, v in phase_ms.items()}
    phases["h2d_GBps"] = h2d / (phases["h2d_ms"] * 1e-3) / 1e9 if phases["h2d_ms"] > 0 else None
    phases["d2h_GBps"] = d2h / (phases["d2h_ms"] * 1e-3) / 1e9 if phases["d2h_ms"] > 0 else None

    # The extra sections are single-GPU measurements: the N = 1 line carries them, and a
    # multi-rank run does not hold its GPUs for them.
    skip = args.skip_extras or world > 1
    batched = None if skip else batched_vs_per_room(args)
    adjoint = None if skip else adjoint_cost(args)
    inversion = None if skip else batched_adjoint_cost(args)
    precision = None if skip else precision_check(args)
    slabs = None if skip else slab_overhead(args)
    pressure_only = None if skip else pressure_only_cost(args)
    time_blocking = None if skip else time_blocking_cost(args)

    clock_record = clocks.summary()
    if clock_record.get("sm_mhz"):
        # Launch time in SM clock cycles at the median loaded clock: separates the code's cost
        # from the clock the power cap allowed (ms x MHz = thousands of cycles).
        avg_ms = roofline.get("avg_launch_ms") or 0.0
        roofline["launch_kcycles_at_median_sm_clock"] = avg_ms * clock_record["sm_mhz"]
        roofline["median_sm_mhz"] = clock_record["sm_mhz"]
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {**config_dict(args, grid),
                   "launch": {**launch_dict(geometry),
                              "chosen_by": "--launch" if args.launch else "ac_fdtd_b200.autotune"}},
        "roofline": roofline,
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "path": f"CudaAcousticFDTD.set_state (pinned host) -> run({T}) -> "
                        "recorded_pressure, get_state (pinned host)",
                "phases_per_step": phases},
        "gpu_launches": launches,
        "clocks": clock_record,
        "batched": batched,
        "adjoint": adjoint,
        "batched_inversion": inversion,
        "precision": precision,
        "slabs_one_gpu": slabs,
        "pressure_only": pressure_only,
        "time_blocking": time_blocking,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.size, budget_s=args.cpu_budget)
        if not args.skip_extras:
            line["comparators"] = comparators(args)
    elif rank == 0:
        line["cpu_baseline"] = None
    solver.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        line["extras_summary"] = extras_summary(line)     # last key: the end of the line
        print(json.dumps(line), flush=True)


def extras_summary(line: dict) -> dict:
    """The headline figures of the extra sections, compact, so that the end of the JSON line
    (what a log tail keeps) carries them."""
    def get(*path):
        node = line
        for key in path:
            if not isinstance(node, dict) or key not in node:
                return None
            node = node[key]
        return float(f"{node:.5g}") if isinstance(node, float) else node

    return {
        "gcups": get("value"), "e2e_gcups": get("e2e", "value"), "frac": get("roofline", "frac"),
        "e2e_h2d_ms": get("e2e", "phases_per_step", "h2d_ms"),
        "e2e_run_ms": get("e2e", "phases_per_step", "run_ms"),
        "e2e_d2h_ms": get("e2e", "phases_per_step", "d2h_ms"),
        "cpu_ref_gcups": get("cpu_baseline", "value"),
        "batched_speedup": get("batched", "speedup"),
        "batched_ceiling": get("batched", "batching_ceiling_speedup"),
        "small_rooms_speedup": get("batched", "small_rooms", "speedup"),
        "grad_ratio_walls": get("adjoint", "walls_and_signal", "ratio"),
        "grad_ratio_air": get("adjoint", "walls_signal_and_air", "ratio"),
        "inversion_ratio": get("batched_inversion", "ratio"),
        "fp32_rel_l2_384": get("precision", "room_384", "fp32_vs_fp64", "rel_l2"),
        "fp64_gcups_384": get("precision", "room_384", "fp64_gcups"),
        "torch_cuda_gcups_384": get("comparators", "gpu", "room_384_fp32", "gcups"),
        "c_fp64_gcups_384": get("comparators", "cpu", "c_fp64_room_384", "gcups"),
        "numpy_gcups_64": get("comparators", "cpu", "numpy_fp64_room_64", "gcups"),
        "pressure_only_gcups": get("pressure_only", "pressure_only", "gcups"),
        "pressure_only_frac": get("pressure_only", "pressure_only", "hbm_frac_of_measured"),
        "pressure_only_speedup": get("pressure_only", "speedup_over_fused"),
        "time_blocking_speedup": get("time_blocking", "speedup"),
    }


def reference_package():
    """The unmodified reference package installed under ``baseline/_ref`` (git-ignored, made
    by ``__graft_entry__.build()``), or None. Appended to the path, so only ``ac_fdtd`` itself
    can resolve from there."""
    path = ROOT / "baseline" / "_ref"
    if not (path / "ac_fdtd" / "__init__.py").exists():
        return None
    if str(path) not in sys.path:
        sys.path.append(str(path))
    import ac_fdtd

    return ac_fdtd


def _as_reference(ref, grid, objects: dict):
    """The reference's own value objects with the same parameters as ours."""
    import dataclasses

    rgrid = ref.Grid(dx=grid.dx, nx=grid.nx, ny=grid.ny, nz=grid.nz)
    kinds = {"walls": ref.WallAdmittances, "absorbing_layer": ref.AbsorbingLayer,
             "air_absorption": ref.AirAbsorption}
    out = {}
    for key, value in objects.items():
        if value is not None:
            out[key] = kinds[key](**{f.name: getattr(value, f.name)
                                     for f in dataclasses.fields(value)})
    return rgrid, out


def comparators(args) -> dict:
    """Comparators beside the C fp32 reference arm, each through the reference's own code path
    (never this package's kernels):

    * ``gpu``: the reference's whole-array Torch backend ``TorchAcousticFDTD(device="cuda")``
      (ac-fdtd ``src/ac_fdtd/torch_backend.py:234-316``) on this GPU -- the 384^3 room in fp32
      over a bounded sample after 3 warm-up steps, and the 64^3 plain room (walls 0.15, 2000
      steps) in fp64 and fp32 in full -- beside this package on the same 64^3 runs;
    * ``cpu``: the reference's C backend in fp64 on the 384^3 room (bounded sample), C fp64
      and the NumPy reference in full on the 64^3 room, and the per-room C run over the 64
      uneven rooms (a bounded number of steps per room), on this host's cores.
    """
    import torch

    from ac_fdtd_b200 import AIR, CudaAcousticFDTD, gaussian_pulse
    from ac_fdtd_b200.sources import gaussian_derivative_pulse
    from ac_fdtd_b200.workloads import plain_room_small, uneven_rooms

    ref = reference_package()
    out = {"reference_package": "baseline/_ref/ac_fdtd (unmodified)" if ref else None}
    grid1, objects1, source1, receivers1 = plain_room_small()
    T1 = 2000

    def small_signal(dt):      # d/dt of the 1 kHz Gaussian, as the 64^3 configuration has it
        return gaussian_derivative_pulse(T1, dt, 1000.0)

    gpu = {}
    if ref is None:
        gpu["unavailable"] = "the reference package is not installed under baseline/_ref"
    else:
        from ac_fdtd.torch_backend import TorchAcousticFDTD

        grid, objects, points = workload(args.size)
        rgrid, robjects = _as_reference(ref, grid, objects)
        solver = TorchAcousticFDTD(rgrid, device="cuda", dtype=torch.float32, **robjects)
        solver.add_volume_source(points[0], ref.gaussian_pulse(args.time_steps, solver.dt, 4000.0))
        for point in points[1:]:
            solver.add_pressure_receiver(point)
        solver.run(3)
        steps = 100
        ms = _device_ms(lambda: solver.run(steps), torch)
        gpu["room_384_fp32"] = {
            "gcups": grid.n_cells * steps / (ms * 1e-3) / 1e9,
            "sample": f"{steps} leapfrog steps of the {args.size}^3 room after 3 warm-up steps, "
                      f"{ms:.0f} ms, CUDA events",
        }
        del solver
        torch.cuda.empty_cache()
        rgrid1, robjects1 = _as_reference(ref, grid1, objects1)
        for dtype, tdtype in ((np.float64, torch.float64), (np.float32, torch.float32)):
            name = np.dtype(dtype).name
            solver = TorchAcousticFDTD(rgrid1, device="cuda", dtype=tdtype, **robjects1)
            solver.add_volume_source(source1, small_signal(solver.dt))
            for point in receivers1:
                solver.add_pressure_receiver(point)
            ms = _device_ms(lambda: solver.run(T1), torch)
            torch_rec = solver.recorded_pressure
            ours = CudaAcousticFDTD(grid1, dtype=dtype, **objects1)
            from ac_fdtd_b200.autotune import apply_tuned

            apply_tuned(ours)
            ours.add_volume_source(source1, small_signal(ours.dt))
            for point in receivers1:
                ours.add_pressure_receiver(point)
            ours.run(3)          # warm-up: graph capture
            ours.reset_state()
            ours.step_index = 0
            ours_ms = _device_ms(lambda: ours.run(T1), torch)
            ours_rec = ours.recorded_pressure
            ours.close()
            gpu[f"room_64_{name}"] = {
                "reference_torch_gcups": grid1.n_cells * T1 / (ms * 1e-3) / 1e9,
                "ours_gcups": grid1.n_cells * T1 / (ours_ms * 1e-3) / 1e9,
                "speedup": ms / ours_ms,
                "receiver_max_diff_over_peak": float(np.max(np.abs(ours_rec - torch_rec))
                                                     / np.max(np.abs(torch_rec))),
                "sample": f"{T1} steps in full, one run, CUDA events",
            }
            del solver
    out["gpu"] = gpu

    cpu = {"host_cpus": os.cpu_count(), "cpu_model": cpu_model()}
    from oracle import ref_c

    if ref_c.available():
        grid, objects, points = workload(args.size)
        solver = ref_c.RefCSolver(grid, AIR, dtype=np.float64, threads=0, **objects)
        solver.add_volume_source(points[0], gaussian_pulse(args.time_steps, solver.dt, 4000.0))
        for point in points[1:]:
            solver.add_pressure_receiver(point)
        solver.run(2)
        steps = 60
        t0 = time.perf_counter()
        solver.run(steps)
        elapsed = time.perf_counter() - t0
        cpu["c_fp64_room_384"] = {"gcups": grid.n_cells * steps / elapsed / 1e9,
                                  "threads": solver.threads,
                                  "sample": f"{steps} leapfrog steps after 2, {elapsed:.1f} s"}
        del solver
        solver = ref_c.RefCSolver(grid1, AIR, dtype=np.float64, threads=0, **objects1)
        solver.add_volume_source(source1, small_signal(solver.dt))
        for point in receivers1:
            solver.add_pressure_receiver(point)
        t0 = time.perf_counter()
        solver.run(T1)
        elapsed = time.perf_counter() - t0
        cpu["c_fp64_room_64"] = {"gcups": grid1.n_cells * T1 / elapsed / 1e9,
                                 "threads": solver.threads,
                                 "sample": f"{T1} steps in full, {elapsed:.1f} s"}
        rooms = uneven_rooms()
        per_room_steps = 10
        cells = 0
        elapsed = 0.0
        threads = 0
        for spec, source, receivers in rooms:
            solver = ref_c.RefCSolver(spec["grid"], AIR, dtype=np.float32, threads=0,
                                      walls=spec["walls"], air_absorption=spec["air_absorption"])
            threads = solver.threads
            solver.add_volume_source(source, gaussian_pulse(args.batch_steps, solver.dt, 2000.0))
            for point in receivers:
                solver.add_pressure_receiver(point)
            t0 = time.perf_counter()
            solver.run(per_room_steps)
            elapsed += time.perf_counter() - t0
            cells += spec["grid"].n_cells
        cpu["c_fp32_uneven_rooms_per_room"] = {
            "gcups": cells * per_room_steps / elapsed / 1e9, "threads": threads,
            "sample": f"each of the 64 rooms for {per_room_steps} steps ({elapsed:.1f} s)"}
    else:
        cpu["c"] = "unavailable: oracle/_ref not built"
    if ref is not None:
        solver = ref.AcousticFDTD(ref.Grid(dx=grid1.dx, nx=grid1.nx, ny=grid1.ny, nz=grid1.nz),
                                  walls=ref.WallAdmittances.from_absorption(0.15))
        solver.add_volume_source(source1, small_signal(solver.dt))
        for point in receivers1:
            solver.add_pressure_receiver(point)
        t0 = time.perf_counter()
        solver.run(T1)
        elapsed = time.perf_counter() - t0
        cpu["numpy_fp64_room_64"] = {"gcups": grid1.n_cells * T1 / elapsed / 1e9, "threads": 1,
                                     "sample": f"{T1} steps in full, {elapsed:.1f} s"}
    out["cpu"] = cpu
    return out


def pressure_only_cost(args) -> dict:
    """The pressure-only scheme against the p-v leapfrog on the headline room without its sponge
    and air (neither exists in the second-order pressure equation): 384^3 fp32, the six walls,
    the source and four receivers, 1000 steps each from rest. Kernel time from CUDA events
    around every launch (one kernel per step in both schemes), run time from events around the
    run; receivers compared between the schemes."""
    import torch

    from ac_fdtd_b200 import CudaAcousticFDTD, gaussian_pulse
    from ac_fdtd_b200.autotune import apply_tuned

    grid, objects, points = workload(args.size)
    walls = objects["walls"]
    T = 1000
    peak, peak_kind = measured_peak_hbm()
    out = {"workload": f"{args.size}^3 fp32, the headline room's walls, no sponge, no air, "
                       f"{len(points) - 1} receivers, {T} steps from rest"}
    recordings = {}
    for scheme, bytes_per_cell in (("fused", 32), ("pressure_only", 12)):
        solver = CudaAcousticFDTD(grid, dtype=np.float32, walls=walls, scheme=scheme)
        launch = launch_dict(apply_tuned(solver, schemes=(scheme,)))
        solver.add_volume_source(points[0], gaussian_pulse(T, solver.dt, 4000.0))
        for point in points[1:]:
            solver.add_pressure_receiver(point)

        def run(solver=solver):
            solver.reset_state()
            solver.step_index = 0
            solver.run(T)

        run()
        run_ms = min(_device_ms(run, torch) for _ in range(2))
        recordings[scheme] = solver.recorded_pressure
        solver.reset_state()
        solver.step_index = 0
        solver.profile(True)
        solver.run(200)
        first_ms, second_ms, launches = solver.profile_read()
        solver.profile(False)
        kernel_ms = (first_ms + second_ms) / max(launches, 1)
        solver.close()
        achieved = grid.n_cells * bytes_per_cell / (kernel_ms * 1e-3) / 1e9
        out[scheme] = {
            "gcups": grid.n_cells * T / (run_ms * 1e-3) / 1e9, "bytes_per_cell": bytes_per_cell,
            "avg_launch_ms": kernel_ms, "achieved_GBps": achieved,
            f"hbm_frac_of_{peak_kind}": achieved / peak,
            # one kernel per step in both schemes: the whole graph-replayed run over its bytes
            f"run_hbm_frac_of_{peak_kind}": grid.n_cells * T * bytes_per_cell / (run_ms * 1e-3) / 1e9 / peak,
            "kernel": "lean_sweep<false,walls,0>" if scheme == "fused" else "pressure_only_sweep<float,walls>",
            "launch": launch,
        }
    rec = recordings["pressure_only"]
    out["speedup_over_fused"] = out["pressure_only"]["gcups"] / out["fused"]["gcups"]
    out["receivers_vs_fused_fp32"] = _errors(rec, recordings["fused"])
    return out


def time_blocking_cost(args) -> dict:
    """Two steps per launch (temporal blocking, ``set_time_blocking(2)``) against the one-step
    lean sweep on the headline room (walls, sponge, air, the source and receivers), 400 steps
    from rest each, device time from CUDA events around the run; recordings compared bit for
    bit. Algorithmic DRAM bytes per cell-step: 56 one step at a time, 28 two at a time (plus the
    first-step pressure ring, which stays in L2)."""
    import torch

    from ac_fdtd_b200 import CudaAcousticFDTD, gaussian_pulse

    grid, objects, points = workload(args.size)
    T = 400
    peak, peak_kind = measured_peak_hbm()
    out = {"workload": f"the headline room, {args.size}^3 fp32, {T} steps from rest"}
    recordings = {}
    for steps_per_launch, bytes_per_cell in ((1, 56), (2, 28)):
        solver = CudaAcousticFDTD(grid, dtype=np.float32, scheme="fused", **objects)
        if steps_per_launch == 2:
            solver.set_time_blocking(2)
        solver.add_volume_source(points[0], gaussian_pulse(T, solver.dt, 4000.0))
        for point in points[1:]:
            solver.add_pressure_receiver(point)

        def run(solver=solver):
            solver.reset_state()
            solver.step_index = 0
            solver.run(T)

        run()
        run_ms = min(_device_ms(run, torch) for _ in range(2))
        recordings[steps_per_launch] = solver.recorded_pressure
        solver.close()
        gcups = grid.n_cells * T / (run_ms * 1e-3) / 1e9
        out[f"steps_per_launch_{steps_per_launch}"] = {
            "gcups": gcups, "bytes_per_cell_step": bytes_per_cell,
            f"hbm_frac_of_{peak_kind}": gcups * bytes_per_cell / peak,
            "kernel": "lean_sweep<true,true,3>" if steps_per_launch == 1 else "lean_pair_sweep<true,true,3>",
        }
    out["speedup"] = out["steps_per_launch_2"]["gcups"] / out["steps_per_launch_1"]["gcups"]
    out["recordings_bitwise_equal"] = bool(np.array_equal(recordings[1], recordings[2]))
    return out


def slab_overhead(args) -> dict:
    """The x-slab decomposition's own cost with every part on this GPU: the headline room whole
    and cut into 2 and 4 slabs (300 steps), recordings compared bit for bit. Two sweeps: the
    pressure sweep stores the boundary planes into the neighbours' ghosts (acf_run_slabs);
    fused scheme: one lean step per part and step, storing its boundary planes into the
    neighbours' next-copy ghosts, the parts' launches replayed from one CUDA graph."""
    out = {"workload": f"the headline room, {args.size}^3 fp32, 300 steps, every part on one GPU"}
    for scheme, path in (("two_sweeps", "exchange fused into the pressure sweep"),
                         ("fused", "ghost stores fused into each part's lean step")):
        out[scheme] = {"exchange": path, **_slab_runs(args, scheme)}
    return out


def _slab_runs(args, scheme: str) -> dict:
    import torch

    from ac_fdtd_b200 import CudaAcousticFDTD, gaussian_pulse
    from ac_fdtd_b200.slabs import SlabGroup

    grid, objects, points = workload(args.size)
    T, warm = 300, 20
    out = {}
    whole_recording = None
    for parts in (1, 2, 4):
        room = (CudaAcousticFDTD(grid, dtype=np.float32, scheme=scheme, **objects) if parts == 1
                else SlabGroup(grid, dtype=np.float32, parts=parts, scheme=scheme, **objects))
        room.add_volume_source(points[0], gaussian_pulse(T + warm, room.dt, 4000.0))
        for point in points[1:]:
            room.add_pressure_receiver(point)
        room.run(warm)
        room.synchronize()
        ms = _device_ms(lambda room=room: room.run(T), torch)
        recording = room.recorded_pressure
        if whole_recording is None:
            whole_recording = recording
        out[f"parts_{parts}"] = {
            "gcups": grid.n_cells * T / (ms * 1e-3) / 1e9,
            "recordings_bitwise_equal_to_whole_room": bool(np.array_equal(recording, whole_recording)),
        }
        room.close()
    return out


def _errors(single, double) -> dict:
    """Relative L2 over every receiver and sample, and peak |error| over peak |p|."""
    a = np.asarray(single, dtype=np.float64)
    b = np.asarray(double, dtype=np.float64)
    return {"rel_l2": float(np.linalg.norm(a - b) / np.linalg.norm(b)),
            "peak": float(np.max(np.abs(a - b)) / np.max(np.abs(b)))}


def precision_check(args) -> dict:
    """FP32 receiver signals against FP64 on the same rooms, and the FP64 throughput at the
    headline size. The FP64 path performs the NumPy reference's float64 arithmetic bit for bit
    (tests/test_parity_gpu.py), so it stands in for the reference at sizes NumPy cannot run."""
    import torch

    from ac_fdtd_b200 import CudaAcousticFDTD, RoomBatch, WallAdmittances, gaussian_pulse
    from ac_fdtd_b200.autotune import apply_tuned
    from ac_fdtd_b200.workloads import differentiable_room, uneven_rooms

    out = {}
    # the headline room, T steps from rest in each precision
    grid, objects, points = workload(args.size)
    T = args.time_steps
    recordings, times, schemes = {}, {}, {}
    for dtype in (np.float32, np.float64):
        solver = CudaAcousticFDTD(grid, dtype=dtype, **objects)
        schemes[np.dtype(dtype).name] = launch_dict(apply_tuned(solver))
        solver.add_volume_source(points[0], gaussian_pulse(T, solver.dt, 4000.0))
        for point in points[1:]:
            solver.add_pressure_receiver(point)
        times[np.dtype(dtype).name] = _device_ms(lambda: solver.run(T), torch)
        recordings[dtype] = solver.recorded_pressure
        solver.close()
    f64_gcups = grid.n_cells * T / (times["float64"] * 1e-3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    out["room_384"] = {
        "workload": f"the headline room, {args.size}^3, {T} steps from rest, {len(points) - 1} receivers",
        "fp32_vs_fp64": _errors(recordings[np.float32], recordings[np.float64]),
        "fp64_gcups": f64_gcups,
        f"fp64_hbm_frac_of_{peak_kind}_at_112_B_per_cell": f64_gcups * 112 / peak,
        "fp64_launch": schemes["float64"],
        "note": "one run including its CUDA-graph capture, timed with CUDA events",
    }

    # the differentiable room (128^3, its true walls), adjoint-steps long
    grid4, true_xi, _, source, receivers = differentiable_room()
    T4 = args.adjoint_steps
    rec4 = {}
    for dtype in (np.float32, np.float64):
        solver = CudaAcousticFDTD(grid4, dtype=dtype, walls=WallAdmittances(*true_xi))
        solver.add_volume_source(source, gaussian_pulse(T4, solver.dt, 2000.0))
        for point in receivers:
            solver.add_pressure_receiver(point)
        solver.run(T4)
        rec4[dtype] = solver.recorded_pressure
        solver.close()
    out["differentiable_128"] = {"workload": f"128^3, {T4} steps, 4 receivers",
                                 "fp32_vs_fp64": _errors(rec4[np.float32], rec4[np.float64])}

    # the 64 uneven rooms, batched, batch-steps long: the worst room
    rooms = uneven_rooms()
    T3 = args.batch_steps
    rec3 = {}
    for dtype in (np.float32, np.float64):
        batch = RoomBatch([r[0] for r in rooms], dtype=dtype)
        for r, (_, src, recs) in enumerate(rooms):
            batch.add_volume_source(r, src, gaussian_pulse(T3, batch.dt(r), 2000.0))
            for point in recs:
                batch.add_pressure_receiver(r, point)
        batch.run(T3)
        rec3[dtype] = [batch.recorded_pressure(r) for r in range(len(rooms))]
        batch.close()
    per_room = [_errors(a, b) for a, b in zip(rec3[np.float32], rec3[np.float64])]
    out["uneven_rooms"] = {"workload": f"64 uneven rooms, {T3} steps, 2 receivers each",
                           "fp32_vs_fp64_worst_room": {
                               "rel_l2": max(e["rel_l2"] for e in per_room),
                               "peak": max(e["peak"] for e in per_room)},
                           "fp32_vs_fp64_median_room_rel_l2": float(np.median([e["rel_l2"] for e in per_room]))}
    return out


def _device_ms(fn, torch) -> float:
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    fn()
    end.record()
    torch.cuda.synchronize()
    return start.elapsed_time(end)


def batched_vs_per_room(args) -> dict:
    """64 uneven rooms (60-200 cells per axis, fp32, walls + ISO air): one RoomBatch against the
    same rooms run one after another, each as its own CudaAcousticFDTD (CUDA graphs in both).
    The same comparison on 64 small rooms (24-64 cells per axis), where launch gaps dominate the
    per-room arm, shows what batching buys when each room alone cannot fill the GPU."""
    from ac_fdtd_b200.workloads import uneven_rooms

    T = args.batch_steps
    out = _batch_vs_rooms(uneven_rooms(), T, args)
    out["workload"] = (f"64 rooms 3-10 m per axis at dx 5 cm ({out['cells']} cells, 60-200 per "
                       f"axis), fp32, walls alpha~U(0.05,0.5), ISO air T~U(15,25) C RH~U(30,70) %, "
                       f"1 source + 2 receivers per room, {T} steps (CUDA graphs in both arms)")
    small = _batch_vs_rooms(uneven_rooms(seed=6, lengths=(1.2, 3.2)), T, args)
    small["workload"] = (f"64 small rooms 1.2-3.2 m per axis at dx 5 cm ({small['cells']} cells, "
                         f"24-64 per axis), otherwise as above, {T} steps")
    out["small_rooms"] = small
    return out


def _batch_vs_rooms(rooms, T: int, args) -> dict:
    import torch

    from ac_fdtd_b200 import CudaAcousticFDTD, RoomBatch, gaussian_pulse
    from ac_fdtd_b200.autotune import apply_tuned_batch

    specs = [r[0] for r in rooms]
    cells = int(sum(spec["grid"].n_cells for spec in specs))
    batch = RoomBatch(specs, dtype=np.float32)
    batch_geometry = apply_tuned_batch(batch)
    for r, (spec, source, receivers) in enumerate(rooms):
        batch.add_volume_source(r, source, gaussian_pulse(T, batch.dt(r), 2000.0))
        for point in receivers:
            batch.add_pressure_receiver(r, point)

    def run_batch():
        batch.step_index = 0
        batch.run(T)

    for _ in range(max(1, args.warmup - 1)):
        run_batch()
    batch_ms = min(_device_ms(run_batch, torch) for _ in range(2))
    launches = batch.launch_count()
    batch.close()

    # each room on its own, one after another, in each scheme; the faster one is the per-room arm
    per_room = {}
    for scheme in ("two_sweeps", "fused"):
        solvers = []
        for spec, source, receivers in rooms:
            solver = CudaAcousticFDTD(spec["grid"], dtype=np.float32, walls=spec["walls"],
                                      air_absorption=spec["air_absorption"], scheme=scheme)
            solver.add_volume_source(source, gaussian_pulse(T, solver.dt, 2000.0))
            for point in receivers:
                solver.add_pressure_receiver(point)
            solvers.append(solver)

        def run_rooms():
            for solver in solvers:
                solver.step_index = 0
                solver.run(T)

        for _ in range(max(1, args.warmup - 1)):
            run_rooms()
        per_room[scheme] = min(_device_ms(run_rooms, torch) for _ in range(2))
        for solver in solvers:
            solver.close()
    best_scheme = min(per_room, key=per_room.get)
    per_room_ms = per_room[best_scheme]
    peak, peak_kind = measured_peak_hbm()
    batched_gcups = cells * T / (batch_ms * 1e-3) / 1e9
    per_room_gcups = cells * T / (per_room_ms * 1e-3) / 1e9
    batch_bytes = 56 if batch_geometry[0] == "fused" else 72
    room_bytes = 56 if best_scheme == "fused" else 72
    per_room_frac = per_room_gcups * room_bytes / peak
    return {
        "cells": cells,
        "batched_gcups": batched_gcups,
        "per_room_gcups": per_room_gcups,
        "per_room_gcups_by_scheme": {k: cells * T / (v * 1e-3) / 1e9 for k, v in per_room.items()},
        "speedup": per_room_ms / batch_ms,
        f"batched_hbm_frac_of_{peak_kind}": batched_gcups * batch_bytes / peak,
        "bytes_per_cell": batch_bytes,
        f"per_room_hbm_frac_of_{peak_kind}": per_room_frac,
        "per_room_scheme": best_scheme,
        "per_room_bytes_per_cell": room_bytes,
        # a batch moves at most the peak, on the fused step's 56 bytes per cell at the least:
        # against the per-room arm no batching can be faster than this
        "batching_ceiling_speedup": (peak / 56) / per_room_gcups,
        "launches_in_setup_and_runs": launches,
        "batch_launch": {"scheme": batch_geometry[0], "block_threads": batch_geometry[1],
                         "planes": batch_geometry[2], "ctas_per_sm": batch_geometry[3],
                         "chosen_by": "ac_fdtd_b200.autotune"},
    }


def adjoint_cost(args) -> dict:
    """Cost of one gradient against one forward run: 128^3 fp32, 3000 steps, L2 misfit of four
    receivers to the signals of the true admittances, from a start perturbed by up to 30 %."""
    import torch

    from ac_fdtd_b200 import AirAbsorption, CudaAcousticFDTD, WallAdmittances, gaussian_pulse
    from ac_fdtd_b200.adjoint import DifferentiableRoom
    from ac_fdtd_b200.autotune import apply_tuned
    from ac_fdtd_b200.workloads import differentiable_room

    T = args.adjoint_steps
    grid, true_xi, start_xi, source, receivers = differentiable_room()
    out = {"workload": f"differentiable room 128^3 fp32, {T} steps, 4 receivers, gradient wrt 6 "
                       f"wall admittances + {T} source samples"}
    for label, air in (("walls_and_signal", None),
                       ("walls_signal_and_air", AirAbsorption(temperature=20.0, relative_humidity=50.0))):
        wrt = ("signal", "walls") if air is None else ("signal", "walls", "air")
        forward = CudaAcousticFDTD(grid, dtype=np.float32, walls=WallAdmittances(*start_xi),
                                   air_absorption=air)
        forward_launch = launch_dict(apply_tuned(forward))     # against the fastest forward
        room = DifferentiableRoom(grid, dtype=np.float32, walls=WallAdmittances(*true_xi),
                                  air_absorption=air, max_steps=T, wrt=wrt)
        signal = gaussian_pulse(T, room.dt, 2000.0)
        for solver in (forward, room.solver):
            solver.add_volume_source(source, signal)
            for point in receivers:
                solver.add_pressure_receiver(point)
        target = room.forward(T).astype(np.float64)
        room.set_parameters(walls=WallAdmittances(*start_xi))

        def run_forward():
            forward.step_index = 0
            forward.run(T)

        def gradient():
            rec = room.forward(T)
            room.backward(rec.astype(np.float64) - target)

        run_forward()
        gradient()
        forward_ms = min(_device_ms(run_forward, torch) for _ in range(3))
        gradient_ms = min(_device_ms(gradient, torch) for _ in range(3))
        out[label] = {"forward_ms": forward_ms, "gradient_ms": gradient_ms,
                      "ratio": gradient_ms / forward_ms,
                      "checkpoint_every": room.checkpoint_every if air is not None else None,
                      "forward_launch": forward_launch}
        forward.close()
        room.solver.close()
    return out


def batched_adjoint_cost(args) -> dict:
    """One gradient of the batched patch inversion: 16 rooms (96-160 cells per axis), 4 x 4
    patches per wall (1536 admittances), air + one sponge face, 8 receivers per room, L2 misfit
    to the signals of the true patches from a start perturbed by up to 30 %."""
    import torch

    from ac_fdtd_b200 import RoomBatch, gaussian_pulse
    from ac_fdtd_b200.adjoint import DifferentiableBatch
    from ac_fdtd_b200.workloads import patch_inversion_rooms

    T = args.inversion_steps
    rooms = patch_inversion_rooms()
    specs = [r[0] for r in rooms]
    cells = int(sum(spec["grid"].n_cells for spec in specs))
    inversion = DifferentiableBatch(specs, dtype=np.float32, max_steps=T)
    forward = RoomBatch([dict(spec, walls=start) for spec, start, _, _ in rooms], dtype=np.float32)
    from ac_fdtd_b200.autotune import apply_tuned_batch

    forward_geometry = apply_tuned_batch(forward)      # the fastest plain forward
    for r, (spec, start, source, receivers) in enumerate(rooms):
        for batch in (inversion.batch, forward):
            batch.add_volume_source(r, source, gaussian_pulse(T, batch.dt(r), 2000.0))
            for point in receivers:
                batch.add_pressure_receiver(r, point)
    targets = [rec.astype(np.float64) for rec in inversion.forward(T)]
    for r, (_, start, _, _) in enumerate(rooms):
        inversion.set_walls(r, start)

    def gradient():
        recordings = inversion.forward(T)
        inversion.backward([rec.astype(np.float64) - tgt for rec, tgt in zip(recordings, targets)])

    def run_forward():
        forward.step_index = 0
        forward.run(T)

    run_forward()
    forward_ms = min(_device_ms(run_forward, torch) for _ in range(2))
    gradient()
    gradient_ms = min(_device_ms(gradient, torch) for _ in range(2))
    inversion.batch.close()
    forward.close()
    return {
        "workload": f"16 rooms 96-160 cells per axis ({cells} cells), fp32, 4x4 patches per wall "
                    f"(1536 admittances), ISO air 20 C, 16-cell sponge on one face, 8 receivers "
                    f"per room, {T} steps; gradient wrt all patches and source samples",
        "forward_ms": forward_ms, "gradient_ms": gradient_ms, "ratio": gradient_ms / forward_ms,
        "gradient_steps_per_s": 1000.0 / gradient_ms,
        "forward_gcups": cells * T / (forward_ms * 1e-3) / 1e9,
        "forward_launch": {"scheme": forward_geometry[0], "block_threads": forward_geometry[1],
                           "planes": forward_geometry[2], "ctas_per_sm": forward_geometry[3]},
    }


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=3)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=["ours", "reference"], default="ours")
    parser.add_argument("--size", type=int, default=384)
    parser.add_argument("--time-steps", type=int, default=4000)
    parser.add_argument("--cpu-budget", type=float, default=12.0)
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--skip-extras", action="store_true",
                        help="skip the batched-room and adjoint-cost measurements")
    parser.add_argument("--batch-steps", type=int, default=3000)
    parser.add_argument("--walls-only", action="store_true",
                        help="the headline room without its sponge and air (for the "
                             "pressure-only scheme, --launch pressure_only,128,8)")
    parser.add_argument("--launch", default="",
                        help="fixed geometry instead of the autotuner: 'two_sweeps|fused,threads,planes' "
                             "or 'staged,rows,stages,planes,vector'")
    parser.add_argument("--adjoint-steps", type=int, default=3000)
    parser.add_argument("--inversion-steps", type=int, default=2500)
    parser.add_argument("--slabs", action="store_true",
                        help="cut the room into one x slab per rank (strong scaling) instead of "
                             "running a replica per rank")
    args = parser.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.slabs:
        run_slab_mode(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
