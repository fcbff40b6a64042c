#!/usr/bin/env python
"""Benchmark of the D3Q27 cumulant time step (MLUPS and HBM-roofline fraction).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME] [--storage f32|f16|bf16]

A "step" is one coarse time step (updateAllGrids) of the whole domain.
One process per GPU (torchrun for N > 1); domains are independent replicas,
so scaling is weak and there is no data-path collective.  Rank 0 prints one
JSON line.  ``--impl reference`` times the reference algorithm's CPU
implementation (the C oracle, all host threads) on the same workload.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

BYTES_PER_POP = {"f32": 4, "f16": 2, "bf16": 2, "f64": 8}
A_STORE = {"f32": 0, "f16": 1, "bf16": 2, "f64": 3}  # LBM_STORE_* of include/lbm3_b200.h


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------- workloads
def make_case(name: str, storage: str):
    import lbm3_b200 as L
    from lbm3_b200 import _abi as A
    st = {"f32": A.LBM_STORE_F32, "f16": A.LBM_STORE_F16, "bf16": A.LBM_STORE_BF16, "f64": A.LBM_STORE_F64}[storage]
    if name.startswith("sphere"):
        # flow around a sphere: single level, icosphere of 20,480 triangles with
        # D = 24 cells at (64, 64, 64) on the 256x128x128 grid (scaled with the
        # grid for other sizes), velocity inlet u = 0.04, non-reflective
        # pressure outlet, strict-velocity sides, nu = 0.0096 (Re 100)
        dims = name[len("sphere"):] or "256x128x128"
        nx, ny, nz = (int(v) for v in dims.split("x"))
        k = nx / 256.0
        s = L.flow_around_sphere(nx, ny, nz, diameter=24.0 * k, center=(64.0 * k, ny / 2.0, nz / 2.0),
                                 storage=st)
        desc = (f"flow around a sphere {nx}x{ny}x{nz} single level: icosphere 20480 triangles, "
                f"D={24.0 * k:g} cells at ({64.0 * k:g},{ny / 2.0:g},{nz / 2.0:g}), IBB, velocity inlet u=0.04, "
                f"non-reflective pressure outlet, strict-velocity sides, nu=0.0096 (Re 100)")
        return s.case, desc, s
    if name.startswith("msphere"):
        # flow around a sphere on three levels: base 128x64x64, refinement
        # boxes of 96x64x64 level-1 and 112x80x80 level-2 cells around the
        # sphere (D = 48 finest cells), Re 300, inlet u = 0.04
        from lbm3_b200.cases import multilevel_sphere
        dims = name[len("msphere"):] or "128x64x64"
        nx, ny, nz = (int(v) for v in dims.split("x"))
        s = multilevel_sphere(nx, ny, nz, storage=st)
        desc = (f"multilevel sphere: 3 levels (ratio 2), base {nx}x{ny}x{nz}, refinement boxes of 96x64x64 "
                f"level-1 and 112x80x80 level-2 cells, icosphere of 20480 triangles with D=48 finest cells, "
                f"wall refinement 2, velocity inlet u=0.04, non-reflective outlet, Re=300")
        return s.case, desc, s
    if name.startswith("xchannel") or name.startswith("yzchannel"):
        # the sphere configuration's channel without the body, with only the x
        # faces open (periodic sides) or only the y/z faces open (periodic x):
        # the open-boundary cost per face kind
        xonly = name.startswith("xchannel")
        dims = name[len("xchannel" if xonly else "yzchannel"):] or "256x128x128"
        nx, ny, nz = (int(v) for v in dims.split("x"))
        c = L.open_channel(nx, ny, nz, u_in=0.04, nu_lattice=0.0096, sides="periodic" if xonly else "velocity",
                           storage=st)
        if not xonly:
            for f in (A.FACE_XMIN, A.FACE_XMAX):
                c.face[f] = A.LbmFaceBC(A.LBM_BC_PERIODIC, 0, 0, 0, 7.0, 0.0, 0.0, 0.0, 0.0)
        desc = (f"channel {nx}x{ny}x{nz} without a body, " +
                ("velocity inlet and non-reflective outlet on x, periodic y and z" if xonly
                 else "periodic x, velocity boundaries on the y and z faces") + ", nu=0.0096")
        return c, desc, None
    if name == "box256x128x128":
        # the 256x128x128 single-level grid of the flow-around-sphere
        # configuration, fully periodic and without the obstacle
        c = L.periodic_box(254, 126, 126, nu_lattice=0.0096, ux=0.04, storage=st)
        desc = ("periodic box 256x128x128 cells incl. ghosts (sphere-config grid, no obstacle, "
                "no open boundaries), nu=0.0096, u=0.04")
        return c, desc, None
    if name == "tgv64":
        s = L.tgv_plain_method(storage=st)
        return s.case, "Taylor-Green vortex 64^3 periodic (66^3 incl. ghosts), u0=0.05, nu=0.01", s
    if name == "tgv128":
        s = L.taylor_green(128, storage=st)
        return s.case, "Taylor-Green vortex Re1600 Ma0.1 128^3 periodic (130^3 incl. ghosts)", s
    raise SystemExit(f"unknown workload {name}")


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples every 100 ms while the timed region runs; only the
    samples taken inside the [start, stop] window are summarised."""
    FIELDS = ("timestamp,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.file = None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.file, stderr=subprocess.DEVNULL)
            # wait for the first sample so the window is covered from its start
            deadline = time.time() + 5.0
            while time.time() < deadline and os.path.getsize(self.file.name) == 0:
                time.sleep(0.05)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def start(self):
        self.t0 = datetime.datetime.now()

    def stop(self):
        self.t1 = datetime.datetime.now()
        time.sleep(0.25)  # let the sampler flush one more line

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.file is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.file.flush()
        rows = [[c.strip() for c in l.split(",")] for l in Path(self.file.name).read_text().splitlines()
                if l.strip()]
        os.unlink(self.file.name)
        if self.uuid:
            rows = [r for r in rows if len(r) > 1 and r[1] == self.uuid] or rows
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lo = self.t0 - datetime.timedelta(milliseconds=100) if self.t0 else None
        hi = self.t1 + datetime.timedelta(milliseconds=100) if self.t1 else None
        for r in rows:
            try:
                ts = datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f")
                if lo and hi and not (lo <= ts <= hi):
                    continue
                sm.append(float(r[2]))
                smax = float(r[3])
                power.append(float(r[4]))
            except (ValueError, IndexError):
                continue
            for nme, v in zip(names, r[6:10]):
                if v.lower() == "active":
                    reasons.add(nme)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "power_w_median": statistics.median(power) if power else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------- CPU legs
def oracle_grid(case):
    """The oracle on the workload, every table built by the oracle itself
    (its own restatement of the reference's setup chain)."""
    import oracle as O
    return O.OracleGrid(case)


def time_oracle(case, target_s: float, min_steps: int = 1, max_steps: int | None = None):
    """Time whole oracle time steps (collide-stream, open boundary, periodic
    copy: updateSingleGrid) on the host cores: returns (MLUPS, steps,
    seconds, threads)."""
    g = oracle_grid(case)
    import oracle as O
    cells = g.g.fluidUpdates
    g.step(1)  # warm the pages
    steps, t0 = 0, time.perf_counter()
    while True:
        g.step(1)
        steps += 1
        el = time.perf_counter() - t0
        if steps >= min_steps and (el >= target_s or (max_steps is not None and steps >= max_steps)):
            break
    g.close()
    return cells * steps / el / 1e6, steps, el, O.threads()


def workload_config(desc: str, cells: int, updates: int, storage: str, world: int) -> dict:
    """The `config` object both arms print for a workload."""
    bpp = BYTES_PER_POP[storage]
    pop_bytes = updates * 27 * bpp
    return {"workload": desc, "cells": cells, "fluid_updates_per_step": updates, "storage": storage,
            "compute": "f32",
            "l2": "inputs larger than L2 (populations %.0f MB > 126 MB)" % (pop_bytes / 1e6)
            if pop_bytes > 126e6 else "inputs smaller than L2",
            "parallelism": f"replicas x{world}"}


def run_reference(args):
    """CPU implementation of the reference algorithm (the C oracle on all host
    threads, tables built by the oracle itself) on the same workload.  Every
    timed step is one whole time step; the number of timed steps is capped so
    the run stays within --ref-seconds."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    world = int(os.environ.get("WORLD_SIZE", "1"))
    case, desc, _ = make_case(args.workload, args.storage)
    import oracle as O
    g = oracle_grid(case)
    n, updates = g.cell_count, int(g.g.fluidUpdates)
    # warm-up steps, then an estimate of the step time
    t0 = time.perf_counter()
    g.step(1)
    est = max(time.perf_counter() - t0, 1e-6)
    for _ in range(max(0, min(args.warmup, 3) - 1)):
        g.step(1)
    timed = int(max(1, min(args.steps, args.ref_seconds / est)))
    t0 = time.perf_counter()
    g.step(timed)
    el = time.perf_counter() - t0
    g.close()
    mlups = updates * timed / el / 1e6
    line = {
        "impl": "reference", "metric": "MLUPS", "value": round(mlups, 3), "unit": "MLUPS",
        "n_gpus": args.gpus, "steps": timed, "warmup": args.warmup,
        "ms_per_step": round(1e3 * el / timed, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(desc, n, updates, args.storage, world),
        "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS", "cores": O.threads(), "kind": "port",
                         "sample": f"{timed} whole time steps (collide-stream + open boundary + periodic copy) "
                                   f"of the {n}-cell grid of {args.steps} requested, capped at "
                                   f"{args.ref_seconds:g} s: C restatement of the reference time step on "
                                   f"oracle-built tables, OpenMP, {O.threads()} threads, FP32 populations"},
        "e2e": {"value": round(mlups, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- ranks
def max_over_ranks(value: float, dist, device: str) -> float:
    """The largest `value` over all ranks (the slowest rank sets the job
    time); `dist` is torch.distributed or None for a single process."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(updates_per_step: int, steps: int, world: int, seconds: float) -> float:
    """MLUPS of the whole job: every rank advances its own replica of the
    workload, all ranks are done after `seconds`."""
    return updates_per_step * steps * world / seconds / 1e6


# ---------------------------------------------------------------- GPU leg
def run_ours(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    import lbm3_b200 as L
    case, desc, tgv = make_case(args.workload, args.storage)
    stream = torch.cuda.Stream()
    g = L.build_grids(case)
    g.set_stream(stream.cuda_stream)
    info = g.info()
    updates = g.fluid_updates_per_iteration
    with torch.cuda.stream(stream):
        g.update_all_grids(args.warmup)
    g.synchronize()

    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
        uuid = "GPU-" + uuid if not uuid.startswith("GPU-") else uuid
    except Exception:
        pass

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(uuid) as clk:
        clk.start()
        # the step schedule replayed as CUDA graphs, CUDA events on the grid stream
        ms = g.time_steps_graph(args.steps)
        clk.stop()
    torch.cuda.synchronize()
    # collide-stream kernel time: a pass of direct launches, each bracketed by events
    kt_steps = max(2, min(args.steps, 400))
    g.time_steps(kt_steps)
    kernel_ms, launches = g.last_kernel_time()
    all_launches = int(round(g.last_launch_count() / kt_steps * args.steps))
    if dist:
        dist.barrier()
    ms_max = max_over_ranks(ms, dist, "cuda")
    value = whole_job_rate(updates, args.steps, world, ms_max * 1e-3)

    # roofline of the dominant kernel (collide-stream): algorithmic bytes =
    # 2 x 27 populations per fluid cell update at the storage width, summed
    # over the collide launches of a coarse step (one per level substep)
    bpp = BYTES_PER_POP[args.storage]
    alg_bytes = updates * 2 * 27 * bpp
    per_launch_ms = kernel_ms / max(launches, 1)
    per_step_kernel_ms = kernel_ms / kt_steps
    achieved = alg_bytes / (per_step_kernel_ms * 1e-3) / 1e9
    peak, peak_kind = peaks()
    traffic = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        tr = json.loads(tfile.read_text()).get(f"{args.workload}:{args.storage}")
        if tr:
            traffic = int(tr)  # bytes per launch, like algorithmic_bytes_per_launch

    # end to end through the public API: upload the initial state from pinned
    # host memory, then run steps that each read the step's observable back
    e2e_steps = max(10, min(args.steps // 10, 200))
    levels = g.level_count()
    pinned = [torch.from_numpy(g.populations(l)).pin_memory() for l in range(levels)]
    import numpy as np
    f_np = [t.numpy() for t in pinned]
    upload_bytes = sum(a.nbytes for a in f_np)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for l in range(levels):
        g.set_populations(f_np[l], l)
    sphere = tgv is not None and (hasattr(tgv, "drag_coefficient") or hasattr(tgv, "diameter_finest"))
    for _ in range(e2e_steps):
        g.update_all_grids(1)
        if sphere:
            g.wall_force(0)                    # drag and torque, 6 doubles
        elif tgv is not None:
            g.kinetic_energy(tgv.u_initial_phys, tgv.domain_length)
        else:
            g.kinetic_energy(1.0, 1000.0)
    g.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_value = whole_job_rate(updates, e2e_steps, world, max_over_ranks(e2e_s, dist, "cuda"))
    del np

    extras = storage_comparison(args, value, torch) if (rank == 0 and world == 1 and not args.no_extras) else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        mlups, steps, el, thr = time_oracle(case, target_s=args.cpu_seconds)
        cpu = {"value": round(mlups, 3), "unit": "MLUPS", "cores": thr, "kind": "port",
               "sample": f"{steps} full steps of the same workload ({el:.1f} s, FP32) by the C restatement "
                         f"of the reference time step on the host cores (OpenMP)"}

    clocks = clk.summary()
    g.close()
    if rank == 0:
        line = {
            "metric": "MLUPS", "value": round(value, 2), "unit": "MLUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": args.storage if args.storage != "f32" else "f32", "data": "synthetic",
            "config": workload_config(desc, info.cell_count, updates, args.storage, world),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_kind})",
                         "kernel": {"pair": "collidePair", "packed": "collidePacked", "prefetch": "collidePrefetch",
                                    "tma": "collideBulkTma", "simple": "collideStream"}.get(
                             os.environ.get("LBM3_COLLIDE_KERNEL", "pair") or "pair", "collidePair")
                         + " (bulk segments + wall-adjacent cells, one persistent launch)",
                         "kernel_ms_per_launch": round(per_launch_ms, 5),
                         "collide_launches_per_step": round(launches / kt_steps, 3),
                         "algorithmic_bytes_per_launch": int(alg_bytes * kt_steps / max(launches, 1)),
                         "traffic_unit": "bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)"},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_value, 2), "unit": "MLUPS",
                    "h2d_bytes_per_step": int(upload_bytes // e2e_steps), "d2h_bytes_per_step": 48 if sphere else 8,
                    "steps": e2e_steps,
                    "note": "initial populations uploaded from pinned host memory inside the timed "
                            "region; every step reads its tracked observable back (tracker period 1: "
                            + ("wall force and torque" if sphere else "kinetic energy") + ")"},
            "gpu_launches": all_launches,
            "clocks": clocks,
        }
        if extras:
            line.update(extras)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def time_batch(cases, steps: int, warmup: int, torch) -> float:
    """MLUPS of independent domains advanced together by update_batch, one
    stream each, device-timed from a start event all streams wait on to an
    end event that waits on all of them."""
    import lbm3_b200 as L
    grids = [L.build_grids(c) for c in cases]
    streams = [torch.cuda.Stream() for _ in grids]
    for g, s in zip(grids, streams):
        g.set_stream(s.cuda_stream)
    L.update_batch(grids, warmup)
    torch.cuda.synchronize()
    main = torch.cuda.current_stream()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(main)
    for s in streams:
        s.wait_event(start)
    L.update_batch(grids, steps)
    for s in streams:
        ev = torch.cuda.Event()
        ev.record(s)
        main.wait_event(ev)
    end.record(main)
    end.synchronize()
    ms = start.elapsed_time(end)
    updates = sum(g.fluid_updates_per_iteration for g in grids)
    for g in grids:
        g.close()
    return updates * steps / (ms * 1e-3) / 1e6


def time_packed(cases, steps: int, warmup: int) -> tuple:
    """MLUPS of independent single-level domains advanced as one packed batch
    (one persistent collide-stream launch over the packed block table of all
    of them, one open-boundary and one periodic launch per step, step pairs
    replayed as a CUDA graph), device-timed on the batch stream; and the
    batch's kernel launches per step."""
    import lbm3_b200 as L
    grids = [L.build_grids(c) for c in cases]
    with L.PackedBatch(grids) as b:
        b.update(warmup + (warmup & 1))
        ms = b.time_steps(steps)
        launches = b.info().launches_per_step
    updates = sum(g.fluid_updates_per_iteration for g in grids)
    for g in grids:
        g.close()
    return updates * steps / (ms * 1e-3) / 1e6, launches


def storage_comparison(args, f32_value: float, torch) -> dict:
    """The metric's comparison: the same workload with FP16-shifted storage,
    and the FP16-shifted batched form (8 Taylor-Green 64^3 domains, the plain
    method's configuration, one stream each) against the plain FP32 kernel
    on one domain of that configuration and on this workload."""
    import lbm3_b200 as L
    out = {}
    if args.storage == "f32":
        c16, _, _ = make_case(args.workload, "f16")
        g = L.build_grids(c16)
        s = torch.cuda.Stream()
        g.set_stream(s.cuda_stream)
        g.update_all_grids(args.warmup)
        steps = max(2, min(args.steps, 2000))
        ms = g.time_steps_graph(steps)
        v16 = g.fluid_updates_per_iteration * steps / (ms * 1e-3) / 1e6
        g.close()
        out["storage_f16"] = {"value": round(v16, 2), "unit": "MLUPS", "ratio_vs_f32": round(v16 / f32_value, 4),
                              "workload": "same workload, FP16-shifted populations, FP32 arithmetic"}
    # the multilevel configuration: three levels, substep schedule replayed as graphs
    cm, dm, _ = make_case("msphere128x64x64", args.storage)
    g = L.build_grids(cm)
    s = torch.cuda.Stream()
    g.set_stream(s.cuda_stream)
    g.update_all_grids(args.warmup)
    steps = max(2, min(args.steps, 1000))
    ms = g.time_steps_graph(steps)
    vm = g.fluid_updates_per_iteration * steps / (ms * 1e-3) / 1e6
    g.time_steps(min(steps, 200))
    kms, klaunch = g.last_kernel_time()
    out["multilevel_sphere"] = {
        "value": round(vm, 2), "unit": "MLUPS", "ms_per_coarse_step": round(ms / steps, 5),
        "fluid_updates_per_coarse_step": g.fluid_updates_per_iteration,
        "cells_per_level": [g.info(l).cell_count for l in range(g.level_count())],
        "collide_share_of_step": round(kms / min(steps, 200) / (ms / steps), 4),
        "workload": dm + "; MLUPS counts level-L updates 2^L times per coarse step"}
    g.close()
    tgv32 = L.tgv_plain_method().case
    g = L.build_grids(tgv32)
    s = torch.cuda.Stream()
    g.set_stream(s.cuda_stream)
    g.update_all_grids(args.warmup)
    ms = g.time_steps_graph(1000)
    plain = g.fluid_updates_per_iteration * 1000 / (ms * 1e-3) / 1e6
    g.close()
    tgv16 = [L.tgv_plain_method(storage=A_STORE["f16"]).case for _ in range(8)]
    batched, launches = time_packed(tgv16, 500, args.warmup)
    streams = time_batch(tgv16, 500, args.warmup, torch)
    out["batched_f16"] = {
        "value": round(batched, 2), "unit": "MLUPS",
        "workload": "8 Taylor-Green 64^3 domains (66^3 with ghosts), FP16-shifted, one packed batch: one "
                    "persistent collide-stream launch over all domains' work items and one periodic-ghost "
                    "launch per step, step pairs replayed as CUDA graphs",
        "launches_per_step": launches,
        "plain_f32_single_domain": round(plain, 2),
        "ratio_vs_plain_f32_same_configuration": round(batched / plain, 4),
        "ratio_vs_plain_f32_this_workload": round(batched / f32_value, 4),
        "one_stream_per_domain": round(streams, 2)}
    return out


def run_batch(args, copies: int, base: str):
    """Many-domain batch: `copies` independent domains of workload `base`.
    Single-level domains without rotors advance as one packed batch (one
    persistent collide-stream launch over all domains' work items per step,
    graph replay), device-timed on the batch stream; otherwise each domain
    runs on its own stream, advanced together by update_batch, timed from a
    start event every domain stream waits on to an end event that waits on
    all of them."""
    import torch
    import lbm3_b200 as L
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        raise SystemExit("batch workloads run on one GPU")
    torch.cuda.set_device(0)
    made = [make_case(base, args.storage) for _ in range(copies)]
    desc = made[0][1]
    grids = [L.build_grids(c) for c, _, _ in made]
    streams = [torch.cuda.Stream() for _ in grids]
    for g, s in zip(grids, streams):
        g.set_stream(s.cuda_stream)
    packed = None
    if args.storage != "f64" and all(g.level_count() == 1 and g.case.rotor_count == 0 for g in grids):
        packed = L.PackedBatch(grids)
    per_step_launches = 0
    if packed is not None:
        per_step_launches = packed.info().launches_per_step
    else:
        for g in grids:
            g.time_steps(1)
            per_step_launches += g.last_launch_count()
    advance = packed.update if packed is not None else (lambda n: L.update_batch(grids, n))
    advance(args.warmup + (args.warmup & 1))
    torch.cuda.synchronize()
    updates = sum(g.fluid_updates_per_iteration for g in grids)
    main_stream = torch.cuda.current_stream()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(0).uuid)
        uuid = "GPU-" + uuid if not uuid.startswith("GPU-") else uuid
    except Exception:
        pass
    with ClockSampler(uuid) as clk:
        clk.start()
        if packed is not None:
            ms = packed.time_steps(args.steps)
        else:
            start.record(main_stream)
            for s in streams:
                s.wait_event(start)
            L.update_batch(grids, args.steps)
            for s in streams:
                ev = torch.cuda.Event()
                ev.record(s)
                main_stream.wait_event(ev)
            end.record(main_stream)
            end.synchronize()
            ms = start.elapsed_time(end)
        clk.stop()
    value = whole_job_rate(updates, args.steps, 1, ms * 1e-3)
    bpp = BYTES_PER_POP[args.storage]
    alg_bytes = updates * 2 * 27 * bpp
    achieved = alg_bytes / (ms / args.steps * 1e-3) / 1e9
    peak, peak_kind = peaks()
    # end to end: upload every domain's state from pinned memory, then steps that
    # each read every domain's kinetic energy back
    import numpy as np
    e2e_steps = max(10, min(args.steps // 10, 200))
    states = [torch.from_numpy(g.populations()).pin_memory().numpy() for g in grids]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for g, f0 in zip(grids, states):
        g.set_populations(f0)
    for _ in range(e2e_steps):
        advance(1)
        for g, (_, _, tg) in zip(grids, made):
            g.kinetic_energy(tg.u_initial_phys, tg.domain_length) if tg is not None else g.kinetic_energy(1.0, 1000.0)
    e2e_s = time.perf_counter() - t0
    clocks = clk.summary()
    h2d = sum(f.nbytes for f in states)
    if packed is not None:
        packed.close()
    for g in grids:
        g.close()
    del np
    line = {
        "metric": "MLUPS", "value": round(value, 2), "unit": "MLUPS", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.storage, "data": "synthetic",
        "config": {"workload": f"batch of {copies} independent domains, each: {desc}", "domains": copies,
                   "fluid_updates_per_step": updates, "storage": args.storage, "compute": "f32",
                   "l2": "all domains' populations %.0f MB" % (alg_bytes / 2 / 1e6),
                   "parallelism": "packed batch" if packed is not None else "one stream per domain"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None,
                     "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_kind})",
                     "kernel": "whole batch step (all kernels of all domains)",
                     "algorithmic_bytes_per_step": alg_bytes},
        "cpu_baseline": None,
        "e2e": {"value": round(whole_job_rate(updates, e2e_steps, 1, e2e_s), 2), "unit": "MLUPS",
                "h2d_bytes_per_step": int(h2d // e2e_steps), "d2h_bytes_per_step": 8 * copies, "steps": e2e_steps},
        "gpu_launches": per_step_launches * args.steps,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_serving(args):
    """Serving stream of the serving configuration: seeded requests (2e x e x e
    channels, e from {32, 48, 64, 96, 128}, ellipsoid or icosphere obstacle,
    Re 20-200, 2,000-10,000 steps, FP16 storage) with Poisson arrivals at 80%
    of the capacity the serving loop itself delivers (admission, builds and
    stepping, measured on a saturated calibration stream), served by the
    continuous-batching loop; value = aggregate MLUPS, plus p50/p99
    time-to-result.  The request count is bounded by --requests."""
    import numpy as np
    import torch
    from lbm3_b200 import serving as S
    torch.cuda.set_device(0)
    edges_all = [32, 48, 64, 96, 128]

    def stream(seed: int, count: int):
        rng = np.random.default_rng(seed)
        edges = rng.choice(edges_all, size=count)
        steps = rng.integers(2000, 10001, size=count)
        reqs = [S.channel_request(q, int(e), rng, int(n)) for q, (e, n) in enumerate(zip(edges, steps))]
        # submission: each request is planned once; footprint and work travel with it
        for r in reqs:
            p = L.Plan(r.case)
            r.footprint = int(p.info().grid_memory_bytes)
            r.updates = int(p.fluid_updates_per_iteration)
            p.close()
        return reqs

    import lbm3_b200 as L
    budget = int(args.hbm_budget_gb * (1 << 30))
    # capacity of the serving loop: a saturated stream (everything arrives at 0)
    cal = stream(54321, args.calibration_requests)
    t0 = time.perf_counter()
    cal_res = S.Server(hbm_budget=budget, max_slots=16, chunk_steps=100).run(cal)
    cal_wall = time.perf_counter() - t0
    cap = S.summarize(cal_res, cal_wall)["mlups"]
    reqs = stream(12345, args.requests)
    work = [r.updates * int(r.steps) / 1e6 for r in reqs]
    load = 0.8
    rate = load * cap / float(np.mean(work))          # requests per second
    rng = np.random.default_rng(777)
    t = 0.0
    for r in reqs:
        t += float(rng.exponential(1.0 / rate))
        r.arrival = t
    server = S.Server(hbm_budget=budget, max_slots=16, chunk_steps=100)
    t0 = time.perf_counter()
    results = server.run(reqs)
    wall = time.perf_counter() - t0
    summ = S.summarize(results, wall)
    offered = sum(work) / reqs[-1].arrival if reqs[-1].arrival > 0 else None
    line = {
        "metric": "MLUPS", "value": round(summ["mlups"], 2), "unit": "MLUPS", "n_gpus": 1,
        "steps": int(sum(int(r.steps) for r in reqs)), "warmup": 0, "ms_per_step": None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f16", "data": "synthetic",
        "config": {"workload": f"serving stream of {len(reqs)} requests: 2e x e x e channels, e in {edges_all}, "
                               "ellipsoid/icosphere obstacle, Re 20-200, 2000-10000 steps, FP16 storage, Poisson "
                               "arrivals at 80% of the serving loop's measured capacity",
                   "requests": len(reqs), "hbm_budget_gb": args.hbm_budget_gb,
                   "capacity_mlups": round(cap, 1), "capacity_sample": f"{len(cal)} requests arriving at once, "
                   f"{cal_wall:.1f} s", "offered_load_fraction": load,
                   "arrival_rate_per_s": round(rate, 4),
                   "offered_mlups": round(offered, 1) if offered else None,
                   "parallelism": "continuous batching: the resident domains of each storage type advance as one "
                                  "packed batch (one persistent collide-stream launch per step), rebuilt as "
                                  "requests join and leave; grids built on 2 host threads"},
        "serving": {"requests": summ["requests"], "p50_s": round(summ["p50_s"], 4), "p99_s": round(summ["p99_s"], 4),
                    "wall_s": round(wall, 3)},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="sphere256x128x128",
                    help="sphere256x128x128 (default; sphereNXxNYxNZ scales it), box256x128x128, tgv64, tgv128, "
                         "batchK_<workload> (K domains on K streams), serving (continuous-batching request stream)")
    ap.add_argument("--storage", choices=["f32", "f16", "bf16", "f64"], default="f32")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-seconds", type=float, default=90.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the FP16 and batched comparisons")
    ap.add_argument("--requests", type=int, default=48, help="serving: requests in the measured stream")
    ap.add_argument("--calibration-requests", type=int, default=12, help="serving: saturated capacity sample")
    ap.add_argument("--hbm-budget-gb", type=float, default=120.0, help="serving: device memory for resident domains")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload.startswith("batch"):
        copies, base = args.workload[len("batch"):].split("_", 1)
        return run_batch(args, int(copies), base)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
