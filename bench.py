"""Benchmark of the B200 ideal-MHD step: zone-updates/s of the 3D decaying-turbulence box.

Workload (one GPU): 3D decaying turbulence on a periodic 256^3 grid, MC-limited PLM +
HLLD + CT-contact vector-potential constrained transport, SSP-RK2 at CFL 0.3, float32
state (pressure recovery in float64); seeded Gaussian random velocity and potential
fields with a k^-2 spectrum on 1 <= |k| <= 8, rms Mach 1, rms |B| = 1. One zone-update is
one cell advanced by one full RK2 step; a bench step is one RK2 step of the whole box.
With N GPUs (torchrun) every rank advances its own box (replicas, seeded by rank: weak
scaling, no data-path collective); `value` is the zone-updates of all ranks over the
slowest rank's time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--cells 256] [--impl reference]

`--impl reference` times the CPU implementation of the same step (the NumPy
restatement of the reference's MHD3D step, the reference being pure Python) on all
host cores, each process a bounded 32^3 sample of the workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "zone-updates/s on 1 B200 (batched FP32 vs plain FP64) at stated L1 err; % HBM roofline"
UNIT = "zone-updates/s"
BYTES_PER_ZONE_UPDATE = 5 * 8 * 4  # 5 state passes x 8 values (5 cell + 3 edge) x float32
WORKLOAD = ("3D decaying turbulence, periodic {n}^3, MC-PLM + HLLD + CT, SSP-RK2, CFL 0.3, "
            "float32 state (float64 pressure recovery), k^-2 seeded fields, Mach 1, |B|_rms 1")


def parse():
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=100)
    parser.add_argument("--warmup", type=int, default=5)
    parser.add_argument("--cells", type=int, default=256)
    parser.add_argument("--impl", default="ours", choices=["ours", "reference"])
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--no-e2e", action="store_true")
    parser.add_argument("--no-accuracy", action="store_true")
    parser.add_argument("--lx", type=int, default=32)
    parser.add_argument("--no-plain", action="store_true")
    return parser.parse_args()


# ---- CPU side ---------------------------------------------------------------------------------
def _cpu_sample(args):
    """One process's bounded sample: the oracle MHD3D step on a small turbulence box."""
    n, steps, seed = args
    from oracle.mesh import Hierarchy
    from oracle.mhd3d import MHD3D
    from wellbalanced_b200.problems import turbulence_3d

    rho, velocity, p, potential = turbulence_3d(n, seed=seed)
    model = MHD3D(Hierarchy((n,) * 3, ((0.0, 1.0),) * 3, (True,) * 3), limiter="mc", cfl=0.3)
    model.set_state(rho, velocity, p, vector_potential=potential)
    model.step()  # warm-up
    start = time.perf_counter()
    for _ in range(steps):
        model.step()
    return n**3 * steps, time.perf_counter() - start


def cpu_baseline(n=64, steps=3):
    """The oracle's NumPy 3D step on one core (zone-updates/s)."""
    cells, seconds = _cpu_sample((n, steps, 0))
    return {
        "value": cells / seconds,
        "unit": UNIT,
        "cores": 1,
        "kind": "port",
        "sample": f"NumPy restatement of the reference MHD3D step, 3D turbulence {n}^3, {steps} RK2 steps after 1 warm-up, 1 process",
    }


def reference_arm(args):
    import multiprocessing as mp

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    n = 32
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        pool.map(_cpu_sample, [(n, 0, s) for s in range(cores)])  # spin up, import
        per_step = []
        for step in range(args.warmup + args.steps):
            start = time.perf_counter()
            results = pool.map(_cpu_sample, [(n, 1, s) for s in range(cores)])
            wall = time.perf_counter() - start
            if step >= args.warmup:
                per_step.append((sum(c for c, _ in results), wall))
    total_cells = sum(c for c, _ in per_step)
    total_time = sum(t for _, t in per_step)
    value = total_cells / total_time
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * total_time / len(per_step),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD.format(n=args.cells) + f"; CPU sample {n}^3 per process"},
        "cpu_baseline": {
            "value": value,
            "unit": UNIT,
            "cores": cores,
            "kind": "port",
            "sample": f"{cores} processes, each one RK2 step of a {n}^3 box of the workload per bench step "
                      "(NumPy restatement of the reference MHD3D step; the reference is pure Python)",
        },
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- GPU side ---------------------------------------------------------------------------------
class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = [r.split(",") for r in out.strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, flag in zip(names, r[5:9], strict=True):
                if flag.strip().lower() == "active":
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": float(rows[0][2]) if rows[0][2].strip().replace(".", "").isdigit() else None,
            "reasons": sorted(reasons),
            "samples": len(rows),
        }


def peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per stage launch from the committed ncu summary, if present."""
    path = ROOT / "profiles" / "stage3d_turbulence.md"
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_launch_256:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    baseline = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        baseline = cpu_baseline()  # before any GPU work

    import numpy as np
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    from wellbalanced_b200.mhd3d import MHD3D

    n = args.cells
    model = MHD3D.turbulence(n, seed=rank, precision=32, lx=args.lx)
    eng = model.engine
    model.advance(args.warmup)
    torch.cuda.synchronize()

    # timed region: K RK2 steps, state resident in HBM
    eng.stage_events = []
    launches0 = eng.launches
    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    model.advance(args.steps, check=False)
    end.record()
    torch.cuda.synchronize()
    barrier()
    clock_info = clocks.stop()
    launches = eng.launches - launches0
    seconds = start.elapsed_time(end) / 1e3
    stage_ms = [s.elapsed_time(e) for s, e in eng.stage_events]
    eng.stage_events = None
    if int(eng.bad.item()):
        raise FloatingPointError("bad cells during the benchmark")
    t = torch.tensor([seconds], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    seconds = float(t.item())
    cells = n**3
    value = world * cells * args.steps / seconds

    # end to end through the public API with host buffers: per step, the state pool is
    # copied from pinned host memory, advanced one step and copied back
    e2e = None
    if not args.no_e2e:
        host = model.save()
        torch.cuda.synchronize()
        e2e_steps = max(3, min(args.steps, 20))
        barrier()
        torch.cuda.synchronize()
        s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s2.record()
        for _ in range(e2e_steps):
            model.load(host)
            model.advance(1, check=False)
            model.save(host)
        e2.record()
        torch.cuda.synchronize()
        barrier()
        t2 = torch.tensor([s2.elapsed_time(e2) / 1e3], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t2, op=dist.ReduceOp.MAX)
        nbytes = host.numel() * host.element_size()
        e2e = {
            "value": world * cells * e2e_steps / float(t2.item()),
            "unit": UNIT,
            "h2d_bytes_per_step": int(nbytes),
            "d2h_bytes_per_step": int(nbytes),
            "path": "MHD3D.load(pinned host pool) + MHD3D.advance(1) + MHD3D.save(pinned host pool)",
        }

    # the plain float64 GPU step (the reference's dataflow, kernel by kernel) on the same box
    plain = None
    if rank == 0 and not args.no_plain:
        plain = plain_step(n, rank, cells)

    # accuracy of the float32 step against the float64 device step from the same state
    accuracy = None
    if rank == 0 and not args.no_accuracy:
        accuracy = accuracy_check(n, rank)

    if rank == 0:
        peak, peak_kind = peaks()
        launch_s = statistics.mean(stage_ms) / 1e3 if stage_ms else float("nan")
        achieved = BYTES_PER_ZONE_UPDATE / 2 * cells / launch_s / 1e9
        traffic = profile_traffic()
        if traffic is not None:
            traffic *= cells / 256**3  # the summary's figure is per launch at 256^3
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": 1e3 * seconds / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {
                "workload": WORKLOAD.format(n=n),
                "cells_per_gpu": cells,
                "parallelism": f"replicas x{world}",
                "l2": "inputs larger than L2 (state pool {:.2f} GB per copy)".format(
                    eng.state.numel() * eng.state.element_size() / 1e9),
                "tile": {"y": eng.layout.tile_shape[0], "z": eng.layout.tile_shape[1], "x_planes": args.lx},
            },
            "roofline": {
                "bound": "hbm",
                "achieved": achieved,
                "peak": peak,
                "unit": "GB/s",
                "frac": achieved / peak,
                "traffic": traffic,
                "kernel": "wb::stage3d_kernel<float, 2>",
                "algorithmic_bytes_per_launch": BYTES_PER_ZONE_UPDATE / 2 * cells,
                "mean_launch_ms": 1e3 * launch_s,
                "peak_kind": peak_kind,
            },
            "gpu_launches": launches,
            "clocks": clock_info,
        }
        if baseline is not None:
            line["cpu_baseline"] = baseline
        if e2e is not None:
            line["e2e"] = e2e
        if accuracy is not None:
            line["accuracy"] = accuracy
        if plain is not None:
            line["plain_fp64"] = plain
            line["plain_fp64"]["speedup_of_value"] = value / world / plain["value"]
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def plain_step(n, seed, cells, steps=3):
    """zone-updates/s of the plain float64 GPU step (`wellbalanced_b200.plain.PlainMHD3D`)."""
    import torch

    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.plain import PlainMHD3D
    from wellbalanced_b200.problems import turbulence_3d

    rho, velocity, p, potential = turbulence_3d(n, seed=seed)
    model = PlainMHD3D(AMRHierarchy((n,) * 3, ((0.0, 1.0),) * 3, periodic=(True,) * 3), limiter="mc", cfl=0.3)
    model.set_state(rho, velocity, p, vector_potential=potential)
    model.step()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(steps):
        model.step()
    end.record()
    torch.cuda.synchronize()
    seconds = start.elapsed_time(end) / 1e3
    del model
    torch.cuda.empty_cache()
    return {"value": cells * steps / seconds, "unit": UNIT, "ms_per_step": 1e3 * seconds / steps, "steps": steps,
            "what": "PlainMHD3D: the reference MHD3D dataflow on the device, float64, per-kernel, intermediates in HBM"}


def accuracy_check(n, seed, steps=10):
    """Relative L1 errors of float32 against float64 device steps from the same state."""
    import numpy as np
    import torch

    from wellbalanced_b200.mhd3d import MHD3D

    ref = MHD3D.turbulence(n, seed=seed, precision=64)
    low = MHD3D.turbulence(n, seed=seed, precision=32)
    for _ in range(steps):
        dt = ref.step()
        low.step(dt)
    torch.cuda.synchronize()
    out = {"steps": steps, "against": "float64 device step from the same state (float64 step == reference to 1e-12 in the tests)"}
    for key, f in (("density", 0), ("energy", 4)):
        (patch,) = ref.hierarchy.patches
        a = ref._read(patch, f).to(torch.float64)
        b = low._read(patch, f).to(torch.float64)
        out[f"rel_l1_{key}"] = float(torch.sum(torch.abs(b - a)) / torch.sum(torch.abs(a)))
    out["div_b"] = low.divergence()
    del ref, low
    torch.cuda.empty_cache()
    return out


if __name__ == "__main__":
    main()
