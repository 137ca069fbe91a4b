"""Benchmark of the B200 ideal-MHD step: zone-updates/s.

Workloads (``--workload``; one zone-update = one cell advanced by one full RK2 step):

* ``turbulence`` (default): 3D decaying turbulence on a periodic 256^3 grid,
  MC-limited PLM + HLLD + CT-contact vector-potential constrained transport, SSP-RK2 at
  CFL 0.3, float32 state (pressure recovery in float64); seeded Gaussian random velocity
  and potential fields with a k^-2 spectrum on 1 <= |k| <= 8, rms Mach 1, rms |B| = 1.
* ``batch``: 4096 independent periodic 2D Orszag-Tang problems (sides drawn from
  {32, 48, ..., 256}, field and velocity amplitudes scaled by seeded factors in
  [0.5, 1.5]), each at its own CFL 0.4 step, float32; all instances advanced by one launch
  per kernel (the timed steps launch directly; the same steps replayed from a CUDA graph
  are reported beside them).
* ``harris``: a 2D Harris current sheet on [-1, 1] x [-2, 2], base 128 x 256, periodic in
  x and outflow in y, refined three times on the current (|J| dx > 1e-7, boxes of 16-24
  fine cells a side where the tags allow: ~1600 uneven patches, 5.6e5 cells), float32 with
  float64 refluxing; every level advances at the finest CFL 0.4 step, all patches in one
  launch per kernel.

With N GPUs (torchrun) every rank advances its own copy of the workload (replicas,
seeded by rank: weak scaling, no data-path collective); `value` is the zone-updates of
all ranks over the slowest rank's time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload turbulence|batch|harris]

`--impl reference` times the CPU implementation of the same step (the NumPy restatement
of the reference's step, the reference being pure Python) on all host cores, each process
a bounded sample of the workload per bench step.
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


def parse():
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=100)
    parser.add_argument("--warmup", type=int, default=5)
    parser.add_argument("--workload", default="turbulence", choices=["turbulence", "batch", "harris"])
    parser.add_argument("--cells", type=int, default=256, help="turbulence: cells per side")
    parser.add_argument("--count", type=int, default=4096, help="batch: number of instances")
    parser.add_argument("--impl", default="ours", choices=["ours", "reference"])
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--no-e2e", action="store_true")
    parser.add_argument("--no-accuracy", action="store_true")
    parser.add_argument("--no-plain", action="store_true")
    parser.add_argument("--partition", action="store_true",
                        help="turbulence on N GPUs as ONE box of N slabs of --cells^3 (patches per rank, "
                             "halo exchange over NCCL, a global dt) instead of N replicas")
    parser.add_argument("--no-extra", action="store_true",
                        help="turbulence at one GPU: skip the batch and Harris configurations measured beside it")
    parser.add_argument("--lx", default="auto", help="turbulence: x-planes per tile (an integer, or auto: tuned)")
    parser.add_argument("--tile3d", default=None,
                        help="turbulence with an integer --lx: the stage kernel's TYxTZ tile shape (default 16x16)")
    return parser.parse_args()


# ---- workloads ---------------------------------------------------------------------------------
HARRIS_BASE = (128, 256)
HARRIS_BOUNDS = ((-1.0, 1.0), (-2.0, 2.0))
HARRIS_LEVELS = 3
#: the refinement rule of the Harris workload: |J| dx above 1e-7 (the current sheet and its
#: seeded perturbation out to |y| ~ 0.4), clustered into boxes of 8 to 12 coarse cells a
#: side (refined patches of 12-24 cells, most 16-24): ~1600 uneven patches and 5.6e5 cells
#: over three levels
HARRIS_THRESHOLD = 1e-7
HARRIS_PATCH = 12  # coarse cells a side at most, so refined patches of at most 24 cells
HARRIS_MIN_PATCH = 8  # coarse cells a side at least, where the tagged region allows


def _harris_model(cls, precision, seed, *, levels=HARRIS_LEVELS, base=HARRIS_BASE, **options):
    """The Harris-sheet workload: set on the base level, then refined on the current."""
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.problems import harris_sheet

    density, pressure, potential = harris_sheet(*base, seed=seed, bounds=HARRIS_BOUNDS)
    mesh = AMRHierarchy(base, HARRIS_BOUNDS, periodic=(True, False))
    model = cls(mesh, limiter="mc", cfl=0.4, precision=precision, **options)
    model.set_state(density, (0.0, 0.0, 0.0), pressure, vector_potential=potential)
    for _ in range(levels):
        model.regrid(model.current_tags(HARRIS_THRESHOLD, levels=levels), max_patch_size=HARRIS_PATCH,
                     min_patch_size=HARRIS_MIN_PATCH)
    return model


def _harris_on(mesh, cls, precision, seed, **options):
    """The Harris-sheet state set directly on a given hierarchy (all levels)."""
    from wellbalanced_b200.problems import harris_sheet

    density, pressure, potential = harris_sheet(*mesh.shape, seed=seed, bounds=HARRIS_BOUNDS)
    model = cls(mesh, limiter="mc", cfl=0.4, precision=precision, **options)
    model.set_state(density, (0.0, 0.0, 0.0), pressure, vector_potential=potential)
    return model


def _copy_mesh(mesh):
    from wellbalanced_b200.mesh import AMRHierarchy

    out = AMRHierarchy(mesh.shape, mesh.bounds, mesh.periodic)
    for p in mesh.patches:
        if p.level:
            out.add_patch(p.level, p.box)
    return out


#: set by main() when the workload's state fits in L2: a buffer larger than L2 that is
#: rewritten before every timed step, outside its CUDA events
L2_FLUSH = None


def _flush_buffer(engine, device_index):
    """A device buffer of twice the L2 size when both state pools fit in L2, else None."""
    import torch

    l2 = getattr(torch.cuda.get_device_properties(device_index), "L2_cache_size", 126 * 2**20) or 126 * 2**20
    pools = 2 * engine.state.numel() * engine.state.element_size()
    if pools >= l2:
        return None
    return torch.empty(2 * l2 // 4, dtype=torch.float32, device=engine.state.device)


def _device_seconds(step, steps, flush=None):
    """Device seconds of `steps` calls of `step` (CUDA events); with `flush`, the L2 is
    overwritten before every call, outside the events, and the per-call times summed."""
    import torch

    if flush is None:
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(steps):
            step()
        end.record()
        torch.cuda.synchronize()
        return start.elapsed_time(end) / 1e3
    pairs = []
    for _ in range(steps):
        flush.fill_(1.0)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        step()
        end.record()
        pairs.append((start, end))
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in pairs) / 1e3


def _time_steps(step, steps):
    """Device seconds of `steps` calls of `step` after one warm-up call (CUDA events)."""
    import torch

    step()
    torch.cuda.synchronize()
    return _device_seconds(step, steps, L2_FLUSH)


def _rel_l1(ref, low, patches, steps):
    """Relative L1 of density and energy of `low` against `ref` over the given patches."""
    import torch

    out = {"steps": steps,
           "bound": 1e-5,
           "against": "float64 device step from the same state (float64 step == reference to 1e-12 in the tests)"}
    for key, f in (("density", 0), ("energy", 4)):
        num = den = 0.0
        for pr, pl in patches:
            a = ref._read(pr, f).to(torch.float64)
            b = low._read(pl, f).to(torch.float64)
            num += float(torch.sum(torch.abs(b - a)))
            den += float(torch.sum(torch.abs(a)))
        out[f"rel_l1_{key}"] = num / den
    return out


def _drift(before, after):
    """Largest change of a conserved total relative to the largest total."""
    scale = max(abs(v) for v in before.values()) or 1.0
    return max(abs(after[k] - before[k]) for k in before) / scale


def describe(timings):
    return {str(k): round(float(v), 4) for k, v in sorted(timings.items())} if timings else None


class Turbulence:
    @property
    def bytes_per_zone_update(self):
        # 5 state passes x 8 values (5 cell + 3 edge) x the state's bytes
        return 5 * 8 * (4 if self.precision == 32 else 8)

    @property
    def kernel(self):
        ty, tz = self.engine.layout.tile_shape
        state = "float" if self.precision == 32 else "double"
        return f"wb::stage3d_kernel<{state}, float, 2, false, {ty}, {tz}>"

    def __init__(self, args, rank):
        from wellbalanced_b200.mhd3d import MHD3D

        self.n = args.cells
        self.rank = rank
        self.args = args
        self.precision = getattr(args, "precision", 32)
        lx = args.lx if args.lx == "auto" else int(args.lx)
        self.model = MHD3D.turbulence(self.n, seed=rank, precision=self.precision, lx=lx)
        self.engine = self.model.engine
        if args.tile3d and lx != "auto":
            from wellbalanced_b200.autotune import _set_tile

            _set_tile(self.engine, tuple(int(v) for v in args.tile3d.split("x")))
        self.lx = self.model.lx
        self.cells = self.n**3

    #: the Mach-1 box leaves the method's positivity range after ~700 steps (in the
    #: reference's float64 arithmetic too): longer timed runs restart from the post-warm-up
    #: state every `max_steps` steps, outside the timed events
    max_steps = 300

    def advance(self, steps):
        self.model.advance(steps, check=False)

    def restore(self, state, time):
        self.engine.state.copy_(state)
        self.engine.dt_ready = False
        self.engine.time.copy_(time)
        self.model.time = float(time[0].item())

    @staticmethod
    def describe(args):
        state = ("float32 state (float64 pressure recovery)" if getattr(args, "precision", 32) == 32 else
                 "float32 arithmetic on a float64 state (float64 pressure recovery, potential differences, "
                 "flux differences and updates)")
        return (f"3D decaying turbulence, periodic {args.cells}^3, MC-PLM + HLLD + CT, SSP-RK2, CFL 0.3, "
                f"{state}, k^-2 seeded fields, Mach 1, |B|_rms 1")

    def config(self):
        eng = self.engine
        return {
            "workload": self.describe(self.args),
            "cells_per_gpu": self.cells,
            "tile": {"y": eng.layout.tile_shape[0], "z": eng.layout.tile_shape[1], "x_planes": self.lx},
            "autotune_ms_per_launch": describe(self.model.lx_timings),
        }

    def plain(self, steps=3):
        """zone-updates/s of the plain float64 GPU step (`wellbalanced_b200.plain.PlainMHD3D`)."""
        from wellbalanced_b200.mesh import AMRHierarchy
        from wellbalanced_b200.plain import PlainMHD3D
        from wellbalanced_b200.problems import turbulence_3d

        n = self.n
        rho, velocity, p, potential = turbulence_3d(n, seed=self.rank)
        model = PlainMHD3D(AMRHierarchy((n,) * 3, ((0.0, 1.0),) * 3, periodic=(True,) * 3), limiter="mc", cfl=0.3)
        model.set_state(rho, velocity, p, vector_potential=potential)
        seconds = _time_steps(model.step, steps)
        return {"value": self.cells * steps / seconds, "unit": UNIT, "ms_per_step": 1e3 * seconds / steps,
                "steps": steps,
                "what": "PlainMHD3D: the reference MHD3D dataflow on the device, float64, per-kernel, intermediates in HBM"}

    #: the configuration's horizon: 100 RK2 steps
    horizon = 100

    def accuracy(self, steps=None):
        import torch

        from wellbalanced_b200.mhd3d import MHD3D

        steps = self.horizon if steps is None else steps
        ref = MHD3D.turbulence(self.n, seed=self.rank, precision=64)
        low = MHD3D.turbulence(self.n, seed=self.rank, precision=self.precision)
        before = low.totals()
        for _ in range(steps):
            low.step(ref.step())
        out = _rel_l1(ref, low, list(zip(ref.hierarchy.patches, low.hierarchy.patches, strict=True)), steps)
        out["div_b"] = low.divergence()
        out["totals_drift"] = _drift(before, low.totals())
        del ref, low
        torch.cuda.empty_cache()
        return out


class PartitionedTurbulence(Turbulence):
    """The turbulence workload as one periodic box of N slabs of n^3 cells along x, one slab
    per rank (`AMRHierarchy(..., comm=group)`: the rank's patch, its halos exchanged with
    the neighbour ranks over NCCL every fill, dt the global minimum): weak scaling of one
    problem rather than N replicas. Every slab holds the same seeded n^3 fields, so the box
    is periodic with period n along x."""

    def __init__(self, args, rank):
        import torch.distributed as dist

        from wellbalanced_b200.mesh import AMRHierarchy
        from wellbalanced_b200.mhd3d import MHD3D
        from wellbalanced_b200.problems import conserved_3d, turbulence_3d

        world = dist.get_world_size() if dist.is_initialized() else 1
        self.n, self.rank, self.args, self.world = args.cells, rank, args, world
        self.precision = getattr(args, "precision", 32)
        n = self.n
        lx = 32 if args.lx == "auto" else int(args.lx)
        mesh = AMRHierarchy((n * world, n, n), ((0.0, float(world)), (0.0, 1.0), (0.0, 1.0)), periodic=(True,) * 3,
                            comm=dist.group.WORLD if world > 1 else None, split=(world, 1, 1))
        self.model = MHD3D(mesh, limiter="mc", cfl=0.3, precision=self.precision, lx=lx)
        rho, velocity, p, potential = turbulence_3d(n, seed=0, gamma=self.model.gamma)
        cells = conserved_3d(rho, velocity, p, potential, (1.0 / n,) * 3, gamma=self.model.gamma)
        extras = ((0, 1, 1), (1, 0, 1), (1, 1, 0))
        for patch in self.model._local():
            for f, value in enumerate(cells):
                self.model._write(patch, f, value)
            for c, value in enumerate(potential):
                self.model._write(patch, 5 + c, value, extras[c])
        self.model._after_state()
        self.model._ready = True
        self.engine = self.model.engine
        self.lx = lx
        self.cells = n**3
        self.model.lx_timings = None

    @staticmethod
    def describe(args):
        return (f"3D decaying turbulence as one periodic box of N slabs of {args.cells}^3 (one per GPU, halos over "
                "NCCL, global dt), MC-PLM + HLLD + CT, SSP-RK2, CFL 0.3, float32 state")

    def config(self):
        out = super().config()
        out["partition"] = f"{self.world} slabs of {self.n}^3 along x, one per rank"
        return out

    def plain(self, steps=3):
        return None

    def accuracy(self, steps=None):
        return None


def _kernel2d(engine):
    tx, ty = engine.layout.tile_shape
    return f"wb::stage2d_kernel<float, 2, false, {tx}, {ty}>"


class BatchWorkload:
    bytes_per_zone_update = 5 * 7 * 4  # 5 state passes x 7 values (6 cell + 1 node) x float32

    @property
    def kernel(self):
        return _kernel2d(self.engine)

    def __init__(self, args, rank):
        from wellbalanced_b200.batch import Batch

        self.count = args.count
        self.rank = rank
        self.args = args
        self.batch = Batch.orszag_tang(self.count, seed=rank, precision=32, tile="auto")
        self.engine = self.batch.engine
        self.cells = self.batch.cells

    def advance(self, steps):
        for _ in range(steps):
            self.batch._step_launches()
        self.batch.steps += steps

    def graph_timing(self, steps):
        """ms per step of the same steps replayed from one captured CUDA graph."""
        self.batch.capture()
        seconds = _time_steps(lambda: self.batch.advance(1, check=False), steps)
        self.batch._graph = None
        return 1e3 * seconds / steps

    @staticmethod
    def describe(args):
        return (f"{args.count} independent periodic 2D Orszag-Tang problems, sides from {{32, 48, ..., 256}} "
                "(seeded per rank), amplitudes x U[0.5, 1.5], MC-PLM + HLLD + CT, SSP-RK2, per-instance "
                "CFL 0.4 dt, float32 state, one launch per kernel for all instances")

    def config(self):
        sides = [s for s, _ in self.batch.sides]
        return {
            "workload": self.describe(self.args),
            "cells_per_gpu": self.cells,
            "instances": self.count,
            "mean_side": float(sum(sides) / len(sides)),
            "tile": {"x": self.engine.layout.tile_shape[0], "y": self.engine.layout.tile_shape[1]},
            "autotune_tile_ms_per_launch": self.batch.tile_timings,
        }

    def plain(self, count=8, steps=2):
        """The plain float64 GPU step looped over a seeded subset of the instances."""
        from wellbalanced_b200.mesh import AMRHierarchy
        from wellbalanced_b200.plain import PlainMHD2D
        from wellbalanced_b200.problems import orszag_tang_2d, orszag_tang_sizes

        sides, bf, vf = orszag_tang_sizes(self.count, seed=self.rank)
        models, cells = [], 0
        for k in range(count):
            n = int(sides[k])
            model = PlainMHD2D(AMRHierarchy((n, n), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, True)), limiter="mc",
                               cfl=0.4)
            model.set_conserved(*orszag_tang_2d(n, bf[k], vf[k]))
            models.append(model)
            cells += n * n

        def step_all():
            for model in models:
                model.step()

        seconds = _time_steps(step_all, steps)
        return {"value": cells * steps / seconds, "unit": UNIT, "ms_per_step": 1e3 * seconds / steps, "steps": steps,
                "what": f"PlainMHD2D (the reference MHD2D dataflow per kernel, float64) looped over the first {count} "
                        "instances of the batch"}

    #: the configuration's horizon: 200 steps per instance
    horizon = 200

    def accuracy(self, steps=None):
        import torch

        from wellbalanced_b200.mesh import AMRHierarchy
        from wellbalanced_b200.mhd import MHD2D
        from wellbalanced_b200.problems import orszag_tang_2d, orszag_tang_sizes

        steps = self.horizon if steps is None else steps
        sides, bf, vf = orszag_tang_sizes(self.count, seed=self.rank)
        k = int(max(range(len(sides)), key=lambda i: sides[i]))
        n = int(sides[k])
        models = []
        for precision in (64, 32):
            model = MHD2D(AMRHierarchy((n, n), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, True)), limiter="mc",
                          cfl=0.4, precision=precision)
            model.set_conserved(*orszag_tang_2d(n, bf[k], vf[k]))
            models.append(model)
        ref, low = models
        before = low.totals()
        for _ in range(steps):
            low.step(ref.step())
        out = _rel_l1(ref, low, list(zip(ref.hierarchy.patches, low.hierarchy.patches, strict=True)), steps)
        out["instance"] = f"{n}^2 (instance {k})"
        out["div_b"] = low.divergence()
        out["totals_drift"] = _drift(before, low.totals())
        del ref, low, models
        torch.cuda.empty_cache()
        return out


class Harris:
    bytes_per_zone_update = 5 * 7 * 4

    @property
    def kernel(self):
        return _kernel2d(self.engine)

    def __init__(self, args, rank):
        from wellbalanced_b200.mhd import MHD2D

        self.rank = rank
        self.model = _harris_model(MHD2D, 32, rank, tile="auto")
        self.engine = self.model.engine
        self.cells = int(sum(p.shape[0] * p.shape[1] for p in self.model.hierarchy.patches))

    def advance(self, steps):
        self.model.advance(steps, check=False)

    def graph_timing(self, steps):
        """ms per step of the same steps replayed from one captured CUDA graph."""
        self.model.capture()
        seconds = _time_steps(lambda: self.model.advance(1, check=False), steps)
        self.model._graph = None
        return 1e3 * seconds / steps

    def schedule_timing(self, steps):
        """ms and launches per step of the two schedules of the refined step: the small ops
        between the stages as separate launches (fill, restrict, register, rate), and as two
        op programs (device work lists drained by one launch each)."""
        eng = self.engine
        default = eng.use_programs
        out = {}
        for name, programs in (("separate_launches", False), ("op_programs", True)):
            eng.use_programs = programs
            eng.dt_ready = False
            self.model.advance(2, check=False)
            first = eng.launches
            seconds = _time_steps(lambda: self.model.advance(1, check=False), steps)
            out[name] = {"ms_per_step": 1e3 * seconds / steps,
                         "launches_per_step": (eng.launches - first) / (steps + 1),
                         "value": self.cells * steps / seconds}
        eng.use_programs = default
        eng.dt_ready = False
        out["default"] = "op_programs" if default else "separate_launches"
        return out

    def regrid_timing(self):
        """Milliseconds of one regrid of the hierarchy on its own rule (|J| dx above the
        threshold on every level, the same boxes): the device tags read back, then the
        clustering, the new op lists and the device transfer (`MHD2D.regrid`). Leaves the
        model on the new hierarchy."""
        import torch

        model = self.model
        torch.cuda.synchronize()
        start = time.perf_counter()
        tags = model.current_tags(HARRIS_THRESHOLD, levels=HARRIS_LEVELS)
        tagged = time.perf_counter()
        model.regrid(tags, max_patch_size=HARRIS_PATCH, min_patch_size=HARRIS_MIN_PATCH)
        torch.cuda.synchronize()
        done = time.perf_counter()
        self.engine = model.engine
        self.cells = int(sum(p.shape[0] * p.shape[1] for p in model.hierarchy.patches))
        return {"tags_ms": 1e3 * (tagged - start), "regrid_ms": 1e3 * (done - tagged),
                "patches_after": len(model.hierarchy.patches),
                "what": "one regrid on the current tags: device tags read back (tags_ms); host clustering, "
                        "op lists and engine, device transfer (regrid_ms)"}

    @staticmethod
    def describe(args):
        return (f"2D Harris sheet on [-1,1]x[-2,2], base {HARRIS_BASE[0]}x{HARRIS_BASE[1]}, periodic x, "
                f"outflow y, {HARRIS_LEVELS} refined levels on |J| dx > {HARRIS_THRESHOLD} (patches of "
                f"{2 * HARRIS_MIN_PATCH}-{2 * HARRIS_PATCH} cells a side where the tags allow), MC-PLM + HLLD + CT, SSP-RK2, CFL 0.4 at the finest dx, "
                "float32 state with float64 refluxing, all patches in one launch per kernel")

    def config(self):
        h = self.model.hierarchy
        refined = [p.shape for p in h.patches if p.level]
        return {
            "workload": self.describe(None),
            "cells_per_gpu": self.cells,
            "patches": len(h.patches),
            "patches_per_level": {str(lv): len(h.patches_at_level(lv)) for lv in range(h.max_level + 1)},
            "refined_patch_sides": [min(min(s) for s in refined), max(max(s) for s in refined)] if refined else None,
            "tile": {"x": self.engine.layout.tile_shape[0], "y": self.engine.layout.tile_shape[1]},
            "autotune_tile_ms_per_launch": self.model.tile_timings,
        }

    def plain(self, steps=2):
        from wellbalanced_b200.plain import PlainMHD2D

        model = _harris_on(_copy_mesh(self.model.hierarchy), PlainMHD2D, 64, self.rank)
        seconds = _time_steps(model.step, steps)
        return {"value": self.cells * steps / seconds, "unit": UNIT, "ms_per_step": 1e3 * seconds / steps,
                "steps": steps,
                "what": "PlainMHD2D (the reference MHD2D dataflow per kernel, float64) on the same hierarchy"}

    #: steps of the accuracy comparison (the configuration states no horizon)
    horizon = 100

    def accuracy(self, steps=None):
        import torch

        from wellbalanced_b200.mhd import MHD2D

        steps = self.horizon if steps is None else steps
        ref = _harris_on(_copy_mesh(self.model.hierarchy), MHD2D, 64, self.rank)
        low = _harris_on(_copy_mesh(self.model.hierarchy), MHD2D, 32, self.rank)
        before = low.totals()
        for _ in range(steps):
            low.step(ref.step())
        base = list(zip(ref.hierarchy.patches_at_level(0), low.hierarchy.patches_at_level(0), strict=True))
        out = _rel_l1(ref, low, base, steps)
        out["against"] = "float64 device step from the same state on the same hierarchy (base level, restricted)"
        out["div_b"] = low.divergence()
        out["composite_div_b"] = low.composite_divergence()
        out["totals_drift"] = _drift(before, low.totals())
        del ref, low
        torch.cuda.empty_cache()
        return out


WORKLOADS = {"turbulence": Turbulence, "batch": BatchWorkload, "harris": Harris}


# ---- CPU legs (the oracle: NumPy restatement of the reference's step) ---------------------------
def _cpu_sample(job):
    """One process's bounded sample: (zone-updates, seconds) of `steps` oracle steps."""
    workload, seed, steps, n3d = job
    if workload == "turbulence":
        from oracle.mesh import Hierarchy
        from oracle.mhd3d import MHD3D
        from wellbalanced_b200.problems import turbulence_3d

        rho, velocity, p, potential = turbulence_3d(n3d, seed=seed)
        model = MHD3D(Hierarchy((n3d,) * 3, ((0.0, 1.0),) * 3, (True,) * 3), limiter="mc", cfl=0.3)
        model.set_state(rho, velocity, p, vector_potential=potential)
        cells = n3d**3
    elif workload == "batch":
        from oracle.mesh import Hierarchy
        from oracle.mhd2d import MHD2D
        from wellbalanced_b200.problems import orszag_tang_2d, orszag_tang_sizes

        sides, bf, vf = orszag_tang_sizes(seed + 1, seed=0)
        n = int(sides[seed])
        model = MHD2D(Hierarchy((n, n), ((0.0, 1.0), (0.0, 1.0)), (True, True)), limiter="mc", cfl=0.4)
        model.set_conserved(*orszag_tang_2d(n, bf[seed], vf[seed]))
        cells = n * n
    else:
        from oracle.mesh import Hierarchy
        from oracle.mhd2d import MHD2D
        from wellbalanced_b200.problems import harris_sheet

        density, pressure, potential = harris_sheet(*HARRIS_BASE, seed=seed, bounds=HARRIS_BOUNDS)
        model = MHD2D(Hierarchy(HARRIS_BASE, HARRIS_BOUNDS, (True, False)), limiter="mc", cfl=0.4)
        model.set_state(density, (0.0, 0.0, 0.0), pressure, vector_potential=potential)
        cells = HARRIS_BASE[0] * HARRIS_BASE[1]
    if steps == 0:
        return 0, 0.0
    model.step()  # warm-up
    start = time.perf_counter()
    for _ in range(steps):
        model.step()
    return cells * steps, time.perf_counter() - start


CPU_SAMPLES = {
    "turbulence": "3D turbulence 64^3",
    "batch": "the batch's first Orszag-Tang instance",
    "harris": "the Harris sheet's 128x256 base level (unrefined)",
}


def cpu_baseline(workload):
    """The oracle's step on one core (zone-updates/s), a bounded sample of the workload."""
    cells, seconds = _cpu_sample((workload, 0, 3, 64))
    return {"value": cells / seconds, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"NumPy restatement of the reference step, {CPU_SAMPLES[workload]}, 3 RK2 steps after 1 warm-up, "
                      "1 process"}


#: cells a side of the turbulence box each host process steps in the reference arm: large
#: enough that the two-cell ghost layers are a small share of the work (a third of a 32^3
#: box's haloed arrays are ghosts, 17% of a 64^3 box's)
REFERENCE_BOX = 64


def reference_arm(args):
    import multiprocessing as mp

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        pool.map(_cpu_sample, [(args.workload, s, 0, REFERENCE_BOX) for s in range(cores)])  # spin up, import
        per_step = []
        for step in range(args.warmup + args.steps):
            start = time.perf_counter()
            results = pool.map(_cpu_sample, [(args.workload, s, 1, REFERENCE_BOX) for s in range(cores)])
            wall = time.perf_counter() - start
            if step >= args.warmup:
                per_step.append((sum(c for c, _ in results), wall))
    total_cells = sum(c for c, _ in per_step)
    total_time = sum(t for _, t in per_step)
    value = total_cells / total_time
    sample = {"turbulence": f"a {REFERENCE_BOX}^3 turbulence box of the same seeded fields",
              "batch": "one Orszag-Tang instance of the batch",
              "harris": "the 128x256 Harris base level"}[args.workload]
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
        "config": {"workload": WORKLOADS[args.workload].describe(args), "cpu_sample": sample},
        "cpu_baseline": {
            "value": value,
            "unit": UNIT,
            "cores": cores,
            "kind": "port",
            "sample": f"{cores} processes, each one RK2 step of {sample} per bench step (after a warm-up step; "
                      "NumPy restatement of the reference step; the reference is pure Python)",
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


PROFILES = {"turbulence": "stage3d_turbulence.md", "batch": "stage2d_batch.md", "harris": "stage2d_harris.md"}


def profile_figure(workload, key):
    """A per-cell figure (`key: value` line) of the committed ncu summary of the workload,
    or None."""
    path = ROOT / "profiles" / PROFILES[workload]
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        if line.strip().startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def profile_traffic(workload, cells):
    """DRAM bytes per stage launch from the committed ncu summary of the workload (its
    per-cell figure times this run's cells), or None."""
    per_cell = profile_figure(workload, "traffic_bytes_per_cell_launch")
    return None if per_cell is None else per_cell * cells


def issue_roofline(workload, cells, launch_s, clock_info):
    """The stage kernel against its instruction-issue ceiling: the warp instructions of one
    launch (the ncu summary's per-cell count times this run's cells) over the live launch
    time, against one warp instruction per cycle on each of the four schedulers of every SM
    at the SM clock sampled during the timed region (else the maximum clock)."""
    import torch

    per_cell = profile_figure(workload, "warp_instructions_per_cell_launch")
    if per_cell is None or not launch_s > 0:
        return None
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = None
    if clock_info:
        mhz = clock_info.get("sm_mhz") or clock_info.get("sm_max_mhz")
    if not mhz:
        return None
    achieved = per_cell * cells / launch_s
    peak = 4.0 * sms * mhz * 1e6
    return {"achieved": achieved, "peak": peak, "unit": "warp instructions/s", "frac": achieved / peak,
            "warp_instructions_per_cell_launch": per_cell, "sm_mhz": mhz, "sms": sms}


def measure(work, args, rank, world, local, barrier, *, steps, warmup, e2e=True, graph=True):
    """Time `steps` RK2 steps of `work` after `warmup` untimed ones (barrier and device
    synchronisation on both sides, CUDA events, max over ranks), then the graph replay and
    the end-to-end leg. Returns the raw figures of the run."""
    import torch
    import torch.distributed as dist

    global L2_FLUSH
    eng = work.engine
    L2_FLUSH = _flush_buffer(eng, local)
    work.advance(warmup)
    torch.cuda.synchronize()

    # timed region: K RK2 steps, state resident in HBM
    eng.stage_events = []
    launches0 = eng.launches
    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    chunk = getattr(work, "max_steps", None) or steps
    saved = (eng.state.clone(), eng.time.clone()) if steps > chunk else None
    seconds, left = 0.0, steps
    while left > 0:
        n = min(chunk, left)
        if L2_FLUSH is None:
            seconds += _device_seconds(lambda: work.advance(n), 1)
        else:
            seconds += _device_seconds(lambda: work.advance(1), n, L2_FLUSH)
        left -= n
        if left > 0:
            work.restore(*saved)  # outside the timed events
    del saved
    barrier()
    clock_info = clocks.stop()
    launches = eng.launches - launches0
    stage_ms = [s.elapsed_time(e) for s, e in eng.stage_events]
    eng.stage_events = None
    if int(eng.bad.item()):
        raise FloatingPointError("bad cells during the benchmark")
    t = torch.tensor([seconds], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    seconds = float(t.item())
    out = {"seconds": seconds, "value": world * work.cells * steps / seconds, "launches": launches,
           "stage_ms": stage_ms, "clocks": clock_info, "steps": steps, "warmup": warmup}
    out["graph_ms"] = work.graph_timing(min(steps, 50)) if graph and hasattr(work, "graph_timing") else None

    # end to end with host buffers: per step, the state pool is copied in from pinned host
    # memory, advanced one step and copied back
    out["e2e"] = None
    if e2e:
        pool = eng.state
        host = torch.empty(pool.shape, dtype=pool.dtype, pin_memory=True)
        host.copy_(pool)
        torch.cuda.synchronize()
        e2e_steps = max(3, min(steps, 20))
        barrier()
        torch.cuda.synchronize()

        def round_trip():
            pool.copy_(host, non_blocking=True)
            eng.dt_ready = False  # the step's dt from the state copied in
            work.advance(1)
            host.copy_(pool, non_blocking=True)

        e2e_seconds = _device_seconds(round_trip, e2e_steps, L2_FLUSH)
        barrier()
        t2 = torch.tensor([e2e_seconds], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t2, op=dist.ReduceOp.MAX)
        nbytes = host.numel() * host.element_size()
        out["e2e"] = {
            "value": world * work.cells * e2e_steps / float(t2.item()),
            "unit": UNIT,
            "h2d_bytes_per_step": int(nbytes),
            "d2h_bytes_per_step": int(nbytes),
            "path": "state pool copied in from pinned host memory, one step, copied back (every step)",
        }
    return out


def roofline(name, work, run):
    """The stage kernel's HBM roofline of a measured run (rank 0)."""
    peak, peak_kind = peaks()
    cells = work.cells
    launch_s = statistics.mean(run["stage_ms"]) / 1e3 if run["stage_ms"] else float("nan")
    per_launch = work.bytes_per_zone_update / 2 * cells
    achieved = per_launch / launch_s / 1e9
    return {
        "bound": "hbm",
        "achieved": achieved,
        "peak": peak,
        "unit": "GB/s",
        "frac": achieved / peak,
        # the committed ncu figures are of the float32-state kernels
        "traffic": profile_traffic(name, cells) if getattr(work, "precision", 32) == 32 else None,
        "kernel": work.kernel,
        "algorithmic_bytes_per_launch": per_launch,
        "mean_launch_ms": 1e3 * launch_s,
        "peak_kind": peak_kind,
        "issue": issue_roofline(name, cells, launch_s, run["clocks"]) if getattr(work, "precision", 32) == 32 else None,
    }


def workload_config(work, world, args, steps):
    eng = work.engine
    config = work.config()
    config["parallelism"] = (f"one box in {world} slabs (patches per rank, NCCL halos)"
                             if getattr(work, "world", None) else f"replicas x{world}")
    limit = getattr(work, "max_steps", None)
    if limit and steps > limit:
        config["timed_runs"] = (f"{-(-steps // limit)} runs of at most {limit} steps, each from the state "
                                "after warm-up (restored outside the timed events)")
    pool_gb = eng.state.numel() * eng.state.element_size() / 1e9
    if L2_FLUSH is None:
        config["l2"] = "inputs larger than L2 (state pool {:.2f} GB per copy)".format(pool_gb)
    else:
        config["l2"] = ("L2 flushed before every timed step, outside its CUDA events (a {:.0f} MB write; "
                        "state pool {:.3f} GB per copy, smaller than L2)").format(L2_FLUSH.numel() * 4 / 1e6, pool_gb)
    return config


#: the configurations measured beside the headline in the default run: (workload, state
#: precision, steps, warm-up); the float32-state headline's twin with a float64 state
#: meets the L1 bound over the longest horizons (Orszag-Tang 256^2 to t = 0.5)
EXTRA_WORKLOADS = {"turbulence_mixed": ("turbulence", "mixed", 20, 3), "batch": ("batch", 32, 20, 3),
                   "harris": ("harris", 32, 50, 5)}


def extra_workload(name, args, rank, world, local, barrier):
    """One more configuration measured in the same run (value, roofline, graph replay,
    plain float64 step, accuracy over its horizon), as a `workloads` entry."""
    import copy

    import torch

    kind, precision, steps, warmup = EXTRA_WORKLOADS[name]
    args = copy.copy(args)
    args.precision = precision
    work = WORKLOADS[kind](args, rank)
    run = measure(work, args, rank, world, local, barrier, steps=steps, warmup=warmup, e2e=False)
    entry = {
        "value": run["value"],
        "unit": UNIT,
        "ms_per_step": 1e3 * run["seconds"] / steps,
        "steps": steps,
        "warmup": warmup,
        "gpu_launches": run["launches"],
        "launches_per_step": run["launches"] / steps,
        "config": workload_config(work, world, args, steps),
        "roofline": roofline(kind, work, run),
        "precision": precision,
        "clocks": run["clocks"],
    }
    if run["graph_ms"] is not None:
        entry["graph"] = {"ms_per_step": run["graph_ms"], "value": world * work.cells / (run["graph_ms"] / 1e3),
                          "what": "the same steps replayed from one captured CUDA graph"}
    if hasattr(work, "schedule_timing"):
        entry["schedules"] = work.schedule_timing(steps)
    if rank == 0 and not args.no_plain and kind != args.workload:
        entry["plain_fp64"] = work.plain()
        entry["plain_fp64"]["speedup_of_value"] = run["value"] / world / entry["plain_fp64"]["value"]
    if rank == 0 and not args.no_accuracy:
        entry["accuracy"] = work.accuracy()
    if hasattr(work, "regrid_timing"):
        entry["regrid"] = work.regrid_timing()  # last: it moves the model to a new hierarchy
    del work
    torch.cuda.empty_cache()
    return entry


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
        baseline = cpu_baseline(args.workload)  # before any GPU work

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    if args.partition and args.workload != "turbulence":
        raise SystemExit("--partition splits the turbulence box")
    work = (PartitionedTurbulence if args.partition else WORKLOADS[args.workload])(args, rank)
    run = measure(work, args, rank, world, local, barrier, steps=args.steps, warmup=args.warmup,
                  e2e=not args.no_e2e)
    value, seconds = run["value"], run["seconds"]
    plain = work.plain() if rank == 0 and not args.no_plain else None
    accuracy = work.accuracy() if rank == 0 and not args.no_accuracy else None
    config = workload_config(work, world, args, args.steps) if rank == 0 else None
    line_roofline = roofline(args.workload, work, run) if rank == 0 else None
    graph = None
    if run["graph_ms"] is not None:
        graph = {"ms_per_step": run["graph_ms"], "value": world * work.cells / (run["graph_ms"] / 1e3),
                 "what": "the same steps replayed from one captured CUDA graph"}

    # the other configurations, measured in the same run at one GPU (the headline's
    # scaling lines carry the headline workload only)
    extras = {}
    if world == 1 and args.workload == "turbulence" and not args.no_extra:
        del work
        torch.cuda.empty_cache()
        for name in EXTRA_WORKLOADS:
            extras[name] = extra_workload(name, args, rank, world, local, barrier)

    if rank == 0:
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
            "config": config,
            "roofline": line_roofline,
            "gpu_launches": run["launches"],
            "clocks": run["clocks"],
        }
        if graph is not None:
            line["graph"] = graph
        if baseline is not None:
            line["cpu_baseline"] = baseline
        if run["e2e"] is not None:
            line["e2e"] = run["e2e"]
        if accuracy is not None:
            line["accuracy"] = accuracy
        if plain is not None:
            line["plain_fp64"] = plain
            line["plain_fp64"]["speedup_of_value"] = value / world / plain["value"]
        if extras:
            line["workloads"] = extras
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
