"""Many independent 2D problems advanced together: one launch per kernel for all of them.

`Batch` holds N periodic 2D problems of any sizes in one device pool (one patch each,
`Layout.merge`), each with its own time step: the rate kernel reduces per instance and
the stage kernels read each tile's instance dt, so one launch of each kernel advances
every instance by its own CFL step. A step (rate, dt, two stages, two halo fills) can be
captured in a CUDA graph and replayed.

``Batch.orszag_tang(count, seed)`` builds the batched Orszag–Tang workload: sides drawn
from {32, 48, ..., 256}, field and velocity amplitudes scaled by seeded factors in
[0.5, 1.5] (`wellbalanced_b200.problems.orszag_tang_sizes`).
"""

from __future__ import annotations

import numpy as np
import torch

from wellbalanced_b200 import _lib
from wellbalanced_b200.engine import Engine
from wellbalanced_b200.mesh import HALO, AMRHierarchy, Layout
from wellbalanced_b200.mhd import LIMITER_CODES
from wellbalanced_b200.problems import orszag_tang_2d, orszag_tang_sizes


class Batch:
    """N independent periodic 2D MHD problems on the device (ideal MHD, fused stages)."""

    def __init__(self, sides, *, gamma=5.0 / 3.0, limiter="mc", cfl=0.4, precision=32, device="cuda",
                 bounds=((0.0, 1.0), (0.0, 1.0)), tile=None):
        if limiter not in LIMITER_CODES:
            raise ValueError(f"limiter is one of {sorted(LIMITER_CODES)}")
        if not 0.0 < cfl <= 1.0:
            raise ValueError("cfl must be in (0, 1]")
        self.sides = [tuple(int(v) for v in (s if np.ndim(s) else (s, s))) for s in sides]
        self.count = len(self.sides)
        self.gamma = float(gamma)
        self.limiter = limiter
        self.cfl = float(cfl)
        self.precision = _lib.precision_code(precision)
        parts = {}
        layouts = []
        self.hierarchies = []
        for shape in self.sides:
            if shape not in parts:
                h = AMRHierarchy(shape, bounds, periodic=(True, True))
                parts[shape] = (h, Layout(h, precision=self.precision))
            h, layout = parts[shape]
            self.hierarchies.append(h)
            layouts.append(layout)
        self.layout = Layout.merge(layouts)
        self.engine = Engine(None, precision=self.precision, limiter=LIMITER_CODES.index(limiter), gamma=self.gamma,
                             mean_field=(0.0, 0.0), device=device, layout=self.layout)
        self._patch_starts = np.cumsum([0] + [1] * self.count)
        self.steps = 0
        self._graph = None
        # tile shape of the stage kernel: None (default), (tx, ty), or "auto" (tuned in
        # finish_state, on the batch's own patch sizes)
        self._auto_tile = tile == "auto"
        self.tile = None if tile is None or self._auto_tile else tuple(tile)
        self.tile_timings = None
        if self.tile is not None:
            from wellbalanced_b200.autotune import _set_tile

            _set_tile(self.engine, self.tile)

    @classmethod
    def orszag_tang(cls, count, *, seed=0, precision=32, **options):
        sides, b_factor, v_factor = orszag_tang_sizes(count, seed=seed)
        batch = cls(sides, precision=precision, **options)
        host = np.zeros(batch.layout.pool_size, dtype=np.float32 if batch.precision == 32 else np.float64)
        for k in range(count):
            fields, az = orszag_tang_2d(int(sides[k]), b_factor[k], v_factor[k], gamma=batch.gamma)
            batch._write_host(host, k, fields, az)
        batch.engine.state.copy_(torch.from_numpy(host))
        batch.finish_state()
        return batch

    def _write_host(self, host, k, fields, az):
        """Instance k's conserved cells and A_z into a host copy of the pool."""
        from wellbalanced_b200.mesh import Patch

        nx, ny = self.sides[k]
        patch = Patch(0, ((0, nx), (0, ny)), index=k)
        for f, value in enumerate(fields):
            self.layout.patch_view(host, patch, f)[HALO : HALO + nx, HALO : HALO + ny] = value
        self.layout.patch_view(host, patch, 6)[HALO : HALO + nx + 1, HALO : HALO + ny + 1] = az

    # state ---------------------------------------------------------------------------------------
    def _view(self, k, f, node=False):
        from wellbalanced_b200.mesh import Patch

        nx, ny = self.sides[k]
        patch = Patch(0, ((0, nx), (0, ny)), index=k)
        view = self.layout.patch_view(self.engine.state, patch, f)
        e = 1 if node else 0
        return view[HALO : HALO + nx + e, HALO : HALO + ny + e]

    def set_instance(self, k, fields, az):
        """Conserved cell arrays (rho, mx, my, mz, E, bz) and nodal A_z of instance k."""
        for f, value in enumerate(fields):
            self._view(k, f).copy_(torch.as_tensor(np.ascontiguousarray(value)))
        self._view(k, 6, node=True).copy_(torch.as_tensor(np.ascontiguousarray(az)))

    def finish_state(self):
        self.engine.fill(self.engine.state)
        if self._auto_tile:
            from wellbalanced_b200.autotune import tune_tile2d

            self.tile, timings = tune_tile2d(self.engine)
            self.tile_timings = timings or self.tile_timings
            self._graph = None
        self.engine.time.zero_()
        self.steps = 0

    def instance_state(self, k):
        names = ("density", "momentum_x", "momentum_y", "momentum_z", "energy", "bz")
        out = {name: self._view(k, f).to(torch.float64).cpu().numpy() for f, name in enumerate(names)}
        out["az"] = self._view(k, 6, node=True).to(torch.float64).cpu().numpy()
        return out

    @property
    def cells(self):
        return int(sum(nx * ny for nx, ny in self.sides))

    # stepping ------------------------------------------------------------------------------------
    def _step_launches(self):
        eng = self.engine
        groups = eng.layout.groups
        with eng.launching():
            eng.rate()
            eng.finalize_dt(self.cfl, advance=True)
            eng.heun_step(groups[1:], groups)

    def capture(self):
        """Capture one step (all launches) in a CUDA graph; `advance` then replays it. The
        recording takes one step of every instance."""
        self._graph = self.engine.capture(self._step_launches)
        self.steps += 1

    def advance(self, steps, *, check=True):
        """``steps`` steps of every instance (each at its own stable dt)."""
        eng = self.engine
        if check:
            eng.bad.zero_()
        for _ in range(steps):
            if self._graph is not None:
                self._graph.replay()
            else:
                self._step_launches()
        self.steps += steps
        if check and int(eng.bad.item()):
            raise FloatingPointError("non-positive density or pressure (or non-finite values) in the batch")

    def times(self):
        return self.engine.time.cpu().numpy()
