r"""MHD in two dimensions on the device: the drop-in for ``carafe.mhd.MHD2D``.

Same constructor keywords, test problems and methods as the reference
(``src/carafe/mhd.py:410-1226``): ``set_state``, ``stable_step``, ``step``, ``run``,
``current_tags``, ``regrid``, ``divergence``, ``composite_divergence``, ``totals``,
``dataset``, ``leaf_values``. The state lives in device pools; a step is the fused
stage kernels of ``libwb200.so`` (``wb_stage2d``) with the halo, restriction and
flux-register op lists (`wellbalanced_b200.engine`).

Extra keyword ``precision``: 64 (float64 state and arithmetic, the reference's), 32
(float32 state and arithmetic, the pressure recovery in float64) or "mixed" (float32
reconstruction, HLLD and CT on a float64 state: the conserved and potential updates, the
pressure recovery, the face fields' potential differences and the flux differences in
float64).

Numerics as the reference: MUSCL/PLM reconstruction with the limiter of
``carafe.limiters``, HLLD, CT-contact electric field on the nodes, Heun (SSP-RK2),
vector-potential constrained transport (div B = 0 to round-off), outflow or wall faces,
one time step for all levels.
"""

from __future__ import annotations

from collections.abc import Callable
from typing import Any

import numpy as np
import torch

from wellbalanced_b200 import _lib

from wellbalanced_b200.dataset import Dataset, Variable
from wellbalanced_b200.engine import Engine
from wellbalanced_b200.mesh import HALO, AMRHierarchy

__all__ = ["CONSERVED", "MHD2D", "LIMITER_CODES", "harris_sheets"]

CONSERVED = ("density", "momentum_x", "momentum_y", "momentum_z", "energy", "bz")
LIMITER_CODES = ("minmod", "vanleer", "mc", "none")
BOUNDARIES = ("outflow", "wall")

Value = float | np.ndarray | Callable[..., Any]


class MHD2D:
    """2.5D ideal MHD on the device (see the module docstring).

    Args: as ``carafe.mhd.MHD2D`` (hierarchy, gamma, mean_field, resistivity, limiter,
    cfl, conduction, gravity, boundaries, prefix), plus ``precision`` (32, 64 or "mixed")
    and ``device``.
    """

    def __init__(
        self,
        hierarchy: AMRHierarchy,
        *,
        gamma: float = 5.0 / 3.0,
        mean_field: tuple[float, float] = (0.0, 0.0),
        resistivity: float = 0.0,
        limiter: str = "vanleer",
        cfl: float = 0.4,
        conduction: tuple[float, float] = (0.0, 0.0),
        gravity: tuple[float, float] = (0.0, 0.0),
        boundaries: dict[str, str] | None = None,
        prefix: str = "mhd_",
        precision: int | str = 64,
        device: str = "cuda",
        tile: tuple[int, int] | str | None = None,
    ) -> None:
        if hierarchy.ndim != 2:
            raise ValueError("MHD2D needs a 2D hierarchy")
        if hierarchy.cylindrical or hierarchy.graded:
            raise NotImplementedError("MHD2D is Cartesian on uniform levels: no r–z metric, no graded axes")
        if limiter not in LIMITER_CODES:
            raise ValueError(f"limiter is one of {sorted(LIMITER_CODES)}")
        if not 0.0 < cfl <= 1.0:
            raise ValueError("cfl must be in (0, 1]")
        if gamma <= 1.0:
            raise ValueError("gamma must be larger than 1")
        if not resistivity >= 0.0:
            raise ValueError("resistivity must be non-negative")
        if not min(conduction) >= 0.0:
            raise ValueError("the conductivities must be non-negative")
        kinds = {"x": "outflow", "y": "outflow"}
        for axis_name, kind in (boundaries or {}).items():
            if axis_name not in kinds or kind not in BOUNDARIES:
                raise ValueError(
                    f"boundaries maps 'x' or 'y' to one of {BOUNDARIES}, got {axis_name!r}: {kind!r}"
                )
            axis = "xy".index(axis_name)
            if hierarchy.periodic[axis]:
                raise ValueError(f"the hierarchy is periodic along {axis_name}")
            if kind == "wall" and mean_field[axis] != 0.0:
                raise ValueError(f"a wall normal to {axis_name} needs a zero mean field along it")
            kinds[axis_name] = kind
        self.hierarchy = hierarchy
        self.gamma = float(gamma)
        self.mean_field = (float(mean_field[0]), float(mean_field[1]))
        self.resistivity = float(resistivity)
        self.limiter = limiter
        self.cfl = float(cfl)
        self.conduction = (float(conduction[0]), float(conduction[1]))
        self.gravity = (float(gravity[0]), float(gravity[1]))
        self.walls = tuple(kinds[name] == "wall" for name in "xy")
        self.names = {name: prefix + name for name in CONSERVED}
        self.potential = prefix + "az"
        self.periodic = tuple(hierarchy.periodic)
        self.precision = _lib.precision_code(precision)
        self.device = device
        # tile shape of the stage kernel: None (the default), (tx, ty), or "auto" (tuned
        # when the state is first set; ideal MHD only)
        self._auto_tile = tile == "auto"
        self.tile = None if tile is None or self._auto_tile else tuple(tile)
        self.tile_timings = None
        self._build_engine()
        self.time = 0.0
        self.steps = 0
        self.period = float("nan")
        self._ready = False

    def _local(self):
        """The patches this rank holds (every patch without a partition)."""
        from wellbalanced_b200.distributed import local_patches

        return local_patches(self)

    def _single_rank(self, what):
        if getattr(self, "_group", None) is not None:
            raise NotImplementedError(f"{what} on a hierarchy partitioned over ranks")

    #: whether steps run the fused stage kernels (False: the per-kernel float64 path)
    _fused = True

    def _build_engine(self):
        self._graph = None
        walls = tuple((w, w) for w in self.walls)
        options = dict(precision=self.precision, limiter=LIMITER_CODES.index(self.limiter), gamma=self.gamma,
                       mean_field=self.mean_field, device=self.device)
        from wellbalanced_b200.distributed import solver_engine, solver_group

        # a hierarchy over several ranks (AMRHierarchy(..., comm=group)): this rank's patches
        self._group = solver_group(self.hierarchy)
        if self._group is not None:
            self.engine = solver_engine(self.hierarchy, self._group, walls=walls, **options)
        else:
            self.engine = Engine(self.hierarchy, walls=walls, **options)
        groups = self.engine.layout.groups
        self._groups_all = groups
        self._groups_potential = groups[1:]
        physics = (self.resistivity, self.conduction[0], self.conduction[1], self.gravity[0], self.gravity[1])
        if any(physics):
            self.engine.physics = tuple(float(v) for v in physics)
        # the conduction limit depends on the density: on a refined hierarchy each level's
        # smallest density goes with that level's spacing (carafe/mhd.py:942-960)
        self.engine.per_level_dt = self.engine.max_level > 0 and max(self.conduction) > 0.0
        if self.tile is not None and self._fused:
            if self.engine.physics is not None and self.tile != self.engine.layout.default_tile:
                raise ValueError("resistivity, conduction and gravity run on the default tile shape")
            from wellbalanced_b200.autotune import _set_tile

            _set_tile(self.engine, self.tile)

    # construction of common cases (carafe/mhd.py:486-671) -----------------------------------------
    @classmethod
    def alfven_wave(cls, cells: int, *, amplitude: float = 0.1, **options: Any):
        hierarchy = AMRHierarchy((2 * cells, cells), ((0.0, 2.0), (0.0, 1.0)), periodic=(True, True))
        angle = np.arctan2(2.0, 1.0)
        kx, ky = np.cos(angle), np.sin(angle)
        wavelength = 2.0 / np.sqrt(5.0)
        k = 2.0 * np.pi / wavelength

        def phase(x, y):
            return k * (kx * x + ky * y)

        def velocity(x, y):
            b_perp = amplitude * np.sin(phase(x, y))
            return (b_perp * ky, -b_perp * kx, -amplitude * np.cos(phase(x, y)))

        model = cls(hierarchy, mean_field=(kx, ky), **options)
        model.set_state(
            1.0,
            velocity,
            0.1,
            vector_potential=lambda x, y: amplitude / k * np.cos(phase(x, y)),
            bz=lambda x, y: amplitude * np.cos(phase(x, y)),
        )
        model.period = float(wavelength)
        return model, model.dataset()

    @classmethod
    def rayleigh_taylor(cls, cells: int, *, field: float = 0.0, amplitude: float = 0.01, **options: Any) -> MHD2D:
        """Single-mode Rayleigh-Taylor instability on ``cells x 3 cells`` (``carafe/mhd.py:626-671``):
        density 2 over 1 on [-0.25, 0.25] x [-0.75, 0.75], periodic in x, walls in y, gravity
        -0.1 along y, pressure 2.5 - 0.1 rho y, gamma 1.4, v_y = amplitude (1 + cos 4 pi x)
        (1 + cos 3 pi y) / 4, uniform field ``field`` along x."""
        hierarchy = AMRHierarchy((cells, 3 * cells), ((-0.25, 0.25), (-0.75, 0.75)), periodic=(True, False))
        options = {"gamma": 1.4, **options}
        model = cls(hierarchy, mean_field=(field, 0.0), gravity=(0.0, -0.1), boundaries={"y": "wall"}, **options)

        def density(x, y):
            return np.where(y > 0.0, 2.0, 1.0)

        def velocity(x, y):
            rise = amplitude * (1.0 + np.cos(4.0 * np.pi * x)) * (1.0 + np.cos(3.0 * np.pi * y)) / 4.0
            return (0.0 * x, rise, 0.0 * x)

        model.set_state(density, velocity, lambda x, y: 2.5 - 0.1 * density(x, y) * y)
        return model

    @classmethod
    def orszag_tang(cls, cells: int, **options: Any) -> MHD2D:
        hierarchy = AMRHierarchy((cells, cells), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, True),
                                 split=options.pop("split", None))
        model = cls(hierarchy, **options)
        b0 = 1.0 / np.sqrt(4.0 * np.pi)
        model.set_state(
            25.0 / (36.0 * np.pi),
            lambda x, y: (-np.sin(2 * np.pi * y), np.sin(2 * np.pi * x), 0.0 * x),
            5.0 / (12.0 * np.pi),
            vector_potential=lambda x, y: b0 * (np.cos(4 * np.pi * x) / (4 * np.pi) + np.cos(2 * np.pi * y) / (2 * np.pi)),
        )
        return model

    @classmethod
    def rotor(cls, cells: int, **options: Any) -> MHD2D:
        hierarchy = AMRHierarchy((cells, cells), ((0.0, 1.0), (0.0, 1.0)))
        options = {"gamma": 1.4, **options}
        model = cls(hierarchy, mean_field=(5.0 / np.sqrt(4.0 * np.pi), 0.0), **options)
        r0, r1, speed = 0.1, 0.115, 2.0

        def taper(x, y):
            r = np.hypot(x - 0.5, y - 0.5)
            return r, np.clip((r1 - r) / (r1 - r0), 0.0, 1.0)

        def density(x, y):
            r, f = taper(x, y)
            return np.where(r <= r0, 10.0, 1.0 + 9.0 * f)

        def velocity(x, y):
            r, f = taper(x, y)
            omega = np.where(r <= r0, speed / r0, f * speed / np.maximum(r, r0))
            return (-omega * (y - 0.5), omega * (x - 0.5), 0.0 * x)

        model.set_state(density, velocity, 1.0)
        return model

    @classmethod
    def blast_wave(cls, cells: int, **options: Any) -> MHD2D:
        hierarchy = AMRHierarchy((cells, (3 * cells) // 2), ((-0.5, 0.5), (-0.75, 0.75)), periodic=(True, True))
        field = 1.0 / np.sqrt(2.0)
        options = {"limiter": "minmod", **options}
        model = cls(hierarchy, mean_field=(field, field), **options)
        model.set_state(1.0, (0.0, 0.0, 0.0), lambda x, y: np.where(np.hypot(x, y) < 0.1, 10.0, 0.1))
        return model

    # state ---------------------------------------------------------------------------------------
    @staticmethod
    def _evaluate(value: Value, x: np.ndarray, y: np.ndarray) -> np.ndarray:
        if callable(value):
            return np.broadcast_to(np.asarray(value(x, y), dtype=float), x.shape)
        return np.broadcast_to(np.asarray(value, dtype=float), x.shape)

    def _coordinates(self, patch, node):
        h = self.hierarchy
        dx = h.spacing(patch.level)
        axes = []
        for a, (lo, hi) in enumerate(patch.box):
            start = h.lower_bound[a]
            if node:
                axes.append(start + np.arange(lo, hi + 1) * dx[a])
            else:
                axes.append(start + (np.arange(lo, hi) + 0.5) * dx[a])
        return np.meshgrid(*axes, indexing="ij")

    def _cell_field(self, patch, az):
        dx, dy = self.hierarchy.spacing(patch.level)
        bxf = (az[:, 1:] - az[:, :-1]) / dy + self.mean_field[0]
        byf = -(az[1:, :] - az[:-1, :]) / dx + self.mean_field[1]
        return 0.5 * (bxf[:-1] + bxf[1:]), 0.5 * (byf[:, :-1] + byf[:, 1:])

    def _write(self, patch, field, values):
        self.engine.dt_ready = False
        n = values.shape
        view = self.engine.view(self.engine.state, patch, field)
        view[HALO : HALO + n[0], HALO : HALO + n[1]] = torch.from_numpy(np.require(values, requirements=("C", "W"))).to(
            view.device, view.dtype
        )

    def _read(self, patch, field, node=False, pool=None):
        pool = self.engine.state if pool is None else pool
        n = [s + (1 if node else 0) for s in patch.shape]
        view = self.engine.view(pool, patch, field)
        return view[HALO : HALO + n[0], HALO : HALO + n[1]]

    def set_state(self, density, velocity, pressure, *, vector_potential: Value = 0.0, bz: Value = 0.0) -> None:
        """Set the state on every patch (``carafe/mhd.py:683-737``)."""
        gamma = self.gamma
        for patch in self._local():
            x, y = self._coordinates(patch, False)
            xn, yn = self._coordinates(patch, True)
            rho = self._evaluate(density, x, y)
            if callable(velocity):
                u, v, w = (np.broadcast_to(c, x.shape) for c in velocity(x, y))
            elif isinstance(velocity, tuple | list) and len(velocity) == 3:
                u, v, w = (self._evaluate(c, x, y) for c in velocity)
            else:
                raise ValueError("velocity is a function or three values")
            p = self._evaluate(pressure, x, y)
            if np.any(rho <= 0.0) or np.any(p <= 0.0):
                raise ValueError("the density and the pressure must be positive")
            az = self._evaluate(vector_potential, xn, yn)
            bx, by = self._cell_field(patch, az)
            bzv = self._evaluate(bz, x, y)
            energy = p / (gamma - 1.0) + 0.5 * rho * (u**2 + v**2 + w**2) + 0.5 * (bx**2 + by**2 + bzv**2)
            for f, value in enumerate((rho, rho * u, rho * v, rho * w, energy, bzv)):
                self._write(patch, f, value)
            self._write(patch, 6, az)
        self._after_state()

    def set_conserved(self, fields, az) -> None:
        """Set a one-patch level 0 from conserved arrays ``(rho, mx, my, mz, E, bz)`` and ``A_z``."""
        (patch,) = self.hierarchy.patches_at_level(0)
        for f, value in enumerate(fields):
            self._write(patch, f, np.asarray(value, dtype=float))
        self._write(patch, 6, np.asarray(az, dtype=float))
        self._after_state()

    def _after_state(self, tune=True):
        """The halos and the restriction of a new state; with `tune`, the autotuner's tile
        (a regrid keeps the tile tuned before it: `tune` False)."""
        self.engine.dt_ready = False
        eng = self.engine
        if self.hierarchy.max_level > 0:
            eng.restrict(eng.state, self._groups_all)
        eng.fill(eng.state)
        if tune and self._auto_tile and self._fused and eng.physics is None and getattr(self, "_group", None) is None:
            from wellbalanced_b200.autotune import tune_tile2d

            self.tile, timings = tune_tile2d(eng)
            self.tile_timings = timings or self.tile_timings
        self.time = 0.0
        self.steps = 0
        eng.time.zero_()
        self._ready = True

    def _check_ready(self) -> None:
        if not self._ready:
            raise RuntimeError("set the state first (set_state)")

    # time stepping -------------------------------------------------------------------------------
    def stable_step(self) -> float:
        """The largest stable step (``carafe/mhd.py:930-963``)."""
        self._check_ready()
        eng = self.engine
        eng.rate()
        eng.finalize_dt(self.cfl, self.resistivity, max(self.conduction))
        return float(eng.dt[0].item())

    def _raise_if_bad(self):
        if self.engine.use_programs and self.engine.program_error():
            raise RuntimeError("an op program's phase wait ran out (its device error word is set)")
        if int(self.engine.bad.item()):
            raise FloatingPointError(f"non-positive density or pressure (or non-finite values) at t = {self.time}")

    def step(self, dt: float | None = None) -> float:
        """Advance by one step of Heun's method (SSP-RK2); return the step taken."""
        self._check_ready()
        eng = self.engine
        if dt is None:
            dt = self.stable_step()
        else:
            eng.dt.fill_(float(dt))
        eng.bad.zero_()
        eng.heun_step(self._groups_potential, self._groups_all)
        self._raise_if_bad()
        self.time += float(dt)
        self.steps += 1
        eng.time.fill_(self.time)
        return float(dt)

    def run(self, duration: float, *, max_steps: int = 1_000_000) -> int:
        """Advance by ``duration`` (the last step shortened to land on it); return the steps."""
        self._check_ready()
        if not np.isfinite(duration) or duration < 0.0:
            raise ValueError("duration must be a finite, non-negative time")
        end = self.time + duration
        taken = 0
        while self.time < end * (1.0 - 1e-14) and taken < max_steps:
            dt = min(self.stable_step(), end - self.time)
            self.step(dt)
            taken += 1
        return taken

    def _one_step(self):
        """The launches of one step at the stable dt (dt, time and state on the device).
        With op programs (refined hierarchies) dt is already on the device: `_prime`
        before the first step, then each step's second program leaves the next one."""
        eng = self.engine
        if eng.use_programs:
            eng.programmed_step(self._groups_potential, self._groups_all, self.cfl, self.resistivity, max(self.conduction))
            return
        with eng.launching():
            eng.rate()
            eng.finalize_dt(self.cfl, self.resistivity, max(self.conduction), advance=True)
            eng.heun_step(self._groups_potential, self._groups_all)

    def _prime(self):
        if self.engine.use_programs and not self.engine.dt_ready:
            self.engine.prime_dt(self.cfl, self.resistivity, max(self.conduction))

    def capture(self) -> None:
        """Record one step (rate, dt, both stages, halos, reflux, restriction) in a CUDA
        graph that `advance` replays. The recording takes one step. A regrid drops it."""
        self._single_rank("capture")
        self._check_ready()
        self._prime()
        self._graph = self.engine.capture(self._one_step)
        self.steps += 1
        self.time = float(self.engine.time[0].item())

    def advance(self, steps: int, *, check: bool = True) -> None:
        """``steps`` steps at the stable dt with no host synchronisation (checked at the end
        unless ``check`` is false; the bad-cell count then stays in ``engine.bad``)."""
        self._check_ready()
        eng = self.engine
        eng.bad.zero_()
        self._prime()
        for _ in range(steps):
            if self._graph is not None:
                self._graph.replay()
            else:
                self._one_step()
        self.steps += steps
        if check:
            self.time = float(eng.time[0].item())
            self._raise_if_bad()

    def save(self, host=None):
        """Copy the device state pool into ``host`` (a pinned CPU tensor, allocated if None);
        returns it once the copy has landed."""
        pool = self.engine.state
        if host is None:
            host = torch.empty(pool.shape, dtype=pool.dtype, pin_memory=True)
        host.copy_(pool, non_blocking=True)
        torch.cuda.current_stream(pool.device).synchronize()
        return host

    def load(self, host) -> None:
        """Replace the device state pool by ``host`` (from `save`, same hierarchy and precision)."""
        self.engine.dt_ready = False
        pool = self.engine.state
        if tuple(host.shape) != tuple(pool.shape) or host.dtype != pool.dtype:
            raise ValueError("the saved state belongs to another layout or precision")
        pool.copy_(host, non_blocking=True)
        self._ready = True

    # refinement ----------------------------------------------------------------------------------
    def current_tags(self, threshold: float, levels: int) -> dict[int, np.ndarray]:
        """Tag cells where ``|J_z|`` (the mean over the cell's four nodes) times the cell
        size exceeds ``threshold`` (``carafe/mhd.py:1011-1041``): one kernel over every
        cell of the tagged levels (``wb_current_tags``)."""
        self._single_rank("current_tags")
        from wellbalanced_b200.regrid import device_tags

        return device_tags(self, threshold, levels)

    def regrid(self, tags: dict[int, np.ndarray], **options: Any) -> None:
        """Regrid on ``tags`` (``carafe/mhd.py:1043-1056``): new patches over the tagged
        cells (`AMRHierarchy.regrid` options: ``max_patch_size``, ``buffer``), the conserved
        fields moved with their integrals kept, ``A_z`` interpolated (div B stays zero)."""
        self._single_rank("regrid")
        from wellbalanced_b200.regrid import regrid_model

        regrid_model(self, tags, **options)

    def _field_extras(self):
        return [(0, 0)] * 6 + [(1, 1)]

    def _gather_field(self, patch, f):
        return self.gather(patch, f, node=f == 6)

    def _write_field(self, patch, f, values):
        self._write(patch, f, values)

    # diagnostics ---------------------------------------------------------------------------------
    def divergence(self) -> float:
        """The largest ``|div B|`` times the cell size (float64 from the stored ``A_z``)."""
        self._check_ready()
        largest = 0.0
        for patch in self._local():
            dx, dy = self.hierarchy.spacing(patch.level)
            az = self._read(patch, 6, node=True).to(torch.float64)
            bxf = (az[:, 1:] - az[:, :-1]) / dy + self.mean_field[0]
            byf = -(az[1:, :] - az[:-1, :]) / dx + self.mean_field[1]
            div = (bxf[1:] - bxf[:-1]) / dx + (byf[:, 1:] - byf[:, :-1]) / dy
            largest = max(largest, float(torch.max(torch.abs(div))) * min(dx, dy))
        from wellbalanced_b200.distributed import all_reduce

        return all_reduce(self, [largest], "max")[0]

    def composite_divergence(self) -> float:
        """The largest mismatch of shared coarse/fine ``A_z`` nodes relative to the largest face flux."""
        self._single_rank("composite_divergence")
        self._check_ready()
        h = self.hierarchy
        worst, scale = 0.0, 0.0
        for fine in h.patches:
            if fine.level == 0:
                continue
            fine_az = self._read(fine, 6, node=True).to(torch.float64).cpu().numpy()
            scale = max(scale, float(np.max(np.abs(np.diff(fine_az, axis=0)))), float(np.max(np.abs(np.diff(fine_az, axis=1)))))
            for coarse in h.patches_at_level(fine.level - 1):
                coarse_az = self._read(coarse, 6, node=True).to(torch.float64).cpu().numpy()
                (fx0, fx1), (fy0, fy1) = fine.box
                for i in range(fx0 // 2, fx1 // 2 + 1):
                    for j in range(fy0 // 2, fy1 // 2 + 1):
                        if not (i in (fx0 // 2, fx1 // 2) or j in (fy0 // 2, fy1 // 2)):
                            continue
                        ci, cj = i - coarse.box[0][0], j - coarse.box[1][0]
                        if not (0 <= ci < coarse_az.shape[0] and 0 <= cj < coarse_az.shape[1]):
                            continue
                        worst = max(worst, abs(coarse_az[ci, cj] - fine_az[2 * i - fx0, 2 * j - fy0]))
        return worst / scale if scale else 0.0

    def _covered(self, patch):
        return covered_cells(self.hierarchy, patch)

    def totals(self) -> dict[str, float]:
        """Integrals of the conserved fields over the domain from the leaf cells (float64)."""
        self._check_ready()
        out = dict.fromkeys(CONSERVED, 0.0)
        for patch in self._local():
            volume = float(np.prod(self.hierarchy.spacing(patch.level)))
            leaf = torch.from_numpy(~self._covered(patch)).to(self.engine.device)
            for f, name in enumerate(CONSERVED):
                values = self._read(patch, f).to(torch.float64)
                out[name] += float(torch.sum(values[leaf])) * volume
        from wellbalanced_b200.distributed import all_reduce

        return dict(zip(out, all_reduce(self, list(out.values()), "sum"), strict=True))

    def gather(self, patch, field: int, node=False) -> np.ndarray:
        return self._read(patch, field, node=node).to(torch.float64).cpu().numpy()

    def state(self) -> dict[str, np.ndarray]:
        """Level-0 conserved fields and ``A_z`` as float64 host arrays."""
        h = self.hierarchy
        nx, ny = h.level_shape(0)
        out = {name: np.full((nx, ny), np.nan) for name in CONSERVED}
        out["az"] = np.full((nx + 1, ny + 1), np.nan)
        for patch in h.patches_at_level(0):
            (i0, i1), (j0, j1) = patch.box
            for f, name in enumerate(CONSERVED):
                out[name][i0:i1, j0:j1] = self.gather(patch, f)
            out["az"][i0 : i1 + 1, j0 : j1 + 1] = self.gather(patch, 6, node=True)
        return out

    #: the variables of `leaf_values` besides the coordinates and the level
    LEAF_VARIABLES = ("density", "velocity_x", "velocity_y", "velocity_z", "pressure", "magnetic_field_x",
                      "magnetic_field_y", "magnetic_field_z", "current_z")

    def _leaf_block(self, patch) -> torch.Tensor:
        """(9, nx, ny) float64 on the device: the primitive variables of the patch's cells
        (mhd_primitive_pyccel.py:23-87) and J_z at the cell as the mean of its four corner
        nodes (carafe/mhd.py:1089-1096), from the haloed state."""
        state = self.engine.state
        nx, ny = patch.shape
        dx, dy = self.hierarchy.spacing(patch.level)
        view = [self.engine.view(state, patch, f).to(torch.float64) for f in range(7)]
        az = view[6]                                      # haloed nodes (nx + 5, ny + 5)
        bxf = (az[:, 1:] - az[:, :-1]) / dy + self.mean_field[0]   # [I, J]: node I of cell J
        byf = -(az[1:, :] - az[:-1, :]) / dx + self.mean_field[1]  # [I, J]: cell I, node J
        cells = (slice(HALO, HALO + nx), slice(HALO, HALO + ny))
        rho, mx, my, mz, energy, bz = (v[cells] for v in view[:6])
        bx = 0.5 * (bxf[HALO : HALO + nx, HALO : HALO + ny] + bxf[HALO + 1 : HALO + nx + 1, HALO : HALO + ny])
        by = 0.5 * (byf[HALO : HALO + nx, HALO : HALO + ny] + byf[HALO : HALO + nx, HALO + 1 : HALO + ny + 1])
        u, v, w = mx / rho, my / rho, mz / rho
        p = (self.gamma - 1.0) * (energy - 0.5 * rho * (u * u + v * v + w * w) - 0.5 * (bx * bx + by * by + bz * bz))
        # J_z at haloed nodes I, J in [1, n + 4): dB_y/dx - dB_x/dy
        jz = (byf[1:, 1:-1] - byf[:-1, 1:-1]) / dx - (bxf[1:-1, 1:] - bxf[1:-1, :-1]) / dy
        corner = torch.zeros_like(rho)
        for a in (0, 1):
            for b in (0, 1):
                corner = corner + jz[HALO - 1 + a : HALO - 1 + a + nx, HALO - 1 + b : HALO - 1 + b + ny]
        return torch.stack([rho, u, v, w, p, bx, by, bz, 0.25 * corner])

    def leaf_values(self) -> dict[str, np.ndarray]:
        """The primitive variables on the leaf cells of the hierarchy (carafe/mhd.py:1059-1111).

        One value per leaf cell (a cell no finer patch covers): ``x``, ``y`` (the centres),
        ``level``, the variables of `dataset` and ``current_z`` (the mean of the corners).
        The cells come patch by patch in the hierarchy's order, each patch's in row-major
        (x, y) order.
        """
        self._check_ready()
        h = self.hierarchy
        self.engine.fill(self.engine.state)
        parts: dict[str, list[np.ndarray]] = {name: [] for name in ("x", "y", "level", *self.LEAF_VARIABLES)}
        for patch in h.patches:
            leaf = ~self._covered(patch)
            block = self._leaf_block(patch)[:, torch.from_numpy(leaf).to(self.engine.device)].cpu().numpy()
            x, y = self._coordinates(patch, node=False)
            parts["x"].append(x[leaf])
            parts["y"].append(y[leaf])
            parts["level"].append(np.full(int(leaf.sum()), patch.level))
            for name, values in zip(self.LEAF_VARIABLES, block, strict=True):
                parts[name].append(values)
        return {name: np.concatenate(values) for name, values in parts.items()}

    def dataset(self, level: int = 0) -> Dataset:
        """The primitive variables of ``level`` over its cell centres (``mhd.py:1177-1226``)."""
        self._check_ready()
        h = self.hierarchy
        nx, ny = h.level_shape(level)
        dx, dy = h.spacing(level)
        x = h.lower_bound[0] + (np.arange(nx) + 0.5) * dx
        y = h.lower_bound[1] + (np.arange(ny) + 0.5) * dy
        fields = {name: np.full((nx, ny), np.nan) for name in (*CONSERVED, "bx", "by")}
        for patch in h.patches_at_level(level):
            (i0, i1), (j0, j1) = patch.box
            for f, name in enumerate(CONSERVED):
                fields[name][i0:i1, j0:j1] = self.gather(patch, f)
            bx, by = self._cell_field(patch, self.gather(patch, 6, node=True))
            fields["bx"][i0:i1, j0:j1] = bx
            fields["by"][i0:i1, j0:j1] = by
        rho = fields["density"]
        u = fields["momentum_x"] / rho
        v = fields["momentum_y"] / rho
        w = fields["momentum_z"] / rho
        b2 = fields["bx"] ** 2 + fields["by"] ** 2 + fields["bz"] ** 2
        p = (self.gamma - 1.0) * (fields["energy"] - 0.5 * rho * (u**2 + v**2 + w**2) - 0.5 * b2)
        dims = ("x", "y")
        data = {
            "density": Variable(dims, rho, r"$\rho$"),
            "velocity_x": Variable(dims, u, r"$u_x$"),
            "velocity_y": Variable(dims, v, r"$u_y$"),
            "velocity_z": Variable(dims, w, r"$u_z$"),
            "pressure": Variable(dims, p, r"$p$"),
            "magnetic_field_x": Variable(dims, fields["bx"], r"$B_x$"),
            "magnetic_field_y": Variable(dims, fields["by"], r"$B_y$"),
            "magnetic_field_z": Variable(dims, fields["bz"], r"$B_z$"),
            "magnetic_pressure": Variable(dims, 0.5 * b2, r"$|\mathbf{B}|^2/2$"),
        }
        coords = {"x": Variable("x", x, r"$x$"), "y": Variable("y", y, r"$y$")}
        return Dataset(data, coords=coords, attrs={"time": self.time, "level": level, "gamma": self.gamma})


def covered_cells(hierarchy, patch) -> np.ndarray:
    """The cells of a 2D patch that a patch of the next level covers (bool, patch shape)."""
    mask = np.zeros(patch.shape, dtype=bool)
    for fine in hierarchy.patches_at_level(patch.level + 1):
        idx = []
        for a in range(2):
            (flo, fhi), (lo, hi) = fine.box[a], patch.box[a]
            s, e = max(flo // 2, lo), min(fhi // 2, hi)
            if s >= e:
                break
            idx.append(slice(s - lo, e - lo))
        else:
            mask[tuple(idx)] = True
    return mask


def _locate(hierarchy, leaf, points):
    """The index in `leaf` of the leaf cell holding each point ((2, n) array): the finest
    level whose leaf cells contain it."""
    lower = np.asarray(hierarchy.lower_bound, dtype=float)
    owner = {}
    for level in range(hierarchy.max_level + 1):
        spacing = np.asarray(hierarchy.spacing(level))
        mine = leaf["level"] == level
        table = np.full(hierarchy.level_shape(level), -1, dtype=np.int64)
        i = np.floor((leaf["x"][mine] - lower[0]) / spacing[0]).astype(np.int64)
        j = np.floor((leaf["y"][mine] - lower[1]) / spacing[1]).astype(np.int64)
        table[i, j] = np.flatnonzero(mine)
        owner[level] = (table, spacing)
    found = np.full(points.shape[1], -1, dtype=np.int64)
    for level in range(hierarchy.max_level, -1, -1):
        table, spacing = owner[level]
        i = np.floor((points[0] - lower[0]) / spacing[0]).astype(np.int64)
        j = np.floor((points[1] - lower[1]) / spacing[1]).astype(np.int64)
        i = np.clip(i, 0, table.shape[0] - 1)
        j = np.clip(j, 0, table.shape[1] - 1)
        hit = table[i, j]
        found = np.where(found < 0, hit, found)
    if np.any(found < 0):
        raise ValueError("a point lies outside the leaf cells")
    return found


def sheet_diagnostics(model, leaf=None) -> dict:
    """The reconnected flux and the plasmoids of the lower sheet of `harris_sheets`
    (carafe/mhd.py:1291-1329).

    Along the line ``y = Ly / 4``: ``psi = (1/2) int |B_y| dx`` at the finest spacing,
    the O-points (B_y turning from positive to negative along x) and X-points, and the
    largest ``|J_z|``. ``leaf``: the `MHD2D.leaf_values` already computed.
    """
    mesh = model.hierarchy
    leaf = model.leaf_values() if leaf is None else leaf
    (x0, x1), (y0, y1) = mesh.bounds
    line = y0 + 0.25 * (y1 - y0)
    finest = mesh.spacing(mesh.max_level)[0]
    x = x0 + (np.arange(round((x1 - x0) / finest)) + 0.5) * finest
    below = _locate(mesh, leaf, np.array([x, np.full_like(x, line - 1e-9)]))
    above = _locate(mesh, leaf, np.array([x, np.full_like(x, line + 1e-9)]))
    by = 0.5 * (leaf["magnetic_field_y"][below] + leaf["magnetic_field_y"][above])
    psi = 0.5 * float(np.sum(np.abs(by)) * finest)
    sign = np.sign(by)
    turns = sign * np.roll(sign, -1) < 0
    return {
        "time": model.time,
        "psi": psi,
        "o_points": int(np.sum(turns & (sign > 0))),
        "x_points": int(np.sum(turns & (sign < 0))),
        "max_current": float(np.max(np.abs(leaf["current_z"]))),
        "leaf_cells": int(leaf["density"].size),
    }


def harris_sheets(hierarchy, *, width, beta=0.2, perturbation=1e-3, noise=0.0, seed=0):
    """Two Harris sheets in a periodic box: arguments of ``set_state`` (``mhd.py:1232-1288``)."""
    (x0, x1), (y0, y1) = hierarchy.bounds
    lx, ly = x1 - x0, y1 - y0
    first, second = y0 + 0.25 * ly, y0 + 0.75 * ly
    rng = np.random.default_rng(seed)
    modes = np.arange(2, 11)
    phases = rng.uniform(0.0, 2.0 * np.pi, (2, modes.size))
    amplitudes = noise * rng.standard_normal((2, modes.size)) / modes

    def potential(x, y):
        a = width * (np.log(np.cosh((y - first) / width)) - np.log(np.cosh((y - second) / width))) - (y - y0)
        for sheet, (centre, sign) in enumerate(((first, 1.0), (second, -1.0))):
            shape = np.exp(-(((y - centre) / (2.0 * width)) ** 2))
            wave = perturbation * np.cos(2.0 * np.pi * (x - x0) / lx)
            for mode, phase, amp in zip(modes, phases[sheet], amplitudes[sheet], strict=True):
                wave = wave + amp * np.cos(2.0 * np.pi * mode * (x - x0) / lx + phase)
            a = a + sign * wave * shape
        return a

    def pressure(x, y):
        bx = np.tanh((y - first) / width) - np.tanh((y - second) / width) - 1.0
        return 0.5 * (1.0 + beta) - 0.5 * bx * bx

    return {"density": 1.0, "velocity": (0.0, 0.0, 0.0), "pressure": pressure, "vector_potential": potential}
