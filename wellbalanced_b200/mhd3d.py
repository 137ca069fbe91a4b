r"""MHD in three dimensions on the device: the drop-in for ``carafe.mhd3d.MHD3D``.

Same constructor keywords, test problems and methods as the reference
(``src/carafe/mhd3d.py:182-965``). The state (density, momentum, energy on the cells;
the vector potential on the edges) lives in device pools; a step is the fused 3D stage
kernel of ``libwb200.so`` (``wb_stage3d``: primitives, MUSCL + HLLD along the three
axes, CT-contact edge fields, cell and edge updates in one pass per stage) with the halo
and restriction op lists. ``precision`` 64 (the reference's arithmetic), 32, or "mixed"
(float32 reconstruction, HLLD and CT on a float64 state).
"""

from __future__ import annotations

from typing import Any

import numpy as np
import torch

from wellbalanced_b200 import _lib

from wellbalanced_b200.dataset import Dataset, Variable
from wellbalanced_b200.engine import Engine
from wellbalanced_b200.mesh import HALO, AMRHierarchy
from wellbalanced_b200.mhd import LIMITER_CODES

__all__ = ["CONSERVED_3D", "MHD3D"]

CONSERVED_3D = ("density", "momentum_x", "momentum_y", "momentum_z", "energy")
_EXTRA = ((0, 1, 1), (1, 0, 1), (1, 1, 0))  # node axes of the x-, y-, z-edge potentials


def _cyclic(axis):
    return axis, (axis + 1) % 3, (axis + 2) % 3


class MHD3D:
    """3D ideal MHD on the device (see the module docstring)."""

    def __init__(
        self,
        hierarchy: AMRHierarchy,
        *,
        gamma: float = 5.0 / 3.0,
        mean_field: tuple[float, float, float] = (0.0, 0.0, 0.0),
        resistivity: float = 0.0,
        limiter: str = "vanleer",
        cfl: float = 0.3,
        gravity: tuple[float, float, float] = (0.0, 0.0, 0.0),
        prefix: str = "mhd_",
        precision: int | str = 64,
        device: str = "cuda",
        lx: int | str = 32,
    ) -> None:
        if hierarchy.ndim != 3:
            raise ValueError("MHD3D needs a 3D hierarchy")
        if hierarchy.cylindrical or hierarchy.graded:
            raise NotImplementedError("MHD3D is Cartesian on uniform levels: no graded axes")
        if limiter not in LIMITER_CODES:
            raise ValueError(f"limiter is one of {sorted(LIMITER_CODES)}")
        if not 0.0 < cfl <= 1.0:
            raise ValueError("cfl must be in (0, 1]")
        if gamma <= 1.0:
            raise ValueError("gamma must be larger than 1")
        if not resistivity >= 0.0:
            raise ValueError("resistivity must be non-negative")
        if len(mean_field) != 3 or len(gravity) != 3:
            raise ValueError("mean_field and gravity have three components")
        self.hierarchy = hierarchy
        self.gamma = float(gamma)
        self.mean_field = tuple(float(b) for b in mean_field)
        self.resistivity = float(resistivity)
        self.limiter = limiter
        self.cfl = float(cfl)
        self.gravity = tuple(float(g) for g in gravity)
        self.names = {name: prefix + name for name in CONSERVED_3D}
        self.potential = tuple(prefix + name for name in ("ax", "ay", "az"))
        self.periodic = tuple(hierarchy.periodic)
        self.precision = _lib.precision_code(precision)
        self.device = device
        # x-planes per tile of the stage kernel; "auto": tuned when the state is first set
        self._auto_lx = lx == "auto"
        self.lx = 32 if self._auto_lx else int(lx)
        self.lx_timings = None
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

    #: whether steps run the fused stage kernel (False: the per-kernel float64 path)
    _fused = True

    def _build_engine(self):
        self._graph = None
        options = dict(precision=self.precision, limiter=LIMITER_CODES.index(self.limiter), gamma=self.gamma,
                       mean_field=self.mean_field, device=self.device)
        from wellbalanced_b200.distributed import solver_engine, solver_group

        # a hierarchy over several ranks (AMRHierarchy(..., comm=group)): this rank's patches
        self._group = solver_group(self.hierarchy)
        if self._group is not None:
            self.engine = solver_engine(self.hierarchy, self._group, lx=self.lx, **options)
        else:
            self.engine = Engine(self.hierarchy, lx=self.lx, **options)
        groups = self.engine.layout.groups
        self._groups_all = groups
        self._groups_potential = groups[1:]
        physics = (self.resistivity, *self.gravity)
        if any(physics):
            self.engine.physics = tuple(float(v) for v in physics)

    # test problems (carafe/mhd3d.py:236-346) -----------------------------------------------------
    @classmethod
    def orszag_tang(cls, cells: int, layers: int = 4, **options: Any) -> MHD3D:
        hierarchy = AMRHierarchy(
            (cells, cells, layers), ((0.0, 1.0), (0.0, 1.0), (0.0, layers / cells)), periodic=(True, True, True)
        )
        model = cls(hierarchy, **options)
        b0 = 1.0 / np.sqrt(4.0 * np.pi)
        model.set_state(
            25.0 / (36.0 * np.pi),
            lambda x, y, z: (-np.sin(2 * np.pi * y), np.sin(2 * np.pi * x), 0.0 * x),
            5.0 / (12.0 * np.pi),
            vector_potential=(
                0.0,
                0.0,
                lambda x, y, z: b0 * (np.cos(4 * np.pi * x) / (4 * np.pi) + np.cos(2 * np.pi * y) / (2 * np.pi)),
            ),
        )
        return model

    @classmethod
    def alfven_wave(cls, cells: int, *, amplitude: float = 0.1, **options: Any):
        hierarchy = AMRHierarchy(
            (2 * cells, cells, cells), ((0.0, 2.0), (0.0, 1.0), (0.0, 1.0)), periodic=(True, True, True)
        )
        wavevector = 2.0 * np.pi * np.array([0.5, 1.0, 1.0])
        k = float(np.linalg.norm(wavevector))
        n = wavevector / k
        e1 = np.cross(n, [0.0, 0.0, 1.0])
        e1 /= np.linalg.norm(e1)
        e2 = np.cross(n, e1)

        def perpendicular(x, y, z):
            phase = wavevector[0] * x + wavevector[1] * y + wavevector[2] * z
            s, c = np.sin(phase), np.cos(phase)
            return [amplitude * (s * e1[i] + c * e2[i]) for i in range(3)]

        def potential(i):
            return lambda x, y, z: perpendicular(x, y, z)[i] / k

        model = cls(hierarchy, mean_field=tuple(n), **options)
        model.set_state(
            1.0,
            lambda x, y, z: [-b for b in perpendicular(x, y, z)],
            0.1,
            vector_potential=(potential(0), potential(1), potential(2)),
        )
        model.period = 2.0 / 3.0
        return model, model.dataset()

    @classmethod
    def blast_wave(cls, cells: int, **options: Any) -> MHD3D:
        hierarchy = AMRHierarchy(
            (cells, cells, (3 * cells) // 2), ((-0.5, 0.5), (-0.5, 0.5), (-0.75, 0.75)), periodic=(True, True, True)
        )
        field = 1.0 / np.sqrt(3.0)
        options = {"limiter": "minmod", **options}
        model = cls(hierarchy, mean_field=(field, field, field), **options)
        model.set_state(1.0, (0.0, 0.0, 0.0), lambda x, y, z: np.where(x**2 + y**2 + z**2 < 0.01, 10.0, 0.1))
        return model

    @classmethod
    def turbulence(cls, cells: int, *, seed: int = 0, **options: Any) -> MHD3D:
        """Decaying turbulence on the periodic unit cube (`wellbalanced_b200.problems.turbulence_3d`)."""
        from wellbalanced_b200.problems import turbulence_3d

        hierarchy = AMRHierarchy((cells,) * 3, ((0.0, 1.0),) * 3, periodic=(True, True, True))
        options = {"limiter": "mc", "cfl": 0.3, **options}
        model = cls(hierarchy, **options)
        rho, velocity, p, potential = turbulence_3d(cells, seed=seed, gamma=model.gamma)
        model.set_state(rho, velocity, p, vector_potential=potential)
        return model

    # state ---------------------------------------------------------------------------------------
    @staticmethod
    def _evaluate(value, *coordinates):
        shape = coordinates[0].shape
        if callable(value):
            return np.broadcast_to(np.asarray(value(*coordinates), dtype=float), shape)
        return np.broadcast_to(np.asarray(value, dtype=float), shape)

    def _coordinates(self, patch, extra):
        h = self.hierarchy
        dx = h.spacing(patch.level)
        axes = []
        for a, (lo, hi) in enumerate(patch.box):
            start = h.lower_bound[a]
            if extra[a]:
                axes.append(start + np.arange(lo, hi + 1) * dx[a])
            else:
                axes.append(start + (np.arange(lo, hi) + 0.5) * dx[a])
        return np.meshgrid(*axes, indexing="ij")

    def _face_fields(self, potential, spacing):
        faces = []
        for a in range(3):
            _, b, c = _cyclic(a)
            faces.append(
                np.diff(potential[c], axis=b) / spacing[b] - np.diff(potential[b], axis=c) / spacing[c] + self.mean_field[a]
            )
        return faces

    @staticmethod
    def _cell_fields(faces):
        out = []
        for a, f in enumerate(faces):
            n = f.shape[a]
            out.append(0.5 * (np.take(f, np.arange(0, n - 1), axis=a) + np.take(f, np.arange(1, n), axis=a)))
        return out

    def _slices(self, patch, extra):
        return tuple(slice(HALO, HALO + n + e) for n, e in zip(patch.shape, extra, strict=True))

    def _write(self, patch, field, values, extra=(0, 0, 0)):
        self.engine.dt_ready = False
        view = self.engine.view(self.engine.state, patch, field)
        view[self._slices(patch, extra)] = torch.from_numpy(np.require(values, requirements=("C", "W"))).to(view.device, view.dtype)

    def _read(self, patch, field, extra=(0, 0, 0), pool=None):
        pool = self.engine.state if pool is None else pool
        return self.engine.view(pool, patch, field)[self._slices(patch, extra)]

    def set_state(self, density, velocity, pressure, *, vector_potential=(0.0, 0.0, 0.0)) -> None:
        """Set the state on every patch (``carafe/mhd3d.py:388-441``)."""
        gamma = self.gamma
        h = self.hierarchy
        for patch in self._local():
            x, y, z = self._coordinates(patch, (0, 0, 0))
            rho = self._evaluate(density, x, y, z)
            if callable(velocity):
                u, v, w = (np.broadcast_to(c, x.shape) for c in velocity(x, y, z))
            elif isinstance(velocity, tuple | list) and len(velocity) == 3:
                u, v, w = (self._evaluate(c, x, y, z) for c in velocity)
            else:
                raise ValueError("velocity is a function or three values")
            p = self._evaluate(pressure, x, y, z)
            if np.any(rho <= 0.0) or np.any(p <= 0.0):
                raise ValueError("the density and the pressure must be positive")
            potential = []
            for c, value in enumerate(vector_potential):
                extra = _EXTRA[c]
                at = self._coordinates(patch, extra)
                shape = tuple(n + e for n, e in zip(patch.shape, extra, strict=True))
                if isinstance(value, np.ndarray) and value.shape == shape:
                    array = np.asarray(value, dtype=float)
                else:
                    array = np.array(self._evaluate(value, *at))
                potential.append(array)
                self._write(patch, 5 + c, array, extra)
            bx, by, bz = self._cell_fields(self._face_fields(tuple(potential), h.spacing(patch.level)))
            energy = p / (gamma - 1.0) + 0.5 * rho * (u**2 + v**2 + w**2) + 0.5 * (bx**2 + by**2 + bz**2)
            for f, value in enumerate((rho, rho * u, rho * v, rho * w, energy)):
                self._write(patch, f, value)
        self._after_state()

    def set_conserved(self, fields, potential) -> None:
        """Set a one-patch level 0 from conserved arrays and edge potentials."""
        (patch,) = self.hierarchy.patches_at_level(0)
        for f, value in enumerate(fields):
            self._write(patch, f, np.asarray(value, dtype=float))
        for c, value in enumerate(potential):
            self._write(patch, 5 + c, np.asarray(value, dtype=float), _EXTRA[c])
        self._after_state()

    def _after_state(self, tune=True):
        """The halos and the restriction of a new state; with `tune`, the autotuner's x-plane
        count (a regrid keeps the count tuned before it: `tune` False)."""
        self.engine.dt_ready = False
        eng = self.engine
        if self.hierarchy.max_level > 0:
            eng.restrict(eng.state, self._groups_all)
        eng.fill(eng.state)
        if tune and self._auto_lx:
            from wellbalanced_b200.autotune import tune_lx

            self.lx, timings = tune_lx(eng)
            self.lx_timings = timings or self.lx_timings
        self.time = 0.0
        self.steps = 0
        eng.time.zero_()
        self._ready = True

    def _check_ready(self):
        if not self._ready:
            raise RuntimeError("set the state first (set_state)")

    # time stepping -------------------------------------------------------------------------------
    def stable_step(self) -> float:
        self._check_ready()
        eng = self.engine
        eng.rate()
        eng.finalize_dt(self.cfl, self.resistivity, 0.0)
        return float(eng.dt[0].item())

    def _raise_if_bad(self):
        if self.engine.use_programs and self.engine.program_error():
            raise RuntimeError("an op program's phase wait ran out (its device error word is set)")
        if int(self.engine.bad.item()):
            raise FloatingPointError(f"non-positive density or pressure (or non-finite values) at t = {self.time}")

    def step(self, dt: float | None = None) -> float:
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
            eng.programmed_step(self._groups_potential, self._groups_all, self.cfl, self.resistivity, 0.0)
            return
        with eng.launching():
            eng.rate()
            eng.finalize_dt(self.cfl, self.resistivity, 0.0, advance=True)
            eng.heun_step(self._groups_potential, self._groups_all)

    def _prime(self):
        if self.engine.use_programs and not self.engine.dt_ready:
            self.engine.prime_dt(self.cfl, self.resistivity, 0.0)

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
        """``steps`` steps at the stable dt with no host synchronisation."""
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

    # raw device state (checkpoint / host buffers) ------------------------------------------------
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
        """Tag cells where ``|J|`` (central differences of the cell field) times the cell
        size exceeds ``threshold`` (``carafe/mhd3d.py:771-801``): one kernel over every
        cell of the tagged levels (``wb_current_tags``)."""
        self._single_rank("current_tags")
        from wellbalanced_b200.regrid import device_tags

        return device_tags(self, threshold, levels)

    def regrid(self, tags: dict[int, np.ndarray], **options: Any) -> None:
        """Regrid on ``tags`` (``carafe/mhd3d.py:803-816``); the potential is interpolated and
        restricted, so the field stays divergence-free."""
        self._single_rank("regrid")
        from wellbalanced_b200.regrid import regrid_model

        regrid_model(self, tags, **options)

    def _field_extras(self):
        return [(0, 0, 0)] * 5 + list(_EXTRA)

    def _gather_field(self, patch, f):
        return self.gather(patch, f)

    def _write_field(self, patch, f, values):
        extra = (0, 0, 0) if f < 5 else _EXTRA[f - 5]
        self._write(patch, f, values, extra)

    # diagnostics ---------------------------------------------------------------------------------
    def _potentials(self, patch):
        return tuple(self._read(patch, 5 + c, _EXTRA[c]).to(torch.float64) for c in range(3))

    def divergence(self) -> float:
        self._check_ready()
        largest = 0.0
        for patch in self._local():
            spacing = self.hierarchy.spacing(patch.level)
            pot = self._potentials(patch)
            div = 0.0
            for a in range(3):
                _, b, c = _cyclic(a)
                face = torch.diff(pot[c], dim=b) / spacing[b] - torch.diff(pot[b], dim=c) / spacing[c] + self.mean_field[a]
                div = div + torch.diff(face, dim=a) / spacing[a]
            largest = max(largest, float(torch.max(torch.abs(div))) * min(spacing))
        from wellbalanced_b200.distributed import all_reduce

        return all_reduce(self, [largest], "max")[0]

    def _covered(self, patch):
        mask = np.zeros(patch.shape, dtype=bool)
        for fine in self.hierarchy.patches_at_level(patch.level + 1):
            idx = []
            for a in range(3):
                (flo, fhi), (lo, hi) = fine.box[a], patch.box[a]
                s, e = max(flo // 2, lo), min(fhi // 2, hi)
                if s >= e:
                    break
                idx.append(slice(s - lo, e - lo))
            else:
                mask[tuple(idx)] = True
        return mask

    def totals(self) -> dict[str, float]:
        """Integrals of the conserved fields from the leaf cells (float64)."""
        self._check_ready()
        out = dict.fromkeys(CONSERVED_3D, 0.0)
        for patch in self._local():
            volume = float(np.prod(self.hierarchy.spacing(patch.level)))
            leaf = torch.from_numpy(~self._covered(patch)).to(self.engine.device)
            for f, name in enumerate(CONSERVED_3D):
                out[name] += float(torch.sum(self._read(patch, f).to(torch.float64)[leaf])) * volume
        from wellbalanced_b200.distributed import all_reduce

        return dict(zip(out, all_reduce(self, list(out.values()), "sum"), strict=True))

    def gather(self, patch, field):
        extra = (0, 0, 0) if field < 5 else _EXTRA[field - 5]
        return self._read(patch, field, extra).to(torch.float64).cpu().numpy()

    def state(self) -> dict[str, np.ndarray]:
        (patch,) = self.hierarchy.patches_at_level(0)
        out = {name: self._read(patch, f).to(torch.float64).cpu().numpy() for f, name in enumerate(CONSERVED_3D)}
        for c, key in enumerate(("ax", "ay", "az")):
            out[key] = self._read(patch, 5 + c, _EXTRA[c]).to(torch.float64).cpu().numpy()
        return out

    def dataset(self, level: int = 0) -> Dataset:
        self._check_ready()
        h = self.hierarchy
        shape = h.level_shape(level)
        spacing = h.spacing(level)
        axes = [h.lower_bound[a] + (np.arange(shape[a]) + 0.5) * spacing[a] for a in range(3)]
        names = (*CONSERVED_3D, "bx", "by", "bz")
        fields = {name: np.full(shape, np.nan) for name in names}
        for patch in h.patches_at_level(level):
            index = tuple(slice(lo, hi) for lo, hi in patch.box)
            for f, name in enumerate(CONSERVED_3D):
                fields[name][index] = self._read(patch, f).to(torch.float64).cpu().numpy()
            pot = tuple(p.cpu().numpy() for p in self._potentials(patch))
            for name, value in zip(("bx", "by", "bz"), self._cell_fields(self._face_fields(pot, spacing)), strict=True):
                fields[name][index] = value
        rho = fields["density"]
        u, v, w = (fields[f"momentum_{a}"] / rho for a in "xyz")
        b2 = fields["bx"] ** 2 + fields["by"] ** 2 + fields["bz"] ** 2
        p = (self.gamma - 1.0) * (fields["energy"] - 0.5 * rho * (u**2 + v**2 + w**2) - 0.5 * b2)
        dims = ("x", "y", "z")
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
        coords = {name: Variable(name, values, f"${name}$") for name, values in zip(dims, axes, strict=True)}
        return Dataset(data, coords=coords, attrs={"time": self.time, "level": level, "gamma": self.gamma})
