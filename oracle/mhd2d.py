"""CPU float64 MHD2D step on an oracle hierarchy (test infrastructure only).

ORACLE — imported only by the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline leg. A restatement of the reference solver ``carafe.mhd.MHD2D``
(``src/carafe/mhd.py``): the same fields, halos, kernels and Heun step, on the patch
hierarchy of ``oracle.mesh``.

* constructor and validation — ``mhd.py:410-483``;
* test problems — ``mhd.py:486-671`` (Alfvén, Orszag–Tang, rotor, blast, RT);
* ``set_state`` — ``mhd.py:683-737``;
* halos and boundaries — ``mhd.py:298-353, 744-777``;
* ``_patch_fluxes`` / ``_advance`` — ``mhd.py:844-927``;
* ``stable_step`` / ``step`` / ``run`` — ``mhd.py:930-1008``;
* ``current_tags`` — ``mhd.py:1011-1041``;
* diagnostics — ``mhd.py:1114-1226``;
* ``harris_sheets`` — ``mhd.py:1232-1288``.
"""

from __future__ import annotations

from typing import Any

import numpy as np

from oracle import kernels as K
from oracle.mesh import FluxRegister, Hierarchy

HALO = 2
CONSERVED = ("density", "momentum_x", "momentum_y", "momentum_z", "energy", "bz")
_FLUX_ROWS = ((0, 1, 2, 3, 4, 6), (0, 2, 1, 3, 4, 6))
_WALL_ROWS = [0, 2, 3, 4, 6]


def outflow_cells(array, axis, lower, upper):
    """Zero-gradient halo cells along ``axis`` (``mhd.py:298-305``)."""
    h = HALO
    moved = np.moveaxis(array, axis, 0)
    if lower:
        moved[:h] = moved[h]
    if upper:
        moved[-h:] = moved[-h - 1]


def outflow_nodes(array, axis, lower, upper):
    """Halo nodes extrapolated linearly along ``axis`` (``mhd.py:308-324``)."""
    h = HALO
    moved = np.moveaxis(array, axis, 0)
    if lower:
        edge, inner = moved[h].copy(), moved[h + 1].copy()
        for k in range(1, h + 1):
            moved[h - k] = edge + k * (edge - inner)
    if upper:
        edge, inner = moved[-h - 1].copy(), moved[-h - 2].copy()
        for k in range(1, h + 1):
            moved[-h - 1 + k] = edge + k * (edge - inner)


def wall_cells(array, axis, lower, upper, sign=1.0):
    """Mirrored halo cells, ``sign`` -1 for the normal momentum (``mhd.py:327-338``)."""
    h = HALO
    moved = np.moveaxis(array, axis, 0)
    if lower:
        for k in range(h):
            moved[h - 1 - k] = sign * moved[h + k]
    if upper:
        n = moved.shape[0]
        for k in range(h):
            moved[n - h + k] = sign * moved[n - h - 1 - k]


def wall_nodes(array, axis, lower, upper):
    """Halo nodes odd about the wall node (``mhd.py:341-353``)."""
    h = HALO
    moved = np.moveaxis(array, axis, 0)
    if lower:
        wall = moved[h].copy()
        for k in range(1, h + 1):
            moved[h - k] = 2.0 * wall - moved[h + k]
    if upper:
        n = moved.shape[0]
        wall = moved[n - h - 1].copy()
        for k in range(1, h + 1):
            moved[n - h - 1 + k] = 2.0 * wall - moved[n - h - 1 - k]


class MHD2D:
    """Oracle MHD2D; same keyword arguments as the reference constructor."""

    def __init__(
        self,
        hierarchy: Hierarchy,
        *,
        gamma=5.0 / 3.0,
        mean_field=(0.0, 0.0),
        resistivity=0.0,
        limiter="vanleer",
        cfl=0.4,
        conduction=(0.0, 0.0),
        gravity=(0.0, 0.0),
        boundaries=None,
        prefix="mhd_",
    ):
        if hierarchy.ndim != 2:
            raise ValueError("MHD2D needs a 2D hierarchy")
        if limiter not in K.LIMITER_CODES:
            raise ValueError(f"limiter is one of {sorted(K.LIMITER_CODES)}")
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
            if axis_name not in kinds or kind not in ("outflow", "wall"):
                raise ValueError(f"boundaries maps 'x' or 'y' to outflow/wall, got {axis_name!r}")
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
        for name in CONSERVED:
            hierarchy.allocate_field(self.names[name], halo=HALO, conservative=True)
        hierarchy.allocate_field(self.potential, halo=HALO, centering="node")
        self.periodic = tuple(hierarchy.periodic)
        self.register = FluxRegister(hierarchy)
        self.time = 0.0
        self.steps = 0
        self.period = float("nan")
        self._ready = False

    # test problems -----------------------------------------------------------------------
    @classmethod
    def orszag_tang(cls, cells, split=None, **options):
        hierarchy = Hierarchy((cells, cells), ((0.0, 1.0), (0.0, 1.0)), (True, True), split)
        model = cls(hierarchy, **options)
        b0 = 1.0 / np.sqrt(4.0 * np.pi)
        model.set_state(
            25.0 / (36.0 * np.pi),
            lambda x, y: (-np.sin(2 * np.pi * y), np.sin(2 * np.pi * x), 0.0 * x),
            5.0 / (12.0 * np.pi),
            vector_potential=lambda x, y: b0
            * (np.cos(4 * np.pi * x) / (4 * np.pi) + np.cos(2 * np.pi * y) / (2 * np.pi)),
        )
        return model

    @classmethod
    def alfven_wave(cls, cells, *, amplitude=0.1, **options):
        hierarchy = Hierarchy((2 * cells, cells), ((0.0, 2.0), (0.0, 1.0)), (True, True))
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
    def rotor(cls, cells, **options):
        hierarchy = Hierarchy((cells, cells), ((0.0, 1.0), (0.0, 1.0)))
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
    def blast_wave(cls, cells, **options):
        hierarchy = Hierarchy(
            (cells, (3 * cells) // 2), ((-0.5, 0.5), (-0.75, 0.75)), (True, True)
        )
        field = 1.0 / np.sqrt(2.0)
        options = {"limiter": "minmod", **options}
        model = cls(hierarchy, mean_field=(field, field), **options)
        model.set_state(1.0, (0.0, 0.0, 0.0), lambda x, y: np.where(np.hypot(x, y) < 0.1, 10.0, 0.1))
        return model

    @classmethod
    def rayleigh_taylor(cls, cells, *, field=0.0, amplitude=0.01, **options):
        hierarchy = Hierarchy((cells, 3 * cells), ((-0.25, 0.25), (-0.75, 0.75)), (True, False))
        options = {"gamma": 1.4, **options}
        model = cls(
            hierarchy,
            mean_field=(field, 0.0),
            gravity=(0.0, -0.1),
            boundaries={"y": "wall"},
            **options,
        )

        def density(x, y):
            return np.where(y > 0.0, 2.0, 1.0)

        def velocity(x, y):
            vy = amplitude * (1 + np.cos(4 * np.pi * x)) * (1 + np.cos(3 * np.pi * y))
            return (0.0 * x, vy / 4.0, 0.0 * x)

        model.set_state(density, velocity, lambda x, y: 2.5 - 0.1 * density(x, y) * y)
        return model

    # state -------------------------------------------------------------------------------
    @staticmethod
    def _evaluate(value, x, y):
        if callable(value):
            return np.broadcast_to(np.asarray(value(x, y), dtype=float), x.shape)
        return np.broadcast_to(np.asarray(value, dtype=float), x.shape)

    def cell_field(self, patch, az):
        dx, dy = self.hierarchy.spacing(patch.level)
        bxf = (az[:, 1:] - az[:, :-1]) / dy + self.mean_field[0]
        byf = -(az[1:, :] - az[:-1, :]) / dx + self.mean_field[1]
        return 0.5 * (bxf[:-1] + bxf[1:]), 0.5 * (byf[:, :-1] + byf[:, 1:])

    def set_state(self, density, velocity, pressure, *, vector_potential=0.0, bz=0.0):
        hierarchy = self.hierarchy
        gamma = self.gamma
        for patch in hierarchy.patches:
            x, y = patch.coordinates(hierarchy, (0, 0))
            xn, yn = patch.coordinates(hierarchy, (1, 1))
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
            patch.field(self.potential).local[...] = az
            bx, by = self.cell_field(patch, az)
            bzv = self._evaluate(bz, x, y)
            values = {
                "density": rho,
                "momentum_x": rho * u,
                "momentum_y": rho * v,
                "momentum_z": rho * w,
                "energy": p / (gamma - 1.0)
                + 0.5 * rho * (u**2 + v**2 + w**2)
                + 0.5 * (bx**2 + by**2 + bzv**2),
                "bz": bzv,
            }
            for name, value in values.items():
                patch.field(self.names[name]).local[...] = value
        for name in self.names.values():
            hierarchy.restrict(name)
        hierarchy.restrict(self.potential)
        self.time = 0.0
        self.steps = 0
        self._ready = True

    def set_conserved(self, fields, az):
        """A one-patch level 0 from conserved cell arrays (rho, m_x, m_y, m_z, E, B_z) and
        nodal A_z (a test-side setter; the reference sets states through `set_state`)."""
        (patch,) = self.hierarchy.patches_at_level(0)
        for name, value in zip(CONSERVED, fields, strict=True):
            patch.field(self.names[name]).local[...] = value
        patch.field(self.potential).local[...] = az
        self.time = 0.0
        self.steps = 0
        self._ready = True

    def _check_ready(self):
        if not self._ready:
            raise RuntimeError("set the state first (set_state)")

    # halos -------------------------------------------------------------------------------
    def fill_halos(self):
        hierarchy = self.hierarchy
        names = [*self.names.values(), self.potential]
        coarse = {}
        for level in range(hierarchy.max_level + 1):
            for name in names:
                hierarchy.exchange_level(name, level, coarse.get(name))
            shape = hierarchy.level_shape(level)
            for patch in hierarchy.patches_at_level(level):
                for axis in range(2):
                    if self.periodic[axis]:
                        continue
                    lower = patch.box[axis][0] == 0
                    upper = patch.box[axis][1] == shape[axis]
                    if not (lower or upper):
                        continue
                    potential = patch.field(self.potential).local_with_halos
                    if not self.walls[axis]:
                        for name in self.names.values():
                            outflow_cells(patch.field(name).local_with_halos, axis, lower, upper)
                        outflow_nodes(potential, axis, lower, upper)
                        continue
                    normal = ("momentum_x", "momentum_y")[axis]
                    for key, name in self.names.items():
                        wall_cells(
                            patch.field(name).local_with_halos,
                            axis,
                            lower,
                            upper,
                            -1.0 if key == normal else 1.0,
                        )
                    wall_nodes(potential, axis, lower, upper)
            coarse = {name: hierarchy.padded(name, level) for name in names}

    # right-hand side ---------------------------------------------------------------------
    def primitive(self, patch):
        dx, dy = self.hierarchy.spacing(patch.level)
        nx, ny = patch.shape
        cells = (nx + 2 * HALO, ny + 2 * HALO)
        prim = np.empty((8, *cells))
        bxf = np.empty((cells[0] + 1, cells[1]))
        byf = np.empty((cells[0], cells[1] + 1))
        ecc = np.empty(cells)
        bad = K.mhd_primitive(
            *(patch.field(self.names[name]).local_with_halos for name in CONSERVED),
            patch.field(self.potential).local_with_halos,
            dx,
            dy,
            *self.mean_field,
            self.gamma,
            prim,
            bxf,
            byf,
            ecc,
        )
        return prim, bxf, byf, ecc, bad

    def current(self, bxf, byf, level):
        dx, dy = self.hierarchy.spacing(level)
        return (byf[1:, 1:-1] - byf[:-1, 1:-1]) / dx - (bxf[1:-1, 1:] - bxf[1:-1, :-1]) / dy

    def wall_sides(self, patch):
        shape = self.hierarchy.level_shape(patch.level)
        return tuple(
            (
                self.walls[axis] and patch.box[axis][0] == 0,
                self.walls[axis] and patch.box[axis][1] == shape[axis],
            )
            for axis in range(2)
        )

    def patch_fluxes(self, patch):
        prim, bxf, byf, ecc, bad = self.primitive(patch)
        if bad:
            raise FloatingPointError(
                f"non-positive density or pressure on the level-{patch.level} patch "
                f"{patch.box} at t = {self.time}"
            )
        nx, ny = patch.shape
        cells = (nx + 2 * HALO, ny + 2 * HALO)
        fx = np.empty((7, cells[0] - 3, cells[1]))
        fy = np.empty((7, cells[0], cells[1] - 3))
        ez = np.empty((nx + 1, ny + 1))
        code = K.LIMITER_CODES.index(self.limiter)
        K.mhd_sweep(prim, bxf, 0, code, self.gamma, fx)
        K.mhd_sweep(prim, byf, 1, code, self.gamma, fy)
        K.ct_contact(fx[5], fy[5], fx[0], fy[0], ecc, ez)
        dx, dy = self.hierarchy.spacing(patch.level)
        if max(self.conduction) > 0.0:
            K.mhd_conductive(prim, bxf, byf, dx, dy, *self.conduction, fx, fy)
        if self.resistivity:
            K.mhd_resistive(prim, bxf, byf, dx, dy, self.resistivity, fx, fy, ez)
        (left, right), (bottom, top) = self.wall_sides(patch)
        if left:
            ez[0, :] = 0.0
            fx[_WALL_ROWS, 0, :] = 0.0
        if right:
            ez[-1, :] = 0.0
            fx[_WALL_ROWS, -1, :] = 0.0
        if bottom:
            ez[:, 0] = 0.0
            fy[_WALL_ROWS, :, 0] = 0.0
        if top:
            ez[:, -1] = 0.0
            fy[_WALL_ROWS, :, -1] = 0.0
        return fx, fy, ez

    def advance(self, dt, scale):
        hierarchy = self.hierarchy
        self.fill_halos()
        fluxes = {id(p): self.patch_fluxes(p) for p in hierarchy.patches}
        gx, gy = self.gravity
        sources = {}
        if gx or gy:
            for patch in hierarchy.patches:
                rho = patch.field(self.names["density"]).local.copy()
                mx = patch.field(self.names["momentum_x"]).local
                my = patch.field(self.names["momentum_y"]).local
                sources[id(patch)] = (rho * gx, rho * gy, (mx * gx + my * gy).copy())
        h = HALO

        def block(patch, x_row, y_row):
            nx, ny = patch.shape
            fx, fy, _ = fluxes[id(patch)]
            return fx[x_row, :, h : h + ny], fy[y_row, h : h + nx, :]

        for name, x_row, y_row in zip(CONSERVED, *_FLUX_ROWS, strict=True):
            self.register.update(
                self.names[name],
                lambda patch, x_row=x_row, y_row=y_row: block(patch, x_row, y_row),
                dt,
                scale=scale,
            )
        for patch in hierarchy.patches:
            potential = patch.field(self.potential).local
            potential -= dt * fluxes[id(patch)][2]
            if gx or gy:
                force_x, force_y, work = sources[id(patch)]
                patch.field(self.names["momentum_x"]).local[...] += dt * force_x
                patch.field(self.names["momentum_y"]).local[...] += dt * force_y
                patch.field(self.names["energy"]).local[...] += dt * work

    # time stepping -----------------------------------------------------------------------
    def stable_step(self):
        self._check_ready()
        hierarchy = self.hierarchy
        smallest = np.inf
        out = np.empty(2)
        for patch in hierarchy.patches:
            dx, dy = hierarchy.spacing(patch.level)
            K.mhd_rate(
                *(patch.field(self.names[name]).local_with_halos for name in CONSERVED),
                patch.field(self.potential).local_with_halos,
                HALO,
                dx,
                dy,
                *self.mean_field,
                self.gamma,
                out,
            )
            smallest = min(smallest, 1.0 / out[0])
            diffusivity = max(
                self.resistivity, (self.gamma - 1.0) * max(self.conduction) / float(out[1])
            )
            if diffusivity > 0.0:
                smallest = min(smallest, 0.5 / (diffusivity * (dx**-2 + dy**-2)))
        return self.cfl * float(smallest)

    def step(self, dt=None):
        self._check_ready()
        if dt is None:
            dt = self.stable_step()
        hierarchy = self.hierarchy
        names = [*self.names.values(), self.potential]
        start = {
            (id(p), n): np.array(p.field(n).local) for p in hierarchy.patches for n in names
        }
        self.advance(dt, 0.5 * dt)
        hierarchy.restrict(self.potential)
        self.advance(dt, 0.5 * dt)
        for patch in hierarchy.patches:
            for name in names:
                array = patch.field(name).local
                array += start[id(patch), name]
                array *= 0.5
        for name in self.names.values():
            self.register.reflux(name)
        hierarchy.restrict(self.potential)
        self.time += dt
        self.steps += 1
        return dt

    def run(self, duration, *, max_steps=1_000_000):
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

    # refinement --------------------------------------------------------------------------
    def current_tags(self, threshold, levels):
        self._check_ready()
        hierarchy = self.hierarchy
        self.fill_halos()
        h = HALO
        tags = {
            level: np.zeros(hierarchy.level_shape(level), dtype=bool)
            for level in range(min(levels, hierarchy.max_level + 1))
        }
        for patch in hierarchy.patches:
            if patch.level not in tags:
                continue
            nx, ny = patch.shape
            dx, dy = hierarchy.spacing(patch.level)
            _, bxf, byf, _, _ = self.primitive(patch)
            jz = np.abs(self.current(bxf, byf, patch.level))
            cell = 0.25 * sum(
                jz[h - 1 + a : h - 1 + a + nx, h - 1 + b : h - 1 + b + ny]
                for a in (0, 1)
                for b in (0, 1)
            )
            (i0, i1), (j0, j1) = patch.box
            tags[patch.level][i0:i1, j0:j1] |= cell * max(dx, dy) > threshold
        return tags

    # diagnostics -------------------------------------------------------------------------
    def divergence(self):
        largest = 0.0
        for patch in self.hierarchy.patches:
            dx, dy = self.hierarchy.spacing(patch.level)
            az = patch.field(self.potential).local
            bxf = (az[:, 1:] - az[:, :-1]) / dy + self.mean_field[0]
            byf = -(az[1:, :] - az[:-1, :]) / dx + self.mean_field[1]
            div = (bxf[1:] - bxf[:-1]) / dx + (byf[:, 1:] - byf[:, :-1]) / dy
            largest = max(largest, float(np.max(np.abs(div))) * min(dx, dy))
        return largest

    def totals(self):
        return {name: self.hierarchy.integral(self.names[name]) for name in CONSERVED}

    def dataset(self, level=0):
        """Primitive variables of ``level`` as a dict of ``(nx, ny)`` arrays (NaN if absent)."""
        hierarchy = self.hierarchy
        nx, ny = hierarchy.level_shape(level)
        fields = {name: np.full((nx, ny), np.nan) for name in (*CONSERVED, "bx", "by")}
        for patch in hierarchy.patches_at_level(level):
            (i0, i1), (j0, j1) = patch.box
            for name in CONSERVED:
                fields[name][i0:i1, j0:j1] = patch.field(self.names[name]).local
            bx, by = self.cell_field(patch, np.array(patch.field(self.potential).local))
            fields["bx"][i0:i1, j0:j1] = bx
            fields["by"][i0:i1, j0:j1] = by
        rho = fields["density"]
        u = fields["momentum_x"] / rho
        v = fields["momentum_y"] / rho
        w = fields["momentum_z"] / rho
        b2 = fields["bx"] ** 2 + fields["by"] ** 2 + fields["bz"] ** 2
        p = (self.gamma - 1.0) * (fields["energy"] - 0.5 * rho * (u**2 + v**2 + w**2) - 0.5 * b2)
        return {
            "density": rho,
            "velocity_x": u,
            "velocity_y": v,
            "velocity_z": w,
            "pressure": p,
            "magnetic_field_x": fields["bx"],
            "magnetic_field_y": fields["by"],
            "magnetic_field_z": fields["bz"],
            "magnetic_pressure": 0.5 * b2,
            "energy": fields["energy"],
        }

    def state(self) -> dict[str, Any]:
        """The level-0 conserved fields and ``A_z`` (one patch per level assumed)."""
        hierarchy = self.hierarchy
        nx, ny = hierarchy.level_shape(0)
        out = {name: np.full((nx, ny), np.nan) for name in CONSERVED}
        out["az"] = np.full((nx + 1, ny + 1), np.nan)
        for patch in hierarchy.patches_at_level(0):
            (i0, i1), (j0, j1) = patch.box
            for name in CONSERVED:
                out[name][i0:i1, j0:j1] = patch.field(self.names[name]).local
            out["az"][i0 : i1 + 1, j0 : j1 + 1] = patch.field(self.potential).local
        return out


def harris_sheets(hierarchy, *, width, beta=0.2, perturbation=1e-3, noise=0.0, seed=0):
    """Arguments of ``set_state`` for two Harris sheets (``mhd.py:1232-1288``)."""
    (x0, x1), (y0, y1) = hierarchy.bounds
    lx, ly = x1 - x0, y1 - y0
    first, second = y0 + 0.25 * ly, y0 + 0.75 * ly
    rng = np.random.default_rng(seed)
    modes = np.arange(2, 11)
    phases = rng.uniform(0.0, 2.0 * np.pi, (2, modes.size))
    amplitudes = noise * rng.standard_normal((2, modes.size)) / modes

    def potential(x, y):
        a = width * (
            np.log(np.cosh((y - first) / width)) - np.log(np.cosh((y - second) / width))
        ) - (y - y0)
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

    return {
        "density": 1.0,
        "velocity": (0.0, 0.0, 0.0),
        "pressure": pressure,
        "vector_potential": potential,
    }
