"""CPU float64 MHD3D step on an oracle hierarchy (test infrastructure only).

ORACLE — imported only by the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline leg. A restatement of the reference solver ``carafe.mhd3d.MHD3D``
(``src/carafe/mhd3d.py``), vectorised over whole blocks:

* face and cell fields from the edge potential — ``mhd3d.py:361-386``;
* primitive variables and their check — ``mhd3d.py:475-509``;
* sweeps along each axis in the cyclic frame — ``mhd3d.py:511-528``;
* the CT-contact edge field on every plane — ``mhd3d.py:530-559``;
* resistive edge field and energy flux — ``mhd3d.py:561-602``;
* ``_patch_fluxes`` / ``_advance`` / ``stable_step`` / ``step`` — ``mhd3d.py:604-754``;
* test problems — ``mhd3d.py:236-346``.

Also the seeded decaying-turbulence initial state (k^-2 Gaussian random fields) of the
3D turbulence workload, shared by the tests and the benchmark.
"""

from __future__ import annotations

import numpy as np

from oracle import kernels as K
from oracle.mesh import FluxRegister, Hierarchy
from oracle.mhd2d import HALO, outflow_cells, outflow_nodes

CONSERVED_3D = ("density", "momentum_x", "momentum_y", "momentum_z", "energy")
_POTENTIAL = (("ax", "x-edge"), ("ay", "y-edge"), ("az", "z-edge"))


def cyclic(axis):
    return axis, (axis + 1) % 3, (axis + 2) % 3


def along(array, axis, start, stop):
    index = [slice(None)] * array.ndim
    index[axis] = slice(start, stop)
    return array[tuple(index)]


def pair_mean(array, axis, start, count):
    return 0.5 * (along(array, axis, start, start + count) + along(array, axis, start + 1, start + 1 + count))


def field_at_face(face, normal, node, shape):
    h = HALO
    face = pair_mean(face, normal, h - 1, shape[normal] + 1)
    face = pair_mean(face, node, h, shape[node])
    other = 3 - normal - node
    return along(face, other, h, h + shape[other])


class MHD3D:
    """Oracle MHD3D; same keyword arguments as the reference constructor."""

    def __init__(
        self,
        hierarchy: Hierarchy,
        *,
        gamma=5.0 / 3.0,
        mean_field=(0.0, 0.0, 0.0),
        resistivity=0.0,
        limiter="vanleer",
        cfl=0.3,
        gravity=(0.0, 0.0, 0.0),
        prefix="mhd_",
    ):
        if hierarchy.ndim != 3:
            raise ValueError("MHD3D needs a 3D hierarchy")
        if limiter not in K.LIMITER_CODES:
            raise ValueError(f"limiter is one of {sorted(K.LIMITER_CODES)}")
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
        self.potential = tuple(prefix + name for name, _ in _POTENTIAL)
        for name in CONSERVED_3D:
            hierarchy.allocate_field(self.names[name], halo=HALO, conservative=True)
        for name, (_, centering) in zip(self.potential, _POTENTIAL, strict=True):
            hierarchy.allocate_field(name, halo=HALO, centering=centering)
        self.periodic = tuple(hierarchy.periodic)
        self.register = FluxRegister(hierarchy)
        self.time = 0.0
        self.steps = 0
        self.period = float("nan")
        self._ready = False

    # test problems -----------------------------------------------------------------------
    @classmethod
    def orszag_tang(cls, cells, layers=4, **options):
        hierarchy = Hierarchy(
            (cells, cells, layers), ((0.0, 1.0), (0.0, 1.0), (0.0, layers / cells)), (True,) * 3
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
                lambda x, y, z: b0
                * (np.cos(4 * np.pi * x) / (4 * np.pi) + np.cos(2 * np.pi * y) / (2 * np.pi)),
            ),
        )
        return model

    @classmethod
    def alfven_wave(cls, cells, *, amplitude=0.1, **options):
        hierarchy = Hierarchy(
            (2 * cells, cells, cells), ((0.0, 2.0), (0.0, 1.0), (0.0, 1.0)), (True,) * 3
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
    def blast_wave(cls, cells, **options):
        hierarchy = Hierarchy(
            (cells, cells, (3 * cells) // 2),
            ((-0.5, 0.5), (-0.5, 0.5), (-0.75, 0.75)),
            (True,) * 3,
        )
        field = 1.0 / np.sqrt(3.0)
        options = {"limiter": "minmod", **options}
        model = cls(hierarchy, mean_field=(field, field, field), **options)
        model.set_state(
            1.0,
            (0.0, 0.0, 0.0),
            lambda x, y, z: np.where(x**2 + y**2 + z**2 < 0.01, 10.0, 0.1),
        )
        return model

    # state -------------------------------------------------------------------------------
    @staticmethod
    def _evaluate(value, *coordinates):
        shape = coordinates[0].shape
        if callable(value):
            return np.broadcast_to(np.asarray(value(*coordinates), dtype=float), shape)
        return np.broadcast_to(np.asarray(value, dtype=float), shape)

    def face_fields(self, potential, spacing):
        faces = []
        for a in range(3):
            _, b, c = cyclic(a)
            faces.append(
                np.diff(potential[c], axis=b) / spacing[b]
                - np.diff(potential[b], axis=c) / spacing[c]
                + self.mean_field[a]
            )
        return faces

    @staticmethod
    def cell_fields(faces):
        return [
            0.5 * (along(f, a, 0, f.shape[a] - 1) + along(f, a, 1, f.shape[a]))
            for a, f in enumerate(faces)
        ]

    def set_state(self, density, velocity, pressure, *, vector_potential=(0.0, 0.0, 0.0)):
        hierarchy = self.hierarchy
        gamma = self.gamma
        for patch in hierarchy.patches:
            x, y, z = patch.coordinates(hierarchy, (0, 0, 0))
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
            for name, value in zip(self.potential, vector_potential, strict=True):
                at = patch.coordinates(hierarchy, patch.field(name).extra)
                if isinstance(value, np.ndarray) and value.shape == patch.field(name).local.shape:
                    patch.field(name).local[...] = value
                else:
                    patch.field(name).local[...] = self._evaluate(value, *at)
                potential.append(np.asarray(patch.field(name).local))
            bx, by, bz = self.cell_fields(
                self.face_fields(tuple(potential), hierarchy.spacing(patch.level))
            )
            values = {
                "density": rho,
                "momentum_x": rho * u,
                "momentum_y": rho * v,
                "momentum_z": rho * w,
                "energy": p / (gamma - 1.0)
                + 0.5 * rho * (u**2 + v**2 + w**2)
                + 0.5 * (bx**2 + by**2 + bz**2),
            }
            for name, value in values.items():
                patch.field(self.names[name]).local[...] = value
        for name in (*self.names.values(), *self.potential):
            hierarchy.restrict(name)
        self.time = 0.0
        self.steps = 0
        self._ready = True

    def set_conserved(self, fields, potential):
        """Set level 0 (one patch) from conserved arrays and edge potentials directly."""
        (patch,) = self.hierarchy.patches_at_level(0)
        for name, value in zip(CONSERVED_3D, fields, strict=True):
            patch.field(self.names[name]).local[...] = value
        for name, value in zip(self.potential, potential, strict=True):
            patch.field(name).local[...] = value
        self.time = 0.0
        self.steps = 0
        self._ready = True

    def _check_ready(self):
        if not self._ready:
            raise RuntimeError("set the state first (set_state)")

    # halos -------------------------------------------------------------------------------
    def fill_halos(self):
        hierarchy = self.hierarchy
        names = [*self.names.values(), *self.potential]
        coarse = {}
        for level in range(hierarchy.max_level + 1):
            for name in names:
                hierarchy.exchange_level(name, level, coarse.get(name))
            shape = hierarchy.level_shape(level)
            for patch in hierarchy.patches_at_level(level):
                for axis in range(3):
                    if self.periodic[axis]:
                        continue
                    lower = patch.box[axis][0] == 0
                    upper = patch.box[axis][1] == shape[axis]
                    if not (lower or upper):
                        continue
                    for name in self.names.values():
                        outflow_cells(patch.field(name).local_with_halos, axis, lower, upper)
                    for name in self.potential:
                        outflow_nodes(patch.field(name).local_with_halos, axis, lower, upper)
            coarse = {name: hierarchy.padded(name, level) for name in names}

    # right-hand side ---------------------------------------------------------------------
    def primitive(self, patch):
        spacing = self.hierarchy.spacing(patch.level)
        potential = tuple(np.asarray(patch.field(n).local_with_halos) for n in self.potential)
        faces = self.face_fields(potential, spacing)
        cells = self.cell_fields(faces)
        rho, mx, my, mz, energy = (
            np.asarray(patch.field(self.names[n]).local_with_halos) for n in CONSERVED_3D
        )
        with np.errstate(divide="ignore", invalid="ignore"):
            u, v, w = mx / rho, my / rho, mz / rho
            bx, by, bz = cells
            p = (self.gamma - 1.0) * (
                energy - 0.5 * rho * (u**2 + v**2 + w**2) - 0.5 * (bx**2 + by**2 + bz**2)
            )
        prim = np.stack((rho, u, v, w, p, bx, by, bz))
        h = HALO
        inner = prim[(slice(None), *(slice(h, -h),) * 3)]
        if not (np.all(np.isfinite(inner)) and np.all(inner[0] > 0) and np.all(inner[4] > 0)):
            raise FloatingPointError(
                f"non-positive density or pressure on the level-{patch.level} patch "
                f"{patch.box} at t = {self.time}"
            )
        return prim, faces, cells

    def sweep(self, prim, face, axis):
        """Fluxes through the faces normal to ``axis``, physical axis order, frame rows."""
        s, b, c = cyclic(axis)
        q = prim[[0, 1 + s, 1 + b, 1 + c, 4, 5 + b, 5 + c]]
        n = q.shape[1 + axis]
        normal = along(face, axis, 2, n - 1)
        code = K.LIMITER_CODES.index(self.limiter)
        return K.sweep_lines(q, normal, code, self.gamma, axis)

    def edge_field(self, prim, sweeps, patch):
        fields = []
        for c in range(3):
            _, a, b = cyclic(c)
            cell = prim[5 + a] * prim[1 + b] - prim[5 + b] * prim[1 + a]
            order = (c, a, b)
            fa = sweeps[a][[0, 5]]  # a-faces: mass, flux of B_b (= -E_c)
            fb = sweeps[b][[0, 6]]  # b-faces: mass, flux of B_a (= +E_c)
            fa = np.transpose(fa, (0, *(1 + i for i in order)))
            fb = np.transpose(fb, (0, *(1 + i for i in order)))
            cell = np.transpose(cell, order)
            na, nb, nc = (patch.shape[i] for i in (a, b, c))
            h = HALO
            sl = slice(h, h + nc)
            out = K.ct_nodes(fa[1][sl], fb[1][sl], fa[0][sl], fb[0][sl], cell[sl], na + 1, nb + 1)
            fields.append(np.transpose(out, np.argsort(order)))
        return fields

    def resistive(self, faces, patch, edges, fluxes):
        h = HALO
        eta = self.resistivity
        spacing = self.hierarchy.spacing(patch.level)
        shape = patch.shape
        current = []
        for c in range(3):
            _, a, b = cyclic(c)
            parts = []
            for axis, field, sign in ((a, faces[b], 1.0), (b, faces[a], -1.0)):
                derivative = np.diff(field, axis=axis) / spacing[axis]
                index = [slice(h, h + shape[i]) for i in range(3)]
                index[a] = slice(h, h + shape[a] + 1)
                index[b] = slice(h, h + shape[b] + 1)
                index[axis] = slice(h - 1, h + shape[axis])
                parts.append(sign * derivative[tuple(index)])
            current.append(parts[0] + parts[1])
        for c in range(3):
            edges[c] += eta * current[c]
        for s in range(3):
            _, b, c = cyclic(s)
            jb = pair_mean(current[b], c, 0, shape[c])
            jc = pair_mean(current[c], b, 0, shape[b])
            fluxes[s] += eta * (
                jb * field_at_face(faces[c], s, c, shape) - jc * field_at_face(faces[b], s, b, shape)
            )

    def patch_fluxes(self, patch):
        prim, faces, _ = self.primitive(patch)
        sweeps = [self.sweep(prim, faces[s], s) for s in range(3)]
        edges = self.edge_field(prim, sweeps, patch)
        h = HALO
        shape = patch.shape
        fluxes = {name: [] for name in CONSERVED_3D}
        for s in range(3):
            frame = cyclic(s)
            index = [slice(None)] * 4
            for t in range(3):
                if t != s:
                    index[1 + t] = slice(h, h + shape[t])
            block = sweeps[s][tuple(index)]
            fluxes["density"].append(block[0])
            for row, axis in zip((1, 2, 3), frame, strict=True):
                fluxes[("momentum_x", "momentum_y", "momentum_z")[axis]].append(block[row])
            fluxes["energy"].append(np.array(block[4]))
        if self.resistivity:
            self.resistive(faces, patch, edges, fluxes["energy"])
        return fluxes, edges

    def advance(self, dt, scale):
        hierarchy = self.hierarchy
        self.fill_halos()
        results = {id(p): self.patch_fluxes(p) for p in hierarchy.patches}
        g = self.gravity
        sources = {}
        if any(g):
            for patch in hierarchy.patches:
                rho = np.array(patch.field(self.names["density"]).local)
                momentum = [
                    np.asarray(patch.field(self.names[f"momentum_{a}"]).local) for a in "xyz"
                ]
                work = sum(m * ga for m, ga in zip(momentum, g, strict=True))
                sources[id(patch)] = (rho, np.array(work))
        for name in CONSERVED_3D:
            self.register.update(
                self.names[name],
                lambda patch, name=name: tuple(results[id(patch)][0][name]),
                dt,
                scale=scale,
            )
        for patch in hierarchy.patches:
            edges = results[id(patch)][1]
            for name, field in zip(self.potential, edges, strict=True):
                patch.field(name).local[...] -= dt * field
            if any(g):
                rho, work = sources[id(patch)]
                for a, ga in zip("xyz", g, strict=True):
                    if ga:
                        patch.field(self.names[f"momentum_{a}"]).local[...] += dt * ga * rho
                patch.field(self.names["energy"]).local[...] += dt * work

    # time stepping -----------------------------------------------------------------------
    def stable_step(self):
        self._check_ready()
        hierarchy = self.hierarchy
        smallest = np.inf
        for patch in hierarchy.patches:
            spacing = hierarchy.spacing(patch.level)
            potential = tuple(np.asarray(patch.field(n).local) for n in self.potential)
            field = self.cell_fields(self.face_fields(potential, spacing))
            rho, *momentum, energy = (
                np.asarray(patch.field(self.names[n]).local) for n in CONSERVED_3D
            )
            velocity = [m / rho for m in momentum]
            p = (self.gamma - 1.0) * (
                energy - 0.5 * rho * sum(v**2 for v in velocity) - 0.5 * sum(b**2 for b in field)
            )
            rate = sum(
                (
                    np.abs(velocity[a])
                    + K.fast_speed(rho, p, field[a], field[(a + 1) % 3], field[(a + 2) % 3], self.gamma)
                )
                / spacing[a]
                for a in range(3)
            )
            smallest = min(smallest, 1.0 / float(np.max(rate)))
            if self.resistivity:
                smallest = min(smallest, 0.5 / (self.resistivity * sum(d**-2 for d in spacing)))
        return self.cfl * float(smallest)

    def step(self, dt=None):
        self._check_ready()
        if dt is None:
            dt = self.stable_step()
        hierarchy = self.hierarchy
        names = [*self.names.values(), *self.potential]
        start = {(id(p), n): np.array(p.field(n).local) for p in hierarchy.patches for n in names}
        self.advance(dt, 0.5 * dt)
        for name in self.potential:
            hierarchy.restrict(name)
        self.advance(dt, 0.5 * dt)
        for patch in hierarchy.patches:
            for name in names:
                array = patch.field(name).local
                array += start[id(patch), name]
                array *= 0.5
        for name in self.names.values():
            self.register.reflux(name)
        for name in self.potential:
            hierarchy.restrict(name)
        self.time += dt
        self.steps += 1
        return dt

    def run(self, duration, *, max_steps=1_000_000):
        self._check_ready()
        end = self.time + duration
        taken = 0
        while self.time < end * (1.0 - 1e-14) and taken < max_steps:
            dt = min(self.stable_step(), end - self.time)
            self.step(dt)
            taken += 1
        return taken

    # diagnostics -------------------------------------------------------------------------
    def divergence(self):
        largest = 0.0
        for patch in self.hierarchy.patches:
            spacing = self.hierarchy.spacing(patch.level)
            potential = tuple(np.asarray(patch.field(n).local) for n in self.potential)
            faces = self.face_fields(potential, spacing)
            div = sum(np.diff(f, axis=a) / spacing[a] for a, f in enumerate(faces))
            largest = max(largest, float(np.max(np.abs(div))) * min(spacing))
        return largest

    def totals(self):
        return {name: self.hierarchy.integral(self.names[name]) for name in CONSERVED_3D}

    def state(self):
        (patch,) = self.hierarchy.patches_at_level(0)
        out = {name: np.array(patch.field(self.names[name]).local) for name in CONSERVED_3D}
        for key, name in zip(("ax", "ay", "az"), self.potential, strict=True):
            out[key] = np.array(patch.field(name).local)
        return out

    def dataset(self, level=0):
        hierarchy = self.hierarchy
        shape = hierarchy.level_shape(level)
        names = (*CONSERVED_3D, "bx", "by", "bz")
        fields = {name: np.full(shape, np.nan) for name in names}
        for patch in hierarchy.patches_at_level(level):
            index = tuple(slice(lo, hi) for lo, hi in patch.box)
            for name in CONSERVED_3D:
                fields[name][index] = patch.field(self.names[name]).local
            potential = tuple(np.array(patch.field(n).local) for n in self.potential)
            cells = self.cell_fields(self.face_fields(potential, hierarchy.spacing(patch.level)))
            for name, value in zip(("bx", "by", "bz"), cells, strict=True):
                fields[name][index] = value
        rho = fields["density"]
        u, v, w = (fields[f"momentum_{a}"] / rho for a in "xyz")
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
