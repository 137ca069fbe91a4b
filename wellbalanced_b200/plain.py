"""The plain float64 GPU step: the reference's dataflow on the device, kernel by kernel.

`PlainMHD2D` / `PlainMHD3D` keep the surface of `MHD2D` / `MHD3D` but advance the way
the reference does (``carafe/mhd.py:844-994``, ``carafe/mhd3d.py:475-754``): per patch
and stage, the haloed block is gathered into contiguous arrays, the reference's block
kernels run one by one through the C ABI (``mhd_primitive``, ``mhd_sweep`` per axis —
after the reference's transposes in 3D —, ``ct_contact`` — all planes of a 3D block in
one launch —, ``mhd_conductive``, ``mhd_resistive``), every intermediate (primitive
variables, face fields, fluxes, edge fields) lives in HBM, and the flux-register update
(the fine-minus-coarse fluxes of every coarse-fine interface, from the sweeps' own fluxes),
gravity sources, potential update and Heun combine are device array operations. It is
the float64 baseline the fused kernels are measured against, and in 3D it carries the
terms the fused 3D kernel leaves out (resistivity, gravity).
"""

from __future__ import annotations

import torch

from wellbalanced_b200 import _lib
from wellbalanced_b200.kernels import KERNELS
from wellbalanced_b200.mesh import HALO
from wellbalanced_b200.mhd import CONSERVED, MHD2D
from wellbalanced_b200.mhd3d import CONSERVED_3D, MHD3D

_FLUX_ROWS = ((0, 1, 2, 3, 4, 6), (0, 2, 1, 3, 4, 6))
_WALL_ROWS = [0, 2, 3, 4, 6]


def _face_ops(engine):
    import numpy as np

    ops = engine.layout.face_flux_ops
    return [] if ops is None or ops.size == 0 else list(np.atleast_1d(ops))


def _register_update(engine, blocks):
    """reg += (mean of the fine faces - the coarse face) at every coarse-fine interface
    face, from the per-patch flux blocks of a stage (patchwork's FluxRegister.update as
    carafe/mhd.py:906-919 calls it; the slots of the device register, which `Engine.reflux`
    applies with 0.5 dt after the step).

    ``blocks(patch_index, axis)``: a tensor (fields, ...) of that patch's fluxes through
    its faces normal to ``axis``, indexed [field, face along axis, transverse haloed or
    interior indices] as `_plane` reads them.
    """
    reg = engine.register
    for op in _face_ops(engine):
        axis, length, width = int(op["axis"]), int(op["len"]), int(op["width"])
        coarse = _plane(blocks(int(op["coarse"]), axis), op, "coarse", length // width, width, 1)
        fine = _plane(blocks(int(op["fine"]), axis), op, "fine", length // width, width, 2)
        if int(op["ndim"]) == 2:
            total = fine[:, :, 0] + fine[:, :, 1]
            count = 2.0
        else:
            total = fine[:, :, 0, :, 0] + fine[:, :, 0, :, 1] + fine[:, :, 1, :, 0] + fine[:, :, 1, :, 1]
            count = 4.0
        values = total.reshape(total.shape[0], -1) / count - coarse.reshape(coarse.shape[0], -1)
        off = int(op["reg_off"])
        reg[off : off + values.numel()] += values.reshape(-1)


def _plane(flux, op, side, n1, n2, step):
    """The faces of one side of an op from a flux block: 2D (fields, n1[, 2]); 3D (fields,
    n1[, 2], n2[, 2]). ``flux`` is indexed [field, normal face, t1, t2] after `_oriented`."""
    plane = int(op[f"{side}_plane"]) - HALO
    t0 = [int(v) for v in op[f"{side}_t0"]]
    if int(op["ndim"]) == 2:
        rows = flux[:, plane, t0[0] : t0[0] + step * n1]
        return rows.reshape(rows.shape[0], n1, step) if step == 2 else rows
    rows = flux[:, plane, t0[0] : t0[0] + step * n1, t0[1] : t0[1] + step * n2]
    return rows.reshape(rows.shape[0], n1, step, n2, step) if step == 2 else rows


def _stream():
    return torch.cuda.current_stream().cuda_stream


class PlainMHD2D(MHD2D):
    """`MHD2D` advanced by the per-kernel float64 path (resistive / conductive / gravity too)."""

    _fused = False

    def __init__(self, hierarchy, **options):
        options["precision"] = 64
        super().__init__(hierarchy, **options)
        self._work = {}

    def _buffers(self, patch):
        work = self._work.get(patch.index)
        if work is None:
            nx, ny = patch.shape
            X, Y = nx + 2 * HALO, ny + 2 * HALO
            new = lambda *shape: torch.empty(shape, dtype=torch.float64, device=self.engine.device)  # noqa: E731
            work = {
                "prim": new(8, X, Y), "bxf": new(X + 1, Y), "byf": new(X, Y + 1), "ecc": new(X, Y),
                "fx": new(7, X - 3, Y), "fy": new(7, X, Y - 3), "ez": new(nx + 1, ny + 1),
            }
            self._work[patch.index] = work
        return work

    def _patch_fluxes(self, patch):
        """The reference's ``_patch_fluxes`` (carafe/mhd.py:844-887) with device kernels."""
        eng = self.engine
        nx, ny = patch.shape
        X, Y = nx + 2 * HALO, ny + 2 * HALO
        cons = [eng.view(eng.state, patch, f)[:X, :Y].contiguous() for f in range(6)]
        az = eng.view(eng.state, patch, 6)[: X + 1, : Y + 1].contiguous()
        w = self._buffers(patch)
        dx, dy = self.hierarchy.spacing(patch.level)
        _lib.call("wb_mhd_primitive", *(c.data_ptr() for c in cons), az.data_ptr(), X, Y, dx, dy, *self.mean_field,
                  self.gamma, w["prim"].data_ptr(), w["bxf"].data_ptr(), w["byf"].data_ptr(), w["ecc"].data_ptr(),
                  eng.bad.data_ptr(), _stream())
        code = ("minmod", "vanleer", "mc", "none").index(self.limiter)
        KERNELS["mhd_sweep"](w["prim"], w["bxf"], 0, code, self.gamma, w["fx"])
        KERNELS["mhd_sweep"](w["prim"], w["byf"], 1, code, self.gamma, w["fy"])
        fx, fy, ez = w["fx"], w["fy"], w["ez"]
        KERNELS["ct_contact"](fx[5], fy[5], fx[0], fy[0], w["ecc"], ez)
        if max(self.conduction) > 0.0:
            KERNELS["mhd_conductive"](w["prim"], w["bxf"], w["byf"], dx, dy, *self.conduction, fx, fy)
        if self.resistivity:
            KERNELS["mhd_resistive"](w["prim"], w["bxf"], w["byf"], dx, dy, self.resistivity, fx, fy, ez)
        shape = self.hierarchy.level_shape(patch.level)
        sides = [(self.walls[a] and patch.box[a][0] == 0, self.walls[a] and patch.box[a][1] == shape[a]) for a in range(2)]
        (left, right), (bottom, top) = sides
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

    def _advance(self, dt, scale):
        """One forward-Euler stage (carafe/mhd.py:889-927)."""
        eng = self.engine
        eng.fill(eng.state)
        fluxes = {p.index: self._patch_fluxes(p) for p in self.hierarchy.patches}
        if self.hierarchy.max_level > 0:
            # x-faces: [row, face, haloed y]; y-faces [row, haloed x, face] -> [row, face, haloed x]
            def blocks(index, axis):
                rows = list(_FLUX_ROWS[axis])
                return fluxes[index][0][rows] if axis == 0 else fluxes[index][1][rows].transpose(1, 2)

            _register_update(eng, blocks)
        gx, gy = self.gravity
        sources = {}
        if gx or gy:
            for p in self.hierarchy.patches:
                rho = self._read(p, 0).clone()
                sources[p.index] = (rho * gx, rho * gy, (self._read(p, 1) * gx + self._read(p, 2) * gy).clone())
        h = HALO
        for p in self.hierarchy.patches:
            nx, ny = p.shape
            dx, dy = self.hierarchy.spacing(p.level)
            fx, fy, ez = fluxes[p.index]
            for f, (xr, yr) in enumerate(zip(*_FLUX_ROWS, strict=True)):
                bx = fx[xr, :, h : h + ny]
                by = fy[yr, h : h + nx, :]
                divergence = (bx[1:] - bx[:-1]) / dx + (by[:, 1:] - by[:, :-1]) / dy
                self._read(p, f).sub_(dt * divergence)
            self._read(p, 6, node=True).sub_(dt * ez)
            if gx or gy:
                fxs, fys, work = sources[p.index]
                self._read(p, 1).add_(dt * fxs)
                self._read(p, 2).add_(dt * fys)
                self._read(p, 4).add_(dt * work)

    def stable_step(self):
        self._check_ready()
        eng = self.engine
        eng.fill(eng.state)
        smallest = float("inf")
        out = torch.empty(2, dtype=torch.float64, device=eng.device)
        for p in self.hierarchy.patches:
            nx, ny = p.shape
            X, Y = nx + 2 * HALO, ny + 2 * HALO
            dx, dy = self.hierarchy.spacing(p.level)
            cons = [eng.view(eng.state, p, f)[:X, :Y].contiguous() for f in range(6)]
            az = eng.view(eng.state, p, 6)[: X + 1, : Y + 1].contiguous()
            KERNELS["mhd_rate"](*cons, az, HALO, dx, dy, *self.mean_field, self.gamma, out)
            rate, rho_min = out.tolist()
            smallest = min(smallest, 1.0 / rate)
            diffusivity = max(self.resistivity, (self.gamma - 1.0) * max(self.conduction) / rho_min)
            if diffusivity > 0.0:
                smallest = min(smallest, 0.5 / (diffusivity * (dx**-2 + dy**-2)))
        return self.cfl * smallest

    def step(self, dt=None):
        """Heun's method as the reference (carafe/mhd.py:965-994)."""
        self._check_ready()
        eng = self.engine
        if dt is None:
            dt = self.stable_step()
        eng.bad.zero_()
        start = eng.state.clone()
        self._advance(dt, 0.5 * dt)
        if self.hierarchy.max_level > 0:
            eng.restrict(eng.state, self._groups_potential)
        self._advance(dt, 0.5 * dt)
        eng.state.add_(start)
        eng.state.mul_(0.5)
        if self.hierarchy.max_level > 0:
            eng.dt.fill_(float(dt))
            eng.reflux(eng.state)
            eng.restrict(eng.state, self._groups_all)
        eng.fill(eng.state)
        self._raise_if_bad()
        self.time += float(dt)
        self.steps += 1
        return float(dt)

    def advance(self, steps):
        for _ in range(steps):
            self.step()


def _cyclic(axis):
    return axis, (axis + 1) % 3, (axis + 2) % 3


class PlainMHD3D(MHD3D):
    """`MHD3D` advanced by the reference's 3D dataflow on the device (float64)."""

    _fused = False

    def __init__(self, hierarchy, **options):
        options["precision"] = 64
        super().__init__(hierarchy, **options)

    def _haloed(self, patch):
        eng = self.engine
        nx, ny, nz = patch.shape
        X, Y, Z = nx + 4, ny + 4, nz + 4
        cons = [eng.view(eng.state, patch, f)[:X, :Y, :Z] for f in range(5)]
        pot = (
            eng.view(eng.state, patch, 5)[:X, : Y + 1, : Z + 1],
            eng.view(eng.state, patch, 6)[: X + 1, :Y, : Z + 1],
            eng.view(eng.state, patch, 7)[: X + 1, : Y + 1, :Z],
        )
        return cons, pot

    def _primitive3(self, patch):
        """carafe/mhd3d.py:475-509 on the device."""
        spacing = self.hierarchy.spacing(patch.level)
        cons, pot = self._haloed(patch)
        faces = []
        for a in range(3):
            _, b, c = _cyclic(a)
            faces.append(torch.diff(pot[c], dim=b) / spacing[b] - torch.diff(pot[b], dim=c) / spacing[c] + self.mean_field[a])
        cells = [0.5 * (f.narrow(a, 0, f.shape[a] - 1) + f.narrow(a, 1, f.shape[a] - 1)) for a, f in enumerate(faces)]
        rho, mx, my, mz, energy = cons
        u, v, w = mx / rho, my / rho, mz / rho
        bx, by, bz = cells
        p = (self.gamma - 1.0) * (energy - 0.5 * rho * (u**2 + v**2 + w**2) - 0.5 * (bx**2 + by**2 + bz**2))
        prim = torch.stack((rho, u, v, w, p, bx, by, bz))
        inner = prim[:, HALO:-HALO, HALO:-HALO, HALO:-HALO]
        bad = (~torch.isfinite(inner).all(dim=0)) | (inner[0] <= 0) | (inner[4] <= 0)
        self.engine.bad.add_(bad.sum())
        return prim, faces

    def _sweep(self, prim, face, axis):
        """carafe/mhd3d.py:511-528: frame rows, transpose, one mhd_sweep over all lines."""
        frame = _cyclic(axis)
        rows = [0, *(1 + a for a in frame), 4, *(5 + a for a in frame)]
        moved = prim[rows].permute(0, *(1 + a for a in frame))
        n, nb, nc = moved.shape[1:]
        lines = moved.reshape(8, n, nb * nc).contiguous()
        normal = face.permute(frame).reshape(n + 1, nb * nc).contiguous()
        flux = torch.empty((7, n - 3, nb * nc), dtype=torch.float64, device=prim.device)
        code = ("minmod", "vanleer", "mc", "none").index(self.limiter)
        KERNELS["mhd_sweep"](lines, normal, 0, code, self.gamma, flux)
        return flux.reshape(7, n - 3, nb, nc)

    def _edge_field(self, prim, sweeps, patch):
        """carafe/mhd3d.py:530-559: ct_contact on every plane normal to each edge direction."""
        h = HALO
        fields = []
        for c in range(3):
            _, a, b = _cyclic(c)
            cell = prim[5 + a] * prim[1 + b] - prim[5 + b] * prim[1 + a]
            frame = (c, a, b)
            cell = cell.permute(frame).contiguous()
            fa = sweeps[a][[0, 5]].permute(3, 0, 1, 2).contiguous()
            fb = sweeps[b][[0, 6]].permute(2, 0, 3, 1).contiguous()
            na, nb, nc = (patch.shape[i] for i in frame[1:] + frame[:1])
            X, Y = cell.shape[1], cell.shape[2]
            out = torch.empty((nc, na + 1, nb + 1), dtype=torch.float64, device=prim.device)
            sl = slice(h, h + nc)
            args = [fa[sl, 1].contiguous(), fb[sl, 1].contiguous(), fa[sl, 0].contiguous(), fb[sl, 0].contiguous(),
                    cell[sl].contiguous()]
            _lib.call("wb_ct_contact_planes", *(t.data_ptr() for t in args), X, Y, na + 1, nb + 1, nc, out.data_ptr(),
                      _stream())
            inverse = [frame.index(i) for i in range(3)]
            fields.append(out.permute(inverse))
        return fields

    def _patch_fluxes(self, patch):
        prim, faces = self._primitive3(patch)
        sweeps = [self._sweep(prim, faces[s], s) for s in range(3)]
        edges = self._edge_field(prim, sweeps, patch)
        h = HALO
        shape = patch.shape
        fluxes = {name: [] for name in CONSERVED_3D}
        for s in range(3):
            frame = _cyclic(s)
            block = sweeps[s][:, :, h : h + shape[frame[1]], h : h + shape[frame[2]]]
            inverse = [0, *(1 + frame.index(i) for i in range(3))]
            block = block.permute(inverse)
            fluxes["density"].append(block[0])
            for row, axis in zip((1, 2, 3), frame, strict=True):
                fluxes[("momentum_x", "momentum_y", "momentum_z")[axis]].append(block[row])
            fluxes["energy"].append(block[4])
        if self.resistivity:
            self._resistive(faces, patch, edges, fluxes["energy"])
        return fluxes, edges

    def _resistive(self, faces, patch, edges, energy):
        """eta J on the edge field, eta J x B on the energy fluxes (carafe/mhd3d.py:561-602).

        J_c = d_a B_b - d_b B_a on the c-edges of the block from the haloed face fields; a
        face normal to s gains eta (J_b B_c - J_c B_b), J the mean of the face's two edges
        along each direction and B the mean of the four faces around it.
        """
        h = HALO
        eta = self.resistivity
        spacing = self.hierarchy.spacing(patch.level)
        shape = patch.shape
        current = []
        for c in range(3):
            _, a, b = _cyclic(c)
            total = 0.0
            for axis, field, sign in ((a, faces[b], 1.0), (b, faces[a], -1.0)):
                derivative = torch.diff(field, dim=axis) / spacing[axis]
                index = [slice(h, h + shape[i]) for i in range(3)]
                index[a] = slice(h, h + shape[a] + 1)
                index[b] = slice(h, h + shape[b] + 1)
                index[axis] = slice(h - 1, h + shape[axis])
                total = total + sign * derivative[tuple(index)]
            current.append(total)
        for c in range(3):
            edges[c] = edges[c] + eta * current[c]

        def pair_mean(t, axis, start, count):
            return 0.5 * (t.narrow(axis, start, count) + t.narrow(axis, start + 1, count))

        def field_at_face(face, normal, node):
            face = pair_mean(face, normal, h - 1, shape[normal] + 1)  # cells -> nodes along the normal
            face = pair_mean(face, node, h, shape[node])  # nodes -> cells along the face's own axis
            other = 3 - normal - node
            return face.narrow(other, h, shape[other])

        for s in range(3):
            _, b, c = _cyclic(s)
            jb = pair_mean(current[b], c, 0, shape[c])
            jc = pair_mean(current[c], b, 0, shape[b])
            energy[s] = energy[s] + eta * (jb * field_at_face(faces[c], s, c) - jc * field_at_face(faces[b], s, b))

    def _advance(self, dt, scale):
        eng = self.engine
        eng.fill(eng.state)
        results = {p.index: self._patch_fluxes(p) for p in self.hierarchy.patches}
        if self.hierarchy.max_level > 0:
            # interior blocks [face along axis, ...] -> [field, face, t1, t2] with haloed
            # transverse indices (two zero-padded halo layers in front)
            def blocks(index, axis):
                t1, t2 = (b for b in range(3) if b != axis)  # the ops' transverse axes, in order
                stacked = torch.stack([results[index][0][name][axis] for name in CONSERVED_3D])
                oriented = stacked.permute(0, 1 + axis, 1 + t1, 1 + t2)
                return torch.nn.functional.pad(oriented, (HALO, 0, HALO, 0))

            _register_update(eng, blocks)
        g = self.gravity
        sources = {}
        if any(g):
            # rho g on the momentum and m . g on the energy, from the stage's input state
            for p in self.hierarchy.patches:
                rho = self._read(p, 0).clone()
                work = sum(self._read(p, 1 + a) * ga for a, ga in enumerate(g))
                sources[p.index] = (rho, work.clone())
        for p in self.hierarchy.patches:
            spacing = self.hierarchy.spacing(p.level)
            fluxes, edges = results[p.index]
            for f, name in enumerate(CONSERVED_3D):
                divergence = 0.0
                for a, flux in enumerate(fluxes[name]):
                    divergence = divergence + torch.diff(flux, dim=a) / spacing[a]
                self._read(p, f).sub_(dt * divergence)
            for c in range(3):
                extra = ((0, 1, 1), (1, 0, 1), (1, 1, 0))[c]
                self._read(p, 5 + c, extra).sub_(dt * edges[c])
            if any(g):
                rho, work = sources[p.index]
                for a, ga in enumerate(g):
                    if ga:
                        self._read(p, 1 + a).add_(dt * ga * rho)
                self._read(p, 4).add_(dt * work)

    def stable_step(self):
        self._check_ready()
        eng = self.engine
        eng.rate()
        eng.finalize_dt(self.cfl, self.resistivity, 0.0)
        return float(eng.dt[0].item())

    def step(self, dt=None):
        self._check_ready()
        eng = self.engine
        if dt is None:
            dt = self.stable_step()
        eng.bad.zero_()
        start = eng.state.clone()
        self._advance(dt, 0.5 * dt)
        if self.hierarchy.max_level > 0:
            eng.restrict(eng.state, self._groups_potential)
        self._advance(dt, 0.5 * dt)
        eng.state.add_(start)
        eng.state.mul_(0.5)
        if self.hierarchy.max_level > 0:
            eng.dt.fill_(float(dt))
            eng.reflux(eng.state)
            eng.restrict(eng.state, self._groups_all)
        eng.fill(eng.state)
        self._raise_if_bad()
        self.time += float(dt)
        self.steps += 1
        return float(dt)

    def advance(self, steps, check=True):
        for _ in range(steps):
            self.step()
