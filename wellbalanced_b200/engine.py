"""Device state and step driver shared by `MHD2D` and `MHD3D`.

Holds the two state pools of the Heun step (the state U and the stage U1), the layout
of a hierarchy (`wellbalanced_b200.mesh.Layout`) uploaded to the device, and launches
through the C ABI:

* ``fill(pool)`` — patchwork's ``exchange_halos`` plus the boundary faces, level by
  level: interpolation from the level below, same-level copies, outflow / wall faces;
* ``restrict(pool, groups)`` — patchwork's ``restrict``;
* ``stage(...)`` — one fused RK stage over every tile;
* ``rate()`` / ``finalize_dt()`` — the stable step on the device.

One step is the reference's ``step`` (``carafe/mhd.py:965-994``,
``carafe/mhd3d.py:726-754``): stage 1 into U1, restrict the potential, fill U1, stage 2
back into U with the Heun combine, reflux, restrict, fill. torch is used for device
memory and streams only; every numerical kernel is in ``libwb200.so``.
"""

from __future__ import annotations

import contextlib
import ctypes

import numpy as np
import torch

from wellbalanced_b200 import _lib
from wellbalanced_b200.mesh import Layout, _concat, number_faces, size_ops

_DTYPES = {32: torch.float32, 64: torch.float64, _lib.MATH32_STATE64: torch.float64}


def _ptr(t):
    return ctypes_ptr(t)


def ctypes_ptr(t):
    if t is None:
        return None
    return t.data_ptr()


def _device_bytes(array, device, dtype):
    """A uint8 device tensor holding a numpy structured array in the C layout ``dtype``
    (None if empty). NumPy may repack a padded structured dtype (``np.concatenate`` does),
    so the records are cast back to the exact layout the kernels read."""
    if array is None or array.size == 0:
        return None
    array = np.ascontiguousarray(np.asarray(array).astype(dtype, copy=False))
    if array.dtype != dtype or array.dtype.itemsize != dtype.itemsize:
        raise TypeError(f"op records of dtype {array.dtype} do not have the C layout {dtype}")
    return torch.from_numpy(array.view(np.uint8).reshape(-1).copy()).to(device)


class Engine:
    """Device pools + op lists of one hierarchy; the kernels' launch sequence."""

    def __init__(self, hierarchy, *, precision=32, walls=None, limiter=1, gamma=5.0 / 3.0, mean_field=(0.0, 0.0, 0.0),
                 instances=None, device="cuda", lx=32, stream=None, layout=None):
        precision = _lib.precision_code(precision)
        if not torch.cuda.is_available():
            raise RuntimeError("wellbalanced_b200 needs a CUDA device (there is no CPU path)")
        _lib.load()
        self.device = torch.device(device)
        self.precision = precision
        self.dtype = _DTYPES[precision]
        self.limiter = int(limiter)
        self.gamma = float(gamma)
        self.mean_field = tuple(float(b) for b in mean_field) + (0.0,) * (3 - len(mean_field))
        self.layout = layout if layout is not None else Layout(
            hierarchy, walls=walls, precision=precision, lx=lx, instances=instances)
        L = self.layout
        self.ndim = L.ndim
        #: finest level of the layout (the hierarchy's property walks every patch)
        self.max_level = int(L.max_level)
        self.state = torch.zeros(L.pool_size, dtype=self.dtype, device=self.device)
        self.stage_pool = torch.zeros(L.pool_size, dtype=self.dtype, device=self.device)
        self.patches = _device_bytes(L.rows, self.device, _lib.PATCH)
        self.tiles = _device_bytes(L.tiles, self.device, _lib.TILE)
        self.ntiles = int(L.tiles.size)
        self.chunk_patch = torch.from_numpy(L.chunk_patch).to(self.device)
        self.chunk_start = torch.from_numpy(L.chunk_start).to(self.device)
        self.nchunks = int(L.chunk_patch.size)
        self.inv_dx2_sum = torch.from_numpy(L.inv_dx2_sum).to(self.device)
        levels = np.ascontiguousarray(getattr(L, "inv_dx2_levels", L.inv_dx2_sum[:, None]), dtype=np.float64)
        #: levels of the per-(instance, level) diffusion limit
        self.nlevels = int(levels.shape[1])
        self.inv_dx2_levels = torch.from_numpy(levels.reshape(-1)).to(self.device)
        self.level_keys = torch.zeros(max(self.nlevels * L.ninstances, 1), dtype=torch.int64, device=self.device)
        #: reduce the smallest density per level (set by the solvers when a diffusion limit
        #: applies on a refined hierarchy: each level's own density and spacing decide)
        self.per_level_dt = False
        # op lists on the device, each cut for the op kernels by its size (`size_ops`)
        def upload(ops, dtype):
            ops = size_ops(ops) if np.asarray(ops).size else np.zeros(0, dtype)
            return _device_bytes(ops, self.device, dtype), int(ops.size)

        self.copy_phases = [
            (*upload(same, _lib.COPY_OP), [upload(b, _lib.COPY_OP) for b in bnd]) for same, bnd in L.copy_phases
        ]
        self.interp_levels = [upload(ops, _lib.INTERP_OP) for ops in L.interp_levels]
        self.restrict_levels = {
            level: {g: upload(ops, _lib.RESTRICT_OP) for g, ops in groups.items()}
            for level, groups in L.restrict_levels.items()
        }
        # the ops of every field group of a level in one list: the groups write different
        # fields of the coarse level and read only the fine one, so one launch runs them all
        self.restrict_merged = {}
        for level, groups in L.restrict_levels.items():
            if len(groups) > 1:
                ops = _concat(list(groups.values()), _lib.RESTRICT_OP)
                self.restrict_merged[level] = (frozenset(groups), *upload(ops, _lib.RESTRICT_OP))
        n = L.ninstances
        self.ninstances = n
        self.dt = torch.zeros(n, dtype=torch.float64, device=self.device)
        self.keys = torch.zeros(2 * n, dtype=torch.int64, device=self.device)
        self.time = torch.zeros(n, dtype=torch.float64, device=self.device)
        self.end = torch.zeros(n, dtype=torch.float64, device=self.device)
        self.bad = torch.zeros(1, dtype=torch.int64, device=self.device)
        #: the 2D stage kernel's boundary-face fluxes (float64, allocated on first use): the
        #: register reads the fine faces there instead of recomputing them
        self.bflux = None
        self.staged_fluxes = True
        face_ops, self.nface_faces = number_faces(L.face_flux_ops)
        self.face_flux_ops = _device_bytes(face_ops, self.device, _lib.FACE_FLUX_OP)
        self.nface = int(L.face_flux_ops.size)
        self.reflux_ops = _device_bytes(L.reflux_ops, self.device, _lib.REFLUX_OP)
        self.nreflux = int(L.reflux_ops.size)
        counts = [int(ops.size) for ops in L.reflux_phases]
        starts = np.cumsum([0, *counts])[: len(counts)]
        #: (first op, op count) of each reflux phase in `reflux_ops`
        self.reflux_phases = [(int(a), c) for a, c in zip(starts, counts, strict=True) if c]
        self.register = torch.zeros(max(L.register_size, 1), dtype=torch.float64, device=self.device)
        self.stream = stream
        #: kernels launched by this engine (counted per C-ABI call)
        self.launches = 0
        #: optional list collecting (start, end) CUDA events around each stage kernel
        self.stage_events = None
        #: non-ideal terms, None for ideal MHD: 2D (eta, kappa_par, kappa_perp, gx, gy),
        #: 3D (eta, gx, gy, gz)
        self.physics = None
        #: a level's interpolation and same-level copies in one launch (`wb_fill_ops`)
        self.fused_fill = True
        #: run stage 1's flux-register kernel on a second stream, beside the restriction
        #: and halo fill of the stage pool (it reads U, which those do not write)
        self.overlap_fluxes = True
        self._flux_stream = None
        self._flux_events = None
        #: the launching stream's handle while a step issues its launches (looked up once)
        self._step_stream = None
        #: run the reflux, restriction, halo-fill and stable-step phases between the stage
        #: kernels as op programs (`wb_run_program`, one launch each: six launches per
        #: refined step instead of ~26). Off by default: on the B200 the separate launches
        #: finish the ~2300-patch Harris step in 0.62 ms against 0.74 ms for the programs,
        #: whose in-kernel phase waits cost more than the launch boundaries they replace
        self.use_programs = False
        self._programs = {}
        #: dt on the device belongs to the current state (set by `prime_dt` and each
        #: programmed step; cleared by every other launch or write that changes the state)
        self.dt_ready = False

    # low-level launches ----------------------------------------------------------------------
    def _s(self):
        if self._step_stream is not None:
            return self._step_stream
        return self._main().cuda_stream

    def _main(self):
        return self.stream if self.stream is not None else torch.cuda.current_stream(self.device)

    def fill(self, pool, levels=None):
        """Halos of every patch of `pool`, level by level (coarse first)."""
        for level in range(len(self.copy_phases)):
            if levels is None or level in levels:
                self._fill_level(pool, level)

    def _fill_level(self, pool, level):
        """Interpolation from the level below, same-level copies, boundary faces."""
        prec = self.precision
        s = self._s()
        same, nsame, boundary = self.copy_phases[level]
        interp, ninterp = self.interp_levels[level]
        if ninterp and nsame and self.fused_fill:
            # the layout's interpolation ops skip the points the copies write: one launch
            _lib.call("wb_fill_ops", prec, pool.data_ptr(), self.patches.data_ptr(), interp.data_ptr(), ninterp,
                      same.data_ptr(), nsame, s)
            self.launches += 1
        else:
            if ninterp:
                _lib.call("wb_interp_ops", prec, pool.data_ptr(), self.patches.data_ptr(), interp.data_ptr(), ninterp,
                          s)
                self.launches += 1
            if nsame:
                _lib.call("wb_copy_ops", prec, pool.data_ptr(), self.patches.data_ptr(), same.data_ptr(), nsame, s)
                self.launches += 1
        for ops, nops in boundary:
            if nops:
                _lib.call("wb_copy_ops", prec, pool.data_ptr(), self.patches.data_ptr(), ops.data_ptr(), nops, s)
                self.launches += 1

    def restrict(self, pool, groups):
        """Coarse values under finer patches from the fine ones (finest level first)."""
        key = frozenset(groups)
        for level in range(self.max_level, 0, -1):
            merged = self.restrict_merged.get(level)
            if merged is not None and merged[0] == key:
                ops, nops = merged[1], merged[2]
                if nops:
                    _lib.call("wb_restrict_ops", self.precision, pool.data_ptr(), self.patches.data_ptr(),
                              ops.data_ptr(), nops, self._s())
                    self.launches += 1
                continue
            for g in groups:
                self._restrict_level(pool, level, g)

    def _restrict_level(self, pool, level, g):
        ops, nops = self.restrict_levels[level][g]
        if nops:
            _lib.call("wb_restrict_ops", self.precision, pool.data_ptr(), self.patches.data_ptr(), ops.data_ptr(),
                      nops, self._s())
            self.launches += 1

    def _uses_staged_fluxes(self):
        """Whether the register takes the fine faces from the 2D stage kernel's boundary-face
        output (ideal 2D refined hierarchies; the non-ideal terms and 3D recompute them)."""
        return self.staged_fluxes and self.ndim == 2 and self.nface > 0 and self.physics is None

    def _stage_bflux(self):
        if self.bflux is None:
            self.bflux = torch.zeros(max(int(self.layout.bflux_size), 1), dtype=torch.float64, device=self.device)
        return self.bflux

    def stage(self, src, base, dst, bflux=None):
        b = self.mean_field
        s = self._s()
        if self.ntiles == 0:
            return
        if bflux is None and self._uses_staged_fluxes():
            bflux = self._stage_bflux()
        timing = self.stage_events is not None
        if timing:
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(torch.cuda.current_stream(self.device) if self.stream is None else self.stream)
        self.launches += 1
        if self.ndim == 2 and self.physics is not None:
            if tuple(self.layout.tile_shape) != tuple(self.layout.default_tile):
                raise ValueError("the non-ideal 2D stage kernel runs on the default tile shape")
            _lib.call("wb_stage2d_physics", self.precision, src.data_ptr(), None if base is None else base.data_ptr(),
                      dst.data_ptr(), self.patches.data_ptr(), self.tiles.data_ptr(), self.ntiles, self.dt.data_ptr(),
                      self.gamma, b[0], b[1], self.limiter, *self.physics, self.bad.data_ptr(), s)
        elif self.ndim == 2:
            tx, ty = self.layout.tile_shape
            _lib.call("wb_stage2d_tiled", self.precision, src.data_ptr(), None if base is None else base.data_ptr(),
                      dst.data_ptr(), self.patches.data_ptr(), self.tiles.data_ptr(), self.ntiles, self.dt.data_ptr(),
                      self.gamma, b[0], b[1], self.limiter, tx, ty, self.bad.data_ptr(),
                      None if bflux is None else bflux.data_ptr(), s)
        elif self.physics is not None:
            if tuple(self.layout.tile_shape) != tuple(self.layout.default_tile):
                raise ValueError("the non-ideal 3D stage kernel runs on the default tile shape")
            _lib.call("wb_stage3d_physics", self.precision, src.data_ptr(),
                      None if base is None else base.data_ptr(), dst.data_ptr(), self.patches.data_ptr(),
                      self.tiles.data_ptr(), self.ntiles, self.dt.data_ptr(), self.gamma, b[0], b[1], b[2],
                      self.limiter, self.layout.lx, *self.physics, self.bad.data_ptr(), s)
        else:
            ty, tz = self.layout.tile_shape
            _lib.call("wb_stage3d_tiled", self.precision, src.data_ptr(), None if base is None else base.data_ptr(),
                      dst.data_ptr(), self.patches.data_ptr(), self.tiles.data_ptr(), self.ntiles, self.dt.data_ptr(),
                      self.gamma, b[0], b[1], b[2], self.limiter, self.layout.lx, ty, tz, self.bad.data_ptr(),
                      None if bflux is None else bflux.data_ptr(), s)
        if timing:
            end.record(torch.cuda.current_stream(self.device) if self.stream is None else self.stream)
            self.stage_events.append((start, end))

    def rate(self, pool=None):
        pool = self.state if pool is None else pool
        b = self.mean_field
        if self.per_level_dt:
            _lib.call("wb_rate_levels", self.precision, self.ndim, pool.data_ptr(), self.patches.data_ptr(),
                      self.layout.npatches, self.chunk_patch.data_ptr(), self.chunk_start.data_ptr(), self.nchunks,
                      b[0], b[1], b[2], self.gamma, self.keys.data_ptr(), self.ninstances,
                      self.level_keys.data_ptr(), self.nlevels, self._s())
        else:
            _lib.call("wb_rate", self.precision, self.ndim, pool.data_ptr(), self.patches.data_ptr(),
                      self.layout.npatches, self.chunk_patch.data_ptr(), self.chunk_start.data_ptr(), self.nchunks,
                      b[0], b[1], b[2], self.gamma, self.keys.data_ptr(), self.ninstances, self._s())
        self.launches += 2 if self.nchunks else 1

    def finalize_dt(self, cfl, eta=0.0, kappa=0.0, *, clip_to_end=False, advance=False):
        end = self.end.data_ptr() if clip_to_end else None
        if self.per_level_dt:
            _lib.call("wb_finalize_dt_levels", self.keys.data_ptr(), self.ninstances, float(cfl), float(eta),
                      float(kappa), self.gamma, self.level_keys.data_ptr(), self.inv_dx2_levels.data_ptr(),
                      self.nlevels, self.time.data_ptr(), end, self.dt.data_ptr(), int(advance), self._s())
        else:
            _lib.call("wb_finalize_dt", self.keys.data_ptr(), self.ninstances, float(cfl), float(eta), float(kappa),
                      self.gamma, self.inv_dx2_sum.data_ptr(), self.time.data_ptr(), end, self.dt.data_ptr(),
                      int(advance), self._s())
        self.launches += 1

    def rate_values(self):
        """(max rate, min density) per instance, on the host."""
        keys = self.keys.view(torch.int64).cpu().numpy().view(np.uint64).reshape(-1, 2)
        out = np.empty(keys.shape)
        for index, k in np.ndenumerate(keys):
            k = int(k)
            bits = (k & 0x7FFFFFFFFFFFFFFF) if k >> 63 else (~k & 0xFFFFFFFFFFFFFFFF)
            out[index] = np.frombuffer(np.uint64(bits).tobytes(), dtype=np.float64)[0]
        return out

    def face_fluxes(self, pool, stream=None):
        """Register += fine-mean minus coarse fluxes of every coarse-fine interface face
        (on `stream`, else the engine's stream). `pool` is the input of the stage just
        launched: with staged fluxes its fine faces are read from that stage's output."""
        if self.nface:
            s = stream.cuda_stream if stream is not None else self._s()
            b = self.mean_field
            if self.physics is not None:
                eta, kappa_par, kappa_perp = self.physics[:3] if self.ndim == 2 else (self.physics[0], 0.0, 0.0)
            if self.physics is not None and (eta or kappa_par or kappa_perp):
                _lib.call("wb_face_flux_ops_physics", self.precision, pool.data_ptr(), self.patches.data_ptr(),
                          self.face_flux_ops.data_ptr(), self.nface, b[0], b[1], b[2], self.gamma, self.limiter, eta,
                          kappa_par, kappa_perp, self.register.data_ptr(), s)
            elif self._uses_staged_fluxes():
                # the fine faces as the stage kernel that read `pool` wrote them
                _lib.call("wb_face_flux_ops_staged", self.precision, pool.data_ptr(), self.patches.data_ptr(),
                          self.face_flux_ops.data_ptr(), self.nface, self.nface_faces, b[0], b[1], b[2], self.gamma,
                          self.limiter, self._stage_bflux().data_ptr(), self.register.data_ptr(), s)
            else:
                _lib.call("wb_face_flux_ops", self.precision, pool.data_ptr(), self.patches.data_ptr(),
                          self.face_flux_ops.data_ptr(), self.nface, b[0], b[1], b[2], self.gamma, self.limiter,
                          self.register.data_ptr(), s)
            self.launches += 1

    def reflux(self, pool):
        """Coarse cells beside fine patches take the register's correction (then cleared)."""
        size = _lib.REFLUX_OP.itemsize
        for start, count in self.reflux_phases:
            _lib.call("wb_reflux_apply", self.precision, pool.data_ptr(), self.patches.data_ptr(),
                      self.reflux_ops.data_ptr() + start * size, count, self.register.data_ptr(),
                      self.dt.data_ptr(), self._s())
            self.launches += 1

    def capture(self, step):
        """A CUDA graph of the launches `step()` issues. `step` runs once outside the graph
        first (lazy loading and launch attributes happen there, not in the recording)."""
        stream = torch.cuda.Stream(self.device)
        stream.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(stream):
            step()
        torch.cuda.current_stream(self.device).wait_stream(stream)
        torch.cuda.synchronize(self.device)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            step()
        torch.cuda.synchronize(self.device)
        return graph

    def heun_step(self, groups_potential, groups_all):
        """One Heun step with the dt already in self.dt (device), refluxed and restricted."""
        self.dt_ready = False
        with self.launching():
            self._heun_launches(groups_potential, groups_all)

    @contextlib.contextmanager
    def launching(self):
        """A run of launches on the engine's stream as it is now (its handle looked up once,
        not per launch)."""
        outer = self._step_stream
        if outer is None:
            self._step_stream = self._main().cuda_stream
        try:
            yield
        finally:
            self._step_stream = outer

    def _heun_launches(self, groups_potential, groups_all):
        U, U1 = self.state, self.stage_pool
        refined = self.max_level > 0
        self.stage(U, None, U1)
        side = None
        if self.overlap_fluxes and self.nface:
            # stage 1's register kernel beside the restriction and fill of U1 (small,
            # latency-bound launches that leave the SMs idle), not beside the stage kernel
            if self._flux_stream is None:
                self._flux_stream = torch.cuda.Stream(self.device)
                self._flux_events = (torch.cuda.Event(), torch.cuda.Event())
            side, main = self._flux_stream, self._main()
            forked, joined = self._flux_events
            forked.record(main)
            side.wait_event(forked)
        self.face_fluxes(U, side)
        if refined:
            self.restrict(U1, groups_potential)
        self.fill(U1)
        if side is not None:
            joined.record(side)
            main.wait_event(joined)  # stage 1's fluxes have read U before stage 2 writes it
        self.stage(U1, U, U)
        self.face_fluxes(U1)
        self.reflux(U)
        if refined:
            self.restrict(U, groups_all)
        self.fill(U)

    # op programs ------------------------------------------------------------------------------
    def _fill_phases(self, pool):
        """Phases of the halo fill of every level of pool (0: the state, 1: the stage pool),
        as `fill` launches them."""
        phases = []
        for level in range(len(self.copy_phases)):
            same, nsame, boundary = self.copy_phases[level]
            interp, ninterp = self.interp_levels[level]
            # the interpolation ops are trimmed to the points no copy writes: one phase
            phases.append([s for s in (("interp", pool, interp, ninterp), ("copy", pool, same, nsame)) if s[3]])
            phases.extend([("copy", pool, ops, nops)] for ops, nops in boundary if nops)
        return phases

    def _restrict_phases(self, pool, groups):
        """Phases of the restriction of `groups` in pool, finest level first, as `restrict`
        launches them."""
        key = frozenset(groups)
        phases = []
        for level in range(self.max_level, 0, -1):
            merged = self.restrict_merged.get(level)
            if merged is not None and merged[0] == key:
                phases.append([("restrict", pool, merged[1], merged[2])] if merged[2] else [])
            else:
                phases.append([("restrict", pool, *self.restrict_levels[level][g]) for g in groups
                               if self.restrict_levels[level][g][1]])
        return phases

    def _program(self, phases, dt_params=None):
        """An op program (segment records, parameters, counters) from phases of segments
        (kind, pool, ops tensor or None, count[, aux tensor]); empty phases dropped."""
        phases = [p for p in phases if p]
        rows = []
        for k, phase in enumerate(phases):
            for seg in phase:
                kind, pool, ops, count = seg[:4]
                aux = seg[4] if len(seg) > 4 else None
                rows.append((_lib.SEGMENT_KINDS[kind], pool, k, int(count), 0, 0,
                             0 if ops is None else ops.data_ptr(), 0 if aux is None else aux.data_ptr()))
        if len(rows) > _lib.PROGRAM_MAX_SEGMENTS:
            raise ValueError(f"an op program of {len(rows)} segments (at most {_lib.PROGRAM_MAX_SEGMENTS})")
        segments = np.array(rows, dtype=_lib.PROGRAM_SEGMENT) if rows else np.zeros(0, _lib.PROGRAM_SEGMENT)
        params = _lib.ProgramParams()
        for a in range(3):
            params.b0[a] = self.mean_field[a]
        params.gamma = self.gamma
        params.ndim = self.ndim
        params.ninstances = self.ninstances
        params.nlevels = self.nlevels
        params.reg = self.register.data_ptr()
        params.dt = self.dt.data_ptr()
        params.time = self.time.data_ptr()
        params.keys = self.keys.data_ptr()
        params.inv_dx2_sum = self.inv_dx2_sum.data_ptr()
        params.inv_dx2_levels = self.inv_dx2_levels.data_ptr()
        if self.per_level_dt:
            params.level_keys = self.level_keys.data_ptr()
        if dt_params is not None:
            params.cfl, params.dt_eta, params.dt_kappa = dt_params
        counters = torch.zeros(3 + len(phases), dtype=torch.int32, device=self.device)
        return segments, params, counters

    def programs(self, groups_potential, groups_all, dt_params=None):
        """The two op programs of a step: after stage 1 the restriction of the stage pool's
        potential and its halo fill; after stage 2 the reflux, the state's restriction and
        halo fill and, with dt_params (cfl, eta, kappa), the time advanced by this step's
        dt first and the next step's dt from the new state last."""
        key = (tuple(groups_potential), tuple(groups_all), dt_params, self.per_level_dt)
        found = self._programs.get(key)
        if found is None:
            first = self._restrict_phases(1, groups_potential) + self._fill_phases(1)
            second = [[("advance_time", 0, None, 1), ("init_keys", 0, None, 1)]] if dt_params is not None else []
            size = _lib.REFLUX_OP.itemsize
            second += [[("reflux", 0, self.reflux_ops[start * size:], count)] for start, count in self.reflux_phases]
            second += self._restrict_phases(0, groups_all) + self._fill_phases(0)
            if dt_params is not None:
                if self.nchunks:
                    second.append([("rate", 0, self.chunk_patch, self.nchunks, self.chunk_start)])
                second.append([("finalize_dt", 0, None, 1)])
            found = (self._program(first), self._program(second, dt_params))
            self._programs[key] = found
        return found

    def run_program(self, program):
        segments, params, counters = program
        if segments.size == 0:
            return
        _lib.call("wb_run_program", self.precision, self.state.data_ptr(), self.stage_pool.data_ptr(),
                  self.patches.data_ptr(), segments.ctypes.data, int(segments.size), ctypes.addressof(params),
                  counters.data_ptr(), self._s())
        self.launches += 1

    def program_error(self):
        """The error bits the op programs have set since the last call (0: none); cleared."""
        bits = 0
        for pair in self._programs.values():
            for _, _, counters in pair:
                bits |= int(counters[2].item())
                counters[2].zero_()
        return bits

    def prime_dt(self, cfl, eta=0.0, kappa=0.0):
        """dt of the next programmed step from the current state (time not advanced)."""
        with self.launching():
            self.rate()
            self.finalize_dt(cfl, eta, kappa, advance=False)
        self.dt_ready = True

    def programmed_step(self, groups_potential, groups_all, cfl, eta=0.0, kappa=0.0):
        """One Heun step through op programs at the dt on the device (`prime_dt` before the
        first, then each step leaves the next one): stage 1, the register's face fluxes
        (beside program 1), program 1, stage 2, face fluxes, program 2. Equal, bit for
        bit, to rate, finalize_dt(advance) and `heun_step` at the same dt."""
        first, second = self.programs(groups_potential, groups_all, (float(cfl), float(eta), float(kappa)))
        with self.launching():
            U, U1 = self.state, self.stage_pool
            self.stage(U, None, U1)
            side = None
            if self.overlap_fluxes and self.nface:
                if self._flux_stream is None:
                    self._flux_stream = torch.cuda.Stream(self.device)
                    self._flux_events = (torch.cuda.Event(), torch.cuda.Event())
                side, main = self._flux_stream, self._main()
                forked, joined = self._flux_events
                forked.record(main)
                side.wait_event(forked)
            self.face_fluxes(U, side)
            self.run_program(first)
            if side is not None:
                joined.record(side)
                main.wait_event(joined)  # stage 1's fluxes have read U before stage 2 writes it
            self.stage(U1, U, U)
            self.face_fluxes(U1)
            self.run_program(second)
        self.dt_ready = True  # the second program left the next step's dt

    # host views --------------------------------------------------------------------------------
    def view(self, pool, patch, field):
        return self.layout.patch_view(pool, patch, field)
