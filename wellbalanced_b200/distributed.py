"""A hierarchy partitioned over ranks: patches per GPU, halo exchange, a global time step.

The reference decomposes by whole patches over MPI ranks (``carafe/mhd.py:96-98``,
``tests/unit/test_mhd_mpi.py:31-51``): each rank advances its patches, patchwork's halo
exchange, restriction and flux register move data between ranks, and the time step is an
allreduce MIN (``carafe/mhd.py:963``). Here:

* `partition` gives every patch an owner: per level, Morton order of the patch origins
  cut into ``world`` runs of nearly equal cell counts;
* `RankLayout` is the part of a global `wellbalanced_b200.mesh.Layout` one rank holds: its
  patches (renumbered, packed into its own pool), tiles and rate chunks, and the op lists
  of the patches it writes: halos (copies, interpolation from below, boundary faces) of
  its patches, restriction into and face fluxes / reflux of its coarse patches. An op
  whose source patch lives on another rank reads a *proxy*: the box of the source patch
  the op's footprint covers (every field), shipped from the owner into a dense block of
  this rank's pool and described by a patch row with the source's haloed coordinates, so
  the op itself is unchanged. Shipping happens in *rounds*, one per point of the step
  where a source must be current: halo fill of each level, the face fluxes of a stage,
  the restriction of each level and field group. In a round every owner packs its boxes
  (copy ops, ``wb_copy_ops``) into mailboxes, one contiguous slice per peer, the slices
  are exchanged, and the receiving ops run;
* `DistributedEngine` runs a step on a RankLayout (its fill, restriction and face fluxes
  take their rounds first; dt is the global max rate and min density, an all-reduce MAX
  of the order-preserving keys with the min key bit-complemented);
* `LocalCluster` holds every rank of a partition in one process on one device and moves
  the mailboxes by device copies: the same ops, for checking a partition on one GPU.

Exchange and reduction go through a transport object: `TorchTransport` (process groups:
NCCL between GPUs, gloo on CPUs) or any object with the same two methods.
"""

from __future__ import annotations

import numpy as np
import torch

from wellbalanced_b200 import _lib
from wellbalanced_b200.engine import Engine, _device_bytes
from wellbalanced_b200.mesh import _concat, size_ops, split_box_ops

#: patch-row flag of a dense block that stands for a box of a patch (kProxy in layout.cuh)
PROXY = 1 << 30


def _morton(point, bits=16):
    code = 0
    for b in range(bits):
        for a, v in enumerate(point):
            code |= ((int(v) >> b) & 1) << (b * len(point) + a)
    return code


def partition(hierarchy, world):
    """Owner rank of every patch (list indexed by patch index): each level's patches in
    Morton order of their origins, cut into ``world`` runs of nearly equal cell counts."""
    owner = [0] * len(hierarchy.patches)
    for level in range(hierarchy.max_level + 1):
        patches = hierarchy.patches_at_level(level)
        order = sorted(patches, key=lambda p: _morton([lo for lo, _ in p.box]))
        cells = np.array([int(np.prod(p.shape)) for p in order], dtype=float)
        target = cells.sum() / world
        running, rank = 0.0, 0
        for p, c in zip(order, cells, strict=True):
            if running + 0.5 * c > target * (rank + 1) and rank < world - 1:
                rank += 1
            owner[p.index] = rank
            running += c
    return owner


# read footprints of the op kernels (csrc/halo.cu, csrc/reflux.cu), as inclusive boxes of
# haloed indices of the source patch ---------------------------------------------------------
def _copy_footprints(op):
    """(source, lo, hi) of each source a copy op reads: src1 + m1 p, and src2 where w2 != 0."""
    out = []
    n = [int(v) for v in op["n"]]
    for key, s, m in (("src1", "s1", "m1"), ("src2", "s2", "m2")):
        if key == "src2" and float(op["w2"]) == 0.0:
            continue
        src = int(op[key]) if key == "src1" or int(op["src2"]) >= 0 else int(op["src1"])
        first = [int(op[s][a]) for a in range(3)]
        last = [int(op[s][a]) + int(op[m][a]) * (n[a] - 1) for a in range(3)]
        out.append((src, [min(x, y) for x, y in zip(first, last)], [max(x, y) for x, y in zip(first, last)]))
    return out


def _interp_footprint(op):
    """The coarse points an interpolation op reads (linear along cell axes, the coincident
    node or the 4-point midpoint along node axes)."""
    lo, hi = [0, 0, 0], [0, 0, 0]
    for a in range(int(op["ndim"])):
        node = (int(op["node_mask"]) >> a) & 1
        first = int(op["d"][a]) - 2 + int(op["fine_lo"][a])
        cmin, cmax = None, None
        for g in range(first, first + int(op["n"][a])):
            if node:
                c0, cnt = (g // 2, 1) if g % 2 == 0 else (g // 2 - 1, 4)
            else:
                c0, cnt = (g // 2 - 1, 2) if g % 2 == 0 else (g // 2, 2)
            cmin = c0 if cmin is None else min(cmin, c0)
            cmax = c0 + cnt - 1 if cmax is None else max(cmax, c0 + cnt - 1)
        lo[a] = cmin - int(op["coarse_lo"][a]) + 2
        hi[a] = cmax - int(op["coarse_lo"][a]) + 2
    return int(op["coarse"]), lo, hi


def _restrict_footprint(op):
    """The fine points a restriction op reads: 2 per coarse point along cell axes, 1 along
    node axes."""
    lo, hi = [0, 0, 0], [0, 0, 0]
    for a in range(3):
        cnt = 2 if a < int(op["ndim"]) and not (int(op["node_mask"]) >> a) & 1 else 1
        lo[a] = int(op["f"][a])
        hi[a] = int(op["f"][a]) + 2 * (int(op["n"][a]) - 1) + cnt - 1
    return int(op["fine"]), lo, hi


def _flux_footprint(op):
    """The fine points a face-flux op reads around its fine faces: along the normal the
    four cells of the reconstruction and their upper potentials (normal index - 2 .. + 2),
    across it one more on each side for the resistive and conductive terms (- 1 .. + 2)."""
    lo, hi = [0, 0, 0], [0, 0, 0]
    axis = int(op["axis"])
    lo[axis], hi[axis] = int(op["fine_plane"]) - 2, int(op["fine_plane"]) + 2
    length, width = int(op["len"]), int(op["width"])
    spans = [(int(op["t1"]), int(op["fine_t0"][0]), length // width)]
    if int(op["ndim"]) == 3:
        spans.append((int(op["t2"]), int(op["fine_t0"][1]), width))
    for t, t0, count in spans:
        lo[t], hi[t] = t0 - 1, t0 + 2 * count + 1
    return int(op["fine"]), lo, hi


def _rounds(layout):
    """The exchange rounds of a step, in a fixed order every rank agrees on."""
    levels = len(layout.copy_phases)
    out = [("fill", level) for level in range(levels)] + [("flux",)]
    for level in range(1, levels):
        out += [("restrict", level, g) for g in layout.restrict_levels[level]]
    return out


def _needs(layout, owner, rank):
    """For each round, the boxes of other ranks' patches the ops of `rank` read:
    {round: {source patch: (lo, hi)}} (inclusive haloed indices, clipped to the source)."""
    rows = layout.rows
    needs = {key: {} for key in _rounds(layout)}

    def need(key, src, lo, hi, clip=False):
        if owner[src] == rank:
            return
        extent = [int(rows[src]["n"][a]) + 4 if a < layout.ndim else 0 for a in range(3)]
        if clip:
            lo = [max(v, 0) for v in lo]
            hi = [min(v, e) for v, e in zip(hi, extent)]
        if any(v < 0 for v in lo) or any(v > e for v, e in zip(hi, extent)):
            raise RuntimeError(f"an op reads outside the haloed patch {src}: {lo}..{hi}")
        box = needs[key].get(src)
        if box is not None:
            lo = [min(x, y) for x, y in zip(box[0], lo)]
            hi = [max(x, y) for x, y in zip(box[1], hi)]
        needs[key][src] = (lo, hi)

    for level, (same, boundary) in enumerate(layout.copy_phases):
        key = ("fill", level)
        for op in np.atleast_1d(same):
            if owner[int(op["dst"])] == rank:
                for src, lo, hi in _copy_footprints(op):
                    need(key, src, lo, hi)
        for ops in boundary:
            for op in np.atleast_1d(ops):
                if owner[int(op["dst"])] == rank and any(owner[src] != rank for src, _, _ in _copy_footprints(op)):
                    raise NotImplementedError("a boundary op reading another rank's patch")
        for op in np.atleast_1d(layout.interp_levels[level]):
            if owner[int(op["fine"])] == rank:
                need(key, *_interp_footprint(op))
    for op in np.atleast_1d(layout.face_flux_ops):
        if owner[int(op["coarse"])] == rank:
            need(("flux",), *_flux_footprint(op), clip=True)
    for level in range(1, len(layout.copy_phases)):
        for g, ops in layout.restrict_levels[level].items():
            for op in np.atleast_1d(ops):
                if owner[int(op["coarse"])] == rank:
                    need(("restrict", level, g), *_restrict_footprint(op))
    return needs


class Round:
    """One exchange round of a rank: pack ops (own boxes -> mailboxes), the pool slices
    sent to / received from each peer ((start, length) per peer rank), and the proxy row
    of each received source patch."""

    def __init__(self):
        self.pack_ops = []
        self.send = {}
        self.recv = {}
        self.proxies = {}


class RankLayout:
    """One rank's share of a global Layout (see the module docstring)."""

    def __init__(self, layout, owner, rank):
        self.rank = rank
        self.world = max(owner) + 1
        self.ndim = layout.ndim
        self.nfields = layout.nfields
        self.groups = layout.groups
        self.precision = layout.precision
        self.lx = layout.lx
        self.tile_shape = layout.tile_shape
        self.default_tile = getattr(layout, "default_tile", layout.tile_shape)
        self.walls = layout.walls
        self.max_level = layout.max_level
        self.h = None
        local = [g for g in range(layout.npatches) if owner[g] == rank]
        self.local = local
        gmap = {g: i for i, g in enumerate(local)}
        self._gmap = gmap
        self.own = [layout.own[g] for g in local]
        rows = [r.copy() for r in layout.rows[local]]
        offset = 0
        for r in rows:
            r["off"] = offset
            r["instance"] = 0
            r["bflux"] = -1
            offset += int(r["fstride"]) * self.nfields
        # proxies address their blocks through the source's haloed coordinates: keep the
        # mailboxes above the largest shift that needs, so every row offset stays >= 0
        offset = max(offset, max((int(r["fstride"]) for r in layout.rows), default=0))
        nf = self.nfields

        def dense_row(src, lo, hi):
            """A patch row over a dense block of every field of box lo..hi of `src`."""
            nonlocal offset
            n = [h - l + 1 for l, h in zip(lo, hi)]
            volume = n[0] * n[1] * n[2]
            row = layout.rows[src].copy()
            row["fstride"] = volume
            if self.ndim == 2:
                row["pitch0"], row["pitch1"] = n[1], 0
                shift = lo[0] * n[1] + lo[1]
            else:
                row["pitch0"], row["pitch1"] = n[1] * n[2], n[2]
                shift = lo[0] * n[1] * n[2] + lo[1] * n[2] + lo[2]
            row["instance"], row["bflux"] = 0, -1
            row["flags"] = int(row["flags"]) | PROXY
            start = offset
            offset += nf * volume
            return row, start, shift, n

        plans = [_needs(layout, owner, r) for r in range(self.world)]
        self.rounds = {}
        for key in _rounds(layout):
            rd = Round()
            for peer in range(self.world):  # this rank's boxes for each peer
                first = None
                for src in sorted(plans[peer][key]):
                    if owner[src] != rank or peer == rank:
                        continue
                    lo, hi = plans[peer][key][src]
                    row, start, shift, n = dense_row(src, lo, hi)
                    if n[0] * n[1] * n[2] >= 2**31:  # the copy kernel indexes an op's points in 32 bits
                        raise ValueError(f"a mailbox box of {n} points")
                    row["off"] = start  # the pack op writes box index 0.. here
                    rows.append(row)
                    first = start if first is None else first
                    op = np.zeros((), dtype=_lib.COPY_OP)
                    op["dst"], op["src1"], op["src2"] = len(rows) - 1, gmap[src], -1
                    op["field_lo"], op["field_hi"], op["negate"] = 0, nf, -1
                    op["n"], op["d"], op["s1"], op["m1"] = n, [0, 0, 0], lo, [1, 1, 1]
                    op["s2"], op["m2"], op["w1"], op["w2"] = [0, 0, 0], [0, 0, 0], 1.0, 0.0
                    rd.pack_ops.append(op)
                if first is not None:
                    rd.send[peer] = (first, offset - first)
            for peer in range(self.world):  # the boxes each peer sends this rank
                first = None
                for src in sorted(plans[rank][key]):
                    if owner[src] != peer:
                        continue
                    lo, hi = plans[rank][key][src]
                    row, start, shift, _ = dense_row(src, lo, hi)
                    row["off"] = start - shift
                    if int(row["off"]) < 0:
                        raise RuntimeError("proxy offset below the pool")
                    rows.append(row)
                    rd.proxies[src] = len(rows) - 1
                    first = start if first is None else first
                if first is not None:
                    rd.recv[peer] = (first, offset - first)
            rd.pack_ops = split_box_ops(_concat(rd.pack_ops, _lib.COPY_OP))
            self.rounds[key] = rd

        def index(key, g):
            return gmap[g] if owner[g] == rank else self.rounds[key].proxies[g]

        copy_phases, interp_levels = [], []
        for level, (same, boundary) in enumerate(layout.copy_phases):
            key = ("fill", level)
            kept = []
            for op in np.atleast_1d(same):
                if owner[int(op["dst"])] != rank:
                    continue
                o = op.copy()
                o["dst"], o["src1"] = gmap[int(op["dst"])], index(key, int(op["src1"]))
                o["src2"] = index(key, int(op["src2"])) if int(op["src2"]) >= 0 else -1
                kept.append(o)
            local_boundary = []
            for ops in boundary:
                mine = []
                for op in np.atleast_1d(ops):
                    if owner[int(op["dst"])] != rank:
                        continue
                    o = op.copy()
                    for k in ("dst", "src1", "src2"):
                        if int(o[k]) >= 0:
                            o[k] = gmap[int(o[k])]
                    mine.append(o)
                local_boundary.append(_concat(mine, _lib.COPY_OP))
            copy_phases.append((_concat(kept, _lib.COPY_OP), local_boundary))
            interp = []
            for op in np.atleast_1d(layout.interp_levels[level]):
                if owner[int(op["fine"])] != rank:
                    continue
                o = op.copy()
                o["fine"], o["coarse"] = gmap[int(op["fine"])], index(key, int(op["coarse"]))
                interp.append(o)
            interp_levels.append(_concat(interp, _lib.INTERP_OP))
        self.copy_phases = copy_phases
        self.interp_levels = interp_levels
        self.restrict_levels = {}
        for level, groups in layout.restrict_levels.items():
            self.restrict_levels[level] = {}
            for g, ops in groups.items():
                mine = []
                for op in np.atleast_1d(ops):
                    if owner[int(op["coarse"])] != rank:
                        continue
                    o = op.copy()
                    o["coarse"], o["fine"] = gmap[int(op["coarse"])], index(("restrict", level, g), int(op["fine"]))
                    mine.append(o)
                self.restrict_levels[level][g] = _concat(mine, _lib.RESTRICT_OP)
        faces = []
        for op in np.atleast_1d(layout.face_flux_ops):
            if owner[int(op["coarse"])] != rank:
                continue
            o = op.copy()
            o["coarse"], o["fine"] = gmap[int(op["coarse"])], index(("flux",), int(op["fine"]))
            faces.append(o)
        self.face_flux_ops = _concat(faces, _lib.FACE_FLUX_OP)
        self.reflux_phases = []
        for ops in layout.reflux_phases:
            mine = []
            for op in np.atleast_1d(ops):
                if owner[int(op["coarse"])] == rank:
                    o = op.copy()
                    o["coarse"] = gmap[int(op["coarse"])]
                    mine.append(o)
            self.reflux_phases.append(_concat(mine, _lib.REFLUX_OP))
        self.register_size = layout.register_size
        self.rows = np.array(rows, dtype=_lib.PATCH) if rows else np.zeros(0, _lib.PATCH)
        self.npatches = len(local)
        # slack after the last mailbox, one field of the largest patch: the pool ends no
        # closer to a block than any of its patches' own stencils reach
        self.pool_size = offset + max((int(r["fstride"]) for r in layout.rows), default=0)
        tiles = layout.tiles[np.isin(layout.tiles["patch"], local)].copy()
        tiles["patch"] = [gmap[int(t)] for t in tiles["patch"]]
        self.tiles = tiles
        keep = np.isin(layout.chunk_patch, local)
        self.chunk_patch = np.array([gmap[int(c)] for c in layout.chunk_patch[keep]], dtype=np.int32)
        self.chunk_start = layout.chunk_start[keep].astype(np.int32)
        self.inv_dx2_sum = layout.inv_dx2_sum[:1].copy()
        self.inv_dx2_levels = getattr(layout, "inv_dx2_levels", layout.inv_dx2_sum[:, None])[:1].copy()
        self.instances = np.zeros(len(local), dtype=np.int32)
        self.ninstances = 1

    @property
    def reflux_ops(self):
        return _concat(self.reflux_phases, _lib.REFLUX_OP)

    def owns(self, patch):
        """Whether the hierarchy's patch lives on this rank."""
        return patch.index in self._gmap

    def patch_view(self, pool, p, f):
        """A view of field f of this rank's patch p (a hierarchy patch) in `pool`."""
        r = self.rows[self._gmap[p.index]]
        start = int(r["off"] + f * r["fstride"])
        if self.ndim == 2:
            X, P0 = p.shape[0] + 5, int(r["pitch0"])
            return pool[start : start + X * P0].reshape(X, P0)[:, : p.shape[1] + 5]
        X, Y = p.shape[0] + 5, p.shape[1] + 5
        P0, P1 = int(r["pitch0"]), int(r["pitch1"])
        return pool[start : start + X * P0].reshape(X, Y, P1)[:, :, : p.shape[2] + 5]

    def block(self, local_index):
        """(start, size) of a local patch's fields in the rank's pool."""
        r = self.rows[local_index]
        return int(r["off"]), int(r["fstride"]) * self.nfields

    def mailbox_range(self):
        """(start, end) of the pool's mailbox area (after the local patches)."""
        end = max((self.block(i)[0] + self.block(i)[1] for i in range(self.npatches)), default=0)
        return end, self.pool_size


def _keys_to_max_form(keys):
    """Keys (max rate, min density) per instance as int64 values whose MAX all-reduce gives
    the max rate key and the complement of the min density key (uint64 order kept: the
    rate keys of non-negative rates all have the top bit set, the complemented density
    keys all have it clear, so the signed order agrees with the unsigned one)."""
    k = keys.view(torch.int64).clone().view(-1, 2)
    k[:, 1] = torch.bitwise_not(k[:, 1])
    return k


def _keys_from_max_form(k, keys):
    k = k.clone()
    k[:, 1] = torch.bitwise_not(k[:, 1])
    keys.view(torch.int64).copy_(k.view(-1))


class TorchTransport:
    """Exchange and reductions over a ``torch.distributed`` process group. With NCCL the
    point-to-point transfers are ordered on the launching stream (`stream_ordered`); with
    gloo the mailboxes go through host memory."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        #: NCCL orders its transfers after the launching stream's pending work
        self.stream_ordered = dist.get_backend(group) == "nccl"

    def _host(self, view):
        return view if self.stream_ordered else view.cpu()

    def exchange(self, pool, send, recv):
        ops, landed = [], []
        for peer, (start, length) in sorted(send.items()):
            ops.append(self.dist.P2POp(self.dist.isend, self._host(pool[start : start + length]), peer, self.group))
        for peer, (start, length) in sorted(recv.items()):
            box = pool[start : start + length]
            buffer = self._host(box)
            landed.append((box, buffer))
            ops.append(self.dist.P2POp(self.dist.irecv, buffer, peer, self.group))
        if ops:
            for request in self.dist.batch_isend_irecv(ops):
                request.wait()
        for box, buffer in landed:
            if buffer is not box:
                box.copy_(buffer)

    def reduce_min_keys(self, keys):
        """All-reduce MIN of order-preserving keys (as a MAX of their complements)."""
        k = torch.bitwise_not(keys.view(torch.int64))
        if self.stream_ordered:
            self.dist.all_reduce(k, op=self.dist.ReduceOp.MAX, group=self.group)
        else:
            host = k.cpu()
            self.dist.all_reduce(host, op=self.dist.ReduceOp.MAX, group=self.group)
            k.copy_(host)
        keys.view(torch.int64).copy_(torch.bitwise_not(k))

    def reduce_keys(self, keys):
        k = _keys_to_max_form(keys)
        if self.stream_ordered:
            self.dist.all_reduce(k, op=self.dist.ReduceOp.MAX, group=self.group)
        else:
            host = k.cpu()
            self.dist.all_reduce(host, op=self.dist.ReduceOp.MAX, group=self.group)
            k.copy_(host)
        _keys_from_max_form(k, keys)


class DistributedEngine(Engine):
    """`Engine` on one rank's share of a hierarchy: fills, restriction and face fluxes
    take their exchange rounds first; dt is global."""

    def __init__(self, rank_layout, transport, **options):
        super().__init__(None, layout=rank_layout, **options)
        self.transport = transport
        self.overlap_fluxes = False  # the flux round's exchange runs on the engine's stream
        # exchange rounds run between the levels' fills and restrictions: no op programs
        self.use_programs = False
        # the fine faces of an interface may live on another rank: recomputed from proxies
        self.staged_fluxes = False
        self.rounds = {}
        for key, rd in rank_layout.rounds.items():
            ops = size_ops(rd.pack_ops) if rd.pack_ops.size else rd.pack_ops
            self.rounds[key] = (_device_bytes(ops, self.device, _lib.COPY_OP), int(ops.size), rd.send, rd.recv)

    def pack(self, pool, key):
        """Copy this rank's boxes of round `key` into their mailboxes."""
        ops, nops, _, _ = self.rounds[key]
        if nops:
            _lib.call("wb_copy_ops", self.precision, pool.data_ptr(), self.patches.data_ptr(), ops.data_ptr(), nops,
                      self._s())
            self.launches += 1

    def exchange(self, pool, key):
        """Pack, then swap the mailboxes of round `key` with the peers. A transport on the
        device's stream (NCCL: its sends start after the pack on that stream and the
        stream waits for its receives) needs no host synchronisation; any other transport
        gets the packed mailboxes after the stream has drained."""
        self.pack(pool, key)
        _, _, send, recv = self.rounds[key]
        if send or recv:
            if not getattr(self.transport, "stream_ordered", False):
                torch.cuda.current_stream(self.device).synchronize()
            self.transport.exchange(pool, send, recv)

    def fill(self, pool, levels=None):
        for level in range(len(self.copy_phases)):
            if levels is None or level in levels:
                self.exchange(pool, ("fill", level))
                self._fill_level(pool, level)

    def restrict(self, pool, groups):
        for level in range(self.layout.max_level, 0, -1):
            for g in groups:
                self.exchange(pool, ("restrict", level, g))
                self._restrict_level(pool, level, g)

    def face_fluxes(self, pool, stream=None):
        if self.layout.max_level > 0:
            self.exchange(pool, ("flux",))
        Engine.face_fluxes(self, pool)

    def finalize_dt(self, cfl, eta=0.0, kappa=0.0, *, clip_to_end=False, advance=False):
        self.transport.reduce_keys(self.keys)
        if self.per_level_dt:
            self.transport.reduce_min_keys(self.level_keys)
        Engine.finalize_dt(self, cfl, eta, kappa, clip_to_end=clip_to_end, advance=advance)

    def step(self, cfl):
        """One Heun step of this rank's patches at the global stable dt."""
        self.rate()
        self.finalize_dt(cfl, advance=True)
        groups = self.layout.groups
        self.heun_step(groups[1:], groups)


class LocalCluster:
    """Every rank of a partition in one process on one device, in lockstep: the ops of
    `DistributedEngine`, with the mailboxes moved by device copies between the pools."""

    def __init__(self, layout, owner, **options):
        world = max(owner) + 1
        self.layout = layout
        self.parts = [RankLayout(layout, owner, r) for r in range(world)]
        self.engines = [DistributedEngine(part, transport=None, **options) for part in self.parts]

    def _round(self, pool_name, key):
        pools = [getattr(e, pool_name) for e in self.engines]
        for e, pool in zip(self.engines, pools, strict=True):
            e.pack(pool, key)
        for r, e in enumerate(self.engines):
            for peer, (start, length) in e.rounds[key][3].items():
                s_start, s_length = self.engines[peer].rounds[key][2][r]
                if s_length != length:
                    raise RuntimeError("mailboxes of a rank pair do not match")
                pools[r][start : start + length].copy_(pools[peer][s_start : s_start + s_length])
        return pools

    def fill(self, pool_name):
        for level in range(len(self.layout.copy_phases)):
            pools = self._round(pool_name, ("fill", level))
            for e, pool in zip(self.engines, pools, strict=True):
                e._fill_level(pool, level)

    def restrict(self, pool_name, groups):
        for level in range(self.layout.max_level, 0, -1):
            for g in groups:
                pools = self._round(pool_name, ("restrict", level, g))
                for e, pool in zip(self.engines, pools, strict=True):
                    e._restrict_level(pool, level, g)

    def face_fluxes(self, pool_name):
        pools = self._round(pool_name, ("flux",))
        for e, pool in zip(self.engines, pools, strict=True):
            Engine.face_fluxes(e, pool)

    def reduce_keys(self):
        forms = torch.stack([_keys_to_max_form(e.keys) for e in self.engines])
        top = forms.max(dim=0).values
        for e in self.engines:
            _keys_from_max_form(top, e.keys)

    def step(self, cfl, eta=0.0, kappa=0.0):
        """One Heun step of every rank at the global stable dt, in the order of
        `Engine.heun_step`."""
        for e in self.engines:
            e.rate()
        self.reduce_keys()
        for e in self.engines:
            Engine.finalize_dt(e, cfl, eta, kappa, advance=True)
        groups = self.layout.groups
        refined = self.layout.max_level > 0
        for e in self.engines:
            e.stage(e.state, None, e.stage_pool)
        self.face_fluxes("state")
        if refined:
            self.restrict("stage_pool", groups[1:])
        self.fill("stage_pool")
        for e in self.engines:
            e.stage(e.stage_pool, e.state, e.state)
        self.face_fluxes("stage_pool")
        for e in self.engines:
            e.reflux(e.state)
        if refined:
            self.restrict("state", groups)
        self.fill("state")


# ---- the solvers on a partitioned hierarchy ------------------------------------------------
def solver_group(hierarchy):
    """The process group of a hierarchy (``AMRHierarchy(..., comm=group)``, as the reference
    passes its MPI communicator) when it spans more than one rank, else None."""
    comm = getattr(hierarchy, "comm", None)
    if comm is None:
        return None
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size(comm) <= 1:
        return None
    return comm


def solver_engine(hierarchy, group, *, walls=None, lx=32, **options):
    """A `DistributedEngine` on this rank's share of the hierarchy: the patches of every
    level in Morton order, cut into runs of nearly equal cells per rank (`partition`)."""
    import torch.distributed as dist

    from wellbalanced_b200.mesh import Layout

    layout = Layout(hierarchy, walls=walls, precision=_lib.precision_code(options.get("precision", 32)), lx=lx)
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    owner = partition(hierarchy, world)
    return DistributedEngine(RankLayout(layout, owner, rank), TorchTransport(group), **options)


def local_patches(model):
    """The hierarchy's patches this rank holds (all of them without a partition)."""
    layout = model.engine.layout
    if hasattr(layout, "owns"):
        return [p for p in model.hierarchy.patches if layout.owns(p)]
    return list(model.hierarchy.patches)


def all_reduce(model, values, op):
    """values (a list of floats) reduced over the model's ranks (op "sum" or "max")."""
    group = getattr(model, "_group", None)
    if group is None:
        return values
    import torch.distributed as dist

    t = torch.tensor(values, dtype=torch.float64)
    if dist.get_backend(group) == "nccl":
        t = t.to(model.engine.device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM if op == "sum" else dist.ReduceOp.MAX, group=group)
    return [float(v) for v in t.cpu()]
