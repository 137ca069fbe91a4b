"""A level partitioned over ranks: patches per GPU, halo exchange, a global time step.

The reference decomposes by whole patches over MPI ranks (``carafe/mhd.py:96-98``,
``tests/unit/test_mhd_mpi.py:31-51``): each rank advances its patches, patchwork's halo
exchange moves ghost layers between ranks, and the time step is an allreduce MIN
(``carafe/mhd.py:963``). Here, for one level (uniform grids split into patches):

* `partition` gives every patch an owner: Morton order of the patch origins, cut into
  ``world`` runs of nearly equal cell counts;
* `RankLayout` is the part of a global `wellbalanced_b200.mesh.Layout` one rank holds: its
  patches (renumbered, packed into its own pool), its tiles and rate chunks, its local
  halo copies, and the exchange plan. A same-level copy whose source patch lives on
  another rank becomes a pack op on the sender (source box -> a "mailbox", a dense block
  at the end of the sender's pool) and an unpack op on the receiver (its mailbox -> the
  halo box). Both sides walk the global op list in order, so the mailboxes of a pair of
  ranks line up; each peer's mailboxes are one contiguous slice of the pool, sent whole.
  Pack, unpack and local copies are the ordinary copy ops (``wb_copy_ops``);
* `DistributedEngine` runs a step on a RankLayout: fill = pack, exchange (one grouped
  send/recv per peer over ``torch.distributed``, NCCL on GPUs), local copies and unpacks,
  boundary faces; dt = the global max rate and min density (an all-reduce MAX of the
  order-preserving keys, the min key bit-complemented) before ``finalize_dt``;
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
from wellbalanced_b200.mesh import _concat


def _morton(point, bits=16):
    code = 0
    for b in range(bits):
        for a, v in enumerate(point):
            code |= ((int(v) >> b) & 1) << (b * len(point) + a)
    return code


def partition(hierarchy, world):
    """Owner rank of every patch of a one-level hierarchy (list indexed by patch index)."""
    if hierarchy.max_level != 0:
        raise NotImplementedError("the partition covers one level; refined hierarchies run on one rank")
    patches = hierarchy.patches
    order = sorted(patches, key=lambda p: _morton([lo for lo, _ in p.box]))
    cells = np.array([int(np.prod(p.shape)) for p in order], dtype=float)
    target = cells.sum() / world
    owner = [0] * len(patches)
    running, rank = 0.0, 0
    for p, c in zip(order, cells, strict=True):
        if running + 0.5 * c > target * (rank + 1) and rank < world - 1:
            rank += 1
        owner[p.index] = rank
        running += c
    return owner


class RankLayout:
    """One rank's share of a one-level global Layout (see the module docstring)."""

    def __init__(self, layout, owner, rank):
        if layout.max_level != 0:
            raise NotImplementedError("the partition covers one level")
        self.rank = rank
        self.world = max(owner) + 1
        self.ndim = layout.ndim
        self.nfields = layout.nfields
        self.groups = layout.groups
        self.precision = layout.precision
        self.lx = layout.lx
        self.tile_shape = layout.tile_shape
        self.walls = layout.walls
        self.max_level = 0
        self.h = None
        local = [g for g in range(layout.npatches) if owner[g] == rank]
        self.local = local
        gmap = {g: i for i, g in enumerate(local)}
        self.own = [layout.own[g] for g in local]
        rows = layout.rows[local].copy()
        offset = 0
        for r in rows:
            r["off"] = offset
            r["instance"] = 0
            offset += int(r["fstride"]) * self.nfields
        mailbox_rows = []

        def mailbox(op):
            """A dense block for op's box and fields at the end of the pool: (row, start)."""
            nonlocal offset
            n = [int(v) for v in op["n"]]
            volume = n[0] * n[1] * n[2]
            row = np.zeros((), dtype=_lib.PATCH)
            row["fstride"] = volume
            row["off"] = offset - int(op["field_lo"]) * volume  # field f at off + f * volume
            if int(row["off"]) < 0:
                raise ValueError("mailbox offset below the pool")
            if self.ndim == 2:
                row["pitch0"], row["pitch1"] = n[1], 0
            else:
                row["pitch0"], row["pitch1"] = n[1] * n[2], n[2]
            row["n"] = [n[0] - 5, n[1] - 5, n[2] - 5 if self.ndim == 3 else 1]
            row["flags"], row["level"], row["bflux"] = 0, 0, -1
            index = len(rows) + len(mailbox_rows)
            mailbox_rows.append(row)
            start = offset
            offset += (int(op["field_hi"]) - int(op["field_lo"])) * volume
            return index, start

        same, boundary = layout.copy_phases[0]
        local_ops, pack_ops, unpack_ops = [], [], []
        outgoing = {peer: [] for peer in range(self.world)}
        incoming = {peer: [] for peer in range(self.world)}
        for op in same:
            dst, src = int(owner[op["dst"]]), int(owner[op["src1"]])
            if op["src2"] >= 0 and int(owner[op["src2"]]) != src:
                raise NotImplementedError("two-source copies across ranks")
            if dst == rank and src == rank:
                o = op.copy()
                o["dst"], o["src1"] = gmap[int(op["dst"])], gmap[int(op["src1"])]
                o["src2"] = gmap[int(op["src2"])] if op["src2"] >= 0 else -1
                local_ops.append(o)
            elif src == rank:
                outgoing[dst].append(op)
            elif dst == rank:
                incoming[src].append(op)
        self.send, self.recv = {}, {}
        for peer in range(self.world):
            if outgoing[peer]:
                first = None
                for op in outgoing[peer]:
                    box, start = mailbox(op)
                    first = start if first is None else first
                    o = np.zeros((), dtype=_lib.COPY_OP)
                    o["dst"], o["src1"], o["src2"] = box, gmap[int(op["src1"])], -1
                    o["field_lo"], o["field_hi"], o["negate"] = op["field_lo"], op["field_hi"], -1
                    o["n"], o["d"] = op["n"], [0, 0, 0]
                    o["s1"], o["m1"] = op["s1"], op["m1"]
                    o["w1"], o["w2"] = 1.0, 0.0
                    pack_ops.append(o)
                self.send[peer] = (first, offset - first)
        for peer in range(self.world):
            if incoming[peer]:
                first = None
                for op in incoming[peer]:
                    box, start = mailbox(op)
                    first = start if first is None else first
                    o = op.copy()
                    o["dst"], o["src1"], o["src2"] = gmap[int(op["dst"])], box, -1
                    o["s1"], o["m1"] = [0, 0, 0], [1, 1, 1]
                    unpack_ops.append(o)
                self.recv[peer] = (first, offset - first)
        self.rows = np.concatenate([rows, np.array(mailbox_rows, dtype=_lib.PATCH)]) if mailbox_rows else rows
        self.npatches = len(local)
        self.pool_size = offset
        self.pack_ops = _concat(pack_ops, _lib.COPY_OP)
        boundary_local = []
        for ops in boundary:
            kept = [op.copy() for op in ops if owner[op["dst"]] == rank]
            for o in kept:
                for key in ("dst", "src1", "src2"):
                    if o[key] >= 0:
                        o[key] = gmap[int(o[key])]
            boundary_local.append(_concat(kept, _lib.COPY_OP))
        self.copy_phases = [(_concat(local_ops + unpack_ops, _lib.COPY_OP), boundary_local)]
        tiles = layout.tiles[np.isin(layout.tiles["patch"], local)].copy()
        tiles["patch"] = [gmap[int(t)] for t in tiles["patch"]]
        self.tiles = tiles
        keep = np.isin(layout.chunk_patch, local)
        self.chunk_patch = np.array([gmap[int(c)] for c in layout.chunk_patch[keep]], dtype=np.int32)
        self.chunk_start = layout.chunk_start[keep].astype(np.int32)
        self.inv_dx2_sum = layout.inv_dx2_sum[:1].copy()
        self.instances = np.zeros(len(local), dtype=np.int32)
        self.ninstances = 1
        self.interp_levels = [np.zeros(0, _lib.INTERP_OP)]
        self.restrict_levels = {0: {}}
        self.face_flux_ops = np.zeros(0, _lib.FACE_FLUX_OP)
        self.reflux_phases = [np.zeros(0, _lib.REFLUX_OP) for _ in range(2 * self.ndim)]
        self.register_size = 0

    @property
    def reflux_ops(self):
        return np.zeros(0, _lib.REFLUX_OP)

    def block(self, local_index):
        """(start, size) of a local patch's fields in the rank's pool."""
        r = self.rows[local_index]
        return int(r["off"]), int(r["fstride"]) * self.nfields


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
    """Exchange and reductions over a ``torch.distributed`` process group."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group

    def exchange(self, pool, send, recv):
        ops = []
        for peer, (start, length) in sorted(send.items()):
            ops.append(self.dist.P2POp(self.dist.isend, pool[start : start + length], peer, self.group))
        for peer, (start, length) in sorted(recv.items()):
            ops.append(self.dist.P2POp(self.dist.irecv, pool[start : start + length], peer, self.group))
        if ops:
            for request in self.dist.batch_isend_irecv(ops):
                request.wait()

    def reduce_keys(self, keys):
        k = _keys_to_max_form(keys)
        self.dist.all_reduce(k, op=self.dist.ReduceOp.MAX, group=self.group)
        _keys_from_max_form(k, keys)


class DistributedEngine(Engine):
    """`Engine` on one rank's share of a level: fills exchange halos, dt is global."""

    def __init__(self, rank_layout, transport, **options):
        super().__init__(None, layout=rank_layout, **options)
        self.transport = transport
        self.pack = _device_bytes(rank_layout.pack_ops, self.device, _lib.COPY_OP)
        self.npack = int(rank_layout.pack_ops.size)

    def pack_mailboxes(self, pool):
        if self.npack:
            _lib.call("wb_copy_ops", self.precision, pool.data_ptr(), self.patches.data_ptr(), self.pack.data_ptr(),
                      self.npack, self._s())
            self.launches += 1

    def local_fill(self, pool):
        """Local copies, unpacks of received mailboxes and boundary faces."""
        Engine.fill(self, pool)

    def fill(self, pool, levels=None):
        self.pack_mailboxes(pool)
        L = self.layout
        if L.send or L.recv:
            torch.cuda.current_stream(self.device).synchronize()
            self.transport.exchange(pool, L.send, L.recv)
        self.local_fill(pool)

    def finalize_dt(self, cfl, eta=0.0, kappa=0.0, *, clip_to_end=False, advance=False):
        self.transport.reduce_keys(self.keys)
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
        self.parts = [RankLayout(layout, owner, r) for r in range(world)]
        self.engines = [DistributedEngine(part, transport=None, **options) for part in self.parts]

    def fill(self, pool_name):
        pools = [getattr(e, pool_name) for e in self.engines]
        for e, pool in zip(self.engines, pools, strict=True):
            e.pack_mailboxes(pool)
        for r, part in enumerate(self.parts):
            for peer, (start, length) in part.recv.items():
                s_start, s_length = self.parts[peer].send[r]
                if s_length != length:
                    raise RuntimeError("mailboxes of a rank pair do not match")
                pools[r][start : start + length].copy_(pools[peer][s_start : s_start + s_length])
        for e, pool in zip(self.engines, pools, strict=True):
            e.local_fill(pool)

    def reduce_keys(self):
        forms = torch.stack([_keys_to_max_form(e.keys) for e in self.engines])
        top = forms.max(dim=0).values
        for e in self.engines:
            _keys_from_max_form(top, e.keys)

    def step(self, cfl):
        """One Heun step of every rank at the global stable dt."""
        for e in self.engines:
            e.rate()
        self.reduce_keys()
        for e in self.engines:
            Engine.finalize_dt(e, cfl, advance=True)
        for e in self.engines:
            e.stage(e.state, None, e.stage_pool)
        self.fill("stage_pool")
        for e in self.engines:
            e.stage(e.stage_pool, e.state, e.state)
        self.fill("state")
