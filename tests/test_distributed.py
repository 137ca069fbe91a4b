"""A hierarchy partitioned over ranks (CPU, gloo): exchange rounds, halos, restriction,
face-flux proxies and the global time step.

Each rank builds the same global layout and keeps its share (`RankLayout`). Every round
packs the boxes other ranks read into mailboxes, swaps them (grouped send/recv), and the
rank's own ops run on its patches and the received proxies, applied here by the NumPy
emulation of the kernels. The mailbox area starts as NaN, so an op reading outside the
boxes shipped to it shows up. The halos after the level-by-level fill and the coarse
values after the restriction must equal, bit for bit, the single-process sequence over
the whole hierarchy; the proxies of the face-flux round must hold the fine patches'
values over the faces' stencils; the all-reduce of the order-preserving rate / density
keys must give the global max rate and min density. Ranks are spawned processes on
127.0.0.1.
"""

from __future__ import annotations

import datetime
import os
import socket
import struct

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

CASES = [
    # shape, periodic, split, world, refined patches (level, box)
    ((24, 16), (True, True), (3, 2), 2, ()),
    ((24, 16), (True, False), (4, 2), 3, ()),
    ((12, 10, 8), (True, True, False), (2, 2, 1), 2, ()),
    ((24, 16), (True, True), (2, 2), 2, ((1, ((10, 30), (6, 22))), (1, ((30, 44), (4, 14))))),
    ((24, 16), (True, False), (3, 2), 3, ((1, ((0, 16), (8, 24))), (1, ((16, 40), (10, 20))),
                                          (2, ((4, 28), (20, 40))))),
    ((12, 10, 8), (True, True, True), (2, 1, 1), 2, ((1, ((4, 14), (2, 12), (4, 12))),
                                                     (1, ((14, 20), (6, 16), (2, 8))))),
]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _key(x):
    bits = struct.unpack("<Q", struct.pack("<d", x))[0]
    return (~bits & 0xFFFFFFFFFFFFFFFF) if bits >> 63 else (bits | 1 << 63)


def _as_int64(u):
    return u - (1 << 64) if u >= 1 << 63 else u


def _worker(rank, world, port, case, out):
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        out.put(_work(rank, world, case))
    except Exception as error:  # report instead of leaving the other ranks waiting
        out.put((rank, repr(error), 0, [], False, 0))
    finally:
        torch.distributed.destroy_process_group()


def _hierarchy(case):
    from wellbalanced_b200.mesh import AMRHierarchy

    shape, periodic, split, _, refined = CASES[case]
    h = AMRHierarchy(shape, ((0.0, 1.0),) * len(shape), periodic, split=split)
    for level, box in refined:
        h.add_patch(level, box)
    return h


def _blocks_differ(pool, expect, layout, part):
    worst = 0.0
    nf = layout.nfields
    for i, g in enumerate(part.local):
        a, size = int(layout.rows[g]["off"]), int(layout.rows[g]["fstride"]) * nf
        b, _ = part.block(i)
        diff = np.abs(pool[b : b + size] - expect[a : a + size])
        worst = max(worst, float(np.nanmax(diff)) if diff.size else 0.0)
        if np.isnan(diff).any() != np.isnan(expect[a : a + size]).any():
            worst = np.inf
    return worst


def _work(rank, world, case):
    from tests import _emulate
    from wellbalanced_b200.distributed import RankLayout, TorchTransport, _flux_footprint, partition
    from wellbalanced_b200.mesh import Layout

    h = _hierarchy(case)
    layout = Layout(h, precision=64)
    owner = partition(h, world)
    part = RankLayout(layout, owner, rank)
    transport = TorchTransport()
    rng = np.random.default_rng(case)
    whole = rng.normal(size=layout.pool_size)
    expect = whole.copy()
    _emulate.fill(expect, layout)
    pool_t = torch.full((part.pool_size,), float("nan"), dtype=torch.float64)
    pool = pool_t.numpy()
    nf = layout.nfields
    for i, g in enumerate(part.local):
        a, size = int(layout.rows[g]["off"]), int(layout.rows[g]["fstride"]) * nf
        b, _ = part.block(i)
        pool[b : b + size] = whole[a : a + size]

    def exchange(key):
        rd = part.rounds[key]
        _emulate.apply_copy(pool, part.rows, rd.pack_ops)
        transport.exchange(pool_t, rd.send, rd.recv)

    # halos, level by level
    for level, (same, boundary) in enumerate(part.copy_phases):
        exchange(("fill", level))
        _emulate.apply_interp(pool, part.rows, part.interp_levels[level])
        _emulate.apply_copy(pool, part.rows, same)
        for ops in boundary:
            _emulate.apply_copy(pool, part.rows, ops)
    worst = _blocks_differ(pool, expect, layout, part)
    # the face-flux proxies hold the fine patches' stencils
    exchange(("flux",))
    flux_bad = 0
    for op in np.atleast_1d(part.face_flux_ops):
        fine = int(op["fine"])
        if fine < part.npatches:
            continue
        g = [src for src, row in part.rounds[("flux",)].proxies.items() if row == fine][0]
        _, lo, hi = _flux_footprint(op)
        P, Q = part.rows[fine], layout.rows[g]
        extent = [int(Q["n"][a]) + 4 if a < layout.ndim else 0 for a in range(3)]
        lo = [max(v, 0) for v in lo]
        hi = [min(v, e) for v, e in zip(hi, extent, strict=True)]
        for i in range(lo[0], hi[0] + 1):
            for j in range(lo[1], hi[1] + 1):
                for k in range(lo[2], hi[2] + 1):
                    for f in range(nf):
                        mine = pool[int(P["off"]) + f * int(P["fstride"]) + _emulate.offset_of(P, i, j, k)]
                        theirs = expect[int(Q["off"]) + f * int(Q["fstride"]) + _emulate.offset_of(Q, i, j, k)]
                        flux_bad += int(not (mine == theirs))
    # restriction, finest level first
    for level in range(layout.max_level, 0, -1):
        for g in layout.groups:
            _emulate.apply_restrict(expect, layout.rows, layout.restrict_levels[level][g])
            exchange(("restrict", level, g))
            _emulate.apply_restrict(pool, part.rows, part.restrict_levels[level][g])
    worst = max(worst, _blocks_differ(pool, expect, layout, part))
    # global time step: max rate and min density over the ranks
    rate, rho = 1.0 + rank * 0.75, 2.0 - rank * 0.5
    keys = torch.tensor([_as_int64(_key(rate)), _as_int64(_key(rho))], dtype=torch.int64)
    transport.reduce_keys(keys)
    want = [_as_int64(_key(1.0 + (world - 1) * 0.75)), _as_int64(_key(2.0 - (world - 1) * 0.5))]
    peers = sorted({p for rd in part.rounds.values() for p in rd.send})
    return rank, worst, len(part.local), peers, keys.tolist() == want, flux_bad


@pytest.mark.parametrize("case", range(len(CASES)))
def test_partitioned_hierarchy_equals_the_single_process_sequence(case):
    world = CASES[case][3]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = [out.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sum(r[2] for r in results) == len(_hierarchy(case).patches), results  # every patch has one owner
    for rank, worst, nlocal, peers, keys_ok, flux_bad in results:
        assert nlocal > 0 and peers, (rank, worst, nlocal, peers)
        assert worst == 0.0, (rank, worst)
        assert keys_ok, rank
        assert flux_bad == 0, (rank, flux_bad)


def test_partition_balances_cells_in_morton_order():
    from wellbalanced_b200.distributed import partition
    from wellbalanced_b200.mesh import AMRHierarchy

    h = AMRHierarchy((64, 64), ((0.0, 1.0), (0.0, 1.0)), (True, True), split=(4, 4))
    owner = partition(h, 4)
    counts = np.bincount(owner, minlength=4)
    assert list(counts) == [4, 4, 4, 4]
    # Morton runs: each rank's patches form a 2 x 2 block of the 4 x 4 split
    for r in range(4):
        boxes = [p.box for p in h.patches if owner[p.index] == r]
        xs = {b[0][0] for b in boxes}
        ys = {b[1][0] for b in boxes}
        assert len(xs) == 2 and len(ys) == 2
    # refined levels are balanced level by level
    h.add_patch(1, ((16, 48), (16, 48)))
    h.add_patch(1, ((80, 112), (80, 112)))
    owner = partition(h, 2)
    fine = [owner[p.index] for p in h.patches_at_level(1)]
    assert sorted(fine) == [0, 1]


def test_refined_plans_ship_boxes_inside_the_source_patches():
    """Every rank's proxies lie inside their source patches' haloed arrays, and the
    mailbox slices of every rank pair line up."""
    from wellbalanced_b200.distributed import RankLayout, partition
    from wellbalanced_b200.mesh import Layout

    for case in range(3, len(CASES)):
        h = _hierarchy(case)
        layout = Layout(h, precision=64)
        world = CASES[case][3]
        owner = partition(h, world)
        parts = [RankLayout(layout, owner, r) for r in range(world)]
        crossing = 0
        for r, part in enumerate(parts):
            for key, rd in part.rounds.items():
                for peer, (_, length) in rd.recv.items():
                    assert parts[peer].rounds[key].send[r][1] == length, (case, key, r, peer)
                    crossing += 1
        assert crossing > 0, case
