"""A level partitioned over ranks (CPU, gloo): halo exchange and the global time step.

Each rank builds the same global layout, keeps its share (`RankLayout`) and fills the
halos of its patches by pack -> grouped send/recv -> local copies and unpacks ->
boundary faces (the copy ops applied by the NumPy emulation of the copy kernel); every
point of every rank's patches must equal the single-process fill of the whole level.
The all-reduce of the order-preserving rate / density keys must give the global max rate
and min density. Ranks are spawned processes on 127.0.0.1.
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
    # shape, periodic, split, world
    ((24, 16), (True, True), (3, 2), 2),
    ((24, 16), (True, False), (4, 2), 3),
    ((12, 10, 8), (True, True, False), (2, 2, 1), 2),
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
        out.put((rank, repr(error), 0, [], False))
    finally:
        torch.distributed.destroy_process_group()


def _work(rank, world, case):
    from tests import _emulate
    from wellbalanced_b200.distributed import RankLayout, TorchTransport, partition
    from wellbalanced_b200.mesh import AMRHierarchy, Layout

    shape, periodic, split, _ = CASES[case]
    h = AMRHierarchy(shape, ((0.0, 1.0),) * len(shape), periodic, split=split)
    layout = Layout(h, precision=64)
    owner = partition(h, world)
    part = RankLayout(layout, owner, rank)
    rng = np.random.default_rng(case)
    whole = rng.normal(size=layout.pool_size)
    expect = whole.copy()
    _emulate.fill(expect, layout)
    pool_t = torch.zeros(part.pool_size, dtype=torch.float64)
    pool = pool_t.numpy()
    nf = layout.nfields
    for i, g in enumerate(part.local):
        a, size = int(layout.rows[g]["off"]), int(layout.rows[g]["fstride"]) * nf
        b, _ = part.block(i)
        pool[b : b + size] = whole[a : a + size]
    _emulate.apply_copy(pool, part.rows, part.pack_ops)
    TorchTransport().exchange(pool_t, part.send, part.recv)
    same, boundary = part.copy_phases[0]
    _emulate.apply_copy(pool, part.rows, same)
    for ops in boundary:
        _emulate.apply_copy(pool, part.rows, ops)
    worst = 0.0
    for i, g in enumerate(part.local):
        a, size = int(layout.rows[g]["off"]), int(layout.rows[g]["fstride"]) * nf
        b, _ = part.block(i)
        worst = max(worst, float(np.max(np.abs(pool[b : b + size] - expect[a : a + size]))))
    # global time step: max rate and min density over the ranks
    rate, rho = 1.0 + rank * 0.75, 2.0 - rank * 0.5
    keys = torch.tensor([_as_int64(_key(rate)), _as_int64(_key(rho))], dtype=torch.int64)
    TorchTransport().reduce_keys(keys)
    want = [_as_int64(_key(1.0 + (world - 1) * 0.75)), _as_int64(_key(2.0 - (world - 1) * 0.5))]
    return rank, worst, len(part.local), sorted(part.send), keys.tolist() == want


@pytest.mark.parametrize("case", range(len(CASES)))
def test_partitioned_fill_equals_the_whole_level(case):
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
    assert sum(r[2] for r in results) == int(np.prod(CASES[case][2]))  # every patch has one owner
    for rank, worst, nlocal, peers, keys_ok in results:
        assert nlocal > 0 and peers, (rank, worst, nlocal, peers)
        assert worst == 0.0, (rank, worst)
        assert keys_ok, rank


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
