"""The device regrid transfer's op lists (CPU): every point of every new patch is written
by the prolongation from the level below (levels >= 1), kept-value ops cover exactly the
points an old patch of the same level held, positivity ops visit every new cell of a level
>= 1 once (as a child of a parent cell of the level below), and every index an op makes its
kernel read or write lies inside the haloed arrays of its patches (the bounds of
csrc/transfer.cu)."""

from __future__ import annotations

import itertools

import numpy as np
import pytest

from wellbalanced_b200.mesh import HALO, AMRHierarchy, field_groups
from wellbalanced_b200.regrid import transfer_ops


def _hierarchies(ndim, periodic):
    shape = (16,) * ndim
    old = AMRHierarchy(shape, ((0.0, 1.0),) * ndim, periodic=periodic)
    box1 = tuple((6, 20) for _ in range(ndim))
    old.add_patch(1, box1)
    rng = np.random.default_rng(ndim)
    tags = {0: rng.random(shape) < 0.15}
    tags[0][tuple(slice(4, 9) for _ in range(ndim))] = True
    h1 = old.regrid(tags, max_patch_size=6)
    t1 = {0: tags[0], 1: np.zeros(h1.level_shape(1), dtype=bool)}
    t1[1][tuple(slice(10, 16) for _ in range(ndim))] = True
    new = h1.regrid(t1, max_patch_size=6)
    return old, new


def _haloed(p, ndim):
    return [p.shape[a] + 5 for a in range(ndim)]


@pytest.mark.parametrize("ndim, periodic", [(2, (True, True)), (2, (True, False)), (3, (True, True, True))])
def test_transfer_ops_cover_and_stay_in_bounds(ndim, periodic):
    old, new = _hierarchies(ndim, periodic)
    assert new.max_level == 2
    groups = field_groups(ndim)
    ops = transfer_ops(old, new, groups, ndim)
    assert len(ops) == new.max_level + 1
    for level, (prolong, kept, positivity) in enumerate(ops):
        for g in groups:
            for f in new.patches_at_level(level):
                n = [f.shape[a] + ((g.node_mask >> a) & 1) for a in range(ndim)]
                hit = np.zeros(n, dtype=bool)
                for op in prolong[(prolong["fine"] == f.index) & (prolong["field_lo"] == g.lo)]:
                    c = new.patches[int(op["coarse"])]
                    assert c.level == level - 1
                    for q in itertools.product(*[range(int(op["n"][a])) for a in range(ndim)]):
                        fi = [int(op["d"][a]) + q[a] for a in range(ndim)]
                        assert all(0 <= fi[a] < _haloed(f, ndim)[a] for a in range(ndim))
                        hit[tuple(fi[a] - HALO for a in range(ndim))] = True
                        gl = [fi[a] - HALO + int(op["fine_lo"][a]) for a in range(ndim)]
                        for a in range(ndim):
                            node = (g.node_mask >> a) & 1
                            base = gl[a] >> 1
                            reach = [base, base + (gl[a] & 1)] if node else [base - 1, base + 1]
                            for cc in reach:
                                ch = cc - int(op["coarse_lo"][a]) + HALO
                                assert 0 <= ch < _haloed(c, ndim)[a], (level, a, cc)
                if level:
                    assert hit.all(), (level, f.box, g)
                # kept values: within both patches' arrays
                for op in kept[(kept["dst"] == f.index) & (kept["field_lo"] == g.lo)]:
                    o = old.patches[int(op["src1"])]
                    assert o.level == level
                    for a in range(ndim):
                        assert 0 <= op["d"][a] and op["d"][a] + op["n"][a] <= _haloed(f, ndim)[a]
                        assert 0 <= op["s1"][a] and op["s1"][a] + op["n"][a] <= _haloed(o, ndim)[a]
        if level:
            for f in new.patches_at_level(level):
                seen = np.zeros(f.shape, dtype=np.int64)
                for op in positivity[positivity["fine"] == f.index]:
                    c = new.patches[int(op["coarse"])]
                    assert c.level == level - 1 and int(op["ndim"]) == ndim
                    for q in itertools.product(*[range(int(op["n"][a])) for a in range(ndim)]):
                        parent = [int(op["c0"][a]) + q[a] for a in range(ndim)]
                        # the parent's cell and its nodes (cell + 1) inside the coarse array
                        assert all(HALO <= parent[a] < HALO + c.shape[a] for a in range(ndim))
                        # its level index matches its children's
                        for o in itertools.product((0, 1), repeat=ndim):
                            x = [int(op["f0"][a]) + 2 * q[a] + o[a] for a in range(ndim)]
                            assert all(HALO <= x[a] < HALO + f.shape[a] for a in range(ndim))
                            level_x = [x[a] - HALO + f.box[a][0] for a in range(ndim)]
                            level_parent = [parent[a] - HALO + c.box[a][0] for a in range(ndim)]
                            assert [v // 2 for v in level_x] == level_parent
                            seen[tuple(x[a] - HALO for a in range(ndim))] += 1
                assert (seen == 1).all(), (level, f.box)
