"""Host-side op lists of the device mesh against the oracle's halo exchange (CPU).

The copy / interpolation / boundary ops that `wellbalanced_b200.mesh.Layout` builds are
applied to a host pool by a NumPy emulation of the CUDA kernels (``tests/_emulate.py``)
and must fill every halo point exactly as the oracle's ``fill_halos`` does
(same-level patches, periodic images, outflow and wall faces, coarse-fine
interpolation), for 2D and 3D layouts.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle.mesh import Hierarchy
from oracle.mhd2d import MHD2D as OracleMHD2D
from oracle.mhd3d import MHD3D as OracleMHD3D
from tests import _emulate
from wellbalanced_b200.mesh import AMRHierarchy, Layout

CASES_2D = [
    # shape, bounds, periodic, split, fine boxes, boundaries
    ((8, 6), ((0.0, 1.0), (0.0, 1.0)), (True, True), None, [], None),
    ((12, 10), ((0.0, 1.0), (0.0, 1.0)), (True, True), (2, 3), [], None),
    ((8, 6), ((0.0, 1.0), (0.0, 1.0)), (False, False), None, [], None),
    ((8, 9), ((0.0, 1.0), (0.0, 1.0)), (False, True), (2, 1), [], None),
    ((8, 8), ((0.0, 1.0), (0.0, 1.0)), (True, False), None, [], {"y": "wall"}),
    ((8, 8), ((0.0, 1.0), (0.0, 1.0)), (False, False), None, [], {"x": "wall", "y": "wall"}),
    ((16, 12), ((0.0, 1.0), (0.0, 1.0)), (True, True), None, [(1, ((8, 20), (6, 18)))], None),
    ((16, 12), ((0.0, 1.0), (0.0, 1.0)), (True, True), (2, 2), [(1, ((0, 12), (4, 16))), (1, ((20, 32), (8, 24)))], None),
    ((12, 12), ((0.0, 1.0), (0.0, 1.0)), (False, False), None, [(1, ((0, 8), (8, 24)))], None),
]


def _fill_oracle_and_pool(oracle_model, layout, pool, rng, nfields, extras):
    h = oracle_model.hierarchy
    names = [*oracle_model.names.values()]
    names += list(oracle_model.potential) if isinstance(oracle_model.potential, tuple) else [oracle_model.potential]
    for level in range(h.max_level + 1):
        shape = h.level_shape(level)
        for f, name in enumerate(names):
            extra = extras[f]
            values = rng.normal(size=tuple(n + e for n, e in zip(shape, extra, strict=True)))
            # periodic duplicates of the last node plane agree with the first
            for a, e in enumerate(extra):
                if e and h.periodic[a]:
                    first = np.take(values, [0], axis=a)
                    index = [slice(None)] * values.ndim
                    index[a] = slice(shape[a], shape[a] + 1)
                    values[tuple(index)] = first
            for patch in h.patches_at_level(level):
                index = tuple(slice(lo, hi + e) for (lo, hi), e in zip(patch.box, extra, strict=True))
                local = values[index]
                patch.field(name).local[...] = local
                dev = layout.h.patches[h.patches.index(patch)]
                view = layout.patch_view(pool, dev, f)
                view[tuple(slice(2, 2 + s) for s in local.shape)] = local
    return names


def _compare(oracle_model, layout, pool, names, extras):
    h = oracle_model.hierarchy
    worst = 0.0
    for patch in h.patches:
        dev = layout.h.patches[h.patches.index(patch)]
        for f, name in enumerate(names):
            expect = patch.field(name).local_with_halos
            got = layout.patch_view(pool, dev, f)[tuple(slice(0, s) for s in expect.shape)]
            worst = max(worst, float(np.max(np.abs(got - expect))))
    return worst


@pytest.mark.parametrize("case", range(len(CASES_2D)))
def test_2d_ops_fill_halos_like_the_oracle(case):
    shape, bounds, periodic, split, fine, boundaries = CASES_2D[case]
    oracle_h = Hierarchy(shape, bounds, periodic, split)
    device_h = AMRHierarchy(shape, bounds, periodic, split=split)
    for level, box in fine:
        oracle_h.add_patch(level, box)
        device_h.add_patch(level, box)
    model = OracleMHD2D(oracle_h, boundaries=boundaries)
    walls = tuple((w, w) for w in model.walls)
    layout = Layout(device_h, walls=walls, precision=64)
    pool = np.zeros(layout.pool_size)
    extras = [(0, 0)] * 6 + [(1, 1)]
    rng = np.random.default_rng(case)
    names = _fill_oracle_and_pool(model, layout, pool, rng, 7, extras)
    model.fill_halos()
    _emulate.fill(pool, layout)
    assert _compare(model, layout, pool, names, extras) < 1e-13


CASES_3D = [
    ((4, 5, 6), (True, True, True), None),
    ((6, 4, 5), (False, True, False), None),
    ((6, 6, 6), (True, True, True), (2, 1, 2)),
]


@pytest.mark.parametrize("case", range(len(CASES_3D)))
def test_3d_ops_fill_halos_like_the_oracle(case):
    shape, periodic, split = CASES_3D[case]
    bounds = ((0.0, 1.0),) * 3
    oracle_h = Hierarchy(shape, bounds, periodic, split)
    device_h = AMRHierarchy(shape, bounds, periodic, split=split)
    model = OracleMHD3D(oracle_h)
    layout = Layout(device_h, precision=64)
    pool = np.zeros(layout.pool_size)
    extras = [(0, 0, 0)] * 5 + [(0, 1, 1), (1, 0, 1), (1, 1, 0)]
    rng = np.random.default_rng(10 + case)
    names = _fill_oracle_and_pool(model, layout, pool, rng, 8, extras)
    model.fill_halos()
    _emulate.fill(pool, layout)
    assert _compare(model, layout, pool, names, extras) < 1e-13


def test_tiles_cover_every_computed_node_once():
    h = AMRHierarchy((40, 24), ((0.0, 1.0), (0.0, 1.0)), (False, True), split=(2, 1))
    layout = Layout(h, precision=32)
    tx, ty = layout.tile_shape
    for p in h.patches:
        own = [p.shape[a] + (1 if layout.own[p.index][a] else 0) for a in range(2)]
        count = np.zeros(own, dtype=int)
        for t in layout.tiles[layout.tiles["patch"] == p.index]:
            count[t["x0"] : t["x0"] + tx, t["y0"] : t["y0"] + ty] += 1
        assert np.all(count == 1)
    # the non-periodic x boundary is computed by its patch, the shared plane is not
    assert layout.own[0] == (False, False) and layout.own[1] == (True, False)


@pytest.mark.parametrize("case", [6, 7, 8])
def test_2d_restriction_ops_match_the_oracle(case):
    from oracle.mhd2d import MHD2D as OracleMHD2D

    shape, bounds, periodic, split, fine, boundaries = CASES_2D[case]
    oracle_h = Hierarchy(shape, bounds, periodic, split)
    device_h = AMRHierarchy(shape, bounds, periodic, split=split)
    for level, box in fine:
        oracle_h.add_patch(level, box)
        device_h.add_patch(level, box)
    model = OracleMHD2D(oracle_h, boundaries=boundaries)
    layout = Layout(device_h, precision=64)
    pool = np.zeros(layout.pool_size)
    extras = [(0, 0)] * 6 + [(1, 1)]
    rng = np.random.default_rng(20 + case)
    names = _fill_oracle_and_pool(model, layout, pool, rng, 7, extras)
    for name in names:
        oracle_h.restrict(name)
    for level in range(layout.h.max_level, 0, -1):
        for g in layout.groups:
            _emulate.apply_restrict(pool, layout.rows, layout.restrict_levels[level][g])
    # compare the computed points (the oracle also writes duplicate nodes the device fills)
    for patch in oracle_h.patches:
        dev = layout.h.patches[oracle_h.patches.index(patch)]
        for f, name in enumerate(names):
            expect = patch.field(name).local
            got = layout.patch_view(pool, dev, f)[tuple(slice(2, 2 + s) for s in expect.shape)]
            own = [s - (0 if (f < 6 or layout.own[dev.index][a]) else 1) for a, s in enumerate(expect.shape)]
            np.testing.assert_allclose(got[: own[0], : own[1]], expect[: own[0], : own[1]], atol=1e-14)
