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
    # a fine level over the whole periodic domain, and a second level inside it
    ((8, 8), ((0.0, 1.0), (0.0, 1.0)), (True, True), None, [(1, ((0, 16), (0, 16))), (2, ((8, 24), (4, 20)))], None),
    # two fine patches that together span the periodic x axis
    ((8, 8), ((0.0, 1.0), (0.0, 1.0)), (True, True), None, [(1, ((0, 8), (4, 12))), (1, ((8, 16), (4, 12)))], None),
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


@pytest.mark.parametrize("case", [6, 7, 8, 9, 10])
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
    # node planes a fine patch does not compute are stale copies until the next halo fill:
    # the restriction must not read them
    for dev in layout.h.patches:
        if dev.level == 0:
            continue
        view = layout.patch_view(pool, dev, 6)
        for a in range(2):
            if not layout.own[dev.index][a]:
                index = [slice(None)] * 2
                index[a] = 2 + dev.shape[a]
                view[tuple(index)] = np.nan
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


def test_merged_layouts_fill_each_instance_independently():
    parts = []
    for shape in ((8, 6), (12, 10), (8, 6)):
        h = AMRHierarchy(shape, ((0.0, 1.0), (0.0, 1.0)), periodic=(True, True))
        parts.append((h, Layout(h, precision=64)))
    merged = Layout.merge([layout for _, layout in parts])
    assert merged.ninstances == 3 and list(merged.instances) == [0, 1, 2]
    rng = np.random.default_rng(5)
    pool = rng.normal(size=merged.pool_size)
    _emulate.fill(pool, merged)
    start = 0
    for k, (h, layout) in enumerate(parts):
        single = pool[start : start + layout.pool_size].copy()
        expect = single.copy()
        _emulate.fill(expect, layout)
        np.testing.assert_array_equal(single, expect)
        start += layout.pool_size


def test_reflux_phases_touch_disjoint_cells():
    """A coarse cell between fine patches takes corrections from several RefluxOps; the
    ops of one phase (one launch) must never share a cell, and a cell takes its
    corrections in the (axis, side) order of the interfaces, whatever the grouping."""
    boxes = [((0, 8), (0, 14)), ((14, 20), (0, 4)), ((0, 4), (14, 18)), ((8, 20), (14, 28)), ((0, 20), (28, 36)),
             ((0, 6), (44, 52)), ((8, 20), (36, 52)), ((0, 8), (52, 64)), ((24, 28), (0, 16)), ((28, 40), (0, 8)),
             ((28, 38), (8, 20)), ((56, 64), (0, 20)), ((20, 24), (22, 48)), ((60, 64), (28, 36))]
    h = AMRHierarchy((16, 16), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, True))
    h.add_patch(1, ((0, 32), (0, 32)))
    for box in boxes:
        h.add_patch(2, box)
    layout = Layout(h, precision=64)
    assert 2 <= len(layout.reflux_phases) <= 4
    shared = 0
    seen_any = {}
    order = {}  # cell -> (axis, side) ranks of its corrections, in launch order
    for ops in layout.reflux_phases:
        seen = set()
        for op in ops:
            axis = 1 - int(op["t1"])  # 2D: the normal is the other axis
            rank = 2 * axis + (0 if float(op["sign"]) > 0 else 1)
            for s in range(int(op["len"])):
                s1, s2 = divmod(s, int(op["width"]))
                idx = [int(v) for v in op["c"]]
                idx[int(op["t1"])] += s1
                if int(op["t2"]) >= 0:
                    idx[int(op["t2"])] += s2
                cell = (int(op["coarse"]), *idx)
                assert cell not in seen
                seen.add(cell)
                shared += cell in seen_any
                seen_any[cell] = True
                order.setdefault(cell, []).append(rank)
    assert shared > 0  # the configuration does have cells corrected from two sides
    assert all(ranks == sorted(ranks) for ranks in order.values())


def test_op_records_keep_the_c_layout():
    """Every record array handed to the kernels has the exact C struct layout (NumPy
    repacks padded structured dtypes when concatenating; the upload casts back)."""
    import torch

    from wellbalanced_b200 import _lib
    from wellbalanced_b200.engine import _device_bytes

    h = AMRHierarchy((16, 16), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, True))
    h.add_patch(1, ((4, 12), (8, 20)))
    h.add_patch(1, ((12, 20), (8, 16)))
    single = Layout(h, precision=64)
    merged = Layout.merge([single, single])
    for layout in (single, merged):
        arrays = [(layout.rows, _lib.PATCH), (layout.tiles, _lib.TILE), (layout.face_flux_ops, _lib.FACE_FLUX_OP),
                  (layout.reflux_ops, _lib.REFLUX_OP)]
        arrays += [(ops, _lib.REFLUX_OP) for ops in layout.reflux_phases]
        arrays += [(ops, _lib.INTERP_OP) for ops in layout.interp_levels]
        for same, boundary in layout.copy_phases:
            arrays += [(same, _lib.COPY_OP)] + [(ops, _lib.COPY_OP) for ops in boundary]
        for groups in layout.restrict_levels.values():
            arrays += [(ops, _lib.RESTRICT_OP) for ops in groups.values()]
        for array, dtype in arrays:
            assert array.dtype == dtype and array.dtype.itemsize == dtype.itemsize
            if array.size:
                raw = _device_bytes(array, torch.device("cpu"), dtype)
                assert raw.numel() == array.size * dtype.itemsize
                back = raw.numpy().view(dtype)
                assert back.tobytes() == np.ascontiguousarray(array).tobytes()
    # a repacked array is cast back field by field
    packed = np.concatenate([single.reflux_ops, single.reflux_ops])
    assert packed.dtype.itemsize != _lib.REFLUX_OP.itemsize
    raw = _device_bytes(packed, torch.device("cpu"), _lib.REFLUX_OP).numpy().view(_lib.REFLUX_OP)
    for name in _lib.REFLUX_OP.names:
        np.testing.assert_array_equal(raw[name], packed[name])


@pytest.mark.parametrize("case", [6, 7, 8, 9, 10])
def test_flux_register_ops_stay_inside_their_patches(case):
    """FaceFluxOps read a 4-cell stencil (and the node after it) across each face, and
    RefluxOps write interior cells only: check every index against the haloed extents."""
    shape, bounds, periodic, split, fine, boundaries = CASES_2D[case]
    h = AMRHierarchy(shape, bounds, periodic, split=split)
    for level, box in fine:
        h.add_patch(level, box)
    layout = Layout(h, precision=64)
    rows = layout.rows
    for op in layout.face_flux_ops:
        a, t1 = int(op["axis"]), int(op["t1"])
        for patch, plane, t0, step in ((op["coarse"], op["coarse_plane"], op["coarse_t0"][0], 1),
                                       (op["fine"], op["fine_plane"], op["fine_t0"][0], 2)):
            n = rows[patch]["n"]
            # haloed indices: cells plane-2 .. plane+1 of n+4, the node after them of n+5
            assert 0 <= plane - 2 and plane + 1 < n[a] + 4
            # transverse: interior cells only
            last = t0 + step * int(op["len"]) - 1
            assert 2 <= t0 and last < n[t1] + 2
    for op in layout.reflux_ops:
        n = rows[op["coarse"]]["n"]
        t1 = int(op["t1"])
        c = [int(v) for v in op["c"]][:2]
        for axis in range(2):
            hi = c[axis] + (int(op["len"]) - 1 if axis == t1 else 0)
            assert 2 <= c[axis] and hi < 2 + n[axis]
