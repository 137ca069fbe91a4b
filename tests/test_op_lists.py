"""Host-side op lists of the halo kernels (CPU): the cuts that size them for the kernels
and the trimmed interpolation ops of the single-launch level fill.

Cutting a box into ops, and trimming a level's interpolation ops to the halo points no
same-level copy writes, must leave the fill's result unchanged bit for bit (applied
here by the NumPy emulation of the kernels), and the trimmed interpolation ops must
write no point a copy of the same level writes (they share one launch).
"""

from __future__ import annotations

import itertools

import numpy as np
import pytest

from tests import _emulate
from tests.test_distributed import CASES, _hierarchy


def _points(op, start_key):
    d, n = op[start_key], op["n"]
    return {
        (int(op["dst"] if "dst" in op.dtype.names else op["fine"]), f, *p)
        for f in range(int(op["field_lo"]), int(op["field_hi"]))
        for p in itertools.product(*(range(int(d[a]), int(d[a] + n[a])) for a in range(3)))
    }


def _seeded_pool(layout, seed=0):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(layout.pool_size)


@pytest.mark.parametrize("case", [3, 4, 5])
def test_trimmed_interpolation_writes_no_copied_point_and_fills_the_same(case):
    from wellbalanced_b200.mesh import Layout

    layout = Layout(_hierarchy(case), precision=64)
    full = layout._interp_ops()
    trimmed_any = False
    for level in range(1, len(layout.interp_levels)):
        same = layout.copy_phases[level][0]
        copied = set().union(*(_points(op, "d") for op in same)) if same.size else set()
        interp = layout.interp_levels[level]
        written = set().union(*(_points(op, "d") for op in interp)) if interp.size else set()
        assert not written & copied
        # together they still cover every point the untrimmed interpolation wrote
        before = set().union(*(_points(op, "d") for op in full[level])) if full[level].size else set()
        assert before <= written | copied
        trimmed_any |= len(written) < len(before)
    assert trimmed_any

    expect = _seeded_pool(layout)
    got = expect.copy()
    for level, (same, boundary) in enumerate(layout.copy_phases):
        _emulate.apply_interp(expect, layout.rows, full[level])
        _emulate.apply_copy(expect, layout.rows, same)
        for ops in boundary:
            _emulate.apply_copy(expect, layout.rows, ops)
    _emulate.fill(got, layout)
    assert np.array_equal(got, expect)


@pytest.mark.parametrize("case", range(len(CASES)))
def test_ops_cut_for_the_kernels_fill_the_same(case):
    from wellbalanced_b200.mesh import Layout, size_ops, split_box_ops

    layout = Layout(_hierarchy(case), precision=64)
    expect = _seeded_pool(layout, 1)
    got = expect.copy()
    for level, (same, boundary) in enumerate(layout.copy_phases):
        interp = layout.interp_levels[level]
        _emulate.apply_interp(expect, layout.rows, interp)
        _emulate.apply_copy(expect, layout.rows, same)
        for ops in boundary:
            _emulate.apply_copy(expect, layout.rows, ops)
        cut = [size_ops(interp) if interp.size else interp, split_box_ops(same, 5) if same.size else same]
        for ops in cut:
            assert ops.size == 0 or int(np.prod(ops["n"].astype(np.int64), axis=1).max()) <= 1024
        _emulate.apply_interp(got, layout.rows, cut[0])
        _emulate.apply_copy(got, layout.rows, cut[1])
        for ops in boundary:
            _emulate.apply_copy(got, layout.rows, split_box_ops(ops, 7) if ops.size else ops)
    assert np.array_equal(got, expect)
    for level, groups in layout.restrict_levels.items():
        for g, ops in groups.items():
            if ops.size:
                a, b = expect.copy(), expect.copy()
                _emulate.apply_restrict(a, layout.rows, ops)
                _emulate.apply_restrict(b, layout.rows, split_box_ops(ops, 3))
                assert np.array_equal(a, b)


def test_op_points_follow_the_list_size():
    from wellbalanced_b200.mesh import OP_WAVE, op_points

    assert op_points(1) == 64
    assert op_points(64 * OP_WAVE) == 64
    assert op_points(64 * OP_WAVE + 1) == 128
    assert op_points(10**9) == 1024


def test_face_numbering_maps_every_face_to_its_op():
    """The staged register's flat face numbering (CPU): each op's `first` is the prefix sum of
    the lengths, and the binary search the kernel runs over `first` returns, for every face,
    the op holding it and its position in the op."""
    from wellbalanced_b200.mesh import AMRHierarchy, Layout, number_faces

    mesh = AMRHierarchy((32, 32), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, False))
    mesh.add_patch(1, ((12, 40), (20, 44)))
    mesh.add_patch(1, ((40, 60), (8, 30)))
    mesh.add_patch(2, ((30, 60), (48, 80)))
    layout = Layout(mesh)
    ops, total = number_faces(layout.face_flux_ops)
    assert ops.size == layout.face_flux_ops.size > 0
    assert total == int(layout.face_flux_ops["len"].sum())
    seen = []
    for face in range(total):
        lo, hi = 0, ops.size - 1
        while lo < hi:  # the kernel's search: the last op whose first face is not after `face`
            mid = (lo + hi + 1) >> 1
            if ops["first"][mid] <= face:
                lo = mid
            else:
                hi = mid - 1
        s = face - int(ops["first"][lo])
        assert 0 <= s < int(ops["len"][lo])
        seen.append((lo, s))
    assert seen == [(i, s) for i in range(ops.size) for s in range(int(ops["len"][i]))]
    # the numbering leaves the other fields alone
    for name in ops.dtype.names:
        if name != "first":
            np.testing.assert_array_equal(ops[name], layout.face_flux_ops[name])
