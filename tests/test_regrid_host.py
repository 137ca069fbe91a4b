"""Regridding's host logic (CPU): clustering, prolongation, and the transfer driven on the oracle.

The reference's AMR regrid properties (``tests/unit/test_mhd_amr.py:69-89``: each regrid
keeps the totals, the field stays divergence-free, refined runs stay conservative) are
checked here with the oracle's MHD2D as the solver and this package's clustering and
transfer rules, so the rules are pinned without a GPU.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle.mesh import Hierarchy
from oracle.mhd2d import MHD2D as OracleMHD2D
from wellbalanced_b200.mesh import AMRHierarchy
from wellbalanced_b200.regrid import (
    _merge_periodic_planes,
    cluster_tags,
    nesting_mask,
    prolong_cells,
    prolong_potential,
)

K = 2.0 * np.pi


def test_cluster_boxes_cover_every_grown_tag_of_thin_3d_shells():
    """Thin spherical shells and scattered cells on a periodic 32^3 level (the multi-blast's
    tag pattern): the boxes cover every tagged cell grown by the buffer, do not overlap,
    and respect the largest side."""
    n = 32
    rng = np.random.default_rng(0)
    x = (np.arange(n) + 0.5) / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    tags = np.zeros((n, n, n), dtype=bool)
    for _ in range(8):
        c = rng.uniform(0.15, 0.85, 3)
        r = rng.uniform(0.1, 0.25)
        tags |= np.abs(np.sqrt((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) - r) < 0.03
    tags |= rng.random(tags.shape) < 0.01
    boxes = cluster_tags(tags, buffer=1, max_size=8, periodic=(True,) * 3)
    held = np.zeros(tags.shape, dtype=int)
    for box in boxes:
        assert all(1 <= hi - lo <= 8 for lo, hi in box)
        held[tuple(slice(lo, hi) for lo, hi in box)] += 1
    assert held.max() == 1
    grown = tags.copy()
    for a in range(3):
        grown = grown | np.roll(grown, 1, axis=a) | np.roll(grown, -1, axis=a)
    assert np.all(held[grown] == 1)


def test_cluster_boxes_cover_the_tags_and_do_not_overlap():
    rng = np.random.default_rng(3)
    tags = np.zeros((32, 24), dtype=bool)
    tags[4:9, 3:20] = True
    tags[20:30, 10:14] = True
    tags |= rng.random(tags.shape) < 0.01
    boxes = cluster_tags(tags, buffer=1, max_size=12, periodic=(True, False))
    covered = np.zeros(tags.shape, dtype=int)
    for box in boxes:
        assert all(hi - lo <= 12 and hi - lo >= 2 for lo, hi in box)
        covered[tuple(slice(lo, hi) for lo, hi in box)] += 1
    assert covered.max() == 1
    # every tagged cell that may hold a finer patch is covered
    allowed = nesting_mask(tags.shape, [((0, 32), (0, 24))], (True, False))
    assert np.all(covered[tags & allowed] == 1)


def test_nesting_keeps_a_cell_inside_the_parent_patches():
    parents = [((4, 12), (4, 12))]
    mask = nesting_mask((16, 16), parents, (False, False))
    assert mask[5:11, 5:11].all()
    assert not mask[4].any() and not mask[:, 11].any()


def test_prolongation_keeps_integrals_and_coincident_nodes():
    rng = np.random.default_rng(1)
    coarse = rng.random((6, 5))
    fine = prolong_cells(coarse, (True, False))
    mean = 0.25 * (fine[0::2, 0::2] + fine[1::2, 0::2] + fine[0::2, 1::2] + fine[1::2, 1::2])
    np.testing.assert_allclose(mean, coarse, rtol=0, atol=1e-15)
    assert fine.min() >= coarse.min() - 1e-15 and fine.max() <= coarse.max() + 1e-15
    az = rng.random((7, 6))
    fine_az = prolong_potential(az, (1, 1))
    np.testing.assert_array_equal(fine_az[0::2, 0::2], az)
    edge = rng.random((6, 7, 7))  # an x-edge potential: cell axis x, node axes y and z
    fine_edge = prolong_potential(edge, (0, 1, 1))
    assert fine_edge.shape == (12, 13, 13)
    np.testing.assert_array_equal(fine_edge[0::2, 0::2, 0::2], edge)


def test_periodic_duplicate_planes_take_the_kept_value():
    values = np.arange(25.0).reshape(5, 5)
    mask = np.zeros((5, 5), dtype=bool)
    mask[4, 1:3] = True  # kept values on the last x plane only
    mask[0, 3] = True  # and one on the first
    _merge_periodic_planes(values, mask, (1, 1), (True, False), (4, 4))
    np.testing.assert_array_equal(values[0], values[4])
    assert values[0, 1] == 21.0 and values[0, 2] == 22.0 and values[0, 3] == 3.0
    assert mask[0, 1:4].all() and mask[4, 1:4].all()


def _orszag_tang(hierarchy):
    model = OracleMHD2D(hierarchy)
    model.set_state(
        25.0 / (36.0 * np.pi),
        (lambda x, y: -np.sin(K * y), lambda x, y: np.sin(K * x), 0.0),
        5.0 / (12.0 * np.pi),
        vector_potential=lambda x, y: (np.cos(2 * K * x) / (2 * K) + np.cos(K * y) / K) / np.sqrt(4 * np.pi),
        bz=lambda x, y: 0.1 * np.cos(K * x),
    )
    return model


def _regrid_oracle(model, mesh, tags, merge=True, **options):
    """The transfer of `wellbalanced_b200.regrid.regrid_model`, applied to the oracle's patches."""
    names = [*model.names.values(), model.potential]
    extras = [(0, 0)] * 6 + [(1, 1)]
    h = model.hierarchy
    old = {}
    for level in range(h.max_level + 1):
        shape = h.level_shape(level)
        arrays = []
        for name, extra in zip(names, extras, strict=True):
            values = np.zeros(tuple(n + e for n, e in zip(shape, extra, strict=True)))
            mask = np.zeros(values.shape, dtype=bool)
            for p in h.patches_at_level(level):
                index = tuple(slice(lo, hi + e) for (lo, hi), e in zip(p.box, extra, strict=True))
                values[index] = p.field(name).local
                mask[index] = True
            if merge:
                _merge_periodic_planes(values, mask, extra, h.periodic, shape)
            arrays.append((values, mask))
        old[level] = arrays
    new_mesh = mesh.regrid(tags, **options)
    oh = Hierarchy(h.shape, h.bounds, h.periodic)
    for p in new_mesh.patches:
        if p.level:
            oh.add_patch(p.level, p.box)
    out = OracleMHD2D(oh)
    new = {}
    for level in range(new_mesh.max_level + 1):
        arrays = []
        for f, (name, extra) in enumerate(zip(names, extras, strict=True)):
            if level == 0:
                result = old[0][f][0]
            else:
                coarse = new[level - 1][f]
                fine = prolong_potential(coarse, extra) if any(extra) else prolong_cells(coarse, h.periodic)
                result = fine if level not in old else np.where(old[level][f][1], old[level][f][0], fine)
            arrays.append(result)
            for p in oh.patches_at_level(level):
                index = tuple(slice(lo, hi + e) for (lo, hi), e in zip(p.box, extra, strict=True))
                p.field(name).local[...] = result[index]
        new[level] = arrays
    out._ready = True
    for name in names:
        oh.restrict(name)
    return out, new_mesh


def _three_regrids(merge):
    mesh = AMRHierarchy((16, 16), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, True))
    model = _orszag_tang(Hierarchy((16, 16), ((0.0, 1.0), (0.0, 1.0)), (True, True)))
    start = model.totals()
    for _ in range(3):
        before = model.totals()
        # boxes of at most 12 coarse cells: fine patches meet across the periodic boundaries
        model, mesh = _regrid_oracle(model, mesh, model.current_tags(0.1, 2), merge=merge, max_patch_size=12)
        after = model.totals()
        for name in before:
            assert abs(after[name] - before[name]) < 1e-14, name
        for _ in range(4):
            model.step()
    end = model.totals()
    return mesh, max(abs(end[name] - start[name]) for name in start)


def test_three_regrids_keep_the_totals_on_the_oracle():
    mesh, drift = _three_regrids(merge=True)
    assert mesh.max_level == 2 and len(mesh.patches_at_level(2)) > 4
    assert drift < 1e-14


def test_unmerged_periodic_planes_break_conservation():
    """Without merging the periodic duplicate planes, fine patches that meet across the
    periodic boundary start from different A_z and their shared-face fluxes disagree."""
    _, drift = _three_regrids(merge=False)
    assert drift > 1e-12


@pytest.mark.parametrize("periodic", [(False, False), (True, False)])
def test_cluster_boxes_respect_the_parents_and_cover_the_nestable_tags(periodic):
    """Clustering a refined level under two parent patches (outflow and periodic x): every
    box lies in the nestable region (inside the parents by the nesting margin), the boxes are
    disjoint, at most `max_size` a side, and every grown tag of the nestable region is
    covered; boxes reach the smallest side where free nestable cells allow."""
    rng = np.random.default_rng(7)
    shape = (48, 40)
    parents = [((0, 20), (4, 36)), ((20, 44), (8, 30))]
    tags = rng.random(shape) < 0.06
    tags[10:16, 12:20] = True
    boxes = cluster_tags(tags, buffer=1, max_size=8, min_size=8, parents=parents, periodic=periodic)
    allowed = nesting_mask(shape, parents, periodic)
    held = np.zeros(shape, dtype=int)
    for box in boxes:
        assert all(1 <= hi - lo <= 8 for lo, hi in box)
        region = tuple(slice(lo, hi) for lo, hi in box)
        assert allowed[region].all()
        held[region] += 1
    assert held.max() == 1
    grown = tags.copy()
    for a in range(2):
        up = np.roll(grown, 1, axis=a)
        down = np.roll(grown, -1, axis=a)
        if not periodic[a]:
            edge = [slice(None)] * 2
            edge[a] = 0
            up[tuple(edge)] = False
            edge[a] = -1
            down[tuple(edge)] = False
        grown = grown | up | down
    assert np.all(held[grown & allowed] == 1)
    # a box below the smallest side (4 cells here: min_size 8 on the refined level) has no
    # room left along that axis: each neighbouring slab is outside the level, outside the
    # nestable region, or holds part of another box
    for box in boxes:
        for a, (lo, hi) in enumerate(box):
            if hi - lo >= 4:
                continue
            for slab in ((hi, hi + 1), (lo - 1, lo)):
                if slab[0] < 0 or slab[1] > shape[a]:
                    continue
                region = tuple(slice(*slab) if b == a else slice(*box[b]) for b in range(2))
                assert held[region].any() or not allowed[region].all(), (box, a, slab)
