"""Regridding on the current (GPU): the reference's AMR properties.

``tests/unit/test_mhd_amr.py:69-89`` (three regrids of an Orszag–Tang vortex: each regrid
keeps the totals, the composite divergence stays at round-off, two refined levels) and
``tests/unit/test_mhd3d.py:83-92`` (3D regrid on the current of an Alfvén wave).
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

K = 2.0 * np.pi


def _orszag_tang(n, precision=64):
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    mesh = AMRHierarchy((n, n), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, True))
    model = MHD2D(mesh, precision=precision)
    model.set_state(
        25.0 / (36.0 * np.pi),
        (lambda x, y: -np.sin(K * y), lambda x, y: np.sin(K * x), 0.0),
        5.0 / (12.0 * np.pi),
        vector_potential=lambda x, y: (np.cos(2 * K * x) / (2 * K) + np.cos(K * y) / K) / np.sqrt(4 * np.pi),
        bz=lambda x, y: 0.1 * np.cos(K * x),
    )
    return model


def test_regrids_conserve_and_keep_the_field_divergence_free():
    model = _orszag_tang(16)
    start = model.totals()
    for _ in range(3):
        before = model.totals()
        model.regrid(model.current_tags(0.1, levels=2), max_patch_size=16)
        after = model.totals()
        for name in before:
            assert abs(after[name] - before[name]) < 1e-14, name
        assert model.composite_divergence() < 1e-12
        for _ in range(4):
            model.step()
    assert model.hierarchy.max_level == 2
    end = model.totals()
    for name in start:
        assert abs(end[name] - start[name]) < 1e-13
    assert model.divergence() < 1e-12
    assert model.composite_divergence() < 1e-12
    assert float(np.nanmin(model.dataset(2).pressure.values)) > 0.0


def test_3d_regrid_on_the_current():
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd3d import MHD3D

    model, _ = MHD3D.alfven_wave(8, precision=64)
    model.regrid(model.current_tags(0.1, levels=1), max_patch_size=8)
    assert model.hierarchy.max_level == 1
    assert len(model.hierarchy.patches_at_level(1)) > 1
    start = model.totals()
    model.run(0.05)
    assert abs(model.totals()["energy"] - start["energy"]) < 1e-13
    assert model.divergence() < 1e-14
