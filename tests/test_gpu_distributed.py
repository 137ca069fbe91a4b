"""A partitioned hierarchy on one GPU (`LocalCluster`): every rank's engine, its
mailboxes packed, moved by device copies, read through proxies; the steps must equal,
bitwise, the steps of one engine holding the whole hierarchy (same kernels, same global
dt). Single levels and refined hierarchies (halos interpolated from, restriction into and
face fluxes against patches of other ranks), ideal and with the non-ideal terms. The
mailbox areas start as NaN, so a kernel reading outside the boxes shipped to it fails
the comparison."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _check(model, world, steps=4):
    from wellbalanced_b200.distributed import LocalCluster, partition

    eng = model.engine
    layout = eng.layout
    owner = partition(model.hierarchy, world)
    cluster = LocalCluster(layout, owner, precision=eng.precision, limiter=eng.limiter, gamma=eng.gamma,
                           mean_field=eng.mean_field)
    nf = layout.nfields
    for part, e in zip(cluster.parts, cluster.engines, strict=True):
        e.physics = eng.physics
        start, end = part.mailbox_range()
        for pool in (e.state, e.stage_pool):
            pool[start:end] = float("nan")
        for i, g in enumerate(part.local):
            a, size = int(layout.rows[g]["off"]), int(layout.rows[g]["fstride"]) * nf
            b, _ = part.block(i)
            e.state[b : b + size].copy_(eng.state[a : a + size])
    eta = getattr(model, "resistivity", 0.0)
    kappa = max(getattr(model, "conduction", (0.0,)))
    for _ in range(steps):
        model.advance(1)
        cluster.step(model.cfl, eta, kappa)
    torch.cuda.synchronize()
    for part, e in zip(cluster.parts, cluster.engines, strict=True):
        assert float(e.dt[0].item()) == float(eng.dt[0].item())
        for i, g in enumerate(part.local):
            a, size = int(layout.rows[g]["off"]), int(layout.rows[g]["fstride"]) * nf
            b, _ = part.block(i)
            assert torch.equal(e.state[b : b + size], eng.state[a : a + size]), (part.rank, g)


def test_partitioned_2d_steps_equal_the_whole_level():
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    k = 2.0 * np.pi
    model = MHD2D(AMRHierarchy((48, 32), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, False), split=(3, 2)),
                  precision=32, limiter="mc")
    model.set_state(
        25.0 / (36.0 * np.pi),
        (lambda x, y: -np.sin(k * y), lambda x, y: np.sin(k * x), 0.0),
        5.0 / (12.0 * np.pi),
        vector_potential=lambda x, y: (np.cos(2 * k * x) / (2 * k) + np.cos(k * y) / k) / np.sqrt(4 * np.pi),
    )
    _check(model, 2)
    _check(model, 3)


def test_partitioned_3d_steps_equal_the_whole_level():
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd3d import MHD3D
    n, k = 24, 2.0 * np.pi
    model = MHD3D(AMRHierarchy((n,) * 3, ((0.0, 1.0),) * 3, periodic=(True,) * 3, split=(2, 2, 1)), precision=32,
                  limiter="mc", cfl=0.3)
    model.set_state(
        lambda x, y, z: 1.0 + 0.2 * np.sin(k * (x + y)),
        (lambda x, y, z: 0.5 * np.sin(k * y), lambda x, y, z: 0.5 * np.sin(k * z), lambda x, y, z: 0.5 * np.sin(k * x)),
        1.0,
        vector_potential=(lambda x, y, z: 0.1 * np.cos(k * z), lambda x, y, z: 0.1 * np.cos(k * x),
                          lambda x, y, z: 0.1 * np.cos(k * y)),
    )
    _check(model, 2)
    _check(model, 3)


def _refined_2d(precision, **options):
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    h = AMRHierarchy((32, 16), ((-1.0, 1.0), (-0.5, 0.5)), periodic=(True, False), split=(2, 2))
    h.add_patch(1, ((16, 40), (8, 24)))
    h.add_patch(1, ((40, 56), (4, 20)))
    h.add_patch(2, ((40, 72), (20, 44)))
    model = MHD2D(h, limiter="minmod", precision=precision, **options)
    model.set_state(lambda x, y: 1.0 + 0.5 * np.exp(-((x + 0.3) ** 2 + y**2) / 0.02), (2.0, 1.0, 0.3),
                    lambda x, y: 1.0 + 0.2 * np.cos(np.pi * x),
                    vector_potential=lambda x, y: 0.1 * np.maximum(0.3 - np.hypot(x, y), 0.0),
                    bz=lambda x, y: 0.1 * np.sin(np.pi * x))
    return model


def test_partitioned_refined_2d_steps_equal_the_whole_hierarchy():
    _check(_refined_2d(64), 2)
    _check(_refined_2d(64), 3)
    _check(_refined_2d(32), 3)
    _check(_refined_2d(64, resistivity=2e-3, conduction=(2e-2, 1e-3), gravity=(0.0, -0.1)), 2)


def test_partitioned_refined_3d_steps_equal_the_whole_hierarchy():
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd3d import MHD3D

    k = 2.0 * np.pi
    for options in ({}, {"resistivity": 0.01, "gravity": (0.0, 0.0, -0.1)}):
        h = AMRHierarchy((16, 8, 8), ((0.0, 2.0), (0.0, 1.0), (0.0, 1.0)), periodic=(True,) * 3, split=(2, 1, 1))
        h.add_patch(1, ((8, 20), (4, 12), (2, 10)))
        h.add_patch(1, ((20, 28), (2, 10), (4, 14)))
        model = MHD3D(h, precision=64, limiter="mc", cfl=0.3, mean_field=(0.3, 0.2, 0.1), lx=8, **options)
        model.set_state(
            lambda x, y, z: 1.0 + 0.2 * np.sin(k * (x + y)),
            (lambda x, y, z: 0.5 * np.sin(k * y), lambda x, y, z: 0.5 * np.sin(k * z), 0.0),
            1.0,
            vector_potential=(lambda x, y, z: 0.1 * np.cos(k * z), lambda x, y, z: 0.1 * np.cos(k * x),
                              lambda x, y, z: 0.1 * np.cos(k * y)),
        )
        _check(model, 2, steps=3)
