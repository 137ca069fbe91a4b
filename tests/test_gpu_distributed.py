"""A partitioned level on one GPU (`LocalCluster`): every rank's engine, its mailboxes
packed, moved by device copies and unpacked; the steps must equal, bitwise, the steps of
one engine holding the whole level (same kernels, same global dt)."""

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
        for i, g in enumerate(part.local):
            a, size = int(layout.rows[g]["off"]), int(layout.rows[g]["fstride"]) * nf
            b, _ = part.block(i)
            e.state[b : b + size].copy_(eng.state[a : a + size])
    for _ in range(steps):
        model.advance(1)
        cluster.step(model.cfl)
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
