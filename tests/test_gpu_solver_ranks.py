"""The solvers on a hierarchy partitioned over ranks (GPU, two gloo ranks on one device).

As the reference's MPI tests (``tests/unit/test_mhd_mpi.py:31-51`` with
``_mpi_mhd_job.py`` / ``_mpi_mhd3d_job.py``): every rank builds the solver on the
hierarchy of a process group (``AMRHierarchy(..., comm=group)``), which holds only its
patches, and also the same case on a one-rank hierarchy; after steps at the global stable
step, the rank's patches equal the one-rank run's bit for bit and the global totals agree.
The two ranks exchange their mailboxes through host memory (gloo), so their kernels never
wait on one another.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

K = 2.0 * np.pi


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _mesh2d(comm):
    from wellbalanced_b200.mesh import AMRHierarchy

    mesh = AMRHierarchy((32, 16), ((-1.0, 1.0), (-0.5, 0.5)), periodic=(True, False), comm=comm, split=(2, 1))
    mesh.add_patch(1, ((8, 24), (8, 24)))
    mesh.add_patch(1, ((36, 56), (6, 26)))
    return mesh


def _mesh3d(comm):
    from wellbalanced_b200.mesh import AMRHierarchy

    mesh = AMRHierarchy((12, 12, 12), ((0.0, 1.0),) * 3, periodic=(True, True, True), comm=comm, split=(2, 1, 1))
    mesh.add_patch(1, ((4, 12), (6, 18), (4, 20)))
    mesh.add_patch(1, ((14, 22), (6, 18), (4, 20)))
    return mesh


def _model(ndim, comm, precision):
    if ndim == 2:
        from wellbalanced_b200.mhd import MHD2D

        model = MHD2D(_mesh2d(comm), limiter="mc", precision=precision, resistivity=1e-3, conduction=(1e-2, 1e-3))
        model.set_state(lambda x, y: 1.0 + 0.5 * np.exp(-((x + 0.3) ** 2 + y**2) / 0.02), (1.0, 0.5, 0.2),
                        lambda x, y: 1.0 + 0.2 * np.cos(np.pi * x),
                        vector_potential=lambda x, y: 0.1 * np.maximum(0.3 - np.hypot(x, y), 0.0),
                        bz=lambda x, y: 0.1 * np.sin(np.pi * x))
        return model
    from wellbalanced_b200.mhd3d import MHD3D

    model = MHD3D(_mesh3d(comm), limiter="mc", precision=precision)
    model.set_state(lambda x, y, z: 1.0 + 0.2 * np.sin(K * (x + y)),
                    (lambda x, y, z: 0.5 * np.sin(K * y), 0.2, lambda x, y, z: 0.3 * np.sin(K * x)), 1.0,
                    vector_potential=(0.0, lambda x, y, z: 0.05 * np.cos(K * x), lambda x, y, z: 0.1 * np.cos(K * y)))
    return model


def _job(rank, world, port, ndim, precision):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        torch.cuda.set_device(0)
        part = _model(ndim, dist.group.WORLD, precision)
        single = _model(ndim, None, precision)
        local = [p.index for p in part._local()]
        assert 0 < len(local) < len(part.hierarchy.patches)
        start = single.totals()
        for _ in range(3):
            assert part.step() == single.step()
        part.advance(2)
        single.advance(2)
        assert part.time == single.time
        nfields = 7 if ndim == 2 else 8
        for patch in part._local():
            twin = single.hierarchy.patches[patch.index]
            for f in range(nfields):
                if ndim == 2:
                    a, b = part.gather(patch, f, node=f == 6), single.gather(twin, f, node=f == 6)
                else:
                    a, b = part.gather(patch, f), single.gather(twin, f)
                np.testing.assert_array_equal(a, b, err_msg=f"rank {rank} patch {patch.index} field {f}")
        totals, want = part.totals(), single.totals()
        for key in want:
            assert abs(totals[key] - want[key]) <= 1e-14 * max(1.0, abs(want[key])), key
            if ndim == 3:  # periodic: nothing leaves the box
                assert abs(totals[key] - start[key]) <= 1e-12 * max(1.0, abs(start[key])), key
        assert part.divergence() == single.divergence()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ndim, precision", [(2, 64), (2, 32), (3, 64)])
def test_partitioned_solver_equals_one_rank(ndim, precision):
    import torch.multiprocessing as mp

    mp.spawn(_job, args=(2, _free_port(), ndim, precision), nprocs=2, join=True)
