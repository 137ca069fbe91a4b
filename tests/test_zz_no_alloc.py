"""wb_rate_static (GPU): the rate reduction with its keys in static device scratch.

Compared with the existing entry point (wb_rate, keys in a caller buffer, decoded on the
host) on two calls in a row — a high-rate state, then a lower-rate one, so a scratch not
re-initialised between calls would return the first call's maximum — for batched 2D
float32 instances of different sizes and a 3D float64 hierarchy with refined patches.
This file is collected last and must pass alone as well.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _rate_static(engine, ninstances=None, out=None):
    from wellbalanced_b200 import _lib

    n = engine.ninstances if ninstances is None else ninstances
    if out is None:
        out = torch.full((2 * n,), float("nan"), dtype=torch.float64, device=engine.device)
    b = engine.mean_field
    lib = _lib.load()
    status = lib.wb_rate_static(engine.precision, engine.ndim, engine.state.data_ptr(), engine.patches.data_ptr(),
                                engine.layout.npatches, engine.chunk_patch.data_ptr(), engine.chunk_start.data_ptr(),
                                engine.nchunks, b[0], b[1], b[2], engine.gamma, n, out.data_ptr(),
                                torch.cuda.current_stream(engine.device).cuda_stream)
    return status, out


def _existing(engine):
    engine.rate()
    return engine.rate_values()


def _scaled_batch(speed):
    from wellbalanced_b200.batch import Batch
    from wellbalanced_b200.problems import orszag_tang_2d

    batch = Batch([32, 48, 32], precision=32)
    for k, side in enumerate(batch.sides):
        fields, az = orszag_tang_2d(side[0], 1.0 + 0.1 * k, speed * (1.0 + 0.2 * k), gamma=batch.gamma)
        batch.set_instance(k, fields, az)
    batch.finish_state()
    return batch


def test_batched_instances_match_the_existing_entry_point_on_two_calls():
    fast, slow = _scaled_batch(3.0), _scaled_batch(0.5)
    for batch in (fast, slow):  # two calls in a row, the second on lower rates
        status, out = _rate_static(batch.engine)
        assert status == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(-1, 2)
        expect = _existing(batch.engine)
        np.testing.assert_array_equal(got, expect)
    assert np.all(_existing(slow.engine)[:, 0] < _existing(fast.engine)[:, 0])


def test_refined_3d_matches_the_existing_entry_point_on_two_calls():
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd3d import MHD3D

    mesh = AMRHierarchy((8, 8, 8), ((0.0, 1.0),) * 3, periodic=(True, True, True))
    mesh.add_patch(1, ((4, 12), (4, 12), (4, 12)))
    model = MHD3D(mesh, precision=64)
    for amplitude in (2.0, 0.25):
        model.set_state(
            1.0,
            (lambda x, y, z, a=amplitude: a * np.sin(2 * np.pi * y), 0.0, 0.0),
            1.0,
            vector_potential=(0.0, 0.0, lambda x, y, z: 0.1 * np.cos(2 * np.pi * x)),
        )
        status, out = _rate_static(model.engine)
        assert status == 0
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy().reshape(-1, 2), _existing(model.engine))


def test_more_instances_than_the_scratch_holds_are_rejected():
    from wellbalanced_b200 import _lib

    batch = _scaled_batch(1.0)
    out = torch.zeros(2, dtype=torch.float64, device=batch.engine.device)
    status, _ = _rate_static(batch.engine, ninstances=4097, out=out)
    assert status == -4
    assert "4096 instances" in _lib.load().wb_last_error().decode()


def test_a_patch_beyond_the_instance_count_makes_every_value_nan():
    """A patch whose instance index is not below the count given is skipped by the rate
    kernel (nothing is written outside the instances' slots) and the whole output is NaN;
    the next call with the right count is correct again."""
    batch = _scaled_batch(1.0)
    status, out = _rate_static(batch.engine, ninstances=2)
    assert status == 0
    torch.cuda.synchronize()
    assert np.all(np.isnan(out.cpu().numpy()))
    status, out = _rate_static(batch.engine)
    assert status == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy().reshape(-1, 2), _existing(batch.engine))
