"""Batched independent problems (GPU): every instance evolves as if alone.

`wellbalanced_b200.Batch` advances N periodic Orszag–Tang problems of different sizes,
each at its own CFL step, by one launch per kernel; each instance must equal the same
problem advanced alone by `MHD2D`, and graph replay must equal direct launches.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def test_batched_instances_equal_single_runs():
    from wellbalanced_b200.batch import Batch
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D
    from wellbalanced_b200.problems import orszag_tang_2d, orszag_tang_sizes

    sides, bf, vf = orszag_tang_sizes(5, seed=3, sides=(32, 48, 64))
    batch = Batch(sides, precision=64, limiter="mc", cfl=0.4)
    for k in range(5):
        fields, az = orszag_tang_2d(int(sides[k]), bf[k], vf[k])
        batch.set_instance(k, fields, az)
    batch.finish_state()
    batch.advance(6)
    times = batch.times()
    assert len(set(np.round(times, 12))) > 1  # each instance took its own steps
    for k in (0, 3):
        fields, az = orszag_tang_2d(int(sides[k]), bf[k], vf[k])
        n = int(sides[k])
        single = MHD2D(AMRHierarchy((n, n), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, True)), limiter="mc", cfl=0.4,
                       precision=64)
        single.set_conserved(fields, az)
        for _ in range(6):
            single.step()
        np.testing.assert_allclose(single.time, times[k], rtol=1e-13)
        got, want = batch.instance_state(k), single.state()
        for key in want:
            np.testing.assert_allclose(got[key], want[key], rtol=1e-12, atol=1e-12, err_msg=key)


def test_graph_replay_equals_direct_launches():
    from wellbalanced_b200.batch import Batch

    a = Batch.orszag_tang(6, seed=1, precision=32)
    b = Batch.orszag_tang(6, seed=1, precision=32)
    a.advance(4)
    b.capture()
    b.advance(3)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(a.engine.state.cpu().numpy(), b.engine.state.cpu().numpy())
    np.testing.assert_array_equal(a.times(), b.times())
