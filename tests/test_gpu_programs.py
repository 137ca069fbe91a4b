"""Op programs (GPU): the reflux, restriction, halo-fill and stable-step phases of a
refined step in one launch each (`wb_run_program`).

A step through programs must equal, bit for bit, the step through the standalone launches
at the same dt (the same device bodies and arithmetic per point): refined 2D and 3D
hierarchies in float32, float64 and the mixed precision, with the non-ideal terms and the
per-level conduction limit, directly and replayed from a CUDA graph. A phase wait that
never completes ends after its bounded wait with the program's error bit set, and the
next launch runs normally.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _refined_2d(precision, **options):
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    mesh = AMRHierarchy((32, 16), ((-1.0, 1.0), (-0.5, 0.5)), periodic=(True, False))
    mesh.add_patch(1, ((16, 48), (8, 24)))
    mesh.add_patch(2, ((40, 72), (20, 36)))
    model = MHD2D(mesh, limiter="mc", precision=precision, mean_field=(0.1, 0.05), **options)
    model.set_state(lambda x, y: 1.0 + 0.5 * np.exp(-((x + 0.1) ** 2 + y**2) / 0.02), (1.0, 0.5, 0.3),
                    lambda x, y: 1.0 + 0.2 * np.cos(np.pi * x),
                    vector_potential=lambda x, y: 0.1 * np.maximum(0.3 - np.hypot(x, y), 0.0),
                    bz=lambda x, y: 0.1 * np.sin(np.pi * x))
    return model


def _refined_3d(precision, **options):
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd3d import MHD3D

    mesh = AMRHierarchy((12, 12, 12), ((0.0, 1.0),) * 3, periodic=(True, True, True))
    mesh.add_patch(1, ((6, 18), (6, 18), (4, 20)))
    model = MHD3D(mesh, precision=precision, limiter="mc", **options)
    k = 2.0 * np.pi
    model.set_state(lambda x, y, z: 1.0 + 0.2 * np.sin(k * (x + y)),
                    (lambda x, y, z: 0.5 * np.sin(k * y), 0.2, lambda x, y, z: 0.3 * np.sin(k * x)), 1.0,
                    vector_potential=(0.0, lambda x, y, z: 0.05 * np.cos(k * x), lambda x, y, z: 0.1 * np.cos(k * y)))
    return model


def _pair(build, precision, **options):
    a, b = build(precision, **options), build(precision, **options)
    assert a.engine.max_level > 0 and not a.engine.use_programs  # separate launches by default
    a.engine.use_programs = True
    return a, b


CASES = [
    ("2d float32", _refined_2d, 32, {}),
    ("2d float64 non-ideal", _refined_2d, 64, dict(resistivity=2e-3, conduction=(2e-2, 1e-3), gravity=(0.0, -0.1))),
    ("2d mixed", _refined_2d, "mixed", {}),
    ("3d float32", _refined_3d, 32, {}),
    ("3d float64 resistive", _refined_3d, 64, dict(resistivity=1e-3)),
]


@pytest.mark.parametrize("name, build, precision, options", CASES, ids=[c[0] for c in CASES])
def test_programmed_steps_equal_the_standalone_launches(name, build, precision, options):
    programmed, standalone = _pair(build, precision, **options)
    launches = programmed.engine.launches
    programmed.advance(6)
    per_step = (programmed.engine.launches - launches) / 6
    standalone.advance(6)
    assert programmed.time == standalone.time
    assert torch.equal(programmed.engine.state, standalone.engine.state), name
    # the programmed step leaves the next step's dt; the standalone path forms it on demand
    kappa = max(standalone.conduction) if hasattr(standalone, "conduction") else 0.0
    standalone.engine.prime_dt(standalone.cfl, standalone.resistivity, kappa)
    assert torch.equal(programmed.engine.dt, standalone.engine.dt)
    # stage kernels, face fluxes and two programs per step (and the priming rate / dt)
    assert per_step <= 8, per_step


def test_programmed_graph_replays_equal_direct_programmed_steps():
    direct, graphed = _refined_2d(32), _refined_2d(32)
    graphed.capture()  # takes one step
    direct.advance(1)
    graphed.advance(5)
    direct.advance(5)
    assert graphed.time == direct.time
    assert torch.equal(graphed.engine.state, direct.engine.state)


def test_conduction_limit_per_level_through_programs():
    """The per-level conduction limit (each level's smallest density with its spacing) in
    the program's rate and dt phases equals the standalone rate and finalize kernels."""
    programmed, standalone = _pair(_refined_2d, 64, conduction=(0.5, 0.1))
    assert programmed.engine.per_level_dt
    for _ in range(3):
        programmed.advance(1)
        standalone.advance(1)
        standalone.engine.prime_dt(standalone.cfl, standalone.resistivity, max(standalone.conduction))
        assert torch.equal(programmed.engine.dt, standalone.engine.dt)
    assert torch.equal(programmed.engine.state, standalone.engine.state)


def test_a_phase_wait_that_never_completes_sets_the_error_bit():
    """The ticket counter starts past the first item, so phase 0 never completes and the
    first wait of phase 1 runs out after its bounded wait: the error word gets bit 2, no
    later phase runs, the launch returns, and the counters are left for the next launch."""
    from wellbalanced_b200 import _lib

    model = _refined_2d(32)
    eng = model.engine
    first, _ = eng.programs(model._groups_potential, model._groups_all)
    segments, params, counters = first
    assert int(segments["phase"].max()) >= 1
    counters[0] = 1  # no block takes the first ticket (an item of phase 0)
    torch.cuda.synchronize()
    lib = _lib.load()
    status = lib.wb_run_program(eng.precision, eng.state.data_ptr(), eng.stage_pool.data_ptr(),
                                eng.patches.data_ptr(), segments.ctypes.data, int(segments.size),
                                ctypes.addressof(params), counters.data_ptr(),
                                torch.cuda.current_stream().cuda_stream)
    assert status == 0
    torch.cuda.synchronize()
    words = counters.cpu().numpy()
    assert words[2] & 2
    assert words[0] == 0 and words[1] == 0 and not words[3:].any()
    counters[2] = 0
    eng.run_program(first)  # the next launch runs normally
    torch.cuda.synchronize()
    assert int(counters[2].item()) == 0


def test_program_arguments_are_checked():
    from wellbalanced_b200 import _lib

    model = _refined_2d(32)
    eng = model.engine
    first, _ = eng.programs(model._groups_potential, model._groups_all)
    segments, params, counters = first
    bad = segments.copy()
    bad["phase"][-1] = int(bad["phase"][-1]) + 2  # a gap in the phases
    lib = _lib.load()
    status = lib.wb_run_program(eng.precision, eng.state.data_ptr(), eng.stage_pool.data_ptr(),
                                eng.patches.data_ptr(), bad.ctypes.data, int(bad.size), ctypes.addressof(params),
                                counters.data_ptr(), None)
    assert status == -1 and b"phase" in lib.wb_last_error()
