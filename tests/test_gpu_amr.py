"""Refined patches on the device: halos from coarser levels, restriction, refluxing (GPU).

The device float64 step on hierarchies with refined patches against the oracle's AMR
step (the same semantics, restated on the CPU: `oracle.mesh`), patch by patch, and the
reference's own properties of refined runs (``tests/unit/test_mhd.py:164-211``,
``tests/unit/test_mhd3d.py:72-80``): conserved totals to round-off, div B and the
composite divergence at round-off, the refined solution close to the uniform one.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _refined_state():
    return dict(
        density=lambda x, y: 1.0 + 0.5 * np.exp(-((x + 0.3) ** 2 + y**2) / 0.02),
        velocity=(2.0, 1.0, 0.3),
        pressure=lambda x, y: 1.0 + 0.2 * np.cos(np.pi * x),
        vector_potential=lambda x, y: 0.1 * np.maximum(0.3 - np.hypot(x, y), 0.0),
        bz=lambda x, y: 0.1 * np.sin(np.pi * x),
    )


def _pair(cells=16, precision=64, **options):
    from oracle.mesh import Hierarchy
    from oracle.mhd2d import MHD2D as OracleMHD2D
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    box = ((cells - cells // 2, cells + cells // 2), (cells // 2, 3 * cells // 2))
    oh = Hierarchy((2 * cells, cells), ((-1.0, 1.0), (-0.5, 0.5)), (True, True))
    oh.add_patch(1, box)
    dh = AMRHierarchy((2 * cells, cells), ((-1.0, 1.0), (-0.5, 0.5)), periodic=(True, True))
    dh.add_patch(1, box)
    oracle = OracleMHD2D(oh, limiter="minmod", **options)
    device = MHD2D(dh, limiter="minmod", precision=precision, **options)
    state = _refined_state()
    oracle.set_state(state["density"], state["velocity"], state["pressure"],
                     vector_potential=state["vector_potential"], bz=state["bz"])
    device.set_state(state["density"], state["velocity"], state["pressure"],
                     vector_potential=state["vector_potential"], bz=state["bz"])
    return oracle, device


def test_refined_2d_conduction_step_takes_each_levels_density_with_its_spacing():
    """The conduction limit of the time step (carafe/mhd.py:942-960) pairs each patch's
    smallest density with that patch's own spacing. The thinnest gas sits on the coarse
    level, outside the fine patch: the device's own dt (no dt passed) equals the
    oracle's stable_step on every step, not the stricter limit of the coarse density at
    the fine spacing."""
    from oracle.mesh import Hierarchy
    from oracle.mhd2d import MHD2D as OracleMHD2D
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    cells = 16
    box = ((cells - cells // 2, cells + cells // 2), (cells // 2, 3 * cells // 2))
    oh = Hierarchy((2 * cells, cells), ((-1.0, 1.0), (-0.5, 0.5)), (True, True))
    oh.add_patch(1, box)
    dh = AMRHierarchy((2 * cells, cells), ((-1.0, 1.0), (-0.5, 0.5)), periodic=(True, True))
    dh.add_patch(1, box)
    options = dict(conduction=(0.5, 0.1), mean_field=(0.1, 0.05))
    oracle = OracleMHD2D(oh, limiter="minmod", **options)
    device = MHD2D(dh, limiter="minmod", precision=64, **options)
    state = dict(
        density=lambda x, y: 1.0 - 0.6 * np.exp(-((x - 0.8) ** 2 + y**2) / 0.01),
        velocity=(0.2, 0.1, 0.0),
        pressure=1.0,
        vector_potential=lambda x, y: 0.05 * np.cos(np.pi * x),
    )
    for model in (oracle, device):
        model.set_state(state["density"], state["velocity"], state["pressure"],
                        vector_potential=state["vector_potential"])
    for _ in range(4):
        expect = oracle.step()
        got = device.step()
        assert got == pytest.approx(expect, rel=1e-13)
    # the coarse density at the fine spacing would have given a step 2.5x shorter
    rho_min = min(float(np.min(p.field(oracle.names["density"]).local)) for p in oh.patches)
    fine = sum(d**-2 for d in oh.spacing(1))
    assert got > 1.5 * oracle.cfl * 0.5 / ((oracle.gamma - 1.0) * 0.5 / rho_min * fine)


def test_refined_2d_matches_the_oracle_patch_by_patch():
    oracle, device = _pair()
    for _ in range(12):
        dt = oracle.step()
        device.step(dt)
    for op, dp in zip(oracle.hierarchy.patches, device.hierarchy.patches, strict=True):
        for f, name in enumerate(oracle.names.values()):
            np.testing.assert_allclose(device.gather(dp, f), op.field(name).local, rtol=1e-11, atol=1e-12,
                                       err_msg=f"level {op.level} {name}")
        np.testing.assert_allclose(device.gather(dp, 6, node=True), op.field(oracle.potential).local,
                                   rtol=1e-11, atol=1e-12)


def test_refined_2d_with_resistivity_conduction_and_gravity_matches_the_oracle():
    """The flux register carries the resistive and conductive face terms (the reference
    records its fluxes after adding them, carafe/mhd.py:866-872, 906-919): the refined
    non-ideal step matches the oracle's patch by patch, and without gravity the composite
    totals stay at round-off."""
    physics = dict(resistivity=2e-3, conduction=(2e-2, 1e-3), mean_field=(0.1, 0.05))
    oracle, device = _pair(gravity=(0.05, -0.1), **physics)
    for _ in range(12):
        dt = oracle.step()
        device.step(dt)
    for op, dp in zip(oracle.hierarchy.patches, device.hierarchy.patches, strict=True):
        for f, name in enumerate(oracle.names.values()):
            np.testing.assert_allclose(device.gather(dp, f), op.field(name).local, rtol=1e-11, atol=1e-12,
                                       err_msg=f"level {op.level} {name}")
        np.testing.assert_allclose(device.gather(dp, 6, node=True), op.field(oracle.potential).local,
                                   rtol=1e-11, atol=1e-12)
    _, model = _pair(**physics)
    before = model.totals()
    for _ in range(20):
        model.step()
    after = model.totals()
    for name in before:
        assert abs(after[name] - before[name]) < 1e-12, name
    assert model.divergence() < 1e-14


def _oracle_leaf_values(oracle):
    """The reference's leaf_values (carafe/mhd.py:1059-1111) restated on the oracle, with
    the device's cell order (patch by patch, row-major)."""
    from wellbalanced_b200.mhd import covered_cells

    h = oracle.hierarchy
    oracle.fill_halos()
    parts = {}
    for patch in h.patches:
        nx, ny = patch.shape
        prim, bxf, byf, _, _ = oracle.primitive(patch)
        jz = oracle.current(bxf, byf, patch.level)
        corner = 0.25 * sum(jz[1 + a : 1 + a + nx, 1 + b : 1 + b + ny] for a in (0, 1) for b in (0, 1))
        values = np.stack([*(q[2 : 2 + nx, 2 : 2 + ny] for q in prim), corner])
        leaf = ~covered_cells(h, patch)
        for i, value in enumerate(values):
            parts.setdefault(i, []).append(value[leaf])
    return [np.concatenate(parts[i]) for i in range(9)]


def test_leaf_values_and_sheet_diagnostics_match_the_oracle():
    from wellbalanced_b200.mhd import MHD2D, sheet_diagnostics

    oracle, device = _pair()
    for _ in range(5):
        device.step(oracle.step())
    leaf = device.leaf_values()
    want = _oracle_leaf_values(oracle)
    for name, expected in zip(MHD2D.LEAF_VARIABLES, want, strict=True):
        np.testing.assert_allclose(leaf[name], expected, rtol=1e-11, atol=1e-12, err_msg=name)
    assert leaf["level"].max() == 1 and leaf["x"].size == leaf["density"].size
    mine = sheet_diagnostics(device, leaf)
    theirs = sheet_diagnostics(device, {**leaf, **dict(zip(MHD2D.LEAF_VARIABLES, want, strict=True))})
    assert mine["o_points"] == theirs["o_points"] and mine["x_points"] == theirs["x_points"]
    assert abs(mine["psi"] - theirs["psi"]) < 1e-12 and abs(mine["max_current"] - theirs["max_current"]) < 1e-10


def test_refined_2d_conserves_and_keeps_div_b_zero():
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    _, model = _pair()
    before = model.totals()
    model.run(0.2)
    after = model.totals()
    for name in before:
        assert abs(after[name] - before[name]) < 1e-12
    assert model.divergence() < 1e-14
    assert model.composite_divergence() < 1e-14
    # close to the uniform solution (test_mhd.py:193-211)
    _, refined = _pair()
    refined.run(0.1)
    uniform = MHD2D(AMRHierarchy((32, 16), ((-1.0, 1.0), (-0.5, 0.5)), periodic=(True, True)), limiter="minmod",
                    precision=64)
    s = _refined_state()
    uniform.set_state(s["density"], s["velocity"], s["pressure"], vector_potential=s["vector_potential"], bz=s["bz"])
    uniform.run(0.1)
    difference = refined.dataset().density.values - uniform.dataset().density.values
    assert float(np.abs(difference).max()) < 0.05


def test_refined_2d_float32_drift_is_at_float32_round_off():
    _, model = _pair(precision=32)
    before = model.totals()
    for _ in range(50):
        model.step()
    after = model.totals()
    for name in before:
        assert abs(after[name] - before[name]) < 1e-5 * max(1.0, abs(before[name])), name
    assert model.divergence() < 1e-12
    assert model.composite_divergence() < 1e-6


def _alfven_pair(precision=64, device_cls=None, **options):
    from oracle.mesh import Hierarchy
    from oracle.mhd3d import MHD3D as OracleMHD3D
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd3d import MHD3D

    MHD3D = device_cls or MHD3D  # noqa: N806

    wavevector = 2 * np.pi * np.array([0.5, 1.0, 1.0])
    k = np.linalg.norm(wavevector)
    n = wavevector / k
    e1 = np.cross(n, [0.0, 0.0, 1.0])
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(n, e1)

    def perpendicular(x, y, z):
        phase = wavevector[0] * x + wavevector[1] * y + wavevector[2] * z
        return [0.1 * (np.sin(phase) * e1[i] + np.cos(phase) * e2[i]) for i in range(3)]

    def potential(i):
        return lambda x, y, z: perpendicular(x, y, z)[i] / k

    bounds = ((0.0, 2.0), (0.0, 1.0), (0.0, 1.0))
    oh = Hierarchy((16, 8, 8), bounds, (True,) * 3)
    oh.add_patch(1, ((8, 20), (4, 12), (2, 10)))
    dh = AMRHierarchy((16, 8, 8), bounds, periodic=(True,) * 3)
    dh.add_patch(1, ((8, 20), (4, 12), (2, 10)))
    models = (OracleMHD3D(oh, mean_field=tuple(n), **options),
              MHD3D(dh, mean_field=tuple(n), precision=precision, **options))
    for m in models:
        m.set_state(1.0, lambda x, y, z: [-b for b in perpendicular(x, y, z)], 0.1,
                    vector_potential=(potential(0), potential(1), potential(2)))
    return models


def test_refined_3d_matches_the_oracle_and_conserves():
    oracle, device = _alfven_pair()
    before = device.totals()
    for _ in range(6):
        dt = oracle.step()
        device.step(dt)
    for op, dp in zip(oracle.hierarchy.patches, device.hierarchy.patches, strict=True):
        names = [*oracle.names.values(), *oracle.potential]
        for f, name in enumerate(names):
            np.testing.assert_allclose(device.gather(dp, f), op.field(name).local, rtol=1e-11, atol=1e-12,
                                       err_msg=f"level {op.level} {name}")
    after = device.totals()
    for name in before:
        assert abs(after[name] - before[name]) < 1e-14 * max(1.0, abs(before[name])) * 100
    assert device.divergence() < 1e-14


def test_refined_3d_with_resistivity_and_gravity_matches_the_oracle():
    """The fused 3D kernel's resistive and gravity terms on a refined hierarchy: the flux
    register carries eta (J x B) on the recomputed coarse and fine faces (the reference
    records the energy fluxes after adding it, carafe/mhd3d.py:630-632, 651-657)."""
    oracle, device = _alfven_pair(resistivity=0.01, gravity=(0.02, -0.05, 0.03))
    for _ in range(6):
        dt = oracle.step()
        device.step(dt)
    for op, dp in zip(oracle.hierarchy.patches, device.hierarchy.patches, strict=True):
        names = [*oracle.names.values(), *oracle.potential]
        for f, name in enumerate(names):
            np.testing.assert_allclose(device.gather(dp, f), op.field(name).local, rtol=1e-11, atol=1e-12,
                                       err_msg=f"level {op.level} {name}")
    _, device = _alfven_pair(resistivity=0.01)
    before = device.totals()
    for _ in range(6):
        device.step()
    after = device.totals()
    for name in before:
        assert abs(after[name] - before[name]) < 1e-12 * max(1.0, abs(before[name])), name
    assert device.divergence() < 1e-14


def test_graph_replay_equals_direct_steps_on_a_refined_hierarchy():
    """`capture` records one step of the whole hierarchy; replays equal direct launches."""
    import torch

    _, a = _pair(precision=32)
    _, b = _pair(precision=32)
    a.advance(5)
    b.capture()
    b.advance(4)
    torch.cuda.synchronize()
    assert a.steps == b.steps == 5
    assert a.time == b.time
    np.testing.assert_array_equal(a.engine.state.cpu().numpy(), b.engine.state.cpu().numpy())


def test_plain_float64_paths_reflux_like_the_oracle():
    """The per-kernel float64 paths on refined hierarchies: the flux register from the
    sweeps' own fluxes and the reflux after the step (patchwork's FluxRegister as the
    reference calls it), patch by patch against the oracle, in 2D (with resistivity and
    conduction) and 3D."""
    from oracle.mesh import Hierarchy
    from oracle.mhd2d import MHD2D as OracleMHD2D
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.plain import PlainMHD2D, PlainMHD3D

    cells = 16
    box = ((cells - cells // 2, cells + cells // 2), (cells // 2, 3 * cells // 2))
    for options in ({}, {"resistivity": 2e-3, "conduction": (2e-2, 1e-3)}):
        oh = Hierarchy((2 * cells, cells), ((-1.0, 1.0), (-0.5, 0.5)), (True, True))
        oh.add_patch(1, box)
        dh = AMRHierarchy((2 * cells, cells), ((-1.0, 1.0), (-0.5, 0.5)), periodic=(True, True))
        dh.add_patch(1, box)
        oracle = OracleMHD2D(oh, limiter="minmod", **options)
        plain = PlainMHD2D(dh, limiter="minmod", **options)
        s = _refined_state()
        for m in (oracle, plain):
            m.set_state(s["density"], s["velocity"], s["pressure"], vector_potential=s["vector_potential"], bz=s["bz"])
        for _ in range(6):
            plain.step(oracle.step())
        for op, dp in zip(oracle.hierarchy.patches, plain.hierarchy.patches, strict=True):
            for f, name in enumerate(oracle.names.values()):
                np.testing.assert_allclose(plain.gather(dp, f), op.field(name).local, rtol=1e-11, atol=1e-12,
                                           err_msg=f"level {op.level} {name} {options}")
    oracle, plain = _alfven_pair(device_cls=PlainMHD3D, resistivity=0.01)
    for _ in range(4):
        plain.step(oracle.step())
    for op, dp in zip(oracle.hierarchy.patches, plain.hierarchy.patches, strict=True):
        names = [*oracle.names.values(), *oracle.potential]
        for f, name in enumerate(names):
            np.testing.assert_allclose(plain.gather(dp, f), op.field(name).local, rtol=1e-11, atol=1e-12,
                                       err_msg=f"3D level {op.level} {name}")


@pytest.mark.parametrize("dims", [2, 3])
def test_fused_level_fill_and_overlapped_fluxes_equal_the_plain_sequence(dims):
    """The single-launch level fill (`wb_fill_ops`, interpolation ops trimmed to the points
    no copy writes) and the second stream of the flux register change no bit of a step
    against separate interpolation and copy launches on one stream."""
    import torch

    def make():
        return _pair(precision=32)[1] if dims == 2 else _alfven_pair(precision=32)[1]

    fused, plain = make(), make()
    plain.engine.fused_fill = False
    plain.engine.overlap_fluxes = False
    assert fused.engine.nface > 0
    pool_a, pool_b = fused.engine.state.clone(), plain.engine.state.clone()
    fused.engine.fill(pool_a)
    plain.engine.fill(pool_b)
    torch.cuda.synchronize()
    assert torch.equal(pool_a, pool_b)
    for _ in range(3):
        fused.advance(1)
        plain.advance(1)
    torch.cuda.synchronize()
    assert fused.time == plain.time
    assert torch.equal(fused.engine.state, plain.engine.state)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [32, 64, "mixed"])
def test_staged_fine_fluxes_equal_the_recomputed_register(precision):
    """2D ideal refined steps with the register's fine faces read from the stage kernels'
    boundary-face output equal steps whose register recomputes them: bit for bit where the
    faces are float32 arithmetic (every float32 face runs the same explicit lane code), to
    rounding in float64 (the compiler contracts the two kernels' float64 arithmetic
    differently); the staged run keeps the composite totals to round-off."""
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    models = []
    for staged in (True, False):
        mesh = AMRHierarchy((32, 32), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, True))
        mesh.add_patch(1, ((12, 40), (20, 44)))
        mesh.add_patch(2, ((30, 60), (48, 80)))
        model = MHD2D(mesh, limiter="mc", precision=precision)
        model.set_state(lambda x, y: 1.0 + 0.4 * np.exp(-((x - 0.5) ** 2 + (y - 0.55) ** 2) / 0.01),
                        (0.6, -0.3, 0.1), lambda x, y: 1.0 + 0.3 * np.cos(2 * np.pi * x),
                        vector_potential=lambda x, y: 0.05 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y),
                        bz=0.1)
        model.engine.staged_fluxes = staged
        models.append(model)
    assert models[0].engine._uses_staged_fluxes() and not models[1].engine._uses_staged_fluxes()
    start = models[0].totals()
    for _ in range(6):
        dts = [m.step() for m in models]
        if precision != 64:
            assert dts[0] == dts[1]
    a, b = models[0].engine.state, models[1].engine.state
    if precision == 64:
        assert torch.allclose(a, b, rtol=1e-12, atol=1e-13)
    else:
        assert torch.equal(a, b)
        assert torch.equal(models[0].engine.register, models[1].engine.register)
    end = models[0].totals()
    tol = 1e-6 if precision == 32 else 1e-13  # a float32 state rounds every update
    for key in start:
        assert abs(end[key] - start[key]) < tol * max(1.0, abs(start[key])), key
