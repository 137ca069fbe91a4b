"""The fused device step (MHD2D / MHD3D) against the reference's own runs (GPU).

float64 state: the reference's step to 1e-12 (the golden runs of the reference's
``MHD2D``/``MHD3D`` — Orszag–Tang, all limiters, outflow rotor, uniform state, multi-patch
level, Alfvén wave, z-uniform 3D, 3D blast, 3D turbulence). float32 state: the stated
L1 error against the float64 reference, div B at round-off from the stored potential.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).with_name("golden")


@pytest.fixture(scope="module")
def runs2d():
    return np.load(GOLDEN / "runs2d.npz")


@pytest.fixture(scope="module")
def runs3d():
    return np.load(GOLDEN / "runs3d.npz")


def close(state, runs, prefix, tol):
    for key, value in state.items():
        np.testing.assert_allclose(value, runs[f"{prefix}_{key}"], rtol=tol, atol=tol, err_msg=f"{prefix}: {key}")


def rel_l1(a, b):
    return float(np.sum(np.abs(a - b)) / np.sum(np.abs(b)))


# --- 2D ---------------------------------------------------------------------------------------
def test_orszag_tang_steps_match_the_reference(runs2d):
    from wellbalanced_b200.mhd import MHD2D

    model = MHD2D.orszag_tang(32, precision=64)
    dts = [model.step() for _ in range(5)]
    np.testing.assert_allclose(dts, runs2d["ot32_5_dts"], rtol=1e-13)
    close(model.state(), runs2d, "ot32_5", 1e-12)


def test_orszag_tang_run_keeps_div_b_zero_and_conserves(runs2d):
    from wellbalanced_b200.mhd import MHD2D

    model = MHD2D.orszag_tang(32, precision=64)
    before = model.totals()
    model.run(0.1)
    after = model.totals()
    assert model.steps == int(runs2d["ot32_run_steps"])
    assert model.divergence() < 1e-14
    for name in before:
        assert abs(after[name] - before[name]) < 1e-13
    close(model.state(), runs2d, "ot32_run", 1e-11)
    assert float(model.dataset().pressure.min()) > 0.0


@pytest.mark.parametrize("limiter", ["minmod", "vanleer", "mc", "none"])
def test_every_limiter_matches_the_reference(runs2d, limiter):
    from wellbalanced_b200.mhd import MHD2D

    model = MHD2D.orszag_tang(24, limiter=limiter, precision=64)
    for _ in range(8):
        model.step()
    close(model.state(), runs2d, f"ot24_{limiter}", 1e-12)


def test_outflow_rotor_uniform_and_alfven_match_the_reference(runs2d):
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    model = MHD2D.rotor(32, precision=64)
    model.run(0.02)
    close(model.state(), runs2d, "rotor32", 1e-11)
    model = MHD2D(AMRHierarchy((8, 6), ((0.0, 1.0), (0.0, 1.0))), mean_field=(0.3, -0.2), limiter="mc", precision=64)
    model.set_state(1.0, (0.2, -0.1, 0.05), 0.5, bz=0.4)
    model.run(0.2)
    close(model.state(), runs2d, "uniform8x6", 1e-12)
    model, _ = MHD2D.alfven_wave(16, limiter="none", precision=64)
    model.run(model.period)
    close(model.state(), runs2d, "alfven16", 1e-11)


def test_brio_wu_along_both_axes_matches_the_reference(runs2d):
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    for axis in (0, 1):
        cells = 64
        if axis == 0:
            mesh = AMRHierarchy((cells, 2), ((0.0, 1.0), (0.0, 2.0 / cells)), periodic=(False, True))
        else:
            mesh = AMRHierarchy((2, cells), ((0.0, 2.0 / cells), (0.0, 1.0)), periodic=(True, False))
        model = MHD2D(mesh, gamma=2.0, mean_field=(0.75, 0.0) if axis == 0 else (0.0, 0.75), precision=64)
        sign = 1.0 if axis == 0 else -1.0

        def s(x, y, axis=axis):
            return x if axis == 0 else y

        model.set_state(
            lambda x, y: np.where(s(x, y) < 0.5, 1.0, 0.125),
            (0.0, 0.0, 0.0),
            lambda x, y: np.where(s(x, y) < 0.5, 1.0, 0.1),
            vector_potential=lambda x, y: sign * np.abs(s(x, y) - 0.5),
        )
        model.run(0.1)
        close(model.state(), runs2d, f"briowu{axis}", 1e-11)


def test_a_multi_patch_level_matches_the_reference():
    from wellbalanced_b200.mhd import MHD2D

    golden = np.load(GOLDEN / "multipatch.npz")
    model = MHD2D.orszag_tang(32, split=(2, 3), precision=64)
    for _ in range(5):
        model.step()
    np.testing.assert_allclose(model.state()["density"], golden["split_density"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("precision", [32, "mixed"])
def test_float32_orszag_tang_error_against_the_float64_reference(runs2d, precision):
    """Orszag-Tang 64^2 to t = 0.5 with float32 arithmetic (float32 or float64 state)
    against the reference's float64 run: relative L1 of density and energy within 1e-5,
    div B at round-off."""
    from wellbalanced_b200.mhd import MHD2D

    model = MHD2D.orszag_tang(64, limiter="mc", cfl=0.4, precision=precision)
    model.run(0.5)
    state = model.state()
    err_rho = rel_l1(state["density"], runs2d["ot64_mc_density"])
    err_e = rel_l1(state["energy"], runs2d["ot64_mc_energy"])
    print(f"{precision} OT 64^2 to t=0.5: rel L1 rho {err_rho:.3e}, E {err_e:.3e}, steps {model.steps}")
    assert err_rho < 1e-5 and err_e < 1e-5
    assert model.divergence() < 1e-12


def test_float32_near_degenerate_harris_sheet_tracks_float64():
    """A Harris sheet at rest has HLLD faces whose star denominator
    rho (S - u)(S - S_M) - B_n^2 nearly vanishes (Alfven speed close to the fast speed,
    small tangential field). Evaluated in float32 it cancels to noise: the float32 step
    drifted by 1e-3 per step and went negative. The float32 kernels redo those faces'
    wave speeds and star states in float64; float32 must then track float64 closely."""
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D
    from wellbalanced_b200.problems import harris_sheet

    bounds = ((-1.0, 1.0), (-2.0, 2.0))
    density, pressure, potential = harris_sheet(256, 512, seed=0, bounds=bounds)
    models = []
    for precision in (64, 32):
        model = MHD2D(AMRHierarchy((256, 512), bounds, periodic=(True, False)), limiter="mc", cfl=0.4,
                      precision=precision)
        model.set_state(density, (0.0, 0.0, 0.0), pressure, vector_potential=potential)
        models.append(model)
    ref, low = models
    for _ in range(6):
        low.step(ref.step())
    (pr,), (pl,) = ref.hierarchy.patches, low.hierarchy.patches
    for f in (0, 2, 4):  # density, m_y (near zero: absolute only), energy
        a, b = ref.gather(pr, f), low.gather(pl, f)
        assert np.max(np.abs(b - a)) < 2e-5, f
        if f != 2:
            assert np.sum(np.abs(b - a)) / np.sum(np.abs(a)) < 1e-6, f


def test_fused_step_with_gravity_resistivity_and_conduction_matches_the_reference(runs2d):
    """The non-ideal terms inside the fused 2D stage kernel (walls + gravity, resistivity,
    Braginskii conduction) against the reference's own runs; float32 close to them."""
    from wellbalanced_b200.mhd import MHD2D

    cases = [
        ("rt8", lambda p: MHD2D.rayleigh_taylor(8, field=0.05, precision=p), 20),
        ("ot16_resistive", lambda p: MHD2D.orszag_tang(16, resistivity=1e-3, conduction=(1e-2, 1e-3), precision=p), 3),
        ("rt8_resistive", lambda p: MHD2D.rayleigh_taylor(8, resistivity=1e-3, conduction=(1e-3, 0.0), field=0.05,
                                                          precision=p), 3),
    ]
    for name, make, steps in cases:
        model = make(64)
        assert model.engine.physics is not None
        for _ in range(steps):
            model.step()
        close(model.state(), runs2d, name, 1e-12)
        low = make(32)
        for _ in range(steps):
            low.step()
        state = low.state()
        for key in ("density", "energy"):
            assert rel_l1(state[key], runs2d[f"{name}_{key}"]) < 1e-6, (name, key)


def test_negative_pressure_is_reported():
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    model = MHD2D(AMRHierarchy((8, 8), periodic=(True, True)), precision=64)
    model.set_state(1.0, (0.0, 0.0, 0.0), 1e-3)
    (patch,) = model.hierarchy.patches
    view = model.engine.view(model.engine.state, patch, 4)
    view[5, 5] = -1.0
    with pytest.raises(FloatingPointError, match="pressure"):
        model.step(1e-3)


# --- 3D ---------------------------------------------------------------------------------------
def test_z_uniform_3d_matches_the_reference(runs3d):
    from wellbalanced_b200.mhd3d import MHD3D

    flat = MHD3D.orszag_tang(16, layers=2, precision=64)
    for dt in runs3d["ot3d16_dts"]:
        flat.step(float(dt))
    close(flat.state(), runs3d, "ot3d16", 1e-12)


def test_3d_alfven_blast_and_outflow_match_the_reference(runs3d):
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd3d import MHD3D

    model, _ = MHD3D.alfven_wave(8, limiter="none", precision=64)
    model.run(0.1)
    close(model.state(), runs3d, "alfven3d8", 1e-12)
    # The blast's quiescent exterior has exactly zero mass flux, where CT-contact's upwind
    # pick (ct_contact_pyccel.py:17-24) is discontinuous: the reference algorithm itself
    # moves by 4e-5 after these 6 steps when its energy is perturbed by 1e-15 (oracle
    # experiment), so this case is compared within that envelope, conservation exactly.
    model = MHD3D.blast_wave(12, precision=64)
    before = model.totals()
    model.run(0.01)
    close(model.state(), runs3d, "blast3d12", 1e-4)
    after = model.totals()
    for name in before:
        assert abs(after[name] - before[name]) < 1e-12 * max(1.0, abs(before[name]))
    assert model.divergence() < 1e-14
    mesh = AMRHierarchy((6, 4, 5), ((0.0, 1.0),) * 3, periodic=(False, True, False))
    model = MHD3D(mesh, mean_field=(0.3, -0.2, 0.5), precision=64)
    model.set_state(1.2, (0.1, -0.2, 0.3), 0.7)
    for _ in range(4):
        model.step()
    close(model.state(), runs3d, "uniform3d", 1e-12)
    mesh = AMRHierarchy((8, 6, 7), ((0.0, 1.0),) * 3, periodic=(False, True, False))
    model = MHD3D(mesh, mean_field=(0.3, -0.2, 0.5), limiter="mc", precision=64)
    model.set_state(
        lambda x, y, z: 1.0 + 0.3 * np.exp(-((x - 0.4) ** 2 + (y - 0.5) ** 2 + (z - 0.6) ** 2) / 0.05),
        (0.1, -0.2, 0.3),
        lambda x, y, z: 0.7 + 0.2 * np.cos(2 * np.pi * y),
        vector_potential=(
            lambda x, y, z: 0.05 * np.sin(2 * np.pi * y) * z,
            lambda x, y, z: 0.05 * x * z,
            lambda x, y, z: 0.05 * np.cos(2 * np.pi * y) * x,
        ),
    )
    for _ in range(4):
        model.step()
    close(model.state(), runs3d, "outflow3d", 1e-12)


def _turbulence(precision):
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd3d import MHD3D
    from wellbalanced_b200.problems import turbulence_3d

    rho, velocity, p, potential = turbulence_3d(16, seed=7)
    model = MHD3D(AMRHierarchy((16,) * 3, ((0.0, 1.0),) * 3, periodic=(True,) * 3), limiter="mc", cfl=0.3,
                  precision=precision)
    model.set_state(rho, velocity, p, vector_potential=potential)
    return model


def test_3d_turbulence_float64_matches_the_reference(runs3d):
    model = _turbulence(64)
    close(model.state(), runs3d, "turb16_init", 1e-14)
    dts = [model.step() for _ in range(4)]
    np.testing.assert_allclose(dts, runs3d["turb16_dts"], rtol=1e-13)
    close(model.state(), runs3d, "turb16", 1e-12)


def test_3d_turbulence_float32_error_and_div_b(runs3d):
    model = _turbulence(32)
    before = model.totals()
    for dt in runs3d["turb16_dts"]:
        model.step(float(dt))
    state = model.state()
    err_rho = rel_l1(state["density"], runs3d["turb16_density"])
    err_e = rel_l1(state["energy"], runs3d["turb16_energy"])
    print(f"float32 turbulence 16^3, 4 steps: rel L1 rho {err_rho:.3e}, E {err_e:.3e}")
    assert err_rho < 1e-5 and err_e < 1e-5
    assert model.divergence() < 1e-12
    after = model.totals()
    assert abs(after["density"] - before["density"]) < 1e-5


def test_3d_negative_pressure_is_reported():
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd3d import MHD3D

    model = MHD3D(AMRHierarchy((4, 4, 4), ((0.0, 1.0),) * 3, periodic=(True,) * 3), precision=64)
    model.set_state(1.0, (0.0, 0.0, 0.0), 1.0)
    (patch,) = model.hierarchy.patches
    model.engine.view(model.engine.state, patch, 4)[3, 3, 3] = -1.0
    with pytest.raises(FloatingPointError, match="pressure"):
        model.step(1e-3)


# --- the plain float64 step (per-kernel, the reference's dataflow) -----------------------------
def test_plain_2d_step_matches_the_reference_with_walls_gravity_resistivity(runs2d):
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.plain import PlainMHD2D

    model = PlainMHD2D(AMRHierarchy((32, 32), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, True)))
    b0 = 1.0 / np.sqrt(4.0 * np.pi)
    model.set_state(
        25.0 / (36.0 * np.pi),
        lambda x, y: (-np.sin(2 * np.pi * y), np.sin(2 * np.pi * x), 0.0 * x),
        5.0 / (12.0 * np.pi),
        vector_potential=lambda x, y: b0 * (np.cos(4 * np.pi * x) / (4 * np.pi) + np.cos(2 * np.pi * y) / (2 * np.pi)),
    )
    dts = [model.step() for _ in range(5)]
    np.testing.assert_allclose(dts, runs2d["ot32_5_dts"], rtol=1e-13)
    close(model.state(), runs2d, "ot32_5", 1e-12)
    # Rayleigh-Taylor: walls along y, gravity, a field along x (carafe/mhd.py:626-671)
    rt = PlainMHD2D(
        AMRHierarchy((8, 24), ((-0.25, 0.25), (-0.75, 0.75)), periodic=(True, False)),
        gamma=1.4, mean_field=(0.05, 0.0), gravity=(0.0, -0.1), boundaries={"y": "wall"},
    )

    def density(x, y):
        return np.where(y > 0.0, 2.0, 1.0)

    rt.set_state(
        density,
        lambda x, y: (0.0 * x, 0.01 * (1 + np.cos(4 * np.pi * x)) * (1 + np.cos(3 * np.pi * y)) / 4.0, 0.0 * x),
        lambda x, y: 2.5 - 0.1 * density(x, y) * y,
    )
    for _ in range(20):
        rt.step()
    close(rt.state(), runs2d, "rt8", 1e-12)
    # resistive + Braginskii-conductive Orszag-Tang
    model = PlainMHD2D(AMRHierarchy((16, 16), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, True)),
                       resistivity=1e-3, conduction=(1e-2, 1e-3))
    model.set_state(
        25.0 / (36.0 * np.pi),
        lambda x, y: (-np.sin(2 * np.pi * y), np.sin(2 * np.pi * x), 0.0 * x),
        5.0 / (12.0 * np.pi),
        vector_potential=lambda x, y: b0 * (np.cos(4 * np.pi * x) / (4 * np.pi) + np.cos(2 * np.pi * y) / (2 * np.pi)),
    )
    for _ in range(3):
        model.step()
    close(model.state(), runs2d, "ot16_resistive", 1e-12)


def test_plain_3d_step_matches_the_reference(runs3d):
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.plain import PlainMHD3D
    from wellbalanced_b200.problems import turbulence_3d

    rho, velocity, p, potential = turbulence_3d(16, seed=7)
    model = PlainMHD3D(AMRHierarchy((16,) * 3, ((0.0, 1.0),) * 3, periodic=(True,) * 3), limiter="mc", cfl=0.3)
    model.set_state(rho, velocity, p, vector_potential=potential)
    dts = [model.step() for _ in range(4)]
    np.testing.assert_allclose(dts, runs3d["turb16_dts"], rtol=1e-13)
    close(model.state(), runs3d, "turb16", 1e-12)


def test_autotuned_x_march_gives_the_same_steps():
    """`lx="auto"` times the stage kernel for each tile shape and x-march length and keeps
    the fastest. The x-march changes no arithmetic (bitwise the same steps); another tile
    shape is another instantiation of the kernel, whose compiled multiply-adds may round
    differently, so the steps agree to float32 rounding."""
    import torch

    from wellbalanced_b200.autotune import CANDIDATES
    from wellbalanced_b200.mhd3d import MHD3D

    tuned = MHD3D.turbulence(24, seed=2, precision=32, lx="auto")
    fixed = MHD3D.turbulence(24, seed=2, precision=32, lx=8)
    ty, tz = tuned.engine.layout.tile_shape
    assert tuned.lx in CANDIDATES and tuned.lx_timings
    assert f"{ty}x{tz}/{tuned.lx}" == min(tuned.lx_timings, key=tuned.lx_timings.get)
    for _ in range(3):
        fixed.step(tuned.step())
    torch.cuda.synchronize()
    if tuned.engine.layout.tile_shape == fixed.engine.layout.tile_shape:
        assert torch.equal(tuned.engine.state, fixed.engine.state)
    else:
        assert torch.allclose(tuned.engine.state, fixed.engine.state, rtol=1e-5, atol=1e-6)
    # same shape, another x-march: bitwise
    other = MHD3D.turbulence(24, seed=2, precision=32, lx=16)
    other.engine.layout.set_tile(tuned.engine.layout.tile_shape)
    from wellbalanced_b200.autotune import _set_lx

    _set_lx(other.engine, 16)
    again = MHD3D.turbulence(24, seed=2, precision=32, lx=8)
    again.engine.layout.set_tile(tuned.engine.layout.tile_shape)
    _set_lx(again.engine, 8)
    for _ in range(3):
        again.step(other.step())
    torch.cuda.synchronize()
    assert torch.equal(other.engine.state, again.engine.state)


def test_plain_3d_resistivity_and_gravity_match_the_reference(runs3d):
    """The per-kernel float64 3D path with resistivity (the reference's own run) and with
    gravity (against the oracle's 3D step, which restates carafe/mhd3d.py:635-671)."""
    from oracle.mesh import Hierarchy
    from oracle.mhd3d import MHD3D as OracleMHD3D
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.plain import PlainMHD3D

    k = 2.0 * np.pi
    model = PlainMHD3D(AMRHierarchy((4, 4, 16), ((0.0, 1.0),) * 3, periodic=(True,) * 3), resistivity=0.01)
    model.set_state(1.0, (0.0, 0.0, 0.0), 1.0,
                    vector_potential=(lambda x, y, z: np.cos(k * z) / k, lambda x, y, z: np.sin(k * z) / k, 0.0))
    for _ in range(5):
        model.step()
    close(model.state(), runs3d, "resistive3d", 1e-12)

    def state(m):
        m.set_state(lambda x, y, z: 1.0 + 0.3 * (z > 0.5), (0.0, 0.0, lambda x, y, z: 0.05 * np.sin(k * x)),
                    lambda x, y, z: 2.0 - 0.2 * z,
                    vector_potential=(0.0, lambda x, y, z: 0.05 * np.cos(k * x) / k, 0.0))
        return m

    options = dict(gravity=(0.0, 0.0, -0.2), resistivity=0.005, limiter="minmod", mean_field=(0.0, 0.0, 0.1))
    device = state(PlainMHD3D(AMRHierarchy((6, 6, 8), ((0.0, 1.0),) * 3, periodic=(True,) * 3), **options))
    oracle = state(OracleMHD3D(Hierarchy((6, 6, 8), ((0.0, 1.0),) * 3, (True,) * 3), **options))
    for _ in range(4):
        device.step(oracle.step())
    want = oracle.state()
    got = device.state()
    for key in want:
        np.testing.assert_allclose(got[key], want[key], rtol=1e-12, atol=1e-12, err_msg=key)


def test_fused_3d_resistivity_and_gravity_match_the_reference(runs3d):
    """The fused 3D stage kernel with resistivity (the reference's own resistive run) and
    with resistivity, gravity and a mean field (against the oracle's 3D step), in float64
    to 1e-12 and in float32 to float32 round-off."""
    from oracle.mesh import Hierarchy
    from oracle.mhd3d import MHD3D as OracleMHD3D
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd3d import MHD3D

    k = 2.0 * np.pi
    model = MHD3D(AMRHierarchy((4, 4, 16), ((0.0, 1.0),) * 3, periodic=(True,) * 3), resistivity=0.01,
                  precision=64)
    model.set_state(1.0, (0.0, 0.0, 0.0), 1.0,
                    vector_potential=(lambda x, y, z: np.cos(k * z) / k, lambda x, y, z: np.sin(k * z) / k, 0.0))
    for _ in range(5):
        model.step()
    close(model.state(), runs3d, "resistive3d", 1e-12)

    def state(m):
        m.set_state(lambda x, y, z: 1.0 + 0.3 * (z > 0.5), (0.0, 0.0, lambda x, y, z: 0.05 * np.sin(k * x)),
                    lambda x, y, z: 2.0 - 0.2 * z,
                    vector_potential=(lambda x, y, z: 0.03 * np.sin(k * y) / k,
                                      lambda x, y, z: 0.05 * np.cos(k * x) / k, 0.0))
        return m

    options = dict(gravity=(0.05, 0.0, -0.2), resistivity=0.005, limiter="minmod", mean_field=(0.0, 0.05, 0.1))
    shape = (20, 18, 24)  # several tiles along y and z, tiles of 16 planes along x
    oracle = state(OracleMHD3D(Hierarchy(shape, ((0.0, 1.0),) * 3, (True,) * 3), **options))
    fused64 = state(MHD3D(AMRHierarchy(shape, ((0.0, 1.0),) * 3, periodic=(True,) * 3), precision=64, lx=16,
                          **options))
    fused32 = state(MHD3D(AMRHierarchy(shape, ((0.0, 1.0),) * 3, periodic=(True,) * 3), precision=32, lx=16,
                          **options))
    for _ in range(4):
        dt = oracle.step()
        fused64.step(dt)
        fused32.step(dt)
    want = oracle.state()
    got64, got32 = fused64.state(), fused32.state()
    for key in want:
        np.testing.assert_allclose(got64[key], want[key], rtol=1e-12, atol=1e-12, err_msg=key)
        scale = float(np.max(np.abs(want[key])))
        assert float(np.max(np.abs(got32[key] - want[key]))) < 2e-5 * max(scale, 1.0), key
    assert fused64.divergence() < 1e-13


def test_every_2d_tile_shape_gives_the_same_steps():
    """The 2D stage kernel on each tile shape it is built for: a face's flux and a cell's
    update use the same arithmetic whichever tile holds them, so the steps are bitwise
    those of the default shape (patch sizes that are not multiples of the tiles)."""
    from wellbalanced_b200 import _lib
    from wellbalanced_b200.autotune import tune_tile2d
    from wellbalanced_b200.mhd import MHD2D

    for precision in (32, 64, "mixed"):
        reference = MHD2D.orszag_tang(40, precision=precision, limiter="mc")
        for _ in range(3):
            reference.step()
        want = reference.engine.state.clone()
        for tile in _lib.tile_shapes_2d(precision):
            model = MHD2D.orszag_tang(40, precision=precision, limiter="mc", tile=tile)
            assert model.engine.layout.tile_shape == tile
            for _ in range(3):
                model.step()
            assert torch.equal(model.engine.state, want), (precision, tile)
        tuned = MHD2D.orszag_tang(40, precision=precision, limiter="mc", tile="auto")
        assert tuned.tile in _lib.tile_shapes_2d(precision)
        for _ in range(3):
            tuned.step()
        assert torch.equal(tuned.engine.state, want)
        best, timings = tune_tile2d(tuned.engine, use_cache=False)
        assert set(timings) == {f"{tx}x{ty}" for tx, ty in _lib.tile_shapes_2d(precision)}
        assert all(v > 0 for v in timings.values())


def test_every_3d_tile_shape_gives_the_same_steps():
    """The 3D stage kernel on each tile shape it is built for (with the rim threads of the
    smaller tile) gives the steps of the default shape, float32 and float64, on a box whose
    sides are not multiples of the tiles: to rounding, since each shape is a separate
    instantiation whose compiled multiply-adds may round differently (a wrong index would
    show at O(1))."""
    from wellbalanced_b200 import _lib
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd3d import MHD3D

    k = 2.0 * np.pi

    def model(precision, tile=None, lx=8):
        m = MHD3D(AMRHierarchy((20, 18, 26), ((0.0, 1.0),) * 3, periodic=(True, True, False)), precision=precision,
                  limiter="mc", cfl=0.3, lx=lx)
        if tile is not None:
            from wellbalanced_b200.autotune import _set_lx

            m.engine.layout.set_tile(tile)
            _set_lx(m.engine, lx)
        m.set_state(lambda x, y, z: 1.0 + 0.2 * np.sin(k * (x + y)),
                    (lambda x, y, z: 0.5 * np.sin(k * y), lambda x, y, z: 0.5 * np.sin(k * z),
                     lambda x, y, z: 0.5 * np.sin(k * x)),
                    1.0,
                    vector_potential=(lambda x, y, z: 0.1 * np.cos(k * z), lambda x, y, z: 0.1 * np.cos(k * x),
                                      lambda x, y, z: 0.1 * np.cos(k * y)))
        return m

    for precision in (32, 64, "mixed"):
        reference = model(precision)
        for _ in range(3):
            reference.step()
        for tile in _lib.tile_shapes(3, _lib.precision_code(precision)):
            m = model(precision, tile)
            assert m.engine.layout.tile_shape == tile
            for _ in range(3):
                m.step()
            tol = 1e-12 if precision == 64 else 1e-5
            assert torch.allclose(m.engine.state, reference.engine.state, rtol=tol, atol=tol * 0.1), (precision, tile)


def test_saved_state_resumes_bitwise():
    """`save` / `load` of the device pool: steps after a reload repeat the steps after the
    save, bit for bit (2D float32, 3D float64)."""
    from wellbalanced_b200.mhd import MHD2D
    from wellbalanced_b200.mhd3d import MHD3D

    for model in (MHD2D.orszag_tang(32, precision=32, limiter="mc"),
                  MHD3D.orszag_tang(16, precision=64, limiter="mc")):
        for _ in range(3):
            model.step()
        saved, time, steps = model.save(), model.time, model.steps
        dts = [model.step() for _ in range(4)]
        after = model.engine.state.clone()
        model.load(saved)
        model.time, model.steps = time, steps
        model.engine.time.fill_(time)
        again = [model.step() for _ in range(4)]
        assert again == dts
        assert torch.equal(model.engine.state, after)


@pytest.mark.parametrize("precision", [64, 32, "mixed"])
def test_alfven_wave_converges_at_second_order(precision):
    """The reference's convergence tests (tests/unit/test_mhd.py:78-86,
    tests/unit/test_mhd3d.py:13-21): the circularly polarised Alfven wave after one period
    at 8 and 16 cells, unlimited slopes; the error of B_y falls by 2^1.85 (2D) / 2^1.8
    (3D), div B stays at round-off (the curl of the stored potential, taken in float64:
    1e-14 as the reference's bound for a float64 potential, 1e-12 for a float32 one)."""
    from wellbalanced_b200.mhd import MHD2D
    from wellbalanced_b200.mhd3d import MHD3D

    for cls, order in ((MHD2D, 1.85), (MHD3D, 1.8)):
        errors = []
        for cells in (8, 16):
            model, exact = cls.alfven_wave(cells, limiter="none", precision=precision)
            model.run(model.period)
            by = model.dataset()["magnetic_field_y"].values
            errors.append(float(np.mean(np.abs(by - exact["magnetic_field_y"].values))))
            assert model.divergence() < (1e-12 if precision == 32 else 1e-14), cls.__name__
        assert np.log2(errors[0] / errors[1]) > order, (cls.__name__, errors)


def test_config1_orszag_tang_256_to_half_time_against_the_reference_run():
    """Config 1 at its full size and horizon (256^2, MC, CFL 0.4, t = 0.5: 1441 steps)
    against the reference's own run of it (committed fixture).

    * float64: equal to rounding (1e-12).
    * "mixed" (float32 reconstruction, HLLD and CT; float64 state, pressure recovery and
      updates): relative L1 of density and energy within 1e-5.
    * float32 state: the rounding of the stored state to float32 after every stage is by
      itself 1.06e-5 (density) / 1.28e-5 (energy) at this horizon (the reference's float64
      arithmetic with the state rounded to float32 after each stage, a NumPy restatement of
      this run), so a float32 state cannot meet 1e-5 over the whole horizon. It is held to
      3e-5 here as a regression guard (measured on B200: 1.93e-5 / 2.60e-5 with the float32
      faces on explicit-FMA lane arithmetic; 1.66e-5 / 2.16e-5 with compiler-contracted
      scalar arithmetic: the chaotic flow amplifies a different rounding into a different
      realisation of the same size); the float64 state of "mixed" is what meets the bound
      (measured 1.8e-6 / 2.7e-6)."""
    from wellbalanced_b200.mhd import MHD2D

    golden = np.load(GOLDEN / "ot256_full.npz")
    for precision, bound in ((64, 1e-12), ("mixed", 1e-5), (32, 3e-5)):
        model = MHD2D.orszag_tang(256, limiter="mc", cfl=0.4, precision=precision)
        model.run(float(golden["time"]))
        assert model.steps == int(golden["steps"])
        state = model.state()
        err_rho = rel_l1(state["density"], golden["density"])
        err_e = rel_l1(state["energy"], golden["energy"])
        print(f"config 1, precision {precision}: rel L1 rho {err_rho:.3e}, E {err_e:.3e}")
        assert err_rho < bound and err_e < bound, (precision, err_rho, err_e)
        assert model.divergence() < (1e-12 if precision == 32 else 1e-14)


def test_mixed_precision_3d_turbulence_error_div_b_and_totals(runs3d):
    """float32 arithmetic on a float64 state, 3D: the reference's float64 turbulence run to
    1e-5 (relative L1), div B at the float64 round-off of the stored potential, and the
    conserved totals kept to float64 round-off (the state is the accumulator)."""
    model = _turbulence("mixed")
    before = model.totals()
    for dt in runs3d["turb16_dts"]:
        model.step(float(dt))
    state = model.state()
    err_rho = rel_l1(state["density"], runs3d["turb16_density"])
    err_e = rel_l1(state["energy"], runs3d["turb16_energy"])
    print(f"mixed turbulence 16^3, 4 steps: rel L1 rho {err_rho:.3e}, E {err_e:.3e}")
    assert err_rho < 1e-5 and err_e < 1e-5
    assert model.divergence() < 1e-14
    after = model.totals()
    for key in before:
        assert abs(after[key] - before[key]) < 1e-13 * max(1.0, abs(before[key])), key


def test_mixed_precision_refined_2d_keeps_totals_and_composite_div_b():
    """float32 arithmetic on a float64 state on a refined hierarchy: the flux register
    recomputes the interface fluxes with the stage kernel's float32 arithmetic, so the
    composite totals stay at float64 round-off, as in float64 (tests/unit/test_mhd.py:164-211
    of the reference)."""
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    mesh = AMRHierarchy((32, 16), ((-1.0, 1.0), (-0.5, 0.5)), periodic=(True, True))
    mesh.add_patch(1, ((16, 48), (8, 24)))
    model = MHD2D(mesh, limiter="mc", precision="mixed", mean_field=(0.1, 0.05))
    model.set_state(lambda x, y: 1.0 + 0.5 * np.exp(-((x + 0.3) ** 2 + y**2) / 0.02), (2.0, 1.0, 0.3),
                    lambda x, y: 1.0 + 0.2 * np.cos(np.pi * x),
                    vector_potential=lambda x, y: 0.1 * np.maximum(0.3 - np.hypot(x, y), 0.0),
                    bz=lambda x, y: 0.1 * np.sin(np.pi * x))
    before = model.totals()
    for _ in range(10):
        model.step()
    after = model.totals()
    for key in before:
        assert abs(after[key] - before[key]) < 1e-13 * max(1.0, abs(before[key])), key
    assert model.divergence() < 1e-14
    assert model.composite_divergence() < 1e-14
