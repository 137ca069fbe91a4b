"""The oracle against golden vectors generated by the reference itself (CPU).

``tests/golden/make_golden.py`` ran the reference's own ``carafe`` kernels and solvers
(NumPy and Pyccel-as-Python kernels) and stored their outputs; the oracle restatement
must reproduce them to rounding. These pins are what makes the oracle a valid checker
for the CUDA path.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import kernels as K
from oracle.mesh import Hierarchy
from oracle.mhd2d import MHD2D
from oracle.mhd3d import MHD3D

GOLDEN = Path(__file__).with_name("golden")
GAMMA = 5.0 / 3.0
SHAPE = (13, 9)


@pytest.fixture(scope="module")
def kernels():
    return np.load(GOLDEN / "kernels.npz")


@pytest.fixture(scope="module")
def runs2d():
    return np.load(GOLDEN / "runs2d.npz")


@pytest.fixture(scope="module")
def runs3d():
    return np.load(GOLDEN / "runs3d.npz")


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("axis", [0, 1])
@pytest.mark.parametrize("limiter", range(4))
def test_sweep_matches_the_reference(kernels, seed, axis, limiter):
    prim = kernels[f"block{seed}_prim"]
    bn = kernels[f"block{seed}_{'bxf' if axis == 0 else 'byf'}"]
    nx, ny = SHAPE
    flux = np.empty((7, nx - 3, ny) if axis == 0 else (7, nx, ny - 3))
    K.mhd_sweep(prim, bn, axis, limiter, GAMMA, flux)
    for impl in ("numpy", "pyccel"):
        np.testing.assert_allclose(flux, kernels[f"block{seed}_sweep_a{axis}_l{limiter}_{impl}"], rtol=1e-13, atol=1e-13)


def test_hlld_matches_the_reference(kernels):
    flux = K.hlld(kernels["hlld_left"], kernels["hlld_right"], kernels["hlld_bn"], GAMMA)
    np.testing.assert_allclose(flux, kernels["hlld_flux"], rtol=1e-13, atol=1e-13)


def test_ct_primitive_rate_resistive_conductive_match_the_reference(kernels):
    nx, ny = SHAPE
    fx, fy, ecc = kernels["ct_fx"], kernels["ct_fy"], kernels["ct_ecc"]
    ez = np.empty((nx - 3, ny - 3))
    K.ct_contact(fx[5], fy[5], fx[0], fy[0], ecc, ez)
    np.testing.assert_allclose(ez, kernels["ct_ez_pyccel"], rtol=0, atol=1e-14)
    fields = [kernels[f"cons_{k}"] for k in range(6)]
    az = kernels["cons_az"]
    prim = np.empty((8, nx, ny))
    bxf, byf, ecc = np.empty((nx + 1, ny)), np.empty((nx, ny + 1)), np.empty(SHAPE)
    bad = K.mhd_primitive(*fields, az, 0.1, 0.2, 0.3, -0.4, GAMMA, prim, bxf, byf, ecc)
    assert bad == int(kernels["primitive_bad_pyccel"]) == 0
    np.testing.assert_allclose(prim, kernels["primitive_prim_pyccel"], rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(ecc, kernels["primitive_ecc_pyccel"], rtol=1e-14, atol=1e-14)
    out = np.empty(2)
    K.mhd_rate(*fields, az, 2, 0.1, 0.2, 0.3, -0.4, GAMMA, out)
    np.testing.assert_allclose(out, kernels["rate_pyccel"], rtol=1e-14)
    cases = [(0, -1.0), (4, -1.0e3), (1, np.inf), (2, np.nan), (5, -np.inf), (0, np.nan)]
    for (row, value), expected in zip(cases, kernels["bad_counts"], strict=True):
        f2 = [f.copy() for f in fields]
        f2[row][3, 4] = value
        f2[row][7, 1] = value
        count = K.mhd_primitive(*f2, az, 0.1, 0.2, 0.3, -0.4, GAMMA, np.empty((8, nx, ny)),
                                np.empty((nx + 1, ny)), np.empty((nx, ny + 1)), np.empty(SHAPE))
        assert count == expected == 2
    prim1, bxf1, byf1 = kernels["block1_prim"], kernels["block1_bxf"], kernels["block1_byf"]
    fx, fy, ez = kernels["res_fx0"].copy(), kernels["res_fy0"].copy(), kernels["res_ez0"].copy()
    K.mhd_resistive(prim1, bxf1, byf1, 0.1, 0.2, 0.05, fx, fy, ez)
    np.testing.assert_allclose(fx, kernels["res_fx_pyccel"], rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(fy, kernels["res_fy_pyccel"], rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(ez, kernels["res_ez_pyccel"], rtol=1e-13, atol=1e-13)
    fx, fy = kernels["cond_fx0"].copy(), kernels["cond_fy0"].copy()
    K.mhd_conductive(kernels["cond_prim"], kernels["cond_bxf"], kernels["cond_byf"], 0.1, 0.2, 0.3, 0.01, fx, fy)
    np.testing.assert_allclose(fx, kernels["cond_fx_pyccel"], rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(fy, kernels["cond_fy_pyccel"], rtol=1e-13, atol=1e-13)


def _close2(model, runs, prefix, tol=1e-12):
    state = model.state()
    for key, value in state.items():
        np.testing.assert_allclose(value, runs[f"{prefix}_{key}"], rtol=tol, atol=tol, err_msg=f"{prefix} {key}")


def test_orszag_tang_steps_match_the_reference(runs2d):
    model = MHD2D.orszag_tang(32)
    dts = [model.step() for _ in range(5)]
    np.testing.assert_allclose(dts, runs2d["ot32_5_dts"], rtol=1e-14)
    _close2(model, runs2d, "ot32_5")


@pytest.mark.parametrize("limiter", ["minmod", "vanleer", "mc", "none"])
def test_limiters_match_the_reference(runs2d, limiter):
    model = MHD2D.orszag_tang(24, limiter=limiter)
    for _ in range(8):
        model.step()
    _close2(model, runs2d, f"ot24_{limiter}")


def test_outflow_walls_gravity_resistive_match_the_reference(runs2d):
    model = MHD2D.rotor(32)
    model.run(0.02)
    _close2(model, runs2d, "rotor32", 1e-11)
    model = MHD2D.rayleigh_taylor(8, field=0.05)
    for _ in range(20):
        model.step()
    _close2(model, runs2d, "rt8")
    model = MHD2D.orszag_tang(16, resistivity=1e-3, conduction=(1e-2, 1e-3))
    for _ in range(3):
        model.step()
    _close2(model, runs2d, "ot16_resistive")


def test_multi_patch_level_matches_the_reference():
    golden = np.load(GOLDEN / "multipatch.npz")
    model = MHD2D.orszag_tang(32, split=(2, 3))
    for _ in range(5):
        model.step()
    np.testing.assert_allclose(model.state()["density"], golden["split_density"], rtol=1e-13, atol=1e-13)


def _close3(model, runs, prefix, tol=1e-12):
    state = model.state()
    for key, value in state.items():
        np.testing.assert_allclose(value, runs[f"{prefix}_{key}"], rtol=tol, atol=tol, err_msg=f"{prefix} {key}")


def test_3d_runs_match_the_reference(runs3d):
    flat = MHD3D.orszag_tang(16, layers=2)
    for dt in runs3d["ot3d16_dts"]:
        flat.step(dt)
    _close3(flat, runs3d, "ot3d16")
    model = MHD3D.blast_wave(12)
    model.run(0.01)
    _close3(model, runs3d, "blast3d12", 1e-11)


def test_3d_turbulence_matches_the_reference(runs3d):
    from wellbalanced_b200.problems import turbulence_3d

    rho, velocity, p, potential = turbulence_3d(16, seed=7)
    model = MHD3D(Hierarchy((16,) * 3, ((0.0, 1.0),) * 3, (True,) * 3), limiter="mc", cfl=0.3)
    model.set_state(rho, velocity, p, vector_potential=potential)
    _close3(model, runs3d, "turb16_init", 1e-14)
    dts = [model.step() for _ in range(4)]
    np.testing.assert_allclose(dts, runs3d["turb16_dts"], rtol=1e-13)
    _close3(model, runs3d, "turb16", 1e-12)


def test_oracle_refined_non_ideal_runs_conserve():
    """The oracle's flux register on refined hierarchies with the non-ideal terms (the
    reference records its fluxes after adding them): resistive + conductive 2D and
    resistive 3D runs keep their composite totals to round-off (the checker the device's
    refined non-ideal tests compare with)."""
    from oracle.mesh import Hierarchy
    from oracle.mhd2d import MHD2D as OracleMHD2D
    from oracle.mhd3d import MHD3D as OracleMHD3D

    h = Hierarchy((16, 8), ((-1.0, 1.0), (-0.5, 0.5)), (True, True))
    h.add_patch(1, ((8, 24), (4, 12)))
    model = OracleMHD2D(h, limiter="minmod", resistivity=2e-3, conduction=(2e-2, 1e-3), mean_field=(0.1, 0.05))
    model.set_state(lambda x, y: 1.0 + 0.5 * np.exp(-((x + 0.3) ** 2 + y**2) / 0.02), (2.0, 1.0, 0.3),
                    lambda x, y: 1.0 + 0.2 * np.cos(np.pi * x),
                    vector_potential=lambda x, y: 0.1 * np.maximum(0.3 - np.hypot(x, y), 0.0),
                    bz=lambda x, y: 0.1 * np.sin(np.pi * x))
    before = model.totals()
    for _ in range(5):
        model.step()
    after = model.totals()
    for name in before:
        assert abs(after[name] - before[name]) < 1e-13 * max(1.0, abs(before[name])), name

    k = 2.0 * np.pi
    h3 = Hierarchy((8, 8, 8), ((0.0, 1.0),) * 3, (True,) * 3)
    h3.add_patch(1, ((4, 12), (4, 12), (2, 10)))
    model = OracleMHD3D(h3, resistivity=0.01, limiter="minmod")
    model.set_state(lambda x, y, z: 1.0 + 0.2 * np.sin(k * (x + y)),
                    (lambda x, y, z: 0.3 * np.sin(k * y), 0.0, lambda x, y, z: 0.3 * np.sin(k * x)), 1.0,
                    vector_potential=(lambda x, y, z: 0.1 * np.cos(k * z), lambda x, y, z: 0.1 * np.cos(k * x),
                                      lambda x, y, z: 0.1 * np.cos(k * y)))
    before = model.totals()
    for _ in range(3):
        model.step()
    after = model.totals()
    for name in before:
        assert abs(after[name] - before[name]) < 1e-13 * max(1.0, abs(before[name])), name
