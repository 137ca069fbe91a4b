"""The reference's refined-mesh and resistive tests on the device (float64).

Restated from ``tests/unit/test_mhd_amr.py`` and ``tests/unit/test_mhd3d.py`` of the
reference (the problems, the exact solutions and the bounds are theirs): the Alfven wave
at second order across a refined patch, resistive decay at the diffusion rate on one and
two levels and at second order across a coarse-fine edge, the diffusion limit of the
step, a force-free 3D field decaying at the discrete diffusion rate, and a reconnecting
Harris pair on regridded patches following the uniform mesh.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

AMPLITUDE = 0.1
K = 2.0 * np.pi


def _alfven_along_x(n, levels):
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    mesh = AMRHierarchy((n, 4), ((0.0, 1.0), (0.0, 4.0 / n)), periodic=(True, True))
    for level in range(1, levels + 1):
        r = 2**level
        mesh.add_patch(level, ((n * r // 4, 3 * n * r // 4), (0, 4 * r)))
    model = MHD2D(mesh, mean_field=(1.0, 0.0), limiter="none", precision=64)
    model.set_state(1.0, (0.0, lambda x, y: -AMPLITUDE * np.sin(K * x), lambda x, y: -AMPLITUDE * np.cos(K * x)),
                    0.1, vector_potential=lambda x, y: AMPLITUDE * np.cos(K * x) / K,
                    bz=lambda x, y: AMPLITUDE * np.cos(K * x))
    return model


def _alfven_error(n, levels):
    model = _alfven_along_x(n, levels)
    model.run(0.5)
    leaf = model.leaf_values()
    exact = AMPLITUDE * np.sin(K * (leaf["x"] - 0.5))
    return float(np.mean(np.abs(leaf["magnetic_field_y"] - exact)))


def test_the_alfven_wave_converges_at_second_order_across_a_refined_patch():
    errors = np.array([_alfven_error(n, 1) for n in (16, 32)])
    assert np.log2(errors[0] / errors[1]) > 1.85, errors
    assert errors[1] < _alfven_error(32, 0)  # the patch makes the wave more accurate


@pytest.mark.parametrize("levels", [0, 1])
def test_resistivity_damps_the_field_at_the_diffusion_rate(levels):
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    n, eta, amp = 16, 0.02, 1e-3
    mesh = AMRHierarchy((n, n), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, True))
    if levels:
        mesh.add_patch(1, ((n // 2, 3 * n // 2), (n // 2, 3 * n // 2)))
    model = MHD2D(mesh, resistivity=eta, limiter="none", precision=64)
    model.set_state(1.0, (0.0, 0.0, 0.0), 1.0, vector_potential=lambda x, y: amp * np.cos(K * x) / K,
                    bz=lambda x, y: amp * np.cos(K * y))
    start = model.totals()
    model.run(0.25)
    leaf = model.leaf_values()
    decay = np.exp(-eta * K * K * model.time)
    by = np.mean(np.abs(leaf["magnetic_field_y"] - amp * np.sin(K * leaf["x"]) * decay))
    bz = np.mean(np.abs(leaf["magnetic_field_z"] - amp * np.cos(K * leaf["y"]) * decay))
    assert by < (3.6e-3 if levels else 3e-3) * amp * decay, by / (amp * decay)
    assert bz < 4e-3 * amp * decay, bz / (amp * decay)
    assert abs(model.totals()["energy"] - start["energy"]) < 1e-12  # Ohmic heating stays in the energy


def test_the_step_keeps_within_the_diffusion_limit():
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    model = MHD2D(AMRHierarchy((16, 16), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, True)), resistivity=1.0,
                  precision=64)
    model.set_state(1.0, (0.0, 0.0, 0.0), 1e-3)
    dx = 1.0 / 16
    assert model.stable_step() == pytest.approx(model.cfl * 0.5 / (2.0 / dx**2))


def _refined_decay_error(n):
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    eta, amp = 0.02, 1e-3
    mesh = AMRHierarchy((n, n), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, True))
    mesh.add_patch(1, ((n // 2, 3 * n // 2), (n // 2, 3 * n // 2)))
    model = MHD2D(mesh, resistivity=eta, limiter="none", precision=64)
    model.set_state(1.0, (0.0, 0.0, 0.0), 1.0, vector_potential=lambda x, y: amp * np.cos(K * x) / K)
    model.run(0.25)
    leaf = model.leaf_values()
    decay = np.exp(-eta * K * K * model.time)
    exact = amp * np.sin(K * leaf["x"]) * decay
    return float(np.mean(np.abs(leaf["magnetic_field_y"] - exact)) / (amp * decay))


def test_resistive_decay_converges_at_second_order_across_a_coarse_fine_edge():
    coarse, fine = _refined_decay_error(16), _refined_decay_error(32)
    assert np.log2(coarse / fine) > 1.8, (coarse, fine)


def test_resistivity_damps_a_force_free_field_at_the_diffusion_rate():
    """The fused 3D kernel's resistive terms: a Beltrami field decays as exp(-2 eta k^2 t)
    in magnetic pressure, with the discrete wavenumber of the second difference."""
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd3d import MHD3D

    eta, k = 0.01, 2.0 * np.pi
    model = MHD3D(AMRHierarchy((4, 4, 16), ((0.0, 1.0),) * 3, periodic=(True,) * 3), resistivity=eta, precision=64)
    model.set_state(1.0, (0.0, 0.0, 0.0), 1.0,
                    vector_potential=(lambda x, y, z: np.cos(k * z) / k, lambda x, y, z: np.sin(k * z) / k, 0.0))
    before = model.dataset()["magnetic_pressure"].values.mean()
    duration = 0.5
    model.run(duration)
    after = model.dataset()
    ratio = after["magnetic_pressure"].values.mean() / before
    h = 1.0 / 16
    k_discrete = 2.0 * np.sin(k * h / 2) / h
    assert ratio == pytest.approx(np.exp(-2 * eta * k_discrete**2 * duration), rel=2e-3)
    assert np.abs(after["velocity_x"].values).max() < 1e-12


def test_reconnection_on_patches_follows_the_uniform_mesh():
    """Resistive reconnection of a Harris pair on patches regridded every 5 steps on the
    current: the flux psi of the sheet moves as on a uniform mesh of the finest spacing."""
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D, harris_sheets, sheet_diagnostics

    def run(shape, levels):
        mesh = AMRHierarchy(shape, ((0, 4), (0, 2)), periodic=(True, True))
        state = harris_sheets(mesh, width=0.1, perturbation=0.05)
        model = MHD2D(mesh, resistivity=4e-3, precision=64)
        model.set_state(**state)
        for _ in range(levels):
            model.regrid(model.current_tags(0.5, levels=levels), buffer=1)
            model.set_state(**state)
        first = sheet_diagnostics(model)
        while model.time < 0.2:
            if levels and model.steps % 5 == 0:
                model.regrid(model.current_tags(0.5, levels=levels), buffer=1)
            model.step(min(model.stable_step(), 0.2 - model.time))
        return first, sheet_diagnostics(model), model

    first, refined, model = run((32, 16), 1)
    start, uniform, _ = run((64, 32), 0)
    assert model.hierarchy.max_level == 1
    assert refined["leaf_cells"] < 0.75 * uniform["leaf_cells"]
    assert (first["o_points"], first["x_points"]) == (1, 1)
    assert abs(first["psi"] - start["psi"]) < 1e-3 * start["psi"]
    change = abs(uniform["psi"] - start["psi"])
    assert change > 1e-2 * start["psi"]
    assert abs(refined["psi"] - uniform["psi"]) < 0.05 * change, (refined["psi"], uniform["psi"], change)
