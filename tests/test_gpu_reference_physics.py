"""The reference's property tests of conduction, gravity, walls and the resistive energy
flux, on the fused device path (float64).

Restated from ``tests/unit/test_mhd.py:279-362`` and ``tests/unit/test_mhd3d.py:135-141,
192-240`` of the reference (problems, exact solutions and bounds are theirs): a hot spot
diffusing along an aligned field as in 1D, along an oblique field without overshoot,
isotropically without a field; free fall gaining rho g t of momentum (2D and 3D); walls
keeping mass, energy and B_n = 0; the Rayleigh-Taylor layer growing unless a strong
field holds it; and in 3D the energy change of a sheared field at rest being the
divergence of eta J x B along each axis.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

BOX = ((0.0, 1.0), (0.0, 1.0), (0.0, 1.0))


def _hot_spot(field, conduction, cells=64, t=2e-3):
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    hierarchy = AMRHierarchy((cells, cells), ((-1.0, 1.0), (-1.0, 1.0)), periodic=(True, True))
    model = MHD2D(hierarchy, mean_field=field, conduction=conduction, limiter="mc", precision=64)
    model.set_state(1.0, (0.0, 0.0, 0.0), lambda x, y: 1.0 + 0.01 * np.exp(-(x**2 + y**2) / 0.02))
    before = model.totals()["energy"]
    model.run(t)
    data = model.dataset()
    return model, data, (data.pressure / data.density).values, before


def test_conduction_along_an_aligned_field_is_one_dimensional_diffusion():
    kappa, t = 10.0, 2e-3
    model, data, temperature, before = _hot_spot((1.0, 0.0), (kappa, 0.0), t=t)
    chi = (5.0 / 3.0 - 1.0) * kappa
    s2 = 0.01 + 2.0 * chi * t
    x, y = data.x.values[:, None], data.y.values[None, :]
    exact = 1.0 + 0.01 * np.sqrt(0.01 / s2) * np.exp(-(x**2) / (2 * s2) - y**2 / 0.02)
    assert np.abs(temperature - exact).max() < 2e-5
    assert abs(model.totals()["energy"] - before) < 1e-13


def test_oblique_conduction_stays_on_the_field_lines_without_overshoot():
    field = (1.0 / np.sqrt(2.0), 1.0 / np.sqrt(2.0))
    _, _, temperature, _ = _hot_spot(field, (10.0, 0.0))
    assert temperature.min() > 1.0 - 1e-14
    np.testing.assert_allclose(temperature, temperature.T, atol=1e-15)
    along, across = temperature[40, 40] - 1.0, temperature[40, 24] - 1.0
    assert along > 100.0 * across


def test_isotropic_conduction_without_a_field():
    kappa, t = 10.0, 2e-3
    _, data, temperature, _ = _hot_spot((0.0, 0.0), (0.0, kappa), t=t)
    s2 = 0.01 + 2.0 * (2.0 / 3.0) * kappa * t
    x, y = data.x.values[:, None], data.y.values[None, :]
    exact = 1.0 + 0.01 * (0.01 / s2) * np.exp(-(x**2 + y**2) / (2 * s2))
    assert np.abs(temperature - exact).max() < 3e-5


def test_free_fall_gains_the_momentum_of_gravity():
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D
    from wellbalanced_b200.mhd3d import MHD3D

    model = MHD2D(AMRHierarchy((8, 8), periodic=(True, True)), gravity=(0.2, -0.5), precision=64)
    model.set_state(2.0, (0.0, 0.0, 0.0), 1.0)
    model.run(0.3)
    totals = model.totals()
    assert totals["momentum_x"] == pytest.approx(2.0 * 0.2 * 0.3, rel=1e-12)
    assert totals["momentum_y"] == pytest.approx(-2.0 * 0.5 * 0.3, rel=1e-12)
    model = MHD3D(AMRHierarchy((4, 4, 4), BOX, periodic=(True,) * 3), gravity=(0.0, 0.0, -2.0), precision=64)
    model.set_state(1.5, (0.0, 0.0, 0.0), 1.0)
    model.run(0.1)
    np.testing.assert_allclose(model.dataset()["velocity_z"].values, -0.2, atol=1e-13)


def test_walls_conserve_mass_and_energy_and_keep_the_normal_field_zero():
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd import MHD2D

    hierarchy = AMRHierarchy((24, 24))
    model = MHD2D(hierarchy, boundaries={"x": "wall", "y": "wall"}, precision=64)
    model.set_state(1.0, (0.3, -0.2, 0.1),
                    lambda x, y: 1.0 + 2.0 * np.exp(-((x - 0.3) ** 2 + (y - 0.6) ** 2) / 0.005),
                    vector_potential=lambda x, y: 0.1 * np.sin(np.pi * x) * np.sin(np.pi * y), bz=0.2)
    before = model.totals()
    model.run(0.3)
    after = model.totals()
    for name in ("density", "energy", "momentum_z", "bz"):
        assert abs(after[name] - before[name]) < 1e-13, name
    az = model.gather(hierarchy.patches[0], 6, node=True)
    for edge in (az[0], az[-1], az[:, 0], az[:, -1]):
        assert np.abs(edge).max() < 1e-15


def test_rayleigh_taylor_grows_and_a_strong_field_holds_it():
    from wellbalanced_b200.mhd import MHD2D

    free = MHD2D.rayleigh_taylor(16, precision=64)
    free.run(4.0)
    held = MHD2D.rayleigh_taylor(16, field=0.3, precision=64)
    held.run(4.0)
    growing = float(np.abs(free.dataset().velocity_y).max())
    stable = float(np.abs(held.dataset().velocity_y).max())
    assert growing > 0.015 and stable < 0.006, (growing, stable)
    assert free.divergence() < 1e-14


def _sheared(axis, eta):
    from wellbalanced_b200.mesh import AMRHierarchy
    from wellbalanced_b200.mhd3d import MHD3D

    shape = [4, 4, 4]
    across = (axis + 1) % 3
    shape[across] = 32
    k = 2.0 * np.pi
    model = MHD3D(AMRHierarchy(tuple(shape), BOX, periodic=(True,) * 3), resistivity=eta, precision=64)
    potential = [0.0, 0.0, 0.0]
    potential[(axis + 2) % 3] = lambda x, y, z: -np.cos(k * (x, y, z)[across]) / k
    model.set_state(1.0, (0.0, 0.0, 0.0), lambda x, y, z: 10.0 - 0.5 * np.sin(k * (x, y, z)[across]) ** 2,
                    vector_potential=tuple(potential))
    return model


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_the_resistive_energy_flux_is_eta_j_cross_b(axis):
    """With B_axis = sin(k s) at rest the energy changes by -div(eta J x B) =
    eta k^2 cos(2 k s): the run with resistivity minus the run without."""
    eta, duration = 1e-3, 0.002
    across = (axis + 1) % 3
    energies = []
    for resistivity in (eta, 0.0):
        model = _sheared(axis, resistivity)
        (patch,) = model.hierarchy.patches
        start = model.gather(patch, 4)
        model.run(duration, max_steps=100)
        energies.append(model.gather(patch, 4) - start)
    k = 2.0 * np.pi
    s = (np.arange(32) + 0.5) / 32
    expected = eta * k**2 * np.cos(2.0 * k * s)
    rate = (energies[0] - energies[1]) / duration
    rate = rate.mean(axis=tuple(a for a in range(3) if a != across))
    np.testing.assert_allclose(rate, expected, rtol=0.0, atol=0.03 * eta * k**2)
