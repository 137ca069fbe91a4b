"""Host logic of the leaf-cell diagnostics (CPU): `sheet_diagnostics` on given leaf values.

`sheet_diagnostics` (the reference's ``carafe/mhd.py:1291-1329``) samples B_y on the line
y = Ly / 4 through the leaf cells, at the finest spacing, and counts the sign changes
along x. Here the leaf values are made on the host for a uniform level and for a level
with a refined patch over part of the line, from B_y = A sin(2 pi m x / Lx): psi is
(1/2) int |B_y| dx, and there are m O-points and m X-points.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from wellbalanced_b200.mesh import AMRHierarchy
from wellbalanced_b200.mhd import covered_cells, sheet_diagnostics


def _leaf(hierarchy, by):
    parts = {name: [] for name in ("x", "y", "level", "density", "magnetic_field_y", "current_z")}
    for patch in hierarchy.patches:
        leaf = ~covered_cells(hierarchy, patch)
        dx = hierarchy.spacing(patch.level)
        axes = [hierarchy.lower_bound[a] + (np.arange(*patch.box[a]) + 0.5) * dx[a] for a in range(2)]
        x, y = np.meshgrid(*axes, indexing="ij")
        parts["x"].append(x[leaf])
        parts["y"].append(y[leaf])
        parts["level"].append(np.full(int(leaf.sum()), patch.level))
        parts["density"].append(np.ones(int(leaf.sum())))
        parts["magnetic_field_y"].append(by(x[leaf], y[leaf]))
        parts["current_z"].append(np.full(int(leaf.sum()), float(patch.level + 1)))
    return {k: np.concatenate(v) for k, v in parts.items()}


def _check(hierarchy, modes, amplitude=0.3):
    lx = hierarchy.bounds[0][1] - hierarchy.bounds[0][0]

    def by(x, y):
        return amplitude * np.sin(2 * np.pi * modes * (x - hierarchy.bounds[0][0]) / lx)

    leaf = _leaf(hierarchy, by)
    model = SimpleNamespace(hierarchy=hierarchy, time=0.25)
    out = sheet_diagnostics(model, leaf)
    assert out["o_points"] == modes and out["x_points"] == modes
    assert out["leaf_cells"] == leaf["density"].size
    assert out["max_current"] == float(hierarchy.max_level + 1)
    assert out["time"] == 0.25
    # the finest-spacing midpoint sum of |B_y| against the integral (2 / pi) A Lx / 2
    assert abs(out["psi"] - amplitude * lx / np.pi) < 0.02 * amplitude * lx
    return out


def test_sheet_diagnostics_on_a_uniform_level():
    h = AMRHierarchy((64, 128), ((-1.0, 1.0), (-2.0, 2.0)), periodic=(True, False))
    _check(h, 3)


def test_sheet_diagnostics_through_a_refined_patch():
    h = AMRHierarchy((64, 128), ((-1.0, 1.0), (-2.0, 2.0)), periodic=(True, False))
    # the line y = -1 lies at level-0 row 32, level-1 rows 63 | 64
    h.add_patch(1, ((20, 80), (56, 72)))
    out = _check(h, 4)
    uniform = _check(AMRHierarchy((64, 128), ((-1.0, 1.0), (-2.0, 2.0)), periodic=(True, False)), 4)
    assert out["leaf_cells"] == uniform["leaf_cells"] - 30 * 8 + 60 * 16


def test_dataset_variables_combine_element_wise():
    """`dataset()` variables combine like xarray's aligned variables (``ds.pressure /
    ds.density`` is the temperature)."""
    from wellbalanced_b200.dataset import Dataset, Variable

    p = Variable(("x", "y"), np.array([[2.0, 4.0], [6.0, 8.0]]))
    rho = Variable(("x", "y"), np.array([[1.0, 2.0], [3.0, 4.0]]))
    ds = Dataset({"pressure": p, "density": rho})
    t = ds.pressure / ds.density
    assert isinstance(t, Variable) and t.dims == ("x", "y")
    np.testing.assert_array_equal(t.values, 2.0)
    np.testing.assert_array_equal((1.0 - t).values, -1.0)
    np.testing.assert_array_equal((0.5 * p + rho).values, 2 * rho.values)
    np.testing.assert_array_equal(abs(-rho).values, rho.values)
    assert float((p - rho).max()) == 4.0
