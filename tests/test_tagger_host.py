"""The learned tagger's oracle on the CPU: bfloat16 rounding, gradients, stencil features.

`oracle/mlp.py` is the checker of the tagger's CUDA kernels; here it is itself checked:
its bfloat16 rounding against known values, its analytic gradient against central finite
differences of its loss (the smooth model without rounding), and its stencil features
against a direct evaluation on a small patch.
"""

from __future__ import annotations

import numpy as np

from oracle import mlp


def test_bfloat16_rounds_to_nearest_even():
    values = np.array([1.0, 1.0 + 2.0**-8, 1.0 + 3 * 2.0**-8, 1.0 + 2.0**-9, -2.5, 3.0e-39], dtype=np.float32)
    got = mlp.bf16(values)
    want = np.array([1.0, 1.0, 1.0 + 4 * 2.0**-8, 1.0, -2.5, 0.0])
    # 1 + 2^-8 is a tie (rounds to the even 1.0), 1 + 3 * 2^-8 rounds up, 1 + 2^-9 down
    np.testing.assert_array_equal(got[:5], want[:5])
    assert abs(got[5]) < 1e-38


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    params = rng.normal(0.0, 0.3, mlp.PARAMS)
    X = rng.normal(size=(40, mlp.FEATURES))
    y = (rng.random(40) < 0.3).astype(float)
    loss, grad = mlp.loss_and_gradients(params, X, y, 3.0, rounding=False)
    assert np.isfinite(loss)
    for index in list(rng.choice(mlp.PARAMS, 40, replace=False)) + [5312, 1024, 5184]:
        step = 1e-6
        up, down = params.copy(), params.copy()
        up[index] += step
        down[index] -= step
        numeric = (mlp.loss_and_gradients(up, X, y, 3.0, rounding=False)[0]
                   - mlp.loss_and_gradients(down, X, y, 3.0, rounding=False)[0]) / (2 * step)
        assert abs(numeric - grad[index]) <= 1e-6 * max(1.0, abs(numeric)), index


def test_features_of_a_smooth_patch():
    rng = np.random.default_rng(1)
    n, halo = 4, 2
    shape = (n + 5,) * 3
    rho = 1.0 + 0.1 * rng.random(shape)
    energy = 5.0 + rng.random(shape)
    zeros = np.zeros(shape)
    fields = (rho, zeros, zeros, zeros, energy, zeros, zeros, zeros)
    out = mlp.features(fields, (n, n, n), (0.25, 0.25, 0.25), mean_field=(1.0, 0.0, 0.0))
    assert out.shape == (n**3, 16)
    # with uniform B = (1, 0, 0) and no motion: p = (gamma - 1)(E - 1/2), |B| = 1
    i, j, k = 1, 2, 3
    row = out[(i * n + j) * n + k]
    I, J, K = i + halo, j + halo, k + halo
    assert np.isclose(row[0], np.log(rho[I, J, K]))
    assert np.isclose(row[1], np.log((2.0 / 3.0) * (energy[I, J, K] - 0.5)))
    assert np.isclose(row[2], 1.0)
    assert np.isclose(row[3], 0.5 * (np.log(rho[I + 1, J, K]) - np.log(rho[I - 1, J, K])))
    assert np.isclose(row[11], 0.0) and row[14] == 0.0 and row[15] == 0.0
    block = np.log(rho[I - 1 : I + 2, J - 1 : J + 2, K - 1 : K + 2])
    assert np.isclose(row[12], np.max(np.abs(block - np.log(rho[I, J, K]))))
