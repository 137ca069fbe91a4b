"""Test infrastructure: float64 NumPy restatement of the learned tagger's kernels.

The learned refinement tagger has no counterpart in the reference (it predicts where the
plain current tagger of ``carafe/mhd3d.py:771-801`` will flag cells); this module is the
checker of its CUDA kernels (``wellbalanced_b200/csrc/tagger.cu``): the stencil features,
the forward pass and the gradients of the weighted binary cross-entropy. Only tests use
it.

Model: x^ = bf16(x); z1 = bf16(W1) x^ + b1; h1 = relu(z1); z2 = bf16(W2) bf16(h1) + b2;
h2 = relu(z2); z = bf16(W3) . h2 + b3; bf16 is round-to-nearest-even to bfloat16 and the
gradients pass through it unchanged. Parameters: one vector W1 [64][16] | b1 | W2 [64][64]
| b2 | W3 | b3 (5313 values).
"""

from __future__ import annotations

import numpy as np

FEATURES, HIDDEN = 16, 64
SLICES = {
    "W1": slice(0, 1024),
    "b1": slice(1024, 1088),
    "W2": slice(1088, 5184),
    "b2": slice(5184, 5248),
    "W3": slice(5248, 5312),
    "b3": slice(5312, 5313),
}
PARAMS = 5313


def bf16(x):
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float64."""
    bits = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32).astype(np.uint64)
    rounded = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params):
    p = np.asarray(params, dtype=np.float64)
    return {
        "W1": p[SLICES["W1"]].reshape(HIDDEN, FEATURES),
        "b1": p[SLICES["b1"]],
        "W2": p[SLICES["W2"]].reshape(HIDDEN, HIDDEN),
        "b2": p[SLICES["b2"]],
        "W3": p[SLICES["W3"]],
        "b3": p[SLICES["b3"]][0],
    }


def forward(params, X, rounding=True):
    """Logits and the intermediate values of the forward pass for rows of X (N, 16);
    ``rounding=False`` drops the bfloat16 roundings (a smooth model for derivative checks)."""
    r = bf16 if rounding else (lambda v: np.asarray(v, dtype=np.float64))
    w = unpack(params)
    x = r(X)
    z1 = x @ r(w["W1"]).T + w["b1"]
    h1 = r(np.maximum(z1, 0.0))
    z2 = h1 @ r(w["W2"]).T + w["b2"]
    h2 = np.maximum(z2, 0.0)
    z = h2 @ r(w["W3"]) + w["b3"]
    return z, {"x": x, "z1": z1, "h1": h1, "z2": z2, "h2": h2, "round": r}


def loss_and_gradients(params, X, y, pos_weight, rounding=True):
    """Summed weighted BCE-with-logits loss and its gradient (parameter layout)."""
    w = unpack(params)
    z, c = forward(params, X, rounding)
    r = c["round"]
    weight = np.where(y > 0.5, pos_weight, 1.0)
    loss = float(np.sum(weight * (np.maximum(z, 0.0) + np.log1p(np.exp(-np.abs(z))) - y * z)))
    d3 = weight * (1.0 / (1.0 + np.exp(-z)) - y)
    d2 = np.where(c["z2"] > 0.0, d3[:, None] * r(w["W3"])[None, :], 0.0)
    d1 = np.where(c["z1"] > 0.0, d2 @ r(w["W2"]), 0.0)
    grad = np.zeros(PARAMS)
    grad[SLICES["W1"]] = (d1.T @ c["x"]).ravel()
    grad[SLICES["b1"]] = d1.sum(axis=0)
    grad[SLICES["W2"]] = (d2.T @ c["h1"]).ravel()
    grad[SLICES["b2"]] = d2.sum(axis=0)
    grad[SLICES["W3"]] = d3 @ c["h2"]
    grad[SLICES["b3"]] = d3.sum()
    return loss, grad


def cell_quantities(fields, spacing, mean_field=(0.0, 0.0, 0.0), gamma=5.0 / 3.0):
    """(log rho, log p, |B|) of every cell of a haloed 3D patch whose edges exist.

    ``fields``: the 8 haloed arrays (rho, m_x, m_y, m_z, E on cells; A_x, A_y, A_z on
    edges) as node-shaped (X+1, Y+1, Z+1) blocks; returns (3, X, Y, Z).
    """
    rho, mx, my, mz, energy, ax, ay, az = (np.asarray(f, dtype=np.float64) for f in fields)
    dx, dy, dz = spacing
    X, Y, Z = rho.shape[0] - 1, rho.shape[1] - 1, rho.shape[2] - 1
    # face fields: x-faces on (nodes, cells, cells), y-faces on (cells, nodes, cells), ...
    bxf = ((az[:, 1 : Y + 1, :Z] - az[:, :Y, :Z]) / dy - (ay[:, :Y, 1 : Z + 1] - ay[:, :Y, :Z]) / dz
           + mean_field[0])
    byf = ((ax[:X, :, 1 : Z + 1] - ax[:X, :, :Z]) / dz - (az[1 : X + 1, :, :Z] - az[:X, :, :Z]) / dx
           + mean_field[1])
    bzf = ((ay[1 : X + 1, :Y, :] - ay[:X, :Y, :]) / dx - (ax[:X, 1 : Y + 1, :] - ax[:X, :Y, :]) / dy
           + mean_field[2])
    bx = 0.5 * (bxf[:X] + bxf[1 : X + 1])
    by = 0.5 * (byf[:, :Y] + byf[:, 1 : Y + 1])
    bz = 0.5 * (bzf[:, :, :Z] + bzf[:, :, 1 : Z + 1])
    r = rho[:X, :Y, :Z]
    kinetic = 0.5 * (mx[:X, :Y, :Z] ** 2 + my[:X, :Y, :Z] ** 2 + mz[:X, :Y, :Z] ** 2) / r
    p = (gamma - 1.0) * (energy[:X, :Y, :Z] - kinetic - 0.5 * (bx**2 + by**2 + bz**2))
    return np.stack((np.log(np.maximum(r, 1e-30)), np.log(np.maximum(p, 1e-30)), np.sqrt(bx**2 + by**2 + bz**2)))


def features(fields, shape, spacing, mean_field=(0.0, 0.0, 0.0), gamma=5.0 / 3.0, halo=2):
    """Stencil features (N, 16) of a patch's interior cells in (i, j, k) order (unnormalised):
    per quantity the value, the three half central differences and the largest deviation
    over the 26 neighbours; feature 15 is zero."""
    q = cell_quantities(fields, spacing, mean_field, gamma)
    nx, ny, nz = shape
    out = np.zeros((nx, ny, nz, FEATURES))

    def at(a, b, c):
        return q[:, halo + a : halo + a + nx, halo + b : halo + b + ny, halo + c : halo + c + nz]

    centre = at(0, 0, 0)
    deviation = np.zeros_like(centre)
    for a in (-1, 0, 1):
        for b in (-1, 0, 1):
            for c in (-1, 0, 1):
                deviation = np.maximum(deviation, np.abs(at(a, b, c) - centre))
    for v in range(3):
        out[..., v] = centre[v]
        out[..., 3 + 3 * v + 0] = 0.5 * (at(1, 0, 0)[v] - at(-1, 0, 0)[v])
        out[..., 3 + 3 * v + 1] = 0.5 * (at(0, 1, 0)[v] - at(0, -1, 0)[v])
        out[..., 3 + 3 * v + 2] = 0.5 * (at(0, 0, 1)[v] - at(0, 0, -1)[v])
        out[..., 12 + v] = deviation[v]
    return out.reshape(-1, FEATURES)
