"""The reference's block kernels on the device against the reference's own outputs (GPU).

Mirrors ``tests/unit/test_mhd_kernels.py`` of the reference (compiled vs NumPy kernels,
rtol = atol = 1e-12 for the sweep, 1e-14 for CT and the primitives): here the CUDA
kernels, called through the C ABI, against the golden outputs of the reference's
kernels, and against the oracle on larger random blocks.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).with_name("golden")
GAMMA = 5.0 / 3.0
SHAPE = (13, 9)


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def host(t):
    return t.cpu().numpy()


@pytest.fixture(scope="module")
def kernels():
    return np.load(GOLDEN / "kernels.npz")


@pytest.fixture(scope="module")
def K():
    from wellbalanced_b200.kernels import KERNELS

    return KERNELS


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("axis", [0, 1])
@pytest.mark.parametrize("limiter", range(4))
def test_sweep_matches_the_reference(K, kernels, seed, axis, limiter):
    prim = kernels[f"block{seed}_prim"]
    bn = kernels[f"block{seed}_{'bxf' if axis == 0 else 'byf'}"]
    nx, ny = SHAPE
    flux = torch.full((7, nx - 3, ny) if axis == 0 else (7, nx, ny - 3), float("nan"), dtype=torch.float64, device="cuda")
    K["mhd_sweep"](dev(prim), dev(bn), axis, limiter, GAMMA, flux)
    got = host(flux)
    assert np.all(np.isfinite(got))
    for impl in ("numpy", "pyccel"):
        np.testing.assert_allclose(got, kernels[f"block{seed}_sweep_a{axis}_l{limiter}_{impl}"], rtol=1e-12, atol=1e-12)


def test_ct_contact_matches_the_reference(K, kernels):
    nx, ny = SHAPE
    fx, fy, ecc = kernels["ct_fx"], kernels["ct_fy"], kernels["ct_ecc"]
    ez = torch.full((nx - 3, ny - 3), float("nan"), dtype=torch.float64, device="cuda")
    K["ct_contact"](dev(fx[5]), dev(fy[5]), dev(fx[0]), dev(fy[0]), dev(ecc), ez)
    np.testing.assert_allclose(host(ez), kernels["ct_ez_pyccel"], rtol=0, atol=1e-14)


def test_primitive_and_rate_match_the_reference(K, kernels):
    nx, ny = SHAPE
    fields = [dev(kernels[f"cons_{k}"]) for k in range(6)]
    az = dev(kernels["cons_az"])
    prim = torch.full((8, nx, ny), float("nan"), dtype=torch.float64, device="cuda")
    bxf = torch.empty((nx + 1, ny), dtype=torch.float64, device="cuda")
    byf = torch.empty((nx, ny + 1), dtype=torch.float64, device="cuda")
    ecc = torch.empty((nx, ny), dtype=torch.float64, device="cuda")
    bad = K["mhd_primitive"](*fields, az, 0.1, 0.2, 0.3, -0.4, GAMMA, prim, bxf, byf, ecc)
    assert bad == 0
    for got, key in ((prim, "prim"), (bxf, "bxf"), (byf, "byf"), (ecc, "ecc")):
        np.testing.assert_allclose(host(got), kernels[f"primitive_{key}_pyccel"], rtol=1e-14, atol=1e-14)
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    K["mhd_rate"](*fields, az, 2, 0.1, 0.2, 0.3, -0.4, GAMMA, out)
    np.testing.assert_allclose(host(out), kernels["rate_pyccel"], rtol=1e-14)
    assert host(out)[1] == np.min(kernels["cons_0"][2:-2, 2:-2])


@pytest.mark.parametrize(("row", "value"), [(0, -1.0), (4, -1.0e3), (1, np.inf), (2, np.nan), (5, -np.inf), (0, np.nan)])
def test_primitive_counts_the_bad_cells(K, kernels, row, value):
    nx, ny = SHAPE
    fields = [kernels[f"cons_{k}"].copy() for k in range(6)]
    fields[row][3, 4] = value
    fields[row][7, 1] = value
    out = [torch.empty(s, dtype=torch.float64, device="cuda") for s in ((8, nx, ny), (nx + 1, ny), (nx, ny + 1), (nx, ny))]
    bad = K["mhd_primitive"](*map(dev, fields), dev(kernels["cons_az"]), 0.1, 0.2, 0.3, -0.4, GAMMA, *out)
    assert bad == 2


def test_resistive_and_conductive_match_the_reference(K, kernels):
    prim, bxf, byf = (dev(kernels[f"block1_{k}"]) for k in ("prim", "bxf", "byf"))
    fx, fy, ez = dev(kernels["res_fx0"]), dev(kernels["res_fy0"]), dev(kernels["res_ez0"])
    K["mhd_resistive"](prim, bxf, byf, 0.1, 0.2, 0.05, fx, fy, ez)
    for got, key in ((fx, "fx"), (fy, "fy"), (ez, "ez")):
        np.testing.assert_allclose(host(got), kernels[f"res_{key}_pyccel"], rtol=1e-13, atol=1e-13)
    fx, fy = dev(kernels["cond_fx0"]), dev(kernels["cond_fy0"])
    K["mhd_conductive"](dev(kernels["cond_prim"]), dev(kernels["cond_bxf"]), dev(kernels["cond_byf"]), 0.1, 0.2, 0.3,
                        0.01, fx, fy)
    for got, key in ((fx, "fx"), (fy, "fy")):
        np.testing.assert_allclose(host(got), kernels[f"cond_{key}_pyccel"], rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("limiter", range(4))
def test_sweep_matches_the_oracle_on_a_larger_block(K, limiter):
    from oracle import kernels as O

    rng = np.random.default_rng(100 + limiter)
    X, Y = 67, 45
    prim = rng.normal(size=(8, X, Y))
    prim[0] = rng.uniform(0.2, 3.0, (X, Y))
    prim[4] = rng.uniform(0.05, 2.0, (X, Y))
    prim[1, :, 5] += 20.0
    bn_x, bn_y = rng.normal(size=(X + 1, Y)), rng.normal(size=(X, Y + 1))
    bn_x[10:20, 3] = 0.0
    for axis, bn in ((0, bn_x), (1, bn_y)):
        shape = (7, X - 3, Y) if axis == 0 else (7, X, Y - 3)
        expect = np.empty(shape)
        O.mhd_sweep(prim, bn, axis, limiter, GAMMA, expect)
        got = torch.empty(shape, dtype=torch.float64, device="cuda")
        K["mhd_sweep"](dev(prim), dev(bn), axis, limiter, GAMMA, got)
        np.testing.assert_allclose(host(got), expect, rtol=1e-12, atol=1e-12)


def test_host_arrays_are_refused(K, kernels):
    nx, ny = SHAPE
    with pytest.raises(TypeError, match="CUDA|device"):
        K["mhd_sweep"](kernels["block1_prim"], kernels["block1_bxf"], 0, 0, GAMMA, np.empty((7, nx - 3, ny)))
    assert K["mhd_sweep"].selected() == "cuda"
