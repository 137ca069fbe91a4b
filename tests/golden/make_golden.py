"""Generate the golden vectors of the oracle from the reference itself.

Run in a container holding the reference checkout, given by ``--reference`` or the
``WB_REFERENCE`` environment variable (the checkout's root, holding ``src/carafe``)::

    python tests/golden/make_golden.py --reference PATH [--full]

The reference's own ``carafe.mhd.MHD2D`` / ``carafe.mhd3d.MHD3D`` and its kernels
(``carafe/kernels/<name>/<name>_numpy.py`` and ``_pyccel.py`` run as plain Python) are
imported unchanged; the absent dependencies are replaced by ``reference_stubs.py``
(one refinement level). The outputs are small ``.npz`` fixtures next to this script;
the tests compare the oracle and the CUDA path against them. ``--full`` also runs
the Orszag–Tang vortex on 256^2 cells to t = 0.5 (about 11 minutes on one core).
"""

from __future__ import annotations

import argparse
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parents[1]))

import reference_stubs  # noqa: E402

GAMMA = 5.0 / 3.0
SHAPE = (13, 9)


def kernel_block(seed=1):
    """Primitive block with supersonic rows, a near-vacuum cell and zero B_n.

    The construction of ``tests/unit/test_mhd_kernels.py:20-33``.
    """
    rng = np.random.default_rng(seed)
    nx, ny = SHAPE
    prim = rng.normal(size=(8, nx, ny))
    prim[0] = rng.uniform(0.5, 2.0, SHAPE)
    prim[4] = rng.uniform(0.1, 1.0, SHAPE)
    prim[1, :, 6] += 30.0
    prim[2, 8, :] -= 30.0
    prim[4, 5, 3] = 1.0e-3
    bxf = rng.normal(size=(nx + 1, ny))
    byf = rng.normal(size=(nx, ny + 1))
    bxf[4, 2] = byf[2, 4] = 0.0
    return prim, bxf, byf


def conserved_block(seed=3):
    """Conserved block with positive pressure (``test_mhd_kernels.py:95-104``)."""
    rng = np.random.default_rng(seed)
    nx, ny = SHAPE
    rho = rng.uniform(0.5, 2.0, SHAPE)
    momenta = [rng.normal(size=SHAPE) * rho for _ in range(3)]
    bz = rng.normal(size=SHAPE)
    az = 0.1 * rng.normal(size=(nx + 1, ny + 1))
    energy = 20.0 + rng.uniform(size=SHAPE)
    return [rho, *momenta, energy, bz], az


def kernels_golden(out):
    from carafe.kernels.ct_contact import kernel as ct_contact
    from carafe.kernels.mhd_conductive import kernel as mhd_conductive
    from carafe.kernels.mhd_primitive import kernel as mhd_primitive
    from carafe.kernels.mhd_rate import kernel as mhd_rate
    from carafe.kernels.mhd_resistive import kernel as mhd_resistive
    from carafe.kernels.mhd_sweep import kernel as mhd_sweep
    from carafe.mhd import hlld_flux

    data = {}
    nx, ny = SHAPE
    for seed in (1, 2, 3):
        prim, bxf, byf = kernel_block(seed)
        data[f"block{seed}_prim"] = prim
        data[f"block{seed}_bxf"] = bxf
        data[f"block{seed}_byf"] = byf
        for axis in (0, 1):
            for limiter in range(4):
                shape = (7, nx - 3, ny) if axis == 0 else (7, nx, ny - 3)
                for impl in ("numpy", "pyccel"):
                    with reference_stubs.use_host_kernel_implementation(impl):
                        flux = np.full(shape, np.nan)
                        mhd_sweep(prim, (bxf, byf)[axis], axis, limiter, GAMMA, flux)
                    data[f"block{seed}_sweep_a{axis}_l{limiter}_{impl}"] = flux
    rng = np.random.default_rng(2)
    fx = rng.normal(size=(7, nx - 3, ny))
    fy = rng.normal(size=(7, nx, ny - 3))
    fx[0, 3, 4] = fy[0, 2, 5] = 0.0
    ecc = rng.normal(size=SHAPE)
    data.update(ct_fx=fx, ct_fy=fy, ct_ecc=ecc)
    for impl in ("numpy", "pyccel"):
        with reference_stubs.use_host_kernel_implementation(impl):
            ez = np.full((nx - 3, ny - 3), np.nan)
            ct_contact(fx[5], fy[5], fx[0], fy[0], ecc, ez)
        data[f"ct_ez_{impl}"] = ez
    fields, az = conserved_block()
    for k, f in enumerate(fields):
        data[f"cons_{k}"] = f
    data["cons_az"] = az
    for impl in ("numpy", "pyccel"):
        with reference_stubs.use_host_kernel_implementation(impl):
            prim = np.full((8, nx, ny), np.nan)
            bxf = np.full((nx + 1, ny), np.nan)
            byf = np.full((nx, ny + 1), np.nan)
            ecc = np.full(SHAPE, np.nan)
            bad = mhd_primitive(*fields, az, 0.1, 0.2, 0.3, -0.4, GAMMA, prim, bxf, byf, ecc)
            data[f"primitive_bad_{impl}"] = np.array(bad)
            data[f"primitive_prim_{impl}"] = prim
            data[f"primitive_bxf_{impl}"] = bxf
            data[f"primitive_byf_{impl}"] = byf
            data[f"primitive_ecc_{impl}"] = ecc
            rate = np.full(2, np.nan)
            mhd_rate(*fields, az, 2, 0.1, 0.2, 0.3, -0.4, GAMMA, rate)
            data[f"rate_{impl}"] = rate
    # bad-cell counting (test_mhd_kernels.py:123-141)
    cases = [(0, -1.0), (4, -1.0e3), (1, np.inf), (2, np.nan), (5, -np.inf), (0, np.nan)]
    counts = []
    for row, value in cases:
        f2 = [f.copy() for f in fields]
        f2[row][3, 4] = value
        f2[row][7, 1] = value
        with reference_stubs.use_host_kernel_implementation("numpy"):
            prim = np.empty((8, nx, ny))
            bad = mhd_primitive(
                *f2, az, 0.1, 0.2, 0.3, -0.4, GAMMA, prim,
                np.empty((nx + 1, ny)), np.empty((nx, ny + 1)), np.empty(SHAPE),
            )
        counts.append(bad)
    data["bad_counts"] = np.array(counts)
    # resistive / conductive (test_mhd_kernels.py:156-191)
    prim, bxf, byf = kernel_block(1)
    rng = np.random.default_rng(4)
    fx0 = rng.normal(size=(7, nx - 3, ny))
    fy0 = rng.normal(size=(7, nx, ny - 3))
    ez0 = rng.normal(size=(nx - 3, ny - 3))
    data.update(res_fx0=fx0, res_fy0=fy0, res_ez0=ez0)
    for impl in ("numpy", "pyccel"):
        with reference_stubs.use_host_kernel_implementation(impl):
            fx, fy, ez = fx0.copy(), fy0.copy(), ez0.copy()
            mhd_resistive(prim, bxf, byf, 0.1, 0.2, 0.05, fx, fy, ez)
        data[f"res_fx_{impl}"], data[f"res_fy_{impl}"], data[f"res_ez_{impl}"] = fx, fy, ez
    prim_c, bxf_c, byf_c = kernel_block(1)
    prim_c[5:8, 6, 4] = 0.0
    bxf_c[6:8, 4] = byf_c[6, 4:6] = 0.0
    rng = np.random.default_rng(5)
    fx0 = rng.normal(size=(7, nx - 3, ny))
    fy0 = rng.normal(size=(7, nx, ny - 3))
    data.update(cond_prim=prim_c, cond_bxf=bxf_c, cond_byf=byf_c, cond_fx0=fx0, cond_fy0=fy0)
    for impl in ("numpy", "pyccel"):
        with reference_stubs.use_host_kernel_implementation(impl):
            fx, fy = fx0.copy(), fy0.copy()
            mhd_conductive(prim_c, bxf_c, byf_c, 0.1, 0.2, 0.3, 0.01, fx, fy)
        data[f"cond_fx_{impl}"], data[f"cond_fy_{impl}"] = fx, fy
    # HLLD on random states, including B_n = 0, supersonic and degenerate faces
    rng = np.random.default_rng(11)
    count = 1024
    left = rng.normal(size=(7, count))
    right = rng.normal(size=(7, count))
    for side in (left, right):
        side[0] = rng.uniform(0.05, 3.0, count)
        side[4] = rng.uniform(0.01, 3.0, count)
    left[1, :64] += 25.0
    right[1, :64] += 25.0
    left[1, 64:128] -= 25.0
    right[1, 64:128] -= 25.0
    bn = rng.normal(size=count)
    bn[128:192] = 0.0
    left[5:7, 192:256] = 0.0  # degenerate star denominators
    right[5:7, 192:256] = 0.0
    bn[192:256] = 1.0
    left[:, 256:320] = right[:, 256:320]  # consistency F(U, U) = F(U)
    data.update(hlld_left=left, hlld_right=right, hlld_bn=bn)
    data["hlld_flux"] = hlld_flux(left, right, bn, GAMMA)
    np.savez_compressed(out / "kernels.npz", **data)


def _state2d(model):
    (patch,) = model.hierarchy.patches
    out = {
        name: np.array(patch.field(model.names[name]).local)
        for name in ("density", "momentum_x", "momentum_y", "momentum_z", "energy", "bz")
    }
    out["az"] = np.array(patch.field(model.potential).local)
    return out


def runs2d_golden(out):
    from carafe.mhd import MHD2D
    from patchwork import AMRHierarchy

    data = {}

    def store(prefix, model, extra=None):
        for key, value in _state2d(model).items():
            data[f"{prefix}_{key}"] = value
        data[f"{prefix}_time"] = np.array(model.time)
        data[f"{prefix}_steps"] = np.array(model.steps)
        data[f"{prefix}_div"] = np.array(model.divergence())
        totals = model.totals()
        data[f"{prefix}_totals"] = np.array([totals[k] for k in sorted(totals)])
        for key, value in (extra or {}).items():
            data[f"{prefix}_{key}"] = value

    # OT 32^2, 5 steps (test_mhd_kernels.py:79-92)
    model = MHD2D.orszag_tang(32)
    dts = [model.step() for _ in range(5)]
    store("ot32_5", model, {"dts": np.array(dts)})
    # OT 32^2 to t = 0.1 (test_mhd.py:89-97), with the initial totals
    model = MHD2D.orszag_tang(32)
    before = model.totals()
    model.run(0.1)
    store("ot32_run", model, {"totals0": np.array([before[k] for k in sorted(before)])})
    # OT 64^2, MC limiter, CFL 0.4, to t = 0.5: the CPU-sized Orszag-Tang workload
    start = time.perf_counter()
    model = MHD2D.orszag_tang(64, limiter="mc", cfl=0.4)
    model.run(0.5)
    store("ot64_mc", model, {"seconds": np.array(time.perf_counter() - start)})
    # all four limiters, OT 24^2, 8 steps
    for limiter in ("minmod", "vanleer", "mc", "none"):
        model = MHD2D.orszag_tang(24, limiter=limiter)
        for _ in range(8):
            model.step()
        store(f"ot24_{limiter}", model)
    # Brio-Wu along x and y (outflow; test_mhd.py:100-139)
    for axis in (0, 1):
        cells = 64
        if axis == 0:
            mesh = AMRHierarchy((cells, 2), ((0.0, 1.0), (0.0, 2.0 / cells)), periodic=(False, True))
        else:
            mesh = AMRHierarchy((2, cells), ((0.0, 2.0 / cells), (0.0, 1.0)), periodic=(True, False))
        mean = (0.75, 0.0) if axis == 0 else (0.0, 0.75)
        model = MHD2D(mesh, gamma=2.0, mean_field=mean)
        sign = 1.0 if axis == 0 else -1.0

        def s(x, y, axis=axis):
            return x if axis == 0 else y

        model.set_state(
            lambda x, y, s=s: np.where(s(x, y) < 0.5, 1.0, 0.125),
            (0.0, 0.0, 0.0),
            lambda x, y, s=s: np.where(s(x, y) < 0.5, 1.0, 0.1),
            vector_potential=lambda x, y, s=s, sign=sign: sign * np.abs(s(x, y) - 0.5),
        )
        model.run(0.1)
        store(f"briowu{axis}", model)
    # rotor (outflow faces, mean field, gamma 1.4)
    model = MHD2D.rotor(32)
    model.run(0.02)
    store("rotor32", model)
    # blast (minmod default)
    model = MHD2D.blast_wave(32)
    model.run(0.03)
    store("blast32", model)
    # Rayleigh-Taylor: walls and gravity
    model = MHD2D.rayleigh_taylor(8, field=0.05)
    for _ in range(20):
        model.step()
    store("rt8", model)
    # resistive + conductive OT (test_mhd_kernels.py:194-216)
    model = MHD2D.orszag_tang(16, resistivity=1e-3, conduction=(1e-2, 1e-3))
    for _ in range(3):
        model.step()
    store("ot16_resistive", model)
    model = MHD2D.rayleigh_taylor(8, resistivity=1e-3, conduction=(1e-3, 0.0), field=0.05)
    for _ in range(3):
        model.step()
    store("rt8_resistive", model)
    # uniform state with outflow faces (test_mhd.py:142-151)
    model = MHD2D(AMRHierarchy((8, 6), ((0.0, 1.0), (0.0, 1.0))), mean_field=(0.3, -0.2), limiter="mc")
    model.set_state(1.0, (0.2, -0.1, 0.05), 0.5, bz=0.4)
    model.run(0.2)
    store("uniform8x6", model)
    # the Alfven wave, unlimited, one period at 16 cells
    model, _ = MHD2D.alfven_wave(16, limiter="none")
    model.run(model.period)
    store("alfven16", model)
    np.savez_compressed(out / "runs2d.npz", **data)


def runs3d_golden(out):
    from carafe.mhd import MHD2D
    from carafe.mhd3d import MHD3D
    from patchwork import AMRHierarchy

    from wellbalanced_b200.problems import turbulence_3d

    data = {}

    def store(prefix, model):
        (patch,) = model.hierarchy.patches
        for name in ("density", "momentum_x", "momentum_y", "momentum_z", "energy"):
            data[f"{prefix}_{name}"] = np.array(patch.field(model.names[name]).local)
        for key, name in zip(("ax", "ay", "az"), model.potential, strict=True):
            data[f"{prefix}_{key}"] = np.array(patch.field(name).local)
        data[f"{prefix}_time"] = np.array(model.time)
        data[f"{prefix}_div"] = np.array(model.divergence())
        totals = model.totals()
        data[f"{prefix}_totals"] = np.array([totals[k] for k in sorted(totals)])

    # z-uniform OT equals 2D (test_mhd3d.py:24-38)
    flat = MHD3D.orszag_tang(16, layers=2)
    plane = MHD2D.orszag_tang(16)
    dts = []
    for _ in range(10):
        dt = plane.stable_step()
        dts.append(dt)
        plane.step(dt)
        flat.step(dt)
    store("ot3d16", flat)
    data["ot3d16_dts"] = np.array(dts)
    # 3D Alfven wave, unlimited, 8 cells, 0.1
    model, _ = MHD3D.alfven_wave(8, limiter="none")
    model.run(0.1)
    store("alfven3d8", model)
    # 3D blast, minmod, 12 cells
    model = MHD3D.blast_wave(12)
    model.run(0.01)
    store("blast3d12", model)
    # decaying turbulence, MC, CFL 0.3: 16^3, 4 steps (the 3D turbulence workload, small)
    for n, steps in ((16, 4),):
        rho, velocity, p, potential = turbulence_3d(n, seed=7)
        mesh = AMRHierarchy((n, n, n), ((0.0, 1.0),) * 3, periodic=(True,) * 3)
        model = MHD3D(mesh, limiter="mc", cfl=0.3)
        model.set_state(rho, velocity, p, vector_potential=potential)
        store(f"turb{n}_init", model)
        dts = [model.step() for _ in range(steps)]
        store(f"turb{n}", model)
        data[f"turb{n}_dts"] = np.array(dts)
    # outflow faces in 3D, uniform state (test_mhd3d.py:123-132), and a non-uniform one
    mesh = AMRHierarchy((6, 4, 5), ((0.0, 1.0),) * 3, periodic=(False, True, False))
    model = MHD3D(mesh, mean_field=(0.3, -0.2, 0.5))
    model.set_state(1.2, (0.1, -0.2, 0.3), 0.7)
    for _ in range(4):
        model.step()
    store("uniform3d", model)
    mesh = AMRHierarchy((8, 6, 7), ((0.0, 1.0),) * 3, periodic=(False, True, False))
    model = MHD3D(mesh, mean_field=(0.3, -0.2, 0.5), limiter="mc")
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
    store("outflow3d", model)
    # resistive force-free field (test_mhd3d.py:95-120), a few steps
    mesh = AMRHierarchy((4, 4, 16), ((0.0, 1.0),) * 3, periodic=(True,) * 3)
    k = 2.0 * np.pi
    model = MHD3D(mesh, resistivity=0.01)
    model.set_state(
        1.0,
        (0.0, 0.0, 0.0),
        1.0,
        vector_potential=(lambda x, y, z: np.cos(k * z) / k, lambda x, y, z: np.sin(k * z) / k, 0.0),
    )
    for _ in range(5):
        model.step()
    store("resistive3d", model)
    np.savez_compressed(out / "runs3d.npz", **data)


def multipatch_golden(out):
    """OT 32^2 on 2 x 3 patches of one level, 5 steps: the same as one patch."""
    from carafe.mhd import MHD2D

    mesh = reference_stubs.AMRHierarchy((32, 32), ((0.0, 1.0), (0.0, 1.0)), periodic=(True, True), split=(2, 3))
    model = MHD2D(mesh)
    b0 = 1.0 / np.sqrt(4.0 * np.pi)
    model.set_state(
        25.0 / (36.0 * np.pi),
        lambda x, y: (-np.sin(2 * np.pi * y), np.sin(2 * np.pi * x), 0.0 * x),
        5.0 / (12.0 * np.pi),
        vector_potential=lambda x, y: b0
        * (np.cos(4 * np.pi * x) / (4 * np.pi) + np.cos(2 * np.pi * y) / (2 * np.pi)),
    )
    for _ in range(5):
        model.step()
    data = {}
    rho = np.zeros((32, 32))
    for patch in mesh.patches:
        (i0, i1), (j0, j1) = patch.box
        rho[i0:i1, j0:j1] = patch.field(model.names["density"]).local
    data["split_density"] = rho
    np.savez_compressed(out / "multipatch.npz", **data)


def full_golden(out):
    from carafe.mhd import MHD2D

    start = time.perf_counter()
    model = MHD2D.orszag_tang(256, limiter="mc", cfl=0.4)
    before = model.totals()
    steps = model.run(0.5)
    seconds = time.perf_counter() - start
    state = _state2d(model)
    totals = model.totals()
    np.savez_compressed(
        out / "ot256_full.npz",
        density=state["density"],
        energy=state["energy"],
        steps=np.array(steps),
        time=np.array(model.time),
        seconds=np.array(seconds),
        div=np.array(model.divergence()),
        totals0=np.array([before[k] for k in sorted(before)]),
        totals=np.array([totals[k] for k in sorted(totals)]),
    )


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default=os.environ.get("WB_REFERENCE"),
                        help="the reference checkout's root (default: $WB_REFERENCE)")
    parser.add_argument("--full", action="store_true")
    parser.add_argument("--only", default=None)
    args = parser.parse_args()
    if not args.reference:
        parser.error("give the reference checkout with --reference PATH or WB_REFERENCE")
    reference_stubs.install(f"{args.reference}/src")
    jobs = {
        "kernels": kernels_golden,
        "runs2d": runs2d_golden,
        "runs3d": runs3d_golden,
        "multipatch": multipatch_golden,
    }
    if args.full:
        jobs = {"full": full_golden}
    for name, job in jobs.items():
        if args.only and name != args.only:
            continue
        start = time.perf_counter()
        job(HERE)
        print(f"{name}: {time.perf_counter() - start:.1f} s", flush=True)


if __name__ == "__main__":
    main()
