"""Device dispatch of the reference's six block kernels through the C ABI.

``KERNELS[name](*args)`` takes the reference's arguments in the reference's order
(``carafe/kernels/<name>/<name>_pyccel.py``) with device float64 arrays: torch CUDA
tensors or any object exposing ``__cuda_array_interface__`` (e.g. CuPy arrays, what
cunumpy would route to a CUDA implementation). Outputs are written in place; the
reference's return values are returned. Host (NumPy) arrays are refused: this package
has no CPU path.
"""

from __future__ import annotations

import torch

from wellbalanced_b200 import _lib

LIMITER_CODES = ("minmod", "vanleer", "mc", "none")


def _array(a, name):
    """(device pointer, shape) of a C-contiguous float64 device array."""
    if isinstance(a, torch.Tensor):
        if not a.is_cuda:
            raise TypeError(f"{name}: a CUDA tensor is required (this package has no CPU path)")
        if a.dtype != torch.float64:
            raise TypeError(f"{name}: float64 is required, got {a.dtype}")
        if not a.is_contiguous():
            raise ValueError(f"{name}: a C-contiguous array is required")
        return a.data_ptr(), tuple(a.shape)
    iface = getattr(a, "__cuda_array_interface__", None)
    if iface is None:
        raise TypeError(f"{name}: a device array is required (torch CUDA tensor or __cuda_array_interface__)")
    if iface.get("typestr") != "<f8":
        raise TypeError(f"{name}: float64 is required, got {iface.get('typestr')}")
    shape = tuple(iface["shape"])
    strides = iface.get("strides")
    if strides is not None:
        expect, step = [], 8
        for n in reversed(shape):
            expect.append(step)
            step *= n
        if tuple(reversed(expect)) != tuple(strides):
            raise ValueError(f"{name}: a C-contiguous array is required")
    return int(iface["data"][0]), shape


def _need(shape, expected, name):
    if tuple(shape) != tuple(expected):
        raise ValueError(f"{name}: shape {tuple(shape)} != expected {tuple(expected)}")


def _stream():
    return torch.cuda.current_stream().cuda_stream


def mhd_primitive(rho, mx, my, mz, energy, bz, az, dx, dy, b0x, b0y, gamma, prim, bxf, byf, ecc) -> int:
    p_rho, shape = _array(rho, "rho")
    X, Y = shape
    ptrs = [p_rho]
    for a, name in ((mx, "mx"), (my, "my"), (mz, "mz"), (energy, "energy"), (bz, "bz")):
        p, s = _array(a, name)
        _need(s, (X, Y), name)
        ptrs.append(p)
    p_az, s = _array(az, "az")
    _need(s, (X + 1, Y + 1), "az")
    outs = []
    for a, name, expect in ((prim, "prim", (8, X, Y)), (bxf, "bxf", (X + 1, Y)), (byf, "byf", (X, Y + 1)), (ecc, "ecc", (X, Y))):
        p, s = _array(a, name)
        _need(s, expect, name)
        outs.append(p)
    device = rho.device if isinstance(rho, torch.Tensor) else torch.device("cuda")
    bad = torch.zeros(1, dtype=torch.int64, device=device)
    _lib.call("wb_mhd_primitive", *ptrs, p_az, X, Y, float(dx), float(dy), float(b0x), float(b0y), float(gamma),
              *outs, bad.data_ptr(), _stream())
    return int(bad.item())


def mhd_sweep(prim, bn, axis, limiter, gamma, flux) -> None:
    p_prim, s = _array(prim, "prim")
    if len(s) != 3 or s[0] != 8:
        raise ValueError("prim: shape (8, X, Y) is required")
    _, X, Y = s
    p_bn, sb = _array(bn, "bn")
    _need(sb, (X + 1, Y) if axis == 0 else (X, Y + 1), "bn")
    p_f, sf = _array(flux, "flux")
    _need(sf, (7, X - 3, Y) if axis == 0 else (7, X, Y - 3), "flux")
    _lib.call("wb_mhd_sweep", p_prim, p_bn, int(axis), int(limiter), float(gamma), X, Y, p_f, _stream())


def ct_contact(fx_by, gy_bx, fx_rho, gy_rho, ecc, ez) -> None:
    p_ecc, s = _array(ecc, "ecc")
    X, Y = s
    ptrs = []
    for a, name, expect in ((fx_by, "fx_by", (X - 3, Y)), (gy_bx, "gy_bx", (X, Y - 3)), (fx_rho, "fx_rho", (X - 3, Y)),
                            (gy_rho, "gy_rho", (X, Y - 3))):
        p, sh = _array(a, name)
        _need(sh, expect, name)
        ptrs.append(p)
    p_ez, se = _array(ez, "ez")
    _lib.call("wb_ct_contact", *ptrs, p_ecc, X, Y, se[0], se[1], p_ez, _stream())


def mhd_rate(rho, mx, my, mz, energy, bz, az, halo, dx, dy, b0x, b0y, gamma, out) -> None:
    p_rho, shape = _array(rho, "rho")
    X, Y = shape
    ptrs = [p_rho]
    for a, name in ((mx, "mx"), (my, "my"), (mz, "mz"), (energy, "energy"), (bz, "bz")):
        p, s = _array(a, name)
        _need(s, (X, Y), name)
        ptrs.append(p)
    p_az, s = _array(az, "az")
    _need(s, (X + 1, Y + 1), "az")
    p_out, s = _array(out, "out")
    _need(s, (2,), "out")
    _lib.call("wb_mhd_rate", *ptrs, p_az, X, Y, int(halo), float(dx), float(dy), float(b0x), float(b0y), float(gamma),
              p_out, _stream())


def mhd_resistive(prim, bxf, byf, dx, dy, eta, fx, fy, ez) -> None:
    p_prim, s = _array(prim, "prim")
    _, X, Y = s
    p_bx, sb = _array(bxf, "bxf")
    _need(sb, (X + 1, Y), "bxf")
    p_by, sb = _array(byf, "byf")
    _need(sb, (X, Y + 1), "byf")
    p_fx, s1 = _array(fx, "fx")
    _need(s1, (7, X - 3, Y), "fx")
    p_fy, s2 = _array(fy, "fy")
    _need(s2, (7, X, Y - 3), "fy")
    p_ez, s3 = _array(ez, "ez")
    _need(s3, (X - 3, Y - 3), "ez")
    _lib.call("wb_mhd_resistive", p_prim, p_bx, p_by, X, Y, float(dx), float(dy), float(eta), p_fx, p_fy, p_ez, _stream())


def mhd_conductive(prim, bxf, byf, dx, dy, parallel, perpendicular, fx, fy) -> None:
    p_prim, s = _array(prim, "prim")
    _, X, Y = s
    p_bx, sb = _array(bxf, "bxf")
    _need(sb, (X + 1, Y), "bxf")
    p_by, sb = _array(byf, "byf")
    _need(sb, (X, Y + 1), "byf")
    p_fx, s1 = _array(fx, "fx")
    _need(s1, (7, X - 3, Y), "fx")
    p_fy, s2 = _array(fy, "fy")
    _need(s2, (7, X, Y - 3), "fy")
    _lib.call("wb_mhd_conductive", p_prim, p_bx, p_by, X, Y, float(dx), float(dy), float(parallel),
              float(perpendicular), p_fx, p_fy, _stream())


class Kernel:
    """A callable with the reference kernel object's interface (``kernel(...)``, ``selected()``)."""

    def __init__(self, name, function):
        self.name = name
        self._function = function
        self.__doc__ = function.__doc__

    def __call__(self, *args):
        return self._function(*args)

    def selected(self) -> str:
        return "cuda"

    def __repr__(self):
        return f"<wellbalanced_b200 kernel {self.name} (cuda)>"


KERNELS = {
    "mhd_primitive": Kernel("mhd_primitive", mhd_primitive),
    "mhd_sweep": Kernel("mhd_sweep", mhd_sweep),
    "ct_contact": Kernel("ct_contact", ct_contact),
    "mhd_rate": Kernel("mhd_rate", mhd_rate),
    "mhd_resistive": Kernel("mhd_resistive", mhd_resistive),
    "mhd_conductive": Kernel("mhd_conductive", mhd_conductive),
}
