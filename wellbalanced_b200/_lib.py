"""ctypes binding of libwb200.so (the C ABI of include/wellbalanced_b200.h).

The library is built in-tree (``python -m wellbalanced_b200.build``). Loading fails
loudly when it is missing: there is no CPU fallback for any product path.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "libwb200.so"

_lib = None

c_dp = ctypes.c_void_p
c_i64 = ctypes.c_int64
c_int = ctypes.c_int
c_double = ctypes.c_double

# C signatures: name -> argument types (all return int status)
SIGNATURES = {
    "wb_mhd_primitive": [c_dp] * 7 + [c_i64, c_i64] + [c_double] * 5 + [c_dp] * 5 + [c_dp],
    "wb_mhd_sweep": [c_dp, c_dp, c_int, c_int, c_double, c_i64, c_i64, c_dp, c_dp],
    "wb_ct_contact": [c_dp] * 5 + [c_i64] * 4 + [c_dp, c_dp],
    "wb_ct_contact_planes": [c_dp] * 5 + [c_i64] * 5 + [c_dp, c_dp],
    "wb_mhd_rate": [c_dp] * 7 + [c_i64, c_i64, c_int] + [c_double] * 5 + [c_dp, c_dp],
    "wb_mhd_resistive": [c_dp] * 3 + [c_i64, c_i64] + [c_double] * 3 + [c_dp] * 3 + [c_dp],
    "wb_mhd_conductive": [c_dp] * 3 + [c_i64, c_i64] + [c_double] * 4 + [c_dp] * 2 + [c_dp],
    "wb_stage2d": [c_int, c_dp, c_dp, c_dp, c_dp, c_dp, c_int, c_dp, c_double, c_double, c_double, c_int, c_dp,
                   c_dp, c_dp],
    "wb_stage3d": [c_int, c_dp, c_dp, c_dp, c_dp, c_dp, c_int, c_dp, c_double, c_double, c_double, c_double,
                   c_int, c_int, c_dp, c_dp, c_dp],
    "wb_stage2d_physics": [c_int, c_dp, c_dp, c_dp, c_dp, c_dp, c_int, c_dp, c_double, c_double, c_double, c_int,
                           c_double, c_double, c_double, c_double, c_double, c_dp, c_dp],
    "wb_stage3d_physics": [c_int, c_dp, c_dp, c_dp, c_dp, c_dp, c_int, c_dp, c_double, c_double, c_double,
                           c_double, c_int, c_int, c_double, c_double, c_double, c_double, c_dp, c_dp],
    "wb_stage2d_tiled": [c_int, c_dp, c_dp, c_dp, c_dp, c_dp, c_int, c_dp, c_double, c_double, c_double, c_int,
                         c_int, c_int, c_dp, c_dp, c_dp],
    "wb_stage3d_tiled": [c_int, c_dp, c_dp, c_dp, c_dp, c_dp, c_int, c_dp, c_double, c_double, c_double, c_double,
                         c_int, c_int, c_int, c_int, c_dp, c_dp, c_dp],
    "wb_tile_shape": [c_int, c_int, c_dp, c_dp],
    "wb_tile_shapes": [c_int, c_int, c_dp, c_int],
    "wb_rate": [c_int, c_int, c_dp, c_dp, c_int, c_dp, c_dp, c_int, c_double, c_double, c_double, c_double, c_dp,
                c_int, c_dp],
    "wb_finalize_dt": [c_dp, c_int, c_double, c_double, c_double, c_double, c_dp, c_dp, c_dp, c_dp, c_int, c_dp],
    "wb_rate_levels": [c_int, c_int, c_dp, c_dp, c_int, c_dp, c_dp, c_int, c_double, c_double, c_double, c_double,
                       c_dp, c_int, c_dp, c_int, c_dp],
    "wb_finalize_dt_levels": [c_dp, c_int, c_double, c_double, c_double, c_double, c_dp, c_dp, c_int, c_dp, c_dp,
                              c_dp, c_int, c_dp],
    "wb_tag_features": [c_int, c_dp, c_dp, c_dp, c_dp, c_int, c_dp, c_double, c_double, c_double, c_double, c_dp,
                        c_dp, c_dp, c_dp],
    "wb_mlp_forward": [c_dp, ctypes.c_int64, c_dp, c_dp, c_dp],
    "wb_mlp_backward": [c_dp, c_dp, ctypes.c_int64, c_dp, ctypes.c_float, c_dp, c_dp, c_dp],
    "wb_mlp_adam": [c_dp, c_dp, c_dp, c_dp, c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                    c_int, ctypes.c_float, c_dp],
    "wb_rate_static": [c_int, c_int, c_dp, c_dp, c_int, c_dp, c_dp, c_int, c_double, c_double, c_double, c_double,
                       c_int, c_dp, c_dp],
    "wb_copy_ops": [c_int, c_dp, c_dp, c_dp, c_int, c_dp],
    "wb_interp_ops": [c_int, c_dp, c_dp, c_dp, c_int, c_dp],
    "wb_restrict_ops": [c_int, c_dp, c_dp, c_dp, c_int, c_dp],
    "wb_fill_ops": [c_int, c_dp, c_dp, c_dp, c_int, c_dp, c_int, c_dp],
    "wb_face_flux_ops": [c_int, c_dp, c_dp, c_dp, c_int, c_double, c_double, c_double, c_double, c_int, c_dp, c_dp],
    "wb_face_flux_ops_staged": [c_int, c_dp, c_dp, c_dp, c_int, c_int, c_double, c_double, c_double, c_double, c_int,
                                c_dp, c_dp, c_dp],
    "wb_face_flux_ops_physics": [c_int, c_dp, c_dp, c_dp, c_int, c_double, c_double, c_double, c_double, c_int,
                                 c_double, c_double, c_double, c_dp, c_dp],
    "wb_reflux_apply": [c_int, c_dp, c_dp, c_dp, c_int, c_dp, c_dp, c_dp],
    "wb_struct_sizes": [c_dp, c_int],
    "wb_run_program": [c_int, c_dp, c_dp, c_dp, c_dp, c_int, c_dp, c_dp, c_dp],
    "wb_current_tags": [c_int, c_int, c_dp, c_dp, c_dp, c_dp, c_int, c_dp, c_int, c_double, c_double, c_double,
                        c_double, c_dp, c_dp],
    "wb_prolong_ops": [c_int, c_dp, c_dp, c_dp, c_int, c_dp],
    "wb_kept_ops": [c_int, c_dp, c_dp, c_dp, c_dp, c_dp, c_int, c_dp],
    "wb_positivity_ops": [c_int, c_dp, c_dp, c_dp, c_int, c_double, c_double, c_double, c_double, c_dp],
}

#: Every symbol include/wellbalanced_b200.h declares.
EXPORTS = ("wb_version", "wb_last_error", *SIGNATURES)


class WBError(RuntimeError):
    """A failure reported by the C ABI (status and wb_last_error text)."""


#: The precision code of a float64 state advanced with float32 arithmetic
#: (``WB_MATH32_STATE64``): reconstruction, HLLD and CT in float32; the conserved and
#: potential updates (the conservation and div B accumulators), the Heun combine, the
#: pressure recovery and the face fields' potential differences in float64.
MATH32_STATE64 = 6432

#: Codes of the ``precision`` keyword: 32 (float32 state and arithmetic), 64 (float64),
#: "mixed" (float32 arithmetic on a float64 state).
PRECISIONS = {32: 32, 64: 64, "mixed": MATH32_STATE64, MATH32_STATE64: MATH32_STATE64}


def precision_code(value) -> int:
    """The C-ABI precision code of a ``precision`` keyword (32, 64 or "mixed")."""
    try:
        return PRECISIONS[value]
    except (KeyError, TypeError):
        raise ValueError(f"precision is 32, 64 or 'mixed', not {value!r}") from None


def state_bits(code) -> int:
    """Bits of a state value under a precision code (the mixed code keeps float64 state)."""
    return 32 if code == 32 else 64


def load():
    """The loaded library; raises if it is missing (build it first)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIBRARY.exists():
        raise RuntimeError(
            f"{LIBRARY.name} is not built: run `python -m wellbalanced_b200.build` "
            "(the CUDA path has no CPU fallback)"
        )
    lib = ctypes.CDLL(str(LIBRARY))
    lib.wb_version.restype = ctypes.c_char_p
    lib.wb_last_error.restype = ctypes.c_char_p
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    sizes = np.zeros(9, dtype=np.int64)
    status = lib.wb_struct_sizes(sizes.ctypes.data, 9)
    if status != 0:
        raise WBError(lib.wb_last_error().decode())
    expected = [d.itemsize for d in (PATCH, TILE, COPY_OP, INTERP_OP, RESTRICT_OP, FACE_FLUX_OP, REFLUX_OP,
                                     PROGRAM_SEGMENT)] + [ctypes.sizeof(ProgramParams)]
    if list(sizes) != expected:
        raise RuntimeError(f"struct layout mismatch between host and library: {list(sizes)} != {expected}")
    _lib = lib
    return lib


_FUNCTIONS = {}


def call(name, *args):
    """Call a C-ABI function; raise WBError on a negative status."""
    fn = _FUNCTIONS.get(name)
    if fn is None:
        fn = _FUNCTIONS[name] = getattr(load(), name)
    status = fn(*args)
    if status != 0:
        raise WBError(f"{name}: status {status}: {load().wb_last_error().decode()}")
    return status


def tile_shapes_2d(precision) -> list[tuple[int, int]]:
    """The (tx, ty) tile shapes the 2D stage kernel is built for, the default first."""
    return tile_shapes(2, precision)


def tile_shapes(ndim, precision) -> list[tuple[int, int]]:
    """The tile shapes the stage kernel of `ndim` is built for ((tx, ty) in 2D, (ty, tz) in
    3D), the default first."""
    lib = load()
    buf = (ctypes.c_int * 32)()
    count = lib.wb_tile_shapes(int(ndim), precision_code(precision), buf, 16)
    if count < 0:
        raise WBError(f"wb_tile_shapes: status {count}: {lib.wb_last_error().decode()}")
    return [(buf[2 * i], buf[2 * i + 1]) for i in range(min(count, 16))]


def version() -> str:
    return load().wb_version().decode()


# ---- struct mirrors (layout.cuh, halo.cuh) ------------------------------------------------
PATCH = np.dtype(
    {
        "names": ["off", "fstride", "pitch0", "pitch1", "n", "instance", "flags", "level", "dx", "bflux"],
        "formats": ["<i8", "<i8", "<i8", "<i8", ("<i4", 3), "<i4", "<i4", "<i4", ("<f8", 3), "<i8"],
        "offsets": [0, 8, 16, 24, 32, 44, 48, 52, 56, 80],
        "itemsize": 88,
    }
)
TILE = np.dtype({"names": ["patch", "x0", "y0", "z0"], "formats": ["<i4"] * 4, "itemsize": 16})
COPY_OP = np.dtype(
    {
        "names": ["dst", "src1", "src2", "field_lo", "field_hi", "negate", "n", "d", "s1", "m1", "s2", "m2", "w1", "w2"],
        "formats": ["<i4"] * 6 + [("<i4", 3)] * 6 + ["<f8", "<f8"],
        "offsets": [0, 4, 8, 12, 16, 20, 24, 36, 48, 60, 72, 84, 96, 104],
        "itemsize": 112,
    }
)
INTERP_OP = np.dtype(
    {
        "names": ["fine", "coarse", "field_lo", "field_hi", "node_mask", "ndim", "n", "d", "fine_lo", "coarse_lo"],
        "formats": ["<i4"] * 6 + [("<i4", 3)] * 4,
        "offsets": [0, 4, 8, 12, 16, 20, 24, 36, 48, 60],
        "itemsize": 72,
    }
)
RESTRICT_OP = np.dtype(
    {
        "names": ["fine", "coarse", "field_lo", "field_hi", "node_mask", "ndim", "n", "c", "f"],
        "formats": ["<i4"] * 6 + [("<i4", 3)] * 3,
        "offsets": [0, 4, 8, 12, 16, 20, 24, 36, 48],
        "itemsize": 60,
    }
)
FACE_FLUX_OP = np.dtype(
    {
        "names": ["coarse", "fine", "ndim", "axis", "t1", "t2", "coarse_plane", "fine_plane", "coarse_t0", "fine_t0",
                  "len", "width", "first", "pad1", "reg_off"],
        "formats": ["<i4"] * 8 + [("<i4", 2)] * 2 + ["<i4"] * 4 + ["<i8"],
        "offsets": [0, 4, 8, 12, 16, 20, 24, 28, 32, 40, 48, 52, 56, 60, 64],
        "itemsize": 72,
    }
)
REFLUX_OP = np.dtype(
    {
        "names": ["coarse", "len", "width", "ncomp", "c", "t1", "t2", "field", "sign", "dx", "reg_off"],
        "formats": ["<i4", "<i4", "<i4", "<i4", ("<i4", 3), "<i4", "<i4", ("<i4", 8), "<f8", "<f8", "<i8"],
        "offsets": [0, 4, 8, 12, 16, 28, 32, 36, 72, 80, 88],
        "itemsize": 96,
    }
)

# ---- op programs (include/wellbalanced_b200.h: wb_program_segment, wb_program_params) -----
PROGRAM_SEGMENT = np.dtype(
    {
        "names": ["kind", "pool", "phase", "count", "first", "pad", "ops", "aux"],
        "formats": ["<i4"] * 6 + ["<u8", "<u8"],
        "offsets": [0, 4, 8, 12, 16, 20, 24, 32],
        "itemsize": 40,
    }
)
#: WB_SEG_* codes
SEGMENT_KINDS = {"copy": 0, "interp": 1, "restrict": 2, "reflux": 3, "init_keys": 4, "rate": 5, "finalize_dt": 6,
                 "advance_time": 7}
#: WB_PROGRAM_MAX_SEGMENTS
PROGRAM_MAX_SEGMENTS = 64


class ProgramParams(ctypes.Structure):
    """wb_program_params."""

    _fields_ = [
        ("b0", c_double * 3),
        ("gamma", c_double),
        ("cfl", c_double),
        ("dt_eta", c_double),
        ("dt_kappa", c_double),
        ("ndim", ctypes.c_int32),
        ("ninstances", ctypes.c_int32),
        ("nlevels", ctypes.c_int32),
        ("advance", ctypes.c_int32),
        ("reg", c_dp),
        ("dt", c_dp),
        ("time", c_dp),
        ("end", c_dp),
        ("keys", c_dp),
        ("level_keys", c_dp),
        ("inv_dx2_sum", c_dp),
        ("inv_dx2_levels", c_dp),
    ]
