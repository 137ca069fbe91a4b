"""The C-ABI library: it builds, loads and exports every symbol the header declares (CPU).

No compute call is made here (no GPU in this check); the struct layouts the Python host
mirrors must equal the library's.
"""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np

from wellbalanced_b200 import _lib, build

HEADER = Path(__file__).resolve().parents[1] / "include" / "wellbalanced_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(wb_[a-z0-9_]+)\s*\(", text)))


def test_library_builds_and_loads():
    path = build.build()
    assert path.exists()
    lib = _lib.load()
    assert b"wellbalanced_b200" in lib.wb_version()


def test_every_declared_symbol_is_exported():
    build.build()
    raw = ctypes.CDLL(str(_lib.LIBRARY))
    symbols = declared_symbols()
    assert len(symbols) >= 20
    for name in symbols:
        assert hasattr(raw, name), name
    assert set(symbols) == set(_lib.EXPORTS)


def test_struct_layouts_match_the_library():
    lib = _lib.load()
    sizes = np.zeros(7, dtype=np.int64)
    assert lib.wb_struct_sizes(sizes.ctypes.data, 7) == 0
    assert list(sizes) == [88, 16, 112, 72, 60, 72, 96]


def test_bad_arguments_are_reported_without_a_device():
    lib = _lib.load()
    status = lib.wb_mhd_sweep(None, None, 0, 0, 5.0 / 3.0, 13, 9, None, None)
    assert status == -1
    assert b"NULL" in lib.wb_last_error()
    status = lib.wb_stage2d(16, None, None, None, None, None, 0, None, 1.4, 0.0, 0.0, 0, None, None, None)
    assert status == -1
    assert b"precision" in lib.wb_last_error()
    # the fused level fill: bad precision, NULL pool, a negative count
    status = lib.wb_fill_ops(16, None, None, None, 0, None, 0, None)
    assert status == -1 and b"precision" in lib.wb_last_error()
    status = lib.wb_fill_ops(32, None, None, None, 1, None, 0, None)
    assert status == -1 and b"NULL" in lib.wb_last_error()
