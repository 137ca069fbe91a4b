"""wellbalanced_b200: the ideal-MHD step of carafe (max-models/wellbalanced) on B200.

Public names (imported lazily, so ``wellbalanced_b200.problems`` needs no torch):

* `MHD2D`, `MHD3D` — the reference's solver API on the device (fused stage kernels);
* `PlainMHD2D`, `PlainMHD3D` — the reference's per-kernel dataflow on the device;
* `AMRHierarchy` — the patch hierarchy (patchwork's API as the solvers use it);
* `Batch` — many independent problems advanced by one set of launches;
* `kernels` — the reference's six block kernels (``wellbalanced_b200.kernels.<name>.kernel``).
"""

from __future__ import annotations

__all__ = ["AMRHierarchy", "Batch", "MHD2D", "MHD3D", "PlainMHD2D", "PlainMHD3D", "harris_sheets"]

_SOURCES = {
    "AMRHierarchy": "wellbalanced_b200.mesh",
    "MHD2D": "wellbalanced_b200.mhd",
    "harris_sheets": "wellbalanced_b200.mhd",
    "MHD3D": "wellbalanced_b200.mhd3d",
    "PlainMHD2D": "wellbalanced_b200.plain",
    "PlainMHD3D": "wellbalanced_b200.plain",
    "Batch": "wellbalanced_b200.batch",
}


def __getattr__(name):
    if name in _SOURCES:
        import importlib

        return getattr(importlib.import_module(_SOURCES[name]), name)
    raise AttributeError(name)
