"""The reference's block kernels on the device: ``wellbalanced_b200.kernels.<name>.kernel``.

The same layout as ``carafe.kernels`` (``from carafe.kernels.mhd_sweep import kernel``
becomes ``from wellbalanced_b200.kernels.mhd_sweep import kernel``); each kernel takes
device float64 arrays and runs the CUDA version in ``libwb200.so``.
"""

from wellbalanced_b200.kernels._dispatch import KERNELS, LIMITER_CODES

__all__ = ["KERNELS", "LIMITER_CODES"]
