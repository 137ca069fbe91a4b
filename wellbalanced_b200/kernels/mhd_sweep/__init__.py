"""The mhd_sweep kernel on the device (drop-in for ``carafe.kernels.mhd_sweep``)."""

from wellbalanced_b200.kernels._dispatch import KERNELS, LIMITER_CODES

kernel = KERNELS["mhd_sweep"]

__all__ = ["kernel", "LIMITER_CODES"]
