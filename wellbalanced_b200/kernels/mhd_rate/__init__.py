"""The mhd_rate kernel on the device (drop-in for ``carafe.kernels.mhd_rate``)."""

from wellbalanced_b200.kernels._dispatch import KERNELS, LIMITER_CODES

kernel = KERNELS["mhd_rate"]

__all__ = ["kernel", "LIMITER_CODES"]
