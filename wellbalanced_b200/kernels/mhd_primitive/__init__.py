"""The mhd_primitive kernel on the device (drop-in for ``carafe.kernels.mhd_primitive``)."""

from wellbalanced_b200.kernels._dispatch import KERNELS, LIMITER_CODES

kernel = KERNELS["mhd_primitive"]

__all__ = ["kernel", "LIMITER_CODES"]
