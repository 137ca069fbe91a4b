"""The mhd_conductive kernel on the device (drop-in for ``carafe.kernels.mhd_conductive``)."""

from wellbalanced_b200.kernels._dispatch import KERNELS, LIMITER_CODES

kernel = KERNELS["mhd_conductive"]

__all__ = ["kernel", "LIMITER_CODES"]
