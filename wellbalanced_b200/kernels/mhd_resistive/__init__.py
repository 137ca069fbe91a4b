"""The mhd_resistive kernel on the device (drop-in for ``carafe.kernels.mhd_resistive``)."""

from wellbalanced_b200.kernels._dispatch import KERNELS, LIMITER_CODES

kernel = KERNELS["mhd_resistive"]

__all__ = ["kernel", "LIMITER_CODES"]
