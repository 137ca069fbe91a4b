"""The ct_contact kernel on the device (drop-in for ``carafe.kernels.ct_contact``)."""

from wellbalanced_b200.kernels._dispatch import KERNELS, LIMITER_CODES

kernel = KERNELS["ct_contact"]

__all__ = ["kernel", "LIMITER_CODES"]
