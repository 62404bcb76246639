"""Auxiliary functions (paces/aux/__init__.py).

The SciPy-derived scaling-and-squaring `expm_multiply` of the reference is not part of
this implementation (only used with ExpmParams.use_scaling=True).
"""

__all__ = ["cupy_search", "helpers", "expm_multiply", "expm_multiply_simple"]

from . import cupy_search, helpers  # noqa: F401


def expm_multiply(*args, **kwargs):
    raise NotImplementedError("scaling-and-squaring expm_multiply (ExpmParams.use_scaling=True) is not "
                              "implemented; the truncated Taylor series runs on the device")


expm_multiply_simple = expm_multiply
