"""SciPy stand-in for the subset of `cupyx` that paces 1.2.0 uses (test infrastructure only)."""

from . import scipy  # noqa: F401
