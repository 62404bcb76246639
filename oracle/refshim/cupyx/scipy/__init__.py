"""`cupyx.scipy` stand-in (test infrastructure only)."""

from . import sparse, linalg  # noqa: F401
