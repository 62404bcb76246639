"""`cupyx.scipy.linalg` -> `scipy.linalg` (test infrastructure only)."""

from scipy.linalg import expm  # noqa: F401
