"""`cupyx.scipy.sparse.linalg` -> `scipy.sparse.linalg` (test infrastructure only)."""

from scipy.sparse.linalg import aslinearoperator, norm  # noqa: F401
