"""`cupyx.scipy.sparse` -> `scipy.sparse` (test infrastructure only)."""

from scipy.sparse import coo_matrix, csr_matrix, diags, eye, identity, isspmatrix  # noqa: F401

from . import linalg  # noqa: F401
