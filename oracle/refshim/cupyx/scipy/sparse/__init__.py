"""`cupyx.scipy.sparse` -> `scipy.sparse` (test infrastructure only).

One behaviour differs between the two and is reproduced here: CuPy's sparse
`sum(axis=...)` returns an ndarray (shape (n, 1) for axis=1), SciPy's returns an
`np.matrix`, whose `flatten()` is (1, n) and cannot be added in place to a 1-D array
(the reference's total_ham_ones, paces/core/time_evolution.py:403-420, does exactly
that).  The reference builds its term matrices as `coo_matrix(...).tocsr()`
(time_evolution.py:365-372), so the two classes below carry the CuPy behaviour."""

import numpy as _np
from scipy import sparse as _sp
from scipy.sparse import diags, eye, identity, isspmatrix  # noqa: F401

from . import linalg  # noqa: F401


class csr_matrix(_sp.csr_matrix):
    def sum(self, axis=None, dtype=None, out=None):
        res = super().sum(axis=axis, dtype=dtype, out=out)
        return res if axis is None else _np.asarray(res)


class coo_matrix(_sp.coo_matrix):
    def tocsr(self, copy=False):
        return csr_matrix(super().tocsr(copy=copy))
