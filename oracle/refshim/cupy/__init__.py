"""NumPy stand-in for the subset of CuPy that paces 1.2.0 uses.

TEST INFRASTRUCTURE ONLY.  This package exists so that the unmodified
reference (`paces/` of rkevk/paces) can be imported and run on a CPU host to
produce golden fixtures; it is never imported by the product path.

Two CuPy semantics that differ from NumPy are reproduced explicitly:

* CuPy's `argsort` on device arrays is stable; NumPy's default is not.  The
  reference ranks amplitudes with `cupy.abs(vector).argsort()`
  (paces/core/time_evolution.py:859-860), so `abs` here returns an ndarray
  subclass whose `argsort` uses `kind="stable"`.
* CuPy wraps out-of-range integer indices; NumPy raises.  The reference uses
  the escape results of `searchsorted_full_binary` as indices
  (paces/core/time_evolution.py:785, paces/core/hamiltonian.py:368).  The
  search kernel stand-in clamps escapes to len-1, which yields the same
  equality masks (the clamped row is strictly smaller than the query).

The RawKernel sources of paces (paces/models/_kernels/_holstein_kernels.py:96-255,
paces/aux/cupy_search.py:149-228) are dispatched by kernel name to vectorised
NumPy restatements in `_kernels.py`.
"""

import numpy as _np
from numpy import *  # noqa: F401,F403

from . import cuda  # noqa: F401
from ._kernels import RawKernel, ElementwiseKernel  # noqa: F401

ndarray = _np.ndarray
random = _np.random
linalg = _np.linalg
inf = _np.inf
bool_ = _np.bool_


class _StableSortArray(_np.ndarray):
    """ndarray whose argsort is stable, like CuPy's (thrust stable sort)."""

    def argsort(self, axis=-1, kind=None, order=None):  # noqa: D401
        return _np.asarray(self).argsort(axis=axis, kind="stable")


def abs(x, *args, **kwargs):  # noqa: A001
    return _np.abs(x, *args, **kwargs).view(_StableSortArray)


def argsort(a, axis=-1, kind=None, order=None):
    return _np.argsort(_np.asarray(a), axis=axis, kind="stable")


def asnumpy(a, *args, **kwargs):
    return _np.asarray(a)


def array(obj, *args, **kwargs):
    return _np.array(_np.asarray(obj) if isinstance(obj, _StableSortArray) else obj, *args,
                     **kwargs)


class _MemoryPool:
    def __init__(self, *args, **kwargs):
        pass

    def used_bytes(self):
        return 0

    def total_bytes(self):
        return 0

    def free_all_blocks(self):
        pass

    def set_limit(self, size=None):
        pass

    def malloc(self, size):
        raise NotImplementedError("the CPU stand-in has no device memory")


_default_pool = _MemoryPool()


def get_default_memory_pool():
    return _default_pool


def adapt_reference(paces_pkg):
    """Reproduce CuPy's index wrap-around for the one reference helper that needs it.

    `_check_if_trivial` (paces/aux/cupy_search.py:102-111) answers lookups in a
    one-row phonebook with 0/1; callers then index the phonebook with that
    value (paces/core/time_evolution.py:785).  CuPy wraps index 1 to 0 for a
    length-1 axis, NumPy raises.  The wrapped value is 0 in every case, so the
    stand-in returns zeros for escape-allowed calls.  The reference source is
    not modified; only the in-memory function object is wrapped.
    """
    cs = paces_pkg.aux.cupy_search
    original = cs._check_if_trivial

    def _check_if_trivial(phonebook, findme, allow_escapes):
        res = original(phonebook, findme, allow_escapes)
        if res is not None and phonebook.shape[0] == 1:
            res = _np.zeros_like(res)
        return res

    cs._check_if_trivial = _check_if_trivial
