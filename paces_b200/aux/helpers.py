"""Helper functions (paces/aux/helpers.py): decorators of the model API and small utilities."""

import numpy
import torch

from ..config import SEARCHSORTED_TIMING_LEVEL
from .. import layout


def cartesian_product(*arrays):
    """All combinations of the given 1D arrays as rows (paces/aux/helpers.py:10-17)."""
    grids = numpy.meshgrid(*[numpy.asarray(a) for a in arrays], indexing="ij")
    dtype = numpy.result_type(*arrays)
    return numpy.stack([g.reshape(-1) for g in grids], axis=1).astype(dtype, copy=False)


def print_searchsorted_timing(verb, delta_t, size1, size2):
    if verb > SEARCHSORTED_TIMING_LEVEL:
        print("This application of searchsorted took"
              f" {delta_t*1000} ms (arg sizes {size1}, {size2}).")


def obs_attrs(**kwargs):
    """Attach `fname` and `header` to an observable method (paces/aux/helpers.py:27-42)."""
    def wrapper(f):
        for attr, val in kwargs.items():
            setattr(f, attr, val)
        return f
    return wrapper


def debug_lister(dbg_list):
    """Name the debug outputs of a generate_mel_xxx method (paces/aux/helpers.py:45-55)."""
    def wrapper(f):
        f.dbg_list = dbg_list
        return f
    return wrapper


def flatten_dbg_dict(d):
    return [x for lst in [d[k] for k in d] for x in lst]


def cupy_unique(array):
    """Sorted unique rows of a 2D uint32 array (paces/aux/helpers.py:63-75).

    Returns the same type as the input (torch device tensor or NumPy array).  Used by the
    host API only; the time step deduplicates inside the device merge.
    """
    if len(array.shape) != 2:
        raise ValueError("Input array must be 2D.")
    if isinstance(array, torch.Tensor):
        host = layout.rows_i64(array.cpu()).numpy().astype(numpy.uint32)
        out = layout.sort_unique_rows(host)
        return torch.from_numpy(out.view(numpy.int32)).to(array.device).view(torch.uint32)
    return layout.sort_unique_rows(numpy.asarray(array))
