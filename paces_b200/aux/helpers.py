"""Helper functions (paces/aux/helpers.py): decorators of the model API and small utilities."""

import numpy
import torch

from ..config import SEARCHSORTED_TIMING_LEVEL


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


def _device_rows(array):
    """The rows as a contiguous int32 CUDA tensor, and a function that returns a result in the
    input's type (torch tensor on its device, or a NumPy uint32 array)."""
    if isinstance(array, torch.Tensor):
        dev = array.device if array.is_cuda else torch.device("cuda", torch.cuda.current_device())
        if array.dtype in (torch.int32, torch.uint32):
            t = array.to(dev).contiguous().view(torch.int32)
        else:
            t = array.to(dev, torch.int64).to(torch.int32).contiguous()
        if array.dtype == torch.uint32:
            back = lambda x: x.view(torch.uint32)  # noqa: E731
        elif array.dtype == torch.int32:
            back = lambda x: x  # noqa: E731
        else:
            back = lambda x: x.to(torch.int64) & 0xFFFFFFFF  # noqa: E731
        if not array.is_cuda:
            return t, (lambda x: back(x).cpu())
        return t, back
    a = numpy.ascontiguousarray(numpy.asarray(array).astype(numpy.uint32, copy=False))
    t = torch.from_numpy(a.view(numpy.int32)).to("cuda")
    return t, (lambda x: x.cpu().numpy().view(numpy.uint32))


def cupy_unique(array):
    """Sorted unique rows of a 2D uint32 array (paces/aux/helpers.py:63-75: a lexsort and an
    adjacent-row dedup), computed on the GPU by paces_rows_sort_unique.  Returns the same type
    as the input (torch tensor on its device, or a NumPy array)."""
    import ctypes
    from .. import _native as nat
    if len(array.shape) != 2:
        raise ValueError("Input array must be 2D.")
    rows, back = _device_rows(array)
    n, w = int(rows.shape[0]), int(rows.shape[1])
    lib = nat.load()
    out = torch.empty((max(n, 1), w), dtype=torch.int32, device=rows.device)
    cnt = torch.zeros(1, dtype=torch.int64, device=rows.device)
    ws = torch.empty(max(int(lib.paces_rows_sort_bytes(n)), 1), dtype=torch.uint8, device=rows.device)
    stream = ctypes.c_void_p(torch.cuda.current_stream(rows.device).cuda_stream)
    nat.check(lib.paces_rows_sort_unique(ctypes.c_void_p(rows.data_ptr()), n, w, ctypes.c_void_p(out.data_ptr()),
                                         ctypes.c_void_p(cnt.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(),
                                         stream), None, "rows_sort_unique")
    return back(out[: int(cnt.item())])
