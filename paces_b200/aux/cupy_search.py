"""Search helpers (paces/aux/cupy_search.py) on device tensors.

The time step never calls these: its lookups are index maps produced by the device merge
and the merge-path remap.  They serve the host API (e.g. custom observables), operate on
the reference's uint32 row layout; the search runs in libpaces_b200 (paces_rows_lower_bound).
"""

import torch


def searchsorted_full_binary(phonebook, findme, allow_escapes=False):
    """Lower bound of every row of `findme` in the sorted rows of `phonebook`
    (paces/aux/cupy_search.py:78-93), on the GPU by paces_rows_lower_bound.  Escapes return
    len(phonebook); with allow_escapes=False a missing row raises LookupError (the
    reference's kernel asserts)."""
    import ctypes
    from .. import _native as nat
    from .helpers import _device_rows
    pb, _ = _device_rows(phonebook)
    q, _ = _device_rows(findme)
    q = q.to(pb.device)
    if pb.dim() != 2 or q.dim() != 2 or pb.shape[1] != q.shape[1]:
        raise ValueError("Incompatible array shapes.")
    n, nq, w = int(pb.shape[0]), int(q.shape[0]), int(pb.shape[1])
    out = torch.zeros(max(nq, 1), dtype=torch.int64, device=pb.device)
    if nq == 0:
        return out[:0]
    missing = torch.zeros(1, dtype=torch.int32, device=pb.device)
    lib = nat.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream(pb.device).cuda_stream)
    nat.check(lib.paces_rows_lower_bound(ctypes.c_void_p(pb.data_ptr()), n, ctypes.c_void_p(q.data_ptr()), nq, w,
                                         1 if allow_escapes else 0, ctypes.c_void_p(out.data_ptr()),
                                         ctypes.c_void_p(missing.data_ptr()), stream), None, "rows_lower_bound")
    if not allow_escapes and int(missing.item()):
        raise LookupError("Target values not found in phonebook.")
    return out[:nq]


def calc_partition_lens(partition_by, uniquevals):
    """Length of the block of each value of `uniquevals` in the sorted `partition_by`
    (paces/aux/cupy_search.py:16-51)."""
    p = torch.as_tensor(partition_by).to(torch.int64)
    u = torch.as_tensor(uniquevals, device=p.device).to(torch.int64)
    return torch.searchsorted(p, u, right=True) - torch.searchsorted(p, u)


def jagged_to_regular(a, lens):
    """Pad the concatenated blocks of `a` into a regular (blocks x max_len) array."""
    lens = torch.as_tensor(lens)
    mask = lens[:, None] > torch.arange(int(lens.max()), device=lens.device)
    out = torch.zeros(mask.shape, dtype=a.dtype, device=a.device)
    out[mask] = a
    return out
