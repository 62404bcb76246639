"""Search helpers (paces/aux/cupy_search.py) on device tensors.

The time step never calls these: its lookups are index maps produced by the device merge
and the merge-path remap.  They serve the host API (e.g. custom observables), operate on
the reference's uint32 row layout and run on the device with PyTorch.
"""

import torch

from .. import layout


def _lex_less(a, b):
    """Row-wise lexicographic a < b for int64 tensors of uint32 words."""
    res = torch.zeros(a.shape[0], dtype=torch.bool, device=a.device)
    decided = torch.zeros_like(res)
    for w in range(a.shape[1]):
        lt = a[:, w] < b[:, w]
        gt = a[:, w] > b[:, w]
        res |= ~decided & lt
        decided |= lt | gt
    return res


def searchsorted_full_binary(phonebook, findme, allow_escapes=False):
    """Lower bound of every row of `findme` in the sorted rows of `phonebook`
    (paces/aux/cupy_search.py:78-93).  Escapes return len(phonebook); with
    allow_escapes=False a missing row raises LookupError (the reference's kernel asserts)."""
    pb = layout.rows_i64(phonebook)
    q = layout.rows_i64(findme).to(pb.device)
    if pb.shape[1] != q.shape[1]:
        raise ValueError("Incompatible array shapes.")
    n, nq = pb.shape[0], q.shape[0]
    lo = torch.zeros(nq, dtype=torch.int64, device=pb.device)
    if nq == 0 or n == 0:
        return lo
    hi = torch.full((nq,), n, dtype=torch.int64, device=pb.device)
    while bool((lo < hi).any()):
        active = lo < hi
        mid = (lo + hi) // 2
        below = _lex_less(pb[mid.clamp(max=n - 1)], q)
        lo = torch.where(active & below, mid + 1, lo)
        hi = torch.where(active & ~below, mid, hi)
    if not allow_escapes:
        ok = lo < n
        hit = torch.zeros_like(ok)
        hit[ok] = (pb[lo[ok]] == q[ok]).all(dim=1)
        if not bool(hit.all()):
            raise LookupError("Target values not found in phonebook.")
    return lo


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
