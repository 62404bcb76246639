"""Vectorised NumPy restatements of the RawKernel sources shipped with paces 1.2.0.

TEST INFRASTRUCTURE ONLY (CPU stand-in for CuPy, see the package docstring).

Each kernel name used by the reference is mapped to a NumPy function with the
same argument list and the same in-place / result-array semantics:

* add_pte_kernel / rem_pte_kernel / get_occ_pte_kernel / sum_occ_pte_kernel /
  calc_bath_n_b_kernel (and their `_64` twins):
  paces/models/_kernels/_holstein_kernels.py:96-255.
* full_binary / full_binary_noesc (and `_64`): paces/aux/cupy_search.py:149-228.

The field arithmetic uses a 64-bit window over words (word_i, word_i+1) of a
row; adding or subtracting 1 at the field's last bit in that window is the
same carry/borrow rule the CUDA source applies across the word boundary.
"""

import numpy as np


def _pos_of_rows(bs, bit_offset):
    """Exciton position: the leading `bit_offset[0]` bits of word 0 (_holstein_kernels.py:106)."""
    return (bs[:, 0] >> np.uint32(32 - int(bit_offset[0]))).astype(np.int64)


def _window(bs, rows, wi):
    nwords = bs.shape[1]
    hi = bs[rows, wi].astype(np.uint64)
    has_lo = wi + 1 < nwords
    lo = np.zeros_like(hi)
    lo[has_lo] = bs[rows[has_lo], wi[has_lo] + 1]
    return (hi << np.uint64(32)) | lo, has_lo


def _store_window(bs, rows, wi, val, has_lo):
    bs[rows, wi] = (val >> np.uint64(32)).astype(np.uint32)
    bs[rows[has_lo], wi[has_lo] + 1] = (val[has_lo] & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def _field(bs, rows, wi, n2, width):
    val, _ = _window(bs, rows, wi)
    sh = (64 - n2).astype(np.uint64)
    mask = ((np.uint64(1) << width.astype(np.uint64)) - np.uint64(1))
    return ((val >> sh) & mask).astype(np.uint32)


def _widths(bit_offset, word_i, num2bits):
    return (num2bits.astype(np.int64) - (bit_offset.astype(np.int64) - 32 * word_i.astype(np.int64)))


def _add_rem(bs, bit_offset, word_i, num2bits, rownum, rowlen, sign):
    rows = np.arange(int(rownum))
    pos = _pos_of_rows(bs, bit_offset)
    wi = word_i.astype(np.int64)[pos]
    n2 = num2bits.astype(np.int64)[pos]
    val, has_lo = _window(bs, rows, wi)
    inc = np.uint64(1) << (64 - n2).astype(np.uint64)
    val = val + inc if sign > 0 else val - inc
    _store_window(bs, rows, wi, val, has_lo)


def add_pte_kernel(bs, bit_offset, word_i, num2bits, rownum, rowlen):
    _add_rem(bs, bit_offset, word_i, num2bits, rownum, rowlen, +1)


def rem_pte_kernel(bs, bit_offset, word_i, num2bits, rownum, rowlen):
    _add_rem(bs, bit_offset, word_i, num2bits, rownum, rowlen, -1)


def get_occ_pte_kernel(bs, bit_offset, word_i, num2bits, rownum, rowlen, result):
    rows = np.arange(int(rownum))
    pos = _pos_of_rows(bs, bit_offset)
    width = _widths(bit_offset, word_i, num2bits)
    result[:] = _field(bs, rows, word_i.astype(np.int64)[pos], num2bits.astype(np.int64)[pos],
                       width[pos])


def _site_occ(bs, bit_offset, word_i, num2bits, site):
    rows = np.arange(bs.shape[0])
    wi = np.full(rows.shape, int(word_i[site]), dtype=np.int64)
    n2 = np.full(rows.shape, int(num2bits[site]), dtype=np.int64)
    width = _widths(bit_offset, word_i, num2bits)
    return _field(bs, rows, wi, n2, np.full(rows.shape, int(width[site]), dtype=np.int64))


def sum_occ_pte_kernel(bs, bit_offset, word_i, num2bits, rownum, rowlen, result, omega, numsites):
    # sequential accumulation over sites in float64, as in _holstein_kernels.py:195-207
    for site in range(int(numsites)):
        result += _site_occ(bs, bit_offset, word_i, num2bits, site) * omega[site]


def calc_bath_n_b_kernel(bs, bit_offset, word_i, num2bits, rownum, rowlen, result, weights,
                         numsites):
    for site in range(int(numsites)):
        result[site] += (_site_occ(bs, bit_offset, word_i, num2bits, site) * weights).sum()


def _as_bytes_rows(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    be = a.astype(">u4")
    return np.ascontiguousarray(be).view(f"S{4 * a.shape[1]}").reshape(a.shape[0])


def _full_binary(findme, phonebook, phonebooknum, findmenum, rowlen, result, noesc):
    pb = _as_bytes_rows(phonebook[: int(phonebooknum)])
    q = _as_bytes_rows(findme[: int(findmenum)])
    left = np.searchsorted(pb, q, side="left")
    if noesc:
        hit = left < len(pb)
        hit[hit] = pb[left[hit]] == q[hit]
        if not hit.all():
            raise RuntimeError("full_binary_noesc: a looked-up row is not in the phonebook "
                               "(the CUDA kernel asserts here)")
    else:
        # CuPy wraps out-of-range indices; clamp so NumPy indexing behaves the same way.
        left = np.minimum(left, len(pb) - 1)
    result[: int(findmenum)] = left.astype(np.uint32)


def full_binary(findme, phonebook, phonebooknum, findmenum, rowlen, result):
    _full_binary(findme, phonebook, phonebooknum, findmenum, rowlen, result, False)


def full_binary_noesc(findme, phonebook, phonebooknum, findmenum, rowlen, result):
    _full_binary(findme, phonebook, phonebooknum, findmenum, rowlen, result, True)


_DISPATCH = {
    "add_pte_kernel": add_pte_kernel,
    "rem_pte_kernel": rem_pte_kernel,
    "get_occ_pte_kernel": get_occ_pte_kernel,
    "sum_occ_pte_kernel": sum_occ_pte_kernel,
    "calc_bath_n_b_kernel": calc_bath_n_b_kernel,
    "full_binary": full_binary,
    "full_binary_noesc": full_binary_noesc,
}


class RawKernel:
    def __init__(self, code, name, options=(), backend="nvrtc", **kwargs):
        base = name[:-3] if name.endswith("_64") else name
        if base not in _DISPATCH:
            raise NotImplementedError(f"no CPU stand-in for kernel {name}")
        self.name = name
        self._fn = _DISPATCH[base]

    def __call__(self, grid, block, args, **kwargs):
        self._fn(*args)


class ElementwiseKernel:
    """The legacy uint8 search kernels are defined at import time but never reached."""

    def __init__(self, *args, **kwargs):
        self.args = args

    def __call__(self, *args, **kwargs):
        raise NotImplementedError("legacy uint8 search kernels have no CPU stand-in")
