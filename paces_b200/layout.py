"""Host-side packing of basis states into the reference's row layout.

A state (pos, n_0, ..., n_{N-1}) is packed MSB-first into uint32 words, field i taking
ceil(log2(max_dim_i)) bits and possibly straddling two words
(paces/core/hamiltonian.py:140-160, :218-248).  The device keeps its own layout
(phonon fields only, uint64 words, blocked by position) and converts with
paces_keys_from_ref / paces_keys_to_ref; these helpers exist for the host API
(compress_ind_arr, initial bases, files written in the reference's .npy format).
"""

import numpy as np


def bitwidths_for(max_dims):
    """ceil(log2(max_dim)) per field (paces/core/hamiltonian.py:155), exact for integers."""
    out = []
    for d in max_dims:
        d = int(d)
        b = 0
        while (1 << b) < d:
            b += 1
        out.append(b)
    return np.array(out, dtype=np.int64)


def row_words(bitwidths):
    return int((int(np.sum(bitwidths)) + 31) // 32)


def pack_rows(raw, bitwidths):
    """(R, F) occupations -> (R, W) uint32 rows."""
    raw = np.asarray(raw)
    bw = np.asarray(bitwidths, dtype=np.int64)
    R = raw.shape[0]
    W = row_words(bw)
    rows = np.zeros((R, W), dtype=np.uint32)
    off = 0
    for i, b in enumerate(bw):
        if b == 0:
            continue
        col = raw[:, i].astype(np.uint64)
        if np.any(col >> np.uint64(b)):
            raise ValueError(f"value does not fit its {b}-bit field (field {i})")
        wi = off // 32
        end = off + int(b) - 32 * wi          # last bit of the field inside words (wi, wi+1)
        win = col << np.uint64(64 - end)
        rows[:, wi] |= (win >> np.uint64(32)).astype(np.uint32)
        if end > 32:
            rows[:, wi + 1] |= (win & np.uint64(0xFFFFFFFF)).astype(np.uint32)
        off += int(b)
    return rows


def unpack_rows(rows, bitwidths):
    """(R, W) uint32 rows -> (R, F) occupations."""
    rows = np.asarray(rows, dtype=np.uint32)
    bw = np.asarray(bitwidths, dtype=np.int64)
    R, W = rows.shape
    out = np.zeros((R, len(bw)), dtype=np.uint32)
    off = 0
    for i, b in enumerate(bw):
        if b == 0:
            continue
        wi = off // 32
        end = off + int(b) - 32 * wi
        win = rows[:, wi].astype(np.uint64) << np.uint64(32)
        if wi + 1 < W:
            win |= rows[:, wi + 1].astype(np.uint64)
        out[:, i] = ((win >> np.uint64(64 - end)) & np.uint64((1 << int(b)) - 1)).astype(np.uint32)
        off += int(b)
    return out


def sort_unique_rows(rows):
    """Lexicographic order with word 0 most significant, duplicates removed."""
    rows = np.asarray(rows, dtype=np.uint32)
    if rows.shape[0] == 0:
        return rows
    s = rows[np.lexsort(rows.T[::-1])]
    keep = np.ones(s.shape[0], dtype=bool)
    keep[1:] = np.any(s[1:] != s[:-1], axis=1)
    return s[keep]
