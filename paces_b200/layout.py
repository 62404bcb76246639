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


# ---- the same field arithmetic on device tensors (host API helpers, off the time step) ----

def field_table(bitwidths):
    """Per field: bit offset from the row's MSB, width, first word, end bit in its window."""
    bw = np.asarray(bitwidths, dtype=np.int64)
    off = np.concatenate([[0], np.cumsum(bw)[:-1]]).astype(np.int64)
    wi = off // 32
    n2 = off + bw - 32 * wi
    return off, bw, wi, n2


def rows_i64(rows):
    """uint32 rows (torch uint32/int32/int64 or numpy) -> int64 tensor with values < 2^32."""
    import torch
    if isinstance(rows, np.ndarray):
        rows = torch.from_numpy(np.ascontiguousarray(rows, dtype=np.uint32).view(np.int32))
    if rows.dtype == torch.uint32:
        rows = rows.view(torch.int32)
    if rows.dtype == torch.int32:
        return rows.to(torch.int64) & 0xFFFFFFFF
    return rows.to(torch.int64)


def rows_u32(r64):
    import torch
    return r64.to(torch.int32).view(torch.uint32) if r64.numel() else r64.to(torch.int32).view(torch.uint32)


def _window(r64, wi):
    import torch
    n, W = r64.shape
    pad = torch.cat([r64, torch.zeros((n, 1), dtype=r64.dtype, device=r64.device)], dim=1)
    if isinstance(wi, torch.Tensor):
        hi = torch.gather(pad, 1, wi.view(-1, 1)).view(-1)
        lo = torch.gather(pad, 1, (wi + 1).view(-1, 1)).view(-1)
    else:
        hi, lo = pad[:, wi], pad[:, wi + 1]
    return (hi << 32) | lo


def get_field_t(r64, table, idx):
    """Field `idx` (int, or one index per row) of every row."""
    import torch
    off, bw, wi, n2 = table
    if isinstance(idx, torch.Tensor):
        dev = r64.device
        wi_t = torch.as_tensor(wi, device=dev)[idx]
        n2_t = torch.as_tensor(n2, device=dev)[idx]
        bw_t = torch.as_tensor(bw, device=dev)[idx]
        win = _window(r64, wi_t)
        return (win >> (64 - n2_t)) & ((1 << bw_t) - 1)
    win = _window(r64, int(wi[idx]))
    return (win >> int(64 - n2[idx])) & ((1 << int(bw[idx])) - 1)


def add_field_t(r64, table, idx, delta):
    """New rows with field `idx` (int or per-row) increased by `delta` (carry/borrow across words)."""
    import torch
    off, bw, wi, n2 = table
    n, W = r64.shape
    dev = r64.device
    if isinstance(idx, torch.Tensor):
        wi_t = torch.as_tensor(wi, device=dev)[idx]
        n2_t = torch.as_tensor(n2, device=dev)[idx]
    else:
        wi_t = torch.full((n,), int(wi[idx]), dtype=torch.int64, device=dev)
        n2_t = torch.full((n,), int(n2[idx]), dtype=torch.int64, device=dev)
    win = _window(r64, wi_t) + (torch.as_tensor(delta, dtype=torch.int64, device=dev) << (64 - n2_t))
    out = torch.cat([r64, torch.zeros((n, 1), dtype=r64.dtype, device=dev)], dim=1)
    out.scatter_(1, wi_t.view(-1, 1), ((win >> 32) & 0xFFFFFFFF).view(-1, 1))
    lo_idx = (wi_t + 1).view(-1, 1)
    keep_lo = lo_idx < W
    lo_val = torch.where(keep_lo.view(-1), win & 0xFFFFFFFF, torch.gather(out, 1, lo_idx).view(-1))
    out.scatter_(1, lo_idx, lo_val.view(-1, 1))
    return out[:, :W]
