"""The drop-in's row helpers on the GPU (paces_rows_lower_bound, paces_rows_sort_unique):
searchsorted_full_binary and cupy_unique (paces/aux/cupy_search.py:78-93,
paces/aux/helpers.py:63-75) against the reference's own outputs (tests/golden/layout_*.npz)
and against NumPy's lexicographic sort on random rows of 1..16 words, bit for bit."""

import glob
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
LAYOUTS = sorted(glob.glob(os.path.join(GOLDEN, "layout_*.npz")))


def _np_unique_rows(a):
    if a.shape[0] == 0:
        return a
    order = np.lexsort(a.T[::-1])
    s = a[order]
    keep = np.ones(s.shape[0], dtype=bool)
    keep[1:] = np.any(s[1:] != s[:-1], axis=1)
    return s[keep]


@pytest.mark.parametrize("path", LAYOUTS, ids=os.path.basename)
def test_helpers_match_the_reference(path):
    from paces_b200.aux import cupy_search
    from paces_b200.aux.helpers import cupy_unique
    f = np.load(path)
    uniq = cupy_unique(f["unique_in"])                       # NumPy in, NumPy out
    assert isinstance(uniq, np.ndarray) and np.array_equal(uniq, f["unique_out"])
    dev = cupy_unique(torch.from_numpy(f["unique_in"].view(np.int32)).cuda().view(torch.uint32))
    assert dev.is_cuda and np.array_equal(dev.view(torch.int32).cpu().numpy().view(np.uint32), f["unique_out"])
    idx = cupy_search.searchsorted_full_binary(uniq, f["search_hit_q"])
    assert np.array_equal(idx.cpu().numpy(), f["search_hit_idx"].astype(np.int64))
    any_idx = cupy_search.searchsorted_full_binary(uniq, f["search_any_q"], allow_escapes=True).cpu().numpy()
    hit = f["search_any_hit"]
    assert np.array_equal(any_idx[hit], f["search_any_idx"][hit].astype(np.int64))
    if not hit.all():
        with pytest.raises(LookupError):
            cupy_search.searchsorted_full_binary(uniq, f["search_any_q"])


@pytest.mark.parametrize("words,n,hi", [(1, 1, 4), (1, 50000, 1 << 31), (2, 30000, 16), (3, 100000, 1 << 32),
                                        (5, 70000, 3), (8, 9000, 1 << 20), (9, 5000, 2), (16, 3000, 1 << 32)])
def test_random_rows(words, n, hi):
    from paces_b200.aux import cupy_search
    from paces_b200.aux.helpers import cupy_unique
    rng = np.random.default_rng(words * 1000 + n)
    a = rng.integers(0, hi, (n, words), dtype=np.uint64).astype(np.uint32)
    a = np.concatenate([a, a[rng.integers(0, n, n // 3)]])   # duplicates
    want = _np_unique_rows(a)
    got = cupy_unique(a)
    assert np.array_equal(got, want)
    q = np.concatenate([want[rng.integers(0, len(want), 2000)], rng.integers(0, hi, (2000, words),
                                                                              dtype=np.uint64).astype(np.uint32)])
    b = np.ascontiguousarray(want.astype(">u4")).view(f"S{4 * words}").ravel()
    qb = np.ascontiguousarray(q.astype(">u4")).view(f"S{4 * words}").ravel()
    expect = np.searchsorted(b, qb, side="left")
    got_idx = cupy_search.searchsorted_full_binary(want, q, allow_escapes=True).cpu().numpy()
    assert np.array_equal(got_idx, expect)
    hits = want[rng.integers(0, len(want), 500)]
    assert np.array_equal(cupy_search.searchsorted_full_binary(want, hits).cpu().numpy(),
                          np.searchsorted(b, np.ascontiguousarray(hits.astype(">u4")).view(f"S{4 * words}").ravel()))


def test_empty_inputs():
    from paces_b200.aux import cupy_search
    from paces_b200.aux.helpers import cupy_unique
    e = np.zeros((0, 3), dtype=np.uint32)
    assert cupy_unique(e).shape == (0, 3)
    assert cupy_search.searchsorted_full_binary(np.ones((4, 3), np.uint32), e).numel() == 0
    assert cupy_search.searchsorted_full_binary(e, np.ones((2, 3), np.uint32), allow_escapes=True).tolist() == [0, 0]
