"""Host side of the scaling-and-squaring propagation (paces_b200.expm): the choice of Taylor
order and stage count (code fragment 3.1 of Al-Mohy and Higham; the reference vendors it
in paces/aux/_scipy/_expm_multiply.py:395-450) against the reference's own choices on
synthetic norm data (tests/golden/fragment31.npz), and the block 1-norm estimator
(Higham and Tisseur, Algorithm 2.4) against exact norms of small dense operators."""

import os

import numpy as np
import pytest
import torch

from paces_b200 import expm

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_fragment_3_1_matches_the_reference():
    f = np.load(os.path.join(GOLDEN, "fragment31.npz"))
    estimated = 0
    for case, (m_ref, s_ref) in zip(f["cases"], f["choice"]):
        a1 = float(case[0])
        d = {p: float(case[p - 1]) for p in range(2, 11)}
        if not expm.condition_3_13(a1):
            estimated += 1
        assert expm.choose(a1, d=lambda p: d[p]) == (int(m_ref), int(s_ref)), a1
    assert estimated >= 8   # the equation (3.11) branch is exercised


def test_choice_without_estimates_raises_only_where_needed():
    assert expm.choose(10.0) == expm.choose(10.0, d=lambda p: 1.0)
    with pytest.raises(NotImplementedError):
        expm.choose(500.0)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_onenormest_bounds_the_exact_norm(seed):
    rng = np.random.default_rng(seed)
    n = 60
    M = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    M[rng.random((n, n)) < 0.8] = 0
    for p in (1, 2, 3):
        Mp = torch.as_tensor(np.linalg.matrix_power(M, p))
        exact = float(Mp.abs().sum(dim=0).max())
        gen = torch.Generator().manual_seed(seed)
        est = expm.onenormest(lambda X: Mp @ X, lambda X: Mp.conj().T @ X, n, generator=gen, device="cpu")
        assert est <= exact * (1 + 1e-12)
        assert est >= exact / 3
    small = torch.as_tensor(M[:2, :2])
    assert expm.onenormest(lambda X: small @ X, lambda X: small.conj().T @ X, 2, device="cpu") == pytest.approx(
        float(small.abs().sum(dim=0).max()))
