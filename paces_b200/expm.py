"""Parameters of the scaling-and-squaring propagation (ExpmParams(use_scaling=True)).

The reference propagates with expm_multiply_simple(1j * H, psi, t=dt)
(paces/core/time_evolution.py:579-581; paces/aux/_scipy/_expm_multiply.py:106-160), the
algorithm of Al-Mohy and Higham, "Computing the action of the matrix exponential, with an
application to exponential integrators" (SIAM J. Sci. Comput. 33, 2011): with
A = 1j * H, mu = trace(A) / n and the 1-norm of A - mu I, code fragment 3.1 picks the
number of stages s and the order bound m that minimise m * s subject to the bounds
theta_m of the paper's tables; every stage then runs the truncated Taylor series.  The
device does the norms (`paces_hnorms`) and the series (`paces_expm_scaled`); this module
is the small host-side choice between them.

When condition (3.13) fails (t ||A - mu I||_1 above about 63: large time steps), fragment
3.1 chooses by equation (3.11) from estimates of ||A^p||_1 (p = 2 .. p_max + 1), made by
the block 1-norm estimator of Higham and Tisseur ("A block algorithm for matrix 1-norm
estimation", SIAM J. Matrix Anal. Appl. 21, 2000, Algorithm 2.4; the reference vendors
SciPy's version, paces/aux/_scipy/_onenormest.py:11-345) with t = ell = 2 columns and at
most 5 iterations.  Here every product with A runs as the device H row kernel
(`paces_apply_h`) on the estimator's columns.  The estimator draws random +-1 columns;
the reference draws them from CuPy's generator, this module from a seeded torch
generator, so that branch picks the same (m, s) only where both estimates are exact --
parity unpinned for it, and the propagated state is checked against exact propagation
instead.  For the Holstein chain at the time steps paces uses (dt = 0.05,
||H - mu I||_1 of a few tens) condition (3.13) holds by a wide margin.
"""

from __future__ import annotations

import math

# theta_m: the largest t ||A||_1 for which m Taylor terms reach the double-precision
# tolerance (Al-Mohy and Higham 2011, table 3.1; m <= 30 from Higham, Functions of
# Matrices, table A.3).
THETA = {
    1: 2.29e-16, 2: 2.58e-8, 3: 1.39e-5, 4: 3.40e-4, 5: 2.40e-3, 6: 9.07e-3, 7: 2.38e-2, 8: 5.00e-2,
    9: 8.96e-2, 10: 1.44e-1, 11: 2.14e-1, 12: 3.00e-1, 13: 4.00e-1, 14: 5.14e-1, 15: 6.41e-1,
    16: 7.81e-1, 17: 9.31e-1, 18: 1.09, 19: 1.26, 20: 1.44, 21: 1.62, 22: 1.82, 23: 2.01, 24: 2.22,
    25: 2.43, 26: 2.64, 27: 2.86, 28: 3.08, 29: 3.31, 30: 3.54, 35: 4.7, 40: 6.0, 45: 7.2, 50: 8.5,
    55: 9.9,
}
M_MAX = 55
ELL = 2
TOL = 2.0 ** -53


def p_max(m_max=M_MAX):
    """Largest p with p (p - 1) <= m_max + 1."""
    p = int(math.floor(math.sqrt(m_max)))
    while (p + 1) * p <= m_max + 1:
        p += 1
    while p * (p - 1) > m_max + 1:
        p -= 1
    return p


def condition_3_13(a_1_norm, n0=1, m_max=M_MAX, ell=ELL):
    """Whether the 1-norm alone bounds the cost (condition 3.13 of the paper)."""
    pm = p_max(m_max)
    return a_1_norm <= 2 * ell * pm * (pm + 3) * THETA[m_max] / float(n0 * m_max)


def choose(t_a_1_norm, n0=1, d=None):
    """(m, s) of fragment 3.1 for t ||A - mu I||_1; (0, 1) when it is 0.  Where condition
    (3.13) fails, d(p) must give the estimate of ||(t A)^p||_1^(1/p) (equation 3.11)."""
    if t_a_1_norm == 0:
        return 0, 1
    best_m = best_s = None
    if condition_3_13(t_a_1_norm, n0):
        for m, theta in THETA.items():
            s = int(math.ceil(t_a_1_norm / theta))
            if best_m is None or m * s < best_m * best_s:
                best_m, best_s = m, s
        return best_m, best_s
    if d is None:
        raise NotImplementedError(f"t * ||A - mu I||_1 = {t_a_1_norm:.3g} needs 1-norm estimates of powers of A")
    cache = {}

    def dp(p):
        if p not in cache:
            cache[p] = d(p)
        return cache[p]

    for p in range(2, p_max() + 1):
        for m in range(p * (p - 1) - 1, M_MAX + 1):
            if m in THETA:
                s = int(math.ceil(max(dp(p), dp(p + 1)) / THETA[m]))   # alpha_p, equation (3.10)
                if best_m is None or m * s < best_m * best_s:
                    best_m, best_s = m, s
    return best_m, max(best_s, 1)


def onenormest(matmat, rmatmat, n, t=2, itmax=5, generator=None, device=None):
    """Lower bound of ||B||_1 for the n x n operator B given by matmat(X) = B X and
    rmatmat(X) = B^H X on complex [n, t] tensors (Higham and Tisseur 2000, Algorithm 2.4, in
    the form of the reference's _onenormest_core, _onenormest.py:202-345)."""
    import torch
    dev = device
    if t >= n:   # small operator: the exact norm from its columns
        cols = torch.eye(n, dtype=torch.complex128, device=dev)
        A = matmat(cols)
        return float(A.abs().sum(dim=0).max())

    def rand_pm1(shape):
        return (torch.randint(0, 2, shape, generator=generator, device=dev) * 2 - 1).to(torch.complex128)

    def parallel(v, w):   # columns equal up to sign (entries of unit modulus)
        return bool(torch.dot(v, w).real == n)

    def needs_resampling(i, X, Y=None):
        if any(parallel(X[:, i], X[:, j]) for j in range(i)):
            return True
        return Y is not None and any(parallel(X[:, i], Y[:, j]) for j in range(Y.shape[1]))

    X = torch.ones((n, t), dtype=torch.complex128, device=dev)
    for i in range(1, t):
        X[:, i] = rand_pm1((n,))
    for i in range(t):
        while needs_resampling(i, X):
            X[:, i] = rand_pm1((n,))
    X /= float(n)
    ind_hist = torch.zeros(0, dtype=torch.int64, device=dev)
    est_old = 0.0
    S = torch.zeros((n, t), dtype=torch.complex128, device=dev)
    k = 1
    ind = None
    ind_best = None
    while True:
        Y = matmat(X)
        mags = Y.abs().sum(dim=0)
        est = float(mags.max())
        best_j = int(mags.argmax())
        if est > est_old or k == 2:
            if k >= 2:
                ind_best = int(ind[best_j])
        if k >= 2 and est <= est_old:
            est = est_old
            break
        est_old = est
        S_old = S
        if k > itmax:
            break
        S = Y.clone()
        S[S == 0] = 1
        S = S / S.abs()
        if all(any(parallel(S[:, a], S_old[:, b]) for b in range(t)) for a in range(t)):
            break
        for i in range(t):
            while needs_resampling(i, S, S_old):
                S[:, i] = rand_pm1((n,))
        Z = rmatmat(S)
        h = Z.abs().max(dim=1).values
        if k >= 2 and float(h.max()) == float(h[ind_best]):
            break
        ind = torch.argsort(h, descending=True, stable=True)[: t + len(ind_hist)]
        if t > 1:
            seen = torch.isin(ind, ind_hist)
            if bool(seen[:t].all()):
                break
            ind = torch.cat((ind[~seen], ind[seen]))
        X = torch.zeros((n, t), dtype=torch.complex128, device=dev)
        for j in range(t):
            X[int(ind[j]), j] = 1
        new_ind = ind[:t][~torch.isin(ind[:t], ind_hist)]
        ind_hist = torch.cat((ind_hist, new_ind))
        k += 1
    return est
