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

Only the branch of fragment 3.1 that condition (3.13) selects for t ||A - mu I||_1 below
about 63 is provided -- the branch that needs 1-norm estimates of powers of A (the
randomised estimator of Higham and Tisseur) is not built and raises.  For the Holstein
chain at the time steps paces uses (dt = 0.05, ||H - mu I||_1 of a few tens) the
condition holds by a wide margin.
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


def choose(t_a_1_norm, n0=1):
    """(m, s) of fragment 3.1 for t ||A - mu I||_1; (0, 1) when it is 0."""
    if t_a_1_norm == 0:
        return 0, 1
    if not condition_3_13(t_a_1_norm, n0):
        raise NotImplementedError(
            f"t * ||A - mu I||_1 = {t_a_1_norm:.3g} needs 1-norm estimates of powers of A "
            "(fragment 3.1, equation 3.11), which are not built; use smaller time steps")
    best_m = best_s = None
    for m, theta in THETA.items():
        s = int(math.ceil(t_a_1_norm / theta))
        if best_m is None or m * s < best_m * best_s:
            best_m, best_s = m, s
    return best_m, best_s
