"""Auxiliary functions (paces/aux/__init__.py).

expm_multiply_simple is the reference's scaling-and-squaring action of the matrix
exponential (paces/aux/_scipy/_expm_multiply.py:106-202, Al-Mohy and Higham 2011,
algorithm 3.2).  Here it runs on the device for the operator the reference applies it to,
the total Hamiltonian of a time evolution's current basis (`te.create_ham_mat()`, then
expm_multiply_simple(1j * te.ham_mat, v, t)): the trace shift and 1-norm come from the
device H rows, the stages and order from paces_b200.expm (code fragment 3.1), every term
runs in the library's cooperative kernel.  Other operators are not accepted: there is no
host fallback.
"""

__all__ = ["cupy_search", "helpers", "expm_multiply", "expm_multiply_simple"]

import torch

from . import cupy_search, helpers  # noqa: F401


def expm_multiply_simple(A, B, t=1.0, balance=False, return_dbg=False):
    """e^{t A} B for A = +-1j * ham_mat (the reference's call, paces/core/time_evolution.py:
    579-581); B is a vector (or the columns of a matrix) on the operator's basis.  With
    return_dbg also [converged, final_m, c1_plus_c2, term_ratio] of the (last) column."""
    from ..core.time_evolution import HamiltonianOperator
    if balance:
        raise NotImplementedError
    if not isinstance(A, HamiltonianOperator):
        raise TypeError("expm_multiply_simple runs on the device Hamiltonian of a TimeEvolution: pass "
                        "1j * te.ham_mat (after te.create_ham_mat())")
    if len(A.shape) != 2 or A.shape[0] != A.shape[1]:
        raise ValueError('expected A to be like a square matrix')
    if A.shape[1] != B.shape[0]:
        raise ValueError('the matrices A and B have incompatible shapes')
    if A.scale == 1j:
        tt = float(t)
    elif A.scale == -1j:
        tt = -float(t)
    else:
        raise NotImplementedError("the device series propagates exp(t * 1j H): A must be 1j or -1j times ham_mat")
    tr = A._live()
    eng = A.te.engine
    n = A.shape[0]
    Bt = torch.as_tensor(B).to(eng.device, eng.cdtype)
    cols = Bt.reshape(n, -1)
    out = torch.empty_like(cols)
    x = torch.zeros(max(tr.basis.cap, 1), dtype=eng.cdtype, device=eng.device)
    y = torch.empty_like(x)
    dbg = None
    for j in range(cols.shape[1]):
        x.zero_()
        x[:n] = cols[:, j]
        dbg = tr.expm_apply(x, y, tt)
        out[:, j] = y[:n]
    F = out.reshape(Bt.shape)
    return (F, dbg) if return_dbg else F


def expm_multiply(A, B, start=None, stop=None, num=None, endpoint=None, return_dbg=False):
    """e^{A} B when no time grid is given (start, stop, num and endpoint unset), as the
    reference's expm_multiply does then (paces/aux/_scipy/_expm_multiply.py:51-103); time
    grids are not offered."""
    if any(v is not None for v in (start, stop, num, endpoint)):
        raise NotImplementedError("expm_multiply over a time grid is not offered; call expm_multiply_simple "
                                  "per time point")
    return expm_multiply_simple(A, B, return_dbg=return_dbg)
