"""The scaling-and-squaring propagation (ExpmParams(use_scaling=True)) through the
drop-in API against the reference's own run (tests/golden/scaled_n8c16.npz): basis
sizes, term counts, observables at every step and the final basis and amplitudes."""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_scaled_propagation_matches_the_reference(tmp_path):
    import torch
    from paces.config import devices
    from paces.core.time_evolution import CoeffSaveParams, ExpmParams, TimeEvoParams
    from paces.models import holstein
    f = np.load(os.path.join(GOLDEN, "scaled_n8c16.npz"))
    if not devices.configure_called:
        devices.configure()
    nchain, dim, g = 8, 16, 1.0
    terms = {"diag": dict(eps_sys=0.0, hbar_omega=1.0, delta_eps=0.0), "hopping": dict(J=1.0),
             "vib_coupling": dict(g=g)}
    with devices.vector_dev:
        ham = holstein.Hamiltonian(nchain=nchain, max_ho_dims=[dim] * nchain, use_terms=terms, debug_verb=0)
        te = holstein.TimeEvolution(ham, holstein.Observables, ["n_exc", "n_pho"], str(tmp_path),
                                    TimeEvoParams(maxstates=2000, enlarge_steps=1, shuffle_seed=None),
                                    ExpmParams(use_scaling=True), str(tmp_path / "params.log"))
        te.create_nonuniform_basis([1] * nchain, minpos=2, maxpos=3)
        te.create_initial_vector([1.0], [[2] + [0] * nchain])
        te.generate_timeline(np.arange(31) * 0.05, CoeffSaveParams())
        od = tmp_path / "observables"
        np.testing.assert_allclose(np.loadtxt(od / "n_exc.real"), f["n_exc"], rtol=1e-10, atol=1e-13)
        np.testing.assert_allclose(np.loadtxt(od / "n_pho.real"), f["n_pho"], rtol=1e-10, atol=1e-13)
        d, ref = np.loadtxt(od / "diagnostics.log"), f["diagnostics"]
        for col in (5, 6, 9, 10):   # converged, final_m (terms over all stages), numstates, ceiling hits
            assert np.array_equal(d[:, col], ref[:, col]), col
        who = te.whoami.view(torch.int32).cpu().numpy().view(np.uint32)
        assert np.array_equal(who, f["whoami"])
        np.testing.assert_allclose(te.vector.cpu().numpy(), f["vector"], rtol=0, atol=1e-13)


def test_large_steps_use_norm_estimates():
    """A time step so large that condition (3.13) fails: fragment 3.1 chooses (m, s) from
    1-norm estimates of powers of A (equation 3.11, the block estimator over device H rows),
    and the propagated state equals exp(+1j dt H) psi computed densely."""
    import scipy.linalg as sla
    import torch
    from paces_b200 import expm
    from tests import gpu_helpers
    nchain, dim, g = 6, 8, 1.0
    eng = gpu_helpers.engine_for(nchain, dim, g, cap=1 << 12)
    tr, _ = gpu_helpers.grown_trajectory(eng, nchain, 300, initpos=1, dim=dim)
    b, h = tr.basis, tr.h
    S = b.count()
    diag, mats, _ = gpu_helpers.csr_from_table(eng, b, h, 1.0, g)
    H = np.diag(diag) + sum(mm.toarray() for mm in mats.values())
    _, _, dbar = eng.hnorms(b, h)
    _, a1, _ = eng.hnorms(b, h, shift=dbar)
    dt = 80.0 / a1          # t ||A - mu I||_1 = 80: beyond condition (3.13)
    assert not expm.condition_3_13(dt * a1)
    A = 1j * (H - dbar * np.eye(S))
    # the estimates are lower bounds of the exact norms, and close to them
    for p in (2, 3):
        est = tr._norm_power(dt, dbar, p) ** p
        exact = np.abs(np.linalg.matrix_power(dt * A, p)).sum(axis=0).max()
        assert est <= exact * (1 + 1e-10) and est >= exact / 3, (p, est, exact)
    m, s = expm.choose(dt * a1, d=lambda p: tr._norm_power(dt, dbar, p))
    psi0 = tr.vector.clone()
    out = torch.zeros_like(tr.psis[tr.cur])
    eta = np.exp(dt * 1j * dbar / s)
    eng.expm_scaled(b, h, tr.psis[tr.cur], out, dt, dbar, m, s, eta)
    want = sla.expm(1j * dt * H) @ psi0.cpu().numpy()
    np.testing.assert_allclose(out[:S].cpu().numpy(), want, rtol=0, atol=1e-11)


def test_expm_multiply_simple_through_the_drop_in(tmp_path):
    """paces.aux.expm_multiply_simple(1j * te.ham_mat, v, t) -- the reference's own call of its
    scaling-and-squaring routine (paces/core/time_evolution.py:579-581) -- on the device H of
    a drop-in time evolution: equal to dense exp(+-1j t H) v, the operator's products equal to
    the explicit matrix, and a stale operator (after another step) refuses to act."""
    import scipy.linalg as sla
    import torch
    from paces.aux import expm_multiply_simple
    from paces.config import devices
    from paces.core.time_evolution import CoeffSaveParams, ExpmParams, TimeEvoParams
    from paces.models import holstein
    from tests import gpu_helpers
    if not devices.configure_called:
        devices.configure()
    nchain, dim, g = 6, 8, 1.3
    terms = {"diag": dict(eps_sys=0.0, hbar_omega=1.0, delta_eps=0.0), "hopping": dict(J=1.0),
             "vib_coupling": dict(g=g)}
    ham = holstein.Hamiltonian(nchain=nchain, max_ho_dims=[dim] * nchain, use_terms=terms, debug_verb=0)
    te = holstein.TimeEvolution(ham, holstein.Observables, ["n_exc"], str(tmp_path),
                                TimeEvoParams(maxstates=400, enlarge_steps=1, shuffle_seed=None), ExpmParams(),
                                str(tmp_path / "params.log"))
    te.create_nonuniform_basis([1] * nchain, minpos=1, maxpos=2)
    te.create_initial_vector([1.0], [[1] + [0] * nchain])
    te.generate_timeline(np.arange(6) * 0.05, CoeffSaveParams())
    op = te.create_ham_mat()
    tr = te._traj
    diag, mats, _ = gpu_helpers.csr_from_table(te.engine, tr.basis, tr.h, 1.0, g)
    H = np.diag(diag) + sum(mm.toarray() for mm in mats.values())
    v = te.vector.cpu().numpy()
    np.testing.assert_allclose((op @ te.vector).cpu().numpy(), H @ v, rtol=0, atol=1e-13)
    np.testing.assert_allclose(te.total_ham(te.vector, use_ham_mat=True).cpu().numpy(), H @ v, rtol=0, atol=1e-13)
    for t, A in ((0.05, 1j * op), (0.3, 1j * op), (0.05, -1j * op)):
        F, dbg = expm_multiply_simple(A, te.vector, t=t, return_dbg=True)
        sign = 1.0 if A.scale == 1j else -1.0
        want = sla.expm(sign * 1j * t * H) @ v
        np.testing.assert_allclose(F.cpu().numpy(), want, rtol=0, atol=1e-12)
        assert bool(dbg[0]) and dbg[1] > 0
    with pytest.raises(TypeError):
        expm_multiply_simple(torch.eye(3), torch.ones(3))
    with pytest.raises(NotImplementedError):
        expm_multiply_simple(2.0 * op, te.vector)
    te.generate_timeline(np.arange(2) * 0.05 + 1.0, CoeffSaveParams())
    with pytest.raises(RuntimeError):
        op @ te.vector
