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
