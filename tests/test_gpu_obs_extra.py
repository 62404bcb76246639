"""The drop-in's remaining Holstein observables against the reference's own values
(`tests/golden/obs_extra_n7c8.npz`, made by the unmodified reference run on CPU): hopping
energy per bond and <mu(t) mu(0)> at every step, the vibronic coupling energy per site
and the reduced density matrices of two fields (0 is the exciton position) for the last
state, whose basis and amplitudes are compared too.

The exciton starts off the open chain's mirror axis on purpose: started on the axis,
mirror-image states tie exactly at the truncation cut, and which of two tied states is
kept then follows the last bit of their computed amplitudes -- a legitimate difference
between any two implementations (the CPU oracle itself then differs from the reference's
run by 1.8e-7 in small amplitudes)."""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_extra_observables_match_the_reference(tmp_path):
    import torch
    from paces.config import devices
    from paces.core.time_evolution import CoeffSaveParams, ExpmParams, TimeEvoParams
    from paces.models import holstein
    f = np.load(os.path.join(GOLDEN, "obs_extra_n7c8.npz"))
    nchain, dim, g = 7, 8, 1.2
    if not devices.configure_called:
        devices.configure()
    terms = {"diag": dict(eps_sys=0.0, hbar_omega=1.0, delta_eps=0.0), "hopping": dict(J=1.0),
             "vib_coupling": dict(g=g)}
    with devices.vector_dev:
        ham = holstein.Hamiltonian(nchain=nchain, max_ho_dims=[dim] * nchain, use_terms=terms, debug_verb=0)
        te = holstein.TimeEvolution(ham, holstein.Observables, ["n_exc", "hopping", "mu_to_0"], str(tmp_path),
                                    TimeEvoParams(maxstates=3000, enlarge_steps=1, shuffle_seed=None),
                                    ExpmParams(), str(tmp_path / "params.log"))
        te.create_nonuniform_basis([1] * nchain, minpos=1, maxpos=2)
        te.create_initial_vector([1.0], [[1] + [0] * nchain])
        te.generate_timeline(np.arange(31) * 0.05, CoeffSaveParams())
        od = tmp_path / "observables"
        np.testing.assert_allclose(np.loadtxt(od / "n_exc.real"), f["n_exc"], rtol=1e-10, atol=1e-13)
        np.testing.assert_allclose(np.loadtxt(od / "V_hop.real"), f["hop_re"], rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(np.loadtxt(od / "V_hop.imag"), f["hop_im"], rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(np.loadtxt(od / "mu_to_0.real"), f["mu_re"], rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(np.loadtxt(od / "mu_to_0.imag"), f["mu_im"], rtol=1e-10, atol=1e-12)
        obs = te.obsobj
        obs.primer_hook()
        vec = te.vector
        who = te.whoami.view(torch.int32).cpu().numpy().view(np.uint32)
        assert np.array_equal(who, f["whoami"])
        np.testing.assert_allclose(vec.cpu().numpy(), f["vector"], rtol=0, atol=1e-13)
        coupling = obs.calculate_coupling(vec).cpu().numpy()
        np.testing.assert_allclose(coupling, f["coupling"], rtol=1e-10, atol=1e-12)
        for site, key in ((0, "rdm0"), (3, "rdm3")):
            rdm = obs.calculate_rdm(site, vec)
            assert isinstance(rdm, torch.Tensor)
            np.testing.assert_allclose(rdm.cpu().numpy(), f[key], rtol=1e-10, atol=1e-12)
