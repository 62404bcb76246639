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


@pytest.mark.parametrize("precision,geo,J2", [("c128", 1, None), ("c64", 1, None), ("c128", 2, 0.3)])
def test_term_energies_match_the_oracle(precision, geo, J2):
    """paces_term_energies against the oracle's term matrices on the same basis and state:
    per exciton position the hopping and vibronic energies, and the phonon-vacuum sum."""
    import torch
    from oracle import paces_oracle as po
    from paces_b200.engine import Engine, ModelParams
    from tests import gpu_helpers
    nchain, dim, g = (9, 4, 1.3) if geo == 2 else (8, 8, 1.3)
    eng = Engine(ModelParams(nchain=nchain, max_ho_dims=[dim] * nchain, g=g, geo_dim=geo, J2=J2,
                             precision=precision), cap=1 << 15)
    m = po.Model(nchain, [dim] * nchain, g=g, geo_dim=geo, J2=J2)
    b = eng.basis_from_ref(gpu_helpers.initial_rows(nchain, dim, 1))
    for _ in range(3):
        b = eng.expand(b)
    new, h, _ = eng.assemble(b)
    S = new.count()
    asm = po.generate_mel(m, gpu_helpers.ref_rows(eng, b), 0)
    rng = np.random.default_rng(5)
    v = (rng.standard_normal(S) + 1j * rng.standard_normal(S)) / np.sqrt(S)
    psi = torch.zeros(max(new.cap, 1), dtype=eng.cdtype, device=eng.device)
    psi[:S] = torch.as_tensor(v, device=eng.device).to(eng.cdtype)
    vv = psi[:S].cpu().numpy().astype(np.complex128)
    hop, vib, vac = eng.term_energies(new, h, psi)
    pos = po.get_pos(m, asm.new_inds)
    want_hop = np.bincount(pos, weights=(vv.conj() * asm.mats["hopping"].dot(vv)).real, minlength=nchain) + \
        1j * np.bincount(pos, weights=(vv.conj() * asm.mats["hopping"].dot(vv)).imag, minlength=nchain)
    ev = vv.conj() * asm.mats["vib_coupling"].dot(vv)
    want_vib = np.bincount(pos, weights=ev.real, minlength=nchain) + 1j * np.bincount(pos, weights=ev.imag,
                                                                                       minlength=nchain)
    vacuum = po.sum_all_phonons(m, asm.new_inds) == 0
    tol = dict(rtol=1e-11, atol=1e-13) if precision == "c128" else dict(rtol=2e-5, atol=2e-6)
    np.testing.assert_allclose(hop.cpu().numpy(), want_hop, **tol)
    np.testing.assert_allclose(vib.cpu().numpy(), want_vib, **tol)
    np.testing.assert_allclose(vac, vv[vacuum].sum(), **tol)
