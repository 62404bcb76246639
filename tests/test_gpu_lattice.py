"""Lattices beyond the nearest-neighbour chain -- geo_dim > 1 (hopping along every lattice
dimension, paces/models/holstein.py:210-232) and the next-nearest-neighbour hopping2 term
(holstein.py:234-240) -- through the drop-in API against the reference's own runs
(tests/golden/lattice_<name>.npz): observables at every step, basis sizes, the final basis
and amplitudes; and the assembled Hamiltonian of a lattice basis term by term against the
oracle's CSR matrices."""

import os

import numpy as np
import pytest
import torch

from oracle import paces_oracle as po
from tests import gpu_helpers

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
NAMES = ["geo2_n9c8", "hop2_n8c8", "geo2hop2_n16c4", "geo3_n27c4"]


def _config(name):
    f = np.load(os.path.join(GOLDEN, f"lattice_{name}.npz"))
    nchain, geo, dim, g, J2, deps, ms, steps, initpos = f["config"]
    nchain, geo, dim, ms, steps, initpos = (int(x) for x in (nchain, geo, dim, ms, steps, initpos))
    return f, nchain, geo, dim, float(g), None if np.isnan(J2) else float(J2), float(deps), ms, steps, initpos


@pytest.mark.parametrize("name", NAMES)
def test_lattice_timeline_matches_the_reference(tmp_path, name):
    from paces.config import devices
    from paces.core.time_evolution import CoeffSaveParams, ExpmParams, TimeEvoParams
    from paces.models import holstein
    f, nchain, geo, dim, g, J2, deps, ms, steps, initpos = _config(name)
    if not devices.configure_called:
        devices.configure()
    terms = {"diag": dict(eps_sys=0.0, hbar_omega=1.0, delta_eps=deps), "hopping": dict(J=1.0)}
    if J2 is not None:
        terms["hopping2"] = dict(J2=J2)
    terms["vib_coupling"] = dict(g=g)
    with devices.vector_dev:
        ham = holstein.Hamiltonian(nchain=nchain, max_ho_dims=[dim] * nchain, geo_dim=geo, use_terms=terms,
                                   debug_verb=0)
        te = holstein.TimeEvolution(ham, holstein.Observables, ["n_exc", "n_pho", "total_energy"], str(tmp_path),
                                    TimeEvoParams(maxstates=ms, enlarge_steps=1, shuffle_seed=None),
                                    ExpmParams(), str(tmp_path / "params.log"))
        te.create_nonuniform_basis([1] * nchain, minpos=initpos, maxpos=initpos + 1)
        te.create_initial_vector([1.0], [[initpos] + [0] * nchain])
        te.generate_timeline(np.arange(steps + 1) * 0.05, CoeffSaveParams())
    od = tmp_path / "observables"
    np.testing.assert_allclose(np.loadtxt(od / "n_exc.real"), f["n_exc"], rtol=1e-10, atol=1e-13)
    np.testing.assert_allclose(np.loadtxt(od / "n_pho.real"), f["n_pho"], rtol=1e-10, atol=1e-13)
    np.testing.assert_allclose(np.loadtxt(od / "total_energy.real"), f["energy"], rtol=1e-10, atol=1e-12)
    d, ref = np.loadtxt(od / "diagnostics.log"), f["diagnostics"]
    for col in (5, 6, 9, 10):   # converged, final_m, numstates, ceiling hits
        assert np.array_equal(d[:, col], ref[:, col]), col
    who = te.whoami.view(torch.int32).cpu().numpy().view(np.uint32)
    assert np.array_equal(who, f["whoami"])
    np.testing.assert_allclose(te.vector.cpu().numpy(), f["vector"], rtol=0, atol=1e-13)


@pytest.mark.parametrize("name", NAMES)
def test_lattice_hamiltonian_matches_the_oracle(name):
    """paces_expand / paces_assemble on a grown lattice basis: the new basis, the diagonal
    and every term's CSR bit for bit, and one Taylor step, against the oracle."""
    from paces_b200.core.hamiltonian import hmat_to_coo
    from paces_b200.engine import Engine, ModelParams
    import scipy.sparse as sp
    f, nchain, geo, dim, g, J2, deps, ms, steps, initpos = _config(name)
    eng = Engine(ModelParams(nchain=nchain, max_ho_dims=[dim] * nchain, g=g, delta_eps=deps, geo_dim=geo, J2=J2),
                 cap=1 << 16)
    m = po.Model(nchain, [dim] * nchain, g=g, delta_eps=deps, geo_dim=geo, J2=J2)
    rows = gpu_helpers.initial_rows(nchain, dim, initpos)
    b = eng.basis_from_ref(rows)
    ob = po.initial_basis(m, initpos)
    for _ in range(2):
        b = eng.expand(b)
        ob = po.enlarge(m, ob)
    assert np.array_equal(gpu_helpers.ref_rows(eng, b), ob)
    new, h, ceil = eng.assemble(b)
    asm = po.generate_mel(m, ob, 0)
    assert np.array_equal(gpu_helpers.ref_rows(eng, new), asm.new_inds)
    assert int(ceil) == asm.ceiling_hits
    coo, diag = hmat_to_coo(eng, new, h)
    np.testing.assert_array_equal(diag.cpu().numpy(), asm.diag)
    S = new.count()
    assert set(coo) == set(asm.mats)
    for term, (vals, (r, c)) in coo.items():
        got = sp.coo_matrix((vals.cpu().numpy(), (r.cpu().numpy(), c.cpu().numpy())), shape=(S, S)).tocsr()
        got.sort_indices()
        want = asm.mats[term].copy()
        want.sort_indices()
        assert (got != want).nnz == 0, term
    # one Taylor step of a seeded state on this H
    rng = np.random.default_rng(3)
    v = (rng.standard_normal(S) + 1j * rng.standard_normal(S)) / np.sqrt(2 * S)
    psi = torch.zeros(max(new.cap, 1), dtype=torch.complex128, device=eng.device)
    psi[:S] = torch.as_tensor(v, device=eng.device)
    out, _ = eng.taylor(new, h, psi, 0.05)
    want, _ = po.taylor(asm, v, 0.05)
    np.testing.assert_allclose(out[:S].cpu().numpy(), want, rtol=0, atol=1e-14)


def test_lattice_model_checks():
    from paces_b200 import _native as nat
    from paces_b200.engine import Engine, ModelParams, TrajectoryBatch
    with pytest.raises(nat.PacesError):
        Engine(ModelParams(nchain=10, max_ho_dims=[4] * 10, geo_dim=2))
    with pytest.raises(nat.PacesError):
        Engine(ModelParams(nchain=9, max_ho_dims=[4] * 9, geo_dim=2, periodic=True))
    eng = Engine(ModelParams(nchain=9, max_ho_dims=[4] * 9, geo_dim=2), cap=1 << 12)
    tr, _ = gpu_helpers.grown_trajectory(eng, 9, 200, initpos=1, dim=4)
    with pytest.raises(nat.PacesError):
        TrajectoryBatch([tr]).step(evolve=True, dt=0.05)
