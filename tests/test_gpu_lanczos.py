"""GPU parity of the Lanczos propagation (ExpmParams(lanczos_order=m); the reference's
_lanczos, paces/core/time_evolution.py:515-549) against the reference's own runs
(tests/golden/lanczos_*.npz) and the CPU oracle.

complex128: observables 1e-10 relative at every step, basis sizes and the final basis
exact, amplitudes 1e-12; the single step against the oracle on the same basis 1e-13.
complex64 (Krylov vectors in fp32, alpha, beta, the norms and the small exponential in fp64):
within the bound stated in the test against the complex128 run."""

import glob
import os

import numpy as np
import pytest
import torch

from oracle import paces_oracle as po
from tests import gpu_helpers

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "lanczos_*.npz")))


def _cfg(f):
    nchain, dim, g, ms, es, steps, initpos, order, dt = f["config"]
    return (int(nchain), int(dim), float(g), int(ms), int(es), int(steps), int(initpos), int(order), float(dt))


def _device_run(nchain, dim, g, ms, es, steps, initpos, order, dt, precision="c128", periodic=False):
    from paces_b200.engine import Trajectory
    eng = gpu_helpers.engine_for(nchain, dim, g, cap=1 << 12, precision=precision, periodic=periodic)
    m = po.Model(nchain, [dim] * nchain, g=g)
    tr = Trajectory(eng, ms, es, lanczos_order=order)
    tr.set_state(eng.basis_from_ref(po.initial_basis(m, initpos)), torch.ones(1, dtype=torch.complex128,
                                                                               device=eng.device))
    recs = [tr.step(evolve=False)] + [tr.step(evolve=True, dt=dt) for _ in range(steps)]
    return eng, tr, recs


@pytest.mark.parametrize("path", FIXTURES, ids=os.path.basename)
def test_lanczos_trajectory_matches_the_reference(path):
    f = np.load(path)
    nchain, dim, g, ms, es, steps, initpos, order, dt = _cfg(f)
    eng, tr, recs = _device_run(nchain, dim, g, ms, es, steps, initpos, order, dt)
    np.testing.assert_allclose([list(r.n_exc)[:nchain] for r in recs], f["n_exc"][:, 2:], rtol=1e-10, atol=1e-13)
    np.testing.assert_allclose([list(r.n_pho)[:nchain] for r in recs], f["n_pho"][:, 2:], rtol=1e-10, atol=1e-13)
    np.testing.assert_allclose([r.norm for r in recs], f["n_exc"][:, 1], rtol=1e-12)
    np.testing.assert_allclose([r.energy_re for r in recs], f["energy"][:, 2], rtol=1e-10, atol=1e-12)
    diag = f["diagnostics"]
    assert [r.n_states for r in recs] == diag[:, 9].astype(int).tolist()
    for r in recs[1:]:   # the reference's placeholder diagnostics [False, 0, 0, 0]
        assert (r.converged, r.final_m, r.c1_plus_c2, r.term_ratio) == (0, 0, 0.0, 0.0)
    assert np.array_equal(gpu_helpers.ref_rows(eng, tr.basis), f["whoami"])
    np.testing.assert_allclose(tr.vector.cpu().numpy(), f["vector"], rtol=0, atol=1e-12)
    eng.close()


@pytest.mark.parametrize("order", [1, 4, 12, 40, 63])
def test_lanczos_single_step_matches_the_oracle(order):
    """One propagation on a saturated basis against the oracle's restatement, same input."""
    nchain, g = 10, 1.4
    eng = gpu_helpers.engine_for(nchain, 16, g, cap=1 << 15, periodic=True)
    tr, _ = gpu_helpers.grown_trajectory(eng, nchain, 3000, initpos=3)
    for _ in range(4):
        tr.step(evolve=True, dt=0.05)
    b, h = tr.basis, tr.h
    n = b.count()
    psi = torch.zeros(b.cap, dtype=torch.complex128, device=eng.device)
    psi[:n] = tr.vector
    out, dbg = eng.lanczos(b, h, psi, 0.1, order)
    assert dbg == [False, 0, 0.0, 0.0]
    m = po.Model(nchain, [16] * nchain, g=g, periodic=True)
    diag, mats, _ = gpu_helpers.csr_from_table(eng, b, h, 1.0, g)
    asm = po.Assembly(gpu_helpers.ref_rows(eng, b), diag, mats, None, None, 0)
    ref, _ = po.lanczos(asm, psi[:n].cpu().numpy(), 0.1, order)
    np.testing.assert_allclose(out[:n].cpu().numpy(), ref, rtol=0, atol=1e-13)
    # the same input again gives the same output bit for bit (fixed reduction order)
    again, _ = eng.lanczos(b, h, psi, 0.1, order)
    assert torch.equal(again[:n], out[:n])
    eng.close()


def test_lanczos_complex64_within_bound():
    """The complex64 Lanczos step against the complex128 one over 100 steps of dt 0.05 on a
    periodic chain (N=16, g=1.5, maxstates 2^14, order 16): every observable within 1e-5."""
    runs = {}
    for prec in ("c128", "c64"):
        from paces_b200.engine import Trajectory
        eng = gpu_helpers.engine_for(16, 16, 1.5, cap=1 << 16, precision=prec, periodic=True)
        tr, first = gpu_helpers.grown_trajectory(eng, 16, 1 << 14, initpos=3, lanczos_order=16)
        recs = [first] + [tr.step(evolve=True, dt=0.05) for _ in range(100)]
        runs[prec] = gpu_helpers.observables_of(recs, 16)
        eng.close()
    errs = {k: float(np.max(np.abs(runs["c128"][k] - runs["c64"][k]))) for k in runs["c128"]}
    print("Lanczos complex64 vs complex128, max abs error:", errs)
    for k, e in errs.items():
        assert e <= 1e-5, (k, e)


def test_lanczos_through_the_drop_in(tmp_path):
    """ExpmParams(lanczos_order=12) through the reference-facing API writes the reference's
    files with the reference's values (the lanczos_n8c16_m12 run)."""
    from paces.config import devices
    from paces.core.time_evolution import CoeffSaveParams, ExpmParams, TimeEvoParams
    from paces.models import holstein
    f = np.load(os.path.join(GOLDEN, "lanczos_n8c16_m12.npz"))
    nchain, dim, g, ms, es, steps, initpos, order, dt = _cfg(f)
    devices.configure()
    terms = {"diag": dict(eps_sys=0.0, hbar_omega=1.0, delta_eps=0.0), "hopping": dict(J=1.0),
             "vib_coupling": dict(g=g)}
    ham = holstein.Hamiltonian(nchain=nchain, max_ho_dims=[dim] * nchain, use_terms=terms, debug_verb=0)
    te = holstein.TimeEvolution(ham, holstein.Observables, ["n_exc", "n_pho", "total_energy"], str(tmp_path),
                                TimeEvoParams(maxstates=ms, enlarge_steps=es, shuffle_seed=None),
                                ExpmParams(lanczos_order=order), str(tmp_path / "params.log"))
    te.create_nonuniform_basis([1] * nchain, minpos=initpos, maxpos=initpos + 1)
    te.create_initial_vector(vector_coeffs=[1], vector_coo=[[initpos] + nchain * [0]], auto_normalize=True)
    te.generate_timeline(np.arange(steps + 1) * dt, CoeffSaveParams())
    obs = tmp_path / "observables"
    np.testing.assert_allclose(np.loadtxt(obs / "n_exc.real"), f["n_exc"], rtol=1e-10, atol=1e-13)
    np.testing.assert_allclose(np.loadtxt(obs / "n_pho.real"), f["n_pho"], rtol=1e-10, atol=1e-13)
    d = np.loadtxt(obs / "diagnostics.log")
    for col in (5, 6, 7, 8, 9):
        assert np.array_equal(d[:, col], f["diagnostics"][:, col]), col
