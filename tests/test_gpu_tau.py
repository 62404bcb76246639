"""The look-ahead weighting of the truncation (TimeEvoParams.tau != 0; the reference ranks
the states by coherence_weighting_func or norm_weighting_func from the second step on,
paces/core/time_evolution.py:464-476, :560, :854-857):

* the drop-in timeline against the reference's own runs (tests/golden/tau_*_n8c16.npz):
  observables at every step, the final basis and amplitudes;
* the device weights (paces_lookahead_weights) and H 1 against the oracle on the same
  basis and state, and the weighted truncation against the oracle's on the same weights;
* CUDA-graph replay and batched stepping with the weighting give the eager single-
  trajectory results bit for bit; complex64 stays within its error bound."""

import os

import numpy as np
import pytest
import torch

from oracle import paces_oracle as po
from tests import gpu_helpers

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
WEIGHTINGS = ["coherence", "norm"]
# |psi| comes from CUDA's hypot (at most 2 ulp from the exact value) where the reference
# uses the C library's; the coherence weight squares it: 4 ulp, below 1e-15 relative.
# Every other operation rounds as the reference's does.
HYPOT_RTOL = 1e-15


def _dropin_run(tmp_path, weighting, precision=None):
    from paces.config import devices
    from paces.core.time_evolution import CoeffSaveParams, ExpmParams, TimeEvoParams
    from paces.models import holstein
    if not devices.configure_called:
        devices.configure()
    nchain, dim, g = 8, 16, 1.0
    terms = {"diag": dict(eps_sys=0.0, hbar_omega=1.0, delta_eps=0.0), "hopping": dict(J=1.0),
             "vib_coupling": dict(g=g)}
    kw = {} if precision is None else {"use_complex_type": {"c64": np.complex64, "c128": np.complex128}[precision]}
    with devices.vector_dev:
        ham = holstein.Hamiltonian(nchain=nchain, max_ho_dims=[dim] * nchain, use_terms=terms, debug_verb=0, **kw)
        te = holstein.TimeEvolution(ham, holstein.Observables, ["n_exc", "n_pho", "total_energy"], str(tmp_path),
                                    TimeEvoParams(maxstates=1500, enlarge_steps=1, shuffle_seed=None, tau=0.2,
                                                  weighting_name=weighting),
                                    ExpmParams(), str(tmp_path / "params.log"))
        te.create_nonuniform_basis([1] * nchain, minpos=2, maxpos=3)
        te.create_initial_vector([1.0], [[2] + [0] * nchain])
        te.generate_timeline(np.arange(31) * 0.05, CoeffSaveParams())
    return te


@pytest.mark.parametrize("weighting", WEIGHTINGS)
def test_weighted_timeline_matches_the_reference(tmp_path, weighting):
    f = np.load(os.path.join(GOLDEN, f"tau_{weighting}_n8c16.npz"))
    te = _dropin_run(tmp_path, weighting)
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
    # the drop-in's weighting functions on the final state, against the oracle's
    S = te.numstates
    eng = te.engine
    diag, mats, _ = gpu_helpers.csr_from_table(eng, te._traj.basis, te._traj.h, 1.0, 1.0)
    asm = po.Assembly(None, diag, mats, None, None, 0)
    v = te.vector.cpu().numpy()
    want = po.lookahead_weights(asm, v, 0.2, weighting)
    got = te.weighting_func(te.vector, 0.2).cpu().numpy()
    assert got.shape == (S,)
    np.testing.assert_allclose(got, want, rtol=HYPOT_RTOL, atol=0)
    assert np.array_equal(te.total_ham_ones().cpu().numpy(), po.ham_ones(asm))


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_device_weights_and_weighted_truncation_match_the_oracle(precision):
    nchain, dim, g = 10, 16, 1.3
    eng = gpu_helpers.engine_for(nchain, dim, g, cap=1 << 15, precision=precision)
    tr, _ = gpu_helpers.grown_trajectory(eng, nchain, 3000, initpos=3, dim=dim)
    for _ in range(6):
        tr.step(evolve=True, dt=0.05)
    b, h = tr.basis, tr.h
    S = b.count()
    diag, mats, _ = gpu_helpers.csr_from_table(eng, b, h, 1.0, g)
    asm = po.Assembly(None, diag, mats, None, None, 0)
    v = tr.vector.cpu().numpy().astype(np.complex128)
    from paces_b200 import _native as nat
    psi = tr.psis[tr.cur]
    ones = eng.lookahead_weights(b, h, psi, 0.0, nat.WEIGHT_HAM_ONES).cpu().numpy()
    assert np.array_equal(ones, po.ham_ones(asm))
    for name, kind in (("coherence", nat.WEIGHT_COHERENCE), ("norm", nat.WEIGHT_NORM)):
        for tau in (0.05, 0.7):
            w = eng.lookahead_weights(b, h, psi, tau, kind)
            want = po.lookahead_weights(asm, v, tau, name)
            if precision == "c128":
                np.testing.assert_allclose(w.cpu().numpy(), want, rtol=HYPOT_RTOL, atol=0)
            else:   # fp32 amplitudes (and fp32 H psi for the norm weighting)
                scale = np.abs(want).max()
                np.testing.assert_allclose(w.cpu().numpy(), want, rtol=2e-6, atol=2e-6 * scale)
            # the weighted truncation keeps exactly the oracle's selection for these weights
            for ms in (S // 3, S - 1, S + 5):
                sel = eng.truncate_weighted(b, w, ms)
                keys = gpu_helpers.ref_rows(eng, sel)
                who = gpu_helpers.ref_rows(eng, b)
                assert np.array_equal(keys, po.truncate(who, v, ms, weights=w.cpu().numpy()))


def _weighted_runs(graph, steps, weighting, precision="c128"):
    from paces_b200 import _native as nat
    kind = {"coherence": nat.WEIGHT_COHERENCE, "norm": nat.WEIGHT_NORM}[weighting]
    runs = []
    for nchain, dim, g, m, initpos, tau in ((8, 16, 1.0, 1500, 2, 0.2), (12, 16, 1.5, 4000, 5, 0.1)):
        eng = gpu_helpers.engine_for(nchain, dim, g, cap=1 << 13, precision=precision)
        tr, _ = gpu_helpers.grown_trajectory(eng, nchain, m, initpos=initpos, dim=dim, graph=graph,
                                             weighting=kind, tau=tau)
        runs.append(tr)
    return runs


@pytest.mark.parametrize("weighting", WEIGHTINGS)
def test_weighted_graph_and_batch_match_eager(weighting):
    from paces_b200.engine import TrajectoryBatch
    steps = 12
    eager = _weighted_runs(False, steps, weighting)
    recs_e = [[tr.step(evolve=True, dt=0.05) for _ in range(steps)] for tr in eager]
    graphed = _weighted_runs(True, steps, weighting)
    recs_g = [[tr.step(evolve=True, dt=0.05) for _ in range(steps)] for tr in graphed]
    batched = _weighted_runs(False, steps, weighting)
    batch = TrajectoryBatch(batched, n_streams=2)
    recs_b = [[] for _ in batched]
    for _ in range(steps):
        for i, r in enumerate(batch.step(evolve=True, dt=0.05)):
            recs_b[i].append(r)
    batch.close()
    for k in range(len(eager)):
        for ra, rg, rb in zip(recs_e[k], recs_g[k], recs_b[k]):
            for other in (rg, rb):
                for f in ("n_select", "n_states", "final_m", "status", "n_tied"):
                    assert getattr(ra, f) == getattr(other, f), f
                assert ra.norm == other.norm and list(ra.n_exc) == list(other.n_exc)
        n = eager[k].basis.count()
        for other in (graphed[k], batched[k]):
            assert other.basis.count() == n
            assert torch.equal(eager[k].basis.keys[:n], other.basis.keys[:n])
            assert torch.equal(eager[k].vector, other.vector)


def test_weighted_regrow_keeps_the_table():
    """Growing the buffers (what a step that overflows them does before it repeats) keeps
    the current basis' table, which the next weighted step reads."""
    from paces_b200 import _native as nat
    nchain, dim, g = 8, 16, 1.0
    runs = []
    for _ in range(2):
        eng = gpu_helpers.engine_for(nchain, dim, g, cap=1 << 13)
        tr, _ = gpu_helpers.grown_trajectory(eng, nchain, 1500, initpos=2, dim=dim, weighting=nat.WEIGHT_NORM,
                                             tau=0.2)
        runs.append(tr)
    ref, tr = runs
    for k in range(10):
        if k == 4:
            cap = tr.eng.cap
            tr._regrow()
            assert tr.eng.cap > cap
        ra = ref.step(evolve=True, dt=0.05)
        rb = tr.step(evolve=True, dt=0.05)
        assert ra.n_states == rb.n_states and ra.norm == rb.norm and list(ra.n_exc) == list(rb.n_exc)


def test_weighted_step_needs_the_current_table():
    from paces_b200 import _native as nat
    from paces_b200.engine import Trajectory
    nchain, dim = 6, 8
    eng = gpu_helpers.engine_for(nchain, dim, 1.0, cap=1 << 12)
    tr, _ = gpu_helpers.grown_trajectory(eng, nchain, 200, initpos=1, dim=dim, weighting=nat.WEIGHT_COHERENCE,
                                         tau=0.3)
    b, psi = tr.basis.clone(), tr.vector.clone()
    tr2 = Trajectory(eng, 200, 1, weighting=nat.WEIGHT_COHERENCE, tau=0.3)
    tr2.set_state(b, psi)
    with pytest.raises(RuntimeError):
        tr2.step(evolve=True, dt=0.05)
    with pytest.raises(ValueError):
        Trajectory(eng, 200, 1, weighting=nat.WEIGHT_NORM, tau=0.0)


def test_weighted_c64_stays_close(tmp_path):
    f = np.load(os.path.join(GOLDEN, "tau_norm_n8c16.npz"))
    _dropin_run(tmp_path, "norm", precision="c64")
    od = tmp_path / "observables"
    np.testing.assert_allclose(np.loadtxt(od / "n_exc.real")[:, 2:], f["n_exc"][:, 2:], rtol=0, atol=1e-5)
    np.testing.assert_allclose(np.loadtxt(od / "n_pho.real")[:, 2:], f["n_pho"][:, 2:], rtol=0, atol=1e-5)
