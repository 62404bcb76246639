"""Failure paths, each driven on purpose in a form that faults, traps or hangs no GPU, and each
followed by a normal call on the same context that must succeed:

* a lookup that must succeed misses (a host-corrupted query key): the reference's search
  kernel asserts (paces/aux/cupy_search.py:205-228); here PACES_ERR_LOOKUP is raised;
* non-finite amplitudes entering a step: PACES_ERR_NONFINITE;
* the norm explosion check of the reference (paces/core/time_evolution.py:585-589): the
  drop-in raises the same RuntimeError;
* a bounded device wait that runs out: with a 10 ms wait limit one block of the Taylor
  kernel's cooperative launch gives up at its first grid barrier without arriving (the
  arrival nothing else provides), every other block's wait expires, the kernel returns and
  PACES_ERR_TIMEOUT reaches the host -- for the single-trajectory kernel, the fused step and
  the batched persistent launch.
"""

import math

import numpy as np
import pytest
import torch

from oracle import paces_oracle as po
from tests import gpu_helpers

pytestmark = pytest.mark.gpu

WAIT_NS = 10_000_000  # 10 ms


def _nat():
    from paces_b200 import _native
    return _native


def _same_record(a, b):
    for f in ("n_select", "n_enlarged", "n_states", "converged", "final_m", "ceiling_hits", "status"):
        assert getattr(a, f) == getattr(b, f), f
    for f in ("norm", "energy_re", "post_adapt_norm", "post_adapt_energy_re"):
        assert getattr(a, f) == getattr(b, f), f
    assert list(a.n_exc) == list(b.n_exc) and list(a.n_pho) == list(b.n_pho)


def _pair(precision="c128", nchain=8, maxstates=3000, cap=1 << 16):
    """Two identical trajectories on two contexts (one to fail, one as the witness)."""
    out = []
    for _ in range(2):
        eng = gpu_helpers.engine_for(nchain, 16, 1.3, cap=cap, precision=precision, periodic=True)
        tr, _ = gpu_helpers.grown_trajectory(eng, nchain, maxstates, initpos=2)
        for _ in range(3):
            tr.step(evolve=True, dt=0.05)
        out.append(tr)
    return out


def test_lookup_miss_raises_and_the_context_recovers():
    nat = _nat()
    nchain = 8
    eng = gpu_helpers.engine_for(nchain, 16, 1.0, cap=1 << 12)
    tr, _ = gpu_helpers.grown_trajectory(eng, nchain, 500)
    b = tr.basis
    rows = gpu_helpers.ref_rows(eng, b)
    m = po.Model(nchain, [16] * nchain)
    q = rows[:64].copy()
    raw = po.decompress(m, q[17:18])
    raw[0, 1 + 5] = 15                       # 15 phonons on site 5: never reached from the vacuum
    q[17] = po.compress(m, raw)[0]
    assert not po.lookup_with_mask(rows, q[17:18])[1][0]
    keys, pos, n = eng.query_from_ref(q)
    with pytest.raises(nat.PacesError) as err:
        eng.lookup(b, keys, pos, n, must_exist=True)
    assert err.value.code == nat.ERR_LOOKUP
    # the same queries without must_exist: the miss is -1, every other index exact, no status
    idx = eng.lookup(b, keys, pos, n).cpu().numpy()
    expect = np.arange(64)
    expect[17] = -1
    assert np.array_equal(idx, expect)
    assert eng.read_status() == nat.PACES_OK
    good_keys, good_pos, gn = eng.query_from_ref(rows[:64])
    assert np.array_equal(eng.lookup(b, good_keys, good_pos, gn, must_exist=True).cpu().numpy(), np.arange(64))
    rec = tr.step(evolve=True, dt=0.05)
    assert rec.status == nat.PACES_OK and math.isfinite(rec.norm)


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_nonfinite_amplitudes_raise_and_the_state_survives(precision):
    nat = _nat()
    bad, witness = _pair(precision)
    clean = bad.psis[bad.cur].clone()
    bad.psis[bad.cur][5] = float("nan")
    with pytest.raises(nat.PacesError) as err:
        bad.step(evolve=True, dt=0.05)
    assert err.value.code == nat.ERR_NONFINITE
    # the failed step wrote only the other slot: restore the amplitude and step on
    bad.psis[bad.cur].copy_(clean)
    for _ in range(3):
        _same_record(bad.step(evolve=True, dt=0.05), witness.step(evolve=True, dt=0.05))
    assert bad.eng.read_status() == nat.PACES_OK


def test_norm_explosion_raises_in_the_drop_in(tmp_path):
    """A two-term series (ExpmParams(m_star=2)) over a large step grows the norm past the
    cutoff after the first step; the drop-in raises the reference's RuntimeError and a new
    timeline on the same device then runs normally."""
    from paces.config import devices
    from paces.core.time_evolution import CoeffSaveParams, ExpmParams, TimeEvoParams
    from paces.models import holstein
    devices.configure()
    nchain = 6
    terms = {"diag": dict(eps_sys=0.0, hbar_omega=1.0, delta_eps=0.0), "hopping": dict(J=1.0),
             "vib_coupling": dict(g=3.0)}

    def timeline(expm, sub, dt):
        d = tmp_path / sub
        d.mkdir()
        ham = holstein.Hamiltonian(nchain=nchain, max_ho_dims=[16] * nchain, use_terms=terms, debug_verb=0)
        te = holstein.TimeEvolution(ham, holstein.Observables, ["n_exc"], str(d),
                                    TimeEvoParams(maxstates=2000, enlarge_steps=1, shuffle_seed=None), expm,
                                    str(d / "params.log"))
        te.create_nonuniform_basis([1] * nchain, minpos=0, maxpos=1)
        te.create_initial_vector(vector_coeffs=[1], vector_coo=[[0] + nchain * [0]], auto_normalize=True)
        te.generate_timeline(np.arange(6) * dt, CoeffSaveParams(save_every=0))
        return te

    with pytest.raises(RuntimeError, match=r"Norm has exceeded preset explosion cutoff value \(2.0\)!"):
        timeline(ExpmParams(m_star=2), "explode", 0.5)
    te = timeline(ExpmParams(), "normal", 0.05)
    assert abs(float(np.loadtxt(tmp_path / "normal" / "observables" / "n_exc.real")[-1, 1]) - 1.0) < 1e-12
    assert te.numstates > 0


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_taylor_grid_barrier_timeout_returns(precision):
    nat = _nat()
    tr, _ = _pair(precision)
    e, b, h = tr.eng, tr.basis, tr.h
    psi = tr.psis[tr.cur]
    ref, ref_dbg = e.taylor(b, h, psi, 0.05)
    ref = ref[: b.count()].clone()
    e.set_test_hooks(WAIT_NS, 0)
    try:
        with pytest.raises(nat.PacesError) as err:
            e.taylor(b, h, psi, 0.05)
        assert err.value.code == nat.ERR_TIMEOUT
    finally:
        e.set_test_hooks(0, -1)
    out, dbg = e.taylor(b, h, psi, 0.05)
    assert dbg == ref_dbg
    assert torch.equal(out[: b.count()], ref)


def test_step_timeout_leaves_the_state_intact():
    nat = _nat()
    bad, witness = _pair("c64")
    bad.eng.set_test_hooks(WAIT_NS, 1)
    try:
        with pytest.raises(nat.PacesError) as err:
            bad.step(evolve=True, dt=0.05)
        assert err.value.code == nat.ERR_TIMEOUT
    finally:
        bad.eng.set_test_hooks(0, -1)
    for _ in range(3):
        _same_record(bad.step(evolve=True, dt=0.05), witness.step(evolve=True, dt=0.05))


def test_batched_taylor_timeout_returns():
    from paces_b200.engine import TrajectoryBatch
    nat = _nat()
    trs, twins = [], []
    for nchain, g, initpos in ((8, 1.2, 1), (12, 0.8, 4), (6, 1.6, 0)):
        for lst in (trs, twins):
            eng = gpu_helpers.engine_for(nchain, 16, g, cap=1 << 14, precision="c64", periodic=True)
            tr, _ = gpu_helpers.grown_trajectory(eng, nchain, 2000, initpos=initpos)
            lst.append(tr)
    batch = TrajectoryBatch(trs, n_streams=2)
    try:
        batch.set_test_hooks(WAIT_NS, 0)
        with pytest.raises(nat.PacesError) as err:
            batch.step(evolve=True, dt=0.05)
        assert err.value.code == nat.ERR_TIMEOUT
        batch.set_test_hooks(0, -1)
        for _ in range(3):
            recs = batch.step(evolve=True, dt=0.05)
            for r, t in zip(recs, twins):
                _same_record(r, t.step(evolve=True, dt=0.05))
    finally:
        batch.close()
