"""Batched trajectories (paces_batch_step: concurrent stages, one persistent Taylor launch)
and CUDA-graph replay give, trajectory by trajectory, bit-identical results to stepping
each trajectory alone with paces_step."""

import numpy as np
import pytest
import torch

from tests import gpu_helpers

pytestmark = pytest.mark.gpu

# nchain, dim, g, hbar_omega, maxstates, periodic, initpos, dt, site-energy seed
SPECS = [
    (6, 8, 1.0, 1.0, 300, False, 0, 0.05, None),
    (8, 16, 1.5, 0.7, 2000, True, 3, 0.03, None),
    (12, 16, 0.8, 1.3, 5000, True, 5, 0.05, 7),
    (20, 16, 2.0, 1.0, 8000, True, 0, 0.04, None),
    (5, 4, 1.2, 0.9, 100, False, 2, 0.05, None),
]


def _make(precision, cap=1 << 14, graph=False):
    out = []
    for nchain, dim, g, w0, m, periodic, initpos, dt, seed in SPECS:
        site = None if seed is None else list(np.random.default_rng(seed).normal(0, 0.5, nchain))
        eng = gpu_helpers.engine_for(nchain, dim, g, cap=cap, precision=precision, periodic=periodic,
                                     site_eps=site, hbar_omega=w0)
        tr, _ = gpu_helpers.grown_trajectory(eng, nchain, m, initpos=initpos, dim=dim, graph=graph)
        out.append((tr, dt))
    return out


def _state(tr):
    n = tr.basis.count()
    return tr.basis.keys[:n].cpu().numpy().copy(), tr.vector.cpu().numpy().copy()


def _same(ra, rb):
    for f in ("n_select", "n_enlarged", "n_states", "converged", "final_m", "ceiling_hits", "status"):
        assert getattr(ra, f) == getattr(rb, f), f
    for f in ("norm", "energy_re", "post_adapt_norm", "post_adapt_energy_re", "c1_plus_c2", "term_ratio"):
        assert getattr(ra, f) == getattr(rb, f), f
    assert list(ra.n_exc) == list(rb.n_exc) and list(ra.n_pho) == list(rb.n_pho)


def _alone(precision, steps, graph=False):
    runs = _make(precision, graph=graph)
    recs = [[tr.step(evolve=True, dt=dt) for _ in range(steps)] for tr, dt in runs]
    return recs, [_state(tr) for tr, _ in runs]


def _batched(precision, steps, graph=False, cap=1 << 14, n_streams=3):
    from paces_b200.engine import TrajectoryBatch
    runs = _make(precision, cap=cap)
    batch = TrajectoryBatch([tr for tr, _ in runs], n_streams=n_streams, graph=graph)
    recs = [[] for _ in runs]
    for _ in range(steps):
        out = batch.step(evolve=True, dt=[dt for _, dt in runs])
        for i, r in enumerate(out):
            recs[i].append(r)
    states = [_state(tr) for tr, _ in runs]
    batch.close()
    return recs, states


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_batch_matches_single_trajectories(precision):
    steps = 12
    ra, sa = _alone(precision, steps)
    rb, sb = _batched(precision, steps)
    for i in range(len(SPECS)):
        for a, b in zip(ra[i], rb[i]):
            _same(a, b)
        assert np.array_equal(sa[i][0], sb[i][0])
        assert np.array_equal(sa[i][1], sb[i][1])


def test_graph_replay_matches_eager():
    steps = 10
    ra, sa = _alone("c128", steps)
    rg, sg = _alone("c128", steps, graph=True)
    rb, sb = _batched("c128", steps, graph=True)
    for i in range(len(SPECS)):
        for a, g, b in zip(ra[i], rg[i], rb[i]):
            _same(a, g)
            _same(a, b)
        assert np.array_equal(sa[i][1], sg[i][1]) and np.array_equal(sa[i][1], sb[i][1])


def test_batch_grows_buffers_and_repeats_the_step():
    steps = 6
    ra, sa = _alone("c128", steps)
    rb, sb = _batched("c128", steps, cap=64, n_streams=2)
    for i in range(len(SPECS)):
        for a, b in zip(ra[i], rb[i]):
            _same(a, b)
        assert np.array_equal(sa[i][1], sb[i][1])


def test_large_trajectories_step_through_the_single_kernel():
    """Batches whose every trajectory has room for 2^25 states or more run their Taylor
    series through the single-trajectory kernel, one launch each (the capacity decides, so
    small bases in large buffers take that path too): the records and states stay those of
    stepping each trajectory alone."""
    from paces_b200.engine import TrajectoryBatch
    steps = 6
    specs = SPECS[:2]
    ra, sa = [], []
    for big in (False, True):
        runs = []
        for nchain, dim, g, w0, m, periodic, initpos, dt, seed in specs:
            eng = gpu_helpers.engine_for(nchain, dim, g, cap=(1 << 25) if big else (1 << 14), precision="c64",
                                         periodic=periodic, hbar_omega=w0)
            tr, _ = gpu_helpers.grown_trajectory(eng, nchain, m, initpos=initpos, dim=dim)
            runs.append((tr, dt, eng))
        if big:
            batch = TrajectoryBatch([tr for tr, _, _ in runs], n_streams=2)
            recs = [[] for _ in runs]
            for _ in range(steps):
                for i, r in enumerate(batch.step(evolve=True, dt=[dt for _, dt, _ in runs])):
                    recs[i].append(r)
            rb, sb = recs, [_state(tr) for tr, _, _ in runs]
            batch.close()
        else:
            ra = [[tr.step(evolve=True, dt=dt) for _ in range(steps)] for tr, dt, _ in runs]
            sa = [_state(tr) for tr, _, _ in runs]
        for _, _, eng in runs:
            eng.close()
    for i in range(len(specs)):
        for a, b in zip(ra[i], rb[i]):
            _same(a, b)
        assert np.array_equal(sa[i][0], sb[i][0]) and np.array_equal(sa[i][1], sb[i][1])
