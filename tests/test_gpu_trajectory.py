"""GPU parity of whole trajectories (paces_step) against the reference's recorded
observables and diagnostics, and against the CPU oracle."""

import glob
import os

import numpy as np
import pytest
import torch

from oracle import paces_oracle as po

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TRAJS = sorted(glob.glob(os.path.join(GOLDEN, "traj_*.npz")))


def run_device(eng, m, initpos, maxstates, es, steps, dt=0.05, shuffle_seed=None):
    from paces_b200.engine import Trajectory
    tr = Trajectory(eng, maxstates, es, shuffle_seed=shuffle_seed)
    b = eng.basis_from_ref(po.initial_basis(m, initpos))
    psi = torch.ones(1, dtype=torch.complex128, device=eng.device)
    tr.set_state(b, psi)
    recs = [tr.step(evolve=False)]
    for _ in range(steps):
        recs.append(tr.step(evolve=True, dt=dt))
    return tr, recs


@pytest.mark.parametrize("path", TRAJS, ids=os.path.basename)
def test_trajectory_matches_reference(path):
    from tests import gpu_helpers
    f = np.load(path)
    c = f["config"]
    nchain, dim, g, maxstates, es, steps, initpos = (int(c[0]), int(c[1]), float(c[2]), int(c[3]), int(c[4]),
                                                     int(c[5]), int(c[6]))
    eng = gpu_helpers.engine_for(nchain, dim, g, cap=1 << 12)
    m = po.Model(nchain, [dim] * nchain, g=g)
    _, recs = run_device(eng, m, initpos, maxstates, es, steps)
    ne = np.array([list(r.n_exc)[:nchain] for r in recs])
    nph = np.array([list(r.n_pho)[:nchain] for r in recs])
    np.testing.assert_allclose(ne, f["n_exc"][:, 2:], rtol=1e-10, atol=1e-13)
    np.testing.assert_allclose(nph, f["n_pho"][:, 2:], rtol=1e-10, atol=1e-13)
    np.testing.assert_allclose([r.norm for r in recs], f["n_exc"][:, 1], rtol=1e-12)
    diag = f["diagnostics"]
    assert [r.n_states for r in recs] == diag[:, 9].astype(int).tolist()
    assert [r.final_m for r in recs[1:]] == diag[1:, 6].astype(int).tolist()
    assert [bool(r.converged) for r in recs[1:]] == [bool(x) for x in diag[1:, 5]]
    np.testing.assert_allclose([r.post_adapt_norm for r in recs], diag[:, 3], rtol=1e-12)
    np.testing.assert_allclose([r.post_adapt_energy_re for r in recs], diag[:, 4], rtol=1e-11, atol=1e-12)
    assert [r.ceiling_hits for r in recs] == diag[:, 10].astype(int).tolist()
