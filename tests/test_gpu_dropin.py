"""The drop-in: a driver script written against the reference's API (`import paces`) runs
unchanged on the device path and writes the reference's files with the reference's values."""

import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")

DRIVER = r'''
import os
import sys

import numpy

from paces.config import devices
from paces.models import holstein
from paces.core.time_evolution import CoeffSaveParams, ExpmParams, TimeEvoParams

devices.configure()
dirname = sys.argv[1]
nchain, max_ho_dim = 8, 16
term_param_dict = {
    "diag": dict(eps_sys=0.0, hbar_omega=1.0, delta_eps=0.0),
    "hopping": dict(J=1.0),
    "vib_coupling": dict(g=1.5),
}
te_params = TimeEvoParams(maxstates=4000, enlarge_steps=1, diagnostics=True, shuffle_seed=None)
coeff_save_obj = CoeffSaveParams(save_every=20, save_first=True, save_last=True)
with devices.vector_dev:
    hamobj = holstein.Hamiltonian(nchain=nchain, max_ho_dims=[max_ho_dim] * nchain,
                                  use_terms=term_param_dict, debug_verb=0)
    te = holstein.TimeEvolution(hamobj, holstein.Observables, ["n_pho", "n_exc", "total_energy"], dirname,
                                te_params, ExpmParams(), os.path.join(dirname, "params.log"))
    te.create_nonuniform_basis([1] * nchain, minpos=0, maxpos=1)
    te.create_initial_vector(vector_coeffs=[1], vector_coo=[[0] + nchain * [0]], auto_normalize=True)
    te.generate_timeline(numpy.arange(61) * 0.05, coeff_save_obj)
    print("numstates", te.numstates, tuple(te.whoami.shape))
'''


def test_reference_driver_runs_unchanged(tmp_path):
    script = tmp_path / "driver.py"
    script.write_text(DRIVER)
    out = tmp_path / "results"
    out.mkdir()
    env = dict(os.environ, PYTHONPATH=REPO + os.pathsep + os.environ.get("PYTHONPATH", ""))
    res = subprocess.run([sys.executable, str(script), str(out)], cwd=tmp_path, env=env, capture_output=True,
                         text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-3000:]
    f = np.load(os.path.join(GOLDEN, "traj_n8c16.npz"))
    obs = out / "observables"
    for name in ("n_exc", "n_pho"):
        got = np.loadtxt(obs / f"{name}.real")
        np.testing.assert_allclose(got, f[name], rtol=1e-10, atol=1e-13)
        assert np.all(np.loadtxt(obs / f"{name}.imag")[:, 2:] == 0)
        with open(obs / f"{name}.real") as fh:
            assert fh.readline().startswith("#time norm n^{")
    np.testing.assert_allclose(np.loadtxt(obs / "total_energy.real"), f["energy"], rtol=1e-10, atol=1e-12)
    diag = np.loadtxt(obs / "diagnostics.log")
    ref = f["diagnostics"]
    for col in (5, 6, 9, 10):   # converged, final_m, numstates, ceiling_hits
        assert np.array_equal(diag[:, col], ref[:, col]), col
    np.testing.assert_allclose(diag[:, 3], ref[:, 3], rtol=1e-12)     # post_adapt_norm
    np.testing.assert_allclose(diag[:, 4], ref[:, 4], rtol=1e-10, atol=1e-12)  # post_adapt_H
    wf = sorted(os.listdir(out / "wf_coeffs"))
    assert any(n.startswith("whoami_") for n in wf) and any(n.startswith("wf_file_") for n in wf)
    last_who = np.load(out / "wf_coeffs" / [n for n in wf if n.startswith("whoami_")][-1])
    assert last_who.dtype == np.uint32 and last_who.shape[0] == int(ref[-1, 9])
    assert "numstates" in res.stdout
