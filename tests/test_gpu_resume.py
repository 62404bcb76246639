"""Checkpoint and resume in the reference's files: a run that saves its wavefunction and
basis (`wf_coeffs/wf_file_<t>.npy`, `whoami_<t>.npy`, paces/core/time_evolution.py:682-685)
and a second run started from those files with `load_basis_from_file` and the saved vector
(paces/core/time_evolution.py:271-287) continue identically: the resumed run's first step
rebuilds the same basis around the saved state, so every later step repeats the
uninterrupted run bit for bit."""

import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(dirname, t_array, load=None):
    from paces.config import devices
    from paces.core.time_evolution import CoeffSaveParams, ExpmParams, TimeEvoParams
    from paces.models import holstein
    if not devices.configure_called:
        devices.configure()
    nchain, dim = 9, 16
    terms = {"diag": dict(eps_sys=0.0, hbar_omega=1.0, delta_eps=0.0), "hopping": dict(J=1.0),
             "vib_coupling": dict(g=1.4)}
    with devices.vector_dev:
        ham = holstein.Hamiltonian(nchain=nchain, max_ho_dims=[dim] * nchain, use_terms=terms, debug_verb=0)
        te = holstein.TimeEvolution(ham, holstein.Observables, ["n_exc", "n_pho", "total_energy"], dirname,
                                    TimeEvoParams(maxstates=6000, enlarge_steps=1, diagnostics=True,
                                                  shuffle_seed=None),
                                    ExpmParams(), os.path.join(dirname, "params.log"))
        if load is None:
            te.create_nonuniform_basis([1] * nchain, minpos=0, maxpos=1)
            te.create_initial_vector([1.0], [[0] + [0] * nchain])
        else:
            who, wf = load
            te.load_basis_from_file(who)
            te.vector = np.load(wf)
        te.generate_timeline(t_array, CoeffSaveParams(save_every=10, save_first=True, save_last=True))


def test_resume_from_saved_files_continues_the_run(tmp_path):
    full, resumed = tmp_path / "full", tmp_path / "resumed"
    full.mkdir()
    resumed.mkdir()
    t = np.arange(21) * 0.05
    _run(str(full), t)
    who = sorted(glob.glob(str(full / "wf_coeffs" / "whoami_*.npy")))
    wf = sorted(glob.glob(str(full / "wf_coeffs" / "wf_file_*.npy")))
    assert len(who) == len(wf) == 3            # steps 0, 10 and the last
    w10 = [p for p in who if "0.50" in os.path.basename(p)]
    f10 = [p for p in wf if "0.50" in os.path.basename(p)]
    assert len(w10) == len(f10) == 1
    saved = np.load(w10[0])
    assert saved.dtype == np.uint32 and np.load(f10[0]).dtype == np.complex128
    _run(str(resumed), t[10:], load=(w10[0], f10[0]))
    for name in ("n_exc.real", "n_pho.real", "total_energy.real"):
        a = np.loadtxt(full / "observables" / name)
        b = np.loadtxt(resumed / "observables" / name)
        # row 0 of the resumed run is its non-evolving first step at t = 0.5
        assert np.array_equal(a[11:, 0], b[1:, 0])
        np.testing.assert_allclose(b[1:], a[11:], rtol=1e-13, atol=1e-15)
    da = np.loadtxt(full / "observables" / "diagnostics.log")
    db = np.loadtxt(resumed / "observables" / "diagnostics.log")
    for col in (5, 6, 9, 10):   # converged, final_m, numstates, ceiling hits
        assert np.array_equal(da[11:, col], db[1:, col]), col
