"""Generate golden fixtures by running the unmodified reference (rkevk/paces 1.2.0) on CPU.

Usage (in a container that has the reference source; it never runs on the GPU host):

    python tests/golden/gen_golden.py /path/to/reference [--long]

The reference is imported behind `oracle/refshim` (a NumPy stand-in for CuPy).
Nothing of the reference is copied: only its outputs on seeded, synthetic
inputs are stored, as compressed .npz files next to this script.

Fixtures written:
  layout_<name>.npz   compress_ind_arr, field get/add kernels, sum_all_phonons,
                      calculate_bath_n_b, searchsorted_full_binary, cupy_unique
  stages_<name>.npz   per-step stage data of a short trajectory: truncation input
                      and output, generate_mel output (diag, new_inds, CSR per term),
                      remap output, Taylor output and diagnostics, observables
  traj_<name>.npz     observables and diagnostics of every step of a trajectory
  ed_n4.npz           exact-diagonalisation known answer (full Hilbert space)
  obs_extra_n7c8.npz  hopping, mu_to_0, coupling and reduced density matrices
  scaled_n8c16.npz    a trajectory propagated with ExpmParams(use_scaling=True)
  lanczos_<name>.npz  trajectories propagated with ExpmParams(lanczos_order=m)
  tau_<weighting>_n8c16.npz  trajectories truncated by the look-ahead weights (tau=0.2)
  lattice_<name>.npz  geo_dim > 1 lattices and the hopping2 term (open boundaries)
  fragment31.npz      (m, s) of code fragment 3.1 for synthetic norms and norm estimates
"""

import argparse
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

LAYOUTS = {
    # name: (nchain, max_ho_dim) -- 4-bit fields (N=16: W=3, N=32: W=5), 7-bit straddling
    # fields (N=25 as in the reference's example driver), 3-bit fields.
    "n16c16": (16, 16),
    "n32c16": (32, 16),
    "n25c128": (25, 128),
    "n6c8": (6, 8),
}

STAGE_RUNS = {
    # name: (nchain, max_ho_dim, g, maxstates, enlarge_steps, steps, initpos)
    "n6c8": (6, 8, 1.0, 200, 1, 8, 2),
    "n16c16": (16, 16, 1.0, 1500, 1, 5, 0),
    "n32c16": (32, 16, 1.5, 2000, 1, 4, 0),
    "n25c128": (25, 128, 4.0, 1000, 1, 4, 12),
    "n8c16es0": (8, 16, 1.5, 600, 0, 6, 3),
}

TRAJ_RUNS = {
    # name: (nchain, max_ho_dim, g, maxstates, enlarge_steps, steps, initpos)
    "n8c16": (8, 16, 1.5, 4000, 1, 60, 0),
    "n16c16_m4096": (16, 16, 1.0, 4096, 1, 100, 0),
}
LONG_TRAJ_RUNS = {
    # the small plain-method configuration (open chain): N=16, g=1, maxstates=2^16, 200 steps
    "n16c16_m65536": (16, 16, 1.0, 65536, 1, 200, 0),
}


def import_reference(ref_root):
    sys.path.insert(0, os.path.join(REPO, "oracle", "refshim"))
    sys.path.insert(0, ref_root)
    import cupy  # the stand-in
    import paces
    cupy.adapt_reference(paces)
    from paces.config import devices
    if not devices.configure_called:
        devices.configure()
    return paces


def terms(g):
    return {"diag": dict(eps_sys=0.0, hbar_omega=1.0, delta_eps=0.0),
            "hopping": dict(J=1.0), "vib_coupling": dict(g=g)}


def make_objects(paces, nchain, dim, g, maxstates, es, initpos, workdir):
    from paces.models import holstein
    from paces.core.time_evolution import ExpmParams, TimeEvoParams
    from paces.config import devices
    with devices.vector_dev:
        ham = holstein.Hamiltonian(nchain=nchain, max_ho_dims=[dim] * nchain,
                                   use_terms=terms(g), debug_verb=0)
        te = holstein.TimeEvolution(ham, holstein.Observables, ["n_exc", "n_pho", "total_energy"],
                                    workdir, TimeEvoParams(maxstates=maxstates, enlarge_steps=es,
                                                           shuffle_seed=None),
                                    ExpmParams(), os.path.join(workdir, "params.log"))
        te.create_nonuniform_basis([1] * nchain, minpos=initpos, maxpos=initpos + 1)
        te.create_initial_vector([1.0], [[initpos] + [0] * nchain])
    return ham, te


def gen_layout(paces, name, nchain, dim, rng):
    from paces.models import holstein
    from paces.models._kernels import _holstein_kernels as holke
    from paces.aux import cupy_search
    from paces.aux.helpers import cupy_unique
    from paces.config import devices
    ham = holstein.Hamiltonian(nchain=nchain, max_ho_dims=[dim] * nchain, use_terms=terms(1.0),
                               debug_verb=0)
    R = 3000
    raw = np.zeros((R, nchain + 1), dtype=np.uint32)
    raw[:, 0] = rng.integers(0, nchain, R)
    # sparse occupations (most sites empty, like the physical states) plus some dense rows
    occ = rng.integers(0, dim, (R, nchain)) * (rng.random((R, nchain)) < 0.25)
    occ[: R // 10] = rng.integers(0, dim, (R // 10, nchain))
    raw[:, 1:] = occ
    keys = ham.compress_ind_arr(raw.copy())
    out = dict(raw=raw, keys=keys, bitwidths=np.asarray(ham.bitwidths_v),
               posbitwidth=np.int64(ham.posbitwidth))
    out["get_occ"] = holke.get_phonon_at_exc(keys, ham.posbitwidth, ham.qhobitwidth_v)
    n_at = out["get_occ"].astype(np.int64)
    can_up = n_at < dim - 1
    can_dn = n_at > 0
    k_up = keys[can_up].copy()
    holke.add_phonon_at_exc(k_up, ham.posbitwidth, ham.qhobitwidth_v)
    k_dn = keys[can_dn].copy()
    holke.rem_phonon_at_exc(k_dn, ham.posbitwidth, ham.qhobitwidth_v)
    out.update(can_up=can_up, can_dn=can_dn, keys_up=k_up, keys_dn=k_dn)
    out["sum_all"] = ham.sum_all_phonons(keys)
    w = rng.random(R)
    out["bath_weights"] = w
    out["bath_n_b"] = holke.calculate_bath_n_b(w, keys, ham.posbitwidth, ham.qhobitwidth_v)
    # hopping shifts via the generic field adder
    pos = raw[:, 0].astype(np.int64)
    kr = keys[pos < nchain - 1].copy()
    ham.add_n_to_pos(kr, 1)
    kl = keys[pos > 0].copy()
    ham.add_n_to_pos(kl, -1)
    out.update(keys_right=kr, keys_left=kl)
    # unique + search
    dup = np.concatenate([keys, keys[rng.integers(0, R, R // 2)]])
    uniq = cupy_unique(dup)
    out["unique_in"] = dup
    out["unique_out"] = uniq
    q_hit = uniq[rng.integers(0, len(uniq), 2000)]
    out["search_hit_q"] = q_hit
    out["search_hit_idx"] = cupy_search.searchsorted_full_binary(uniq, q_hit, False)
    q_any = ham.compress_ind_arr(np.concatenate(
        [raw[:500], np.column_stack([rng.integers(0, nchain, 500),
                                      rng.integers(0, dim, (500, nchain))])]).astype(np.uint32))
    out["search_any_q"] = q_any
    # the reference clamps nothing here: escapes come back as len(phonebook) from the CUDA
    # kernel; the stand-in clamps them to len-1, so store the boolean hit mask instead
    idx = cupy_search.searchsorted_full_binary(uniq, q_any, True)
    out["search_any_hit"] = np.all(uniq[idx] == q_any, axis=1)
    out["search_any_idx"] = idx
    np.savez_compressed(os.path.join(HERE, f"layout_{name}.npz"), **out)


def gen_stages(paces, name, cfg, workdir):
    nchain, dim, g, maxstates, es, steps, initpos = cfg
    ham, te = make_objects(paces, nchain, dim, g, maxstates, es, initpos, workdir)
    from paces.core.time_evolution import CoeffSaveParams
    rec = {}
    state = {"step": 0}

    orig_select = te._determine_select_whoami
    orig_gen = ham.generate_mel
    orig_post = te._post_assignment_diagnostics
    orig_taylor = te._simple_taylor
    orig_enlarge = ham.enlarge_basis_set

    def k(s):
        return f"s{state['step']}_{s}"

    def select(vector, **kw):
        rec[k("trunc_whoami")] = np.array(te.whoami)
        rec[k("trunc_vector")] = np.array(vector)
        out = orig_select(vector, **kw)
        rec[k("select")] = np.array(out)
        return out

    def enlarge(basis):
        out = orig_enlarge(basis)
        if k("enlarged") not in rec:
            rec[k("enlarged")] = np.array(out)
        return out

    def gen(basis, enlarge_steps=0, log_ind=1.2):
        out = orig_gen(basis, enlarge_steps=enlarge_steps, log_ind=log_ind)
        (diag, new_inds), coo, dbg = out
        rec[k("new_inds")] = np.array(new_inds)
        rec[k("diag")] = np.array(diag)
        rec[k("ceiling_hits")] = np.array([int(x) for x in dbg.get("vib_coupling", [0])])
        return out

    def post():
        rec[k("remap_vector")] = np.array(te.vector)
        for term, m in te.sparse_mats_dict.items():
            m = m.copy()
            m.sort_indices()
            rec[k(f"csr_{term}_indptr")] = m.indptr.astype(np.int64)
            rec[k(f"csr_{term}_indices")] = m.indices.astype(np.int64)
            rec[k(f"csr_{term}_data")] = m.data
        out = orig_post()
        rec[k("post_adapt")] = np.array(out, dtype=np.float64)
        return out

    def taylor(dt):
        rec[k("taylor_in")] = np.array(te.vector)
        res, dbg = orig_taylor(dt)
        rec[k("taylor_out")] = np.array(res)
        rec[k("taylor_dbg")] = np.array([float(dbg[0]), float(dbg[1]), float(dbg[2]),
                                         float(dbg[3])])
        return res, dbg

    te._determine_select_whoami = select
    ham.generate_mel = gen
    ham.enlarge_basis_set = enlarge
    te._post_assignment_diagnostics = post
    te._simple_taylor = taylor

    orig_post_proc = te._postprocess

    def postprocess(t, norm, i):
        rec[k("final_vector")] = np.array(te.vector)
        rec[k("final_whoami")] = np.array(te.whoami)
        orig_post_proc(t, norm, i)
        state["step"] += 1

    te._postprocess = postprocess
    from paces.config import devices
    with devices.vector_dev:
        te.generate_timeline(np.arange(steps + 1) * 0.05, CoeffSaveParams())
    obs = os.path.join(workdir, "observables")
    rec["n_exc"] = np.loadtxt(os.path.join(obs, "n_exc.real"))
    rec["n_pho"] = np.loadtxt(os.path.join(obs, "n_pho.real"))
    rec["energy"] = np.loadtxt(os.path.join(obs, "total_energy.real"))
    rec["diagnostics"] = np.loadtxt(os.path.join(obs, "diagnostics.log"))
    rec["config"] = np.array([nchain, dim, g, maxstates, es, steps, initpos], dtype=np.float64)
    rec["nsteps_recorded"] = np.int64(state["step"])
    np.savez_compressed(os.path.join(HERE, f"stages_{name}.npz"), **rec)


def gen_traj(paces, name, cfg, workdir):
    nchain, dim, g, maxstates, es, steps, initpos = cfg
    ham, te = make_objects(paces, nchain, dim, g, maxstates, es, initpos, workdir)
    from paces.core.time_evolution import CoeffSaveParams
    from paces.config import devices
    with devices.vector_dev:
        te.generate_timeline(np.arange(steps + 1) * 0.05, CoeffSaveParams())
    obs = os.path.join(workdir, "observables")
    np.savez_compressed(
        os.path.join(HERE, f"traj_{name}.npz"),
        n_exc=np.loadtxt(os.path.join(obs, "n_exc.real")),
        n_pho=np.loadtxt(os.path.join(obs, "n_pho.real")),
        energy=np.loadtxt(os.path.join(obs, "total_energy.real")),
        energy_imag=np.loadtxt(os.path.join(obs, "total_energy.imag")),
        diagnostics=np.loadtxt(os.path.join(obs, "diagnostics.log")),
        config=np.array([nchain, dim, g, maxstates, es, steps, initpos], dtype=np.float64))


def gen_obs_extra(paces, workdir):
    """The remaining Holstein observables on an open chain of odd length (N=7, dim 8, g=1.2,
    maxstates 3000, enlarge_steps 1, 30 steps of dt 0.05, exciton starting on site 1 -- off
    the chain's mirror axis, so no two states tie exactly at the truncation cut and the
    amplitudes themselves can be compared): hopping energy per bond and
    <mu(t) mu(0)> at every step (paces/models/holstein.py:325-357, :366-377), and for the
    last state the vibronic coupling energy per site (holstein.py:360-364, computed with the
    term's real key "vib_coupling": the reference method reads a key "coupling" that its
    matrices dictionary does not have) and the reduced density matrices of sites 0 and 3
    (paces/core/observables.py:126-163)."""
    from paces.models import holstein
    from paces.core.time_evolution import CoeffSaveParams, ExpmParams, TimeEvoParams
    from paces.config import devices
    nchain, dim, g = 7, 8, 1.2
    with devices.vector_dev:
        ham = holstein.Hamiltonian(nchain=nchain, max_ho_dims=[dim] * nchain, use_terms=terms(g), debug_verb=0)
        te = holstein.TimeEvolution(ham, holstein.Observables, ["n_exc", "hopping", "mu_to_0"], workdir,
                                    TimeEvoParams(maxstates=3000, enlarge_steps=1, shuffle_seed=None),
                                    ExpmParams(), os.path.join(workdir, "params.log"))
        te.create_nonuniform_basis([1] * nchain, minpos=1, maxpos=2)
        te.create_initial_vector([1.0], [[1] + [0] * nchain])
        te.generate_timeline(np.arange(31) * 0.05, CoeffSaveParams())
        obs = te.obsobj
        vec = te.vector
        allvals = vec.conj() * te.sparse_mats_dict["vib_coupling"].dot(vec)
        coupling = np.asarray(obs._calculate_partitioned_sum(allvals))
        rdm0 = np.asarray(obs.calculate_rdm(0, vec))
        rdm3 = np.asarray(obs.calculate_rdm(3, vec))
    od = os.path.join(workdir, "observables")
    np.savez_compressed(os.path.join(HERE, "obs_extra_n7c8.npz"),
                        hop_re=np.loadtxt(os.path.join(od, "V_hop.real")),
                        hop_im=np.loadtxt(os.path.join(od, "V_hop.imag")),
                        mu_re=np.loadtxt(os.path.join(od, "mu_to_0.real")),
                        mu_im=np.loadtxt(os.path.join(od, "mu_to_0.imag")),
                        n_exc=np.loadtxt(os.path.join(od, "n_exc.real")),
                        coupling=coupling, rdm0=rdm0, rdm3=rdm3, vector=np.asarray(vec),
                        whoami=np.asarray(te.whoami),
                        config=np.array([nchain, dim, g, 3000, 1, 30, 1], dtype=np.float64))


def gen_traj_scaled(paces, workdir):
    """The scaling-and-squaring propagation (ExpmParams(use_scaling=True): the reference's
    expm_multiply_simple on 1j * the total Hamiltonian, paces/core/time_evolution.py:579-581
    and paces/aux/_scipy/_expm_multiply.py:106-202) on an open chain, N=8, dim 16, g=1,
    maxstates 2000, 30 steps of dt 0.05, exciton starting on site 2 (off the mirror axis)."""
    from paces.models import holstein
    from paces.core.time_evolution import CoeffSaveParams, ExpmParams, TimeEvoParams
    from paces.config import devices
    nchain, dim, g = 8, 16, 1.0
    with devices.vector_dev:
        ham = holstein.Hamiltonian(nchain=nchain, max_ho_dims=[dim] * nchain, use_terms=terms(g), debug_verb=0)
        te = holstein.TimeEvolution(ham, holstein.Observables, ["n_exc", "n_pho"], workdir,
                                    TimeEvoParams(maxstates=2000, enlarge_steps=1, shuffle_seed=None),
                                    ExpmParams(use_scaling=True), os.path.join(workdir, "params.log"))
        te.create_nonuniform_basis([1] * nchain, minpos=2, maxpos=3)
        te.create_initial_vector([1.0], [[2] + [0] * nchain])
        te.generate_timeline(np.arange(31) * 0.05, CoeffSaveParams())
        vec, who = np.asarray(te.vector), np.asarray(te.whoami)
    od = os.path.join(workdir, "observables")
    np.savez_compressed(os.path.join(HERE, "scaled_n8c16.npz"),
                        n_exc=np.loadtxt(os.path.join(od, "n_exc.real")),
                        n_pho=np.loadtxt(os.path.join(od, "n_pho.real")),
                        diagnostics=np.loadtxt(os.path.join(od, "diagnostics.log")),
                        vector=vec, whoami=who,
                        config=np.array([nchain, dim, g, 2000, 1, 30, 2], dtype=np.float64))


LANCZOS_RUNS = {
    # name: (nchain, max_ho_dim, g, maxstates, steps, initpos, lanczos_order, dt)
    # open chains off their mirror axis; a short Krylov space over long steps, whose error
    # tells it from the Taylor series; and one whose Krylov space closes exactly (g = 0: the
    # exciton on the end site of a 4-site chain spans 4 vectors, then beta = 0)
    "n8c16_m12": (8, 16, 1.2, 2000, 30, 2, 12, 0.05),
    "n6c8_m25": (6, 8, 1.0, 800, 20, 1, 25, 0.05),
    "n8c16_m3_dt0.15": (8, 16, 1.2, 2000, 20, 2, 3, 0.15),
    "g0_n4c4_m10": (4, 4, 0.0, 500, 10, 0, 10, 0.05),
}


def gen_traj_lanczos(paces, name, cfg, workdir):
    """The Lanczos propagation (ExpmParams(lanczos_order=m): the reference's _lanczos,
    paces/core/time_evolution.py:515-549, selected at :577-578)."""
    from paces.models import holstein
    from paces.core.time_evolution import CoeffSaveParams, ExpmParams, TimeEvoParams
    from paces.config import devices
    nchain, dim, g, maxstates, steps, initpos, order, dt = cfg
    with devices.vector_dev:
        ham = holstein.Hamiltonian(nchain=nchain, max_ho_dims=[dim] * nchain, use_terms=terms(g), debug_verb=0)
        te = holstein.TimeEvolution(ham, holstein.Observables, ["n_exc", "n_pho", "total_energy"], workdir,
                                    TimeEvoParams(maxstates=maxstates, enlarge_steps=1, shuffle_seed=None),
                                    ExpmParams(lanczos_order=order), os.path.join(workdir, "params.log"))
        te.create_nonuniform_basis([1] * nchain, minpos=initpos, maxpos=initpos + 1)
        te.create_initial_vector([1.0], [[initpos] + [0] * nchain])
        te.generate_timeline(np.arange(steps + 1) * dt, CoeffSaveParams())
        vec, who = np.asarray(te.vector), np.asarray(te.whoami)
    od = os.path.join(workdir, "observables")
    np.savez_compressed(os.path.join(HERE, f"lanczos_{name}.npz"),
                        n_exc=np.loadtxt(os.path.join(od, "n_exc.real")),
                        n_pho=np.loadtxt(os.path.join(od, "n_pho.real")),
                        energy=np.loadtxt(os.path.join(od, "total_energy.real")),
                        diagnostics=np.loadtxt(os.path.join(od, "diagnostics.log")),
                        vector=vec, whoami=who,
                        config=np.array([nchain, dim, g, maxstates, 1, steps, initpos, order, dt], dtype=np.float64))


TAU_RUNS = {
    # name: weighting_name -- N=8, dim 16, g=1, maxstates 1500, 30 steps of dt 0.05, tau 0.2
    "tau_coherence_n8c16": "coherence",
    "tau_norm_n8c16": "norm",
}


def gen_traj_tau(paces, name, weighting, workdir):
    """The look-ahead weighting (TimeEvoParams(tau=0.2, weighting_name=...): the truncation
    ranks by coherence_weighting_func or norm_weighting_func from the second step on,
    paces/core/time_evolution.py:464-476, :560, :854-857) on an open chain, N=8, dim 16,
    g=1, maxstates 1500, 30 steps of dt 0.05, exciton starting on site 2 (off the mirror
    axis).  Stores the observables of every step and the last state."""
    from paces.models import holstein
    from paces.core.time_evolution import CoeffSaveParams, ExpmParams, TimeEvoParams
    from paces.config import devices
    nchain, dim, g, ms, tau = 8, 16, 1.0, 1500, 0.2
    with devices.vector_dev:
        ham = holstein.Hamiltonian(nchain=nchain, max_ho_dims=[dim] * nchain, use_terms=terms(g), debug_verb=0)
        te = holstein.TimeEvolution(ham, holstein.Observables, ["n_exc", "n_pho", "total_energy"], workdir,
                                    TimeEvoParams(maxstates=ms, enlarge_steps=1, shuffle_seed=None, tau=tau,
                                                  weighting_name=weighting),
                                    ExpmParams(), os.path.join(workdir, "params.log"))
        te.create_nonuniform_basis([1] * nchain, minpos=2, maxpos=3)
        te.create_initial_vector([1.0], [[2] + [0] * nchain])
        te.generate_timeline(np.arange(31) * 0.05, CoeffSaveParams())
        vec, who = np.asarray(te.vector), np.asarray(te.whoami)
    od = os.path.join(workdir, "observables")
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"),
                        n_exc=np.loadtxt(os.path.join(od, "n_exc.real")),
                        n_pho=np.loadtxt(os.path.join(od, "n_pho.real")),
                        energy=np.loadtxt(os.path.join(od, "total_energy.real")),
                        diagnostics=np.loadtxt(os.path.join(od, "diagnostics.log")),
                        vector=vec, whoami=who,
                        config=np.array([nchain, dim, g, ms, 1, 30, 2, tau], dtype=np.float64))


LATTICE_RUNS = {
    # name: (nchain, geo_dim, max_ho_dim, g, J2 or None, delta_eps, maxstates, steps, initpos)
    # delta_eps != 0 tilts the site energies, which breaks the lattice's mirror symmetries
    # (mirror-image states would tie exactly at the truncation cut)
    "geo2_n9c8": (9, 2, 8, 1.0, None, 0.13, 1500, 20, 1),
    "hop2_n8c8": (8, 1, 8, 1.2, 0.4, 0.13, 1500, 20, 2),
    "geo2hop2_n16c4": (16, 2, 4, 1.0, 0.3, 0.11, 2000, 15, 5),
    "geo3_n27c4": (27, 3, 4, 1.0, None, 0.07, 2000, 12, 4),
}


def gen_lattice(paces, name, cfg, workdir):
    """Lattices beyond the nearest-neighbour chain: geo_dim > 1 (hopping along every lattice
    dimension, paces/models/holstein.py:210-232) and the next-nearest-neighbour "hopping2"
    term (holstein.py:234-240), open boundaries.  Stores the observables of every step and
    the last state."""
    from paces.models import holstein
    from paces.core.time_evolution import CoeffSaveParams, ExpmParams, TimeEvoParams
    from paces.config import devices
    nchain, geo, dim, g, J2, deps, ms, steps, initpos = cfg
    use_terms = {"diag": dict(eps_sys=0.0, hbar_omega=1.0, delta_eps=deps), "hopping": dict(J=1.0)}
    if J2 is not None:
        use_terms["hopping2"] = dict(J2=J2)
    use_terms["vib_coupling"] = dict(g=g)
    with devices.vector_dev:
        ham = holstein.Hamiltonian(nchain=nchain, max_ho_dims=[dim] * nchain, geo_dim=geo, use_terms=use_terms,
                                   debug_verb=0)
        te = holstein.TimeEvolution(ham, holstein.Observables, ["n_exc", "n_pho", "total_energy"], workdir,
                                    TimeEvoParams(maxstates=ms, enlarge_steps=1, shuffle_seed=None),
                                    ExpmParams(), os.path.join(workdir, "params.log"))
        te.create_nonuniform_basis([1] * nchain, minpos=initpos, maxpos=initpos + 1)
        te.create_initial_vector([1.0], [[initpos] + [0] * nchain])
        te.generate_timeline(np.arange(steps + 1) * 0.05, CoeffSaveParams())
        vec, who = np.asarray(te.vector), np.asarray(te.whoami)
    od = os.path.join(workdir, "observables")
    np.savez_compressed(os.path.join(HERE, f"lattice_{name}.npz"),
                        n_exc=np.loadtxt(os.path.join(od, "n_exc.real")),
                        n_pho=np.loadtxt(os.path.join(od, "n_pho.real")),
                        energy=np.loadtxt(os.path.join(od, "total_energy.real")),
                        diagnostics=np.loadtxt(os.path.join(od, "diagnostics.log")),
                        vector=vec, whoami=who,
                        config=np.array([nchain, geo, dim, g, np.nan if J2 is None else J2, deps, ms, steps,
                                         initpos], dtype=np.float64))


def gen_fragment(paces, workdir):
    """Code fragment 3.1 of Al-Mohy and Higham (paces/aux/_scipy/_expm_multiply.py:395-450)
    on synthetic norm data: t ||A||_1 and the 1-norm estimates d(p) = ||A^p||^(1/p) (the
    estimator is bypassed, so the choice is deterministic).  Stores (m, s) per case."""
    from paces.aux._scipy import _expm_multiply as em
    rng = np.random.default_rng(7)
    cases, out = [], []
    for a1 in (5.0, 40.0, 63.0, 64.0, 80.0, 150.0, 400.0, 1000.0):
        for decay in (1.0, 0.8, 0.5, 0.2):
            d = {p: a1 * decay ** (p - 1) * (1 + 0.05 * rng.random()) for p in range(2, 11)}
            info = em.LazyOperatorNormInfo(None, A_1_norm=a1)
            info._d = dict(d)
            m, s = em._fragment_3_1(info, 1, 2.0 ** -53)
            cases.append([a1] + [d[p] for p in range(2, 11)])
            out.append([m, s])
    np.savez_compressed(os.path.join(HERE, "fragment31.npz"), cases=np.array(cases), choice=np.array(out))


def gen_ed(paces, workdir):
    """N=4, max_ho_dims=4, J=g=omega=1: the full space (1024 states) fits, so paces == exact."""
    ham, te = make_objects(paces, 4, 4, 1.0, 100000, 1, 0, workdir)
    from paces.core.time_evolution import CoeffSaveParams
    from paces.config import devices
    with devices.vector_dev:
        te.generate_timeline(np.arange(21) * 0.05, CoeffSaveParams())
    obs = os.path.join(workdir, "observables")
    np.savez_compressed(os.path.join(HERE, "ed_n4.npz"),
                        n_exc=np.loadtxt(os.path.join(obs, "n_exc.real")),
                        n_pho=np.loadtxt(os.path.join(obs, "n_pho.real")))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("reference", help="path of the reference checkout (read only)")
    ap.add_argument("--long", action="store_true", help="also the 2^16-state, 200-step run")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    paces = import_reference(os.path.abspath(args.reference))
    rng = np.random.default_rng(20260101)

    def fresh():
        d = tempfile.mkdtemp(prefix="paces_golden_")
        return d

    jobs = []
    for name, (n, d) in LAYOUTS.items():
        jobs.append((f"layout_{name}", lambda name=name, n=n, d=d: gen_layout(paces, name, n, d, rng)))
    for name, cfg in STAGE_RUNS.items():
        jobs.append((f"stages_{name}", lambda name=name, cfg=cfg: gen_stages(paces, name, cfg, fresh())))
    for name, cfg in TRAJ_RUNS.items():
        jobs.append((f"traj_{name}", lambda name=name, cfg=cfg: gen_traj(paces, name, cfg, fresh())))
    jobs.append(("ed_n4", lambda: gen_ed(paces, fresh())))
    jobs.append(("obs_extra_n7c8", lambda: gen_obs_extra(paces, fresh())))
    jobs.append(("scaled_n8c16", lambda: gen_traj_scaled(paces, fresh())))
    for name, cfg in LANCZOS_RUNS.items():
        jobs.append((f"lanczos_{name}", lambda name=name, cfg=cfg: gen_traj_lanczos(paces, name, cfg, fresh())))
    for name, weighting in TAU_RUNS.items():
        jobs.append((name, lambda name=name, w=weighting: gen_traj_tau(paces, name, w, fresh())))
    jobs.append(("fragment31", lambda: gen_fragment(paces, fresh())))
    for name, cfg in LATTICE_RUNS.items():
        jobs.append((f"lattice_{name}", lambda name=name, cfg=cfg: gen_lattice(paces, name, cfg, fresh())))
    if args.long:
        for name, cfg in LONG_TRAJ_RUNS.items():
            jobs.append((f"traj_{name}", lambda name=name, cfg=cfg: gen_traj(paces, name, cfg, fresh())))
    for jname, fn in jobs:
        if args.only and args.only not in jname:
            continue
        print("generating", jname, flush=True)
        fn()


if __name__ == "__main__":
    main()
