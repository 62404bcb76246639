"""Pin the CPU oracle to the reference: every oracle function against golden fixtures.

The fixtures come from the unmodified reference run on CPU (tests/golden/gen_golden.py).
Keys, sort order, dedup and lookup indices are compared bit-exactly; amplitudes and
observables to 1e-12 (complex128, summation order differs between SciPy and the
reference's NumPy stand-in only in the last bits).
"""

import glob
import os

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import paces_oracle as po

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
LAYOUTS = sorted(glob.glob(os.path.join(GOLDEN, "layout_*.npz")))
STAGES = sorted(glob.glob(os.path.join(GOLDEN, "stages_*.npz")))
TRAJS = sorted(glob.glob(os.path.join(GOLDEN, "traj_*.npz")))


def _model_from_raw(f):
    raw = f["raw"]
    nchain = raw.shape[1] - 1
    bw = f["bitwidths"]
    dim = 2 ** int(bw[1])
    return po.Model(nchain, [dim] * nchain)


@pytest.mark.parametrize("path", LAYOUTS, ids=os.path.basename)
def test_layout_pack_and_fields(path):
    f = np.load(path)
    m = _model_from_raw(f)
    assert np.array_equal(m.bitwidths, f["bitwidths"])
    keys = po.compress(m, f["raw"])
    assert np.array_equal(keys, f["keys"])
    assert np.array_equal(po.decompress(m, keys), f["raw"])
    assert np.array_equal(po.phonon_at_exc(m, keys), f["get_occ"])
    assert np.array_equal(po.sum_all_phonons(m, keys), f["sum_all"])
    pos = po.get_pos(m, keys)
    occ = po.phonon_at_exc(m, keys).astype(np.int64)
    up = keys[f["can_up"]].copy()
    po.add_field(m, up, 1, pos[f["can_up"]] + 1)
    assert np.array_equal(up, f["keys_up"])
    dn = keys[f["can_dn"]].copy()
    po.add_field(m, dn, -1, pos[f["can_dn"]] + 1)
    assert np.array_equal(dn, f["keys_dn"])
    assert np.array_equal(f["can_up"], occ < m.max_ho_dims[0] - 1)
    r = keys[pos < m.nchain - 1].copy()
    po.add_field(m, r, 1, 0)
    assert np.array_equal(r, f["keys_right"])
    l_ = keys[pos > 0].copy()
    po.add_field(m, l_, -1, 0)
    assert np.array_equal(l_, f["keys_left"])
    nb = po.n_pho(m, keys, np.sqrt(f["bath_weights"]))
    np.testing.assert_allclose(nb, f["bath_n_b"], rtol=1e-12)


@pytest.mark.parametrize("path", LAYOUTS, ids=os.path.basename)
def test_layout_unique_and_search(path):
    f = np.load(path)
    u = po.unique_rows(f["unique_in"])
    assert np.array_equal(u, f["unique_out"])
    assert np.array_equal(po.searchsorted(u, f["search_hit_q"]), f["search_hit_idx"])
    idx, found = po.lookup_with_mask(u, f["search_any_q"])
    assert np.array_equal(found, f["search_any_hit"])
    assert np.array_equal(idx[found], f["search_any_idx"][found].astype(np.int64))
    with pytest.raises(LookupError):
        if (~found).any():
            po.searchsorted(u, f["search_any_q"], allow_escapes=False)
        else:
            raise LookupError


def _stage_model(f):
    nchain, dim, g = int(f["config"][0]), int(f["config"][1]), float(f["config"][2])
    return po.Model(nchain, [dim] * nchain, g=g), int(f["config"][3]), int(f["config"][4])


@pytest.mark.parametrize("path", STAGES, ids=os.path.basename)
def test_stage_by_stage(path):
    """Each stage of each step, fed the reference's own inputs, reproduces its outputs."""
    f = np.load(path)
    m, maxstates, es = _stage_model(f)
    nsteps = int(f["nsteps_recorded"])
    assert nsteps >= 3
    for s in range(nsteps):
        k = f"s{s}_"
        sel = po.truncate(f[k + "trunc_whoami"], f[k + "trunc_vector"], maxstates)
        assert np.array_equal(sel, f[k + "select"]), f"truncation differs at step {s}"
        if es >= 1:
            assert np.array_equal(po.enlarge(m, sel), f[k + "enlarged"])
        asm = po.generate_mel(m, sel, es)
        assert np.array_equal(asm.new_inds, f[k + "new_inds"]), f"new_inds differ at step {s}"
        assert np.array_equal(asm.diag, f[k + "diag"])
        assert asm.ceiling_hits == int(f[k + "ceiling_hits"][0])
        for term, mat in asm.mats.items():
            mat = mat.copy()
            mat.sort_indices()
            assert np.array_equal(mat.indptr, f[k + f"csr_{term}_indptr"])
            assert np.array_equal(mat.indices, f[k + f"csr_{term}_indices"])
            assert np.array_equal(mat.data, f[k + f"csr_{term}_data"])
        v = po.remap(f[k + "trunc_whoami"], f[k + "trunc_vector"], asm.new_inds)
        assert np.array_equal(v, f[k + "remap_vector"])
        if k + "taylor_in" in f:
            res, dbg = po.taylor(asm, f[k + "taylor_in"], 0.05)
            np.testing.assert_allclose(res, f[k + "taylor_out"], rtol=0, atol=1e-13)
            assert dbg[0] == bool(f[k + "taylor_dbg"][0])
            assert dbg[1] == int(f[k + "taylor_dbg"][1])
        fv, fw = f[k + "final_vector"], f[k + "final_whoami"]
        np.testing.assert_allclose(po.n_exc(m, fw, fv), f["n_exc"][s, 2:], rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(po.n_pho(m, fw, fv), f["n_pho"][s, 2:], rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(po.total_energy(asm, fv).real, f["energy"][s, 2], rtol=1e-12,
                                   atol=1e-14)


@pytest.mark.parametrize("path", TRAJS, ids=os.path.basename)
def test_trajectory(path):
    """The whole oracle trajectory reproduces the reference's observables and diagnostics."""
    f = np.load(path)
    m, maxstates, es = _stage_model(f)
    steps, initpos = int(f["config"][5]), int(f["config"][6])
    if maxstates > 10000:
        pytest.skip("long trajectory: covered by the GPU parity test")
    t = np.arange(steps + 1) * 0.05
    tr = po.Trajectory(m, po.initial_basis(m, initpos), np.array([1.0 + 0j]), maxstates, es)
    recs = tr.run(t)
    ne = np.array([r.n_exc for r in recs])
    nph = np.array([r.n_pho for r in recs])
    np.testing.assert_allclose(ne, f["n_exc"][:, 2:], rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(nph, f["n_pho"][:, 2:], rtol=1e-10, atol=1e-14)
    diag = f["diagnostics"]
    assert np.array_equal(np.array([r.numstates for r in recs]), diag[:, 9].astype(int))
    assert np.array_equal(np.array([int(r.expm_dbg[1]) for r in recs]), diag[:, 6].astype(int))


def test_exact_diagonalisation_known_answer():
    """N=4, cutoff 4: the adaptive basis covers the full space, so paces == exact dynamics.

    The value at t=1 is the known answer the reference reproduces to all printed digits.
    """
    f = np.load(os.path.join(GOLDEN, "ed_n4.npz"))
    m = po.Model(4, [4] * 4)
    t = np.arange(21) * 0.05
    exact = po.exact_dynamics(m, 5000, t)
    np.testing.assert_allclose(f["n_exc"][:, 2:], exact, atol=1e-12)
    np.testing.assert_allclose(
        f["n_exc"][-1, 2:],
        [0.4217194563555634, 0.4335225805672021, 0.1270492529005554, 0.0177087101766804],
        atol=1e-15)
    tr = po.Trajectory(m, po.initial_basis(m, 0), np.array([1.0 + 0j]), 100000, 1)
    recs = tr.run(t)
    np.testing.assert_allclose(np.array([r.n_exc for r in recs]), exact, atol=1e-12)


def test_periodic_extension_reduces_and_is_exact():
    """Periodic hopping (not in the reference) against exact dynamics on the full space."""
    m = po.Model(3, [4] * 3, g=0.7, periodic=True)
    t = np.arange(11) * 0.05
    exact = po.exact_dynamics(m, 5000, t, init_pos=1)
    tr = po.Trajectory(m, po.initial_basis(m, 1), np.array([1.0 + 0j]), 100000, 1)
    recs = tr.run(t)
    np.testing.assert_allclose(np.array([r.n_exc for r in recs]), exact, atol=1e-12)
    # ring symmetry: starting on the middle site of 3, sites 0 and 2 stay equal
    np.testing.assert_allclose(exact[:, 0], exact[:, 2], atol=1e-12)


def _kron_hamiltonian(L, d, J, g, w0, site, delta_eps, periodic):
    """The Holstein Hamiltonian on the full product space |pos> (x) |n_0 ... n_{L-1}>, each
    oscillator truncated to d levels, written from its definition with Kronecker products
    and independent of the oracle's key packing, images and o-star rule:
    H = J sum_p (|p+1><p| + h.c.) + sum_p e_p |p><p| + w0 sum_s n_s
        + g sum_p |p><p| (b_p + b_p^dagger),  e_p = site[p] + delta_eps * p,
    with the hop L-1 -> 0 present when periodic.  Basis index: pos * d^L + sum_s n_s d^(L-1-s)."""
    I_d = sp.identity(d, format="csr")
    b = sp.diags(np.sqrt(np.arange(1, d, dtype=np.float64)), 1, shape=(d, d), format="csr")  # lowers n
    n_op = sp.diags(np.arange(d, dtype=np.float64), 0, format="csr")

    def on_site(op, s):
        out = sp.identity(1, format="csr")
        for k in range(L):
            out = sp.kron(out, op if k == s else I_d, format="csr")
        return out

    hop = sp.lil_matrix((L, L))
    for p in range(L - 1 if not periodic else L):
        q = (p + 1) % L
        hop[q, p] += J
        hop[p, q] += J
    ph_dim = d ** L
    H = sp.kron(hop.tocsr(), sp.identity(ph_dim, format="csr"), format="csr")
    e = np.asarray(site, dtype=np.float64) + delta_eps * np.arange(L)
    H = H + sp.kron(sp.diags(e), sp.identity(ph_dim, format="csr"), format="csr")
    nsum = sum(on_site(n_op, s) for s in range(L))
    H = H + w0 * sp.kron(sp.identity(L, format="csr"), nsum, format="csr")
    for p in range(L):
        proj = sp.csr_matrix(([1.0], ([p], [p])), shape=(L, L))
        H = H + g * sp.kron(proj, on_site(b + b.T, p), format="csr")
    return H.tocsr()


@pytest.mark.parametrize("L,d,g,w0,periodic,seed,delta_eps,init", [
    (5, 3, 0.8, 1.0, True, None, 0.0, 0),       # a ring of 5: a wrong wrap is visible
    (6, 3, 1.1, 0.7, True, 4, 0.0, 2),          # ring, site disorder, hbar_omega != 1
    (5, 3, 0.9, 1.3, False, 9, 0.25, 1),        # open chain, disorder and a linear potential
], ids=["ring5", "ring6_disorder_w0.7", "open5_disorder_linear"])
def test_extensions_against_an_independent_hamiltonian(L, d, g, w0, periodic, seed, delta_eps, init):
    """Periodic wrap, per-site energies, hbar_omega != 1 and delta_eps against exact dynamics
    of the Hamiltonian built from its definition (_kron_hamiltonian), not from the oracle's
    images: the adaptive-basis oracle run (no truncation) and the oracle's own full-space
    assembly must both equal it, n_exc and n_pho at every step."""
    import scipy.sparse.linalg as spla
    site = np.zeros(L) if seed is None else np.random.default_rng(seed).normal(0.0, 0.5, L)
    m = po.Model(L, [d] * L, g=g, hbar_omega=w0, periodic=periodic, delta_eps=delta_eps,
                 site_eps=None if seed is None else site)
    H = _kron_hamiltonian(L, d, 1.0, g, w0, site, delta_eps, periodic)
    v = np.zeros(H.shape[0], dtype=np.complex128)
    v[init * d ** L] = 1.0
    occ = np.array(list(np.ndindex(*([d] * L))), dtype=np.float64)        # [d^L, L] in index order
    t = np.arange(16) * 0.05
    exact_ne, exact_np = [], []
    for i in range(len(t)):
        if i:
            v = spla.expm_multiply(-1j * 0.05 * H, v)
        p = (np.abs(v) ** 2).reshape(L, d ** L)
        exact_ne.append(p.sum(axis=1))
        exact_np.append(p.sum(axis=0) @ occ)
    exact_ne, exact_np = np.array(exact_ne), np.array(exact_np)
    # the oracle run starts on the full space (a localised start grows its basis over the
    # first steps, and the states it has not reached yet carry ~1e-10 of phonon weight)
    import itertools
    raw = np.array(list(itertools.product(range(L), *([range(d)] * L))), dtype=np.uint32)
    full = po.unique_rows(po.compress(m, raw))
    v0 = np.zeros(full.shape[0], dtype=np.complex128)
    v0[po.searchsorted(full, po.initial_basis(m, init))[0]] = 1.0
    tr = po.Trajectory(m, full, v0, 10 ** 6, 1)
    recs = tr.run(t)
    assert recs[-1].numstates == L * d ** L
    np.testing.assert_allclose(np.array([r.n_exc for r in recs]), exact_ne, atol=1e-12)
    np.testing.assert_allclose(np.array([r.n_pho for r in recs]), exact_np, atol=1e-12)
    np.testing.assert_allclose(po.exact_dynamics(m, 10 ** 5, t, init_pos=init), exact_ne, atol=1e-12)
    if periodic:
        # the same model without the wrap is a different dynamics: the pin discriminates
        open_H = _kron_hamiltonian(L, d, 1.0, g, w0, site, delta_eps, False)
        u = np.zeros(H.shape[0], dtype=np.complex128)
        u[init * d ** L] = 1.0
        u = spla.expm_multiply(-1j * 0.75 * open_H, u)
        assert np.abs((np.abs(u) ** 2).reshape(L, -1).sum(axis=1) - exact_ne[-1]).max() > 1e-3


def test_site_disorder_extension_is_exact():
    m = po.Model(4, [3] * 4, g=0.9, site_eps=np.array([0.3, -0.2, 0.1, 0.0]))
    t = np.arange(11) * 0.05
    exact = po.exact_dynamics(m, 5000, t, init_pos=2)
    tr = po.Trajectory(m, po.initial_basis(m, 2), np.array([1.0 + 0j]), 100000, 1)
    recs = tr.run(t)
    np.testing.assert_allclose(np.array([r.n_exc for r in recs]), exact, atol=1e-12)


def test_scaling_and_squaring_matches_the_reference():
    """The oracle's expm_scaled inside a trajectory against the reference run with
    ExpmParams(use_scaling=True) (tests/golden/scaled_n8c16.npz)."""
    f = np.load(os.path.join(GOLDEN, "scaled_n8c16.npz"))
    nchain, dim, g, maxstates, es, steps, initpos = [int(x) if i != 2 else float(x) for i, x in enumerate(f["config"])]
    m = po.Model(nchain, [dim] * nchain, g=g)
    tr = po.Trajectory(m, po.initial_basis(m, initpos), np.array([1.0 + 0j]), maxstates, es, use_scaling=True)
    recs = tr.run(np.arange(steps + 1) * 0.05)
    ne = np.array([r.n_exc for r in recs])
    np.testing.assert_allclose(ne, f["n_exc"][:, 2:], rtol=1e-10, atol=1e-13)
    diag = f["diagnostics"]
    assert [r.numstates for r in recs] == diag[:, 9].astype(int).tolist()
    assert [int(r.expm_dbg[1]) for r in recs[1:]] == diag[1:, 6].astype(int).tolist()
    assert np.array_equal(tr.whoami, f["whoami"])
    np.testing.assert_allclose(tr.vector, f["vector"], rtol=0, atol=1e-13)


@pytest.mark.parametrize("weighting", ["coherence", "norm"])
def test_lookahead_weighting_matches_the_reference(weighting):
    """The oracle's look-ahead weighting (coherence_weighting_func / norm_weighting_func
    ranking the truncation from the second step on) against the reference's runs with
    TimeEvoParams(tau=0.2) (tests/golden/tau_<weighting>_n8c16.npz), and the fixture
    discriminates: ranking by |psi| alone ends in another basis."""
    f = np.load(os.path.join(GOLDEN, f"tau_{weighting}_n8c16.npz"))
    nchain, dim, g, maxstates, es, steps, initpos, tau = f["config"]
    nchain, dim, maxstates, es, steps, initpos = (int(x) for x in (nchain, dim, maxstates, es, steps, initpos))
    m = po.Model(nchain, [dim] * nchain, g=float(g))
    runs = {}
    for t in (float(tau), 0.0):
        tr = po.Trajectory(m, po.initial_basis(m, initpos), np.array([1.0 + 0j]), maxstates, es, tau=t,
                           weighting=weighting)
        runs[t] = (tr, tr.run(np.arange(steps + 1) * 0.05))
    tr, recs = runs[float(tau)]
    np.testing.assert_allclose(np.array([r.n_exc for r in recs]), f["n_exc"][:, 2:], rtol=1e-10, atol=1e-14)
    assert [r.numstates for r in recs] == f["diagnostics"][:, 9].astype(int).tolist()
    assert np.array_equal(tr.whoami, f["whoami"])
    np.testing.assert_allclose(tr.vector, f["vector"], rtol=0, atol=1e-14)
    plain = runs[0.0][0]
    assert plain.whoami.shape != f["whoami"].shape or not np.array_equal(plain.whoami, f["whoami"])


@pytest.mark.parametrize("name", ["geo2_n9c8", "hop2_n8c8", "geo2hop2_n16c4", "geo3_n27c4"])
def test_lattices_match_the_reference(name):
    """The oracle's hopping channels (geo_dim > 1: hopping along every lattice dimension;
    the next-nearest-neighbour hopping2 term) against the reference's own runs
    (tests/golden/lattice_<name>.npz): observables at every step, basis sizes, the final
    basis and amplitudes."""
    f = np.load(os.path.join(GOLDEN, f"lattice_{name}.npz"))
    nchain, geo, dim, g, J2, deps, ms, steps, initpos = f["config"]
    nchain, geo, dim, ms, steps, initpos = (int(x) for x in (nchain, geo, dim, ms, steps, initpos))
    m = po.Model(nchain, [dim] * nchain, g=float(g), geo_dim=geo, J2=None if np.isnan(J2) else float(J2),
                 delta_eps=float(deps))
    tr = po.Trajectory(m, po.initial_basis(m, initpos), np.array([1.0 + 0j]), ms, 1)
    recs = tr.run(np.arange(steps + 1) * 0.05)
    np.testing.assert_allclose(np.array([r.n_exc for r in recs]), f["n_exc"][:, 2:], rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(np.array([r.n_pho for r in recs]), f["n_pho"][:, 2:], rtol=1e-10, atol=1e-14)
    assert [r.numstates for r in recs] == f["diagnostics"][:, 9].astype(int).tolist()
    assert np.array_equal(tr.whoami, f["whoami"])
    np.testing.assert_allclose(tr.vector, f["vector"], rtol=0, atol=1e-14)


def test_lattice_model_validation():
    with pytest.raises(ValueError):
        po.Model(10, [4] * 10, geo_dim=2)              # 10 is not a square
    with pytest.raises(ValueError):
        po.Model(4, [4] * 4, geo_dim=2, J2=0.5)        # l = 2: no next-nearest neighbour
    with pytest.raises(NotImplementedError):
        po.Model(9, [4] * 9, geo_dim=2, periodic=True)


LANCZOS = sorted(glob.glob(os.path.join(GOLDEN, "lanczos_*.npz")))


@pytest.mark.parametrize("path", LANCZOS, ids=os.path.basename)
def test_lanczos_matches_the_reference(path):
    """The oracle's Lanczos propagation inside a trajectory against the reference's runs with
    ExpmParams(lanczos_order=m) (tests/golden/lanczos_*.npz): observables at every step,
    basis sizes, the placeholder diagnostics, the final basis and amplitudes."""
    f = np.load(path)
    nchain, dim, g, ms, es, steps, initpos, order, dt = f["config"]
    nchain, dim, ms, es, steps, initpos, order = (int(x) for x in (nchain, dim, ms, es, steps, initpos, order))
    m = po.Model(nchain, [dim] * nchain, g=float(g))
    t = np.arange(steps + 1) * float(dt)
    tr = po.Trajectory(m, po.initial_basis(m, initpos), np.array([1.0 + 0j]), ms, es, lanczos_order=order)
    recs = tr.run(t)
    np.testing.assert_allclose(np.array([r.n_exc for r in recs]), f["n_exc"][:, 2:], rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(np.array([r.n_pho for r in recs]), f["n_pho"][:, 2:], rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(np.array([r.norm for r in recs]), f["n_exc"][:, 1], rtol=1e-12)
    diag = f["diagnostics"]
    assert [r.numstates for r in recs] == diag[:, 9].astype(int).tolist()
    assert np.all(diag[1:, 5:9] == 0)      # [False, 0, 0, 0]: the reference's placeholder
    assert np.array_equal(tr.whoami, f["whoami"])
    np.testing.assert_allclose(tr.vector, f["vector"], rtol=0, atol=1e-13)
    # the fixture tells the Krylov path from the Taylor series: the latter records its term
    # counts and stop flags where the Lanczos step writes the placeholder
    taylor = po.Trajectory(m, po.initial_basis(m, initpos), np.array([1.0 + 0j]), ms, es)
    t_recs = taylor.run(t[:3])
    assert int(t_recs[1].expm_dbg[1]) > 0 and bool(t_recs[1].expm_dbg[0])
    if order < 5:  # and a short Krylov space over long steps moves the observables
        dev = np.abs(np.array([r.n_exc for r in t_recs]) - f["n_exc"][:3, 2:]).max()
        assert dev > 1e-6, dev
