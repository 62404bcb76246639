"""Helpers shared by the GPU parity tests: build engines for fixture configurations and
turn the device neighbour table into the reference's per-term CSR matrices."""

import numpy as np
import scipy.sparse as sp

from paces_b200.engine import Engine, ModelParams


def engine_for(nchain, dim, g, cap=1 << 16, precision="c128", periodic=False, site_eps=None, J=1.0,
               hbar_omega=1.0):
    return Engine(ModelParams(nchain=nchain, max_ho_dims=[dim] * nchain, J=J, g=g, periodic=periodic,
                              site_eps=site_eps, precision=precision, hbar_omega=hbar_omega), cap=cap)


def ref_rows(eng, basis):
    return eng.basis_to_ref(basis).cpu().numpy().view(np.uint32)


def csr_from_table(eng, basis, h, J, g):
    """Per-term CSR (hopping, vib_coupling) and the diagonal, rebuilt from the neighbour table."""
    S = basis.count()
    nbr = h.nbr[:S].cpu().numpy().astype(np.int64).T
    meta = h.meta[:S].cpu().numpy().view(np.uint32).astype(np.int64)
    n = (meta >> 8) & 0xFF
    ntot = meta >> 16
    pos = meta & 0xFF
    p = eng.params
    diag = p.eps_sys + p.hbar_omega * ntot.astype(np.float64)
    if p.delta_eps != 0:
        diag = diag + p.delta_eps * pos
    rows = np.arange(S)
    mats = {}
    for term, slots in (("hopping", (0, 1)), ("vib_coupling", (2, 3))):
        r_all, c_all, v_all = [], [], []
        for s in slots:
            ok = nbr[s] >= 0
            r_all.append(rows[ok])
            c_all.append(nbr[s][ok])
            if term == "hopping":
                v_all.append(np.full(ok.sum(), float(J)))
            else:
                k = n[ok] if s == 2 else n[ok] + 1
                v_all.append(np.sqrt(k.astype(np.float64)) * float(g))
        m = sp.coo_matrix((np.concatenate(v_all), (np.concatenate(r_all), np.concatenate(c_all))),
                          shape=(S, S)).tocsr()
        m.sort_indices()
        mats[term] = m
    return diag, mats, pos


def initial_rows(nchain, dim=16, initpos=0):
    """Reference row of the exciton on site `initpos` with the phonon vacuum."""
    from paces_b200 import layout
    raw = np.zeros((1, nchain + 1), dtype=np.uint32)
    raw[0, 0] = initpos
    return layout.pack_rows(raw, layout.bitwidths_for([nchain] + [dim] * nchain))


def grown_trajectory(eng, nchain, maxstates, es=1, initpos=0, dim=16, graph=False, **traj_kw):
    """A trajectory on grow_optimal_basis(fillfac=1) with the exciton on `initpos` in the
    phonon vacuum, after its first (non-evolving) step
    (paces/core/time_evolution.py:290-323, :325-363)."""
    import torch
    from paces_b200.engine import Trajectory
    rows = initial_rows(nchain, dim, initpos)
    tr = Trajectory(eng, maxstates, es, graph=graph, **traj_kw)
    b = eng.basis_from_ref(rows)
    while True:
        nxt = eng.expand(b)
        if nxt.count() > maxstates or nxt.count() == 0:
            break
        b = nxt
    keys, pos, n = eng.query_from_ref(rows)
    idx = int(eng.lookup(b, keys, pos, n, must_exist=True)[0].item())
    psi = torch.zeros(max(b.count(), 1), dtype=eng.cdtype, device=eng.device)
    psi[idx] = 1.0
    tr.set_state(b, psi)
    first = tr.step(evolve=False)
    return tr, first


def observables_of(recs, nchain):
    return {
        "n_exc": np.array([list(r.n_exc)[:nchain] for r in recs]),
        "n_pho": np.array([list(r.n_pho)[:nchain] for r in recs]),
        "energy": np.array([r.energy_re for r in recs]),
        "norm": np.array([r.norm for r in recs]),
    }
