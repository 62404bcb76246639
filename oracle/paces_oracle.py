"""CPU oracle for the paces adaptive-basis time step (Holstein chain, single exciton).

TEST INFRASTRUCTURE ONLY.  This module is a plain NumPy/SciPy restatement of
the reference algorithm, used by `tests/`, by `__graft_entry__.smoke()` as the
checker, and by `bench.py` as the timed CPU baseline.  The product path
(`paces_b200`) never imports it.

Pinning: `tests/test_oracle_pins.py` checks every function here against golden
fixtures produced by the unmodified reference (rkevk/paces 1.2.0) run on CPU
behind `oracle/refshim` (a NumPy stand-in for CuPy); see
`tests/golden/gen_golden.py`.

Keys use the reference layout: each basis state (pos, n_0, ..., n_{N-1}) is
packed MSB-first into W uint32 words, field widths ceil(log2(max_dim)), and a
field may straddle two words (paces/core/hamiltonian.py:140-160, :218-248).

Two features the reference lacks are restated here so the same code can serve
as the oracle for the extended configurations:

* periodic=True: hopping wraps pos L-1 <-> 0 (the reference raises,
  paces/models/holstein.py:183-184).  Requires L >= 3.
* site_eps: per-site exciton energy added to the diagonal
  (paces/models/holstein.py:280-287 has only eps_sys + hbar_omega*sum(n) +
  delta_eps*pos).
With periodic=False and site_eps=None every function reduces to the reference.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np
import scipy.sparse as sp

TAYLOR_TOL_F64 = 2.0 ** -53   # paces/core/time_evolution.py:484
TAYLOR_TOL_F32 = 2.0 ** -24   # single-precision unit roundoff (paces/aux/_scipy/_expm_multiply.py)

# --------------------------------------------------------------------------------------------
# model description and key layout
# --------------------------------------------------------------------------------------------


@dataclasses.dataclass
class Model:
    """Holstein-chain parameters (paces/models/holstein.py:24-66, use_terms dict)."""
    nchain: int
    max_ho_dims: list
    J: float = 1.0
    g: float = 1.0
    eps_sys: float = 0.0
    hbar_omega: float = 1.0
    delta_eps: float = 0.0
    periodic: bool = False
    site_eps: np.ndarray | None = None
    geo_dim: int = 1             # holstein.py:24, :48-51 (lattice_l ** geo_dim == nchain)
    J2: float | None = None      # the "hopping2" term (next-nearest neighbours), holstein.py:234-240

    def __post_init__(self):
        self.max_ho_dims = [int(x) for x in self.max_ho_dims]
        if len(self.max_ho_dims) != self.nchain:
            raise ValueError("nchain should match the number of QHOs.")
        if self.periodic and self.nchain < 3:
            raise ValueError("periodic hopping needs at least 3 sites")
        self.lattice_l = int(np.round(self.nchain ** (1 / self.geo_dim)))
        if self.lattice_l ** self.geo_dim != self.nchain:
            raise ValueError(f"Number of sites {self.nchain} is incompatible with dimension {self.geo_dim}.")
        if self.periodic and (self.geo_dim != 1 or self.J2 is not None):
            raise NotImplementedError("Periodic hopping not yet implemented.")  # holstein.py:183-184
        if self.J2 is not None and self.lattice_l - 1 < 2:
            raise ValueError("Invalid value for base_order of hopping operator.")  # holstein.py:177-178
        max_dims = np.array([self.nchain] + self.max_ho_dims, dtype=np.float64)
        # hamiltonian.py:155 bitwidths = ceil(log2(max_dims))
        self.bitwidths = np.ceil(np.log2(max_dims)).astype(np.int64)
        self.posbitwidth = int(self.bitwidths[0])
        self.totwordwidth = int(math.ceil(self.bitwidths.sum() / 32))       # hamiltonian.py:160
        self.bit_offset = np.concatenate([[0], np.cumsum(self.bitwidths)[:-1]])
        if self.site_eps is not None:
            self.site_eps = np.asarray(self.site_eps, dtype=np.float64)

    @property
    def n_sites(self):
        return self.nchain + 1


def _window(keys, wi):
    """64-bit window of words (wi, wi+1) for every row (wi may vary per row)."""
    rows = np.arange(keys.shape[0])
    wi = np.broadcast_to(np.asarray(wi, dtype=np.int64), rows.shape)
    hi = keys[rows, wi].astype(np.uint64)
    has_lo = wi + 1 < keys.shape[1]
    lo = np.zeros_like(hi)
    lo[has_lo] = keys[rows[has_lo], wi[has_lo] + 1]
    return (hi << np.uint64(32)) | lo, rows, wi, has_lo


def get_field(model: Model, keys, index):
    """n at field `index` (0 = exciton position) -- paces/core/hamiltonian.py:291-318."""
    if np.ndim(index) == 0:
        # one field for every row: plain column arithmetic on the (one or two) words holding it
        i = int(index)
        b0, w = int(model.bit_offset[i]), int(model.bitwidths[i])
        wi = b0 // 32
        n2 = b0 + w - 32 * wi
        val = keys[:, wi].astype(np.uint64) << np.uint64(32)
        if wi + 1 < keys.shape[1]:
            val |= keys[:, wi + 1].astype(np.uint64)
        return ((val >> np.uint64(64 - n2)) & np.uint64((1 << w) - 1)).astype(np.uint32)
    index = np.asarray(index, dtype=np.int64)
    b0 = model.bit_offset[index]
    w = model.bitwidths[index]
    wi = b0 // 32
    n2 = b0 + w - 32 * wi
    val, *_ = _window(keys, wi)
    sh = np.broadcast_to((64 - n2).astype(np.uint64), val.shape)
    mask = (np.uint64(1) << np.broadcast_to(w.astype(np.uint64), val.shape)) - np.uint64(1)
    return ((val >> sh) & mask).astype(np.uint32)


def add_field(model: Model, keys, n, index):
    """In place: field `index` += n with carry/borrow across words.

    paces/core/hamiltonian.py:321-360 and the per-row variant
    paces/models/_kernels/_holstein_kernels.py:96-149 (index may vary per row).
    """
    index = np.asarray(index, dtype=np.int64)
    b0 = model.bit_offset[index]
    w = model.bitwidths[index]
    wi = b0 // 32
    n2 = b0 + w - 32 * wi
    val, rows, wi, has_lo = _window(keys, wi)
    inc = (np.uint64(abs(n)) << np.broadcast_to((64 - n2).astype(np.uint64), val.shape))
    val = val + inc if n > 0 else val - inc
    keys[rows, wi] = (val >> np.uint64(32)).astype(np.uint32)
    keys[rows[has_lo], wi[has_lo] + 1] = (val[has_lo] & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def set_field(model: Model, keys, values, index):
    """In place: field `index` := values (per row)."""
    cur = get_field(model, keys, index).astype(np.int64)
    values = np.broadcast_to(np.asarray(values, dtype=np.int64), cur.shape)
    up = values > cur
    dn = values < cur
    for mask, sign in ((up, 1), (dn, -1)):
        if mask.any():
            sub = keys[mask]
            delta = np.abs(values[mask] - cur[mask])
            for d in np.unique(delta):
                m2 = delta == d
                s2 = sub[m2]
                add_field(model, s2, sign * int(d), index)
                sub[m2] = s2
            keys[mask] = sub


def compress(model: Model, raw):
    """(R, N+1) occupations -> (R, W) uint32 keys.  paces/core/hamiltonian.py:218-248."""
    raw = np.asarray(raw)
    keys = np.zeros((raw.shape[0], model.totwordwidth), dtype=np.uint32)
    for i in range(model.n_sites):
        col = raw[:, i].astype(np.uint64)
        if np.any(col >= (np.uint64(1) << np.uint64(model.bitwidths[i]))):
            raise ValueError(f"occupation exceeds field width at field {i}")
        b0 = int(model.bit_offset[i])
        w = int(model.bitwidths[i])
        wi = b0 // 32
        n2 = b0 + w - 32 * wi
        val = col << np.uint64(64 - n2)
        keys[:, wi] |= (val >> np.uint64(32)).astype(np.uint32)
        if wi + 1 < model.totwordwidth:
            keys[:, wi + 1] |= (val & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    return keys


def decompress(model: Model, keys):
    """(R, W) keys -> (R, N+1) occupations.  paces/core/hamiltonian.py:210-215."""
    out = np.zeros((keys.shape[0], model.n_sites), dtype=np.uint32)
    for i in range(model.n_sites):
        out[:, i] = get_field(model, keys, i)
    return out


def get_pos(model, keys):
    return get_field(model, keys, 0).astype(np.int64)


def phonon_at_exc(model, keys):
    """paces/models/_kernels/_holstein_kernels.py:153-179 (get_occ_pte_kernel)."""
    return get_field(model, keys, get_pos(model, keys) + 1)


def sum_all_phonons(model, keys):
    """Sum_s n_s in float64, accumulated site by site (_holstein_kernels.py:183-210)."""
    res = np.zeros(keys.shape[0], dtype=np.float64)
    for s in range(model.nchain):
        res += get_field(model, keys, s + 1) * 1.0
    return res


# --------------------------------------------------------------------------------------------
# sorting, uniqueness, lookup
# --------------------------------------------------------------------------------------------


def _rows_as_bytes(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return np.ascontiguousarray(a.astype(">u4")).view(f"S{4 * a.shape[1]}").reshape(a.shape[0])


def lexsort_rows(a):
    """Row order with column 0 most significant (paces/aux/helpers.py:71)."""
    return np.lexsort(a.T[::-1])


def unique_rows(a):
    """Sorted unique rows.  paces/aux/helpers.py:63-75 (cupy_unique)."""
    if a.shape[0] == 0:
        return a.copy()
    s = a[lexsort_rows(a)]
    mask = np.empty(s.shape[0], dtype=bool)
    mask[0] = True
    mask[1:] = np.any(s[1:] != s[:-1], axis=1)
    return s[mask]


def searchsorted(phonebook, findme, allow_escapes=False):
    """Lower bound of each row of `findme` in the sorted `phonebook`.

    paces/aux/cupy_search.py:78-93 with the kernel at :149-228.  With
    allow_escapes=False every row must be present (the CUDA kernel asserts).
    Escapes return len(phonebook), as the CUDA kernel does.
    """
    if findme.shape[0] == 0:
        return np.zeros(0, dtype=np.int64)
    pb = _rows_as_bytes(phonebook)
    q = _rows_as_bytes(findme)
    left = np.searchsorted(pb, q, side="left")
    if not allow_escapes:
        hit = left < len(pb)
        hit[hit] = pb[left[hit]] == q[hit]
        if not hit.all():
            raise LookupError("a looked-up basis state is not in the phonebook")
    return left.astype(np.int64)


def lookup_with_mask(phonebook, findme):
    """(index, found) pairs; index valid only where found (used by the remap and o-star mask)."""
    idx = searchsorted(phonebook, findme, allow_escapes=True)
    found = np.zeros(idx.shape[0], dtype=bool)
    ok = idx < phonebook.shape[0]
    found[ok] = np.all(phonebook[idx[ok]] == findme[ok], axis=1)
    return idx, found


# --------------------------------------------------------------------------------------------
# Hamiltonian terms (Holstein), expansion and assembly
# --------------------------------------------------------------------------------------------


def hop_channels(model: Model):
    """The hopping channels in the reference's order: (term, J, base_order, cur_dim) for the
    "hopping" term (order 1) and then the "hopping2" term (order 2), each over the lattice
    dimensions (holstein.py:210-240, _hopping_dim_wrapper)."""
    out = [("hopping", float(model.J), 1, d) for d in range(model.geo_dim)]
    if model.J2 is not None:
        out += [("hopping2", float(model.J2), 2, d) for d in range(model.geo_dim)]
    return out


def channel_images(model: Model, basis, base_order=1, cur_dim=0):
    """Plus / minus hop images of one channel and their masks.  paces/models/holstein.py:151-207:
    the exciton moves by base_order * l**cur_dim; with open boundaries it stays inside its
    row of the l**(cur_dim+1) block.

    Returns (plus_inds, plus_mask, minus_inds_all, minus_mask): plus_inds are the images of
    basis[plus_mask]; minus_inds_all[i] is the image of basis[i] (only meaningful where
    minus_mask).
    """
    L = model.nchain
    pos = get_pos(model, basis)
    if model.periodic:
        plus_mask = np.ones(basis.shape[0], dtype=bool)
        minus_mask = np.ones(basis.shape[0], dtype=bool)
        plus = basis.copy()
        minus = basis.copy()
        set_field(model, plus, (pos + 1) % L, 0)
        set_field(model, minus, (pos - 1) % L, 0)
        return plus, plus_mask, minus, minus_mask
    block = model.lattice_l ** (cur_dim + 1)
    order = base_order * model.lattice_l ** cur_dim
    excpos_mod = pos % block
    plus_mask = excpos_mod < (block - order)
    plus = basis[plus_mask].copy()
    add_field(model, plus, order, 0)
    minus = basis.copy()
    ok = excpos_mod > order - 1
    sub = minus[ok]
    add_field(model, sub, -order, 0)
    minus[ok] = sub
    return plus, plus_mask, minus, ok


def hopping_images(model: Model, basis):
    """Nearest-neighbour hop images along the first lattice dimension (the chain's only
    channel); see channel_images."""
    return channel_images(model, basis, 1, 0)


def vib_images(model: Model, basis):
    """b^dagger / b at the exciton site.  paces/models/holstein.py:242-277."""
    occ = phonon_at_exc(model, basis).astype(np.int64)
    pos = get_pos(model, basis)
    maxd = np.asarray(model.max_ho_dims, dtype=np.int64)[pos]
    plus_mask = occ < (maxd - 1)                      # holstein.py:254 (ceiling)
    plus = basis[plus_mask].copy()
    add_field(model, plus, 1, pos[plus_mask] + 1)
    minus = basis.copy()
    # the reference subtracts on every row (holstein.py:259-260) and masks afterwards; rows
    # with n=0 would borrow from the neighbouring field, so subtract only where n>0 here --
    # the masked rows are discarded either way.
    minus_mask = occ > 0                              # holstein.py:261 (floor)
    sub = minus[minus_mask]
    add_field(model, sub, -1, pos[minus_mask] + 1)
    minus[minus_mask] = sub
    return plus, plus_mask, minus, minus_mask, occ


def enlarge(model: Model, basis):
    """basis U all raw images, unique.  paces/core/hamiltonian.py:550-577."""
    parts = [basis]
    for _, _, order, dim in hop_channels(model):
        hp, _, hm, hmm = channel_images(model, basis, order, dim)
        parts += [hp, hm[hmm]]
    vp, _, vm, vmm, _ = vib_images(model, basis)
    allk = np.concatenate(parts + [vp, vm[vmm]])
    return unique_rows(allk)


def o_star_mask(basis, plus):
    """True where a basis state is NOT a plus image.  paces/core/hamiltonian.py:363-374."""
    if plus.shape[0] == 0:
        return np.ones(basis.shape[0], dtype=bool)
    sortplus = plus[lexsort_rows(plus)]
    _, found = lookup_with_mask(sortplus, basis)
    return ~found


def diag_values(model: Model, keys):
    """eps_sys + hbar_omega*sum(n) (+ delta_eps*pos) (+ site_eps[pos]).  holstein.py:280-287."""
    d = model.eps_sys + model.hbar_omega * sum_all_phonons(model, keys)
    if model.delta_eps != 0:
        d = d + model.delta_eps * get_pos(model, keys)
    if model.site_eps is not None:
        d = d + model.site_eps[get_pos(model, keys)]
    return d


@dataclasses.dataclass
class Assembly:
    new_inds: np.ndarray           # (S, W) sorted unique keys
    diag: np.ndarray               # (S,) float64
    mats: dict                     # term -> scipy CSR (S x S), float64
    basis: np.ndarray              # the enlarged basis B1 the images were generated from
    basis_lookup: np.ndarray       # positions of B1 in new_inds
    ceiling_hits: int


def generate_mel(model: Model, select, enlarge_steps):
    """Images, unique, diagonal, lookups, COO with h.c.  paces/core/hamiltonian.py:383-547."""
    basis = select
    for _ in range(enlarge_steps):
        basis = enlarge(model, basis)
    n = basis.shape[0]
    hop = {}  # term -> [(plus, plus_mask, minus, minus_mask)] per channel, o-star applied
    for term, _, order, dim in hop_channels(model):
        hp, hpm, hm_all, hmm = channel_images(model, basis, order, dim)
        hmm = hmm & o_star_mask(basis, hp)
        hop.setdefault(term, []).append((hp, hpm, hm_all[hmm], hmm))
    vp, vpm, vm_all, vmm, occ = vib_images(model, basis)
    ceiling_hits = int(n - vpm.sum())
    vmm = vmm & o_star_mask(basis, vp)
    vm = vm_all[vmm]
    parts = [basis]
    for chans in hop.values():
        for hp, _, hm, _ in chans:
            parts += [hp, hm]
    new_inds = unique_rows(np.concatenate(parts + [vp, vm]))
    S = new_inds.shape[0]
    if S >= 2 ** 31:
        raise ValueError("The number of states is too large for signed 32-bit-integer indices.")
    diag = diag_values(model, new_inds)
    blook = searchsorted(new_inds, basis)
    g = float(model.g)
    Jt = {term: J for term, J, _, _ in hop_channels(model)}
    triples = {}
    for term, chans in hop.items():
        lst = []
        for hp, hpm, hm, hmm in chans:
            lst += [(hp, np.full(hp.shape[0], Jt[term]), hpm), (hm, np.full(hm.shape[0], Jt[term]), hmm)]
        triples[term] = lst
    triples["vib_coupling"] = [
        (vp, np.sqrt(occ[vpm] + 1, dtype=np.float64) * g, vpm),
        (vm, np.sqrt(occ[vmm], dtype=np.float64) * g, vmm),
    ]
    mats = {}
    for term, lst in triples.items():
        rows, cols, vals = [], [], []
        for inds, v, mask in lst:
            src = blook[mask]
            img = searchsorted(new_inds, inds)
            rows += [img, src]
            cols += [src, img]
            vals += [v, np.conj(v)]
        r = np.concatenate(rows)
        c = np.concatenate(cols)
        v = np.concatenate(vals)
        mats[term] = sp.coo_matrix((v, (r, c)), shape=(S, S)).tocsr()
    return Assembly(new_inds, diag, mats, basis, blook, ceiling_hits)


# --------------------------------------------------------------------------------------------
# truncation, remap, propagation, observables
# --------------------------------------------------------------------------------------------


def truncate(whoami, vector, maxstates, rng=None, weights=None):
    """Keep the `maxstates` largest |psi| states, lexicographically sorted.

    paces/core/time_evolution.py:833-910.  Stable ascending argsort of |psi| and
    the last `maxstates` entries: among equal values at the cut the highest
    original indices are kept (shuffle_seed=None).  With `rng` the tied states
    at the cut are drawn at random instead (the reference's shuffle, whose
    cuRAND stream cannot be reproduced: parity unpinned for that branch).
    `weights` (the look-ahead weights, :854-857) replace |psi| as the ranking.
    """
    w = np.abs(vector) if weights is None else np.asarray(weights)
    order = np.argsort(w, kind="stable")
    ms = int(maxstates)
    if rng is None or len(vector) < ms or w[order[-ms - 1]] < w[order[-ms]]:
        sel = order[-ms:]
    else:
        sv = w[order]
        decision = sv[-ms]
        first = np.searchsorted(sv, decision, "left")
        last = np.searchsorted(sv, decision, "right")
        if (last - first) > 0.9 * len(vector):
            raise ValueError("This operation would shuffle too many states.")
        back = len(vector) - last
        tied = order[first:last]
        sel = np.concatenate([rng.permutation(tied)[: ms - back], order[last:]])
    sel = np.sort(sel)          # whoami is sorted, so index order == lexicographic order
    return whoami[sel]


def ham_ones(asm: Assembly):
    """H applied to a vector of ones: diag + each term matrix's row sums, added in the
    terms' order.  total_ham_ones, paces/core/time_evolution.py:403-420."""
    res = asm.diag.copy()
    for m in asm.mats.values():
        res += np.asarray(m.sum(axis=1)).ravel()
    return res


def lookahead_weights(asm: Assembly, vector, tau, weighting):
    """The truncation weights with look-ahead time tau.

    coherence: |psi|^2 + tau^2 |psi|^2 (H 1)^2   (time_evolution.py:464-469)
    norm:      |psi - 1j tau H psi|              (time_evolution.py:472-476)
    """
    if weighting == "coherence":
        psi_sq = np.abs(vector) ** 2
        return psi_sq + (tau ** 2) * psi_sq * np.power(ham_ones(asm), 2)
    if weighting == "norm":
        return np.abs(vector - 1j * tau * apply_h(asm, vector))
    raise ValueError(f"unknown weighting {weighting!r}")


def remap(old_whoami, vector, new_inds):
    """New psi = old psi on states present in both bases, else 0.  time_evolution.py:781-797."""
    idx, found = lookup_with_mask(old_whoami, new_inds)
    out = np.zeros(new_inds.shape[0], dtype=vector.dtype)
    out[found] = vector[idx[found]]
    return out


def apply_h(asm: Assembly, v):
    """diag*v + sum_term CSR_term @ v.  paces/core/time_evolution.py:382-400."""
    res = asm.diag * v
    for m in asm.mats.values():
        res = res + m.dot(v)
    return res


def taylor(asm: Assembly, v, dt, m_star=100, tol=TAYLOR_TOL_F64):
    """Truncated Taylor series of exp(-i dt H) v.  paces/core/time_evolution.py:482-512.

    Returns (res, [converged, j_ind, c1_plus_c2, term_ratio]).
    """
    converged = False
    term = v
    res = v.copy()
    c1 = np.linalg.norm(res, np.inf)
    c1_plus_c2 = 0.0
    term_ratio = 0.0
    j_ind = 0
    for j_ind in range(m_star):
        coeff = -1j * dt / float(j_ind + 1)
        term = apply_h(asm, term)
        term = term * coeff
        c2 = np.linalg.norm(term, np.inf)
        res += term
        c1_plus_c2 = c1 + c2
        term_ratio = c1_plus_c2 / np.linalg.norm(res, np.inf)
        if term_ratio <= tol:
            converged = True
            break
        c1 = c2
    return res, [converged, j_ind, c1_plus_c2, term_ratio]


def lanczos(asm: Assembly, v, dt, order):
    """exp(-i dt H) v in an (order+1)-dimensional Krylov space.  paces/core/time_evolution.py:
    515-549 (_lanczos): plain Lanczos recurrence without re-orthogonalisation from v/|v|,
    alpha_i = vdot(H q_i - beta_i q_{i-1}, q_i) (complex), beta_{i+1} = |w|, a stop when
    beta < 1e-15; the (order+1)^2 tridiagonal matrix exponentiated densely and its first
    column combined with the Krylov vectors.  Returns (F, [False, 0, 0, 0]) -- the
    reference's placeholder diagnostics."""
    import scipy.linalg
    m = int(order)
    small = np.zeros((m + 1, m + 1), dtype=complex)
    vmat = np.zeros((v.shape[0], m + 1), dtype=complex)
    orig_norm = np.linalg.norm(v)
    normed = v / orig_norm
    w = apply_h(asm, normed)
    a = np.vdot(w, normed)
    w -= a * normed
    small[0, 0] = a
    vmat[:, 0] = normed
    for i in range(1, m + 1):
        b = np.linalg.norm(w)
        if b < 1e-15:
            break
        new = w / b
        w = apply_h(asm, new) - b * normed
        a = np.vdot(w, new)
        w -= a * new
        normed = new
        small[i, i] = a
        small[i - 1, i] = b
        small[i, i - 1] = b
        vmat[:, i] = normed
    leftcol = scipy.linalg.expm(-1j * dt * small)[:, 0]
    return orig_norm * (vmat @ leftcol), [False, 0, 0.0, 0.0]


# theta_m of Al-Mohy and Higham (2011), table 3.1 (m <= 30: Higham, Functions of
# Matrices, table A.3) -- the bounds paces/aux/_scipy/_expm_multiply.py:205-245 tabulates.
_THETA = {
    1: 2.29e-16, 2: 2.58e-8, 3: 1.39e-5, 4: 3.40e-4, 5: 2.40e-3, 6: 9.07e-3, 7: 2.38e-2, 8: 5.00e-2,
    9: 8.96e-2, 10: 1.44e-1, 11: 2.14e-1, 12: 3.00e-1, 13: 4.00e-1, 14: 5.14e-1, 15: 6.41e-1,
    16: 7.81e-1, 17: 9.31e-1, 18: 1.09, 19: 1.26, 20: 1.44, 21: 1.62, 22: 1.82, 23: 2.01, 24: 2.22,
    25: 2.43, 26: 2.64, 27: 2.86, 28: 3.08, 29: 3.31, 30: 3.54, 35: 4.7, 40: 6.0, 45: 7.2, 50: 8.5,
    55: 9.9,
}


def total_matrix(asm: Assembly):
    """diags(diag) + sum of the term matrices.  paces/core/time_evolution.py:375-379."""
    h = sp.diags(asm.diag).tocsr()
    for m in asm.mats.values():
        h = h + m
    return h


def expm_scaled(asm: Assembly, v, t, tol=TAYLOR_TOL_F64):
    """exp(t * 1j H) v by scaling and squaring: expm_multiply_simple(1j * H, v, t) as
    paces/core/time_evolution.py:579-581 calls it (paces/aux/_scipy/_expm_multiply.py:
    106-202).  Only the branch of fragment 3.1 that condition (3.13) selects is restated
    (the one the reference takes for t ||A - mu I||_1 below about 63).

    Returns (F, [converged, final_m, c1_plus_c2, term_ratio])."""
    A = (1j * total_matrix(asm)).tocsr()
    n = A.shape[0]
    mu = A.diagonal().sum() / float(n)
    A = (A - mu * sp.identity(n, format="csr")).tocsr()
    a1 = abs(A).sum(axis=0).max()
    if t * a1 == 0:
        m_star, s = 0, 1
    else:
        m_max, ell = 55, 2
        p = int(math.floor(math.sqrt(m_max)))
        while (p + 1) * p <= m_max + 1:
            p += 1
        if t * a1 > 2 * ell * p * (p + 3) * _THETA[m_max] / float(m_max):
            raise NotImplementedError("1-norm estimation of matrix powers (equation 3.11) is not restated")
        m_star = s = None
        for m, theta in _THETA.items():
            ss = int(math.ceil(t * a1 / theta))
            if m_star is None or m * ss < m_star * s:
                m_star, s = m, ss
    B = np.asarray(v, dtype=np.complex128)
    F = B
    eta = np.exp(t * mu / float(s))
    converged, final_m, c1_plus_c2, term_ratio = False, 0, 0.0, 0.0
    for _ in range(s):
        c1 = np.linalg.norm(B, np.inf)
        for j in range(m_star):
            final_m += 1
            coeff = t / float(s * (j + 1))
            B = coeff * A.dot(B)
            c2 = np.linalg.norm(B, np.inf)
            F = F + B
            c1_plus_c2 = c1 + c2
            term_ratio = c1_plus_c2 / np.linalg.norm(F, np.inf)
            if term_ratio <= tol:
                converged = True
                break
            c1 = c2
        if eta != 1:
            F = eta * F
        B = F
    return F, [converged, final_m, c1_plus_c2, term_ratio]


def n_exc(model, whoami, vector):
    """Sum |psi|^2 per exciton position.  paces/models/holstein.py:311-314, :380-396."""
    pos = get_pos(model, whoami)
    return np.bincount(pos, weights=np.abs(vector) ** 2, minlength=model.nchain)


def n_pho(model, whoami, vector):
    """Sum_states n_site |psi|^2 per site.  holstein.py:317-322, _holstein_kernels.py:215-255."""
    w = np.abs(vector) ** 2
    return np.array([(get_field(model, whoami, s + 1) * w).sum() for s in range(model.nchain)])


def total_energy(asm, vector):
    """<psi|H|psi>.  paces/core/observables.py:95-99."""
    return complex(np.vdot(vector, apply_h(asm, vector)))


# --------------------------------------------------------------------------------------------
# full trajectory (generate_timeline)
# --------------------------------------------------------------------------------------------


def initial_basis(model: Model, minpos, maxpos=None):
    """Single-exciton, phonon-vacuum basis on positions [minpos, maxpos).

    paces/models/holstein.py:427-476 with truncate_d_list = [1]*N.
    """
    if maxpos is None:
        maxpos = minpos + 1
    raw = np.zeros((maxpos - minpos, model.n_sites), dtype=np.uint32)
    raw[:, 0] = np.arange(minpos, maxpos)
    return compress(model, raw)


def grow_optimal_basis(model, whoami, maxstates, n_max=np.inf, fillfac=1.0):
    """paces/core/time_evolution.py:290-319."""
    n = 0
    prev = whoami
    while len(whoami) <= maxstates * fillfac:
        if n >= n_max:
            break
        n += 1
        prev = whoami
        whoami = enlarge(model, prev)
    return prev


@dataclasses.dataclass
class StepRecord:
    t: float
    norm: float
    numstates: int
    n_exc: np.ndarray
    n_pho: np.ndarray
    energy: complex
    post_adapt_norm: float
    post_adapt_energy: float
    expm_dbg: list
    ceiling_hits: int


class Trajectory:
    """A CPU run of `generate_timeline` (paces/core/time_evolution.py:426-458, :552-650)."""

    def __init__(self, model, whoami, vector, maxstates, enlarge_steps, m_star=100,
                 tol=TAYLOR_TOL_F64, diagnostics=True, shuffle_rng=None, renormalize=False,
                 explosion_cutoff=2.0, use_scaling=False, tau=0.0, weighting="coherence", lanczos_order=0):
        self.model = model
        self.whoami = whoami
        self.vector = np.asarray(vector, dtype=np.complex128)
        self.maxstates = maxstates
        self.enlarge_steps = enlarge_steps
        self.m_star = m_star
        self.tol = tol
        self.diagnostics = diagnostics
        self.rng = shuffle_rng
        self.renormalize = renormalize
        self.explosion_cutoff = explosion_cutoff
        self.use_scaling = use_scaling
        self.tau = tau
        self.weighting = weighting
        self.lanczos_order = int(lanczos_order)
        self.asm = None
        self.records = []

    def _new_space(self, weighted=False):
        """paces/core/time_evolution.py:735-807; `weighted` ranks by the look-ahead weights
        computed with the current basis' Hamiltonian (every step but the first, :560)."""
        w = None
        if weighted and self.tau != 0:
            w = lookahead_weights(self.asm, self.vector, self.tau, self.weighting)
        select = truncate(self.whoami, self.vector, self.maxstates, self.rng, weights=w)
        asm = generate_mel(self.model, select, self.enlarge_steps)
        self.vector = remap(self.whoami, self.vector, asm.new_inds)
        self.whoami = asm.new_inds
        self.asm = asm
        pan, pae = -1.0, float("nan")
        if self.diagnostics:
            pan = float(np.linalg.norm(self.vector))
            e = total_energy(asm, self.vector)
            if e.imag > 1e-12:
                raise RuntimeError(f"Energy has non-zero imaginary part: {e.imag}.")
            pae = e.real
        return pan, pae

    def _observe(self, t, expm_dbg, pan, pae):
        norm = float(np.linalg.norm(self.vector))
        rec = StepRecord(t, norm, self.whoami.shape[0], n_exc(self.model, self.whoami, self.vector),
                         n_pho(self.model, self.whoami, self.vector),
                         total_energy(self.asm, self.vector), pan, pae, expm_dbg,
                         self.asm.ceiling_hits)
        self.records.append(rec)
        return rec

    def first_step(self, t):
        """paces/core/time_evolution.py:616-650."""
        pan, pae = self._new_space()
        return self._observe(t, [0, 0, 0, 0], pan, pae)

    def step(self, t, dt):
        """paces/core/time_evolution.py:552-613."""
        pan, pae = self._new_space(weighted=True)
        if self.lanczos_order > 0:              # time_evolution.py:577-578
            self.vector, dbg = lanczos(self.asm, self.vector, dt, self.lanczos_order)
        elif self.use_scaling:
            self.vector, dbg = expm_scaled(self.asm, self.vector, dt)
        else:
            self.vector, dbg = taylor(self.asm, self.vector, dt, self.m_star, self.tol)
        nrm = np.linalg.norm(self.vector)
        if self.renormalize:
            self.vector /= nrm
        elif nrm > self.explosion_cutoff:
            raise RuntimeError("Norm has exceeded preset explosion cutoff value"
                               f" ({self.explosion_cutoff})!")
        return self._observe(t, dbg, pan, pae)

    def run(self, t_array):
        for i, t in enumerate(t_array):
            if i == 0:
                self.first_step(t)
            else:
                self.step(t, t - t_array[i - 1])
        return self.records


def exact_dynamics(model: Model, maxstates_full, t_array, init_pos=0):
    """Full-Hilbert-space reference via scipy expm_multiply (known-answer test, no truncation).

    Builds the complete basis of dimension L*prod(max_ho_dims), the full H with
    the same terms, and propagates |init_pos, vacuum>.  Returns n_exc per time.
    """
    import itertools
    import scipy.sparse.linalg as spla
    L = model.nchain
    ranges = [range(L)] + [range(d) for d in model.max_ho_dims]
    raw = np.array(list(itertools.product(*ranges)), dtype=np.uint32)
    if raw.shape[0] > maxstates_full:
        raise ValueError("Hilbert space too large for exact dynamics")
    keys = unique_rows(compress(model, raw))
    asm = generate_mel(model, keys, 0)
    H = sp.diags(asm.diag) + sum(asm.mats.values())
    init = initial_basis(model, init_pos)
    idx = searchsorted(asm.new_inds, init)
    v = np.zeros(asm.new_inds.shape[0], dtype=np.complex128)
    v[idx[0]] = 1.0
    out = []
    prev_t = t_array[0]
    for t in t_array:
        if t != prev_t:
            v = spla.expm_multiply(-1j * (t - prev_t) * H, v)
        prev_t = t
        out.append(n_exc(model, asm.new_inds, v))
    return np.array(out)
