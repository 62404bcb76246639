"""HamiltonianFramework: the Hilbert-space structure of a model (paces/core/hamiltonian.py).

Basis states are exchanged in the reference's layout: rows of uint32 words, fields packed
MSB-first with ceil(log2(max_dim)) bits each (paces/core/hamiltonian.py:140-160,
:218-248), held as torch.uint32 tensors on the GPU.  The expensive operations --
enlargement, deduplication, matrix elements, lookups -- run in libpaces_b200 on the
device; the model subclass describes itself to the library through `native_model()`.
"""

import abc
import sys
import time
from typing import NamedTuple

import numpy
import torch

from .. import layout
from ..aux.helpers import print_searchsorted_timing
from ..config import devices

if sys.version_info < (3, 10):
    raise RuntimeError("Python >= 3.10 is required.")


class MelTriple(NamedTuple):
    """Matrix elements of one term (paces/core/hamiltonian.py:27-42)."""
    inds: torch.Tensor
    vals: object
    mask: torch.Tensor


class HamiltonianFramework:
    """Abstract base of a model's Hamiltonian (paces/core/hamiltonian.py:46-172).

    A subclass provides `generate_mel_diag` and the off-diagonal terms named in
    `use_terms`, and `native_model()` returning the `paces_b200.engine.ModelParams`
    the device library evaluates.
    """
    __metaclass__ = abc.ABCMeta

    def __init__(self, max_dims, use_terms, use_complex_type=numpy.complex128, use_module=None, wordsize=32,
                 debug_verb=0, search_mindiff=32):
        if not devices.configure_called:
            raise NameError("The CUDA devices must be configured before starting the calculation"
                            " (by calling paces.config.devices.configure with appropriate args).")
        self.input_args = {"max_dims": max_dims, "use_complex_type": use_complex_type,
                           "use_module": "torch", "wordsize": wordsize,
                           "debug_verb": debug_verb, "search_mindiff": search_mindiff}
        self.use_module = torch
        self.complex_type = numpy.dtype(use_complex_type).type
        if self.complex_type not in (numpy.complex128, numpy.complex64):
            raise ValueError("use_complex_type must be numpy.complex128 or numpy.complex64")
        self.debug_verb = debug_verb
        self.search_mindiff = search_mindiff
        self.max_dims_v = numpy.asarray(max_dims)
        self.max_dims_w = self.max_dims_v
        self.n_sites = len(max_dims)
        if wordsize != 32:
            raise NotImplementedError("basis rows are exchanged as uint32 words (wordsize=32)")
        self.wordsize = 32
        self.max_word_dim = 2 ** self.wordsize
        if self.max_dims_v.max() > self.max_word_dim:
            raise ValueError("At least one of the max dimensions exceeds the word size.")
        self.dtype = numpy.uint32
        self.bitwidths_v = layout.bitwidths_for(max_dims)
        self.bitwidths_w = self.bitwidths_v
        self.totwordwidth = layout.row_words(self.bitwidths_v)
        self._fields = layout.field_table(self.bitwidths_v)
        self.use_terms = use_terms
        self.offdiag_terms = {k: self.use_terms[k] for k in self.use_terms if k != "diag"}
        self.extra_dbg_list = []
        for term in self.offdiag_terms:
            func = getattr(self, "generate_mel_" + term)
            if hasattr(func, "dbg_list"):
                self.extra_dbg_list += func.dbg_list
        self._engine = None

    # ---- device engine -------------------------------------------------------------------
    def native_model(self):
        raise NotImplementedError(f"{type(self).__name__} does not describe itself to the device library; "
                                  "only the Holstein chain is implemented on the device")

    @property
    def engine(self):
        if self._engine is None:
            from ..engine import Engine
            with devices.vector_dev:
                self._engine = Engine(self.native_model(), device=devices.vector_dev.torch)
        return self._engine

    @property
    def device(self):
        return devices.vector_dev.torch if torch.cuda.is_available() else torch.device("cpu")

    def _device_rows(self, rows64):
        return layout.rows_u32(rows64).to(self.device)

    def _basis(self, rows):
        """Sorted unique rows -> device basis."""
        r = layout.rows_i64(rows).to(torch.int32).to(self.device)
        return self.engine.basis_from_ref(r)

    # ---- lookups ---------------------------------------------------------------------------
    def searchsorted(self, phonebook, findme, allow_escapes=False):
        """Index of every row of `findme` in the sorted rows of `phonebook`
        (paces/core/hamiltonian.py:175-202).  Runs the library's lookup kernel.  With
        allow_escapes=True a missing row yields -1, an index whose row never equals the query."""
        t0 = time.time()
        eng = self.engine
        pb = self._basis(phonebook)
        q = layout.rows_i64(findme).to(torch.int32).to(self.device)
        keys, pos, n = eng.query_from_ref(q)
        out = eng.lookup(pb, keys, pos, n, must_exist=not allow_escapes)
        print_searchsorted_timing(self.debug_verb, time.time() - t0, pb.count(), n)
        return out

    # ---- packing -------------------------------------------------------------------------
    def decompress_ind_arr(self, arr):
        """Rows -> one column per field (paces/core/hamiltonian.py:210-215)."""
        r64 = layout.rows_i64(arr)
        cols = [layout.get_field_t(r64, self._fields, i) for i in range(self.n_sites)]
        return layout.rows_u32(torch.stack(cols, dim=1)) if cols else r64

    def compress_ind_arr(self, raw_states):
        """One column per field -> packed rows (paces/core/hamiltonian.py:218-248)."""
        if isinstance(raw_states, torch.Tensor):
            raw = raw_states.detach().cpu().to(torch.int64).numpy()
        else:
            raw = numpy.asarray(raw_states)
        rows = layout.pack_rows(raw, self.bitwidths_v)
        return torch.from_numpy(rows.view(numpy.int32)).to(self.device).view(torch.uint32)

    def get_n_at_site(self, arr, index):
        """Field `index` of every row (paces/core/hamiltonian.py:291-318)."""
        return layout.rows_u32(layout.get_field_t(layout.rows_i64(arr), self._fields, index))

    def add_n_at_site(self, arr, n, index):
        """In place: field `index` += n with carries across words (paces/core/hamiltonian.py:321-360).
        `index` may be one index per row."""
        if n == 0:
            return
        new = layout.add_field_t(layout.rows_i64(arr), self._fields, index, n)
        arr.view(torch.int32).copy_(new.to(torch.int32).to(arr.device))

    # ---- matrix elements -----------------------------------------------------------------
    @abc.abstractmethod
    def generate_mel_diag(self, basis_states):
        """Diagonal matrix elements of the given rows (a subclass overrides this)."""
        return

    def enlarge_basis_set(self, basis_states):
        """Basis plus all images under the off-diagonal terms, sorted and unique
        (paces/core/hamiltonian.py:550-577), computed by the device merge."""
        eng = self.engine
        out = eng.expand(self._basis(basis_states))
        return eng.basis_to_ref(out).view(torch.uint32)

    def generate_mel(self, basis_states, enlarge_steps=0, log_ind=1.2):
        """((diag_vals, new_inds), coo_dict, dbg_dict) of the given basis
        (paces/core/hamiltonian.py:383-492).  The COO triples of each term hold both
        directions of every coupling the reference's H contains."""
        if basis_states.shape[1] != self.totwordwidth:
            raise ValueError("Shape of basis states does not match the specified number of bits.")
        eng = self.engine
        b = self._basis(basis_states)
        for _ in range(enlarge_steps):
            b = eng.expand(b)
        new, h, ceil = eng.assemble(b)
        new_inds = eng.basis_to_ref(new).view(torch.uint32)
        coo, diag = hmat_to_coo(eng, new, h)
        return (diag, new_inds), coo, {"vib_coupling": [torch.tensor(ceil)]}


def hmat_to_coo(eng, basis, h):
    """Per-term COO (vals, (rows, cols)) and the diagonal from the device neighbour table."""
    S = basis.count()
    nbr = h.nbr[:S].to(torch.int64)
    meta = h.meta[:S].to(torch.int64) & 0xFFFFFFFF
    n = (meta >> 8) & 0xFF
    ntot = (meta >> 16).to(torch.float64)
    pos = (meta & 0xFF)
    p = eng.params
    diag = p.eps_sys + p.hbar_omega * ntot
    if p.delta_eps != 0:
        diag = diag + p.delta_eps * pos.to(torch.float64)
    if p.site_eps is not None:
        diag = diag + torch.as_tensor(p.site_eps, dtype=torch.float64, device=diag.device)[pos]
    rows = torch.arange(S, device=nbr.device)
    # hopping channels: channel 0 in the int4 rows, the others in xnbr (channel c >= 1 at
    # xnbr[c-1]); lattices with geo_dim d have d channels of "hopping", then d of "hopping2"
    geo = int(getattr(p, "geo_dim", 1) or 1)
    nhop = int(getattr(eng, "nhop", 1))
    cols = {0: (nbr[:, 0], nbr[:, 1])}
    for c in range(1, nhop):
        x = h.xnbr[c - 1, :S].to(torch.int64)
        cols[c] = (x[:, 0], x[:, 1])
    terms = [("hopping", float(p.J), [c for c in range(nhop) if c < geo])]
    if nhop > geo:
        terms.append(("hopping2", float(p.J2), [c for c in range(nhop) if c >= geo]))
    coo = {}
    for term, J, chans in terms:
        r_all, c_all, v_all = [], [], []
        for c in chans:
            for col in cols[c]:
                ok = col >= 0
                r_all.append(rows[ok])
                c_all.append(col[ok])
                v_all.append(torch.full((int(ok.sum()),), J, dtype=torch.float64, device=nbr.device))
        coo[term] = (torch.cat(v_all), (torch.cat(r_all), torch.cat(c_all)))
    r_all, c_all, v_all = [], [], []
    for s in (2, 3):
        ok = nbr[:, s] >= 0
        r_all.append(rows[ok])
        c_all.append(nbr[ok, s])
        k = n[ok] if s == 2 else n[ok] + 1
        v_all.append(torch.sqrt(k.to(torch.float64)) * float(p.g))
    coo["vib_coupling"] = (torch.cat(v_all), (torch.cat(r_all), torch.cat(c_all)))
    return coo, diag
