"""holstein: the single-exciton Holstein chain (paces/models/holstein.py).

Field 0 of a basis row is the exciton position, fields 1..N the phonon occupations of the
sites (paces/models/holstein.py:24-66).  The time step runs on the device with the terms
`hopping` (J, nearest neighbours) and `vib_coupling` (g) and the diagonal `diag`
(eps_sys, hbar_omega, delta_eps); the methods below keep the reference's model API for
custom use (images, matrix elements, observables) on device tensors.

Extensions beyond the reference: `periodic=True` (ring; the reference raises,
holstein.py:183-184) and a per-site exciton energy `use_terms["diag"]["site_eps"]`.
"""

import inspect
import sys
import time

import numpy
import torch

from .. import layout
from ..aux import cupy_search
from ..aux.helpers import cartesian_product, debug_lister, obs_attrs
from ..config import INIT_VERBOSITY_LEVEL
from ..core.hamiltonian import HamiltonianFramework, MelTriple
from ..core.observables import ObservablesFramework
from ..core.time_evolution import TimeEvolutionFramework

_DEVICE_TERMS = {"diag", "hopping", "vib_coupling"}
_OPTIONAL_TERMS = {"hopping2"}


class Hamiltonian(HamiltonianFramework):
    """Holstein Hamiltonian (paces/models/holstein.py:22-287)."""

    def __init__(self, nchain, max_ho_dims, geo_dim=1, periodic=False, **kwargs):
        self.nchain = nchain
        if nchain != len(max_ho_dims):
            raise ValueError("nchain should match the number of QHOs.")
        max_dims = [nchain] + [int(d) for d in max_ho_dims]
        self.geo_dim = geo_dim
        self.lattice_l = int(numpy.round(nchain ** (1 / geo_dim)))
        if self.lattice_l ** geo_dim != nchain:
            raise ValueError(f"Number of sites {nchain} is incompatible with dimension {geo_dim}.")
        if geo_dim > 3:
            raise NotImplementedError("the device path implements lattices of up to 3 dimensions")
        super().__init__(max_dims=max_dims, **kwargs)
        self.input_args["nchain"] = nchain
        self.input_args["max_ho_dims"] = max_ho_dims
        self.input_args["geo_dim"] = geo_dim
        terms = set(self.use_terms)
        if not (_DEVICE_TERMS <= terms <= _DEVICE_TERMS | _OPTIONAL_TERMS):
            raise NotImplementedError(f"the device path implements the terms {sorted(_DEVICE_TERMS)} (and optionally "
                                      f"{sorted(_OPTIONAL_TERMS)}); got {sorted(terms)}")
        if "hopping2" in terms and self.lattice_l - 1 < 2:
            raise ValueError("Invalid value for base_order of hopping operator.")
        self.posbitwidth = int(self.bitwidths_v[0])
        self.qhobitwidth_v = self.bitwidths_v[1:]
        self.qhobitwidth_w = self.qhobitwidth_v
        self.periodic = bool(periodic)
        if self.periodic and nchain < 3:
            raise ValueError("a periodic chain needs at least 3 sites")
        if self.periodic and (geo_dim != 1 or "hopping2" in terms):
            raise NotImplementedError("Periodic hopping not yet implemented.")

    def native_model(self):
        from ..engine import ModelParams
        d = self.use_terms["diag"]
        return ModelParams(nchain=self.nchain, max_ho_dims=[int(x) for x in self.max_dims_v[1:]],
                           J=float(numpy.real(self.use_terms["hopping"]["J"])),
                           g=float(numpy.real(self.use_terms["vib_coupling"]["g"])),
                           eps_sys=float(d["eps_sys"]), hbar_omega=float(d["hbar_omega"]),
                           delta_eps=float(d.get("delta_eps", 0.0)), periodic=self.periodic,
                           site_eps=d.get("site_eps"),
                           precision="c64" if self.complex_type == numpy.complex64 else "c128",
                           geo_dim=int(self.geo_dim),
                           J2=float(numpy.real(self.use_terms["hopping2"]["J2"])) if "hopping2" in self.use_terms
                           else None)

    # ---- fields (paces/models/holstein.py:68-147) ------------------------------------------
    def get_phonon_occ(self, arr, site):
        return self.get_n_at_site(arr, site + 1)

    def get_pos(self, arr):
        return self.get_n_at_site(arr, 0)

    def get_phonon_at_exc(self, arr):
        r64 = layout.rows_i64(arr)
        pos = layout.get_field_t(r64, self._fields, 0)
        return layout.rows_u32(layout.get_field_t(r64, self._fields, pos + 1))

    def sum_all_phonons(self, arr, omega=None):
        """Sum_s omega_s n_s per row in float64, site by site (_holstein_kernels.py:183-210)."""
        r64 = layout.rows_i64(arr)
        if omega is None:
            omega = numpy.ones(self.nchain)
        omega = numpy.broadcast_to(numpy.asarray(omega, dtype=numpy.float64), (self.nchain,))
        res = torch.zeros(r64.shape[0], dtype=torch.float64, device=r64.device)
        for s in range(self.nchain):
            res += layout.get_field_t(r64, self._fields, s + 1).to(torch.float64) * float(omega[s])
        return res

    def add_n_to_qho(self, arr, n, site):
        self.add_n_at_site(arr, n, site + 1)

    def add_n_to_pos(self, arr, n):
        self.add_n_at_site(arr, n, 0)

    def add_phonon_at_exc(self, arr):
        pos = layout.get_field_t(layout.rows_i64(arr), self._fields, 0)
        self.add_n_at_site(arr, 1, pos + 1)

    def rem_phonon_at_exc(self, arr):
        pos = layout.get_field_t(layout.rows_i64(arr), self._fields, 0)
        self.add_n_at_site(arr, -1, pos + 1)

    # ---- images and matrix elements (paces/models/holstein.py:151-287) ---------------------
    def _shift_pos(self, rows, delta):
        """Rows with the exciton moved by delta (+-1), wrapping on a ring."""
        r64 = layout.rows_i64(rows)
        pos = layout.get_field_t(r64, self._fields, 0)
        L = self.nchain
        new = (pos + delta) % L
        out = layout.add_field_t(r64, self._fields, 0, 0)
        for d in numpy.unique((new - pos).cpu().numpy()):
            sel = (new - pos) == int(d)
            out[sel] = layout.add_field_t(r64[sel], self._fields, 0, int(d))
        return layout.rows_u32(out)

    def _o_star(self, basis_states, plus_inds):
        """True where a basis row is not among the plus images (hamiltonian.py:363-374)."""
        if plus_inds.shape[0] == 0:
            return torch.ones(basis_states.shape[0], dtype=torch.bool, device=basis_states.device)
        from ..aux.helpers import cupy_unique
        idx = self.searchsorted(cupy_unique(plus_inds), basis_states, allow_escapes=True)
        return idx < 0

    def _generate_mel_hopping(self, basis_states, t_sys, base_order=1, cur_dim=0, raw_map_to=False):
        """Hop images of one channel (paces/models/holstein.py:150-207): the exciton moves by
        base_order * l**cur_dim and, with open boundaries, stays in its row of the lattice."""
        if base_order < 1 or base_order > self.lattice_l - 1:
            raise ValueError("Invalid value for base_order of hopping operator.")
        pos = layout.get_field_t(layout.rows_i64(basis_states), self._fields, 0)
        block = self.lattice_l ** (cur_dim + 1)
        order = base_order * self.lattice_l ** cur_dim
        if self.periodic:
            plus_mask = torch.ones_like(pos, dtype=torch.bool)
            minus_mask = torch.ones_like(pos, dtype=torch.bool)
        else:
            plus_mask = pos % block < block - order
            minus_mask = pos % block > order - 1
        plus_inds = self._shift_pos(basis_states[plus_mask], +order)
        minus_all = self._shift_pos(basis_states[minus_mask], -order)
        if raw_map_to:
            return [plus_inds, minus_all]
        keep = self._o_star(basis_states, plus_inds)
        mm = minus_mask & keep
        minus_inds = self._shift_pos(basis_states[mm], -order)
        return [MelTriple(plus_inds, t_sys, plus_mask), MelTriple(minus_inds, numpy.conjugate(t_sys), mm)]

    def _hopping_dim_wrapper(self, basis_states, t_sys, order, raw_map_to):
        """One channel per lattice dimension (paces/models/holstein.py:210-222)."""
        res = self._generate_mel_hopping(basis_states, t_sys, order, raw_map_to=raw_map_to)
        for d in range(1, self.geo_dim):
            res += self._generate_mel_hopping(basis_states, t_sys, base_order=order, cur_dim=d, raw_map_to=raw_map_to)
        return res if raw_map_to else (res, None)

    def generate_mel_hopping(self, basis_states, raw_map_to=False):
        """Nearest-neighbour hopping (paces/models/holstein.py:225-231)."""
        return self._hopping_dim_wrapper(basis_states, self.use_terms["hopping"]["J"], 1, raw_map_to)

    def generate_mel_hopping2(self, basis_states, raw_map_to=False):
        """Next-nearest-neighbour hopping (paces/models/holstein.py:234-240)."""
        return self._hopping_dim_wrapper(basis_states, self.use_terms["hopping2"]["J2"], 2, raw_map_to)

    @debug_lister(["ceiling_hits"])
    def generate_mel_vib_coupling(self, basis_states, raw_map_to=False):
        """b^dagger + b at the exciton site (paces/models/holstein.py:242-277)."""
        r64 = layout.rows_i64(basis_states)
        pos = layout.get_field_t(r64, self._fields, 0)
        occ = layout.get_field_t(r64, self._fields, pos + 1)
        maxd = torch.as_tensor(self.max_dims_v[1:].astype(numpy.int64), device=r64.device)[pos]
        plus_mask = occ < maxd - 1
        minus_mask = occ > 0
        plus_inds = basis_states[plus_mask].clone()
        self.add_phonon_at_exc(plus_inds)
        minus_all = basis_states[minus_mask].clone()
        self.rem_phonon_at_exc(minus_all)
        if raw_map_to:
            return plus_inds, minus_all
        ceiling_hits = int(basis_states.shape[0] - int(plus_mask.sum()))
        mm = minus_mask & self._o_star(basis_states, plus_inds)
        minus_inds = basis_states[mm].clone()
        self.rem_phonon_at_exc(minus_inds)
        g = self.use_terms["vib_coupling"]["g"]
        plus_vals = torch.sqrt(occ[plus_mask].to(torch.float64) + 1) * float(numpy.real(g))
        minus_vals = torch.sqrt(occ[mm].to(torch.float64)) * float(numpy.real(numpy.conjugate(g)))
        return (MelTriple(plus_inds, plus_vals, plus_mask), MelTriple(minus_inds, minus_vals, mm)), [ceiling_hits]

    def generate_mel_diag(self, basis_states):
        """eps_sys + hbar_omega sum(n) (+ delta_eps pos) (+ site_eps[pos]) (holstein.py:280-287)."""
        d = self.use_terms["diag"]
        vals = d["eps_sys"] + d["hbar_omega"] * self.sum_all_phonons(basis_states)
        pos = self.get_pos(basis_states).to(torch.int64)
        if d.get("delta_eps", 0) != 0:
            vals = vals + d["delta_eps"] * pos.to(torch.float64)
        if d.get("site_eps") is not None:
            vals = vals + torch.as_tensor(d["site_eps"], dtype=torch.float64, device=vals.device)[pos]
        return vals


class Observables(ObservablesFramework):
    """Holstein observables (paces/models/holstein.py:291-396)."""

    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self.hop_board = None
        self.partition_lens = None

    def primer_hook(self):
        """Lengths of the exciton-position blocks of the basis (holstein.py:299-308)."""
        blk = self.teobj._traj.basis.blk
        self.partition_lens = (blk[1:] - blk[:-1]).to(torch.int64)

    def _from_device(self, vector, key):
        cached = self.teobj._cached_observable(vector, key)
        if cached is not None:
            return cached
        return self.teobj._observables_of(vector)[key]

    @obs_attrs(fname="n_exc", header=" ".join(f"n^{{exc}}_{i}" for i in range(3)) + " etc.")
    def calculate_n_exc(self, vector):
        """Exciton density per site (holstein.py:311-314), from the device."""
        return self._from_device(vector, "n_exc")

    @obs_attrs(fname="n_pho", header=" ".join(f"n^{{pho}}_{i}" for i in range(3)) + " etc.")
    def calculate_n_pho(self, vector):
        """Phonon number per site (holstein.py:317-322), from the device."""
        return self._from_device(vector, "n_pho")

    def _terms(self, vector):
        """(hopping energy per position, vibronic energy per position, vacuum amplitude sum)
        of `vector` on the current basis, from the device (paces_term_energies)."""
        te = self.teobj
        tr = te._traj
        x = torch.zeros(max(tr.basis.cap, 1), dtype=te.engine.cdtype, device=te.engine.device)
        n = vector.numel()
        x[:n] = torch.as_tensor(vector).to(te.engine.device, te.engine.cdtype)
        return te.engine.term_energies(tr.basis, tr.h, x)

    @obs_attrs(fname="V_hop", header=" ".join(f"V_{i}" for i in range(3)) + " etc.")
    def calculate_hopping(self, vector):
        """Hopping energy per bond (holstein.py:325-357)."""
        if self.hamobj.nchain % 2 == 0 and self.hamobj.periodic:
            raise NotImplementedError("This doesn't work for even chain lengths with periodic boundary conditions.")
        hop_int_i = self._terms(vector)[0]
        if self.hop_board is None:
            nc = self.hamobj.nchain
            cb = numpy.array([[1, 0] * ((nc + 1) // 2), [0, 1] * ((nc + 1) // 2)] * ((nc + 1) // 2))[:nc, :nc]
            board = numpy.triu(cb, 1) + numpy.triu(1 - cb).T
            self.hop_board = torch.as_tensor(board, dtype=torch.complex128, device=vector.device)
        result = ((1 - self.hop_board) * hop_int_i - self.hop_board * hop_int_i.conj()).sum(dim=1)
        if self.hamobj.periodic:
            return result
        return result[:-1]

    @obs_attrs(fname="V_vib_coupl", header=" ".join(f"V_{i}" for i in range(3)) + " etc.")
    def calculate_coupling(self, vector):
        """Exciton-phonon coupling energy per site (holstein.py:360-364), from the device."""
        return self._terms(vector)[1]

    @obs_attrs(fname="mu_to_0", header=r"<mu(t) mu(0)>")
    def calculate_mu_to_0(self, vector):
        """Sum of the amplitudes on phonon-vacuum states (holstein.py:366-377), from the device."""
        return self._terms(vector)[2]

    def _calculate_partitioned_sum(self, sumvals):
        """Sum per exciton-position block (holstein.py:380-396)."""
        lens = self.partition_lens
        ids = torch.repeat_interleave(torch.arange(len(lens), device=sumvals.device), lens.to(sumvals.device))
        out = torch.zeros(len(lens), dtype=sumvals.dtype, device=sumvals.device)
        out.index_add_(0, ids, sumvals)
        return out


class TimeEvolution(TimeEvolutionFramework):
    """Holstein time evolution with its initial-basis builders (holstein.py:401-569)."""

    def _set_raw_basis(self, raw):
        rows = layout.sort_unique_rows(layout.pack_rows(numpy.asarray(raw), self.hamobj.bitwidths_v))
        self.whoami = rows

    def create_uniform_truncated_basis(self, truncate_d):
        """Every site with occupations 0..truncate_d-1, every position (holstein.py:406-425)."""
        if self.debug_verb > INIT_VERBOSITY_LEVEL:
            print("Creating initial basis set...", end=" ")
            sys.stdout.flush()
        if truncate_d > self.hamobj.max_dims_v[1:].min():
            raise ValueError("Specified basis truncation value exceeds at least one HO dimension.")
        if self.hamobj.nchain * truncate_d ** self.hamobj.nchain > self.te_params.maxstates:
            raise ValueError("Number of states that would result from this value of truncate_d exceeds maxstates!")
        self.write_current_params_to_file(inspect.currentframe())
        raw = cartesian_product(numpy.arange(self.hamobj.nchain, dtype=numpy.uint32),
                                *[numpy.arange(truncate_d, dtype=numpy.uint32)] * self.hamobj.nchain)
        self._set_raw_basis(raw)
        if self.debug_verb > INIT_VERBOSITY_LEVEL:
            print("Done!")

    def create_nonuniform_basis(self, truncate_d_list, lowest_d_list=None, minpos=0, maxpos=None):
        """Product basis with per-site ranges on positions [minpos, maxpos) (holstein.py:427-476)."""
        function_start_time = time.time()
        if self.debug_verb > INIT_VERBOSITY_LEVEL:
            print("Creating initial basis set...", end=" ")
            sys.stdout.flush()
        nchain = self.hamobj.nchain
        if maxpos is None:
            maxpos = nchain
        if lowest_d_list is None:
            lowest_d_list = numpy.zeros_like(truncate_d_list)
        if len(truncate_d_list) != nchain or len(lowest_d_list) != nchain:
            raise ValueError("Incorrect chain length.")
        if any(lowest_d_list[i] + truncate_d_list[i] > self.hamobj.max_dims_v[i + 1] for i in range(nchain)):
            raise ValueError("Specified truncation value exceeds at least one of the max_ho_dims.")
        if numpy.prod(truncate_d_list) * (maxpos - minpos) > self.te_params.maxstates:
            raise ValueError("Number of states that would result from this value of truncate_d exceeds maxstates!")
        if minpos < 0 or maxpos > nchain or minpos >= maxpos:
            raise ValueError("Invalid minpos or maxpos.")
        self.write_current_params_to_file(inspect.currentframe(), function_start_time)
        ranges = [numpy.arange(minpos, maxpos, dtype=numpy.uint32)]
        ranges += [numpy.arange(lowest_d_list[i], lowest_d_list[i] + truncate_d_list[i], dtype=numpy.uint32)
                   for i in range(nchain)]
        self._set_raw_basis(cartesian_product(*ranges))
        if self.debug_verb > INIT_VERBOSITY_LEVEL:
            print("Done!")

    def create_moving_gaussian_obc_basis(self, super_mu, super_sigma, sigma, maxval):
        """Gaussian phonon envelopes around every exciton position (holstein.py:479-526)."""
        function_start_time = time.time()
        if maxval >= self.hamobj.max_dims_v[1:].max():
            raise ValueError("Specified basis truncation value exceeds the maximal max_ho_dims.")
        self.write_current_params_to_file(inspect.currentframe(), function_start_time)
        nchain = self.hamobj.nchain

        def gauss(x, mu, s):
            return numpy.exp(-0.5 * ((x - mu) / s) ** 2)

        narr = numpy.arange(nchain)
        super_gauss = 1 + maxval * gauss(narr, super_mu, super_sigma)
        parts, total = [], 0
        for i in range(nchain):
            d = gauss(narr, i, sigma)
            part = cartesian_product(*[numpy.arange(super_gauss[i] * d[j], dtype=numpy.uint32)
                                       for j in range(nchain)])
            total += len(part)
            if total > self.te_params.maxstates:
                raise ValueError("The parameters specified for the initial basis set generate"
                                 " a basis set whose size exceeds maxstates.")
            parts.append(numpy.column_stack([numpy.full(len(part), i, dtype=numpy.uint32), part]))
        raw = numpy.concatenate(parts)
        if numpy.any(raw[:, 1:].max(axis=0) >= self.hamobj.max_dims_v[1:]):
            raise ValueError("max_ho_dims exceeded!")
        self._set_raw_basis(raw)

    def create_tensor_init_state(self, bstates, coeffs, excsite, sites="all"):
        """Localised exciton times a product of identical phonon superpositions
        (holstein.py:528-569); needs an existing basis."""
        bstates = numpy.asarray(bstates)
        coeffs = numpy.asarray(coeffs, dtype=complex)
        nchain = self.hamobj.nchain
        if sites != "all" and len(sites) > nchain:
            raise ValueError("Invalid number of sites.")
        if len(bstates) != len(coeffs):
            raise ValueError("Number of coefficients does not match number of states.")
        sitemask = numpy.ones(nchain, dtype=bool) if sites == "all" else \
            numpy.array([i in sites for i in range(nchain)])
        mat = cartesian_product(*([coeffs] * int(sitemask.sum())))
        vector = mat.prod(axis=1)
        if abs(1 - numpy.linalg.norm(vector)) > 1e-12:
            raise ValueError("State is not normalized, aborting.")
        bmask = numpy.append([False], sitemask)
        basis = numpy.zeros((len(vector), nchain + 1), dtype=numpy.int64)
        basis[:, bmask] = cartesian_product(*numpy.tile(bstates, (int(sitemask.sum()), 1)))
        basis[:, 0] = excsite
        self.create_initial_vector(vector, basis, auto_normalize=True)
