"""TimeEvolutionFramework: the adaptive-basis time evolution (paces/core/time_evolution.py).

Every time step runs as one `paces_step` call of libpaces_b200 on the GPU (truncation,
enlargement, merge-based sort/unique, Hamiltonian table, amplitude remap, the whole
Taylor series and the observables) and returns one small record; this module keeps the
reference's API, parameter dataclasses, checks and output files around it.
"""

import abc
import inspect
import os
import pprint
import sys
import time
from dataclasses import dataclass
from typing import Optional

import numpy
import torch

from .. import __version__
from .. import layout
from ..config import (BASE_STEP_LEVEL, HILBERT_SPACE_LEVEL, INIT_VERBOSITY_LEVEL, MEM_INFO_LEVEL, devices)
from .hamiltonian import hmat_to_coo


@dataclass
class CoeffSaveParams:
    """When to save the wavefunction and its basis (paces/core/time_evolution.py:27-53)."""
    save_every: int = 0
    save_first: bool = False
    save_last: bool = False
    max_i: int = 0

    def save_necessary(self, i: int):
        if self.max_i == 0:
            raise ValueError("max_i should be set before calling this method.")
        necessary = (self.save_first and i == 0)
        necessary |= (self.save_last and i == self.max_i)
        if self.save_every != 0:
            necessary |= (self.save_every is not None and i % self.save_every == 0)
        return necessary


@dataclass
class ExpmParams:
    """Matrix-exponential parameters (paces/core/time_evolution.py:57-82).

    The device runs the truncated Taylor series; with lanczos_order > 0 the Lanczos step
    (paces_lanczos, which takes precedence as in the reference, time_evolution.py:577-580),
    else with use_scaling=True the scaling-and-squaring series of paces_b200.expm.
    """
    m_star: int = 100
    explosion_cutoff: float = 2.0
    use_scaling: bool = False
    renormalize: bool = False
    lanczos_order: int = 0


@dataclass
class TimeEvoParams:
    """Time-evolution parameters (paces/core/time_evolution.py:85-119)."""
    maxstates: int
    enlarge_steps: int
    diagnostics: bool = True
    shuffle_seed: Optional[int] = 0
    weighting_name: str = "coherence"
    tau: float = 0.0
    garbage_tol: float = -1
    use_two_streams: bool = False


class TimeEvolutionFramework:
    """Abstract base of the time evolution of a model (paces/core/time_evolution.py:124-211)."""
    __metaclass__ = abc.ABCMeta

    def __init__(self, hamobj, ObsObj, obs_list, dirname, te_params, expm_params, params_file=None):
        self.use_module = hamobj.use_module
        self.debug_verb = hamobj.debug_verb
        self.start_time = time.time()
        if self.debug_verb > INIT_VERBOSITY_LEVEL:
            print("Initializing TimeEvolution object...")
        self.hamobj = hamobj
        self.dirname = dirname
        self.te_params = te_params
        self.expm_params = expm_params
        self.weighting_func = getattr(self, te_params.weighting_name + "_weighting_func")
        if not os.path.exists(self.dirname):
            raise FileNotFoundError(f"The results directory {self.dirname} does not exist.")
        self.obsobj = ObsObj(self, obs_list)
        self.ham_mat = None
        self.cso = None
        self.wf_name_list = None
        self.log_ind = 0
        real_valued = all(all(numpy.imag(value) == 0 for value in paramdict.values()
                              if numpy.isscalar(value))
                          for paramdict in self.hamobj.use_terms.values())
        if not real_valued:
            raise NotImplementedError("Not all functions have been adapted to complex-valued"
                                      " off-diagonal Hamiltonian matrix elements.")
        if params_file is None:
            self.params_file = os.path.join(self.dirname, "paces_params_run_" + str(time.time()) + ".log")
        else:
            self.params_file = params_file
        self.initialize_params_file()
        # device state: staged basis/vector until a trajectory exists
        self._traj = None
        self._staged_basis = None
        self._staged_vector = None
        self._whoami_cache = None
        self._obs_cache = None
        if self.debug_verb > INIT_VERBOSITY_LEVEL:
            print("Finished initialization of TimeEvolution object!\n")

    # ---- parameters file (paces/core/time_evolution.py:217-264) ----------------------------
    def initialize_params_file(self):
        ver_string = f"### paces version {__version__} ###"
        hashes = "#" * len(ver_string) + "\n"
        with open(self.params_file, "w", encoding="utf-8") as pf:
            pf.write(hashes)
            pf.write(ver_string + "\n")
            pf.write(hashes + "\n")
            pf.write(devices.desc_str)
            pf.write("### Hilbert space constructed from"
                     f" {self.hamobj.__class__.__module__}.{self.hamobj.__class__.__name__}"
                     " with the following parameters:\n")
            pf.write(pprint.pformat(self.hamobj.input_args, compact=True) + "\n")
            pf.write("\n### Hamiltonian terms and their parameters:\n")
            pf.write(pprint.pformat(self.hamobj.use_terms, width=1) + "\n")
            pf.write("\n### Observables constructed from"
                     f" {self.obsobj.__class__.__module__}.{self.obsobj.__class__.__name__}"
                     " with the following observables:\n")
            pf.write(pprint.pformat([*self.obsobj.obs_dict]) + "\n")
            pf.write("\n### TimeEvolution constructed from"
                     f" {self.__class__.__module__}.{self.__class__.__name__}"
                     " with the following parameters:\n")
            pf.write(pprint.pformat(self.te_params) + "\n")
            pf.write(pprint.pformat(self.expm_params) + "\n")
            pf.write("\n### End of initialization parameter list\n"
                     "#################################################################\n")

    def write_current_params_to_file(self, frame, start_time=None):
        if start_time is None:
            start_time = time.time()
        localtime = time.asctime(time.localtime(start_time))
        args, _, _, values = inspect.getargvalues(frame)
        arg_list = [(str(i) + "=" + str(values[i])) for i in args if str(i) != "self"]
        mod_obj = f"{self.__class__.__module__}.{self.__class__.__name__}"
        header = f"\nFunction call in {mod_obj} at {start_time} ({localtime} local):\n"
        header += f"  {frame.f_code.co_name}(\n    " + ",\n    ".join(arg_list) + ")\n"
        with open(self.params_file, "a", encoding="utf-8") as params_file:
            params_file.write(header)

    # ---- device state ----------------------------------------------------------------------
    @property
    def engine(self):
        return self.hamobj.engine

    def _trajectory(self):
        if self._traj is None:
            from ..engine import Trajectory
            from .. import _native as nat
            tp, ep = self.te_params, self.expm_params
            weighting = nat.WEIGHT_NONE
            if tp.tau != 0:
                weighting = {"coherence": nat.WEIGHT_COHERENCE, "norm": nat.WEIGHT_NORM}[tp.weighting_name]
            self._traj = Trajectory(self.engine, tp.maxstates, tp.enlarge_steps, m_star=ep.m_star,
                                    diagnostics=tp.diagnostics, shuffle_seed=tp.shuffle_seed,
                                    renormalize=ep.renormalize, explosion_cutoff=ep.explosion_cutoff,
                                    weighting=weighting, tau=tp.tau, lanczos_order=ep.lanczos_order)
        return self._traj

    def _commit_state(self):
        """Move a staged basis/vector into the trajectory's buffers."""
        if self._staged_basis is None:
            return
        b = self._staged_basis
        v = self._staged_vector
        if v is None:
            v = torch.zeros(b.count(), dtype=self.engine.cdtype, device=self.engine.device)
        self._trajectory().set_state(b, v)
        self._staged_basis = None
        self._staged_vector = None

    @property
    def whoami(self):
        """The current basis as reference rows (torch.uint32 on the GPU, sorted)."""
        if self._staged_basis is not None:
            return self.engine.basis_to_ref(self._staged_basis).view(torch.uint32)
        if self._traj is None:
            return None
        if self._whoami_cache is None:
            self._whoami_cache = self.engine.basis_to_ref(self._traj.basis).view(torch.uint32)
        return self._whoami_cache

    @whoami.setter
    def whoami(self, rows):
        self._staged_basis = self.engine.basis_from_ref(layout.rows_i64(rows).to(torch.int32).to(self.engine.device))
        self._staged_vector = None
        self._whoami_cache = None
        self._obs_cache = None

    @property
    def numstates(self):
        if self._staged_basis is not None:
            return self._staged_basis.count()
        return None if self._traj is None else self._traj.basis.count()

    @property
    def vector(self):
        """The current state (complex tensor on the GPU, one amplitude per basis row)."""
        if self._staged_basis is not None:
            return self._staged_vector
        return None if self._traj is None else self._traj.vector

    @vector.setter
    def vector(self, v):
        v = torch.as_tensor(v).to(self.engine.device, self.engine.cdtype)
        if self._staged_basis is not None:
            self._staged_vector = v
        else:
            self._trajectory().vector.copy_(v)
        self._obs_cache = None

    @property
    def sparse_mats_dict(self):
        """Per-term sparse matrices of the current H (torch sparse CSR, float64)."""
        if self._traj is None or self._traj.last is None:
            return None
        coo, _ = hmat_to_coo(self.engine, self._traj.basis, self._traj.h)
        S = self.numstates
        out = {}
        for term, (vals, (rows, cols)) in coo.items():
            out[term] = torch.sparse_coo_tensor(torch.stack([rows, cols]), vals, (S, S)).coalesce().to_sparse_csr()
        return out

    @property
    def diag_vals(self):
        if self._traj is None or self._traj.last is None:
            return None
        return hmat_to_coo(self.engine, self._traj.basis, self._traj.h)[1]

    # ---- initial basis (paces/core/time_evolution.py:271-359) ------------------------------
    def load_basis_from_file(self, loadfile):
        function_start_time = time.time()
        if self.debug_verb > INIT_VERBOSITY_LEVEL:
            print("Loading basis set from file...", end=" ")
            sys.stdout.flush()
        self.write_current_params_to_file(inspect.currentframe(), function_start_time)
        rows = numpy.load(loadfile)
        if rows.shape[1] != self.hamobj.totwordwidth:
            raise ValueError("Loaded basis set doesn't match total number of bits given by hamobj.")
        if rows.dtype != self.hamobj.dtype:
            raise ValueError("Loaded basis set does not match wordsize given by hamobj.")
        self.whoami = rows
        if self.debug_verb > INIT_VERBOSITY_LEVEL:
            print("Done!")

    def grow_optimal_basis(self, n_max=numpy.inf, fillfac=1.0):
        """Enlarge the basis repeatedly while it has at most fillfac*maxstates states
        (paces/core/time_evolution.py:290-319); each enlargement is one device merge."""
        function_start_time = time.time()
        if self.debug_verb > INIT_VERBOSITY_LEVEL:
            print("Growing initial basis set...", end=" ")
            sys.stdout.flush()
        self.write_current_params_to_file(inspect.currentframe(), function_start_time)
        eng = self.engine
        cur = self._staged_basis if self._staged_basis is not None else eng.basis_from_ref(
            self.whoami.view(torch.int32))
        eng._grow(int(2.5 * self.te_params.maxstates * max(fillfac, 1.0)) + 1024)
        initsize = cur.count()
        prev, n = cur, 0
        while cur.count() <= self.te_params.maxstates * fillfac:
            if n >= n_max:
                break
            n += 1
            prev = cur
            cur = eng.expand(prev)
        self._staged_basis = prev
        self._staged_vector = None
        if self.debug_verb > INIT_VERBOSITY_LEVEL:
            print(f"Done! Performed {n} enlargements (grew from {initsize} to {prev.count()} states).")

    def create_initial_vector(self, vector_coeffs, vector_coo, auto_normalize=True):
        """Amplitudes on the given (pos, n_0, ...) coordinates (paces/core/time_evolution.py:325-359)."""
        if self.debug_verb > INIT_VERBOSITY_LEVEL:
            print("Creating the initial state vector...", end=" ")
            sys.stdout.flush()
        vector_coo = numpy.asarray(vector_coo.cpu() if isinstance(vector_coo, torch.Tensor) else vector_coo)
        if vector_coo.ndim != 2:
            raise ValueError("The coo list must be 2D (even if it contains only the entry for one basis state).")
        if numpy.unique(vector_coo, axis=0).shape != vector_coo.shape:
            raise ValueError("There are duplicates in the specified vector coordinates.")
        if vector_coo.shape[0] != len(vector_coeffs):
            raise ValueError("The number of coefficients does not match the number of coordinates.")
        coeffs = numpy.asarray(vector_coeffs, dtype=numpy.complex128)
        if auto_normalize:
            coeffs = coeffs / numpy.linalg.norm(coeffs)
        rows = self.hamobj.compress_ind_arr(vector_coo)
        if self._staged_basis is None:
            self._staged_basis = self.engine.basis_from_ref(self.whoami.view(torch.int32))
        idx = self.hamobj.searchsorted(self.whoami, rows, allow_escapes=False)
        v = torch.zeros(self._staged_basis.count(), dtype=self.engine.cdtype, device=self.engine.device)
        v[idx] = torch.as_tensor(coeffs).to(v.device, v.dtype)
        self._staged_vector = v
        if self.debug_verb > INIT_VERBOSITY_LEVEL:
            print("Done!")

    # ---- Hamiltonian on the current basis -----------------------------------------------------
    def create_matrices(self, diag_params, coo_dict):
        raise NotImplementedError("the Hamiltonian is assembled on the device by every time step")

    def create_ham_mat(self):
        """The total Hamiltonian of the current basis as self.ham_mat (paces/core/time_evolution.py:
        375-379): here a device operator over the step's neighbour table (HamiltonianOperator),
        not an assembled sparse matrix; `ham_mat @ v`, `1j * ham_mat` and
        paces.aux.expm_multiply_simple(1j * ham_mat, v, t) run on the GPU."""
        self.ham_mat = HamiltonianOperator(self)
        return self.ham_mat

    def total_ham(self, vector, use_ham_mat=False):
        """H applied to a vector of the current basis (paces/core/time_evolution.py:382-400)."""
        if use_ham_mat:
            if self.ham_mat is None:
                raise ValueError("use_ham_mat=True needs create_ham_mat() first")
            return self.ham_mat @ vector
        x = torch.as_tensor(vector).to(self.engine.device, self.engine.cdtype).contiguous()
        return self.engine.apply_h(self._traj.basis, self._traj.h, x)

    def _weights(self, vector, tau, weighting):
        """Per-state weights of `vector` on the current basis, computed by the device."""
        n = self.numstates
        x = torch.zeros(max(self._traj.basis.cap, 1), dtype=self.engine.cdtype, device=self.engine.device)
        if vector is not None:
            x[:n] = torch.as_tensor(vector).to(self.engine.device, self.engine.cdtype)[:n]
        return self.engine.lookahead_weights(self._traj.basis, self._traj.h, x, tau, weighting)

    def total_ham_ones(self, use_ham_mat=False):
        """H applied to a vector of ones: diag + the row sums of every term matrix
        (paces/core/time_evolution.py:403-420), float64 on the GPU.  (The reference adds the
        row sums into its diag_vals array in place; here the diagonal is left unchanged.)
        use_ham_mat gives the same numbers: the operator is the same device H."""
        from .. import _native as nat
        return self._weights(None, 0.0, nat.WEIGHT_HAM_ONES)

    def coherence_weighting_func(self, vector, tau):
        """|psi|^2 + tau^2 |psi|^2 (H 1)^2 per state (paces/core/time_evolution.py:464-469)."""
        from .. import _native as nat
        return self._weights(vector, tau, nat.WEIGHT_COHERENCE)

    def norm_weighting_func(self, vector, tau):
        """|psi - 1j tau H psi| per state (paces/core/time_evolution.py:472-476)."""
        from .. import _native as nat
        return self._weights(vector, tau, nat.WEIGHT_NORM)

    # ---- propagation on the current basis --------------------------------------------------
    def _simple_taylor(self, delta_t):
        """exp(-i dt H) applied to the current vector by the device Taylor series
        (paces/core/time_evolution.py:482-512); returns (result, [converged, j, c1+c2, ratio])."""
        out, dbg = self.engine.taylor(self._traj.basis, self._traj.h, self._traj.psis[self._traj.cur], delta_t,
                                      self.expm_params.m_star)
        return out[: self.numstates], dbg

    def _lanczos(self, delta_t):
        raise NotImplementedError("Lanczos propagation (lanczos_order > 0) is not implemented")

    # ---- observables cache -------------------------------------------------------------------
    def _cached_observable(self, vector, key):
        if self._obs_cache is None or self._traj is None:
            return None
        cur = self._traj.vector
        if vector is None or vector.data_ptr() != cur.data_ptr() or vector.numel() != cur.numel():
            return None
        return self._obs_cache.get(key)

    def _observables_of(self, vector):
        x = torch.zeros(self._traj.basis.cap, dtype=self.engine.cdtype, device=self.engine.device)
        x[: vector.numel()] = vector.to(self.engine.cdtype)
        return self.engine.observables(self._traj.basis, self._traj.h, x)

    # ---- the timeline (paces/core/time_evolution.py:426-458, :552-650) -----------------------
    def generate_timeline(self, t_array, coeff_save_obj):
        if self.debug_verb > INIT_VERBOSITY_LEVEL:
            print("Setting up generate_timeline function...")
        self.write_current_params_to_file(inspect.currentframe(), time.time())
        ep, tp = self.expm_params, self.te_params
        if tp.garbage_tol >= 0:
            raise NotImplementedError("garbage_tol is not implemented")
        if tp.use_two_streams:
            raise NotImplementedError("Using two streams does not appear to confer a benefit.")
        self._compute_wf_name_list(t_array)
        self.cso = coeff_save_obj
        self.cso.max_i = len(t_array) - 1
        self._commit_state()
        if self._traj is None:
            raise ValueError("no basis: create an initial basis and vector first")
        if self.debug_verb > INIT_VERBOSITY_LEVEL:
            print("Finished generate_timeline setup! Beginning time evolution...")
        for i, t_curr in enumerate(t_array):
            self.log_ind = 0
            if self.debug_verb > BASE_STEP_LEVEL:
                what = "Began initial timestep (no evolution in this step)" if i == 0 else \
                    f"Initiated timestep from {t_array[i-1]} to {t_curr}"
                print(f"\nCheck {self.log_ind}: {what}.")
            if i == 0:
                rec = self._traj.step(evolve=False)
                expm_dbg = [0, 0, 0, 0]
            else:
                if ep.use_scaling and ep.lanczos_order == 0:
                    rec = self._traj.step_scaled(float(t_curr - t_array[i - 1]))
                else:
                    rec = self._traj.step(evolve=True, dt=float(t_curr - t_array[i - 1]))
                expm_dbg = [bool(rec.converged), int(rec.final_m), float(rec.c1_plus_c2), float(rec.term_ratio)]
                if not ep.renormalize and rec.norm > ep.explosion_cutoff:
                    raise RuntimeError(f"Norm has exceeded preset explosion cutoff value ({ep.explosion_cutoff})!")
            self._whoami_cache = None
            if ep.use_scaling and ep.lanczos_order == 0:
                self.create_ham_mat()   # as the reference does for this path (time_evolution.py:801-803)
            # the reference's threshold is for complex128; complex64 amplitudes carry ~1e-7
            # relative rounding into <psi|H|psi>
            imag_tol = 1e-6 if self.engine.c64 else 1e-12
            if tp.diagnostics and rec.post_adapt_energy_im > imag_tol:
                raise RuntimeError(f"Energy has non-zero imaginary part: {rec.post_adapt_energy_im}.")
            L = self.engine.L
            self._obs_cache = {"n_exc": numpy.array(rec.n_exc[:L]), "n_pho": numpy.array(rec.n_pho[:L]),
                               "energy": complex(rec.energy_re, rec.energy_im), "norm": rec.norm}
            if self.debug_verb > HILBERT_SPACE_LEVEL:
                print(f"      Determined new Hilbert space: {rec.n_select} kept, {rec.n_enlarged} enlarged,"
                      f" {rec.n_states} states.")
            self._postprocess(t_curr, float(rec.norm), i)
            post = [float(rec.post_adapt_norm), float(rec.post_adapt_energy_re)]
            self._save_diagnostic_data(t_curr, float(rec.norm), post, expm_dbg, [rec.ceiling_hits])
            self._print_memory_info()

    def _postprocess(self, t_curr, norm, i):
        if self.debug_verb > BASE_STEP_LEVEL:
            print(f"Check {self.log_ind}: Beginning calculation of observable expectation values.")
        self.obsobj.primer_hook()
        self.obsobj.compute_all_and_write(self.vector, t_curr, norm, self.log_ind)
        if self.cso.save_necessary(i):
            numpy.save(self.wf_name_list[i], self.vector.detach().cpu().numpy())
            numpy.save(self.wf_name_list[i].replace("wf_file_", "whoami_"),
                       self.whoami.view(torch.int32).cpu().numpy().view(numpy.uint32))

    def _print_memory_info(self):
        if self.debug_verb > MEM_INFO_LEVEL:
            print(f"Used {devices.mempool.used_bytes() / 1024**2:1.1f} MiB on vector_dev.")

    def _compute_wf_name_list(self, t_array):
        """File names of the saved wavefunctions (paces/core/time_evolution.py:700-715)."""
        smallest_val = numpy.min(numpy.abs(t_array))
        smallest_diff = numpy.diff(numpy.abs(t_array)).min()
        if smallest_val == 0:
            decnum = numpy.abs(numpy.floor(numpy.log10(smallest_diff))) + 1
        else:
            decnum = numpy.abs(numpy.floor(numpy.log10(min(smallest_val, smallest_diff)))) + 1
        largest_val = numpy.max(numpy.abs(t_array))
        intnum = numpy.abs(numpy.ceil(numpy.log10(largest_val)))
        f_str = "wf_file_{0:0%i.%if}" % (intnum + decnum + 1, decnum)
        wf_coeff_dir = os.path.join(self.dirname, "wf_coeffs")
        if not os.path.exists(wf_coeff_dir):
            os.mkdir(wf_coeff_dir)
        self.wf_name_list = [os.path.join(wf_coeff_dir, f_str.format(i)) for i in t_array]

    def _save_diagnostic_data(self, t_curr, norm, norm_energy, expm_dbg, dbg_vals):
        """One line of diagnostics.log (paces/core/time_evolution.py:718-728)."""
        if self.te_params.diagnostics:
            line = [t_curr, norm, time.time() - self.start_time] + norm_energy + expm_dbg
            line += [self.numstates] + list(dbg_vals)
            with open(self.obsobj.fname_dict["diagnostics"], "a", encoding="utf-8") as diag_f:
                numpy.savetxt(diag_f, line, newline=" ")
                diag_f.write("\n")


class HamiltonianOperator:
    """The total Hamiltonian of a TimeEvolution's current basis as a device linear operator,
    times a scalar: what create_ham_mat builds in the reference (diags(diag_vals) plus the
    term matrices, paces/core/time_evolution.py:375-379), kept as the step's neighbour table.
    `op @ v` is the device H row kernel (paces_apply_h) times the scalar; `c * op` scales it,
    as the reference passes 1j * ham_mat to expm_multiply_simple.  The operator belongs to the
    basis it was created on: after the next time step it raises instead of acting on a
    different basis."""

    def __init__(self, te, scale=1.0, _step=None):
        if te._traj is None or te._traj.last is None:
            raise ValueError("no Hamiltonian yet: take a time step (generate_timeline) first")
        self.te = te
        self.scale = complex(scale)
        self._step = te._traj.step_index if _step is None else _step
        n = te.numstates
        self.shape = (n, n)
        self.dtype = te.engine.cdtype

    def _live(self):
        if self.te._traj.step_index != self._step:
            raise RuntimeError("this Hamiltonian operator belongs to an earlier basis; call create_ham_mat() again")
        return self.te._traj

    def __matmul__(self, vector):
        tr = self._live()
        eng = self.te.engine
        n = self.shape[0]
        x = torch.zeros(max(tr.basis.cap, 1), dtype=eng.cdtype, device=eng.device)
        x[:n] = torch.as_tensor(vector).to(eng.device, eng.cdtype)[:n]
        y = eng.apply_h(tr.basis, tr.h, x)[:n]
        return y if self.scale == 1 else y * self.scale

    def dot(self, vector):
        return self @ vector

    def __mul__(self, c):
        return HamiltonianOperator(self.te, self.scale * complex(c), self._step)

    __rmul__ = __mul__

    def __neg__(self):
        return self * -1.0

    def __repr__(self):
        return f"<HamiltonianOperator {self.shape[0]}x{self.shape[1]} x {self.scale}>"
