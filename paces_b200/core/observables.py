"""ObservablesFramework: observables of a timeline and their output files
(paces/core/observables.py).

Files and formats are the reference's: `<dirname>/observables/<fname>.real` and `.imag`
with the header `#time norm <header>` and one line per step, values written by
numpy.savetxt (paces/core/observables.py:62-71, :101-123), plus `diagnostics.log`
(:73-81).
"""

import abc
import os

import numpy
import torch

from ..aux.helpers import obs_attrs
from ..config import INIT_VERBOSITY_LEVEL, OBSERVABLES_LEVEL


class ObservablesFramework:
    """Abstract base of a model's observables (paces/core/observables.py:13-92).

    Subclass methods `calculate_<name>(self, vector)` carry `@obs_attrs(fname=..., header=...)`
    and return an array (or a scalar); `self.teobj` and `self.hamobj` give access to the
    basis and the Hamiltonian.
    """
    __metaclass__ = abc.ABCMeta

    def __init__(self, teobj, obs_list):
        if teobj.debug_verb > INIT_VERBOSITY_LEVEL:
            print("Initializing Observables object...")
        self.teobj = teobj
        self.hamobj = teobj.hamobj
        self.use_module = teobj.hamobj.use_module
        self.norm = None
        self.obs_dict = {}
        self.fname_dict = {}
        obs_dir = os.path.join(teobj.dirname, "observables")
        if not os.path.exists(obs_dir):
            os.mkdir(obs_dir)
        for key in obs_list:
            try:
                meth = getattr(self, "calculate_" + key)
            except AttributeError as exc:
                raise KeyError(f"Calculation method for {key} not found.") from exc
            self.obs_dict[key] = meth
            try:
                fname = os.path.join(obs_dir, meth.fname)
            except AttributeError as exc:
                raise AttributeError(f"The observables function {meth} is missing a decorator"
                                     " specifying the fname for the observables file.") from exc
            self.fname_dict[key] = fname
            for part in ["real", "imag"]:
                with open(".".join([fname, part]), "w", encoding="utf-8") as f:
                    f.write("#time norm " + meth.header + "\n")
        if self.teobj.te_params.diagnostics:
            extra_dbg = " ".join(self.hamobj.extra_dbg_list)
            if len(extra_dbg) > 0:
                extra_dbg = " " + extra_dbg
            self.fname_dict["diagnostics"] = os.path.join(obs_dir, "diagnostics.log")
            with open(self.fname_dict["diagnostics"], "w", encoding="utf-8") as diag_file:
                diag_file.write("#time norm seconds_since_start post_adapt_norm post_adapt_H"
                                " expm_converged final_m final_expm_term rel_error_expm numstates"
                                + extra_dbg + "\n")

    def primer_hook(self):
        """Per-step preparation before the observables (subclasses may override)."""

    @obs_attrs(fname="total_energy", header="energy")
    def calculate_total_energy(self, vector):
        """<psi|H|psi> (paces/core/observables.py:95-99), from the device."""
        cached = self.teobj._cached_observable(vector, "energy")
        if cached is not None:
            return cached
        return self.teobj._observables_of(vector)["energy"]

    def compute_all_and_write(self, vector, t, norm, log_index):
        """Evaluate every requested observable and append it to its files
        (paces/core/observables.py:101-123)."""
        for i, obsname in enumerate(self.obs_dict):
            result = self.obs_dict[obsname](vector)
            if self.teobj.debug_verb > OBSERVABLES_LEVEL:
                print(f"      {log_index}.{i+1}a: Calculated {obsname}.")
            if isinstance(result, torch.Tensor):
                result = result.detach().cpu().numpy()
            fname = self.fname_dict[obsname]
            for part in ["real", "imag"]:
                with open(".".join([fname, part]), "a", encoding="utf-8") as f:
                    s_data = numpy.append([t, norm], getattr(numpy.asarray(result), part))
                    numpy.savetxt(f, s_data, newline=" ")
                    f.write("\n")
            if self.teobj.debug_verb > OBSERVABLES_LEVEL:
                print(f"      {log_index}.{i+1}b: Saved {obsname} to file.")

    def calculate_rdm(self, site, vector):
        """Reduced density matrix of one site (paces/core/observables.py:126-150)."""
        occs = self.hamobj.get_n_at_site(self.teobj.whoami, site).to(torch.int64)
        dim = int(self.hamobj.max_dims_v[site])
        vecprod = vector * torch.conj(vector)
        diag = torch.zeros(dim, dtype=torch.complex128, device=vector.device)
        diag.index_add_(0, occs, vecprod.to(torch.complex128))
        upper = torch.zeros((dim, dim), dtype=torch.complex128, device=vector.device)
        for k in range(1, dim):
            vp = self._offdiag_n(vector, k, site) * torch.conj(vector)
            this = torch.zeros(dim, dtype=torch.complex128, device=vector.device)
            this.index_add_(0, occs, vp.to(torch.complex128))
            upper += torch.diag(this[k:], k)
        return upper + upper.T.conj() + torch.diag(diag)

    def _offdiag_n(self, vector, n, site):
        """psi shifted by n quanta at `site` (paces/core/observables.py:153-163)."""
        whoami = self.teobj.whoami
        occs = self.hamobj.get_n_at_site(whoami, site).to(torch.int64)
        ok = occs + n < int(self.hamobj.max_dims_v[site])
        # boolean indexing of uint32 tensors is not available on the GPU: select on an int32 view
        plus = whoami.view(torch.int32)[ok].clone().view(torch.uint32)
        self.hamobj.add_n_at_site(plus, n, site)
        idx = self.hamobj.searchsorted(whoami, plus, allow_escapes=True)
        res = torch.zeros_like(vector)
        found = idx >= 0
        src = torch.nonzero(ok).view(-1)[found]
        res[idx[found]] = vector[src]
        return res
