"""Device-side engine: owns the native context and the device buffers of one trajectory.

Everything that touches amplitudes or keys runs in libpaces_b200 (sm_100a); this
module only allocates torch tensors (device memory), passes their pointers through the
C ABI and reads back the one small record each step produces.
"""

from __future__ import annotations

import ctypes
import dataclasses

import numpy as np
import torch

from . import _native as nat

TAYLOR_TOL_C128 = 2.0 ** -53   # paces/core/time_evolution.py:484
TAYLOR_TOL_C64 = 2.0 ** -24    # single-precision unit roundoff


@dataclasses.dataclass
class ModelParams:
    """Holstein chain (paces/models/holstein.py:24-66 with its use_terms dict)."""
    nchain: int
    max_ho_dims: list
    J: float = 1.0
    g: float = 1.0
    eps_sys: float = 0.0
    hbar_omega: float = 1.0
    delta_eps: float = 0.0
    periodic: bool = False
    site_eps: list | None = None
    precision: str = "c128"   # "c128" (reference precision) or "c64"
    geo_dim: int = 1          # lattice dimensions (holstein.py:24-51); nchain = l ** geo_dim
    J2: float | None = None   # the next-nearest-neighbour "hopping2" term (holstein.py:234-240)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class DevBasis:
    """A sorted basis on the device: keys [cap, nw] (uint64 words in int64 storage) and
    block offsets by exciton position blk [nchain+1] (blk[nchain] = number of states)."""

    def __init__(self, eng: "Engine", cap: int):
        self.eng = eng
        self.cap = int(cap)
        self.keys = torch.empty((max(self.cap, 1), eng.nw), dtype=torch.int64, device=eng.device)
        self.blk = torch.zeros(eng.L + 1, dtype=torch.int32, device=eng.device)

    def c(self):
        return nat.Basis(self.keys.data_ptr(), self.blk.data_ptr(), self.cap)

    def count(self) -> int:
        return int(self.blk[self.eng.L].item())

    @classmethod
    def wrap(cls, eng: "Engine", keys, blk, cap):
        """A basis over existing device tensors (no copy)."""
        b = cls.__new__(cls)
        b.eng, b.cap, b.keys, b.blk = eng, int(cap), keys, blk
        return b

    def clone(self) -> "DevBasis":
        n = self.count()
        b = DevBasis(self.eng, max(n, 1))
        b.keys[:n] = self.keys[:n]
        b.blk.copy_(self.blk)
        return b


class DevHMat:
    """Neighbour table [cap, 4] (left, right, down, up; -1 = absent) and row metadata [cap];
    for lattices with more hopping channels also xnbr [nhop-1, cap, 2] (the other channels'
    lower and upper neighbours)."""

    def __init__(self, eng: "Engine", cap: int):
        self.cap = int(cap)
        self.nbr = torch.empty((max(self.cap, 1), 4), dtype=torch.int32, device=eng.device)
        self.meta = torch.empty(max(self.cap, 1), dtype=torch.int32, device=eng.device)
        self.xnbr = None
        if eng.nhop > 1:
            self.xnbr = torch.empty((eng.nhop - 1, max(self.cap, 1), 2), dtype=torch.int32, device=eng.device)

    def c(self):
        return nat.HMat(self.nbr.data_ptr(), self.meta.data_ptr(), self.cap,
                        self.xnbr.data_ptr() if self.xnbr is not None else None)


class Engine:
    def __init__(self, params: ModelParams, device=None, cap: int = 4096):
        self.lib = nat.load()
        if not torch.cuda.is_available():
            raise RuntimeError("paces_b200 needs a CUDA device (sm_100a); none is visible")
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.params = params
        self.L = int(params.nchain)
        self.c64 = params.precision == "c64"
        self.cdtype = torch.complex64 if self.c64 else torch.complex128
        self.tol = TAYLOR_TOL_C64 if self.c64 else TAYLOR_TOL_C128
        dims = (ctypes.c_int32 * self.L)(*[int(x) for x in params.max_ho_dims])
        site = None
        if params.site_eps is not None:
            site = (ctypes.c_double * self.L)(*[float(x) for x in params.site_eps])
        desc = nat.ModelDesc(self.L, 1 if params.periodic else 0, nat.C64 if self.c64 else nat.C128, 0,
                             dims, float(params.eps_sys), float(params.hbar_omega),
                             float(params.delta_eps), float(params.J), float(params.g),
                             site if site is not None else ctypes.POINTER(ctypes.c_double)(),
                             int(params.geo_dim), 0 if params.J2 is None else 1,
                             0.0 if params.J2 is None else float(params.J2))
        self._dims, self._site = dims, site
        ctx = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            nat.check(self.lib.paces_create(ctypes.byref(desc), ctypes.byref(ctx)), None, "paces_create")
        self.ctx = ctx
        self.nw = self.lib.paces_key_words(ctx)
        # bumped by every change of the launch shapes: CUDA graphs captured under other shapes
        # are not replayed
        self.tuning_epoch = 0
        self.nhop = int(self.lib.paces_hop_channels(ctx))  # hopping channels (1: the chain)
        self.ref_words = self.lib.paces_ref_words(ctx)
        self.cap = 0
        self.ws = None
        self._grow(cap)
        self.rec_dev = torch.zeros(ctypes.sizeof(nat.StepRecord), dtype=torch.uint8, device=self.device)
        self.rec_host = torch.zeros(ctypes.sizeof(nat.StepRecord), dtype=torch.uint8).pin_memory()

    # ---- buffers ------------------------------------------------------------------------
    def _grow(self, cap):
        cap = int(max(cap, 64))
        if cap <= self.cap:
            return
        nbytes = ctypes.c_size_t()
        nat.check(self.lib.paces_workspace_bytes(self.ctx, cap, ctypes.byref(nbytes)), self.ctx, "workspace")
        self.ws = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.device)
        self.ws_bytes = int(nbytes.value)
        self.cap = cap

    def workspace(self):
        return _ptr(self.ws), ctypes.c_size_t(self.ws_bytes)

    def new_basis(self, cap=None):
        return DevBasis(self, self.cap if cap is None else cap)

    def new_hmat(self, cap=None):
        return DevHMat(self, self.cap if cap is None else cap)

    def new_vector(self, cap=None):
        return torch.zeros(max(self.cap if cap is None else cap, 1), dtype=self.cdtype, device=self.device)

    def read_status(self):
        st = ctypes.c_int32()
        nat.check(self.lib.paces_read_status(self.ctx, _stream(self.device), ctypes.byref(st)), self.ctx,
                  "read_status")
        return int(st.value)

    def raise_status(self, what):
        st = self.read_status()
        if st != nat.PACES_OK:
            if st == nat.ERR_CAPACITY:
                raise nat.CapacityError(st, what)
            raise nat.PacesError(st, what)

    # ---- layout conversion ----------------------------------------------------------------
    def basis_from_ref(self, ref_rows, cap=None) -> DevBasis:
        """Reference whoami rows (uint32 [n, W], sorted, unique) -> device basis."""
        ref = torch.as_tensor(np.ascontiguousarray(ref_rows).view(np.int32) if isinstance(ref_rows, np.ndarray)
                              else ref_rows)
        ref = ref.to(self.device, torch.int32).contiguous()
        n = int(ref.shape[0])
        if n and int(ref.shape[1]) != self.ref_words:
            raise ValueError(f"rows have {ref.shape[1]} words, the model packs {self.ref_words}")
        b = self.new_basis(max(cap or 0, n, 1))
        pos = torch.empty(max(n, 1), dtype=torch.int32, device=self.device)
        if n:
            nat.check(self.lib.paces_keys_from_ref(self.ctx, _ptr(ref), n, self.ref_words, _ptr(b.keys), _ptr(pos),
                                                   _stream(self.device)), self.ctx, "keys_from_ref")
            self.raise_status("keys_from_ref: occupation or position out of range")
            counts = torch.bincount(pos[:n].long(), minlength=self.L)
            b.blk[1:] = torch.cumsum(counts, 0).to(torch.int32)
            if not bool((pos[1:n] >= pos[: n - 1]).all()):
                raise ValueError("basis rows must be sorted (exciton position is the leading field)")
        return b

    def basis_to_ref(self, b: DevBasis, n=None) -> torch.Tensor:
        n = b.count() if n is None else n
        out = torch.empty((max(n, 1), self.ref_words), dtype=torch.int32, device=self.device)
        if n:
            nat.check(self.lib.paces_keys_to_ref(self.ctx, ctypes.byref(b.c()), self.ref_words, _ptr(out),
                                                 _stream(self.device)), self.ctx, "keys_to_ref")
        return out[:n]

    def query_from_ref(self, ref_rows):
        """Arbitrary reference rows -> (keys, pos) device tensors (no ordering needed)."""
        ref = torch.as_tensor(np.ascontiguousarray(ref_rows).view(np.int32) if isinstance(ref_rows, np.ndarray)
                              else ref_rows).to(self.device, torch.int32).contiguous()
        n = int(ref.shape[0])
        keys = torch.empty((max(n, 1), self.nw), dtype=torch.int64, device=self.device)
        pos = torch.empty(max(n, 1), dtype=torch.int32, device=self.device)
        if n:
            nat.check(self.lib.paces_keys_from_ref(self.ctx, _ptr(ref), n, self.ref_words, _ptr(keys), _ptr(pos),
                                                   _stream(self.device)), self.ctx, "keys_from_ref")
        return keys, pos, n

    # ---- stages ---------------------------------------------------------------------------
    def expand(self, b: DevBasis, out: DevBasis | None = None) -> DevBasis:
        out = out or self.new_basis()
        ws, nb = self.workspace()
        nat.check(self.lib.paces_expand(self.ctx, ctypes.byref(b.c()), ctypes.byref(out.c()), ws, nb,
                                        _stream(self.device)), self.ctx, "expand")
        self.raise_status("expand")
        return out

    def assemble(self, b: DevBasis, out: DevBasis | None = None, h: DevHMat | None = None):
        out = out or self.new_basis()
        h = h or self.new_hmat(out.cap)
        ceil = torch.zeros(1, dtype=torch.int32, device=self.device)
        ws, nb = self.workspace()
        nat.check(self.lib.paces_assemble(self.ctx, ctypes.byref(b.c()), ctypes.byref(out.c()), ctypes.byref(h.c()),
                                          _ptr(ceil), ws, nb, _stream(self.device)), self.ctx, "assemble")
        self.raise_status("assemble")
        return out, h, int(ceil.item())

    def truncate(self, b: DevBasis, psi, maxstates, shuffle=False, seed=0, step=0, out=None) -> DevBasis:
        out = out or self.new_basis()
        ws, nb = self.workspace()
        nat.check(self.lib.paces_truncate(self.ctx, ctypes.byref(b.c()), _ptr(psi), int(maxstates), int(bool(shuffle)),
                                          int(seed), int(step), ctypes.byref(out.c()), ws, nb,
                                          _stream(self.device)), self.ctx, "truncate")
        self.raise_status("truncate")
        return out

    def truncate_weighted(self, b: DevBasis, weights, maxstates, shuffle=False, seed=0, step=0, out=None) -> DevBasis:
        """`truncate` ranking the states by `weights` (float64, one per state) instead of |psi|."""
        out = out or self.new_basis()
        ws, nb = self.workspace()
        if weights.dtype != torch.float64 or weights.device != self.device or weights.numel() < b.count():
            raise ValueError("weights: one float64 per state, on the engine's device")
        nat.check(self.lib.paces_truncate_weighted(self.ctx, ctypes.byref(b.c()), _ptr(weights), int(maxstates),
                                                   int(bool(shuffle)), int(seed), int(step), ctypes.byref(out.c()),
                                                   ws, nb, _stream(self.device)), self.ctx, "truncate_weighted")
        self.raise_status("truncate_weighted")
        return out

    def lookahead_weights(self, b: DevBasis, h: DevHMat, psi, tau, weighting, out=None):
        """Look-ahead weights (weighting = nat.WEIGHT_COHERENCE / WEIGHT_NORM) or H 1
        (nat.WEIGHT_HAM_ONES) of every state of b, as float64 on the device."""
        n = b.count()
        out = torch.empty(max(n, 1), dtype=torch.float64, device=self.device) if out is None else out
        nat.check(self.lib.paces_lookahead_weights(self.ctx, ctypes.byref(b.c()), ctypes.byref(h.c()), _ptr(psi),
                                                   float(tau), int(weighting), _ptr(out), _stream(self.device)),
                  self.ctx, "lookahead_weights")
        self.raise_status("lookahead_weights")
        return out[:n]

    def remap(self, old: DevBasis, old_psi, new: DevBasis, new_psi=None):
        new_psi = self.new_vector(new.cap) if new_psi is None else new_psi
        ws, nb = self.workspace()
        nat.check(self.lib.paces_remap(self.ctx, ctypes.byref(old.c()), _ptr(old_psi), ctypes.byref(new.c()),
                                       _ptr(new_psi), ws, nb, _stream(self.device)), self.ctx, "remap")
        self.raise_status("remap")
        return new_psi

    def taylor(self, b: DevBasis, h: DevHMat, psi_in, dt, m_star=100, tol=None, psi_out=None):
        psi_out = self.new_vector(b.cap) if psi_out is None else psi_out
        info = torch.zeros(ctypes.sizeof(nat.ExpmInfo), dtype=torch.uint8, device=self.device)
        ws, nb = self.workspace()
        nat.check(self.lib.paces_taylor(self.ctx, ctypes.byref(b.c()), ctypes.byref(h.c()), _ptr(psi_in),
                                        _ptr(psi_out), float(dt), int(m_star), float(self.tol if tol is None else tol),
                                        _ptr(info), ws, nb, _stream(self.device)), self.ctx, "taylor")
        self.raise_status("taylor")
        raw = info.cpu().numpy().tobytes()
        e = nat.ExpmInfo.from_buffer_copy(raw)
        return psi_out, [bool(e.converged), int(e.final_m), float(e.c1_plus_c2), float(e.term_ratio)]

    def krylov_bytes(self, cap, order):
        nbytes = ctypes.c_size_t()
        nat.check(self.lib.paces_lanczos_bytes(self.ctx, int(cap), int(order), ctypes.byref(nbytes)), self.ctx,
                  "lanczos_bytes")
        return int(nbytes.value)

    def new_krylov(self, cap, order):
        """Device workspace of the Lanczos step for bases of up to `cap` states."""
        return torch.empty(self.krylov_bytes(cap, order), dtype=torch.uint8, device=self.device)

    def lanczos(self, b: DevBasis, h: DevHMat, psi_in, dt, order, psi_out=None, krylov=None):
        """psi_out = exp(-i dt H) psi_in from order + 1 Lanczos vectors (paces_lanczos)."""
        psi_out = self.new_vector(b.cap) if psi_out is None else psi_out
        krylov = self.new_krylov(b.cap, order) if krylov is None else krylov
        info = torch.zeros(ctypes.sizeof(nat.ExpmInfo), dtype=torch.uint8, device=self.device)
        nat.check(self.lib.paces_lanczos(self.ctx, ctypes.byref(b.c()), ctypes.byref(h.c()), _ptr(psi_in),
                                         _ptr(psi_out), float(dt), int(order), _ptr(info), _ptr(krylov),
                                         int(krylov.numel()), _stream(self.device)), self.ctx, "lanczos")
        self.raise_status("lanczos")
        e = nat.ExpmInfo.from_buffer_copy(info.cpu().numpy().tobytes())
        return psi_out, [bool(e.converged), int(e.final_m), float(e.c1_plus_c2), float(e.term_ratio)]

    def observables(self, b: DevBasis, h: DevHMat, psi, what=nat.OBS_NORM | nat.OBS_ENERGY | nat.OBS_SITES):
        out = torch.zeros(3 + 2 * self.L, dtype=torch.float64, device=self.device)
        ws, nb = self.workspace()
        nat.check(self.lib.paces_observables(self.ctx, ctypes.byref(b.c()), ctypes.byref(h.c()), _ptr(psi),
                                             int(what), _ptr(out), ws, nb, _stream(self.device)), self.ctx,
                  "observables")
        o = out.cpu().numpy()
        return {"norm": o[0], "energy": complex(o[1], o[2]), "n_exc": o[3:3 + self.L],
                "n_pho": o[3 + self.L:3 + 2 * self.L]}

    def hnorms(self, b: DevBasis, h: DevHMat, shift=None):
        """(trace of H, largest row 1-norm of H - shift I, trace / n) on the device."""
        out = torch.zeros(3, dtype=torch.float64, device=self.device)
        sh = None if shift is None else torch.tensor([float(shift)], dtype=torch.float64, device=self.device)
        ws, nb = self.workspace()
        nat.check(self.lib.paces_hnorms(self.ctx, ctypes.byref(b.c()), ctypes.byref(h.c()), _ptr(sh), _ptr(out), ws, nb,
                                        _stream(self.device)), self.ctx, "hnorms")
        return [float(x) for x in out.cpu().tolist()]

    def expm_scaled(self, b: DevBasis, h: DevHMat, psi_in, psi_out, t, shift, m_star, stages, eta, tol=None):
        """psi_out = exp(t * 1j (H - shift I)) psi_in in `stages` stages of at most m_star terms,
        times eta after each stage.  Returns [converged, final_m, c1 + c2, term ratio]."""
        info = torch.zeros(ctypes.sizeof(nat.ExpmInfo), dtype=torch.uint8, device=self.device)
        ws, nb = self.workspace()
        eta = complex(eta)
        nat.check(self.lib.paces_expm_scaled(self.ctx, ctypes.byref(b.c()), ctypes.byref(h.c()), _ptr(psi_in),
                                             _ptr(psi_out), float(t), float(shift), int(m_star), int(stages),
                                             float(self.tol if tol is None else tol), eta.real, eta.imag, _ptr(info),
                                             ws, nb, _stream(self.device)), self.ctx, "expm_scaled")
        self.raise_status("expm_scaled")
        e = nat.ExpmInfo.from_buffer_copy(info.cpu().numpy().tobytes())
        return [bool(e.converged), int(e.final_m), float(e.c1_plus_c2), float(e.term_ratio)]

    def term_energies(self, b: DevBasis, h: DevHMat, psi):
        """Per exciton position the hopping and vibronic energies <psi_p|H_term|psi> (complex
        [L] each) and the sum of the phonon-vacuum amplitudes (paces_term_energies)."""
        out = torch.empty(4 * self.L + 2, dtype=torch.float64, device=self.device)
        ws, nb = self.workspace()
        nat.check(self.lib.paces_term_energies(self.ctx, ctypes.byref(b.c()), ctypes.byref(h.c()), _ptr(psi),
                                               _ptr(out), ws, nb, _stream(self.device)), self.ctx, "term_energies")
        L = self.L
        hop = torch.complex(out[:L], out[L:2 * L])
        vib = torch.complex(out[2 * L:3 * L], out[3 * L:4 * L])
        return hop, vib, complex(out[4 * L].item(), out[4 * L + 1].item())

    def apply_h(self, b: DevBasis, h: DevHMat, x, y=None):
        """y = H x (total_ham)."""
        y = torch.empty_like(x) if y is None else y
        nat.check(self.lib.paces_apply_h(self.ctx, ctypes.byref(b.c()), ctypes.byref(h.c()), _ptr(x), _ptr(y),
                                         _stream(self.device)), self.ctx, "apply_h")
        return y

    def lookup(self, pb: DevBasis, q_keys, q_pos, nq, must_exist=False):
        out = torch.empty(max(nq, 1), dtype=torch.int64, device=self.device)
        ws, nb = self.workspace()
        nat.check(self.lib.paces_lookup(self.ctx, ctypes.byref(pb.c()), _ptr(q_keys), _ptr(q_pos), int(nq),
                                        int(bool(must_exist)), _ptr(out), ws, nb, _stream(self.device)), self.ctx,
                  "lookup")
        if must_exist:
            self.raise_status("lookup: a state that must exist is not in the basis")
        return out[:nq]

    def step(self, old: DevBasis, old_psi, new: DevBasis, new_psi, h: DevHMat, prm: nat.StepParams,
             sync=True):
        ws, nb = self.workspace()
        nat.check(self.lib.paces_step(self.ctx, ctypes.byref(old.c()), _ptr(old_psi), ctypes.byref(new.c()),
                                      _ptr(new_psi), ctypes.byref(h.c()), ctypes.byref(prm), _ptr(self.rec_dev),
                                      ws, nb, _stream(self.device)), self.ctx, "step")
        if not sync:
            return None
        return self.read_record()

    def set_test_hooks(self, wait_limit_ns=0, skip_barrier_block=-1):
        """Test hook of the bounded grid-barrier waits (paces_set_test_hooks): a shorter wait
        limit and a block that skips its arrival, so a test can make a wait run out."""
        nat.check(self.lib.paces_set_test_hooks(self.ctx, int(wait_limit_ns), int(skip_barrier_block)), self.ctx,
                  "set_test_hooks")

    def set_profiling(self, on=True):
        nat.check(self.lib.paces_set_profiling(self.ctx, 1 if on else 0), self.ctx, "set_profiling")

    # ---- learned proposal ---------------------------------------------------------------------
    def selected(self):
        """(basis, |psi| float32 per state, cut float32 [1]) of the last paces_step's
        truncation -- views into the workspace, valid until the next call that uses it."""
        sel, wp, cp = nat.Basis(), ctypes.c_void_p(), ctypes.c_void_p()
        ws, nb = self.workspace()
        nat.check(self.lib.paces_selected_view(self.ctx, ws, nb, ctypes.byref(sel), ctypes.byref(wp), ctypes.byref(cp)),
                  self.ctx, "selected_view")
        base = self.ws.data_ptr()
        cap = int(sel.cap)
        ok, obk, ow, oc = sel.keys - base, sel.blk - base, wp.value - base, cp.value - base
        keys = self.ws[ok:ok + cap * self.nw * 8].view(torch.int64).view(cap, self.nw)
        blk = self.ws[obk:obk + (self.L + 1) * 4].view(torch.int32)
        w = self.ws[ow:ow + cap * 4].view(torch.float32)
        cut = self.ws[oc:oc + 4].view(torch.float32)
        return DevBasis.wrap(self, keys, blk, cap), w, cut

    def proposal_features(self, x: DevBasis, w, cut):
        n = x.count()
        feats = torch.empty((max(4 * n, 1), 16), dtype=torch.bfloat16, device=self.device)
        valid = torch.empty(max(4 * n, 1), dtype=torch.uint8, device=self.device)
        nat.check(self.lib.paces_proposal_features(self.ctx, ctypes.byref(x.c()), _ptr(w), _ptr(cut), _ptr(feats),
                                                   _ptr(valid), _stream(self.device)), self.ctx, "proposal_features")
        return feats[:4 * n], valid[:4 * n]

    def proposal_labels(self, x: DevBasis, y: DevBasis):
        n = x.count()
        lab = torch.empty(max(4 * n, 1), dtype=torch.uint8, device=self.device)
        nat.check(self.lib.paces_proposal_labels(self.ctx, ctypes.byref(x.c()), ctypes.byref(y.c()), _ptr(lab),
                                                 _stream(self.device)), self.ctx, "proposal_labels")
        return lab[:4 * n]

    def proposal_score(self, x: DevBasis, w, cut, params, threshold=0.0, keep=None):
        """Logits of every event of x (tensor cores); keep (optional, uint8 [5][cap]) gets the
        keep mask.  Returns (logits, (existing, kept))."""
        n = x.count()
        logits = torch.empty(max(4 * n, 1), dtype=torch.float32, device=self.device)
        counts = torch.zeros(2, dtype=torch.int32, device=self.device)
        kcap = keep.shape[1] if keep is not None else 0
        nat.check(self.lib.paces_proposal_score(self.ctx, ctypes.byref(x.c()), _ptr(w), _ptr(cut), _ptr(params),
                                                float(threshold), _ptr(keep), int(kcap), _ptr(logits), _ptr(counts),
                                                _stream(self.device)), self.ctx, "proposal_score")
        self.raise_status("proposal_score")
        c = counts.cpu().tolist()
        return logits[:4 * n], (c[0], c[1])

    def stage_times(self):
        """Per-stage device milliseconds of the last profiled step."""
        ms = (ctypes.c_float * 7)()
        nat.check(self.lib.paces_stage_times(self.ctx, ms), self.ctx, "stage_times")
        return dict(zip(nat.STAGES, [float(x) for x in ms]))

    def kernel_launches(self):
        return int(self.lib.paces_kernel_launches(self.ctx))

    def read_record(self) -> nat.StepRecord:
        self.rec_host.copy_(self.rec_dev, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        return nat.StepRecord.from_buffer_copy(self.rec_host.numpy().tobytes())

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.paces_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Trajectory:
    """One adaptive-basis trajectory on the device, stepped by `paces_step`.

    Two basis/amplitude slots alternate: a step reads the current slot and writes the
    other, so a capacity overflow leaves the state intact and the step is retried with
    larger buffers.

    With `graph=True` the evolving steps replay CUDA graphs (one per slot parity and dt)
    captured from `paces_step`, so a step costs one graph launch and one 2 KB record read.
    Tie shuffling hashes the step index into the kernels' arguments and is stepped without
    graphs.  Growing the buffers drops the graphs; the next step captures them again.
    """

    def __init__(self, eng: Engine, maxstates, enlarge_steps, m_star=100, diagnostics=True,
                 shuffle_seed=None, renormalize=False, explosion_cutoff=2.0, cap=None, graph=False,
                 weighting=nat.WEIGHT_NONE, tau=0.0, lanczos_order=0):
        if weighting not in (nat.WEIGHT_NONE, nat.WEIGHT_COHERENCE, nat.WEIGHT_NORM):
            raise ValueError(f"unknown weighting {weighting}")
        if weighting != nat.WEIGHT_NONE and tau == 0:
            raise ValueError("Specify a non-zero tau for this function to use U-weighting.")
        self.weighting = int(weighting)
        self.tau = float(tau)
        if not 0 <= int(lanczos_order) <= nat.MAX_LANCZOS_ORDER:
            raise ValueError(f"lanczos_order must lie in 0..{nat.MAX_LANCZOS_ORDER}")
        self.lanczos_order = int(lanczos_order)
        self.eng = eng
        self.maxstates = int(maxstates)
        self.enlarge_steps = int(enlarge_steps)
        self.m_star = int(m_star)
        self.diagnostics = bool(diagnostics)
        self.shuffle_seed = shuffle_seed
        self.renormalize = bool(renormalize)
        self.explosion_cutoff = float(explosion_cutoff)
        guess = int((2.5 + 2.0 * (self.enlarge_steps + 1)) * self.maxstates) + 1024
        eng._grow(cap or guess)
        self._alloc()
        self.cur = 0
        self.step_index = 0
        self.last = None
        self.use_graph = bool(graph)
        self._graphs = {}
        self.proposal = None  # (packed MLP parameters on the device, threshold) or None

    def _alloc(self):
        e = self.eng
        self.bases = [e.new_basis(), e.new_basis()]
        self.psis = [e.new_vector(), e.new_vector()]
        # with the look-ahead weighting a step reads the current basis' table while it writes
        # the next one: two tables, swapped with the bases (one shared table otherwise)
        h = e.new_hmat()
        self.hs = [h, e.new_hmat() if self.weighting else h]
        self._h_valid = False   # hs[cur] holds the table of bases[cur]
        # the Lanczos step's Krylov vectors (ExpmParams.lanczos_order > 0)
        self.krylov = e.new_krylov(e.cap, self.lanczos_order) if self.lanczos_order else None

    @property
    def h(self) -> DevHMat:
        """The neighbour table of the current basis (written by the last step)."""
        return self.hs[self.cur]

    def _regrow(self, factor=1.6):
        """Grow every buffer, keeping the current state (and its table)."""
        e = self.eng
        self._graphs = {}
        old_b, old_psi, old_h = self.bases[self.cur], self.psis[self.cur], self.hs[self.cur]
        n = old_b.count()
        e._grow(int(e.cap * factor))
        keep_keys, keep_blk, keep_psi = old_b.keys[:n].clone(), old_b.blk.clone(), old_psi[:n].clone()
        keep_h = None
        if self._h_valid and self.weighting:
            keep_h = (old_h.nbr[:n].clone(), old_h.meta[:n].clone(),
                      None if old_h.xnbr is None else old_h.xnbr[:, :n].clone())
        valid = self._h_valid
        self._alloc()
        b = self.bases[self.cur]
        b.keys[:n] = keep_keys
        b.blk.copy_(keep_blk)
        self.psis[self.cur][:n] = keep_psi
        if keep_h is not None:
            self.hs[self.cur].nbr[:n] = keep_h[0]
            self.hs[self.cur].meta[:n] = keep_h[1]
            if keep_h[2] is not None:
                self.hs[self.cur].xnbr[:, :n] = keep_h[2]
        self._h_valid = valid and keep_h is not None

    def set_state(self, basis: DevBasis, psi):
        self._h_valid = False
        n = basis.count()
        while n > self.eng.cap:
            self._regrow()
        b = self.bases[self.cur]
        b.keys[:n] = basis.keys[:n]
        b.blk.copy_(basis.blk)
        v = self.psis[self.cur]
        v.zero_()
        v[:n] = psi[:n].to(self.eng.cdtype)

    @property
    def basis(self) -> DevBasis:
        return self.bases[self.cur]

    @property
    def vector(self):
        return self.psis[self.cur][: self.basis.count()]

    def params(self, evolve, dt, weighted=None):
        """Step parameters; `weighted` (default: evolve) applies the look-ahead weighting,
        which the reference uses on every step but the first (time_evolution.py:560)."""
        p = nat.StepParams()
        p.maxstates = self.maxstates
        p.enlarge_steps = self.enlarge_steps
        p.evolve = 1 if evolve else 0
        p.dt = float(dt)
        p.m_star = self.m_star
        p.diagnostics = 1 if self.diagnostics else 0
        p.tol = self.eng.tol
        p.shuffle = 0 if self.shuffle_seed is None else 1
        p.renormalize = 1 if self.renormalize else 0
        p.shuffle_seed = 0 if self.shuffle_seed is None else int(self.shuffle_seed) & 0xFFFFFFFFFFFFFFFF
        p.step_index = self.step_index
        p.explosion_cutoff = self.explosion_cutoff
        if self.lanczos_order:
            p.lanczos_order = self.lanczos_order
            p.krylov = self.krylov.data_ptr()
            p.krylov_bytes = int(self.krylov.numel())
        if self.proposal is not None:
            p.proposal = 1
            p.proposal_threshold = float(self.proposal[1])
            p.proposal_params = self.proposal[0].data_ptr()
        if self.weighting and (evolve if weighted is None else weighted):
            if not self._h_valid:
                raise RuntimeError("the look-ahead weighting needs the neighbour table of the current basis: "
                                   "take a first (non-evolving) step after setting the state")
            self._old_h_c = self.hs[self.cur].c()
            p.weighting = self.weighting
            p.tau = self.tau
            p.old_h = ctypes.addressof(self._old_h_c)
        return p

    def _capture(self, dt):
        """CUDA graph of one evolving paces_step from the current slot into the other."""
        nxt = 1 - self.cur
        prm = self.params(True, dt)
        dev = self.eng.device
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(dev)
        torch.cuda.synchronize(dev)
        with torch.cuda.graph(g, stream=s, capture_error_mode="relaxed"):
            self.eng.step(self.bases[self.cur], self.psis[self.cur], self.bases[nxt], self.psis[nxt], self.hs[nxt],
                          prm, sync=False)
        return g, prm

    def _graph_step(self, dt):
        key = (self.cur, float(dt), self.eng.tuning_epoch,
               None if self.proposal is None else (self.proposal[0].data_ptr(), float(self.proposal[1])))
        if key not in self._graphs:
            self._graphs[key] = self._capture(dt)
        self._graphs[key][0].replay()
        rec = self.eng.read_record()
        if rec.status == nat.ERR_CAPACITY:
            return None
        if rec.status != nat.PACES_OK:
            raise nat.PacesError(rec.status, "paces_step")
        self.cur = 1 - self.cur
        self.step_index += 1
        self._h_valid = True
        self.last = rec
        return rec

    def step_scaled(self, dt):
        """One time step propagated by scaling and squaring, as the reference does with
        ExpmParams(use_scaling=True): exp(dt * 1j H) applied with expm_multiply_simple
        (paces/core/time_evolution.py:579-581) -- note the sign: the reference's call
        propagates with +1j H where its plain Taylor path uses -1j H.  The new space is
        built by a non-evolving paces_step; the norms, stage count and order come from
        paces_b200.expm; the observables of the propagated state are measured again.
        Returns the step record."""
        rec = self.step(evolve=False, weighted=True)
        e, b, h = self.eng, self.basis, self.h
        psi = self.psis[self.cur]
        out = self.psis[1 - self.cur]
        dbg = self.expm_apply(psi, out, dt)
        psi.copy_(out)
        n = b.count()
        if self.renormalize:
            nrm = torch.linalg.vector_norm(psi[:n].to(torch.complex128)).item()
            psi[:n] /= nrm
        o = e.observables(b, h, psi)
        rec.converged, rec.final_m = int(dbg[0]), int(dbg[1])
        rec.c1_plus_c2, rec.term_ratio = dbg[2], dbg[3]
        rec.norm = float(o["norm"])
        rec.energy_re, rec.energy_im = o["energy"].real, o["energy"].imag
        for i in range(e.L):
            rec.n_exc[i] = float(o["n_exc"][i])
            rec.n_pho[i] = float(o["n_pho"][i])
        if not self.renormalize and rec.norm > self.explosion_cutoff:
            raise RuntimeError(f"Norm has exceeded preset explosion cutoff value ({self.explosion_cutoff})!")
        self.last = rec
        return rec

    def expm_apply(self, psi_in, psi_out, t):
        """psi_out = exp(t * 1j H) psi_in on the current basis by scaling and squaring
        (expm_multiply_simple(1j * H, psi, t), paces/aux/_scipy/_expm_multiply.py:106-202):
        the trace shift and 1-norm from the device H rows, stages and order from
        paces_b200.expm, every term on the device.  psi_in and psi_out hold the basis'
        capacity.  Returns [converged, final_m, c1_plus_c2, term_ratio]."""
        from . import expm
        e, b, h = self.eng, self.basis, self.h
        _, _, dbar = e.hnorms(b, h)
        _, a1, _ = e.hnorms(b, h, shift=dbar)
        ta = abs(t)  # the choice depends on |t| ||A||; a negative t propagates backwards
        m, s = expm.choose(ta * a1, d=lambda p: self._norm_power(ta, dbar, p))
        eta = np.exp(t * 1j * dbar / s)
        return e.expm_scaled(b, h, psi_in, psi_out, t, dbar, m, s, eta, tol=expm.TOL if not e.c64 else e.tol)

    def _norm_power(self, dt, dbar, p):
        """||(dt A)^p||_1^(1/p) for A = 1j (H - dbar I) on the current basis, by the block
        1-norm estimator (expm.onenormest) with every product on the device H rows."""
        from . import expm
        e, b, h = self.eng, self.basis, self.h
        n = b.count()
        cap = max(b.cap, 1)
        xin = torch.zeros(cap, dtype=e.cdtype, device=e.device)
        yout = torch.empty(cap, dtype=e.cdtype, device=e.device)

        def apply(X, sign):
            out = torch.empty_like(X)
            for j in range(X.shape[1]):
                xin[:n] = X[:, j].to(e.cdtype)
                e.apply_h(b, h, xin, yout)
                hx = yout[:n].to(torch.complex128)
                out[:, j] = (sign * 1j * dt) * (hx - dbar * X[:, j])
            return out

        def power(X, sign):
            for _ in range(p):
                X = apply(X, sign)
            return X

        if not hasattr(self, "_norm_gen"):
            self._norm_gen = torch.Generator(device=e.device)
            self._norm_gen.manual_seed(0x5EED)
        est = expm.onenormest(lambda X: power(X, 1.0), lambda X: power(X, -1.0), n, t=expm.ELL, itmax=5,
                              generator=self._norm_gen, device=e.device)
        return est ** (1.0 / p)

    def step(self, evolve=True, dt=0.0, weighted=None):
        """One time step (first step: evolve=False).  Returns the step record.  `weighted`
        (default: evolve) ranks the truncation by the look-ahead weights when the
        trajectory has a weighting."""
        w = evolve if weighted is None else weighted
        if self.use_graph and evolve and w == evolve and self.shuffle_seed is None:
            rec = self._graph_step(dt)
            if rec is not None:
                return rec
        nxt = 1 - self.cur
        for _ in range(12):
            rec = self.eng.step(self.bases[self.cur], self.psis[self.cur], self.bases[nxt], self.psis[nxt],
                                self.hs[nxt], self.params(evolve, dt, w))
            if rec.status == nat.ERR_CAPACITY:
                self._regrow()
                continue
            break
        if rec.status != nat.PACES_OK:
            raise nat.PacesError(rec.status, "paces_step")
        self.cur = nxt
        self.step_index += 1
        self._h_valid = True
        self.last = rec
        return rec

    def step_begin(self, dt, basis_ready):
        """Enqueue one evolving step on the current stream without waiting for it (no CUDA
        graph).  `basis_ready` is a torch.cuda.Event that has been recorded at least once
        (so that its CUDA event exists): the step records it again as soon as the new
        basis and its neighbour table are final, before the remap and the propagation,
        which only read them.  Returns the new slot's (basis, amplitudes, table); the
        amplitudes are final when the step is.  step_end() completes the step."""
        if getattr(self, "_pending", None) is not None:
            raise RuntimeError("step_begin: the previous step_begin has not been ended")
        if not basis_ready.cuda_event:
            raise ValueError("step_begin: record basis_ready once before passing it")
        nxt = 1 - self.cur
        prm = self.params(True, dt)
        prm.basis_ready = basis_ready.cuda_event
        self.eng.step(self.bases[self.cur], self.psis[self.cur], self.bases[nxt], self.psis[nxt], self.hs[nxt], prm,
                      sync=False)
        self._pending = (nxt, float(dt))
        return self.bases[nxt], self.psis[nxt], self.hs[nxt]

    def step_end(self):
        """Wait for the step of step_begin and return (record, repeated).  On a capacity
        overflow the buffers grow and the step runs again through step() (its inputs are
        read only, so the repeat is exact); repeated is then True, the new state lives in
        other buffers and what was copied out after basis_ready is void."""
        if getattr(self, "_pending", None) is None:
            raise RuntimeError("step_end without step_begin")
        nxt, dt = self._pending
        self._pending = None
        rec = self.eng.read_record()
        if rec.status == nat.ERR_CAPACITY:
            self._regrow()
            return self.step(evolve=True, dt=dt), True
        if rec.status != nat.PACES_OK:
            raise nat.PacesError(rec.status, "paces_step")
        self.cur = nxt
        self.step_index += 1
        self._h_valid = True
        self.last = rec
        return rec, False


class TrajectoryBatch:
    """Independent trajectories (each its own Engine: model, key width, dt, maxstates)
    advanced together by `paces_batch_step`: their stages run concurrently on the batch's
    streams and all their Taylor series in one persistent launch.  With `graph=True` each
    batch step replays a CUDA graph (one per slot parity and dt).  A capacity overflow in
    any trajectory grows that trajectory's buffers and repeats the batch step (inputs are
    read only, so the repeat is exact).
    """

    def __init__(self, trajs: list, n_streams=8, graph=False):
        if not trajs or len(trajs) > nat.MAX_BATCH:
            raise ValueError(f"a batch holds 1..{nat.MAX_BATCH} trajectories")
        devs = {t.eng.device for t in trajs}
        precs = {t.eng.c64 for t in trajs}
        if len(devs) != 1 or len(precs) != 1:
            raise ValueError("all trajectories of a batch share one device and one precision")
        self.trajs = list(trajs)
        self.device = trajs[0].eng.device
        self.lib = nat.load()
        self.use_graph = bool(graph)
        self._graphs = {}
        self.proposal = None  # (packed MLP parameters on the device, threshold) or None
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            nat.check(self.lib.paces_batch_create(len(trajs), int(n_streams), ctypes.byref(h)), None, "batch_create")
        self.handle = h
        self.rec_host = torch.zeros((len(trajs), ctypes.sizeof(nat.StepRecord)), dtype=torch.uint8).pin_memory()
        self.repeats = 0  # batch steps run again after a capacity overflow

    def _dts(self, dt):
        if isinstance(dt, (int, float)):
            return (float(dt),) * len(self.trajs)
        dts = tuple(float(x) for x in dt)
        if len(dts) != len(self.trajs):
            raise ValueError("one dt per trajectory")
        return dts

    def _items(self, evolve, dts):
        """C item array for the current slots; the ctypes objects it points to are kept."""
        keep, arr = [], (nat.BatchItem * len(self.trajs))()
        for i, t in enumerate(self.trajs):
            nxt = 1 - t.cur
            ob, nb, hm = t.bases[t.cur].c(), t.bases[nxt].c(), t.hs[nxt].c()
            prm = t.params(evolve, dts[i])
            ws, nbytes = t.eng.workspace()
            keep += [ob, nb, hm, prm]
            arr[i] = nat.BatchItem(t.eng.ctx, ctypes.pointer(ob), _ptr(t.psis[t.cur]), ctypes.pointer(nb),
                                   _ptr(t.psis[nxt]), ctypes.pointer(hm), ctypes.pointer(prm), _ptr(t.eng.rec_dev),
                                   ws, nbytes)
        return arr, keep

    def _launch(self, evolve, dts):
        arr, keep = self._items(evolve, dts)
        rc = self.lib.paces_batch_step(self.handle, arr, len(self.trajs), _stream(self.device))
        if rc != nat.PACES_OK:
            raise nat.PacesError(rc, self.lib.paces_batch_last_error(self.handle).decode(errors="replace"))
        return keep

    def _capture(self, dts):
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(self.device)
        torch.cuda.synchronize(self.device)
        with torch.cuda.graph(g, stream=s, capture_error_mode="relaxed"):
            keep = self._launch(True, dts)
        return g, keep

    def read_records(self):
        for i, t in enumerate(self.trajs):
            self.rec_host[i].copy_(t.eng.rec_dev, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        raw = self.rec_host.numpy()
        return [nat.StepRecord.from_buffer_copy(raw[i].tobytes()) for i in range(len(self.trajs))]

    def kernel_launches(self):
        return int(self.lib.paces_batch_kernel_launches(self.handle))

    def set_test_hooks(self, wait_limit_ns=0, skip_barrier_block=-1):
        """The batch's Taylor launch test hook (paces_batch_set_test_hooks)."""
        nat.check(self.lib.paces_batch_set_test_hooks(self.handle, int(wait_limit_ns), int(skip_barrier_block)),
                  None, "batch_set_test_hooks")

    def set_profiling(self, on=True):
        nat.check(self.lib.paces_batch_set_profiling(self.handle, 1 if on else 0), None, "batch_set_profiling")

    def stage_times(self):
        """Device ms of the last eager batch step: front stages, batched Taylor, back stages."""
        ms = (ctypes.c_float * 3)()
        nat.check(self.lib.paces_batch_stage_times(self.handle, ms), None, "batch_stage_times")
        return dict(zip(nat.BATCH_STAGES, [float(x) for x in ms]))

    def step(self, evolve=True, dt=0.0):
        """One time step of every trajectory (dt: one value, or one per trajectory);
        returns their records."""
        dts = self._dts(dt)
        graphed = self.use_graph and evolve and all(t.shuffle_seed is None for t in self.trajs)
        for _ in range(12):
            if graphed:
                key = (tuple(t.cur for t in self.trajs), dts, tuple(t.eng.tuning_epoch for t in self.trajs))
                if key not in self._graphs:
                    self._graphs[key] = self._capture(dts)
                self._graphs[key][0].replay()
            else:
                self._launch(evolve, dts)
            recs = self.read_records()
            grow = [i for i, r in enumerate(recs) if r.status == nat.ERR_CAPACITY]
            if grow:
                for i in grow:
                    self.trajs[i]._regrow()
                self._graphs = {}
                self.repeats += 1
                continue
            break
        for i, r in enumerate(recs):
            if r.status != nat.PACES_OK:
                raise nat.PacesError(r.status, f"batch item {i}")
        for t, r in zip(self.trajs, recs):
            t.cur = 1 - t.cur
            t.step_index += 1
            t._h_valid = True
            t.last = r
        return recs

    def close(self):
        if getattr(self, "handle", None):
            self._graphs = {}
            self.lib.paces_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
