"""Learned candidate proposal: the MLP, its training on labels from plain runs, and a
trajectory that expands only the images the MLP keeps, with periodic full expansions as
judge and fallback.

No counterpart in the reference.  The network, features and keep rule are defined in
paces_b200/csrc/proposal.cuh; every kernel (features, labels, tensor-core scoring, the
training forward/backward and the Adam step) is in libpaces_b200.

Labels.  The images ("events") of the basis a step truncates to are its candidates; an
event is a positive when its image is in the basis the NEXT step truncates to (it would
have survived), a negative when it is not, and is not a candidate at all when the image
is already in the basis.  Plain runs (full expansion) generate them; the network is
trained on a class-balanced sample with weighted binary cross-entropy.

Threshold.  The keep threshold is the logit quantile that keeps `target_recall` of the
positives of a held-out step.  A LearnedTrajectory runs every `judge_every`-th step with
full expansion, scores that step's candidates anyway, labels them against the next
step's basis and, when fewer than `target_recall` of the positives would have been
kept, lowers the threshold to restore it.
"""

from __future__ import annotations

import ctypes
import dataclasses

import numpy as np
import torch

from . import _native as nat
from .engine import DevBasis, Trajectory, _ptr, _stream

N_IN, N_HID = 16, 64


class ProposalMLP:
    """The 16-64-64-1 network on one device: fp32 master weights, Adam moments, gradients
    and the packed bf16 inference parameters the kernels read."""

    def __init__(self, device, seed=0, master=None):
        self.lib = nat.load()
        self.device = torch.device(device)
        self.n_master = int(self.lib.paces_mlp_master_floats())
        self.n_bytes = int(self.lib.paces_mlp_param_bytes())
        if master is None:
            master = self.init_weights(seed)
        self.master = torch.as_tensor(np.asarray(master, dtype=np.float32)).to(self.device).contiguous()
        self.m1 = torch.zeros_like(self.master)
        self.m2 = torch.zeros_like(self.master)
        self.grads = torch.zeros_like(self.master)
        self.params = torch.zeros(self.n_bytes, dtype=torch.uint8, device=self.device)
        self.t = 0
        self.pack()

    @staticmethod
    def init_weights(seed):
        """He-style normal initialisation, biases zero (layout W1, W2, b1, b2, w3, b3)."""
        rng = np.random.default_rng(seed)
        w1 = rng.normal(0, np.sqrt(2.0 / N_IN), N_HID * N_IN)
        w2 = rng.normal(0, np.sqrt(2.0 / N_HID), N_HID * N_HID)
        w3 = rng.normal(0, np.sqrt(1.0 / N_HID), N_HID)
        return np.concatenate([w1, w2, np.zeros(2 * N_HID), w3, np.zeros(1)]).astype(np.float32)

    def pack(self):
        nat.check(self.lib.paces_mlp_pack(_ptr(self.master), _ptr(self.params), _stream(self.device)), None, "mlp_pack")

    def forward(self, x):
        """Logits of feature rows (bf16 [n, 16]) on CUDA cores."""
        n = int(x.shape[0])
        out = torch.empty(max(n, 1), dtype=torch.float32, device=self.device)
        nat.check(self.lib.paces_mlp_forward(_ptr(self.params), _ptr(x), n, _ptr(out), _stream(self.device)), None,
                  "mlp_forward")
        return out[:n]

    def backward(self, x, y, sw, inv_norm):
        """Accumulate the gradient of inv_norm * sum sw * BCE into self.grads; returns the loss."""
        loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        nat.check(self.lib.paces_mlp_backward(_ptr(self.params), _ptr(x), _ptr(y), _ptr(sw), int(x.shape[0]),
                                              float(inv_norm), _ptr(self.grads), _ptr(loss), _stream(self.device)),
                  None, "mlp_backward")
        return loss

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        self.t += 1
        nat.check(self.lib.paces_mlp_adam(_ptr(self.master), _ptr(self.m1), _ptr(self.m2), _ptr(self.grads), self.t,
                                          float(lr), float(beta1), float(beta2), float(eps), _ptr(self.params),
                                          _stream(self.device)), None, "mlp_adam")

    def fit(self, x, y, sw, epochs=4, batch=8192, lr=2e-3, seed=0):
        """Mini-batch Adam over (x, y, sw); returns the mean loss of every epoch."""
        g = torch.Generator(device=self.device)
        g.manual_seed(seed)
        n = int(x.shape[0])
        losses = []
        for _ in range(epochs):
            perm = torch.randperm(n, device=self.device, generator=g)
            tot = torch.zeros(1, dtype=torch.float64, device=self.device)
            for s in range(0, n, batch):
                idx = perm[s:s + batch]
                xb, yb, wb = x[idx].contiguous(), y[idx].contiguous(), sw[idx].contiguous()
                inv = 1.0 / float(max(wb.sum().item(), 1e-30))
                tot += self.backward(xb, yb, wb, inv) * float(wb.numel())
                self.adam(lr)
            losses.append(float(tot.item()) / n)
        return losses

    def state(self):
        return self.master.cpu().numpy().copy()


@dataclasses.dataclass
class Dataset:
    x: torch.Tensor      # bf16 [n, 16]
    y: torch.Tensor      # float32 [n]
    sw: torch.Tensor     # float32 [n]
    positives: int
    negatives: int


def collect(tr: Trajectory, steps, dt, neg_per_pos=8, max_neg=200_000, max_pos=100_000, seed=0, held_out=None):
    """Run `steps` plain steps of `tr` and gather labelled events of every step but the last
    (steps whose truncation dropped nothing -- the basis still growing -- have no cut and
    give no samples).

    Returns a class-balanced Dataset, and, when held_out is an int k, also the full
    (features, labels) of the k-th collected step for threshold calibration."""
    eng = tr.eng
    gen = torch.Generator(device=eng.device)
    gen.manual_seed(seed)
    xs, ys = [], []
    npos = nneg = 0
    prev = None
    hold = None
    for k in range(steps):
        try:
            tr.step(evolve=True, dt=dt)
        except nat.PacesError as err:
            # a tie shuffle over nearly every state (the reference raises there too): take
            # that step with the deterministic tie rule
            if err.code != nat.ERR_SHUFFLE:
                raise
            seed_, tr.shuffle_seed = tr.shuffle_seed, None
            tr.step(evolve=True, dt=dt)
            tr.shuffle_seed = seed_
        sel, w, cut = eng.selected()
        cur = sel.clone()
        saturated = float(cut.item()) > 0.0
        if prev is not None and saturated:
            px, pf = prev
            lab = eng.proposal_labels(px, cur)
            if held_out is not None and k - 1 == held_out:
                hold = (pf, lab.clone())
            pos = torch.nonzero(lab == 1).flatten()
            neg = torch.nonzero(lab == 0).flatten()
            if pos.numel() > max_pos:
                pos = pos[torch.randperm(pos.numel(), device=eng.device, generator=gen)[:max_pos]]
            keep_neg = min(int(neg.numel()), max(neg_per_pos * int(pos.numel()), 1), max_neg)
            if keep_neg < neg.numel():
                neg = neg[torch.randperm(neg.numel(), device=eng.device, generator=gen)[:keep_neg]]
            idx = torch.cat([pos, neg])
            xs.append(pf[idx])
            ys.append(torch.cat([torch.ones(pos.numel()), torch.zeros(neg.numel())]).to(eng.device))
            npos += int(pos.numel())
            nneg += int(neg.numel())
        # only steps whose truncation dropped states have a cut: their events are the samples
        prev = (cur, eng.proposal_features(cur, w[:cur.count()].clone(), cut.clone())[0]) if saturated else None
    x = torch.cat(xs)
    y = torch.cat(ys).float()
    # balance the classes: each holds half of the total weight
    sw = torch.where(y > 0, 0.5 / max(npos, 1), 0.5 / max(nneg, 1)).float() * float(x.shape[0])
    ds = Dataset(x, y, sw, npos, nneg)
    return (ds, hold) if held_out is not None else ds


def threshold_for_recall(logits, labels, recall):
    """Largest threshold that keeps at least `recall` of the positive events."""
    pos = logits[labels == 1]
    if pos.numel() == 0:
        return float("-inf")
    q = torch.sort(pos).values
    k = int(np.floor((1.0 - recall) * q.numel()))
    k = min(max(k, 0), q.numel() - 1)
    # keep rule is logit > threshold: step just below the k-th smallest positive logit
    return float(np.nextafter(np.float32(q[k].item()), np.float32(-np.inf)))


@dataclasses.dataclass
class JudgeRecord:
    step: int
    recall: float
    threshold_before: float
    threshold_after: float
    candidates: int
    kept: int


class LearnedTrajectory:
    """A trajectory whose expansions keep only the images the MLP scores above the
    threshold.  Every judge_every-th step runs the full expansion instead; its candidates
    are scored and, once the next step has truncated, labelled: the recall the threshold
    had on them is recorded, the network is fine-tuned on them (online_epochs passes of
    Adam over a class-balanced sample, 0 to switch off) and the threshold is re-set to keep
    target_recall of their positives (up or down)."""

    def __init__(self, tr: Trajectory, mlp: ProposalMLP, threshold, judge_every=10, target_recall=0.999,
                 online_epochs=1, online_lr=1e-3, max_pos=10_000, neg_per_pos=4):
        self.tr = tr
        self.mlp = mlp
        self.threshold = float(threshold)
        self.judge_every = int(judge_every)
        self.target_recall = float(target_recall)
        self.online_epochs = int(online_epochs)
        self.online_lr = float(online_lr)
        self.max_pos = int(max_pos)
        self.neg_per_pos = int(neg_per_pos)
        self.k = 0
        self._pending = None
        self.judges: list[JudgeRecord] = []
        self._gen = torch.Generator(device=tr.eng.device)
        self._gen.manual_seed(0)

    def _learn(self, feats, lab):
        dev = feats.device
        pos = torch.nonzero(lab == 1).flatten()
        neg = torch.nonzero(lab == 0).flatten()
        if pos.numel() == 0 or neg.numel() == 0:
            return
        if pos.numel() > self.max_pos:
            pos = pos[torch.randint(0, pos.numel(), (self.max_pos,), device=dev, generator=self._gen)]
        kn = min(int(neg.numel()), self.neg_per_pos * int(pos.numel()))
        neg = neg[torch.randint(0, neg.numel(), (kn,), device=dev, generator=self._gen)]
        x = torch.cat([feats[pos], feats[neg]])
        y = torch.cat([torch.ones(pos.numel(), device=dev), torch.zeros(neg.numel(), device=dev)])
        sw = torch.where(y > 0, 0.5 / pos.numel(), 0.5 / neg.numel()).float() * float(x.shape[0])
        self.mlp.fit(x, y, sw, epochs=self.online_epochs, lr=self.online_lr, seed=self.k)

    def step(self, dt):
        tr, eng = self.tr, self.tr.eng
        judge = self.judge_every > 0 and self.k % self.judge_every == 0
        tr.proposal = None if judge else (self.mlp.params, self.threshold)
        rec = tr.step(evolve=True, dt=dt)
        sel, w, cut = eng.selected()
        if self._pending is not None:
            px, feats, logits, thr_before = self._pending
            lab = eng.proposal_labels(px, sel)
            pos = lab == 1
            npos = int(pos.sum().item())
            recall = float(((logits > thr_before) & pos).sum().item()) / max(npos, 1)
            cand_mask = (lab == 0) | (lab == 1)
            cand = int(cand_mask.sum().item())
            kept = int((cand_mask & (logits > thr_before)).sum().item())
            thr = self.threshold
            if npos:
                if self.online_epochs > 0:
                    self._learn(feats, lab)
                    # the threshold needs the positives' logits only
                    pidx = torch.nonzero(pos).flatten()
                    logits = torch.full_like(logits, float("-inf"))
                    logits[pidx] = self.mlp.forward(feats[pidx].contiguous())
                thr = threshold_for_recall(logits, lab, self.target_recall)
            self.judges.append(JudgeRecord(self.k - 1, recall, thr_before, thr, cand, kept))
            self.threshold = thr
            self._pending = None
        if judge and float(cut.item()) > 0.0:
            x = sel.clone()
            n = x.count()
            ww, cc = w[:n].clone(), cut.clone()
            logits, _ = eng.proposal_score(x, ww, cc, self.mlp.params, self.threshold)
            feats = eng.proposal_features(x, ww, cc)[0] if self.online_epochs > 0 else None
            self._pending = (x, feats, logits.clone(), self.threshold)
        self.k += 1
        return rec
