"""CPU oracle for the learned candidate proposal.

TEST INFRASTRUCTURE ONLY: used by `tests/` to check the device kernels (event features,
labels, the MLP forward / backward / Adam step) and never by the product path.  The
proposal has no counterpart in the reference; this module restates the definitions in
paces_b200/csrc/proposal.cuh in NumPy, with the same rounding points (features and the
first hidden layer rounded to bf16, W1/W2 used as bf16), so the GPU results can be
compared value by value.  Parity against the reference itself does not apply here: the
method's judge is the plain (unfiltered) step, which is pinned separately.

Bases are reference rows (uint32, see paces_oracle).  Events of a basis X with nx states
are e = (j - 1) * nx + i for runs j = 1 (exciton hops right), 2 (left), 3 (phonon created
at the exciton site), 4 (annihilated).
"""

from __future__ import annotations

import numpy as np

from oracle import paces_oracle as po

RUN_FROM_LEFT, RUN_FROM_RIGHT, RUN_UP, RUN_DOWN = 1, 2, 3, 4
N_IN, N_HID = 16, 64
# fp32 master layout: W1 [64*16], W2 [64*64], b1, b2, w3 [64], b3
OFF_W1, OFF_W2 = 0, 1024
OFF_B1 = OFF_W2 + 4096
OFF_B2, OFF_W3, OFF_B3 = OFF_B1 + 64, OFF_B1 + 128, OFF_B1 + 192
N_MASTER = OFF_B3 + 1


def bf16(x):
    """Round float32 values to bf16 (nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def bf16_bits(x):
    return (bf16(x).view(np.uint32) >> 16).astype(np.uint16)


def unpack(model, rows):
    """(pos [n], occupations [n, L]) of reference rows."""
    pos = po.get_field(model, rows, 0).astype(np.int64)
    occ = np.stack([po.get_field(model, rows, s + 1).astype(np.int64) for s in range(model.nchain)], axis=1) \
        if rows.shape[0] else np.zeros((0, model.nchain), dtype=np.int64)
    return pos, occ


def events(model, rows):
    """Images of every event: run j, source i, exists, image position and occupations."""
    pos, occ = unpack(model, rows)
    nx, L = pos.shape[0], model.nchain
    maxd = np.asarray(model.max_ho_dims, dtype=np.int64)
    js, iis, ok, cpos, cocc = [], [], [], [], []
    idx = np.arange(nx)
    for j in (RUN_FROM_LEFT, RUN_FROM_RIGHT, RUN_UP, RUN_DOWN):
        c = occ.copy()
        if j == RUN_FROM_LEFT:
            p = pos + 1
            v = (p < L) | model.periodic
            p = p % L
        elif j == RUN_FROM_RIGHT:
            p = pos - 1
            v = (p >= 0) | model.periodic
            p = p % L
        else:
            p = pos.copy()
            n = occ[idx, pos] if nx else np.zeros(0, dtype=np.int64)
            if j == RUN_UP:
                v = n + 1 < maxd[pos]
                c[idx[v], pos[v]] += 1
            else:
                v = n > 0
                c[idx[v], pos[v]] -= 1
        js.append(np.full(nx, j))
        iis.append(idx)
        ok.append(np.asarray(v, dtype=bool))
        cpos.append(p)
        cocc.append(c)
    return (np.concatenate(js), np.concatenate(iis), np.concatenate(ok), np.concatenate(cpos),
            np.concatenate(cocc))


def features(model, rows, weights, cut=0.0):
    """float32 [4*nx, 16] features (bf16 values) and the exists flags; `cut` is the
    smallest amplitude the truncation kept (0: it dropped nothing)."""
    j, i, ok, cpos, cocc = events(model, rows)
    ne, L = j.shape[0], model.nchain
    maxd = np.asarray(model.max_ho_dims, dtype=np.int64)
    f = np.zeros((ne, N_IN), dtype=np.float32)
    r = np.arange(ne)
    for d in range(-4, 5):
        s = cpos + d
        if model.periodic:
            s = s % L
            inside = np.ones(ne, dtype=bool)
        else:
            inside = (s >= 0) & (s < L)
            s = np.clip(s, 0, L - 1)
        v = cocc[r, s].astype(np.float32) * (np.float32(1) / (maxd[s] - 1).astype(np.float32))
        f[:, d + 4] = np.where(inside, v, np.float32(0))
    f[:, 9] = cocc.sum(axis=1).astype(np.float32) * np.float32(1.0 / 16.0)
    w = np.asarray(weights, dtype=np.float32)[i]
    log_cut = np.log(np.maximum(np.float32(cut), np.float32(1e-30))).astype(np.float32)
    f[:, 10] = (np.log(np.maximum(w, np.float32(1e-30))).astype(np.float32) - log_cut) * np.float32(1.0 / 16.0)
    f[:, 11] = (j == RUN_FROM_LEFT) | (j == RUN_FROM_RIGHT)
    f[:, 12] = j == RUN_UP
    f[:, 13] = j == RUN_DOWN
    nc = cocc[r, cpos].astype(np.float32)
    g = np.float32(model.g)
    elem = np.where((j == RUN_FROM_LEFT) | (j == RUN_FROM_RIGHT), np.float32(model.J),
                    g * np.sqrt(np.where(j == RUN_UP, nc, nc + np.float32(1))).astype(np.float32)).astype(np.float32)
    f[:, 14] = np.log(np.maximum(np.abs(elem), np.float32(1e-30))).astype(np.float32) * np.float32(0.25)
    f[~ok] = 0
    return bf16(f), ok


def _row_set(model, pos, occ):
    raw = np.concatenate([pos[:, None], occ], axis=1)
    keys = po.compress(model, raw)
    return set(map(bytes, keys)), keys


def labels(model, x_rows, y_rows):
    """254 no image, 255 image already in X, 1 image in Y, 0 otherwise."""
    j, i, ok, cpos, cocc = events(model, x_rows)
    xset = set(map(bytes, np.ascontiguousarray(x_rows, dtype=np.uint32)))
    yset = set(map(bytes, np.ascontiguousarray(y_rows, dtype=np.uint32)))
    out = np.full(j.shape[0], 254, dtype=np.uint8)
    if j.shape[0]:
        raw = np.concatenate([cpos[:, None], cocc], axis=1)
        raw[~ok] = 0
        keys = po.compress(model, raw)
        for e in np.nonzero(ok)[0]:
            b = bytes(keys[e])
            out[e] = 255 if b in xset else (1 if b in yset else 0)
    return out


def split(master):
    m = np.asarray(master, dtype=np.float32)
    return (m[OFF_W1:OFF_W2].reshape(N_HID, N_IN), m[OFF_W2:OFF_B1].reshape(N_HID, N_HID), m[OFF_B1:OFF_B2],
            m[OFF_B2:OFF_W3], m[OFF_W3:OFF_B3], m[OFF_B3])


def init_master(seed=0):
    """He-style initialisation of the fp32 master weights."""
    rng = np.random.default_rng(seed)
    m = np.zeros(N_MASTER, dtype=np.float32)
    m[OFF_W1:OFF_W2] = rng.normal(0, np.sqrt(2.0 / N_IN), N_HID * N_IN)
    m[OFF_W2:OFF_B1] = rng.normal(0, np.sqrt(2.0 / N_HID), N_HID * N_HID)
    m[OFF_W3:OFF_B3] = rng.normal(0, np.sqrt(1.0 / N_HID), N_HID)
    return m


def forward(master, x, round_bf16=True):
    """Logits (float64) of feature rows x; W1, W2 and h1 rounded to bf16 like the kernels."""
    W1, W2, b1, b2, w3, b3 = split(master)
    if round_bf16:
        W1, W2 = bf16(W1), bf16(W2)
    x = np.asarray(x, dtype=np.float64)
    z1 = x @ W1.T.astype(np.float64) + b1
    h1 = np.maximum(z1, 0)
    if round_bf16:
        h1 = bf16(h1.astype(np.float32)).astype(np.float64)
    z2 = h1 @ W2.T.astype(np.float64) + b2
    h2 = np.maximum(z2, 0)
    return h2 @ w3.astype(np.float64) + float(b3), (x, z1, h1, z2, h2)


def loss_and_grads(master, x, y, sw, inv_norm, round_bf16=True):
    """inv_norm * sum_s sw_s BCE(logit_s, y_s) and its gradient in the master layout (the
    gradient with respect to the bf16 weights the forward pass uses)."""
    W1, W2, b1, b2, w3, b3 = split(master)
    if round_bf16:
        W1, W2 = bf16(W1), bf16(W2)
    logit, (xx, z1, h1, z2, h2) = forward(master, x, round_bf16)
    y = np.asarray(y, dtype=np.float64)
    sw = np.asarray(sw, dtype=np.float64)
    p = 1.0 / (1.0 + np.exp(-logit))
    loss = float(np.sum(sw * inv_norm * (np.maximum(logit, 0) + np.log1p(np.exp(-np.abs(logit))) - y * logit)))
    dl = sw * (p - y) * inv_norm
    dz2 = (z2 > 0) * dl[:, None] * w3.astype(np.float64)[None, :]
    g = np.zeros(N_MASTER, dtype=np.float64)
    g[OFF_W2:OFF_B1] = (dz2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = dz2.sum(axis=0)
    g[OFF_W3:OFF_B3] = dl @ h2
    g[OFF_B3] = dl.sum()
    dz1 = (dz2 @ W2.astype(np.float64)) * (h1 > 0)
    g[OFF_W1:OFF_W2] = (dz1.T @ xx).ravel()
    g[OFF_B1:OFF_B2] = dz1.sum(axis=0)
    return loss, g


def adam(master, m1, m2, grads, t, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One bias-corrected Adam step (float32), returning new (master, m1, m2)."""
    f = np.float32
    g = np.asarray(grads, dtype=np.float32)
    a = f(beta1) * m1 + (f(1) - f(beta1)) * g
    b = f(beta2) * m2 + (f(1) - f(beta2)) * g * g
    c1 = f(1.0 / (1.0 - beta1 ** t))
    c2 = f(1.0 / (1.0 - beta2 ** t))
    new = master - f(lr) * (a * c1) / (np.sqrt(b * c2) + f(eps))
    return new.astype(np.float32), a.astype(np.float32), b.astype(np.float32)
