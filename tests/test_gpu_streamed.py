"""paces_step_params.basis_ready: the event a step records once its new basis and neighbour
table are final, so another stream can copy them out while the propagation runs.  A step
started with it (Trajectory.step_begin / step_end) gives the same records, basis and
amplitudes as Trajectory.step, bit for bit; the basis copied on a second stream right after
the event equals the step's final basis; a capacity overflow repeats the step; and under
stream capture the event is recorded at every replay."""

import ctypes

import pytest
import torch

import gpu_helpers

pytestmark = pytest.mark.gpu


def _pair(nchain=12, dim=16, maxstates=3000, cap=1 << 14, **kw):
    trs = []
    for _ in range(2):
        eng = gpu_helpers.engine_for(nchain, dim, 1.3, cap=cap, precision="c64", periodic=True)
        tr, _ = gpu_helpers.grown_trajectory(eng, nchain, maxstates, dim=dim, **kw)
        trs.append(tr)
    return trs


def _raw(rec):
    return ctypes.string_at(ctypes.addressof(rec), ctypes.sizeof(rec))


def _streamed_step(tr, dt, ev, side):
    """step_begin, the new basis copied on `side` right after the event, step_end."""
    nb, npsi, nh = tr.step_begin(dt, ev)
    side.wait_event(ev)
    with torch.cuda.stream(side):
        blk = nb.blk.clone()
        keys = nb.keys.clone()
        nbr = nh.nbr.clone()
    rec, repeated = tr.step_end()
    side.synchronize()
    return rec, repeated, blk, keys, nbr


def test_streamed_steps_match_plain_steps():
    ref, st = _pair()
    ev = torch.cuda.Event()
    ev.record()
    side = torch.cuda.Stream()
    for k in range(6):
        ra = ref.step(evolve=True, dt=0.05)
        rb, repeated, blk, keys, nbr = _streamed_step(st, 0.05, ev, side)
        assert not repeated
        assert _raw(ra) == _raw(rb), k
        n = ra.n_states
        assert torch.equal(ref.basis.blk, st.basis.blk)
        assert torch.equal(ref.basis.keys[:n], st.basis.keys[:n])
        assert torch.equal(ref.psis[ref.cur][:n], st.psis[st.cur][:n])
        # what the second stream copied after the event is the final basis and table
        assert torch.equal(blk, st.basis.blk)
        assert torch.equal(keys[:n], st.basis.keys[:n])
        assert torch.equal(nbr[:n], st.h.nbr[:n])


def _shrink_to_state(tr):
    """Buffers and workspace of exactly the current state's size, the state kept: the next
    step's new basis cannot fit."""
    e = tr.eng
    n = tr.basis.count()
    keep = (tr.basis.keys[:n].clone(), tr.basis.blk.clone(), tr.psis[tr.cur][:n].clone())
    nbytes = ctypes.c_size_t()
    assert e.lib.paces_workspace_bytes(e.ctx, n, ctypes.byref(nbytes)) == 0
    e.ws = torch.empty(int(nbytes.value), dtype=torch.uint8, device=e.device)
    e.ws_bytes = int(nbytes.value)
    e.cap = n
    tr._alloc()
    tr.basis.keys[:n] = keep[0]
    tr.basis.blk.copy_(keep[1])
    tr.psis[tr.cur][:n] = keep[2]
    return n


def test_streamed_step_repeats_on_capacity_overflow():
    ref, st = _pair()
    for tr in (ref, st):
        tr.step(evolve=True, dt=0.05)
    n = _shrink_to_state(st)
    ev = torch.cuda.Event()
    ev.record()
    side = torch.cuda.Stream()
    ra = ref.step(evolve=True, dt=0.05)
    rb, repeated, _, _, _ = _streamed_step(st, 0.05, ev, side)
    assert repeated
    m = ra.n_states
    assert m > n or ra.n_enlarged > n
    assert st.eng.cap > n
    assert _raw(ra) == _raw(rb)
    assert torch.equal(ref.basis.keys[:m], st.basis.keys[:m])
    assert torch.equal(ref.psis[ref.cur][:m], st.psis[st.cur][:m])
    # and the next streamed step runs in the grown buffers
    ra = ref.step(evolve=True, dt=0.05)
    rb, repeated, _, keys, _ = _streamed_step(st, 0.05, ev, side)
    assert not repeated and _raw(ra) == _raw(rb)
    assert torch.equal(keys[:ra.n_states], ref.basis.keys[:ra.n_states])


def test_basis_ready_is_recorded_at_every_graph_replay():
    from paces_b200 import _native as nat
    eng = gpu_helpers.engine_for(12, 16, 1.3, cap=1 << 14, precision="c64", periodic=True)
    tr, _ = gpu_helpers.grown_trajectory(eng, 12, 3000)
    tr.step(evolve=True, dt=0.05)
    ev = torch.cuda.Event()
    ev.record()
    side = torch.cuda.Stream()
    cur, nxt = tr.cur, 1 - tr.cur
    prm = tr.params(True, 0.05)
    prm.basis_ready = ev.cuda_event
    args = (tr.bases[cur], tr.psis[cur], tr.bases[nxt], tr.psis[nxt], tr.hs[nxt], prm)
    eng.step(*args, sync=False)  # workspace and buffers settle before the capture
    first = eng.read_record()
    assert first.status == nat.PACES_OK
    n = first.n_states
    final_keys = tr.bases[nxt].keys[:n].clone()
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=torch.cuda.Stream(), capture_error_mode="relaxed"):
        eng.step(*args, sync=False)
    for _ in range(3):
        tr.bases[nxt].keys.zero_()
        g.replay()
        side.wait_event(ev)
        with torch.cuda.stream(side):
            keys = tr.bases[nxt].keys[:n].clone()
        side.synchronize()
        assert torch.equal(keys, final_keys)
    rec = eng.read_record()
    assert rec.status == nat.PACES_OK and rec.n_states == n
    assert _raw(rec) == _raw(first)
