"""Autotuner for the launch shapes of the time step.

These shapes change the speed of a step but never its results (each trajectory's
arithmetic and ordering are fixed by the data, not by the tiling):

* the merge tiles' splitter strides (tile = 17 * stride elements), one for the expansions
  and one for the assembly: larger tiles spend less on splitters and look-back, smaller ones
  fit more blocks per SM;
* the persistent Taylor kernel's blocks per SM (its grid) and its row schedule (rows read
  directly, or 512-row chunks prefetched into shared memory by bulk TMA copies).

`tune(trajectory, dt)` times candidates on the live workload -- eager steps with the
library's stage events -- and keeps, shape by shape, the fastest (the expansion stride by
the expand time and the assembly stride by the assemble time of the same trials, Taylor
blocks by the Taylor time).  `tune_batch` does the same for
a TrajectoryBatch with its phase times.  Choices are cached per (GPU name, key words,
precision, log2 of the basis size) in memory and in a JSON file
($PACES_TUNE_CACHE, default ~/.cache/paces_b200/tuning.json), so a later run of the same
workload on the same GPU model skips the search.
"""

from __future__ import annotations

import json
import math
import os

import torch

from . import _native as nat

CACHE_PATH = os.environ.get("PACES_TUNE_CACHE",
                            os.path.join(os.path.expanduser("~"), ".cache", "paces_b200", "tuning.json"))
_memory: dict = {}
VARIANTS = [0, 1]  # Taylor row schedules: direct, bulk-prefetched
SHAPES = ("merge_stride", "taylor_blocks_per_sm", "taylor_variant", "assemble_stride")


def get_tuning(eng) -> nat.Tuning:
    t = nat.Tuning()
    nat.check(eng.lib.paces_get_tuning(eng.ctx, t), eng.ctx, "get_tuning")
    return t


def set_tuning(eng, merge_stride=None, taylor_blocks_per_sm=None, taylor_variant=None, assemble_stride=None):
    """Set the given shapes, keeping the others; a merge_stride given without assemble_stride
    sets both strides."""
    t = get_tuning(eng)
    if merge_stride is not None:
        t.merge_stride = int(merge_stride)
        t.assemble_stride = int(merge_stride if assemble_stride is None else assemble_stride)
    elif assemble_stride is not None:
        t.assemble_stride = int(assemble_stride)
    if taylor_blocks_per_sm is not None:
        t.taylor_blocks_per_sm = int(taylor_blocks_per_sm)
    if taylor_variant is not None:
        t.taylor_variant = int(taylor_variant)
    nat.check(eng.lib.paces_set_tuning(eng.ctx, t), eng.ctx, "set_tuning")
    eng.tuning_epoch += 1  # graphs captured under the old shapes are not replayed


def stride_candidates(t: nat.Tuning):
    grid = [64, 80, 96, 128, 160, 192, 240]
    return [s for s in grid if t.merge_stride_min <= s <= t.merge_stride_max]


def bps_candidates(t: nat.Tuning):
    return [0] + list(range(1, t.taylor_blocks_per_sm_max))


# bumped when the kernels' tiling changes, so that choices cached for other tiles are not reused
CACHE_LAYOUT = 2


def _key(eng, states):
    name = torch.cuda.get_device_name(eng.device)
    return (f"v{CACHE_LAYOUT}|{name}|nw{eng.nw}|{'c64' if eng.c64 else 'c128'}"
            f"|s{int(round(math.log2(max(states, 1))))}")


def _load_file():
    try:
        with open(CACHE_PATH) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save_file(key, choice):
    try:
        data = _load_file()
        data[key] = choice
        os.makedirs(os.path.dirname(CACHE_PATH), exist_ok=True)
        tmp = CACHE_PATH + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, CACHE_PATH)
    except OSError:
        pass


def _lookup(key, use_cache):
    if not use_cache:
        return None
    if key in _memory:
        return _memory[key]
    return _load_file().get(key)


def _search(apply, measure, strides, bpss, variants, measure_taylor=None):
    """Coordinate search: the strides by their stages' times, then the Taylor schedule and
    grid by the Taylor time.  Every stride trial runs both merges at that stride; when
    measure() reports the expand and assemble stages apart, each merge keeps its own fastest
    stride, else one stride serves both.  The strides are timed in two passes, the second in
    reverse order, and each keeps its faster pass: a basis that still grows during the search
    then favours no end of the candidate list.  measure_taylor (when given) times the Taylor
    candidates on one fixed input, so that no candidate is judged on a step with fewer
    terms.  apply(expansion stride, assembly stride, blocks per SM, variant)."""
    timings = {"merge_stride": {}, "assemble_stride": {}, "taylor": {}}
    split = True
    for order in (list(strides), list(reversed(strides))):
        for s in order:
            apply(s, s, 0, variants[0])
            m = measure()
            split = split and "expand" in m and "assemble" in m
            e, a = (m["expand"], m["assemble"]) if split else (m["merge"], 0.0)
            timings["merge_stride"][s] = min(e, timings["merge_stride"].get(s, e))
            timings["assemble_stride"][s] = min(a, timings["assemble_stride"].get(s, a))
    best_s = min(timings["merge_stride"], key=timings["merge_stride"].get)
    best_a = min(timings["assemble_stride"], key=timings["assemble_stride"].get) if split else best_s
    if not split:
        del timings["assemble_stride"]
    for v in variants:
        for b in bpss:
            apply(best_s, best_a, b, v)
            timings["taylor"][(v, b)] = measure_taylor() if measure_taylor else measure()["taylor"]
    best_v, best_b = min(timings["taylor"], key=timings["taylor"].get)
    apply(best_s, best_a, best_b, best_v)
    timings["taylor"] = {f"variant{v}_bps{b}": ms for (v, b), ms in timings["taylor"].items()}
    return {"merge_stride": best_s, "assemble_stride": best_a, "taylor_blocks_per_sm": best_b,
            "taylor_variant": best_v, "timings_ms": timings}


def tune(tr, dt, steps=2, use_cache=True):
    """Pick the shapes for trajectory `tr` (its engine keeps them).  The candidate steps
    advance the trajectory like ordinary steps.  Returns the choice (and its timings when
    it was searched)."""
    eng = tr.eng
    key = _key(eng, tr.basis.count())
    hit = _lookup(key, use_cache)
    if hit is not None:
        set_tuning(eng, hit["merge_stride"], hit["taylor_blocks_per_sm"], hit.get("taylor_variant"),
                   assemble_stride=hit.get("assemble_stride"))
        return dict(hit, cached=True)
    t0 = get_tuning(eng)
    use_graph, tr.use_graph = tr.use_graph, False
    eng.set_profiling(True)

    def measure():
        tr.step(evolve=True, dt=dt)  # first step after a change: not timed
        acc = {"expand": 0.0, "assemble": 0.0, "taylor": 0.0}
        for _ in range(steps):
            tr.step(evolve=True, dt=dt)
            st = eng.stage_times()
            acc["expand"] += st["expand"]
            acc["assemble"] += st["assemble"]
            acc["taylor"] += st["taylor"]
        return {k: v / steps for k, v in acc.items()}

    def measure_taylor(reps=3):
        # the whole series on the trajectory's current state, the same input for every candidate
        b, h, psi = tr.basis, tr.h, tr.psis[tr.cur]
        out = torch.empty_like(psi)
        stream = torch.cuda.current_stream(eng.device)
        best = None
        for _ in range(reps + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eng.taylor(b, h, psi, dt, psi_out=out)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        return best

    try:
        choice = _search(lambda s, a, b, v: set_tuning(eng, s, b, v, assemble_stride=a), measure,
                         stride_candidates(t0), bps_candidates(t0), VARIANTS, measure_taylor=measure_taylor)
    finally:
        eng.set_profiling(False)
        tr.use_graph = use_graph
    tr._graphs = {}
    _memory[key] = {k: choice[k] for k in SHAPES}
    _save_file(key, _memory[key])
    return dict(choice, cached=False)


def tune_batch(batch, dt, steps=2, use_cache=True):
    """The same search for a TrajectoryBatch: one stride for every trajectory (timed by the
    batch's front phase) and the Taylor grid of its one persistent launch."""
    engs = [t.eng for t in batch.trajs]
    total = sum(t.basis.count() for t in batch.trajs)
    key = "batch|" + _key(engs[0], total) + f"|n{len(engs)}"
    hit = _lookup(key, use_cache)

    def apply(s, a, b, v=None):
        for e in engs:
            t = get_tuning(e)
            clamp = lambda x: min(max(x, t.merge_stride_min), t.merge_stride_max)
            set_tuning(e, clamp(s), b, v, assemble_stride=clamp(a))

    if hit is not None:
        apply(hit["merge_stride"], hit.get("assemble_stride", hit["merge_stride"]), hit["taylor_blocks_per_sm"])
        return dict(hit, cached=True)
    t0 = get_tuning(engs[0])
    use_graph, batch.use_graph = batch.use_graph, False
    batch.set_profiling(True)

    def measure():
        batch.step(evolve=True, dt=dt)
        acc = {"merge": 0.0, "taylor": 0.0}
        for _ in range(steps):
            batch.step(evolve=True, dt=dt)
            st = batch.stage_times()
            acc["merge"] += st["front"]
            acc["taylor"] += st["taylor"]
        return {k: v / steps for k, v in acc.items()}

    try:
        # the batched Taylor launch has one schedule; its grid is tuned, the variant is not
        choice = _search(apply, measure, stride_candidates(t0), bps_candidates(t0), [t0.taylor_variant])
    finally:
        batch.set_profiling(False)
        batch.use_graph = use_graph
    batch._graphs = {}
    for t in batch.trajs:
        t._graphs = {}
    _memory[key] = {k: choice[k] for k in SHAPES}
    _save_file(key, _memory[key])
    return dict(choice, cached=False)
