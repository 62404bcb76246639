"""Benchmark of the adaptive-basis time step (Holstein chain, paces) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision c128|c64] [--maxstates M] [--nchain L] [--g G]

Workload (default): 1D periodic Holstein chain, single exciton, N=32 sites, J=1,
omega0=1, g=1.5, cutoff 15 (4-bit fields, 2 uint64 words per key), dt=0.05,
maxstates=2^22, enlarge_steps=1, exciton on site 0 with phonon vacuum.  A "step" is
one full adaptive time step (truncate -> expand -> sort/unique -> assemble H ->
remap -> Taylor exp(-i dt H) -> observables) once the basis is saturated at
maxstates.  Untimed preparation steps grow the basis to saturation first.

N > 1 (torchrun): independent replicas, one per GPU ("replicas only": the path is
not sharded); value = steps of all ranks / max-over-ranks time.

--impl reference times the CPU restatement of the reference (oracle/paces_oracle.py)
on the host cores, on a bounded sample of the same workload (smaller maxstates,
scaled linearly to the configured maxstates).
"""

import argparse
import ctypes
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=150)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="c64", choices=["c128", "c64"],
                    help="c64: the FP32 form, checked against a complex128 run of the same trajectory; "
                         "c128: the plain FP64 form alone")
    ap.add_argument("--no-compare", action="store_true",
                    help="c64: skip the complex128 comparison run over t = 10/J")
    ap.add_argument("--maxstates", type=int, default=1 << 22)
    ap.add_argument("--nchain", type=int, default=32)
    ap.add_argument("--g", type=float, default=1.5)
    ap.add_argument("--dt", type=float, default=0.05)
    ap.add_argument("--enlarge-steps", type=int, default=1)
    ap.add_argument("--open-chain", action="store_true", help="open boundaries (the reference's only mode)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-serial", action="store_true",
                    help="e2e: copy the new state out and the next input in one after the other")
    ap.add_argument("--e2e-chunk-mb", type=int, default=32, help="e2e: MB per copy of the streamed state")
    ap.add_argument("--no-learned", action="store_true",
                    help="plain: skip the learned form over the metric's window (training takes ~a minute)")
    ap.add_argument("--ref-steps", type=int, default=3,
                    help="reference arm: oracle steps timed at the configuration (each about a minute)")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--workload", default="plain", choices=["plain", "batched", "learned", "longchain"],
                    help="plain: one N=32 chain at maxstates 2^22; batched: 64 trajectories drawn from --seed; "
                         "learned: the learned proposal + complex64 against the plain complex128 run")
    ap.add_argument("--recall", type=float, default=0.999, help="learned: target recall of the keep threshold")
    ap.add_argument("--judge-every", type=int, default=10, help="learned: a full-expansion judge step every n steps")
    ap.add_argument("--train-seeds", type=int, default=8, help="learned: plain training runs (shuffle seeds 0..n-1)")
    ap.add_argument("--learn-from", type=int, default=50, help="learned: plain steps before the proposal is used")
    ap.add_argument("--total-steps", type=int, default=200, help="learned: steps of the compared trajectories")
    ap.add_argument("--realizations", type=int, default=4, help="longchain: disorder realizations batched")
    ap.add_argument("--sigma", type=float, default=0.5, help="longchain: site-energy disorder (Gaussian sigma)")
    ap.add_argument("--compare-steps", type=int, default=0,
                    help="longchain: steps of realization 0 compared against a complex128 run (0: none)")
    ap.add_argument("--weighting", default="none", choices=["none", "coherence", "norm"],
                    help="plain: rank the truncation by the look-ahead weights (TimeEvoParams.weighting_name)")
    ap.add_argument("--tau", type=float, default=0.2, help="plain: look-ahead time of --weighting")
    ap.add_argument("--lanczos-order", type=int, default=0,
                    help="plain: propagate by the Lanczos step of this order (ExpmParams.lanczos_order)")
    ap.add_argument("--no-graph", action="store_true", help="step without CUDA-graph replay")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch shapes (no autotuning)")
    ap.add_argument("--merge-stride", type=int, default=0, help="plain: this merge stride instead of tuning it")
    ap.add_argument("--assemble-stride", type=int, default=0,
                    help="plain, with --merge-stride: the assembly's own stride (default: the same)")
    ap.add_argument("--batch", type=int, default=64, help="trajectories of the batched workload")
    ap.add_argument("--seed", type=int, default=0, help="seed of the batched workload's draws")
    ap.add_argument("--streams", type=int, default=8, help="streams of the batched step")
    return ap.parse_args()


def workload_name(a):
    bc = "open" if a.open_chain else "periodic"
    return (f"holstein_{bc}_n{a.nchain}_cutoff15_g{a.g:g}_maxstates{a.maxstates}_dt{a.dt:g}"
            f"_es{a.enlarge_steps}")


def log(a, *msg):
    if a.verbose:
        print(*msg, file=sys.stderr, flush=True)


# --------------------------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for name, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "samples": len(sm),
                "reasons": sorted(reasons)}


# --------------------------------------------------------------------------------------------
# shared workload setup
# --------------------------------------------------------------------------------------------
def model_params(a, precision):
    from paces_b200.engine import ModelParams
    return ModelParams(nchain=a.nchain, max_ho_dims=[16] * a.nchain, J=1.0, g=a.g, eps_sys=0.0,
                       hbar_omega=1.0, delta_eps=0.0, periodic=not a.open_chain, precision=precision)


def initial_rows(nchain, initpos=0):
    from paces_b200 import layout
    raw = np.zeros((1, nchain + 1), dtype=np.uint32)
    raw[0, 0] = initpos
    return layout.pack_rows(raw, layout.bitwidths_for([nchain] + [16] * nchain))


def start_trajectory(eng, nchain, maxstates, es, initpos=0, graph=False, weighting="none", tau=0.0, lanczos_order=0):
    """grow_optimal_basis(fillfac=1) around the exciton on `initpos` in the phonon vacuum,
    amplitude 1 on that state, then the first (non-evolving) step."""
    import torch
    from paces_b200 import _native as nat
    from paces_b200.engine import Trajectory
    kind = {"none": nat.WEIGHT_NONE, "coherence": nat.WEIGHT_COHERENCE, "norm": nat.WEIGHT_NORM}[weighting]
    tr = Trajectory(eng, maxstates, es, graph=graph, weighting=kind, tau=tau if kind else 0.0,
                    lanczos_order=lanczos_order)
    rows = initial_rows(nchain, initpos)
    b = eng.basis_from_ref(rows)
    while True:
        nxt = eng.expand(b)
        if nxt.count() > maxstates or nxt.count() == 0:
            break
        b = nxt
    keys, pos, n = eng.query_from_ref(rows)
    idx = int(eng.lookup(b, keys, pos, n, must_exist=True)[0].item())
    psi = torch.zeros(max(b.count(), 1), dtype=eng.cdtype, device=eng.device)
    psi[idx] = 1.0
    tr.set_state(b, psi)
    tr.step(evolve=False)
    return tr


def prepare(a, eng, maxstates):
    """Grow the basis (grow_optimal_basis, fillfac=1), first step, then propagate until the
    truncation keeps exactly maxstates states; returns the saturated trajectory."""
    tr = start_trajectory(eng, a.nchain, maxstates, a.enlarge_steps, graph=not a.no_graph,
                          weighting=getattr(a, "weighting", "none"), tau=getattr(a, "tau", 0.0),
                          lanczos_order=getattr(a, "lanczos_order", 0))
    nprep = 1
    while True:
        rec = tr.step(evolve=True, dt=a.dt)
        nprep += 1
        log(a, f"prep step {nprep}: select={rec.n_select} enlarged={rec.n_enlarged} S={rec.n_states} "
               f"m={rec.final_m}")
        if rec.n_select >= maxstates and nprep >= 3:
            break
        if nprep > 400:
            raise RuntimeError("basis did not saturate")
    return tr, nprep


# The metric is quoted over t = 10/J at dt = 0.05: steps 51..200, the first 50 steps (basis growth
# and saturation) are the untimed lead-in.
WINDOW_FROM, WINDOW_TO = 50, 200


def evolving_steps(tr):
    """Evolving steps the trajectory has taken (its first step does not evolve)."""
    return tr.step_index - 1


def autotune_shapes():
    from paces_b200 import autotune
    return autotune.SHAPES


def max_over_ranks(value, dist, device="cuda"):
    """Largest value over all ranks (the timed region's duration); the value itself when
    there is no process group."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def taylor_bytes_per_term(rec, cs):
    """Algorithmic bytes of one Taylor term on S rows: neighbour table (16 B), row metadata
    (4 B), previous term read once, result read and written, new term written (4*cs)."""
    return rec.n_states * (16 + 4 + 4 * cs)


def lanczos_bytes(rec, cs, order):
    """Algorithmic bytes of one Lanczos propagation on S rows with order + 1 vectors: the norm
    pass (S*cs); per vector sweep A (table 16 B, metadata 4 B, the gathered source, q_{i-1}
    read, q_i and w written: 4*cs) and, but for the last vector, sweep B (w read and written,
    q_i read: 3*cs); the final combination (order + 1 vectors read, the result written)."""
    k = order + 1
    return rec.n_states * (cs + k * (20 + 4 * cs) + (k - 1) * 3 * cs + (k + 1) * cs)


def step_bytes(rec, cs, nw, es):
    """Algorithmic bytes of a whole step: truncation (S weights + M kept keys and weights),
    expansion (M keys in, B keys out), assembly (B keys in, S keys and table rows out),
    remap, the Taylor terms and the observables -- each stage's minimal HBM traffic."""
    kb = 8 * nw
    S, B, M = rec.n_states, rec.n_enlarged, rec.n_select
    truncate = S * cs + M * kb                      # read amplitudes, write kept keys
    expand = es * (M * kb + B * kb)                  # read the basis once, write the enlarged basis
    assemble = B * kb + S * kb + S * (16 + 4) + 5 * B * 4 + B * 32   # keys in/out, H table, maps, fill
    remap = 2 * S * kb + 2 * S * cs
    taylor = (rec.final_m + 1) * S * (16 + 4 + 4 * cs)
    obs = 2 * S * (cs + 4 + 16) + S * kb
    return truncate + expand + assemble + remap + taylor + obs


def read_peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_profile_traffic(precision):
    """DRAM bytes per row and Taylor term of the Taylor kernel from the committed ncu summary."""
    p = os.path.join(HERE, "profiles", f"taylor_kernel_{precision}.md")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        m = re.search(r"dram_bytes_per_row_term:\s*([0-9.]+)", f.read())
    return float(m.group(1)) if m else None


# --------------------------------------------------------------------------------------------
# CPU restatement (reference arm and cpu_baseline)
# --------------------------------------------------------------------------------------------
def oracle_at_config(a, dev, steps, warmup):
    """Time the CPU oracle (the NumPy restatement of the reference's step) at the workload's own
    configuration: the same chain and maxstates, from the saturated state at t = WINDOW_FROM * dt.
    That input state comes from a complex128 device run of the same trajectory (the oracle itself
    would need tens of minutes to grow it); the timed steps are the oracle's alone, each a full
    time step of the reference algorithm (truncation, expansion, lexsort/unique, searchsorted
    lookups, COO/CSR assembly, Taylor series with SciPy CSR SpMV, observables, diagnostics).
    Returns (steps/s, description)."""
    import torch
    from oracle import paces_oracle as po
    from paces_b200.engine import Engine
    eng = Engine(model_params(a, "c128"), device=dev)
    tr = start_trajectory(eng, a.nchain, a.maxstates, a.enlarge_steps)
    while evolving_steps(tr) < WINDOW_FROM:
        tr.step(evolve=True, dt=a.dt)
    rows = eng.basis_to_ref(tr.basis).cpu().numpy().view(np.uint32).copy()
    vec = tr.vector.cpu().numpy().astype(np.complex128)
    S0 = int(rows.shape[0])
    eng.close()
    del tr, eng
    torch.cuda.empty_cache()
    model = po.Model(a.nchain, [16] * a.nchain, g=a.g, periodic=not a.open_chain)
    otr = po.Trajectory(model, rows, vec, a.maxstates, a.enlarge_steps)
    t = WINDOW_FROM * a.dt
    for _ in range(warmup):
        t += a.dt
        otr.step(t, a.dt)
    t0 = time.perf_counter()
    for _ in range(steps):
        t += a.dt
        otr.step(t, a.dt)
    wall = time.perf_counter() - t0
    threads = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "MKL_NUM_THREADS", "OPENBLAS_NUM_THREADS")}
    desc = (f"{steps} oracle steps (after {warmup} untimed) of the configuration itself, maxstates={a.maxstates}, "
            f"from the saturated state at step {WINDOW_FROM} (S={S0} -> {otr.records[-1].numstates}), "
            f"{wall:.1f} s; host nproc={os.cpu_count()}, threads {threads}: NumPy lexsort/searchsorted and "
            f"SciPy CSR SpMV run on one core")
    return steps / wall, desc


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    # each oracle step at the configuration takes about a minute: a bounded sample of the
    # requested steps, at the configuration itself (not scaled from a smaller one)
    steps = max(1, min(a.steps, a.ref_steps))
    warmup = min(max(a.warmup, 0), 1)
    value, desc = oracle_at_config(a, f"cuda:{local}", steps, warmup)
    line = {"impl": "reference", "metric": metric_name(a),
            "value": value, "unit": "time-steps/s",
            "n_gpus": a.gpus, "steps": steps, "warmup": warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": workload_config(a, "c128"),
            "sample": f"{steps} of the {a.steps} requested steps (each about a minute of CPU work)",
            "cpu_baseline": {"value": value, "unit": "time-steps/s", "cores": 1, "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": "time-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def metric_name(a):
    """The line's metric: time-steps/s at 4M states, named with the form the value measures."""
    if a.precision == "c64":
        return ("time-steps/s at 4M states: FP32 (complex64, fp64 scalars) vs plain FP64, observable err <=1e-5; "
                "the learned+FP32 form is reported beside it (window.learned_c64)")
    return "time-steps/s at 4M states (plain FP64)"


def workload_config(a, precision):
    return {"workload": workload_name(a), "nchain": a.nchain, "cutoff": 15, "g": a.g, "omega0": 1.0, "J": 1.0,
            "dt": a.dt, "maxstates": a.maxstates, "enlarge_steps": a.enlarge_steps,
            "boundary": "open" if a.open_chain else "periodic", "precision": precision,
            "timed_steps_from": WINDOW_FROM + 1}


# --------------------------------------------------------------------------------------------
# device arm
# --------------------------------------------------------------------------------------------
def run_ours(a):
    import torch
    from paces_b200 import _native as nat
    from paces_b200.engine import Engine

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    eng = Engine(model_params(a, a.precision), device=f"cuda:{local}")
    cs = 8 if a.precision == "c64" else 16
    tr, nprep = prepare(a, eng, a.maxstates)
    tuning = None
    if a.merge_stride:
        from paces_b200 import autotune
        autotune.set_tuning(eng, merge_stride=a.merge_stride, assemble_stride=a.assemble_stride or None)
        t = autotune.get_tuning(eng)
        tuning = {"merge_stride": t.merge_stride, "assemble_stride": t.assemble_stride,
                  "taylor_blocks_per_sm": t.taylor_blocks_per_sm, "taylor_variant": t.taylor_variant}
    elif not a.no_tune:
        from paces_b200 import autotune
        tuning = autotune.tune(tr, a.dt)
        log(a, f"tuning: {tuning}")
    # warm-up: at least W steps, and up to step WINDOW_FROM, so the timed steps are the
    # metric's window (steps 51.. of t = 10/J)
    nwarm = max(a.warmup, WINDOW_FROM - evolving_steps(tr))
    for _ in range(nwarm):
        tr.step(evolve=True, dt=a.dt)
    first_timed = evolving_steps(tr) + 1

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # timed region: K steps, each replaying the step's CUDA graph and reading its record
    recs = []
    barrier()
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(a.steps):
            recs.append(tr.step(evolve=True, dt=a.dt))
        ev1.record(stream)
        ev1.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist)
    clocks = clk.summary()
    barrier()

    # stage split and the Taylor launch time: eager steps with CUDA events between stages
    n_prof = max(3, min(a.steps, 10))
    eng.set_profiling(True)
    stage_sum = {s_: 0.0 for s_ in nat.STAGES}
    prof_recs = []
    launches0 = eng.kernel_launches()
    use_graph, tr.use_graph = tr.use_graph, False
    for _ in range(n_prof):
        prof_recs.append(tr.step(evolve=True, dt=a.dt))
        for k, v in eng.stage_times().items():
            stage_sum[k] += v
    tr.use_graph = use_graph
    launches_per_step = (eng.kernel_launches() - launches0) / n_prof
    launches = int(round(launches_per_step * a.steps))
    eng.set_profiling(False)
    barrier()

    # e2e: the C ABI called with host buffers -- every step copies the state in from pinned
    # host memory, runs paces_step, and copies the new state and its record back out.
    e2e = None
    if not a.no_e2e:
        e2e = run_e2e(a, eng, tr, barrier, dist)

    compare = None
    if a.precision == "c64" and not a.no_compare and a.weighting == "none" and not a.lanczos_order:
        compare = compare_precisions(a, f"cuda:{local}", dist, learned=not a.no_learned)

    total_steps = a.steps * world
    value = total_steps / (ms / 1e3)
    taylor_ms = stage_sum["taylor"] / n_prof
    terms = statistics.mean(r.final_m + 1 for r in recs)
    S_mean = statistics.mean(r.n_states for r in recs)
    if a.lanczos_order:
        taylor_alg = statistics.mean(lanczos_bytes(r, cs, a.lanczos_order) for r in prof_recs)
    else:
        taylor_alg = statistics.mean(taylor_bytes_per_term(r, cs) * (r.final_m + 1) for r in prof_recs)
    achieved = taylor_alg / (taylor_ms / 1e3) / 1e9
    peak, peak_kind = read_peaks()
    per_row_term = read_profile_traffic(a.precision)
    traffic = None if per_row_term is None else per_row_term * S_mean * terms
    step_alg = statistics.mean(step_bytes(r, cs, eng.nw, a.enlarge_steps) for r in recs)
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        v, desc = oracle_at_config(a, f"cuda:{local}", 1, 0)  # one full oracle step at the configuration
        cpu = {"value": v, "unit": "time-steps/s", "cores": 1, "kind": "port", "sample": desc}
    if rank == 0:
        cfg = workload_config(a, a.precision)
        cfg.update({"timed_steps": f"{first_timed}..{first_timed + a.steps - 1}",
                    "states_per_step": int(S_mean), "taylor_terms_per_step": terms, "prep_steps": nprep,
                    "l2": "inputs larger than L2 (state and H table > 126 MB)", "parallelism": f"replicas x{world}",
                    "cuda_graph": not a.no_graph,
                    "weighting": None if a.weighting == "none" else {"name": a.weighting, "tau": a.tau},
                    "propagator": f"lanczos order {a.lanczos_order}" if a.lanczos_order else "taylor",
                    "tuning": None if tuning is None else {k: tuning[k] for k in autotune_shapes()},
                    "form": ("plain method in complex64: amplitudes and SpMV in fp32, norms, stop test and sums in "
                             "fp64; the learned proposal is off in the timed steps (window.learned_c64 measures "
                             "the learned form)") if a.precision == "c64" else "complex128 plain"})
        line = {
            "metric": metric_name(a),
            "value": value, "unit": "time-steps/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": a.precision, "data": "synthetic", "config": cfg,
            "roofline": {"bound": "hbm", "kernel": "lanczos_kernel" if a.lanczos_order else "taylor_kernel",
                         "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None if a.lanczos_order else traffic,
                         "algorithmic_bytes": taylor_alg, "launch_ms": taylor_ms},
            "step_roofline": {"achieved": step_alg / (ms / a.steps / 1e3) / 1e9, "unit": "GB/s",
                              "frac": step_alg / (ms / a.steps / 1e3) / 1e9 / peak},
            "stage_ms": {k: v / n_prof for k, v in stage_sum.items()}, "stage_steps": n_prof,
            "clocks": clocks, "gpu_launches": launches, "cpu_baseline": cpu, "e2e": e2e,
        }
        if compare is not None:
            line.update(compare)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def window_observables(recs, L):
    return {"n_exc": np.array([list(r.n_exc)[:L] for r in recs]), "n_pho": np.array([list(r.n_pho)[:L] for r in recs]),
            "energy": np.array([r.energy_re for r in recs]), "norm": np.array([r.norm for r in recs])}


def timed_steps(fn, n):
    """Run fn() n times on the current stream between two CUDA events; (results, ms)."""
    import torch
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = [fn() for _ in range(n)]
    e1.record(stream)
    e1.synchronize()
    return out, e0.elapsed_time(e1)


def train_proposal(a, dev, lf=WINDOW_FROM):
    """The learned proposal's training on the GPU: keep/drop labels from the first lf steps of
    plain complex64 runs at shuffle seeds 0..train_seeds-1, then the MLP fitted by the library's
    forward/backward/Adam kernels and the keep threshold set for the target recall on held-out
    steps.  Returns (mlp, threshold, info)."""
    import torch
    from paces_b200.engine import Engine
    from paces_b200.proposal import ProposalMLP, collect, threshold_for_recall
    xs, ys, sws, hold = [], [], [], None
    t0 = time.perf_counter()
    for seed in range(a.train_seeds):
        eng = Engine(model_params(a, "c64"), device=dev)
        tr = start_trajectory(eng, a.nchain, a.maxstates, a.enlarge_steps)
        tr.shuffle_seed = seed
        ds, h = collect(tr, lf, a.dt, neg_per_pos=4, max_pos=25_000, seed=seed, held_out=lf - 5)
        xs.append(ds.x)
        ys.append(ds.y)
        sws.append(ds.sw)
        hold = hold or h
        eng.close()
    collect_s = time.perf_counter() - t0
    x, y, sw = torch.cat(xs), torch.cat(ys), torch.cat(sws)
    mlp = ProposalMLP(dev, seed=0)
    t0 = time.perf_counter()
    losses = mlp.fit(x, y, sw, epochs=2, batch=8192, lr=2e-3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    thr0 = threshold_for_recall(mlp.forward(hold[0]), hold[1], a.recall)
    info = {"runs": a.train_seeds, "steps_per_run": lf, "samples": int(x.shape[0]), "positives": int(y.sum().item()),
            "epochs": 2, "loss": losses, "collect_s": collect_s, "train_s": train_s}
    return mlp, thr0, info


def learned_run(a, dev, mlp, thr0, lf=WINDOW_FROM, total=WINDOW_TO):
    """Plain complex64 for lf steps, then the proposal (full-expansion judge every 10th step)
    until step `total`: (records of steps 0..total, ms of steps lf+1..total, the learned
    trajectory, its engine)."""
    from paces_b200.engine import Engine
    from paces_b200.proposal import LearnedTrajectory
    eng = Engine(model_params(a, "c64"), device=dev)
    tr = start_trajectory(eng, a.nchain, a.maxstates, a.enlarge_steps, graph=not a.no_graph)
    recs = [tr.last] + [tr.step(evolve=True, dt=a.dt) for _ in range(lf)]
    lt = LearnedTrajectory(tr, mlp, thr0, judge_every=a.judge_every, target_recall=a.recall)
    window, ms = timed_steps(lambda: lt.step(a.dt), total - lf)
    return recs + window, ms, lt, eng


def compare_precisions(a, dev, dist, total=WINDOW_TO, window_from=WINDOW_FROM, learned=True):
    """The metric's comparison over t = 0 .. total * dt, on fresh runs of the same trajectory:
    complex128 (the FP64 plain oracle), complex64, and with `learned` the learned proposal in
    complex64 (trained first on the GPU).  Time-steps/s of each over steps window_from+1..total
    and the largest difference of every observable from the complex128 run."""
    from paces_b200.engine import Engine
    obs, rate = {}, {}
    for prec in ("c128", "c64"):
        eng = Engine(model_params(a, prec), device=dev)
        tr = start_trajectory(eng, a.nchain, a.maxstates, a.enlarge_steps, graph=not a.no_graph)
        recs = [tr.last] + [tr.step(evolve=True, dt=a.dt) for _ in range(window_from)]
        window, ms = timed_steps(lambda: tr.step(evolve=True, dt=a.dt), total - window_from)
        rate[prec] = (total - window_from) / (max_over_ranks(ms, dist) / 1e3)
        obs[prec] = window_observables(recs + window, a.nchain)
        eng.close()
    training = None
    lt = None
    if learned:
        mlp, thr0, training = train_proposal(a, dev, window_from)
        recs, ms, lt, eng = learned_run(a, dev, mlp, thr0, window_from, total)
        rate["learned_c64"] = (total - window_from) / (max_over_ranks(ms, dist) / 1e3)
        obs["learned_c64"] = window_observables(recs, a.nchain)
        win = recs[window_from + 1:]
        training.update({"target_recall": a.recall, "threshold_start": thr0, "threshold_end": lt.threshold,
                         "states_per_step": statistics.mean(r.n_states for r in win),
                         "enlarged_per_step": statistics.mean(r.n_enlarged for r in win),
                         "judge_steps": len(lt.judges)})
        eng.close()
    err = {form: {k: float(np.max(np.abs(obs["c128"][k] - obs[form][k]))) for k in obs["c128"]}
           for form in obs if form != "c128"}
    out = {"steps": f"{window_from + 1}..{total} of fresh runs (t = {total * a.dt:g}/J)",
           "plain_c128": {"value": rate["c128"], "unit": "time-steps/s"},
           "plain_c64": {"value": rate["c64"], "unit": "time-steps/s"},
           "ratio_c64_vs_c128": rate["c64"] / rate["c128"],
           "observable_error_vs_c128": err, "bound": 1e-5,
           "within_bound": {form: all(v <= 1e-5 for v in e.values()) for form, e in err.items()}}
    if learned:
        out["learned_c64"] = {"value": rate["learned_c64"], "unit": "time-steps/s", "training": training}
        out["ratio_learned_vs_c128"] = rate["learned_c64"] / rate["c128"]
        out["ratio_learned_vs_plain_c64"] = rate["learned_c64"] / rate["c64"]
    return {"window": out}


def run_e2e(a, eng, tr, barrier, dist):
    """The C ABI with the state in pinned host memory: every step copies its input state in
    and its new state (and record) out.  The new state is the next step's input, so each
    chunk of it goes back in as soon as it has landed on the host, on a second copy stream:
    the two directions of the link run at once.  The new basis (and table) starts out as soon
    as the step has built it (paces_step_params.basis_ready), while the remap, the
    propagation and the observables run; the amplitudes follow when the step ends.
    --e2e-serial: one copy after the other, after the step."""
    import torch
    e = eng
    cs = 8 if a.precision == "c64" else 16
    cap = e.cap
    hk = torch.empty((cap, e.nw), dtype=torch.int64).pin_memory()
    hb = torch.empty(e.L + 1, dtype=torch.int32).pin_memory()
    hp = torch.empty(cap, dtype=e.cdtype).pin_memory()
    # with the look-ahead weighting the state includes the basis' neighbour table
    table = bool(tr.weighting)
    if table:
        hn = torch.empty((cap, 4), dtype=torch.int32).pin_memory()
        hm = torch.empty(cap, dtype=torch.int32).pin_memory()

    def basis_pairs(n, b=None, h=None):
        """(device, host) views of the basis part of the state (keys, table), whole rows;
        the block offsets travel on their own."""
        b = tr.basis if b is None else b
        h = tr.h if h is None else h
        out = [(b.keys[:n], hk[:n])]
        if table:
            out += [(h.nbr[:n], hn[:n]), (h.meta[:n], hm[:n])]
        return out

    def pairs(n):
        """(device, host) views of the whole current state."""
        return [(tr.basis.blk, hb), (tr.psis[tr.cur][:n], hp[:n])] + basis_pairs(n)

    def nbytes(n):
        return n * (e.nw * 8 + cs) + (e.L + 1) * 4 + (n * 20 if table else 0)

    n = tr.basis.count()
    for dev, host in pairs(n):
        host.copy_(dev)
    main = torch.cuda.current_stream()
    s_out, s_in = torch.cuda.Stream(), torch.cuda.Stream()
    chunk = max(1, a.e2e_chunk_mb) << 20  # bytes per copy
    basis_ready = torch.cuda.Event()
    basis_ready.record(main)  # creates the event the steps record

    def stream_out_in(dev, host, back, after=None):
        """dev -> host in chunks on s_out; with `back`, each chunk returns to dev on s_in
        once it has landed (and, with `after`, not before that event)."""
        if dev.shape[0] == 0:
            return
        row_bytes = dev.element_size() * (dev.shape[1] if dev.dim() > 1 else 1)
        rows = max(1, chunk // row_bytes)
        if back and after is not None:
            s_in.wait_event(after)
        for r0 in range(0, dev.shape[0], rows):
            with torch.cuda.stream(s_out):
                host[r0:r0 + rows].copy_(dev[r0:r0 + rows], non_blocking=True)
            if back:
                landed = torch.cuda.Event()
                landed.record(s_out)
                s_in.wait_event(landed)
                with torch.cuda.stream(s_in):
                    dev[r0:r0 + rows].copy_(host[r0:r0 + rows], non_blocking=True)

    h2d = d2h = 0
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(main)
    for dev, host in pairs(n):  # the first step's input
        dev.copy_(host, non_blocking=True)
    h2d += nbytes(n)
    for k in range(a.steps):
        nxt = k + 1 < a.steps  # the new state goes back in as the next step's input
        if a.e2e_serial:
            rec = tr.step(evolve=True, dt=a.dt)
            n = rec.n_states
            for dev, host in pairs(n):
                host.copy_(dev, non_blocking=True)
            if nxt:
                for dev, host in pairs(n):
                    dev.copy_(host, non_blocking=True)
        else:
            nbas, npsi, nh = tr.step_begin(a.dt, basis_ready)
            done = torch.cuda.Event()
            done.record(main)
            # the new basis' size, as soon as the basis is final
            s_out.wait_event(basis_ready)
            with torch.cuda.stream(s_out):
                hb.copy_(nbas.blk, non_blocking=True)
            sized = torch.cuda.Event()
            sized.record(s_out)
            sized.synchronize()
            n = int(hb[e.L])
            # the basis goes out while the step runs on; nothing goes back in before the
            # step has ended (its observables read the keys)
            if nxt:
                s_in.wait_event(done)
                with torch.cuda.stream(s_in):
                    nbas.blk.copy_(hb, non_blocking=True)
            for dev, host in basis_pairs(n, nbas, nh):
                stream_out_in(dev, host, nxt)
            s_out.wait_event(done)
            stream_out_in(npsi[:n], hp[:n], nxt)
            main.wait_stream(s_out)
            main.wait_stream(s_in)
            rec, repeated = tr.step_end()
            if repeated:  # a capacity overflow ran the step again in other buffers
                n = rec.n_states
                for dev, host in pairs(n):
                    host.copy_(dev, non_blocking=True)
                if nxt:
                    for dev, host in pairs(n):
                        dev.copy_(host, non_blocking=True)
        d2h += nbytes(n) + ctypes.sizeof(type(rec))
        if nxt:
            h2d += nbytes(n)
        main.synchronize()  # the host holds the new state
    ev1.record(main)
    ev1.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist)
    world = 1 if dist is None else dist.get_world_size()
    return {"value": a.steps * world / (ms / 1e3), "unit": "time-steps/s",
            "h2d_bytes_per_step": h2d // a.steps, "d2h_bytes_per_step": d2h // a.steps,
            "api": "paces_step (C ABI) with the state in pinned host memory"
                   + ("" if a.e2e_serial else "; the new basis streams out from the moment the step has built it, "
                      "the amplitudes when it ends, and each chunk goes back in on a second copy stream")}

# --------------------------------------------------------------------------------------------
# batched workload: independent trajectories advanced together
# --------------------------------------------------------------------------------------------
def batched_specs(seed, n):
    """n Holstein rings drawn from numpy.random.default_rng(seed), one parameter at a time
    in this order: g ~ U[0.5, 2], omega0 ~ U[0.5, 1.5], N uniform over {16, 24, 32},
    maxstates = round(2^U[14, 20]) (log-uniform), exciton site uniform over the ring."""
    rng = np.random.default_rng(seed)
    g = rng.uniform(0.5, 2.0, n)
    w0 = rng.uniform(0.5, 1.5, n)
    N = rng.choice(np.array([16, 24, 32]), n)
    M = np.round(2.0 ** rng.uniform(14.0, 20.0, n)).astype(np.int64)
    site = rng.integers(0, N)
    return [dict(g=float(g[i]), omega0=float(w0[i]), nchain=int(N[i]), maxstates=int(M[i]), site=int(site[i]))
            for i in range(n)]


def warm_up_batch(batch, trajs, warmup, dt, headroom=1.6, extra=30):
    """Untimed batch steps before the timed ones.  An overflow in the timed steps would run
    that batch step again and capture its graphs anew, so every trajectory first gets room
    for `headroom` times its states, and the warm-up goes on (at most `extra` more steps)
    until `warmup` steps in a row have run without a repeat.  Returns the steps taken."""
    grown = False
    for t in trajs:
        need = int(headroom * t.last.n_states) + 64
        if t.eng.cap < need:
            t._regrow(need / t.eng.cap)
            grown = True
    if grown:
        batch._graphs = {}
    steps = quiet = 0
    want = max(warmup, 1)
    while steps < max(warmup, 0) or (quiet < want and steps < max(warmup, 0) + extra):
        r0 = batch.repeats
        batch.step(evolve=True, dt=dt)
        steps += 1
        quiet = quiet + 1 if batch.repeats == r0 else 0
    return steps


def run_batched(a):
    import torch
    from paces_b200 import _native as nat
    from paces_b200.engine import Engine, ModelParams, TrajectoryBatch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    cs = 8 if a.precision == "c64" else 16
    # each rank runs its own draw of the batch (replicas: rank r uses seed + r)
    specs = batched_specs(a.seed + rank, a.batch)
    trajs = []
    for sp in specs:
        eng = Engine(ModelParams(nchain=sp["nchain"], max_ho_dims=[16] * sp["nchain"], J=1.0, g=sp["g"],
                                 hbar_omega=sp["omega0"], periodic=True, precision=a.precision),
                     device=f"cuda:{local}")
        trajs.append(start_trajectory(eng, sp["nchain"], sp["maxstates"], a.enlarge_steps, sp["site"],
                                      graph=not a.no_graph))
    batch = TrajectoryBatch(trajs, n_streams=a.streams, graph=not a.no_graph)
    nprep = 0
    while True:
        recs = batch.step(evolve=True, dt=a.dt)
        nprep += 1
        if all(r.n_select >= sp["maxstates"] for r, sp in zip(recs, specs)) or nprep >= 60:
            break
    tuning = None
    if not a.no_tune:
        from paces_b200 import autotune
        tuning = autotune.tune_batch(batch, a.dt)
    warm_up_batch(batch, trajs, a.warmup, a.dt)
    repeats0 = batch.repeats

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    rounds = []
    barrier()
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(a.steps):
            rounds.append(batch.step(evolve=True, dt=a.dt))
        ev1.record(stream)
        ev1.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist)
    clocks = clk.summary()
    repeated_timed = batch.repeats - repeats0
    barrier()

    # phase split (eager batch steps with events) and the batched Taylor launch
    n_prof = max(3, min(a.steps, 10))
    batch.set_profiling(True)
    batch.use_graph = False
    phase = {k: 0.0 for k in nat.BATCH_STAGES}
    prof = []
    l0 = batch.kernel_launches()
    for _ in range(n_prof):
        prof.append(batch.step(evolve=True, dt=a.dt))
        for k, v in batch.stage_times().items():
            phase[k] += v
    launches_per_step = (batch.kernel_launches() - l0) / n_prof
    batch.set_profiling(False)
    batch.use_graph = not a.no_graph
    barrier()

    # the same trajectories stepped one after another (paces_step each, graphs on)
    seq_steps = 2
    for t in trajs:
        t.use_graph = not a.no_graph
    for _ in range(2):  # captures each trajectory's graphs (both slot parities)
        for t in trajs:
            t.step(evolve=True, dt=a.dt)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(seq_steps):
        for t in trajs:
            t.step(evolve=True, dt=a.dt)
    e1.record(stream)
    e1.synchronize()
    seq_ms = e0.elapsed_time(e1) / seq_steps

    n = len(trajs)
    value = n * a.steps * world / (ms / 1e3)
    taylor_ms = phase["taylor"] / n_prof
    taylor_alg = statistics.mean(sum(taylor_bytes_per_term(r, cs) * (r.final_m + 1) for r in rr) for rr in prof)
    achieved = taylor_alg / (taylor_ms / 1e3) / 1e9
    peak, peak_kind = read_peaks()
    states = statistics.mean(sum(r.n_states for r in rr) for rr in rounds)
    if rank == 0:
        cfg = {"workload": f"holstein_batched_{n}_seed{a.seed}_c64_dt{a.dt:g}_es{a.enlarge_steps}",
               "trajectories": n, "nchain": "uniform {16,24,32}", "g": "U[0.5,2]", "omega0": "U[0.5,1.5]",
               "maxstates": "log-uniform [2^14, 2^20]", "cutoff": 15, "J": 1.0, "dt": a.dt, "boundary": "periodic",
               "precision": a.precision, "states_per_step_all": int(states), "prep_steps": nprep,
               "streams": a.streams, "cuda_graph": not a.no_graph,
               "tuning": None if tuning is None else {k: tuning.get(k) for k in autotune_shapes()},
               "l2": "inputs larger than L2 (all trajectories' states and H tables > 126 MB)",
               "parallelism": f"replicas x{world}",
               "maxstates_drawn": [sp["maxstates"] for sp in specs], "nchain_drawn": [sp["nchain"] for sp in specs]}
        line = {
            "metric": "trajectory time-steps/s (batched trajectories)", "value": value, "unit": "trajectory-steps/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": a.precision,
            "data": "synthetic", "config": cfg,
            "roofline": {"bound": "hbm", "kernel": batch_taylor_kernel(batch), "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                         "algorithmic_bytes": taylor_alg, "launch_ms": taylor_ms},
            "phase_ms": {k: v / n_prof for k, v in phase.items()},
            "sequential_ms_per_step": seq_ms, "batched_speedup": seq_ms / (ms / a.steps),
            "repeated_steps_timed": repeated_timed,
            "clocks": clocks, "gpu_launches": int(round(launches_per_step * a.steps)), "cpu_baseline": None,
            "e2e": None,
        }
        print(json.dumps(line), flush=True)
    batch.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# --------------------------------------------------------------------------------------------
# learned workload: the proposal + complex64 against the plain complex128 run
# --------------------------------------------------------------------------------------------
def run_learned(a):
    import torch
    from paces_b200 import _native as nat
    from paces_b200.engine import Engine

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = f"cuda:{local}"
    steps, lf = a.total_steps, a.learn_from
    stream = torch.cuda.current_stream()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return out, e0.elapsed_time(e1)

    def observables(recs):
        L = a.nchain
        return {"n_exc": np.array([list(r.n_exc)[:L] for r in recs]), "n_pho": np.array([list(r.n_pho)[:L] for r in recs]),
                "energy": np.array([r.energy_re for r in recs]), "norm": np.array([r.norm for r in recs])}

    def plain(precision):
        eng = Engine(model_params(a, precision), device=dev)
        tr = start_trajectory(eng, a.nchain, a.maxstates, a.enlarge_steps, graph=not a.no_graph)
        recs = [tr.last] + [tr.step(evolve=True, dt=a.dt) for _ in range(lf)]
        window, ms = timed(lambda: [tr.step(evolve=True, dt=a.dt) for _ in range(steps - lf)])
        eng.close()
        return recs + window, ms

    # 1. the plain complex128 run (the oracle of the comparison) and the plain complex64 run
    ref, ms128 = plain("c128")
    r64, ms64 = plain("c64")
    # 2. training on the GPU, then 3. the learned run: plain complex64 for learn_from steps, then
    #    the proposal
    mlp, thr0, training = train_proposal(a, dev, lf)
    with ClockSampler(local) as clk:
        recs, ms, lt, eng = learned_run(a, dev, mlp, thr0, lf, steps)
    clocks = clk.summary()
    tr = lt.tr
    # stage split of proposal (non-judge) steps
    eng.set_profiling(True)
    use_graph, tr.use_graph = tr.use_graph, False
    stage = {k: 0.0 for k in nat.STAGES}
    nprof = 0
    l0 = eng.kernel_launches()
    for _ in range(12):
        judge = lt.k % lt.judge_every == 0
        lt.step(a.dt)
        if not judge:
            for k, v in eng.stage_times().items():
                stage[k] += v
            nprof += 1
    launches_per_step = (eng.kernel_launches() - l0) / 12
    tr.use_graph = use_graph
    eng.set_profiling(False)
    eng.close()
    ms = max_over_ranks(ms, dist)

    A, B, C = observables(ref), observables(recs), observables(r64)
    err = {k: float(np.max(np.abs(A[k] - B[k]))) for k in A}
    err64 = {k: float(np.max(np.abs(A[k] - C[k]))) for k in A}
    nwin = steps - lf
    value = nwin * world / (ms / 1e3)
    cs = 8
    taylor_ms = stage["taylor"] / max(nprof, 1)
    win = recs[lf + 1:]
    taylor_alg = statistics.mean(taylor_bytes_per_term(r, cs) * (r.final_m + 1) for r in win)
    peak, peak_kind = read_peaks()
    achieved = taylor_alg / (taylor_ms / 1e3) / 1e9 if taylor_ms > 0 else None
    if rank == 0:
        cfg = {"workload": f"holstein_periodic_n{a.nchain}_cutoff15_g{a.g:g}_maxstates{a.maxstates}_dt{a.dt:g}"
                           f"_es{a.enlarge_steps}_learned_c64",
               "nchain": a.nchain, "g": a.g, "omega0": 1.0, "J": 1.0, "dt": a.dt, "maxstates": a.maxstates,
               "enlarge_steps": a.enlarge_steps, "precision": "c64 (fp64 norms, stop test and sums)",
               "timed_steps": f"{lf + 1}..{steps} (proposal steps and every 10th a full-expansion judge step)",
               "training": training,
               "target_recall": a.recall, "threshold_start": thr0, "threshold_end": lt.threshold,
               "states_per_step_learned": statistics.mean(r.n_states for r in win),
               "states_per_step_plain": statistics.mean(r.n_states for r in ref[lf + 1:]),
               "enlarged_learned": statistics.mean(r.n_enlarged for r in win),
               "enlarged_plain": statistics.mean(r.n_enlarged for r in ref[lf + 1:]),
               "judges": [[j.step, j.recall, j.candidates, j.kept] for j in lt.judges],
               "l2": "inputs larger than L2", "parallelism": f"replicas x{world}", "cuda_graph": not a.no_graph}
        line = {
            "metric": "time-steps/s at 4M states: learned+FP32 vs plain FP64, observable err <=1e-5",
            "value": value, "unit": "time-steps/s", "n_gpus": world, "steps": nwin, "warmup": lf,
            "ms_per_step": ms / nwin, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64", "data": "synthetic", "config": cfg,
            "plain_c128": {"value": nwin / (ms128 / 1e3), "unit": "time-steps/s", "ms_per_step": ms128 / nwin},
            "plain_c64": {"value": nwin / (ms64 / 1e3), "unit": "time-steps/s", "ms_per_step": ms64 / nwin},
            "speedup_vs_plain_c128": ms128 / ms,
            "observable_error": {"learned_c64": err, "plain_c64": err64, "bound": 1e-5,
                                 "within_bound": all(v <= 1e-5 for v in err.values())},
            "roofline": {"bound": "hbm", "kernel": "taylor_kernel", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": None if achieved is None else achieved / peak,
                         "traffic": None, "launch_ms": taylor_ms},
            "stage_ms": {k: v / max(nprof, 1) for k, v in stage.items()},
            "clocks": clocks, "gpu_launches": int(round(launches_per_step * nwin)), "cpu_baseline": None, "e2e": None,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# --------------------------------------------------------------------------------------------
# long chain: N=64 rings with site-energy disorder, realizations batched in one launch
# --------------------------------------------------------------------------------------------
def batch_taylor_kernel(batch):
    """The Taylor kernel a batch step runs: one persistent launch for all, or the single-trajectory
    kernel per trajectory when every trajectory has room for PACES_BATCH_SINGLE_CAP states."""
    from paces_b200 import _native as nat
    if all(t.basis.cap >= nat.BATCH_SINGLE_CAP for t in batch.trajs):
        return f"taylor_kernel x{len(batch.trajs)}"
    return "taylor_batch_kernel"


def longchain_site_eps(seed, nchain, sigma):
    """Site energies of disorder realization `seed`: numpy.random.default_rng(seed).normal(0, sigma, N)."""
    return np.random.default_rng(seed).normal(0.0, sigma, nchain)


def run_longchain(a):
    import torch
    from paces_b200 import _native as nat
    from paces_b200.engine import Engine, ModelParams, TrajectoryBatch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = f"cuda:{local}"
    cs = 8 if a.precision == "c64" else 16

    def params(seed, precision):
        return ModelParams(nchain=a.nchain, max_ho_dims=[16] * a.nchain, J=1.0, g=a.g, hbar_omega=1.0,
                           periodic=True, site_eps=list(longchain_site_eps(seed, a.nchain, a.sigma)),
                           precision=precision)

    seeds = [a.seed + rank * a.realizations + r for r in range(a.realizations)]
    trajs = []
    for sd in seeds:
        eng = Engine(params(sd, a.precision), device=dev)
        trajs.append(start_trajectory(eng, a.nchain, a.maxstates, a.enlarge_steps, graph=not a.no_graph))
    batch = TrajectoryBatch(trajs, n_streams=min(4, a.realizations), graph=not a.no_graph)
    nprep = 0
    while True:
        recs = batch.step(evolve=True, dt=a.dt)
        nprep += 1
        log(a, f"prep {nprep}: " + " ".join(f"{r.n_select}/{r.n_states}" for r in recs))
        if all(r.n_select >= a.maxstates for r in recs) or nprep >= 80:
            break
    tuning = None
    if not a.no_tune:
        from paces_b200 import autotune
        tuning = autotune.tune_batch(batch, a.dt, steps=1)
    for _ in range(max(a.warmup, 0)):
        batch.step(evolve=True, dt=a.dt)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    rounds = []
    barrier()
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(a.steps):
            rounds.append(batch.step(evolve=True, dt=a.dt))
        ev1.record(stream)
        ev1.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist)
    clocks = clk.summary()
    barrier()
    n_prof = 3
    batch.set_profiling(True)
    batch.use_graph = False
    phase = {k: 0.0 for k in nat.BATCH_STAGES}
    prof = []
    l0 = batch.kernel_launches()
    for _ in range(n_prof):
        prof.append(batch.step(evolve=True, dt=a.dt))
        for k, v in batch.stage_times().items():
            phase[k] += v
    launches_per_step = (batch.kernel_launches() - l0) / n_prof
    batch.set_profiling(False)
    taylor_kernel = batch_taylor_kernel(batch)  # before the trajectories are released
    batch.close()
    for t in trajs:
        t.eng.close()
    del trajs, batch
    torch.cuda.empty_cache()

    compare = None
    if a.compare_steps > 0:
        obs = {}
        for prec in ("c128", a.precision):
            eng = Engine(params(seeds[0], prec), device=dev)
            tr = start_trajectory(eng, a.nchain, a.maxstates, a.enlarge_steps, graph=not a.no_graph)
            rr = [tr.last] + [tr.step(evolve=True, dt=a.dt) for _ in range(a.compare_steps)]
            L = a.nchain
            obs[prec] = {"n_exc": np.array([list(r.n_exc)[:L] for r in rr]),
                         "n_pho": np.array([list(r.n_pho)[:L] for r in rr]),
                         "energy": np.array([r.energy_re for r in rr]), "norm": np.array([r.norm for r in rr])}
            eng.close()
            torch.cuda.empty_cache()
        err = {k: float(np.max(np.abs(obs["c128"][k] - obs[a.precision][k]))) for k in obs["c128"]}
        compare = {"realization": seeds[0], "steps": a.compare_steps, "t_end": a.compare_steps * a.dt,
                   "max_abs_error_vs_c128": err}

    n = len(seeds)
    value = n * a.steps * world / (ms / 1e3)
    taylor_ms = phase["taylor"] / n_prof
    taylor_alg = statistics.mean(sum(taylor_bytes_per_term(r, cs) * (r.final_m + 1) for r in rr) for rr in prof)
    achieved = taylor_alg / (taylor_ms / 1e3) / 1e9
    peak, peak_kind = read_peaks()
    if rank == 0:
        cfg = {"workload": f"holstein_periodic_n{a.nchain}_cutoff15_g{a.g:g}_disorder{a.sigma:g}_maxstates{a.maxstates}"
                           f"_dt{a.dt:g}_x{n}",
               "nchain": a.nchain, "g": a.g, "omega0": 1.0, "J": 1.0, "dt": a.dt, "maxstates": a.maxstates,
               "site_energy_sigma": a.sigma, "realization_seeds": seeds, "precision": a.precision,
               "key_words": 4 if a.nchain == 64 else None, "enlarge_steps": a.enlarge_steps,
               "states_per_step": [int(statistics.mean(rr[i].n_states for rr in rounds)) for i in range(n)],
               "prep_steps": nprep, "cuda_graph": not a.no_graph,
               "tuning": None if tuning is None else {k: tuning.get(k) for k in autotune_shapes()},
               "l2": "inputs larger than L2", "parallelism": f"replicas x{world}"}
        line = {
            "metric": "trajectory time-steps/s (N=64 disorder realizations batched)", "value": value,
            "unit": "trajectory-steps/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": a.precision, "data": "synthetic", "config": cfg,
            "roofline": {"bound": "hbm", "kernel": taylor_kernel, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                         "launch_ms": taylor_ms},
            "phase_ms": {k: v / n_prof for k, v in phase.items()}, "compare": compare,
            "clocks": clocks, "gpu_launches": int(round(launches_per_step * a.steps)), "cpu_baseline": None,
            "e2e": None,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.workload == "batched":
        run_batched(a)
    elif a.workload == "learned":
        a.precision = "c64"
        run_learned(a)
    elif a.workload == "longchain":
        # the long-chain configuration unless overridden: N=64, g=2, maxstates 2^24, dt 0.025
        given = {x.split("=")[0] for x in sys.argv[1:] if x.startswith("--")}
        for flag, attr, val in (("--nchain", "nchain", 64), ("--g", "g", 2.0), ("--maxstates", "maxstates", 1 << 24),
                                ("--dt", "dt", 0.025), ("--steps", "steps", 10)):
            if flag not in given:
                setattr(a, attr, val)
        run_longchain(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
