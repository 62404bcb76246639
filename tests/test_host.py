"""CPU tests of the host side: the C ABI exports, the key layout helpers, the drop-in
module paths, and the multi-process (replica) timing reduction under gloo."""

import os
import re
import socket

import numpy as np
import pytest
import torch

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")


def _declared_symbols():
    with open(os.path.join(REPO, "include", "paces_b200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(paces_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import ctypes
    from paces_b200 import _native
    lib = ctypes.CDLL(_native.LIB_PATH)
    declared = _declared_symbols()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(lib, name), name
    # and the ctypes binding covers the whole ABI
    assert set(declared) == set(_native.exported_symbols())
    _native.load()


def test_workspace_query_without_a_device():
    from paces_b200 import _native
    lib = _native.load()
    assert lib.paces_version() == 10300
    assert lib.paces_create(None, None) == 5  # PACES_ERR_BADARG, no device touched


@pytest.mark.parametrize("name", ["n16c16", "n32c16", "n25c128", "n6c8"])
def test_layout_helpers_match_reference_packing(name):
    from paces_b200 import layout
    f = np.load(os.path.join(GOLDEN, f"layout_{name}.npz"))
    bw = f["bitwidths"]
    rows = layout.pack_rows(f["raw"], bw)
    assert np.array_equal(rows, f["keys"])
    assert np.array_equal(layout.unpack_rows(rows, bw), f["raw"])
    assert np.array_equal(layout.sort_unique_rows(f["unique_in"]), f["unique_out"])
    tab = layout.field_table(bw)
    r64 = layout.rows_i64(rows)
    pos = layout.get_field_t(r64, tab, 0)
    assert np.array_equal(layout.get_field_t(r64, tab, pos + 1).numpy(), f["get_occ"])
    up = torch.from_numpy(f["can_up"])
    got = layout.rows_u32(layout.add_field_t(r64[up], tab, pos[up] + 1, 1)).numpy()
    assert np.array_equal(got, f["keys_up"])


def test_drop_in_module_paths():
    import paces
    from paces.config import devices, INIT_VERBOSITY_LEVEL, SEARCHSORTED_TIMING_LEVEL
    from paces.core.hamiltonian import HamiltonianFramework, MelTriple
    from paces.core.observables import ObservablesFramework
    from paces.core.time_evolution import CoeffSaveParams, ExpmParams, TimeEvoParams, TimeEvolutionFramework
    from paces.models import holstein
    import paces_b200
    assert paces.config.devices is paces_b200.config.devices is devices
    assert issubclass(holstein.Hamiltonian, HamiltonianFramework)
    assert issubclass(holstein.Observables, ObservablesFramework)
    assert issubclass(holstein.TimeEvolution, TimeEvolutionFramework)
    assert INIT_VERBOSITY_LEVEL == 0 and SEARCHSORTED_TIMING_LEVEL == 7
    assert ExpmParams().m_star == 100 and TimeEvoParams(1, 1).shuffle_seed == 0
    cso = CoeffSaveParams(save_every=3, save_first=True, save_last=True, max_i=7)
    assert [cso.save_necessary(i) for i in range(8)] == [True, False, False, True, False, False, True, True]
    assert holstein.Observables.calculate_n_exc.fname == "n_exc"
    assert MelTriple._fields == ("inds", "vals", "mask")


def test_framework_needs_configured_devices():
    from paces_b200.config import DeviceConfig
    d = DeviceConfig()
    with pytest.raises(NotImplementedError):
        d.configure(whoami_device_id=0, vector_device_id=1)
    with pytest.raises(NotImplementedError):
        d.configure(unified_memory_bytes=1 << 30)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _replica_worker(rank, world, port, out):
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    ms = bench.max_over_ranks(10.0 + rank, dist, device="cpu")
    out[rank] = ms
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_takes_the_max_over_ranks():
    import torch.multiprocessing as mp
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    mp.start_processes(_replica_worker, args=(2, port, out), nprocs=2, start_method="spawn")
    assert dict(out) == {0: 11.0, 1: 11.0}


def test_bench_names_the_batch_taylor_kernel():
    """bench.py's roofline label follows paces_batch_step's choice: the single-trajectory
    kernel per trajectory when every trajectory has room for PACES_BATCH_SINGLE_CAP states."""
    import types
    import bench
    from paces_b200 import _native as nat
    def batch(*caps):
        return types.SimpleNamespace(trajs=[types.SimpleNamespace(basis=types.SimpleNamespace(cap=c)) for c in caps])
    big = nat.BATCH_SINGLE_CAP
    assert bench.batch_taylor_kernel(batch(big, big, 2 * big, big)) == "taylor_kernel x4"
    assert bench.batch_taylor_kernel(batch(big, big - 1)) == "taylor_batch_kernel"
    assert bench.batch_taylor_kernel(batch(1 << 14)) == "taylor_batch_kernel"
    header = open(os.path.join(os.path.dirname(__file__), "..", "include", "paces_b200.h")).read()
    m = re.search(r"#define PACES_BATCH_SINGLE_CAP \(1 << (\d+)\)", header)
    assert m and (1 << int(m.group(1))) == big


def test_ctypes_structs_match_the_header(tmp_path):
    """Every ctypes mirror of a struct in include/paces_b200.h has the C compiler's size and
    field offsets (gcc on the header alone; no device)."""
    import ctypes
    import shutil
    import subprocess
    from paces_b200 import _native as nat
    if not shutil.which("gcc"):
        pytest.skip("gcc not found")
    mirrors = {"paces_model_desc": nat.ModelDesc, "paces_basis": nat.Basis, "paces_hmat": nat.HMat,
               "paces_step_params": nat.StepParams, "paces_step_record": nat.StepRecord,
               "paces_expm_info": nat.ExpmInfo, "paces_tuning": nat.Tuning, "paces_batch_item": nat.BatchItem}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "paces_b200.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'    printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, *_ in py._fields_:
            lines.append(f'    printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["    return 0;", "}"]
    src, exe = tmp_path / "layout.c", tmp_path / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in filter(None, out):
        cname, what, v = ln.split()
        got[(cname, what)] = int(v)
    for cname, py in mirrors.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, *_ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_batch_warm_up_runs_until_no_step_repeats():
    """bench.warm_up_batch: trajectories short of room grow first (and the batch drops its
    graphs); the warm-up takes at least `warmup` steps and goes on until that many in a row
    ran without a capacity repeat, within the extra steps allowed."""
    import sys
    sys.path.insert(0, REPO)
    import bench

    class Rec:
        def __init__(self, n):
            self.n_states = n

    class Eng:
        def __init__(self, cap):
            self.cap = cap

    class Traj:
        def __init__(self, cap, n):
            self.eng, self.last, self.grown = Eng(cap), Rec(n), []

        def _regrow(self, factor):
            self.grown.append(factor)
            self.eng.cap = int(self.eng.cap * factor)

    class Batch:
        def __init__(self, repeat_at):
            self.repeats, self.n, self.repeat_at, self._graphs = 0, 0, set(repeat_at), {"g": 1}

        def step(self, evolve, dt):
            self.n += 1
            if self.n in self.repeat_at:
                self.repeats += 1

    trajs = [Traj(1000, 900), Traj(10000, 100)]
    b = Batch(repeat_at=[2, 5])
    assert bench.warm_up_batch(b, trajs, 3, 0.05) == 8  # repeats at 2 and 5: quiet from 6 to 8
    assert trajs[0].eng.cap >= 1.6 * 900 and trajs[0].grown and not trajs[1].grown
    assert b._graphs == {}
    b = Batch(repeat_at=range(1, 100))
    assert bench.warm_up_batch(b, [Traj(10000, 10)], 3, 0.05, extra=5) == 8  # bounded
    b = Batch(repeat_at=[])
    assert bench.warm_up_batch(b, [Traj(10000, 10)], 3, 0.05) == 3
    assert b._graphs == {"g": 1}
