"""paces_remap_noalloc: the remap for callers that cannot allocate device memory.

Some hosts own the whole device through their own memory pool, and some loops must not
call cudaMalloc (it can synchronise the device); this entry point takes no workspace and
uses a fixed static scratch array inside the library instead.  The test calls it through
the C ABI twice in a row (the static scratch keeps the first call's contents) and checks
both results against the workspace entry point, paces_remap; it also checks that bases
too large for the static scratch are refused before anything runs.

This file is collected last on purpose: it must pass both alone in a fresh process and
after every other test.
"""

import ctypes
import glob
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _noalloc(eng, old, old_psi, new, new_psi):
    from paces_b200 import _native as nat
    rc = eng.lib.paces_remap_noalloc(eng.ctx, ctypes.byref(old.c()), ctypes.c_void_p(old_psi.data_ptr()),
                                     ctypes.byref(new.c()), ctypes.c_void_p(new_psi.data_ptr()),
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    nat.check(rc, eng.ctx, "paces_remap_noalloc")
    eng.raise_status("paces_remap_noalloc")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "stages_*.npz")))[:3],
                         ids=os.path.basename)
def test_noalloc_remap_matches_workspace_remap(path):
    from tests import gpu_helpers
    f = np.load(path)
    c = f["config"]
    eng = gpu_helpers.engine_for(int(c[0]), int(c[1]), float(c[2]), cap=1 << 14)
    for s in range(1, int(f["nsteps_recorded"])):
        k = f"s{s}_"
        old = eng.basis_from_ref(f[k + "trunc_whoami"])
        new = eng.basis_from_ref(f[k + "new_inds"])
        old_psi = torch.zeros(old.cap, dtype=torch.complex128, device=eng.device)
        n_old = old.count()
        old_psi[:n_old] = torch.as_tensor(f[k + "trunc_vector"]).to(eng.device)
        expect = eng.remap(old, old_psi, new)[: new.count()].cpu().numpy()
        for _ in range(2):  # two calls in a row on the same static scratch
            got = torch.full((new.cap,), complex(7.0, 7.0), dtype=torch.complex128, device=eng.device)
            _noalloc(eng, old, old_psi, new, got)
            np.testing.assert_allclose(got[: new.count()].cpu().numpy(), expect, rtol=0, atol=0)
        assert np.array_equal(expect, f[k + "remap_vector"])


def test_noalloc_remap_refuses_oversized_bases():
    from paces_b200 import _native as nat
    from tests import gpu_helpers
    eng = gpu_helpers.engine_for(6, 8, 1.0, cap=1 << 10)
    small = eng.new_basis(16)
    huge = nat.Basis(small.keys.data_ptr(), small.blk.data_ptr(), 1 << 40)  # capacity only, never touched
    psi = torch.zeros(16, dtype=torch.complex128, device=eng.device)
    rc = eng.lib.paces_remap_noalloc(eng.ctx, ctypes.byref(huge), ctypes.c_void_p(psi.data_ptr()),
                                     ctypes.byref(small.c()), ctypes.c_void_p(psi.data_ptr()),
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == nat.ERR_CAPACITY
    assert b"static scratch" in eng.lib.paces_last_error(eng.ctx)
