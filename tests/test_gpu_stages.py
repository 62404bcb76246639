"""GPU parity: every stage of libpaces_b200 against the reference's golden fixtures and the
CPU oracle, bit-exact for keys, order, dedup and lookup indices; amplitudes and observables
to 1e-12 relative in complex128."""

import glob
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
STAGES = sorted(glob.glob(os.path.join(GOLDEN, "stages_*.npz")))
LAYOUTS = sorted(glob.glob(os.path.join(GOLDEN, "layout_*.npz")))


def _cfg(f):
    c = f["config"]
    return int(c[0]), int(c[1]), float(c[2]), int(c[3]), int(c[4])


@pytest.fixture(scope="module")
def helpers():
    from tests import gpu_helpers
    return gpu_helpers


@pytest.mark.parametrize("path", LAYOUTS, ids=os.path.basename)
def test_layout_roundtrip_and_lookup(path, helpers):
    f = np.load(path)
    raw = f["raw"]
    nchain = raw.shape[1] - 1
    dim = 2 ** int(f["bitwidths"][1])
    eng = helpers.engine_for(nchain, dim, 1.0, cap=1 << 14)
    uniq = f["unique_out"]
    b = eng.basis_from_ref(uniq)
    assert b.count() == len(uniq)
    assert np.array_equal(helpers.ref_rows(eng, b), uniq)
    keys, pos, n = eng.query_from_ref(f["search_any_q"])
    idx = eng.lookup(b, keys, pos, n).cpu().numpy()
    hit = f["search_any_hit"]
    assert np.array_equal(idx >= 0, hit)
    assert np.array_equal(idx[hit], f["search_any_idx"][hit].astype(np.int64))
    keys, pos, n = eng.query_from_ref(f["search_hit_q"])
    idx = eng.lookup(b, keys, pos, n, must_exist=True).cpu().numpy()
    assert np.array_equal(idx, f["search_hit_idx"].astype(np.int64))


@pytest.mark.parametrize("path", STAGES, ids=os.path.basename)
def test_stages_bit_exact(path, helpers):
    f = np.load(path)
    nchain, dim, g, maxstates, es = _cfg(f)
    eng = helpers.engine_for(nchain, dim, g, cap=1 << 15)
    for s in range(int(f["nsteps_recorded"])):
        k = f"s{s}_"
        # truncation
        old = eng.basis_from_ref(f[k + "trunc_whoami"])
        vec = torch.as_tensor(f[k + "trunc_vector"]).to(eng.device)
        sel = eng.truncate(old, vec, maxstates)
        assert np.array_equal(helpers.ref_rows(eng, sel), f[k + "select"]), f"truncation, step {s}"
        # enlargement
        cur = eng.basis_from_ref(f[k + "select"])
        for _ in range(es):
            cur = eng.expand(cur)
        if es >= 1:
            assert np.array_equal(helpers.ref_rows(eng, cur), f[k + "enlarged"]), f"expand, step {s}"
        # new basis + H
        new, h, ceil = eng.assemble(cur)
        assert np.array_equal(helpers.ref_rows(eng, new), f[k + "new_inds"]), f"assemble keys, step {s}"
        assert ceil == int(f[k + "ceiling_hits"][0])
        diag, mats, _ = helpers.csr_from_table(eng, new, h, 1.0, g)
        assert np.array_equal(diag, f[k + "diag"])
        for term, m in mats.items():
            assert np.array_equal(m.indptr, f[k + f"csr_{term}_indptr"]), f"{term} indptr, step {s}"
            assert np.array_equal(m.indices, f[k + f"csr_{term}_indices"]), f"{term} indices, step {s}"
            assert np.array_equal(m.data, f[k + f"csr_{term}_data"]), f"{term} data, step {s}"
        # remap
        v = eng.remap(old, vec, new)[: new.count()].cpu().numpy()
        assert np.array_equal(v, f[k + "remap_vector"]), f"remap, step {s}"
        # Taylor
        if k + "taylor_in" in f:
            tin = torch.zeros(new.cap, dtype=torch.complex128, device=eng.device)
            tin[: new.count()] = torch.as_tensor(f[k + "taylor_in"]).to(eng.device)
            out, dbg = eng.taylor(new, h, tin, 0.05)
            np.testing.assert_allclose(out[: new.count()].cpu().numpy(), f[k + "taylor_out"], rtol=0, atol=1e-14)
            assert dbg[0] == bool(f[k + "taylor_dbg"][0])
            assert dbg[1] == int(f[k + "taylor_dbg"][1])
        # observables
        fv = torch.zeros(new.cap, dtype=torch.complex128, device=eng.device)
        fv[: new.count()] = torch.as_tensor(f[k + "final_vector"]).to(eng.device)
        obs = eng.observables(new, h, fv)
        np.testing.assert_allclose(obs["n_exc"], f["n_exc"][s, 2:], rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(obs["n_pho"], f["n_pho"][s, 2:], rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(obs["energy"].real, f["energy"][s, 2], rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(obs["norm"], f["n_exc"][s, 1], rtol=1e-13)
