"""Site observables for every key layout the site pass tells apart: 4-bit fields (masked in
place at constant positions), wider uniform fields (5 and 8 bits, the width read at run
time), narrower fields (2 and 3 bits, the general broadcast path), one and two key words.
Compared with fp64 sums over the basis rows on the host (calculate_n_exc / calculate_n_pho,
paces/models/holstein.py:311-322); only the order of the additions differs."""

import numpy as np
import pytest

import gpu_helpers

pytestmark = pytest.mark.gpu

# (nchain, max_ho_dim): key bits per state = nchain * ceil(log2(dim))
CASES = [(6, 4), (6, 8), (6, 16), (20, 16), (6, 32), (14, 32), (6, 256), (10, 256)]


@pytest.mark.parametrize("precision", ["c128", "c64"])
@pytest.mark.parametrize("nchain,dim", CASES)
def test_site_observables_by_field_width(nchain, dim, precision):
    from paces_b200 import layout

    eng = gpu_helpers.engine_for(nchain, dim, 1.3, cap=1 << 15, precision=precision, periodic=True)
    tr, _ = gpu_helpers.grown_trajectory(eng, nchain, 3000, initpos=nchain // 2, dim=dim)
    for _ in range(6):
        tr.step(evolve=True, dt=0.05)
    b, psi = tr.basis, tr.vector
    S = b.count()
    assert S > 1000
    got = eng.observables(b, tr.h, psi)

    rows = gpu_helpers.ref_rows(eng, b)
    occ = layout.unpack_rows(rows, layout.bitwidths_for([nchain] + [dim] * nchain)).astype(np.float64)
    z = psi[:S].cpu().numpy().astype(np.complex128)
    w = z.real * z.real + z.imag * z.imag
    pos = occ[:, 0].astype(np.int64)
    n_exc = np.bincount(pos, weights=w, minlength=nchain)[:nchain]
    n_pho = w @ occ[:, 1:]
    assert occ[:, 1:].max() >= 2  # the trajectory has left the one-phonon shell

    np.testing.assert_allclose(got["norm"], np.sqrt(w.sum()), rtol=1e-12)  # the 2-norm
    np.testing.assert_allclose(got["n_exc"], n_exc, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(got["n_pho"], n_pho, rtol=1e-12, atol=1e-15)
