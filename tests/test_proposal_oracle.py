"""CPU checks of the learned-proposal oracle (features, labels, network, gradients, Adam),
which the GPU tests then use as the reference for the device kernels."""

import numpy as np
import pytest

from oracle import paces_oracle as po
from oracle import proposal_oracle as pr


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e38, 1e-30], dtype=np.float32)
    got = pr.bf16(x)
    assert got[0] == 1.0
    assert got[1] == 1.0                      # halfway, even mantissa kept
    assert got[2] == np.float32(1.0 + 2 ** -7)  # above halfway rounds up
    assert got[3] == -2.5
    assert np.isfinite(got[4]) and abs(got[5] - 1e-30) / 1e-30 < 2 ** -8


@pytest.mark.parametrize("periodic", [False, True])
def test_events_and_features_of_a_hand_state(periodic):
    m = po.Model(5, [4] * 5, periodic=periodic)
    raw = np.array([[4, 1, 0, 2, 3, 0],    # exciton on the last site
                    [0, 0, 0, 0, 0, 0]], dtype=np.uint32)
    rows = po.compress(m, raw)
    w = np.array([0.5, 1e-40], dtype=np.float32)
    j, i, ok, cpos, cocc = pr.events(m, rows)
    nx = 2
    # run 1 (hop right) from site 4: only on the ring
    assert ok[0] == periodic and (not periodic or cpos[0] == 0)
    # run 2 (hop left) from site 0: only on the ring
    assert ok[nx + 1] == periodic
    # run 3 (create at site 4, n=0 -> 1), run 4 (annihilate at site 4: n=0, floor)
    assert ok[2 * nx] and cocc[2 * nx, 4] == 1 and not ok[3 * nx]
    f, ok2 = pr.features(m, rows, w)
    assert np.array_equal(ok, ok2)
    e = 2 * nx  # create at the exciton site of state 0: image (4; 1,0,2,3,1)
    occ = [1, 0, 2, 3, 1]
    win = [occ[(4 + d) % 5] / 3 if (periodic or 0 <= 4 + d < 5) else 0.0 for d in range(-4, 5)]
    assert np.allclose(f[e, :9], pr.bf16(np.array(win, dtype=np.float32)))
    assert f[e, 9] == pr.bf16(np.float32(7 / 16))
    assert abs(f[e, 10] - np.log(0.5) / 16 + np.log(1e-30) / 16) < 2 ** -6
    assert list(f[e, 11:14]) == [0, 1, 0] and f[e, 15] == 0
    # creation from n=0 to n'=1 at the exciton site: element g sqrt(1) = g = 1
    assert f[e, 14] == 0
    # the vanishing amplitude of state 1 is clamped at 1e-30 before the log
    assert ok[2 * nx + 1] and f[2 * nx + 1, 10] == 0
    # relative to a cut
    f2, _ = pr.features(m, rows, w, cut=0.25)
    assert abs(f2[e, 10] - np.log(2.0) / 16) < 2 ** -8
    assert np.all(f[~ok] == 0)


def test_labels_against_sets():
    m = po.Model(4, [4] * 4, periodic=True)
    x = po.unique_rows(po.compress(m, np.array([[0, 0, 0, 0, 0], [1, 0, 0, 0, 0], [0, 1, 0, 0, 0]], dtype=np.uint32)))
    y = po.unique_rows(po.compress(m, np.array([[0, 0, 0, 0, 0], [0, 2, 0, 0, 0], [3, 0, 0, 0, 0]], dtype=np.uint32)))
    lab = pr.labels(m, x, y)
    j, i, ok, cpos, cocc = pr.events(m, x)
    for e in range(len(lab)):
        if not ok[e]:
            assert lab[e] == 254
            continue
        img = po.compress(m, np.concatenate([[cpos[e]], cocc[e]])[None, :].astype(np.uint32))[0]
        in_x = any(np.array_equal(img, r) for r in x)
        in_y = any(np.array_equal(img, r) for r in y)
        assert lab[e] == (255 if in_x else int(in_y))
    assert (lab == 1).any() and (lab == 0).any() and (lab == 255).any()


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    master = pr.init_master(1).astype(np.float64)
    x = rng.normal(0, 1, (64, pr.N_IN))
    y = (rng.random(64) < 0.3).astype(np.float64)
    sw = rng.uniform(0.5, 2.0, 64)
    loss, g = pr.loss_and_grads(master, x, y, sw, 1 / 64, round_bf16=False)
    f = lambda mm: pr.loss_and_grads(mm, x, y, sw, 1 / 64, round_bf16=False)[0]
    h = 1e-3
    idx = list(rng.choice(pr.N_MASTER, 40, replace=False)) + [pr.OFF_B3, pr.OFF_W3, pr.OFF_B1, pr.OFF_W1]
    for q in idx:
        mp, mm = master.copy(), master.copy()
        mp[q] += h
        mm[q] -= h
        fd = (f(mp.astype(np.float32)) - f(mm.astype(np.float32))) / (2 * h)
        assert abs(fd - g[q]) <= 2e-2 * max(1e-3, abs(g[q])) + 2e-4, (q, fd, g[q])


def test_adam_first_step_moves_by_lr():
    master = pr.init_master(0)
    g = np.linspace(-1, 1, pr.N_MASTER).astype(np.float32)
    g[g == 0] = 0.5
    new, m1, m2 = pr.adam(master, np.zeros_like(master), np.zeros_like(master), g, 1, 1e-2)
    assert np.allclose(new - master, -1e-2 * np.sign(g), rtol=1e-3, atol=1e-6)
