"""Launch shapes (merge strides, Taylor grid) change speed only: every shape the tuner may
pick gives bit-identical trajectories, and the tuner returns one of them."""

import numpy as np
import pytest

from tests import gpu_helpers

pytestmark = pytest.mark.gpu


def _run(precision, stride=None, bps=None, variant=None, steps=8, astride=None):
    from paces_b200 import autotune
    eng = gpu_helpers.engine_for(16, 16, 1.0, cap=1 << 14, precision=precision, periodic=True)
    if stride is not None or bps is not None or variant is not None:
        autotune.set_tuning(eng, stride, bps, variant, assemble_stride=astride)
    tr, _ = gpu_helpers.grown_trajectory(eng, 16, 20000)
    recs = [tr.step(evolve=True, dt=0.05) for _ in range(steps)]
    n = tr.basis.count()
    out = (recs, tr.basis.keys[:n].cpu().numpy(), tr.vector.cpu().numpy())
    eng.close()
    return out


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_results_do_not_depend_on_launch_shapes(precision):
    ref = _run(precision, variant=0)
    for stride, bps, variant, astride in ((64, 1, 0, None), (96, 2, 1, None), (160, 0, 1, None), (240, 1, 1, None),
                                          (128, 0, 0, None), (128, 0, 1, 224), (224, 1, 0, 80)):
        got = _run(precision, stride, bps, variant, astride=astride)
        for a, b in zip(ref[0], got[0]):
            assert (a.n_states, a.final_m, a.converged) == (b.n_states, b.final_m, b.converged)
            assert list(a.n_exc) == list(b.n_exc) and list(a.n_pho) == list(b.n_pho)
            assert a.energy_re == b.energy_re
        assert np.array_equal(ref[1], got[1]) and np.array_equal(ref[2], got[2])


def test_out_of_range_shapes_are_rejected():
    from paces_b200 import _native as nat
    from paces_b200 import autotune
    eng = gpu_helpers.engine_for(8, 16, 1.0, cap=1 << 10)
    t = autotune.get_tuning(eng)
    assert t.merge_stride == 160 and t.merge_stride_max == 240 and t.merge_stride_min == 64
    assert t.assemble_stride == 192
    for bad in (48, 250, 72):
        with pytest.raises(nat.PacesError):
            autotune.set_tuning(eng, merge_stride=bad)
        with pytest.raises(nat.PacesError):
            autotune.set_tuning(eng, assemble_stride=bad)
    autotune.set_tuning(eng, merge_stride=128, assemble_stride=208)
    t = autotune.get_tuning(eng)
    assert (t.merge_stride, t.assemble_stride) == (128, 208)
    with pytest.raises(nat.PacesError):
        autotune.set_tuning(eng, taylor_blocks_per_sm=t.taylor_blocks_per_sm_max + 1)
    with pytest.raises(nat.PacesError):
        autotune.set_tuning(eng, taylor_variant=2)
    eng.close()


def test_tuner_picks_an_allowed_shape(tmp_path, monkeypatch):
    from paces_b200 import autotune
    monkeypatch.setattr(autotune, "CACHE_PATH", str(tmp_path / "tuning.json"))
    monkeypatch.setattr(autotune, "_memory", {})
    eng = gpu_helpers.engine_for(16, 16, 1.0, cap=1 << 14, periodic=True)
    tr, _ = gpu_helpers.grown_trajectory(eng, 16, 20000)
    choice = autotune.tune(tr, 0.05, steps=1)
    t = autotune.get_tuning(eng)
    assert not choice["cached"]
    assert t.merge_stride == choice["merge_stride"] and t.taylor_blocks_per_sm == choice["taylor_blocks_per_sm"]
    assert t.assemble_stride == choice["assemble_stride"]
    assert set(choice["timings_ms"]["merge_stride"]) == set(autotune.stride_candidates(t))
    assert set(choice["timings_ms"]["assemble_stride"]) == set(autotune.stride_candidates(t))
    assert t.taylor_variant == choice["taylor_variant"] in (0, 1)
    again = autotune.tune(tr, 0.05, steps=1)
    assert again["cached"] and again["merge_stride"] == choice["merge_stride"]
    eng.close()


def test_graphs_follow_the_launch_shapes():
    """A change of launch shapes (set_tuning, or a cached choice the tuner applies) makes the
    next graph step capture anew, for a trajectory and for a batch: no replay runs under the
    shapes it was captured with after they changed."""
    from paces_b200 import autotune
    from paces_b200.engine import TrajectoryBatch
    trs = []
    for _ in range(3):
        eng = gpu_helpers.engine_for(16, 16, 1.0, cap=1 << 14, precision="c64", periodic=True)
        tr, _ = gpu_helpers.grown_trajectory(eng, 16, 20000, graph=True)
        trs.append(tr)
    tr = trs[0]
    for _ in range(2):
        tr.step(evolve=True, dt=0.05)
    before = set(tr._graphs)
    assert len(before) == 2
    epoch = tr.eng.tuning_epoch
    autotune.set_tuning(tr.eng, 240, assemble_stride=240)
    assert tr.eng.tuning_epoch == epoch + 1
    tr.step(evolve=True, dt=0.05)
    new = set(tr._graphs) - before
    assert len(new) == 1 and all(k[2] == tr.eng.tuning_epoch for k in new)

    batch = TrajectoryBatch(trs[1:], n_streams=2, graph=True)
    for _ in range(2):
        batch.step(evolve=True, dt=0.05)
    before = set(batch._graphs)
    assert len(before) == 2
    autotune.set_tuning(trs[2].eng, 240, assemble_stride=240)
    batch.step(evolve=True, dt=0.05)
    new = set(batch._graphs) - before
    assert len(new) == 1
    assert all(k[2] == tuple(t.eng.tuning_epoch for t in trs[1:]) for k in new)
    batch.close()
