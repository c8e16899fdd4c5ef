"""Launch shapes and the autotuner through the C ABI: every integrate z-chunk and raycast
tile shape computes bit-identical volumes, maps and poses (also on volume sizes that are
not multiples of the chunk); autotuning leaves the session's state untouched; a batch
tuned over a mix still steps each session exactly as it steps alone."""
import itertools

import numpy as np
import pytest

from helpers import small_workload
from oglfusionkinectv2_b200 import GFusion, GFusionBatch, _lib as L

pytestmark = pytest.mark.gpu

SHAPES = list(itertools.product((8, 16, 32), (1, 2, 4, 8)))  # rows 1: the persistent sweep


def _state(g):
    return g.getPose(), g.getVolumeRaw(), g.getVerts(), g.getNorms()


def _assert_same(a, b):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("storage", [L.KF_STORAGE_F32F32, L.KF_STORAGE_F16U16, L.KF_STORAGE_RG16I])
def test_every_shape_is_bit_identical(storage):
    w = small_workload(4, size=100, storage=storage)  # 100 = 3 * 32 + 4: ragged last chunk
    frames = [w.frame(k) for k in range(w.n_frames)]
    ref = None
    for zc, rows in SHAPES:
        g = GFusion(w.config, w.intrinsics)
        g.setLaunchShape(zc, rows)
        assert g.launchShape() == (zc, rows)
        g.Reset(w.poses[0])
        for f in frames:
            g.frameStep(f)
        st = _state(g)
        if ref is None:
            ref = st
            assert (st[2][..., 3] > 0).mean() > 0.2
        else:
            _assert_same(st, ref)


def test_autotune_leaves_state_untouched_and_is_remembered():
    w = small_workload(8, size=128, storage=L.KF_STORAGE_F16U16)
    a, b = GFusion(w.config, w.intrinsics), GFusion(w.config, w.intrinsics)
    for s in (a, b):
        s.Reset(w.poses[0])
    for k in range(4):
        a.frameStep(w.frame(k))
        b.frameStep(w.frame(k))
    before = _state(a)
    shape, times = a.autotune(repeats=3)
    assert shape[0] in (8, 16, 32) and shape[1] in (1, 2, 4, 8)
    assert a.launchShape() == shape
    assert len(times) == 7 and all(0 < t < 100 for t in times.values())
    _assert_same(_state(a), before)
    for k in range(4, 8):
        assert a.frameStep(w.frame(k)) == b.frameStep(w.frame(k))
    _assert_same(_state(a), _state(b))
    # a new session of the same volume size, storage and image size starts with the tuned shape
    c = GFusion(w.config, w.intrinsics)
    assert c.launchShape() == shape


def test_invalid_shapes_are_rejected():
    w = small_workload(1, size=32)
    g = GFusion(w.config, w.intrinsics)
    for zc, rows in ((12, 4), (16, 3), (0, 0), (64, 4)):
        with pytest.raises(L.KfError) as e:
            g.setLaunchShape(zc, rows)
        assert e.value.status == L.KF_ERR_INVALID_ARGUMENT
    with pytest.raises(L.KfError):
        g.autotune(repeats=0)
    # the persistent raycast sweep is a session shape only
    batch = GFusionBatch(2)
    with pytest.raises(L.KfError) as e:
        batch.setLaunchShape(16, 1)
    assert e.value.status == L.KF_ERR_INVALID_ARGUMENT


def test_batch_autotune_keeps_results_exact():
    # batched == alone bit for bit holds for the split-BF16 J^T J form (exact fixed-point sums)
    sizes = (64, 96, 100, 128)
    ws = [small_workload(5, size=n, storage=L.KF_STORAGE_F16U16, jtj=L.KF_JTJ_SPLIT_BF16,
                         quirks=L.KF_QUIRKS_TRACKING, seed=0xC0FFEE + 1 + 10 * k) for k, n in enumerate(sizes)]
    batched = [GFusion(w.config, w.intrinsics) for w in ws]
    alone = [GFusion(w.config, w.intrinsics) for w in ws]
    for s, w in zip(batched + alone, ws + ws):
        s.setLaunchShape(16, 4)
        s.Reset(w.poses[0])
    batch = GFusionBatch(len(ws))
    batch.frameStep(batched, [w.frame(0) for w in ws])
    for s, w in zip(alone, ws):
        s.frameStep(w.frame(0))
    before = [_state(s) for s in batched]
    shape, times = batch.autotune(batched, repeats=2)
    assert batch.launchShape() == shape and len(times) == 6
    for s, st in zip(batched, before):
        _assert_same(_state(s), st)
    for k in range(1, 5):
        batch.frameStep(batched, [w.frame(k) for w in ws])
        for s, w in zip(alone, ws):
            s.frameStep(w.frame(k))
    for s, t in zip(batched, alone):
        _assert_same(_state(s), _state(t))
    # every fixed batch shape agrees as well
    for zc, rows in ((8, 2), (32, 8)):
        batch.setLaunchShape(zc, rows)
        batch.frameStep(batched, [w.frame(4) for w in ws])
        for s, w in zip(alone, ws):
            s.frameStep(w.frame(4))
        for s, t in zip(batched, alone):
            _assert_same(_state(s), _state(t))

