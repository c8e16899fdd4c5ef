"""Batched frame steps (kf_batch_*): several sessions of different volume sizes and scenes
stepped together give the same results as each stepped alone.

With the split-BF16 J^T J form the ICP sums are exact fixed-point integers, so poses,
raycast maps and volumes are bit-identical whatever the batch; membership may change from
step to step (continuous batching)."""
import numpy as np
import pytest

from helpers import small_workload
from oglfusionkinectv2_b200 import GFusion, GFusionBatch, _lib as L

pytestmark = pytest.mark.gpu

SIZES = [64, 96, 128, 80]
SEEDS = [0xC0FFEE + 1, 0xC0FFEE + 21, 0xC0FFEE + 71, 0xC0FFEE + 31]


def workloads(n_frames, storage=L.KF_STORAGE_F16U16, jtj=L.KF_JTJ_SPLIT_BF16):
    return [small_workload(n_frames, size=sz, storage=storage, jtj=jtj, quirks=L.KF_QUIRKS_TRACKING, seed=sd)
            for sz, sd in zip(SIZES, SEEDS)]


def fresh(ws):
    gs = []
    for w in ws:
        g = GFusion(w.config, w.intrinsics)
        g.Reset(w.poses[0])
        gs.append(g)
    return gs


def snapshot(g):
    return g.getPose(), g.getVerts(), g.getNorms(), g.getVolumeRaw()


def assert_same(a, b):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_batch_equals_alone_bit_exact():
    F = 6
    ws = workloads(F)
    frames = [[w.frame(k) for k in range(F)] for w in ws]
    alone = fresh(ws)
    tr_alone = np.array([[g.frameStep(frames[i][k]) for k in range(F)] for i, g in enumerate(alone)])
    together = fresh(ws)
    batch = GFusionBatch(8)
    tr_batch = np.array([batch.frameStep(together, [frames[i][k] for i in range(len(ws))]) for k in range(F)]).T
    np.testing.assert_array_equal(tr_alone, tr_batch)
    assert tr_batch[:, -1].all()
    for ga, gb in zip(alone, together):
        assert_same(snapshot(ga), snapshot(gb))
    t = batch.stageTimes()
    assert (t >= 0).all() and t[1] > 0


def test_batch_icp_waves_bit_exact():
    """More members than one ICP wave holds (KF_BATCH_ICP_WAVE = 32): the batched ICP runs as
    two cooperative launches; every member still matches its alone run bit for bit."""
    F, n = 3, 36
    ws = [small_workload(F, size=48, storage=L.KF_STORAGE_F16U16, jtj=L.KF_JTJ_SPLIT_BF16,
                         quirks=L.KF_QUIRKS_TRACKING, seed=0xC0FFEE + 101 + 7 * k) for k in range(n)]
    frames = [[w.frame(k) for k in range(F)] for w in ws]
    alone = fresh(ws)
    for i, g in enumerate(alone):
        for k in range(F):
            g.frameStep(frames[i][k])
    together = fresh(ws)
    batch = GFusionBatch(n)
    for k in range(F):
        batch.frameStep(together, [frames[i][k] for i in range(n)])
    for ga, gb in zip(alone, together):
        np.testing.assert_array_equal(ga.getPose(), gb.getPose())
        np.testing.assert_array_equal(ga.getVerts(), gb.getVerts())


def test_batch_membership_changes():
    """Sessions join and leave between steps; each still matches its alone run."""
    F = 5
    ws = workloads(F)
    frames = [[w.frame(k) for k in range(F)] for w in ws]
    alone = fresh(ws)
    for i, g in enumerate(alone):
        for k in range(F):
            g.frameStep(frames[i][k])
    mixed = fresh(ws)
    batch = GFusionBatch(4)
    nxt = [0] * len(ws)
    plan = [[0, 1, 2, 3], [1], [0, 2], [3, 2, 1], [0], [0, 1, 2, 3], [2, 3], [1, 3], [0, 1, 2, 3], [0, 2, 3], [1]]
    for members in plan:
        members = [m for m in members if nxt[m] < F]
        if not members:
            continue
        batch.frameStep([mixed[m] for m in members], [frames[m][nxt[m]] for m in members])
        for m in members:
            nxt[m] += 1
    for i, g in enumerate(mixed):
        while nxt[i] < F:
            g.frameStep(frames[i][nxt[i]])  # the rest alone
            nxt[i] += 1
    for ga, gb in zip(alone, mixed):
        assert_same(snapshot(ga), snapshot(gb))


def test_batch_fp32_jtj_within_tolerance(tmp_path):
    """The FP32 J^T J form sums per thread and block in FP32, so a different block split
    (a batch gives each session fewer blocks) may round differently.  Per frame, from the
    same state (the alone session's checkpoint loaded into the batched one before every
    step), poses agree within the per-frame tolerance (0.1 mm / 0.01 deg)."""
    F = 5
    ws = [small_workload(F, size=sz, storage=L.KF_STORAGE_F32F32, jtj=L.KF_JTJ_FP32, quirks=L.KF_QUIRKS_TRACKING,
                         seed=0xC0FFEE + sd) for sz, sd in ((128, 21), (112, 71), (96, 1))]
    frames = [[w.frame(k) for k in range(F)] for w in ws]
    alone = fresh(ws)
    together = fresh(ws)
    batch = GFusionBatch(3)
    for k in range(F):
        for i, (ga, gb) in enumerate(zip(alone, together)):
            ga.saveVolume(tmp_path / f"s{i}.kfc")
            gb.loadVolume(tmp_path / f"s{i}.kfc")
        for i, g in enumerate(alone):
            g.frameStep(frames[i][k])
        batch.frameStep(together, [frames[i][k] for i in range(len(ws))])
        for ga, gb in zip(alone, together):
            Pa, Pb = ga.getPose(), gb.getPose()
            assert np.abs(Pa[:3, 3] - Pb[:3, 3]).max() < 1e-4, k
            R = Pa[:3, :3].T @ Pb[:3, :3]
            assert np.degrees(np.arccos(np.clip((np.trace(R) - 1) / 2, -1, 1))) < 0.01, k


def test_batch_rejects_bad_membership():
    ws = workloads(1)
    gs = fresh(ws[:2])
    f = ws[0].frame(0)
    batch = GFusionBatch(2)
    with pytest.raises(L.KfError) as e:
        batch.frameStep([gs[0], gs[0]], [f, f])
    assert e.value.status == L.KF_ERR_INVALID_ARGUMENT
    other = small_workload(1, size=64, storage=L.KF_STORAGE_F32F32, jtj=L.KF_JTJ_SPLIT_BF16)
    g32 = GFusion(other.config, other.intrinsics)
    g32.Reset(other.poses[0])
    with pytest.raises(L.KfError) as e:
        batch.frameStep([gs[0], g32], [f, f])
    assert e.value.status == L.KF_ERR_INVALID_ARGUMENT
    g3 = fresh(ws[2:3])[0]
    with pytest.raises(L.KfError) as e:
        batch.frameStep([gs[0], gs[1], g3], [f, f, f])
    assert e.value.status == L.KF_ERR_CAPACITY
    # a valid step still works after the refusals
    assert batch.frameStep(gs, [f, f]).shape == (2,)


def test_batch_tables_follow_replaced_sessions():
    """A destroyed session's address may come back for the next session created, and a
    session may reallocate its buffers (Reset with delete): the batch must rebuild its
    per-member tables rather than reuse stale ones."""
    ws = workloads(3)
    fr = [[w.frame(k) for k in range(3)] for w in ws]
    batch = GFusionBatch(2)
    a, b = fresh(ws[:2])
    batch.frameStep([a, b], [fr[0][0], fr[1][0]])
    a.close()
    del a
    c = fresh(ws[2:3])[0]  # a different volume size, possibly at a's old address
    batch.frameStep([c, b], [fr[2][0], fr[1][1]])
    b.Reset(ws[1].poses[0], True)  # reallocates b's volume
    batch.frameStep([c, b], [fr[2][1], fr[1][0]])
    ref_c = fresh(ws[2:3])[0]
    ref_c.frameStep(fr[2][0])
    ref_c.frameStep(fr[2][1])
    ref_b = fresh(ws[1:2])[0]
    ref_b.frameStep(fr[1][0])
    assert_same(snapshot(c), snapshot(ref_c))
    assert_same(snapshot(b), snapshot(ref_b))


def test_batch_async_steps_match_sync_steps():
    """Asynchronous steps (device frames): each call returns the previous step's results;
    the sessions end exactly where synchronous steps take them."""
    import torch
    F = 5
    ws = workloads(F)
    frames = [[w.frame(k) for k in range(F)] for w in ws]
    dev = [torch.from_numpy(np.stack(fr).view(np.int16)).cuda() for fr in frames]
    fbytes = 512 * 424 * 2
    sync_s, async_s = fresh(ws), fresh(ws)
    b1, b2 = GFusionBatch(4), GFusionBatch(4)
    torch.cuda.synchronize()
    sync_poses = []
    for k in range(F):
        b1.frameStepDevice(sync_s, [d.data_ptr() + k * fbytes for d in dev])
        sync_poses.append(b1.poses(len(ws)))
    for k in range(F):
        b2.frameStepDeviceAsync(async_s, [d.data_ptr() + k * fbytes for d in dev])
        if k > 0:
            np.testing.assert_array_equal(b2.poses(len(ws)), sync_poses[k - 1])
    b2.sync()
    np.testing.assert_array_equal(b2.poses(len(ws)), sync_poses[-1])
    assert b2.tracked(len(ws)).all()
    for ga, gb in zip(sync_s, async_s):
        assert_same(snapshot(ga), snapshot(gb))


def test_batch_step_graphs_match_direct_launches():
    """Device-frame steps run as per-slot CUDA graphs (captured on first use, replayed,
    recaptured when the membership changes); host-frame steps launch directly.  Both take
    the sessions to the same bits, across a membership change."""
    import torch
    F = 6
    ws = workloads(F)
    frames = [[w.frame(k) for k in range(F)] for w in ws]
    dev = [torch.from_numpy(np.stack(fr).view(np.int16)).cuda() for fr in frames]
    fbytes = 512 * 424 * 2
    direct, graphed = fresh(ws), fresh(ws)
    b1, b2 = GFusionBatch(4), GFusionBatch(4)
    torch.cuda.synchronize()
    for k in range(F):
        members = range(len(ws)) if k < 3 or k >= 5 else range(1, len(ws))  # session 0 sits out
        b1.frameStep([direct[i] for i in members], [frames[i][k] for i in members])
        b2.frameStepDevice([graphed[i] for i in members], [dev[i].data_ptr() + k * fbytes for i in members])
        np.testing.assert_array_equal(b1.poses(len(members)), b2.poses(len(members)))
    for ga, gb in zip(direct, graphed):
        assert_same(snapshot(ga), snapshot(gb))
    # a replayed graph counts its kernels like direct launches do
    assert b2.launchCount() == b1.launchCount()
