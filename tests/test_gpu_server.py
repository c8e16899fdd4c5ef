"""The served form (kf_server_*): admission by slots and device memory, continuous
batching of queued frames, and each session's results equal to running it alone."""
import numpy as np
import pytest

from helpers import small_workload
from oglfusionkinectv2_b200 import GFusion, GFusionServer, _lib as L

pytestmark = pytest.mark.gpu

SPECS = [(96, 0xC0FFEE + 1), (128, 0xC0FFEE + 21), (112, 0xC0FFEE + 71)]


def workloads(n_frames):
    return [small_workload(n_frames, size=sz, storage=L.KF_STORAGE_F16U16, jtj=L.KF_JTJ_SPLIT_BF16,
                           quirks=L.KF_QUIRKS_TRACKING, seed=sd) for sz, sd in SPECS]


def alone_poses(w, frames):
    g = GFusion(w.config, w.intrinsics)
    g.Reset(w.poses[0])
    out = []
    for f in frames:
        g.frameStep(f)
        out.append(g.getPose())
    return out


def drain(server, ids):
    while any(server.pending(i) for i in ids):
        server.step()


def test_server_admission_continuous_batching_and_results():
    F = 5
    ws = workloads(F)
    frames = [[w.frame(k) for k in range(F)] for w in ws]
    ref = [alone_poses(w, fr) for w, fr in zip(ws, frames)]
    v = GFusionServer(max_sessions=2, max_batch=2)
    a = v.open(ws[0].config, ws[0].intrinsics, ws[0].poses[0])
    b = v.open(ws[1].config, ws[1].intrinsics, ws[1].poses[0])
    assert a is not None and b is not None
    assert v.open(ws[2].config, ws[2].intrinsics, ws[2].poses[0]) is None  # no free slot
    # uneven arrivals: a has three frames waiting, b one
    for k in range(3):
        v.submit(a, frames[0][k])
    v.submit(b, frames[1][0])
    assert v.step() == 2  # one frame of each
    P, tracked, done = v.pose(a)
    np.testing.assert_array_equal(P, ref[0][0])
    assert done == 1
    drain(v, [a, b])
    np.testing.assert_array_equal(v.pose(a)[0], ref[0][2])
    np.testing.assert_array_equal(v.pose(b)[0], ref[1][0])
    # a leaves, c takes its slot while b is mid-stream
    for k in range(3, F):
        v.submit(a, frames[0][k])
    drain(v, [a])
    np.testing.assert_array_equal(v.pose(a)[0], ref[0][F - 1])
    v.close_session(a)
    c = v.open(ws[2].config, ws[2].intrinsics, ws[2].poses[0])
    assert c is not None
    for k in range(F):
        v.submit(c, frames[2][k])
        if k + 1 < F:
            v.submit(b, frames[1][k + 1])
        v.step()
    drain(v, [b, c])
    np.testing.assert_array_equal(v.pose(b)[0], ref[1][F - 1])
    np.testing.assert_array_equal(v.pose(c)[0], ref[2][F - 1])
    st = v.stats()
    assert st["frames"] == 3 * F and st["p99_ms"] >= st["p50_ms"] > 0
    assert st["active_sessions"] == 2


def test_server_memory_budget():
    ws = workloads(1)
    v = GFusionServer(hbm_budget_bytes=64 << 20, max_sessions=4, max_batch=4)
    assert v.open(ws[0].config, ws[0].intrinsics, ws[0].poses[0]) is not None  # 96^3: fits
    assert v.open(ws[1].config, ws[1].intrinsics, ws[1].poses[0]) is None  # 128^3 would exceed 64 MB


def test_server_reuses_closed_sessions():
    """A closed session's memory serves the next admission of the same volume size, reset:
    the new session's results equal a fresh one's."""
    F = 3
    ws = workloads(F)
    fr = [[w.frame(k) for k in range(F)] for w in ws]
    v = GFusionServer(max_sessions=2, max_batch=2)
    a = v.open(ws[0].config, ws[0].intrinsics, ws[0].poses[0])
    for k in range(F):
        v.submit(a, fr[0][k])
    drain(v, [a])
    v.close_session(a)
    # same volume size, another scene and start pose
    w2 = small_workload(F, size=SPECS[0][0], storage=L.KF_STORAGE_F16U16, jtj=L.KF_JTJ_SPLIT_BF16,
                        quirks=L.KF_QUIRKS_TRACKING, seed=0xC0FFEE + 41)
    f2 = [w2.frame(k) for k in range(F)]
    b = v.open(w2.config, w2.intrinsics, w2.poses[0])
    for k in range(F):
        v.submit(b, f2[k])
    drain(v, [b])
    np.testing.assert_array_equal(v.pose(b)[0], alone_poses(w2, f2)[-1])


def test_server_prewarm_and_eviction():
    """Prewarmed sessions count against the budget, serve admissions of their size, and are
    released when another size needs the room."""
    ws = workloads(2)
    v = GFusionServer(hbm_budget_bytes=100 << 20, max_sessions=4, max_batch=4)
    assert v.prewarm(ws[0].config, ws[0].intrinsics, 5) == 2  # about 38 MiB each
    a = v.open(ws[0].config, ws[0].intrinsics, ws[0].poses[0])  # takes a warm one
    assert a is not None
    b = v.open(ws[1].config, ws[1].intrinsics, ws[1].poses[0])  # evicts the other warm one
    assert b is not None
    f = [ws[0].frame(0), ws[1].frame(0)]
    v.submit(a, f[0])
    v.submit(b, f[1])
    assert v.step() == 2
    np.testing.assert_array_equal(v.pose(a)[0], alone_poses(ws[0], f[:1])[-1])
    np.testing.assert_array_equal(v.pose(b)[0], alone_poses(ws[1], f[1:])[-1])


def test_server_async_steps_match_alone():
    """Asynchronous served steps: each call enqueues a step and returns the previous one's
    frame count; submissions and an admission happen while a step is on the device, and
    every session's poses equal running it alone."""
    F = 5
    ws = workloads(F)
    frames = [[w.frame(k) for k in range(F)] for w in ws]
    ref = [alone_poses(w, fr) for w, fr in zip(ws, frames)]
    v = GFusionServer(max_sessions=3, max_batch=3)
    a = v.open(ws[0].config, ws[0].intrinsics, ws[0].poses[0])
    b = v.open(ws[1].config, ws[1].intrinsics, ws[1].poses[0])
    seen = {a: [], b: []}

    def collect(n):
        if n:
            ids, poses, _ = v.last_step(3)
            assert len(ids) == n
            for sid, P in zip(ids.tolist(), poses):
                seen[sid].append(P)

    c = None
    for k in range(F):
        v.submit(a, frames[0][k])
        v.submit(b, frames[1][k])
        if k == 2:
            c = v.open(ws[2].config, ws[2].intrinsics, ws[2].poses[0])  # joins mid-stream
            seen[c] = []
        if c is not None:
            v.submit(c, frames[2][k - 2])
        collect(v.step_async())
    for k in range(F - 2, F):  # c's remaining frames, one step each
        v.submit(c, frames[2][k])
        collect(v.step_async())
    collect(v.sync())
    assert v.sync() == 0
    assert v.stats()["frames"] == 3 * F
    for sid, r in ((a, ref[0]), (b, ref[1]), (c, ref[2])):
        assert len(seen[sid]) == F
        for P, Q in zip(seen[sid], r):
            np.testing.assert_array_equal(P, Q)
    v.close_session(c)
