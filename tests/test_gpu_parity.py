"""GPU (CUDA, through the C ABI) vs FP64 oracle parity on identical inputs.

Tolerances (the parity bar): TSDF max-abs <= 1e-3 of the truncation (normalised units) on
every voxel whose evaluation is unambiguous; per-frame pose <= 0.1 mm / 0.01 deg with
teacher forcing; raycast vertex <= 0.5 mm; free-running ATE within 1 mm of the oracle.
"""
import numpy as np
import pytest

import kf_oracle as O
from helpers import integrate_ambiguous, raycast_ambiguous, rot_deg, small_workload
from oglfusionkinectv2_b200 import GFusion, synth, _lib as L

pytestmark = pytest.mark.gpu

STORAGES = [L.KF_STORAGE_F32F32, L.KF_STORAGE_F16U16, L.KF_STORAGE_RG16I]
QUIRKS = {"tracking": L.KF_QUIRKS_TRACKING, "default": L.KF_QUIRKS_DEFAULT,
          "reference": L.KF_QUIRKS_REFERENCE}


def pair(w):
    return GFusion(w.config, w.intrinsics), O.Oracle(w.config, w.intrinsics)


def test_pyramid_parity():
    w = small_workload(3)
    g, o = pair(w)
    f = w.frame(1)
    for s in (g, o):
        s.depthToVertex(f)
        s.vertexToNormal()
    for l in range(3):
        np.testing.assert_allclose(g.getDepthImage(l), o.getDepthImage(l), rtol=1e-6)
        Vg, Vo = g.getVertexMap(l), o.getVertexMap(l)
        assert np.max(np.abs(Vg[..., :3] - Vo[..., :3])) < 2e-6
        Ng, No = g.getNormalMap(l), o.getNormalMap(l)
        np.testing.assert_array_equal(Ng[..., 0] == 2, No[..., 0] == 2)
        valid = No[..., 0] != 2
        err = np.linalg.norm(Ng[..., :3] - No[..., :3], axis=-1)[valid]
        assert np.mean(err < 1e-4) > 0.9999 and err.max() < 1e-2
    # float input path (the reference's depthToVertex(float*))
    g.depthToVertex(f.astype(np.float32) + 0.25)
    o.depthToVertex(f.astype(np.float32) + 0.25)
    np.testing.assert_allclose(g.getDepthImage(0), o.getDepthImage(0), rtol=0)


@pytest.mark.parametrize("storage", STORAGES)
@pytest.mark.parametrize("quirks", ["tracking", "default"])
def test_integrate_parity(storage, quirks):
    w = small_workload(3, size=96, storage=storage, quirks=QUIRKS[quirks])
    g, o = pair(w)
    for s in (g, o):
        s.Reset(w.poses[0])
    for k in (0, 1):
        f = w.frame(k)
        oldF, oldW = o.getVolume()
        if k:
            g.setVolumeRaw(o.getVolumeRaw())  # identical input volume
        for s in (g, o):
            s.setPose(w.poses[k])
            s.depthToVertex(f)
            s.integrate()
        Fg, Wg = g.getVolume()
        Fo, Wo = o.getVolume()
        bad = (np.abs(Fg - Fo) > 1e-3) | (Wg != Wo)
        touched = (Wo > 0) | (Wg > 0)
        idx = np.nonzero(bad)
        amb = integrate_ambiguous(w.config, w.intrinsics, w.poses[k], f, oldF, oldW, idx)
        assert touched.sum() > 1000
        assert bad.sum() <= 1e-3 * touched.sum(), (bad.sum(), touched.sum())
        assert amb.all(), f"{(~amb).sum()} unexplained voxel mismatches"


@pytest.mark.parametrize("storage", STORAGES)
def test_raycast_parity(storage):
    w = small_workload(3, size=128, storage=storage)
    g, o = pair(w)
    o.Reset(w.poses[0])
    for k in (0, 1):
        o.setPose(w.poses[k])
        o.depthToVertex(w.frame(k))
        o.integrate()
    g.setVolumeRaw(o.getVolumeRaw())
    for s in (g, o):
        s.setPose(w.poses[2])
        s.raycast()
    Vg, Ng = g.getVerts(), g.getNorms()
    Vo, No = o.getVerts(), o.getNorms()
    hg, ho = Vg[..., 3] > 0, Vo[..., 3] > 0
    assert ho.mean() > 0.2
    both = hg & ho
    err = np.where(both, np.linalg.norm(Vg[..., :3] - Vo[..., :3], axis=-1), 0.0)
    # every pixel whose hit/miss differs, or whose vertex is more than 0.5 mm off, must be an
    # FP32/FP64 boundary case of the march (a sample within 1e-4 of 0 or of the 0.8 step
    # switch, a sample on tfar, or a refinement with f(t0) - f(t1) < 0.02)
    mism = (hg != ho) | (err > 0.5e-3)
    ys, xs = np.nonzero(mism)
    Fo, _ = o.getVolume()
    amb = raycast_ambiguous(w.config, w.intrinsics, w.poses[2], Fo, (ys, xs))
    assert amb.all(), f"{int((~amb).sum())} unexplained raycast mismatches of {len(xs)}"
    assert mism.mean() < 1e-3, mism.mean()
    # the largest vertex error among the explained pixels stays within two fine steps
    step = min(w.config.volumeDimensions) / max(w.config.volumeSize)
    assert err.max() <= 2 * step, (err.max(), step)
    nb = both & (No[..., 3] > 0) & (Ng[..., 3] > 0)
    cosang = np.clip(np.einsum("ijk,ijk->ij", Ng[..., :3], No[..., :3])[nb], -1, 1)
    assert np.mean(np.degrees(np.arccos(cosang)) < 1.0) > 0.99


def test_raycast_brick_skip_is_exact():
    """kf_raycast skips 8^3 bricks whose flag says they hold no negative value.  The flags
    kf_integrate maintains (a superset: they are never cleared) and the ones rebuilt from an
    uploaded copy of the same volume must give bit-identical maps, from poses inside and
    outside the volume."""
    w = small_workload(6, size=128)
    g = GFusion(w.config, w.intrinsics)
    g.Reset(w.poses[0])
    for k in range(4):
        g.setPose(w.poses[k])
        g.depthToVertex(w.frame(k))
        g.integrate()
    h = GFusion(w.config, w.intrinsics)
    h.Reset(w.poses[0])
    h.setVolumeRaw(g.getVolumeRaw())
    outside = w.poses[0].copy()
    outside[:3, 3] -= 0.6 * outside[:3, 2]  # back the camera out along its view axis
    for pose in (w.poses[4], w.poses[5], outside):
        for s in (g, h):
            s.setPose(pose)
            s.raycast()
        Vg, Vh = g.getVerts(), h.getVerts()
        assert (Vg[..., 3] > 0).mean() > 0.1
        np.testing.assert_array_equal(Vg, Vh)
        np.testing.assert_array_equal(g.getNorms(), h.getNorms())


def _teacher_forced(w, k, track):
    """Both sides track frame k from the pose of frame k-1 against identical reference
    maps (the GPU raycast copied into the oracle) and an identical volume."""
    g, o = pair(w)
    o.Reset(w.poses[0])
    for j in range(k):
        o.setPose(w.poses[j])
        o.depthToVertex(w.frame(j))
        o.integrate()
    g.Reset(w.poses[0])
    g.setVolumeRaw(o.getVolumeRaw())
    for s in (g, o):
        s.setPose(w.poses[k - 1])
        s.raycast()
    o.setRaycast(g.getVerts().astype(np.float64), g.getNorms().astype(np.float64))
    f = w.frame(k)
    for s in (g, o):
        s.depthToVertex(f)
        s.vertexToNormal()
    tg = getattr(g, track)()
    to = getattr(o, track)()
    return g, o, tg, to


@pytest.mark.parametrize("jtj", [L.KF_JTJ_FP32, L.KF_JTJ_SPLIT_BF16])
@pytest.mark.parametrize("quirks", ["tracking", "default", "reference"])
def test_icp_teacher_forced(jtj, quirks):
    w = small_workload(6, size=128, jtj=jtj, quirks=QUIRKS[quirks])
    for k in (2, 4):
        g, o, tg, to = _teacher_forced(w, k, "Track")
        assert tg == to
        Pg, Po = g.getPose(), o.getPose()
        assert np.linalg.norm(Pg[:3, 3] - Po[:3, 3]) <= 1e-4
        assert rot_deg(Pg, Po) <= 0.01
        sg, so = g.getTrackStatus(0), o.getTrackStatus(0)
        assert np.mean(sg == so) > 0.999
        rg, ro = g.getReduction(), o.getReduction()
        assert rg[28] == ro[28]
        assert abs(g.alignmentEnergy() - o.alignmentEnergy()) <= 1e-3 * o.alignmentEnergy() + 1e-7


@pytest.mark.parametrize("quirks", ["tracking", "default"])
def test_sdf_teacher_forced(quirks):
    w = small_workload(5, size=128, quirks=QUIRKS[quirks], tracking=L.KF_TRACK_SDF)
    for k in (2, 3):
        g, o, tg, to = _teacher_forced(w, k, "TrackSDF")
        assert tg == to
        Pg, Po = g.getPose(), o.getPose()
        assert np.linalg.norm(Pg[:3, 3] - Po[:3, 3]) <= 1e-4
        assert rot_deg(Pg, Po) <= 0.01


@pytest.mark.parametrize("storage", [L.KF_STORAGE_F32F32, L.KF_STORAGE_F16U16])
def test_frame_loop_ate_vs_oracle(storage):
    """kinect.cpp:654-695 free-running on both sides over the full 100 frames of the
    128^3 plain workload: trajectories within 1 mm ATE."""
    w = synth.plain_c1(100)
    w.config.storage = storage
    g, o = pair(w)
    for s in (g, o):
        s.Reset(w.poses[0])
    pg, po = [], []
    for k in range(w.n_frames):
        f = w.frame(k)
        tg, to = g.frameStep(f), o.frameStep(f)
        assert tg == to, k
        pg.append(g.getPose())
        po.append(o.getPose())
    assert synth.ate(pg, po) <= 1e-3
    assert synth.ate(pg, w.poses) <= 5e-3  # and it actually tracks the ground truth


def test_frame_step_graph_matches_step_by_step():
    """The captured frame graph and the individual entry points compute the same frame."""
    w = small_workload(4, size=64)
    a, b = GFusion(w.config, w.intrinsics), GFusion(w.config, w.intrinsics)
    for s in (a, b):
        s.Reset(w.poses[0])
    counter = 0
    reset = True
    for k in range(4):
        f = w.frame(k)
        ta = a.frameStep(f)
        b.depthToVertex(f)
        b.vertexToNormal()
        tb = b.Track()
        if tb or reset:
            b.integrate()
            if counter > 2:
                reset = False
        if not tb:
            b.recoverPose()
        counter += 1
        b.raycast()
        assert ta == tb
        np.testing.assert_array_equal(a.getPose(), b.getPose())
    np.testing.assert_array_equal(a.getVolumeRaw(), b.getVolumeRaw())
    np.testing.assert_array_equal(a.getVerts(), b.getVerts())


def test_stage_timing_sampling():
    """kf_set_stage_timing: the frame graphs of every n-th ring slot record the stage
    boundaries (default n = 4), the others the frame only; the frames compute the same."""
    w = small_workload(13, size=64)
    a, b = GFusion(w.config, w.intrinsics), GFusion(w.config, w.intrinsics)
    assert a.stageTiming() == 4
    b.setStageTiming(1)
    with pytest.raises(L.KfError):
        b.setStageTiming(3)
    for s in (a, b):
        s.Reset(w.poses[0])
        s.resetStageStats()
    for k in range(8):
        f = w.frame(k)
        assert a.frameStep(f) == b.frameStep(f)
    ma, na = a.stageStats()
    mb, nb = b.stageStats()
    assert (na, nb) == (2, 8)
    assert np.all(ma[:5] > 0) and np.all(mb[:5] > 0)
    np.testing.assert_array_equal(a.getPose(), b.getPose())
    b.setStageTiming(0)  # frames already run keep their times; no more are timed
    for k in range(8, 13):
        f = w.frame(k)
        assert a.frameStep(f) == b.frameStep(f)
    assert b.stageStats()[1] == 8 and a.stageStats()[1] == 4
    np.testing.assert_array_equal(a.getPose(), b.getPose())
    np.testing.assert_array_equal(a.getVolumeRaw(), b.getVolumeRaw())


def test_async_frame_steps_match_sync_steps():
    """Pipelined frame steps: each call reads the previous frame's result; the session ends
    exactly where synchronous steps take it."""
    w = small_workload(6, size=64)
    a, b = GFusion(w.config, w.intrinsics), GFusion(w.config, w.intrinsics)
    for s in (a, b):
        s.Reset(w.poses[0])
    sync_res = []
    for k in range(w.n_frames):
        t = a.frameStep(w.frame(k))
        sync_res.append((a.getPose(), t))
    for k in range(w.n_frames):
        b.frameStepAsync(w.frame(k))
        if k > 0:
            P, t = b.lastResult()
            np.testing.assert_array_equal(P, sync_res[k - 1][0])
            assert t == sync_res[k - 1][1]
    assert b.frameSync() == sync_res[-1][1]
    np.testing.assert_array_equal(b.lastResult()[0], sync_res[-1][0])
    np.testing.assert_array_equal(a.getVolumeRaw(), b.getVolumeRaw())
    np.testing.assert_array_equal(a.getVerts(), b.getVerts())
    # a synchronous call after an asynchronous one reads the pending result first
    b.frameStepAsync(w.frame(0))
    np.testing.assert_array_equal(b.getPose(), b.lastResult()[0])


def test_pose_library_and_recover():
    """A frame whose every pixel fails the ICP distance gate (a flat wall at 4.2 m, outside
    the volume) is not tracked (AE == 0); both sides then run recoverPose (TrackSDF from
    each pose of the library) and end on the same pose."""
    w = small_workload(8, size=64)
    g, o = pair(w)
    for s in (g, o):
        s.Reset(w.poses[0])
    for k in range(6):
        f = w.frame(k)
        assert g.frameStep(f) == o.frameStep(f)
    assert g.poseLibrarySize() == o.poseLibrarySize() >= 1
    wall = np.full((424, 512), 4200, np.uint16)
    tg, to = g.frameStep(wall), o.frameStep(wall)
    assert tg is False and to is False
    Pg, Po = g.getPose(), o.getPose()
    # the library holds each side's own tracked poses (within the 1 mm trajectory bound)
    assert np.linalg.norm(Pg[:3, 3] - Po[:3, 3]) <= 1e-3


def test_frame_graph_recover_matches_step_by_step():
    """In the frame graph the recover launch is the body of a conditional node that the ICP
    kernel sets when the frame is not tracked: a lost frame (the wall) runs it, a tracked
    one does not, and both match the entry points called one by one, bit for bit."""
    w = small_workload(7, size=64)
    a, b = GFusion(w.config, w.intrinsics), GFusion(w.config, w.intrinsics)
    for s in (a, b):
        s.Reset(w.poses[0])
    wall = np.full((424, 512), 4200, np.uint16)
    frames = [w.frame(k) for k in range(5)] + [wall, w.frame(5)]
    counter, reset, flags = 0, True, []
    for k, f in enumerate(frames):
        ta = a.frameStep(f)
        b.depthToVertex(f)
        b.vertexToNormal()
        tb = b.Track()
        if tb or reset:
            b.integrate()
            if counter > 2:
                reset = False
        if not tb:
            b.recoverPose()
        counter += 1
        b.raycast()
        assert ta == tb, k
        flags.append(ta)
        np.testing.assert_array_equal(a.getPose(), b.getPose())
    # the first frame has no raycast to track against; the next four track; the wall is lost
    assert flags[:6] == [False, True, True, True, True, False], flags
    np.testing.assert_array_equal(a.getVolumeRaw(), b.getVolumeRaw())
    np.testing.assert_array_equal(a.getVerts(), b.getVerts())


def test_errors_are_reported():
    w = small_workload(1, size=32)
    g = GFusion(w.config, w.intrinsics)
    with pytest.raises(ValueError):
        g.depthToVertex(np.zeros((10, 10), np.uint16))
    with pytest.raises(L.KfError) as e:
        g.setVolumeRaw(np.zeros(7, np.uint8))
    assert e.value.status == L.KF_ERR_INVALID_ARGUMENT


def _plane_maps(w, pose, plane_n, plane_h):
    """Analytic world-frame vertex map of the plane n.X = h seen from `pose`, and the hit
    mask; and float millimetre depth of the same view (0 where there is no hit in range)."""
    dirs = w.pixel_rays() @ pose[:3, :3].T
    o = pose[:3, 3]
    n = np.asarray(plane_n, np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        t = (plane_h - n @ o) / (dirs @ n)
    hit = np.isfinite(t) & (t >= 0.5) & (t <= 4.5)
    X = o + dirs * np.where(hit, t, 0.0)[:, None]
    H, W = w.intrinsics.height, w.intrinsics.width
    depth = np.where(hit, t * 1000.0, 0.0).astype(np.float32).reshape(H, W)
    return X.reshape(H, W, 3), hit.reshape(H, W), depth


@pytest.mark.parametrize("jtj", [L.KF_JTJ_FP32, L.KF_JTJ_SPLIT_BF16])
def test_icp_plane_only_rank_guard(jtj):
    """Q22: a view of one plane leaves in-plane translation and rotation about the normal
    unobservable (J^T J of rank 3).  Exact (float) plane depth tracked against exact plane
    reference maps on both sides: the rank guard drops the same three directions on the
    GPU and in the oracle, and both end on the same pose."""
    w = small_workload(3, size=128, jtj=jtj)
    ground = [p for p in w.scene.planes][0]
    pn, ph = np.array(ground[0], np.float64), float(ground[1])
    g, o = pair(w)
    P0, P1 = w.poses[0], w.poses[1]
    X0, hit0, _ = _plane_maps(w, P0, pn, ph)
    _, _, d1 = _plane_maps(w, P1, pn, ph)
    assert hit0.mean() > 0.2 and (d1 > 0).mean() > 0.2
    # raycast normals point back towards the camera
    nrm = -pn if pn @ P0[:3, 3] < ph else pn
    V = np.zeros(hit0.shape + (4,), np.float32)
    N = np.zeros(hit0.shape + (4,), np.float32)
    V[hit0, :3] = X0[hit0]
    V[hit0, 3] = 1.0
    N[hit0, :3] = nrm
    N[hit0, 3] = 1.0
    for s in (g, o):
        s.Reset(P0)
        s.setPose(P0)
        s.raycast()  # sets the association pose; the maps are replaced next
    g.setReferenceMaps(V, N)
    o.setRaycast(V.astype(np.float64), N.astype(np.float64))
    for s in (g, o):
        s.depthToVertex(d1)
        s.vertexToNormal()
    tg, to = g.Track(), o.Track()
    assert tg == to
    Pg, Po = g.getPose(), o.getPose()
    assert np.linalg.norm(Pg[:3, 3] - Po[:3, 3]) <= 1e-4, np.linalg.norm(Pg[:3, 3] - Po[:3, 3])
    assert rot_deg(Pg, Po) <= 0.01
    # the last system was rank-deficient by the guard's measure on both sides
    for red in (g.getReduction(), o.getReduction()):
        Cm = np.zeros((6, 6))
        k = 7
        for i in range(6):
            for j in range(i, 6):
                Cm[i, j] = Cm[j, i] = red[k]
                k += 1
        lam = np.linalg.eigvalsh(Cm)
        assert lam[2] < 1e-5 * lam[-1] and lam[3] > 1e-3 * lam[-1], lam
