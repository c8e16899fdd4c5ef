"""GPU vs FP64 oracle at the benchmarked configuration: 512^3 TSDF over a 3 m cube, FP16
value + uint16 weight, split-BF16 J^T J, FP64 solve, ICP {10,5,4}, the tracking quirk set
(the precision form the frame-rate line is measured on).

Tolerances, as in the smaller parity tests: TSDF max-abs <= 1e-3 (of the truncation: values
are stored divided by mu) on every voxel whose evaluation is unambiguous, and every
mismatch explained as an FP32/FP64 boundary case; teacher-forced pose <= 0.1 mm / 0.01 deg;
free-running trajectory within 1 mm ATE of the oracle.
"""
import numpy as np
import pytest

import kf_oracle as O
from helpers import integrate_ambiguous, rot_deg
from oglfusionkinectv2_b200 import GFusion, synth, _lib as L

pytestmark = pytest.mark.gpu


def c2(n_frames):
    w = synth.precision_c2(n_frames)
    assert w.config.volumeSize == (512, 512, 512)
    assert w.config.storage == L.KF_STORAGE_F16U16 and w.config.jtj == L.KF_JTJ_SPLIT_BF16
    return w


def test_integrate_parity_512():
    """Frame 0 into an empty volume, then frame 1 into identical volumes (the oracle's)."""
    w = c2(2)
    g, o = GFusion(w.config, w.intrinsics), O.Oracle(w.config, w.intrinsics)
    for s in (g, o):
        s.Reset(w.poses[0])
    for k in (0, 1):
        f = w.frame(k)
        oldF, oldW = o.getVolume()
        if k:
            g.setVolumeRaw(o.getVolumeRaw())
        for s in (g, o):
            s.setPose(w.poses[k])
            s.depthToVertex(f)
            s.integrate()
        Fg, Wg = g.getVolume()
        Fo, Wo = o.getVolume()
        diff = np.abs(Fg - Fo)
        bad = (diff > 1e-3) | (Wg != Wo)
        touched = int(((Wo > 0) | (Wg > 0)).sum())
        idx = np.nonzero(bad)
        amb = integrate_ambiguous(w.config, w.intrinsics, w.poses[k], f, oldF, oldW, idx)
        assert touched > 1_000_000, touched
        assert bad.sum() <= 1e-3 * touched, (int(bad.sum()), touched)
        assert amb.all(), f"{int((~amb).sum())} unexplained voxel mismatches"
        # max-abs over every voxel that is not such a boundary case
        diff[idx[0][amb], idx[1][amb], idx[2][amb]] = 0
        assert float(diff.max()) <= 1e-3
        del Fg, Wg, Fo, Wo, diff, bad
    g.close()
    o.close()


def test_icp_teacher_forced_512():
    """Frames 2 and 3 tracked from the previous ground-truth pose against identical
    reference maps and an identical volume."""
    w = c2(4)
    o = O.Oracle(w.config, w.intrinsics)
    o.Reset(w.poses[0])
    for j in range(3):
        o.setPose(w.poses[j])
        o.depthToVertex(w.frame(j))
        o.integrate()
        if j < 1:
            continue
        k = j + 1
        g = GFusion(w.config, w.intrinsics)
        g.Reset(w.poses[0])
        g.setVolumeRaw(o.getVolumeRaw())
        saved = o.getPose()
        for s in (g, o):
            s.setPose(w.poses[k - 1])
            s.raycast()
        o.setRaycast(g.getVerts().astype(np.float64), g.getNorms().astype(np.float64))
        f = w.frame(k)
        for s in (g, o):
            s.depthToVertex(f)
            s.vertexToNormal()
        tg, to = g.Track(), o.Track()
        assert tg and to
        Pg, Po = g.getPose(), o.getPose()
        assert np.linalg.norm(Pg[:3, 3] - Po[:3, 3]) <= 1e-4, np.linalg.norm(Pg[:3, 3] - Po[:3, 3])
        assert rot_deg(Pg, Po) <= 0.01
        sg, so = g.getTrackStatus(0), o.getTrackStatus(0)
        assert np.mean(sg == so) > 0.999
        assert g.getReduction()[28] == o.getReduction()[28]
        g.close()
        o.setPose(saved)
    o.close()


def test_frame_loop_ate_vs_oracle_512():
    """src/kinect.cpp:654-695 free-running on both sides over 24 frames: trajectories
    within 1 mm ATE of each other, and within 5 mm of the ground truth."""
    n = 24
    w = c2(n)
    g, o = GFusion(w.config, w.intrinsics), O.Oracle(w.config, w.intrinsics)
    for s in (g, o):
        s.Reset(w.poses[0])
    pg, po = [], []
    for k in range(n):
        f = w.frame(k)
        tg, to = g.frameStep(f), o.frameStep(f)
        assert tg == to, k
        pg.append(g.getPose())
        po.append(o.getPose())
    ate_oracle = synth.ate(pg, po)
    assert ate_oracle <= 1e-3, ate_oracle
    assert synth.ate(pg, w.poses) <= 5e-3
    g.close()
    o.close()
