"""Volume inspection and persistence through the C ABI: intensity projection (mip.cs) vs the
FP64 oracle, volume checkpoints (save / load / resume), the bounded-wait self-test and the
rejection of non-finite poses."""
import numpy as np
import pytest

import kf_oracle as O
from helpers import small_workload
from oglfusionkinectv2_b200 import GFusion, _lib as L

pytestmark = pytest.mark.gpu

STORAGES = [L.KF_STORAGE_F32F32, L.KF_STORAGE_F16U16, L.KF_STORAGE_RG16I]


@pytest.mark.parametrize("storage", STORAGES)
def test_intensity_projection_parity(storage):
    """Same volume, same pose: per-pixel ray sums agree with the oracle to 1e-4 relative on
    99.9% of pixels; a ray may differ by its last sample where (tfar - tnear) / largeStep
    falls on an integer (a sample value is at most 1)."""
    w = small_workload(3, size=96, storage=storage)
    g, o = GFusion(w.config, w.intrinsics), O.Oracle(w.config, w.intrinsics)
    o.Reset(w.poses[0])
    for k in (0, 1):
        o.setPose(w.poses[k])
        o.depthToVertex(w.frame(k))
        o.integrate()
    g.setVolumeRaw(o.getVolumeRaw())
    outside = w.poses[0].copy()
    outside[:3, 3] -= 0.6 * outside[:3, 2]
    for pose in (w.poses[2], outside):
        for s in (g, o):
            s.setPose(pose)
        mg, mo = g.intensityProjection(), o.intensityProjection()
        assert mg.shape == mo.shape == (w.intrinsics.height, w.intrinsics.width, 4)
        np.testing.assert_array_equal(mg[..., 1:3], 0)
        np.testing.assert_array_equal(mg[..., 3], 1)
        assert (mo[..., 0] > 1.0).mean() > 0.2
        err = np.abs(mg[..., 0] - mo[..., 0])
        assert np.mean(err <= 1e-4 * np.maximum(1.0, mo[..., 0])) > 0.999, np.percentile(err, [50, 99, 99.9])
        assert err.max() <= 1.0 + 1e-3


def _run(s, w, frames):
    return [s.frameStep(w.frame(k)) for k in frames]


def test_checkpoint_resume_is_exact(tmp_path):
    """A session loaded from a checkpoint steps on bit-identically to the saved one."""
    w = small_workload(10, size=64)
    a = GFusion(w.config, w.intrinsics)
    a.Reset(w.poses[0])
    _run(a, w, range(5))
    path = tmp_path / "vol.kfc"
    a.saveVolume(path)
    with open(path, "rb") as f:
        header = f.readline()
    assert header.startswith(b'{"format":"kf-volume-checkpoint","version":1,')
    b = GFusion(w.config, w.intrinsics)
    b.Reset(np.eye(4))
    b.loadVolume(path)
    np.testing.assert_array_equal(a.getPose(), b.getPose())
    np.testing.assert_array_equal(a.getVolumeRaw(), b.getVolumeRaw())
    np.testing.assert_array_equal(a.getVerts(), b.getVerts())
    assert a.poseLibrarySize() == b.poseLibrarySize()
    ta, tb = _run(a, w, range(5, 10)), _run(b, w, range(5, 10))
    assert ta == tb
    np.testing.assert_array_equal(a.getPose(), b.getPose())
    np.testing.assert_array_equal(a.getVolumeRaw(), b.getVolumeRaw())
    np.testing.assert_array_equal(a.getVerts(), b.getVerts())


def test_checkpoint_rejections_leave_session_untouched(tmp_path):
    w = small_workload(3, size=64)
    a = GFusion(w.config, w.intrinsics)
    a.Reset(w.poses[0])
    _run(a, w, range(2))
    good = tmp_path / "good.kfc"
    a.saveVolume(good)
    data = good.read_bytes()
    before_vol, before_pose = a.getVolumeRaw(), a.getPose()

    def expect(path, status):
        with pytest.raises(L.KfError) as e:
            a.loadVolume(path)
        assert e.value.status == status
        np.testing.assert_array_equal(a.getVolumeRaw(), before_vol)
        np.testing.assert_array_equal(a.getPose(), before_pose)

    short = tmp_path / "short.kfc"
    short.write_bytes(data[:-1])
    expect(short, L.KF_ERR_IO)
    junk = tmp_path / "junk.kfc"
    junk.write_bytes(b"not a checkpoint\n" + bytes(64))
    expect(junk, L.KF_ERR_INVALID_ARGUMENT)
    expect(tmp_path / "missing.kfc", L.KF_ERR_IO)
    # a session of another volume size refuses it
    w2 = small_workload(1, size=32)
    c = GFusion(w2.config, w2.intrinsics)
    with pytest.raises(L.KfError) as e:
        c.loadVolume(good)
    assert e.value.status == L.KF_ERR_INVALID_ARGUMENT
    # ... and so does one of the same size with another truncation distance
    w3 = small_workload(1, size=64)
    w3.config.mu *= 1.5
    d = GFusion(w3.config, w3.intrinsics)
    with pytest.raises(L.KfError) as e:
        d.loadVolume(good)
    assert e.value.status == L.KF_ERR_INVALID_ARGUMENT
    # unwritable destination
    with pytest.raises(L.KfError) as e:
        a.saveVolume(tmp_path / "no_such_dir" / "x.kfc")
    assert e.value.status == L.KF_ERR_IO


def test_bounded_wait_times_out_and_session_stays_usable():
    """The self-test's barrier is never completed: the wait gives up after its budget, the
    host reports KF_ERR_TIMEOUT and clears the error, and the next frames match a session
    that never ran the self-test, bit for bit."""
    w = small_workload(4, size=64)
    a, b = GFusion(w.config, w.intrinsics), GFusion(w.config, w.intrinsics)
    for s in (a, b):
        s.Reset(w.poses[0])
    _run(a, w, range(2))
    _run(b, w, range(2))
    assert a.selftestBarrierTimeout(2_000_000) == L.KF_ERR_TIMEOUT
    assert a.selftestBarrierTimeout(1_000) == L.KF_ERR_TIMEOUT
    assert a.selftestBarrierTimeout(10) == L.KF_ERR_INVALID_ARGUMENT
    assert _run(a, w, range(2, 4)) == _run(b, w, range(2, 4))
    np.testing.assert_array_equal(a.getPose(), b.getPose())
    np.testing.assert_array_equal(a.getVolumeRaw(), b.getVolumeRaw())


def test_non_finite_poses_are_rejected():
    w = small_workload(1, size=32)
    g = GFusion(w.config, w.intrinsics)
    g.Reset(w.poses[0])
    before = g.getPose()
    for bad in (np.nan, np.inf, -np.inf):
        p = w.poses[0].copy()
        p[1, 3] = bad
        for call in (g.setPose, g.resetPose, g.Reset):
            with pytest.raises(L.KfError) as e:
                call(p)
            assert e.value.status == L.KF_ERR_INVALID_ARGUMENT
    np.testing.assert_array_equal(g.getPose(), before)
