"""Depth ingest before the pyramid through the C ABI vs the oracle: the Kinect-v2
undistortion map (libfreenect2 Registration) and filter3D.cs, bit-exact; a frame loop
with both stages on."""
import numpy as np
import pytest

import kf_oracle as O
from helpers import small_workload
from oglfusionkinectv2_b200 import GFusion, GFusionBatch, _lib as L

pytestmark = pytest.mark.gpu

IRS = [(365.1, 364.7, 255.3, 208.9, 0.092, -0.27, 0.094, 0.0012, -0.0006),
       (365.0, 365.0, 256.0, 212.0, 0.0, 0.0, 0.0, 0.0, 0.0),
       (360.0, 361.0, 250.0, 205.0, 0.6, -2.0, 4.0, 0.02, -0.03)]


def pair(w):
    return GFusion(w.config, w.intrinsics), O.Oracle(w.config, w.intrinsics)


@pytest.mark.parametrize("ir", IRS)
def test_undistortion_map_is_bit_exact(ir):
    w = small_workload(1, size=32)
    g, o = pair(w)
    with pytest.raises(L.KfError) as e:
        g.getUndistortionMap()
    assert e.value.status == L.KF_ERR_STATE
    for s in (g, o):
        s.setDepthUndistortion(ir)
    np.testing.assert_array_equal(g.getUndistortionMap(), o.getUndistortionMap())


def _noisy_frame(w, k, seed):
    """A rendered frame with holes, out-of-range depths and speckle, so that every branch of
    filter3D.cs is taken."""
    f = w.frame(k).astype(np.int32)
    rng = np.random.default_rng(seed)
    f += rng.integers(-6, 7, f.shape)
    f[rng.random(f.shape) < 0.05] = 0
    f[rng.random(f.shape) < 0.01] = 4500
    f[rng.random(f.shape) < 0.01] = 3
    return np.clip(f, 0, 65535).astype(np.uint16)


@pytest.mark.parametrize("undistort,filt", [(True, False), (False, True), (True, True)])
def test_ingest_level0_is_bit_exact(undistort, filt):
    w = small_workload(2, size=32)
    g, o = pair(w)
    for s in (g, o):
        s.setDepthUndistortion(IRS[0] if undistort else None)
        s.setDepthFilter(filt)
    raw = _noisy_frame(w, 0, 7)
    for inp in (raw, raw.astype(np.float32) + 0.375):
        for s in (g, o):
            s.depthToVertex(inp)
        dg, do = g.getDepthImage(0), o.getDepthImage(0)
        np.testing.assert_array_equal(dg, do.astype(np.float32))
        assert (dg > 0).mean() > 0.3
        for l in (1, 2):
            np.testing.assert_allclose(g.getDepthImage(l), o.getDepthImage(l), rtol=1e-6)
    # off again: the pyramid reads the raw frame
    for s in (g, o):
        s.setDepthUndistortion(None)
        s.setDepthFilter(False)
        s.depthToVertex(raw)
    np.testing.assert_array_equal(g.getDepthImage(0), raw.astype(np.float32))


def test_frame_loop_with_ingest_matches_oracle():
    """Undistortion and filter on in the captured frame graph: same tracked flags as the
    oracle, poses within 1 mm, and the same frames as the step-by-step entry points.  The
    frames carry the workload's own sensor noise and dropouts (with the harsher noise of
    _noisy_frame the 5 mm filter leaves too few pixels for a well-conditioned ICP, and the
    FP64 and FP32 trackers wander apart by millimetres)."""
    w = small_workload(6, size=128)
    g, o = pair(w)
    h = GFusion(w.config, w.intrinsics)
    for s in (g, o, h):
        s.Reset(w.poses[0])
        s.setDepthUndistortion(IRS[0])
        s.setDepthFilter(True)
    for k in range(w.n_frames):
        f = w.frame(k)
        tg, to = g.frameStep(f), o.frameStep(f)
        assert tg == to, k
        assert np.linalg.norm(g.getPose()[:3, 3] - o.getPose()[:3, 3]) < 1e-3
        h.depthToVertex(f)
        np.testing.assert_array_equal(h.getDepthImage(0), g.getDepthImage(0))


def test_batch_refuses_sessions_with_ingest():
    w = small_workload(1, size=32)
    a, b = GFusion(w.config, w.intrinsics), GFusion(w.config, w.intrinsics)
    b.setDepthFilter(True)
    batch = GFusionBatch(2)
    with pytest.raises(L.KfError) as e:
        batch.frameStep([a, b], [w.frame(0), w.frame(0)])
    assert e.value.status == L.KF_ERR_INVALID_ARGUMENT
    b.setDepthFilter(False)
    assert len(batch.frameStep([a, b], [w.frame(0), w.frame(0)])) == 2


def test_invalid_ir_camera_is_rejected():
    w = small_workload(1, size=32)
    g = GFusion(w.config, w.intrinsics)
    for bad in ((0.0,) + IRS[0][1:], IRS[0][:4] + (float("nan"),) + IRS[0][5:]):
        with pytest.raises(L.KfError) as e:
            g.setDepthUndistortion(bad)
        assert e.value.status == L.KF_ERR_INVALID_ARGUMENT
