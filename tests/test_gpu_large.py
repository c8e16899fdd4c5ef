"""Large-volume form (config 5): a 768^3 TSDF over 4 m fused from a room sequence, then full
histoPyramid and scan marching cubes, integer results bit-exact against the FP64 oracle on
the identical TSDF."""
import numpy as np
import pytest

import kf_oracle as O
from oglfusionkinectv2_b200 import GFusion, MCubes, synth, _lib as L

pytestmark = pytest.mark.gpu


def test_large_768_fusion_and_extraction():
    """Frames of the room fused at their ground-truth poses (tracking parity is covered by
    the teacher-forced tests; the reference's SDF tracker drifts on this walk in the FP64
    oracle as on the GPU), then both extraction methods at full size."""
    F = 12
    w = synth.large_c5(F)
    g = GFusion(w.config, w.intrinsics)
    g.Reset(w.poses[0])
    for k in range(F):
        g.setPose(w.poses[k])
        g.depthToVertex(w.frame(k))
        g.integrate()
    raw = g.getVolumeRaw()
    o = O.Oracle(w.config, w.intrinsics)
    o.setVolumeRaw(raw)
    m = MCubes(g)
    for method in (L.KF_MC_HISTOPYRAMID, L.KF_MC_SCAN):
        n_gpu = m.generateMarchingCubes(method)
        n_ref = o.mcExtract(0.0, method)
        assert n_gpu == n_ref and n_gpu > 10000
        np.testing.assert_array_equal(m.getBaseLevel(), o.mcBaseLevel())
        Vg, Vo = m.getVertices(), o.mcVertices()
        assert Vg.shape == Vo.shape and np.max(np.abs(Vg - Vo)) < 1e-4
