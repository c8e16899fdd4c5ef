"""Marching cubes and prefix sum on the GPU vs the FP64 oracle.

Integer outputs are bit-exact on an identical TSDF: every base-level texel (numTri |
cubeIndex << 16), the triangle count, the prefix sums and their totals.  Vertex positions
(float interpolation) agree within 1e-4 voxel.
"""
import ctypes as C

import numpy as np
import pytest

import kf_oracle as O
from helpers import small_workload
from oglfusionkinectv2_b200 import GFusion, GFusionConfig, Intrinsics, MCubes, _lib as L

pytestmark = pytest.mark.gpu

INTR = Intrinsics()


def sphere_raw(n, storage, r=0.3, dim=1.0):
    g = (np.arange(n) + 0.5) * dim / n
    Z, Y, X = np.meshgrid(g, g, g, indexing="ij")
    sd = np.sqrt((X - dim / 2) ** 2 + (Y - dim / 2) ** 2 + (Z - dim / 2) ** 2) - r
    F = np.clip(sd / 0.05, -1, 1).astype(np.float32).ravel()
    W = np.ones(n ** 3, np.float32)
    if storage == L.KF_STORAGE_F32F32:
        return np.concatenate([F, W]).view(np.uint8)
    if storage == L.KF_STORAGE_RG16I:
        return np.concatenate([(F * 32766).astype(np.int32).astype(np.int16), W.astype(np.int16)]).view(np.uint8)
    return np.concatenate([F.astype(np.float16).view(np.uint16), W.astype(np.uint16)]).view(np.uint8)


def both(cfg, raw):
    g = GFusion(cfg, INTR)
    o = O.Oracle(cfg, INTR)
    g.setVolumeRaw(raw)
    o.setVolumeRaw(raw)
    return g, o


def compare(g, o, method, iso=0.0):
    m = MCubes(g)
    m.setIsolevel(iso)
    ng = m.generateMarchingCubes(method)
    no = o.mcExtract(iso, method)
    assert ng == no
    np.testing.assert_array_equal(m.getBaseLevel(), o.mcBaseLevel())
    Vg, Vo = m.getVertices(), o.mcVertices()
    assert Vg.shape == Vo.shape
    if ng:
        assert np.max(np.abs(Vg - Vo)) < 1e-4
    return m, ng


@pytest.mark.parametrize("storage", [L.KF_STORAGE_F32F32, L.KF_STORAGE_F16U16, L.KF_STORAGE_RG16I])
@pytest.mark.parametrize("method", [L.KF_MC_HISTOPYRAMID, L.KF_MC_SCAN])
@pytest.mark.parametrize("quirks", [L.KF_QUIRKS_DEFAULT, L.KF_QUIRKS_TRACKING & ~(L.KF_Q13_MC_FIRST_SEVEN | L.KF_Q15_MC_BORDER_SKIP)])
def test_sphere_bit_exact(storage, method, quirks):
    cfg = GFusionConfig(volumeSize=(64,) * 3, volumeDimensions=(1.0,) * 3, storage=storage, quirks=quirks)
    g, o = both(cfg, sphere_raw(64, storage, r=0.42))
    m, n = compare(g, o, method)
    assert n > 1000


@pytest.mark.parametrize("n", [48, 96, 130])
def test_non_power_of_two(n):
    cfg = GFusionConfig(volumeSize=(n,) * 3, volumeDimensions=(1.0,) * 3, storage=L.KF_STORAGE_F16U16,
                        quirks=L.KF_QUIRKS_TRACKING)
    g, o = both(cfg, sphere_raw(n, L.KF_STORAGE_F16U16))
    for method in (L.KF_MC_HISTOPYRAMID, L.KF_MC_SCAN):
        compare(g, o, method)


def test_fused_volume_bit_exact(tmp_path):
    """A TSDF fused from synthetic frames (oracle), extracted on both sides."""
    w = small_workload(4, size=128)
    o = O.Oracle(w.config, w.intrinsics)
    o.Reset(w.poses[0])
    for k in range(4):
        o.setPose(w.poses[k])
        o.depthToVertex(w.frame(k))
        o.integrate()
    g = GFusion(w.config, w.intrinsics)
    g.setVolumeRaw(o.getVolumeRaw())
    for method in (L.KF_MC_HISTOPYRAMID, L.KF_MC_SCAN):
        m, n = compare(g, o, method)
        assert n > 100
    # exports: same record layout and counts as the oracle's writers
    m.exportMesh(str(tmp_path / "g.stl"))
    o.exportMesh(str(tmp_path / "o.stl"))
    bg, bo = (tmp_path / "g.stl").read_bytes(), (tmp_path / "o.stl").read_bytes()
    assert len(bg) == len(bo) and bg[:84] == bo[:84]
    m.exportPointCloud(str(tmp_path / "g.ply"))
    assert (tmp_path / "g.ply").read_text().splitlines()[2] == f"element vertex {3 * n}"


def test_extract_after_frames_through_the_frame_step():
    w = small_workload(6, size=96)
    g = GFusion(w.config, w.intrinsics)
    g.Reset(w.poses[0])
    for k in range(6):
        g.frameStep(w.frame(k))
    o = O.Oracle(w.config, w.intrinsics)
    o.setVolumeRaw(g.getVolumeRaw())
    compare(g, o, L.KF_MC_HISTOPYRAMID)


def test_prefix_sum_device():
    import torch
    lib = L.load()
    rng = np.random.default_rng(7)
    for n in [0, 1, 4095, 4096, 4097, 123457, 4096 * 4096 + 5]:
        a = rng.integers(0, 7, n, dtype=np.uint32)
        d_in = torch.from_numpy(a.view(np.int32)).cuda()
        d_out = torch.empty_like(d_in)
        tot = C.c_uint32()
        st = lib.kf_prefix_sum_u32(C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), n, C.byref(tot), None)
        assert st == L.KF_OK
        out = d_out.cpu().numpy().view(np.uint32)
        ref, rtot = O.prefix_sum(a)
        np.testing.assert_array_equal(out, ref)
        assert tot.value == rtot
    # uint32 wrap-around, like GLSL uint
    a = np.full(5000, 2 ** 31 + 3, np.uint32)
    d_in = torch.from_numpy(a.view(np.int32)).cuda()
    d_out = torch.empty_like(d_in)
    tot = C.c_uint32()
    assert lib.kf_prefix_sum_u32(C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), a.size, C.byref(tot), None) == 0
    ref, rtot = O.prefix_sum(a)
    np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint32), ref)
    assert tot.value == rtot
