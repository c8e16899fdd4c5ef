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


@pytest.mark.parametrize("storage", [L.KF_STORAGE_F32F32, L.KF_STORAGE_F16U16, L.KF_STORAGE_RG16I])
@pytest.mark.parametrize("method", [L.KF_MC_HISTOPYRAMID, L.KF_MC_SCAN])
def test_face_normals_match_oracle(storage, method):
    """calcNormal (marchingCubes.cs:87-93) per vertex: cross(v1 - v0, v2 - v0) of its
    triangle, w = 0, for both extraction paths."""
    cfg = GFusionConfig(volumeSize=(64,) * 3, volumeDimensions=(1.0,) * 3, storage=storage,
                        quirks=L.KF_QUIRKS_TRACKING & ~(L.KF_Q13_MC_FIRST_SEVEN | L.KF_Q15_MC_BORDER_SKIP))
    g, o = both(cfg, sphere_raw(64, storage))
    m, ng = compare(g, o, method)
    assert ng > 1000
    Ng, No = m.getNormals(), o.mcNormals()
    assert (Ng[:, 3] == 0).all()
    scale = np.linalg.norm(No[:, :3], axis=1).max()
    assert np.max(np.abs(Ng - No)) <= 1e-4 * scale + 1e-6


@pytest.mark.parametrize("storage", [L.KF_STORAGE_F32F32, L.KF_STORAGE_RG16I])
def test_scan_path_shader_units(storage):
    """Q24: the scan path writes marchingCubes.cs's output convention: corners at
    -1 + gridPos * voxelSize, vertex / 128 * voxelSize.x with z negated, w = 1, normals in
    the unscaled shader units (voxelSize = 1000 * dim / size)."""
    q = (L.KF_QUIRKS_TRACKING & ~(L.KF_Q13_MC_FIRST_SEVEN | L.KF_Q15_MC_BORDER_SKIP)) | L.KF_Q24_MC_SHADER_UNITS
    cfg = GFusionConfig(volumeSize=(64,) * 3, volumeDimensions=(1.0,) * 3, storage=storage, quirks=q)
    g, o = both(cfg, sphere_raw(64, storage))
    m = MCubes(g)
    ng = m.generateMarchingCubes(L.KF_MC_SCAN)
    assert ng == o.mcExtract(0.0, L.KF_MC_SCAN) > 1000
    Vg, Vo = m.getVertices(), o.mcVertices()
    assert (Vg[:, 3] == 1).all()
    assert np.max(np.abs(Vg - Vo)) <= 1e-5 * np.abs(Vo).max()
    vs = 1000.0 / 64
    # the same triangles as voxel-index output, mapped by the shader's formula
    cfg2 = GFusionConfig(volumeSize=(64,) * 3, volumeDimensions=(1.0,) * 3, storage=storage,
                         quirks=q & ~L.KF_Q24_MC_SHADER_UNITS)
    g2 = GFusion(cfg2, INTR)
    g2.setVolumeRaw(sphere_raw(64, storage))
    m2 = MCubes(g2)
    assert m2.generateMarchingCubes(L.KF_MC_SCAN) == ng
    Vi = m2.getVertices()[:, :3].astype(np.float64)
    expect = (-1.0 + Vi * vs) / 128.0 * vs * np.array([1.0, 1.0, -1.0])
    assert np.max(np.abs(Vg[:, :3] - expect)) <= 1e-4 * np.abs(expect).max()
    Ng, No = m.getNormals(), o.mcNormals()
    assert np.max(np.abs(Ng - No)) <= 1e-4 * np.linalg.norm(No[:, :3], axis=1).max()


@pytest.mark.parametrize("storage", [L.KF_STORAGE_F32F32, L.KF_STORAGE_F16U16, L.KF_STORAGE_RG16I])
def test_welded_mesh_matches_oracle(storage, tmp_path):
    """The welded mesh: vertex and triangle counts and every index bit-exact with the
    oracle, positions within 1e-6 m, unit normals within 1e-3; the exports carry it."""
    cfg = GFusionConfig(volumeSize=(64,) * 3, volumeDimensions=(1.0,) * 3, storage=storage,
                        quirks=L.KF_QUIRKS_TRACKING & ~(L.KF_Q13_MC_FIRST_SEVEN | L.KF_Q15_MC_BORDER_SKIP))
    g, o = both(cfg, sphere_raw(64, storage))
    m = MCubes(g)
    Pg, Ng, Ig = m.extractMesh()
    Po, No, Io = o.mcMesh(0.0)
    assert len(Pg) == len(Po) > 1000 and len(Ig) == len(Io)
    np.testing.assert_array_equal(Ig, Io)
    assert np.max(np.abs(Pg - Po)) <= 1e-6
    assert np.max(np.abs(Ng - No)) <= 1e-3
    # a closed surface: V - E + F = 2; as many triangles as the scan path's soup
    E = np.unique(np.sort(np.concatenate([Ig[:, [0, 1]], Ig[:, [1, 2]], Ig[:, [2, 0]]]), axis=1), axis=0)
    assert len(Pg) - len(E) + len(Ig) == 2
    assert m.generateMarchingCubes(L.KF_MC_SCAN) == len(Ig)
    # exports
    ply, stl = str(tmp_path / "m.ply"), str(tmp_path / "m.stl")
    m.exportWeldedMeshPly(ply)
    m.exportWeldedMeshStl(stl)
    raw = open(ply, "rb").read()
    head, body = raw.split(b"end_header\n", 1)
    assert f"element vertex {len(Pg)}".encode() in head and f"element face {len(Ig)}".encode() in head
    assert len(body) == len(Pg) * 24 + len(Ig) * 13
    V = np.frombuffer(body[:len(Pg) * 24], np.float32).reshape(-1, 6)
    np.testing.assert_array_equal(V[:, :3], Pg)
    s = open(stl, "rb").read()
    assert int.from_bytes(s[80:84], "little") == len(Ig) and len(s) == 84 + 50 * len(Ig)
    fn = np.frombuffer(s[84:], np.uint8).reshape(-1, 50)[:, :12].copy().view(np.float32)
    c = np.array([0.5, 0.5, 0.5])
    cen = Pg[Ig].mean(axis=1)
    assert np.mean(np.sum(fn * (cen - c), axis=1) > 0) > 0.999  # outward facets
