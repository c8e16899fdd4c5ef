"""Known-answer tests that pin the FP64 oracle (CPU only).

The reference ships no tests or golden vectors and cannot run here (OpenGL compute), so
the oracle is pinned by closed-form cases of each shader, by the marching-cubes table
facts, and by the math helpers against independent numpy/scipy implementations.
"""
import numpy as np
import pytest
import scipy.linalg

import kf_oracle as O
from oglfusionkinectv2_b200 import GFusionConfig, Intrinsics, _lib as L

INTR = Intrinsics()


def cfg(size=64, dim=1.0, mu=0.05, storage=L.KF_STORAGE_F32F32, quirks=L.KF_QUIRKS_DEFAULT, **kw):
    return GFusionConfig(volumeSize=(size,) * 3, volumeDimensions=(dim,) * 3, mu=mu,
                         storage=storage, quirks=quirks, **kw)


def plane_depth(mm):
    return np.full((INTR.height, INTR.width), mm, np.uint16)


# ---- math helpers ---------------------------------------------------------------------
def test_euler_xyz_is_rx_ry_rz():
    a = [0.3, -0.2, 0.7]
    Rx = np.array([[1, 0, 0], [0, np.cos(a[0]), -np.sin(a[0])], [0, np.sin(a[0]), np.cos(a[0])]])
    Ry = np.array([[np.cos(a[1]), 0, np.sin(a[1])], [0, 1, 0], [-np.sin(a[1]), 0, np.cos(a[1])]])
    Rz = np.array([[np.cos(a[2]), -np.sin(a[2]), 0], [np.sin(a[2]), np.cos(a[2]), 0], [0, 0, 1]])
    np.testing.assert_allclose(O.euler_xyz(a), Rx @ Ry @ Rz, atol=1e-15)
    w = np.array([1e-4, -2e-4, 3e-4])  # small angles: I + [w]x
    W = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]])
    np.testing.assert_allclose(O.euler_xyz(w), np.eye(3) + W, atol=1e-7)


@pytest.mark.parametrize("xi", [[0.1, -0.2, 0.3, 0.5, -0.1, 0.2], [1e-8, 0, -1e-8, 1e-3, 0, 0],
                                [0, 0, 0, 0.2, 0.3, 0.4]])
def test_se3_exp_matches_matrix_exponential(xi):
    M = np.zeros((4, 4))
    w, v = xi[:3], xi[3:]
    M[:3, :3] = [[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]]  # Twist, gFusion.cpp:826
    M[:3, 3] = v
    np.testing.assert_allclose(O.se3_exp(xi), scipy.linalg.expm(M), atol=1e-12)


def test_solvers():
    rng = np.random.default_rng(1)
    A = rng.standard_normal((40, 6))
    C = A.T @ A
    b = rng.standard_normal(6)
    x, rank = O.solve_pinv6(C, b)
    assert rank == 6
    np.testing.assert_allclose(x, np.linalg.solve(C, b), rtol=1e-9)
    np.testing.assert_allclose(O.solve_ldlt6(C, b), np.linalg.solve(C, b), rtol=1e-9)
    # rank-deficient: minimum-norm least squares like JacobiSVD::solve
    A2 = A.copy()
    A2[:, 5] = A2[:, 4]
    C2 = A2.T @ A2
    x2, rank2 = O.solve_pinv6(C2, b)
    assert rank2 == 5
    np.testing.assert_allclose(x2, np.linalg.pinv(C2) @ b, rtol=1e-7, atol=1e-9)
    x0, r0 = O.solve_pinv6(np.zeros((6, 6)), b)
    assert r0 == 0 and np.all(x0 == 0)


def test_icp_rank_guard_solve():
    """The ICP step's rank guard: eigen-directions below 1e-5 of the largest eigenvalue
    are dropped, the step is the minimum-norm solution over the rest (JacobiSVD::solve's
    rule with a higher cut)."""
    rng = np.random.default_rng(3)
    A = rng.standard_normal((50, 6)) * np.array([1, 1, 1, 3, 3, 3])
    C = A.T @ A
    b = rng.standard_normal(6)
    x, kept = O.solve_icp_guarded6(C, b)
    assert kept == 6
    np.testing.assert_allclose(x, np.linalg.solve(C, b), rtol=1e-9)
    # rank 3 (a plane: J = [n, p x n] with one normal) plus rounding-size noise
    n = np.array([0.0, -1.0, 0.0])
    P = rng.uniform(-1, 1, (200, 3)) * [1, 0, 1] + [1.0, 1.3, 2.0]
    J = np.hstack([np.tile(n, (200, 1)), np.cross(P, n)])
    Cp = J.T @ J + 1e-13 * np.eye(6)
    bp = J.T @ rng.standard_normal(200)
    xp, kept = O.solve_icp_guarded6(Cp, bp)
    assert kept == 3
    lam, V = np.linalg.eigh(Cp)
    keep = lam >= 1e-5 * lam[-1]
    expect = V[:, keep] @ ((V[:, keep].T @ bp) / lam[keep])
    np.testing.assert_allclose(xp, expect, rtol=1e-7, atol=1e-12)
    # the unobservable directions get no motion: in-plane translation, rotation about n
    assert abs(xp[0]) < 1e-9 and abs(xp[2]) < 1e-9 and abs(xp[4]) < 1e-9
    x0, k0 = O.solve_icp_guarded6(np.zeros((6, 6)), b)
    assert k0 == 0 and np.all(x0 == 0)


def test_prefix_sum_matches_cumsum_and_wraps():
    rng = np.random.default_rng(2)
    for n in [0, 1, 2047, 2048, 2049, 100000]:
        a = rng.integers(0, 16, n, dtype=np.uint32)
        out, tot = O.prefix_sum(a)
        ref = np.concatenate([[0], np.cumsum(a, dtype=np.uint64)[:-1]]).astype(np.uint32) if n else a
        np.testing.assert_array_equal(out, ref)
        assert tot == int(a.sum(dtype=np.uint64)) % 2 ** 32
    big = np.full(3, 2 ** 31, np.uint32)
    out, tot = O.prefix_sum(big)
    assert list(out) == [0, 2 ** 31, 0] and tot == 2 ** 31


def test_mc_tables_consistency():
    """tables.h facts: numVerts == 3 * nrOfTriangles, triTable rows use exactly the cut
    edges of edgeTable, sum(nrOfTriangles) == 820, offsets3 edges join adjacent corners."""
    edge, tri, nv, nt, off = O.mc_tables()
    assert int(nt.sum()) == 820
    np.testing.assert_array_equal(nv, 3 * nt)
    for c in range(256):
        row = tri[c]
        n = int(nv[c])
        assert np.all(row[n:] == -1) and np.all((row[:n] >= 0) & (row[:n] < 12))
        mask = 0
        for e in row[:n]:
            mask |= 1 << int(e)
        assert mask == edge[c]
    d = np.abs(off[:, :3].astype(int) - off[:, 3:].astype(int)).sum(1)
    assert np.all(d == 1)


# ---- pyramid (depthToVert.cs / vertToNorm.cs / glGenerateMipmap) ----------------------
def test_pyramid_plane_known_answer():
    o = O.Oracle(cfg(), INTR)
    d = plane_depth(1500)
    o.depthToVertex(d)
    o.vertexToNormal()
    for l in range(3):
        w, h = INTR.width >> l, INTR.height >> l
        s = float(1 << l)
        V = o.getVertexMap(l)
        u, v = np.meshgrid(np.arange(w), np.arange(h))
        np.testing.assert_allclose(V[..., 2], 1.5)
        np.testing.assert_allclose(V[..., 0], 1.5 * (u - INTR.cx / s) / (INTR.fx / s), atol=1e-12)
        np.testing.assert_allclose(V[..., 1], 1.5 * (v - INTR.cy / s) / (INTR.fy / s), atol=1e-12)
        N = o.getNormalMap(l)
        # column 0 and row 0 are invalid (uint underflow, vertToNorm.cs:23-26)
        assert np.all(N[0, :, 0] == 2) and np.all(N[:, 0, 0] == 2)
        np.testing.assert_allclose(N[1:, 1:, :3], np.broadcast_to([0, 0, -1.0], N[1:, 1:, :3].shape), atol=1e-12)
        assert np.all(N[1:, 1:, 3] == 1)


def test_pyramid_mip_is_box_mean_with_zeros():
    rng = np.random.default_rng(3)
    d = rng.integers(0, 3000, (INTR.height, INTR.width)).astype(np.uint16)
    d[rng.random(d.shape) < 0.3] = 0
    o = O.Oracle(cfg(), INTR)
    o.depthToVertex(d)
    l1 = d.astype(np.float64).reshape(212, 2, 256, 2).mean((1, 3))
    l2 = l1.reshape(106, 2, 128, 2).mean((1, 3))
    np.testing.assert_allclose(o.getDepthImage(1), l1)
    np.testing.assert_allclose(o.getDepthImage(2), l2)


def test_normal_down_neighbour_quirk():
    """Q3: the 'down' neighbour is read from column x-1 (vertToNorm.cs:26)."""
    d = plane_depth(1500)
    d[51, 100] = 0
    for quirks, q3 in [(L.KF_QUIRKS_DEFAULT, True), (L.KF_QUIRKS_DEFAULT & ~L.KF_Q3_DOWN_FROM_LEFT, False)]:
        o = O.Oracle(cfg(quirks=quirks), INTR)
        o.depthToVertex(d)
        o.vertexToNormal()
        N = o.getNormalMap(0)
        assert (N[50, 101, 0] == 2) == q3
        assert (N[50, 100, 0] == 2) == (not q3)


# ---- integrate (integrate.cs) ----------------------------------------------------------
@pytest.mark.parametrize("band", [True, False])
def test_integrate_frontoparallel_plane(band):
    """Identity pose, plane at z = 0.6 m: every voxel column along the optical axis gets
    the closed-form running average of its first observation."""
    q = L.KF_QUIRKS_DEFAULT if band else L.KF_QUIRKS_TRACKING
    c = cfg(size=64, dim=1.0, mu=0.05, quirks=q)
    o = O.Oracle(c, INTR)
    o.Reset(np.eye(4))
    d = plane_depth(600)
    o.depthToVertex(d)
    o.integrate()
    F, W = o.getVolume()
    vs = 1.0 / 64
    for (x, y) in [(1, 1), (5, 3), (0, 0)]:
        for z in range(64):
            pz = (z + 0.5) * vs
            px, py = (x + 0.5) * vs, (y + 0.5) * vs
            u = INTR.fx * px / pz + INTR.cx + 0.5
            v = INTR.fy * py / pz + INTR.cy + 0.5
            if pz < 1e-4 or u > 511 or v > 423:
                assert W[z, y, x] == 0 and F[z, y, x] == 0
                continue
            diff = (0.6 - pz) * np.sqrt(1 + (px / pz) ** 2 + (py / pz) ** 2)
            if diff <= -c.mu:
                ef, ew = 0.0, 0.0
            else:
                sdf = min(1.0, diff / c.mu)
                if not band:
                    ef, ew = max(-1.0, min(1.0, sdf)), 1.0
                elif sdf < 0.2:
                    ef, ew = max(-0.1, min(0.2, sdf)), 1.0
                else:
                    ef, ew = 0.0, 0.0
            assert W[z, y, x] == ew, (x, y, z)
            assert abs(F[z, y, x] - ef) < 1e-6, (x, y, z, F[z, y, x], ef)


@pytest.mark.parametrize("storage", [L.KF_STORAGE_F32F32, L.KF_STORAGE_F16U16, L.KF_STORAGE_RG16I])
def test_integrate_storage_quantisation(storage):
    """RG16I stores int(F*32766) (integrate.cs:48); F16 rounds to nearest half."""
    c = cfg(size=32, dim=1.0, mu=0.05, storage=storage, quirks=L.KF_QUIRKS_TRACKING)
    o = O.Oracle(c, INTR)
    o.Reset(np.eye(4))
    o.depthToVertex(plane_depth(600))
    o.integrate()
    raw = o.getVolumeRaw()
    n = 32 ** 3
    if storage == L.KF_STORAGE_RG16I:
        q = raw[:2 * n].view(np.int16)
        assert q.min() >= -32766 and q.max() <= 32766 and np.any(q != 0)
    elif storage == L.KF_STORAGE_F16U16:
        h = raw[:2 * n].view(np.float16)
        assert np.all(np.isfinite(h)) and np.any(h != 0)
    F, W = o.getVolume()
    ref = O.Oracle(cfg(size=32, dim=1.0, mu=0.05, quirks=L.KF_QUIRKS_TRACKING), INTR)
    ref.Reset(np.eye(4))
    ref.depthToVertex(plane_depth(600))
    ref.integrate()
    F32, W32 = ref.getVolume()
    np.testing.assert_array_equal(W, W32)
    assert np.max(np.abs(F - F32)) <= 1.0 / 32766 + 5e-4


# ---- raycast (raycast.cs) ---------------------------------------------------------------
def test_raycast_plane_hit_depth():
    c = cfg(size=128, dim=1.0, mu=0.05, quirks=L.KF_QUIRKS_TRACKING)
    o = O.Oracle(c, INTR)
    pose = np.eye(4)
    pose[:3, 3] = [0.5, 0.5, -0.2]
    o.Reset(pose)
    o.depthToVertex(plane_depth(700))  # plane at world z = 0.5
    o.integrate()
    o.raycast()
    V = o.getVerts()
    N = o.getNorms()
    hit = V[..., 3] > 0
    assert hit.mean() > 0.2
    # away from the volume's side faces and the image border, where border-clamped taps or
    # never-observed (zero) voxels enter the trilinear footprint
    inner = hit & np.all((V[..., :2] > 0.05) & (V[..., :2] < 0.95), axis=-1)
    inner[:8] = inner[-8:] = False
    inner[:, :8] = inner[:, -8:] = False
    assert inner.sum() > 0.5 * hit.sum()
    assert np.max(np.abs(V[inner][:, 2] - 0.5)) < 0.5e-3
    # the gradient footprint (+-2 voxels) reaches unobserved voxels slightly more often
    nz = np.abs(N[inner][:, 2] + 1)
    assert np.mean(nz < 1e-6) > 0.97 and nz.max() < 2e-3


# ---- depth ingest: libfreenect2 undistortion and filter3D.cs ----------------------------
IR = (365.1, 364.7, 255.3, 208.9, 0.092, -0.27, 0.094, 0.0012, -0.0006)


def _undistort_map_float32(ir, W, H):
    """libfreenect2 Registration's map in numpy float32 (IEEE single, no fused multiply-add),
    the same expressions in the same order."""
    f = np.float32
    fx, fy, cx, cy, k1, k2, k3, p1, p2 = [f(v) for v in ir]
    ys, xs = np.mgrid[0:H, 0:W]
    dx = (xs.astype(f) - cx) / fx
    dy = (ys.astype(f) - cy) / fy
    dx2, dy2 = dx * dx, dy * dy
    r2 = dx2 + dy2
    dxdy2 = f(2) * dx * dy
    kr = f(1) + ((k3 * r2 + k2) * r2 + k1) * r2
    mx = fx * (dx * kr + p2 * (r2 + f(2) * dx2) + p1 * dxdy2) + cx
    my = fy * (dy * kr + p1 * (r2 + f(2) * dy2) + p2 * dxdy2) + cy
    vx, vy = mx + f(0.5), my + f(0.5)
    ok = (vx > -1) & (vx < W) & (vy > -1) & (vy < H)
    idx = np.trunc(vy).astype(np.int64) * W + np.trunc(vx).astype(np.int64)
    return np.where(ok, idx, -1).astype(np.int32)


@pytest.mark.parametrize("ir", [IR, (365.0, 365.0, 256.0, 212.0, 0, 0, 0, 0, 0),
                                (360.0, 361.0, 250.0, 205.0, 0.6, -2.0, 4.0, 0.02, -0.03)])
def test_undistortion_map_matches_float32_model(ir):
    o = O.Oracle(cfg(size=16), INTR)
    o.setDepthUndistortion(ir)
    m = o.getUndistortionMap()
    np.testing.assert_array_equal(m, _undistort_map_float32(ir, INTR.width, INTR.height))
    if ir[4:] == (0, 0, 0, 0, 0) and ir[:4] == (INTR.fx, INTR.fy, INTR.cx, INTR.cy):
        np.testing.assert_array_equal(m.ravel(), np.arange(m.size))  # no distortion: identity
    assert (m >= 0).mean() > 0.5


def test_undistortion_gathers_raw_depth():
    o = O.Oracle(cfg(size=16), INTR)
    raw = (np.arange(INTR.width * INTR.height) % 3000 + 500).astype(np.uint16).reshape(INTR.height, INTR.width)
    o.setDepthUndistortion(IR)
    o.depthToVertex(raw)
    m = o.getUndistortionMap()
    want = np.where(m >= 0, raw.ravel()[np.maximum(m, 0)], 0).reshape(raw.shape)
    np.testing.assert_array_equal(o.getDepthImage(0), want)
    o.setDepthUndistortion(None)
    o.depthToVertex(raw)
    np.testing.assert_array_equal(o.getDepthImage(0), raw)


def test_filter3d_known_answers():
    o = O.Oracle(cfg(size=16), INTR)
    o.setDepthFilter(True)
    H, W = INTR.height, INTR.width
    d = np.full((H, W), 1000, np.uint16)
    d[100, 100] = 1010          # 8.9 mm above its neighbourhood mean (1001.1): removed
    d[200, 200] = 1004          # 3.6 mm above its neighbourhood mean (1000.4): kept
    d[300, 301:304] = 0         # a run of three invalid depths
    d[50, 50] = 4000            # out of range (checkPixel keeps 5 < d < 4000): invalid
    o.depthToVertex(d)
    f = o.getDepthImage(0)
    # borders (x < 2, x > W-2, y < 2, y > H-2) are never written
    assert np.all(f[:2] == 0) and np.all(f[-1] == 0) and np.all(f[:, :2] == 0) and np.all(f[:, -1] == 0)
    assert f[2, 2] == 1000 and f[H - 2, W - 2] == 1000
    assert f[100, 100] == 0 and f[100, 101] == 1000
    assert f[200, 200] == 1004
    assert f[299, 302] == 0      # its 3x3 holds all three zeros: 6 valid, not more than 6
    assert f[301, 302] == 0      # the same three zeros
    assert f[299, 301] == 1000   # two of them: 7 valid, kept
    assert f[300, 301] == 0      # an invalid depth itself is never kept
    assert f[50, 50] == 0 and f[50, 51] == 1000


# ---- intensityProjection (mip.cs) -----------------------------------------------------
def _mip_sample_counts(c, pose, ls):
    """Samples tnear + k * ls < tfar per pixel, from the slab test of mip.cs:61-77."""
    fx, fy, cx, cy = INTR.fx, INTR.fy, INTR.cx, INTR.cy
    ys, xs = np.mgrid[0:INTR.height, 0:INTR.width].astype(np.float64)
    d_cam = np.stack([(xs - cx) / fx, (ys - cy) / fy, np.ones_like(xs)], -1)
    d = d_cam @ pose[:3, :3].T
    o = pose[:3, 3]
    dim = np.array(c.volumeDimensions, np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / d
        tb = -inv * o
        tt = inv * (dim - o)
    tmin, tmax = np.minimum(tt, tb), np.maximum(tt, tb)
    tnear = np.maximum(tmin.max(-1), c.nearPlane)
    tfar = np.minimum(tmax.min(-1), c.farPlane)
    r = (tfar - tnear) / ls
    n = np.where(tnear < tfar, np.ceil(r), 0)
    # where the ratio sits on an integer, rounding decides whether the last sample is in
    on_step = (tnear < tfar) & (np.abs(r - np.rint(r)) < 1e-9)
    return n, on_step


@pytest.mark.parametrize("value", [0.5, -0.25])
def test_intensity_projection_constant_volume(value):
    """A constant TSDF c makes every trilinear sample c, so each pixel's sum is c times
    its sample count when c > 0 and 0 otherwise; y = z = 0 and w = 1 everywhere."""
    c = cfg(size=32, dim=1.0, mu=0.05)
    o = O.Oracle(c, INTR)
    pose = np.eye(4)
    pose[:3, 3] = [0.5, 0.5, -0.2]
    o.Reset(pose)
    n = 32 ** 3
    raw = np.concatenate([np.full(n, value, np.float32), np.ones(n, np.float32)])
    o.setVolumeRaw(raw.view(np.uint8))
    m = o.intensityProjection()
    counts, on_step = _mip_sample_counts(c, pose, 0.75 * c.mu)
    assert (counts > 0).mean() > 0.3 and on_step.mean() < 0.01
    want = counts * value if value > 0 else np.zeros_like(counts)
    err = np.abs(m[..., 0] - want)
    assert np.all(err[~on_step] <= 1e-9 * np.maximum(1.0, np.abs(want[~on_step])))
    assert np.all(err[on_step] <= abs(value) + 1e-9)
    assert np.all(m[..., 1] == 0) and np.all(m[..., 2] == 0) and np.all(m[..., 3] == 1)
    # the central ray enters at z = 0 (t = 0.2) and leaves at z = 1 (t = 1.2)
    if value > 0:
        cy, cx = int(INTR.cy), int(INTR.cx)
        assert counts[cy, cx] == np.ceil(1.0 / (0.75 * c.mu))


def test_intensity_projection_rg16i_scale():
    """On the reference's RG16I volume a stored short s reads as s * 0.00003051944088
    (mip.cs:39-49, 1/32766): a constant short of 16383 sums to 16383/32766 per sample."""
    c = cfg(size=32, dim=1.0, mu=0.05, storage=L.KF_STORAGE_RG16I)
    o = O.Oracle(c, INTR)
    pose = np.eye(4)
    pose[:3, 3] = [0.5, 0.5, -0.2]
    o.Reset(pose)
    n = 32 ** 3
    raw = np.concatenate([np.full(n, 16383, np.int16), np.ones(n, np.int16)])
    o.setVolumeRaw(raw.view(np.uint8))
    m = o.intensityProjection()
    counts, on_step = _mip_sample_counts(c, pose, 0.75 * c.mu)
    want = counts * 16383 * 0.00003051944088
    err = np.abs(m[..., 0] - want)
    assert (counts > 0).mean() > 0.3
    assert np.all(err[~on_step] <= 1e-6 * np.maximum(1.0, want[~on_step]))


# ---- ICP (track.cs / reduce.cs / Track) ---------------------------------------------
def test_icp_recovers_small_motion_on_same_frame():
    from oglfusionkinectv2_b200 import synth
    w = synth.plain_c1(2)
    o = O.Oracle(w.config, w.intrinsics)
    T = w.poses[0]
    o.Reset(T)
    f = w.frame(0)
    o.depthToVertex(f)
    o.vertexToNormal()
    o.integrate()
    o.raycast()
    a = np.deg2rad(0.3)
    D = np.eye(4)
    D[:3, :3] = [[np.cos(a), 0, np.sin(a)], [0, 1, 0], [-np.sin(a), 0, np.cos(a)]]
    D[:3, 3] = [0.006, -0.004, 0.005]
    o.setPose(D @ T)
    assert o.Track()
    dt = np.linalg.norm(o.getPose()[:3, 3] - T[:3, 3])
    assert dt < 1e-3
    # the reduction counts every pixel of the finest level (reduce.cs:209-263)
    assert o.getReduction()[28] == 512 * 424


def test_icp_q1_counts_group_seven_rows():
    from oglfusionkinectv2_b200 import synth
    w = synth.plain_c1(1)
    w.config.quirks |= L.KF_Q1_LAST_GROUP_ONLY
    o = O.Oracle(w.config, w.intrinsics)
    o.Reset(w.poses[0])
    o.depthToVertex(w.frame(0))
    o.vertexToNormal()
    o.integrate()
    o.raycast()
    s = o.icpReduceOnce(0)
    assert s[28] == 512 * 53


# ---- marching cubes (histoPyramids.cs / traverseHistoPyramids.cs / marchingCubes.cs) ---
def sphere_volume(n=64, r=0.3, storage=L.KF_STORAGE_F32F32, quirks=L.KF_QUIRKS_TRACKING):
    c = cfg(size=n, dim=1.0, storage=storage, quirks=quirks)
    o = O.Oracle(c, INTR)
    vs = 1.0 / n
    g = (np.arange(n) + 0.5) * vs
    Z, Y, X = np.meshgrid(g, g, g, indexing="ij")
    sd = np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2 + (Z - 0.5) ** 2) - r
    F = np.clip(sd / 0.05, -1, 1).astype(np.float32)
    if storage == L.KF_STORAGE_F32F32:
        raw = np.concatenate([F.ravel(), np.ones(n ** 3, np.float32)]).view(np.uint8)
    elif storage == L.KF_STORAGE_RG16I:
        raw = np.concatenate([(F.ravel() * 32766).astype(np.int32).astype(np.int16),
                              np.ones(n ** 3, np.int16)]).view(np.uint8)
    else:
        raw = np.concatenate([F.ravel().astype(np.float16).view(np.uint16),
                              np.ones(n ** 3, np.uint16)]).view(np.uint8)
    o.setVolumeRaw(raw)
    return o, c, r


@pytest.mark.parametrize("method", [L.KF_MC_HISTOPYRAMID, L.KF_MC_SCAN])
def test_mc_sphere_on_surface(method):
    o, c, r = sphere_volume()
    n = o.mcExtract(0.0, method)
    assert n > 500
    V = o.mcVertices()
    p = (V[:, :3].astype(np.float64) + 0.5) / 64  # voxel index -> metres
    dist = np.abs(np.linalg.norm(p - 0.5, axis=1) - r)
    assert dist.max() < 0.5 / 64


def test_mc_histopyramid_matches_direct_count():
    """The histoPyramid total equals the sum of per-cube nrOfTriangles of the base level,
    and traversal emits each cube's triangles exactly once."""
    o, c, r = sphere_volume()
    n = o.mcExtract(0.0, L.KF_MC_HISTOPYRAMID)
    base = o.mcBaseLevel()
    assert n == int((base & 0xFFFF).sum())
    V = o.mcVertices().reshape(-1, 3, 4)
    cubes = np.floor(V[:, :, :3].min(1) + 1e-6).astype(int)  # min corner of each triangle
    counts = np.zeros(base.shape, np.int64)
    np.add.at(counts, (cubes[:, 2], cubes[:, 1], cubes[:, 0]), 1)
    np.testing.assert_array_equal(counts, (base & 0xFFFF).astype(np.int64))


def test_mc_non_pow2_padding():
    o, c, r = sphere_volume(n=48, r=0.3)
    n = o.mcExtract(0.0, L.KF_MC_HISTOPYRAMID)
    assert n == int((o.mcBaseLevel() & 0xFFFF).sum()) and n > 0


def test_mc_border_quirk():
    o, c, r = sphere_volume(n=64, r=0.45)  # surface reaches the 10-voxel border band
    n_q = o.mcExtract(0.0, L.KF_MC_HISTOPYRAMID)
    base = o.mcBaseLevel()
    assert np.all(base[:11] == 0) and np.all(base[:, :, 54:] == 0)
    o2, c2, _ = sphere_volume(n=64, r=0.45, quirks=L.KF_QUIRKS_TRACKING & ~L.KF_Q15_MC_BORDER_SKIP)
    assert o2.mcExtract(0.0, L.KF_MC_HISTOPYRAMID) > n_q


def test_stl_and_ply_export(tmp_path):
    o, c, r = sphere_volume(n=32, r=0.3)
    n = o.mcExtract(0.0, L.KF_MC_HISTOPYRAMID)
    stl = tmp_path / "m.stl"
    o.exportMesh(str(stl))
    b = stl.read_bytes()
    assert len(b) == 84 + 50 * n
    assert int.from_bytes(b[80:84], "little") == n
    rec = np.frombuffer(b[84:84 + 50 * n], dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", 9), ("a", "<u2")]))
    np.testing.assert_array_equal(rec["n"], 1.0)
    np.testing.assert_array_equal(rec["v"].reshape(-1, 3), o.mcVertices()[:, :3])
    ply = tmp_path / "m.ply"
    o.exportPointCloud(str(ply))
    lines = ply.read_text().splitlines()
    assert lines[0] == "ply" and lines[2] == f"element vertex {3 * n}"
    assert len(lines) == 7 + 3 * n


def test_welded_mesh_of_a_sphere():
    """The oracle's welded mesh of an analytic sphere TSDF: a closed surface (V - E + F = 2)
    with the classic path's triangle count, vertices on the sphere, unit normals pointing
    out, facets wound counter-clockwise from outside."""
    from oglfusionkinectv2_b200 import GFusionConfig, Intrinsics, _lib as L
    n = 40
    g = (np.arange(n) + 0.5) / n
    Z, Y, X = np.meshgrid(g, g, g, indexing="ij")
    sd = np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2 + (Z - 0.5) ** 2) - 0.3
    F = np.clip(sd / 0.05, -1, 1).astype(np.float32).ravel()
    raw = np.concatenate([F, np.ones(n ** 3, np.float32)]).view(np.uint8)
    cfg = GFusionConfig(volumeSize=(n,) * 3, volumeDimensions=(1.0,) * 3, storage=L.KF_STORAGE_F32F32,
                        quirks=L.KF_QUIRKS_TRACKING & ~(L.KF_Q13_MC_FIRST_SEVEN | L.KF_Q15_MC_BORDER_SKIP))
    o = O.Oracle(cfg, Intrinsics())
    o.setVolumeRaw(raw)
    P, N, I = o.mcMesh(0.0)
    E = np.unique(np.sort(np.concatenate([I[:, [0, 1]], I[:, [1, 2]], I[:, [2, 0]]]), axis=1), axis=0)
    assert len(P) - len(E) + len(I) == 2
    assert o.mcExtract(0.0, L.KF_MC_SCAN) == len(I)
    c = np.array([0.5, 0.5, 0.5])
    r = np.linalg.norm(P - c, axis=1)
    assert np.abs(r - 0.3).max() < 2e-3
    np.testing.assert_allclose(np.linalg.norm(N, axis=1), 1.0, rtol=1e-5)
    assert np.mean(np.sum(N * (P - c), axis=1) > 0) == 1.0
    fn = np.cross(P[I[:, 1]] - P[I[:, 0]], P[I[:, 2]] - P[I[:, 0]])
    assert np.mean(np.sum(fn * (P[I].mean(axis=1) - c), axis=1) > 0) == 1.0
