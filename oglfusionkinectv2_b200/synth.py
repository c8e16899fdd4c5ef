"""Seeded synthetic depth sequences (stand-in for the reference's live Kinect v2 input).

An FP64 analytic ray caster renders uint16 millimetre depth frames of simple scenes
(ground plane, spheres, boxes, room walls) along a camera trajectory, then applies the
Kinect-v2-like corruption the workloads call for: Gaussian depth noise with
sigma(z) = 0.0012 + 0.0019 (z - 0.4)^2 m, depths outside 0.5-4.5 m zeroed, seeded
dropouts, and (room scenes) flying pixels at depth edges.  Pixel (u, v) looks along
K^-1 (u, v, 1), the same convention the fusion code uses (depthToVert.cs:56).

World frame: the TSDF volume spans [0, dim]^3; +y points down (camera y is down).
Poses are camera-to-world 4x4 (row-major numpy).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .gfusion import GFusionConfig, Intrinsics
from . import _lib as L


def splitmix64(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return z ^ (z >> 31)


def look_at(pos, target) -> np.ndarray:
    """Camera-to-world pose at `pos` looking at `target`, camera y along world +y (down)."""
    pos = np.asarray(pos, np.float64)
    z = np.asarray(target, np.float64) - pos
    z /= np.linalg.norm(z)
    down = np.array([0.0, 1.0, 0.0])
    x = np.cross(down, z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    T = np.eye(4)
    T[:3, 0], T[:3, 1], T[:3, 2], T[:3, 3] = x, y, z, pos
    return T


@dataclass
class Scene:
    planes: list = field(default_factory=list)   # (normal, offset): n.x = d
    spheres: list = field(default_factory=list)  # (centre, radius)
    boxes: list = field(default_factory=list)    # (min, max)

    def raycast(self, origin: np.ndarray, dirs: np.ndarray) -> np.ndarray:
        """Smallest positive t along origin + t * dirs (dirs has camera z = 1, so t = depth)."""
        t = np.full(dirs.shape[0], np.inf)
        o = origin
        for n, d in self.planes:
            n = np.asarray(n, np.float64)
            den = dirs @ n
            with np.errstate(divide="ignore", invalid="ignore"):
                tt = (d - o @ n) / den
            tt[(den == 0) | ~(tt > 1e-6)] = np.inf
            t = np.minimum(t, tt)
        for c, r in self.spheres:
            oc = o - np.asarray(c, np.float64)
            a = np.einsum("ij,ij->i", dirs, dirs)
            b = 2.0 * (dirs @ oc)
            cc = oc @ oc - r * r
            disc = b * b - 4 * a * cc
            ok = disc >= 0
            sq = np.sqrt(np.where(ok, disc, 0.0))
            t0 = (-b - sq) / (2 * a)
            t1 = (-b + sq) / (2 * a)
            tt = np.where(t0 > 1e-6, t0, np.where(t1 > 1e-6, t1, np.inf))
            tt[~ok] = np.inf
            t = np.minimum(t, tt)
        for lo, hi in self.boxes:
            lo = np.asarray(lo, np.float64)
            hi = np.asarray(hi, np.float64)
            with np.errstate(divide="ignore", invalid="ignore"):
                inv = 1.0 / dirs
                ta = (lo - o) * inv
                tb = (hi - o) * inv
            tmin = np.nanmax(np.minimum(ta, tb), axis=1)
            tmax = np.nanmin(np.maximum(ta, tb), axis=1)
            hit = (tmax >= tmin) & (tmax > 1e-6)
            tt = np.where(tmin > 1e-6, tmin, tmax)
            tt[~hit] = np.inf
            t = np.minimum(t, tt)
        return t


@dataclass
class Workload:
    name: str
    config: GFusionConfig
    intrinsics: Intrinsics
    scene: Scene
    poses: list            # ground-truth camera-to-world per frame
    seed: int
    dropout: float = 0.02
    flying_pixels: bool = False
    mc_every: int = 0

    @property
    def n_frames(self) -> int:
        return len(self.poses)

    def pixel_rays(self) -> np.ndarray:
        k = self.intrinsics
        u, v = np.meshgrid(np.arange(k.width, dtype=np.float64), np.arange(k.height, dtype=np.float64))
        return np.stack([(u - k.cx) / k.fx, (v - k.cy) / k.fy, np.ones_like(u)], -1).reshape(-1, 3)

    def clean_depth(self, i: int) -> np.ndarray:
        """Noise-free depth in metres (inf for no hit), shape (H, W)."""
        T = self.poses[i]
        dirs = self.pixel_rays() @ T[:3, :3].T
        t = self.scene.raycast(T[:3, 3], dirs)
        return t.reshape(self.intrinsics.height, self.intrinsics.width)

    def frame(self, i: int) -> np.ndarray:
        """uint16 millimetre depth of frame i with the seeded corruption applied."""
        z = self.clean_depth(i)
        rng = np.random.Generator(np.random.PCG64(splitmix64(self.seed * 1000003 + i)))
        if self.flying_pixels:
            # mixed pixels at depth edges: blend with the far neighbour
            zf = np.where(np.isfinite(z), z, 10.0)
            right = np.roll(zf, -1, axis=1)
            edge = np.abs(right - zf) > 0.1
            mix = rng.random(z.shape)
            blend = zf * mix + right * (1 - mix)
            take = edge & (rng.random(z.shape) < 0.5)
            z = np.where(take, blend, z)
        sigma = 0.0012 + 0.0019 * (z - 0.4) ** 2
        with np.errstate(invalid="ignore"):
            zn = z + rng.standard_normal(z.shape) * np.where(np.isfinite(sigma), sigma, 0.0)
        valid = np.isfinite(zn) & (zn >= 0.5) & (zn <= 4.5)
        mm = np.where(valid, np.rint(zn * 1000.0), 0.0)
        drop = rng.random(z.shape) < self.dropout
        mm[drop] = 0
        return mm.astype(np.uint16)

    def frames(self, start: int = 0, stop: int | None = None):
        stop = self.n_frames if stop is None else stop
        for i in range(start, stop):
            yield self.frame(i)

    def frames_torch(self, indices, device="cuda"):
        """The same scene, trajectory and corruption model rendered with torch on `device`
        (FP64 rays, a torch generator seeded per frame): an int16 tensor (n, H, W) holding
        uint16 millimetres.  The noise draws differ from frame(); used where thousands of
        frames are needed (batched and served workloads)."""
        import torch
        k = self.intrinsics
        dev = torch.device(device)
        u = torch.arange(k.width, dtype=torch.float64, device=dev)
        v = torch.arange(k.height, dtype=torch.float64, device=dev)
        vv, uu = torch.meshgrid(v, u, indexing="ij")
        rays = torch.stack([(uu - k.cx) / k.fx, (vv - k.cy) / k.fy, torch.ones_like(uu)], -1).reshape(-1, 3)
        out = torch.empty((len(indices), k.height, k.width), dtype=torch.int16, device=dev)
        gen = torch.Generator(device=dev)
        for j, i in enumerate(indices):
            T = torch.as_tensor(self.poses[i], dtype=torch.float64, device=dev)
            dirs = rays @ T[:3, :3].T
            o = T[:3, 3]
            t = torch.full((dirs.shape[0],), float("inf"), dtype=torch.float64, device=dev)
            for n, d in self.scene.planes:
                nn = torch.as_tensor(n, dtype=torch.float64, device=dev)
                den = dirs @ nn
                tt = (d - o @ nn) / den
                tt = torch.where((den == 0) | ~(tt > 1e-6), torch.full_like(tt, float("inf")), tt)
                t = torch.minimum(t, tt)
            a = (dirs * dirs).sum(1)
            for c, r in self.scene.spheres:
                oc = o - torch.as_tensor(c, dtype=torch.float64, device=dev)
                b = 2.0 * (dirs @ oc)
                cc = oc @ oc - r * r
                disc = b * b - 4 * a * cc
                ok = disc >= 0
                sq = torch.sqrt(torch.clamp(disc, min=0.0))
                t0 = (-b - sq) / (2 * a)
                t1 = (-b + sq) / (2 * a)
                inf = torch.full_like(t0, float("inf"))
                tt = torch.where(t0 > 1e-6, t0, torch.where(t1 > 1e-6, t1, inf))
                t = torch.minimum(t, torch.where(ok, tt, inf))
            for lo, hi in self.scene.boxes:
                lo_t = torch.as_tensor(lo, dtype=torch.float64, device=dev)
                hi_t = torch.as_tensor(hi, dtype=torch.float64, device=dev)
                inv = 1.0 / dirs
                ta = (lo_t - o) * inv
                tb = (hi_t - o) * inv
                tmin = torch.nan_to_num(torch.minimum(ta, tb), nan=-float("inf")).amax(1)
                tmax = torch.nan_to_num(torch.maximum(ta, tb), nan=float("inf")).amin(1)
                hit = (tmax >= tmin) & (tmax > 1e-6)
                tt = torch.where(tmin > 1e-6, tmin, tmax)
                t = torch.minimum(t, torch.where(hit, tt, torch.full_like(tt, float("inf"))))
            z = t.reshape(k.height, k.width)
            gen.manual_seed(splitmix64(self.seed * 1000003 + i) & 0x7FFFFFFFFFFFFFFF)
            if self.flying_pixels:
                zf = torch.where(torch.isfinite(z), z, torch.full_like(z, 10.0))
                right = torch.roll(zf, -1, dims=1)
                edge = (right - zf).abs() > 0.1
                mix = torch.rand(z.shape, generator=gen, dtype=torch.float64, device=dev)
                take = edge & (torch.rand(z.shape, generator=gen, dtype=torch.float64, device=dev) < 0.5)
                z = torch.where(take, zf * mix + right * (1 - mix), z)
            sigma = 0.0012 + 0.0019 * (z - 0.4) ** 2
            noise = torch.randn(z.shape, generator=gen, dtype=torch.float64, device=dev)
            zn = z + noise * torch.where(torch.isfinite(sigma), sigma, torch.zeros_like(sigma))
            valid = torch.isfinite(zn) & (zn >= 0.5) & (zn <= 4.5)
            mm = torch.where(valid, torch.round(zn * 1000.0), torch.zeros_like(zn))
            drop = torch.rand(z.shape, generator=gen, dtype=torch.float64, device=dev) < self.dropout
            mm = torch.where(drop, torch.zeros_like(mm), mm)
            out[j] = mm.to(torch.int32).to(torch.int16)  # uint16 bits (values <= 4500)
        return out


def _orbit_poses(dim: float, n: int, radius: float = 1.2, deg_per_frame: float = 0.5,
                 drift_per_frame: float = 0.002, height: float = -0.25, phase_deg: float = 0.0) -> list:
    c = np.array([dim / 2, dim / 2, dim / 2])
    poses = []
    for k in range(n):
        th = np.deg2rad(phase_deg + deg_per_frame * k)
        # orbit about the world y axis through the cube centre; drift moves the camera up
        # (towards -y) along that axis
        pos = c + np.array([radius * np.sin(th), height - drift_per_frame * k, -radius * np.cos(th)])
        target = c + np.array([0.0, 0.1, 0.0])
        poses.append(look_at(pos, target))
    return poses


def _objects(rng, dim, n_spheres, n_boxes, ground_y, max_axis_dist=0.7):
    """Spheres / boxes resting on the ground plane, near the orbit axis (>= 0.5 m from an
    orbit of radius 1.2 m) and fully inside the volume."""
    c = dim / 2
    spheres, boxes = [], []
    for _ in range(n_spheres):
        r = rng.uniform(0.2, 0.4) * min(1.0, dim / 1.5)
        r = min(r, 0.4)
        rad = rng.uniform(0.0, max(0.0, max_axis_dist - r))
        ang = rng.uniform(0, 2 * np.pi)
        lift = rng.uniform(0.0, 0.3 * dim / 3)
        cy = ground_y - r - lift
        cy = max(cy, r + 0.05)
        spheres.append(((c + rad * np.cos(ang), cy, c + rad * np.sin(ang)), r))
    for _ in range(n_boxes):
        hx, hy, hz = rng.uniform(0.1, 0.25, size=3)
        rad = rng.uniform(0.0, max(0.0, max_axis_dist - max(hx, hz) * 1.5))
        ang = rng.uniform(0, 2 * np.pi)
        cx, cz = c + rad * np.cos(ang), c + rad * np.sin(ang)
        boxes.append(((cx - hx, ground_y - 2 * hy, cz - hz), (cx + hx, ground_y, cz + hz)))
    return spheres, boxes


def plain_c1(n_frames: int = 100, seed: int = 0xC0FFEE + 1) -> Workload:
    """Plain KinectFusion: 128^3 over 1.5 m, float32 TSDF + weight, mu 30 mm, ICP {10,5,4}."""
    dim = 1.5
    rng = np.random.Generator(np.random.PCG64(splitmix64(seed)))
    ground = dim / 2 + 0.6
    spheres, boxes = _objects(rng, dim, 3, 0, ground, max_axis_dist=0.7)
    scene = Scene(planes=[((0.0, 1.0, 0.0), ground)], spheres=spheres, boxes=boxes)
    cfg = GFusionConfig(volumeSize=(128, 128, 128), volumeDimensions=(dim, dim, dim), mu=0.03,
                        maxWeight=100.0, iterations=(10, 5, 4), storage=L.KF_STORAGE_F32F32,
                        jtj=L.KF_JTJ_FP32, quirks=L.KF_QUIRKS_TRACKING)
    return Workload("c1_plain_128", cfg, Intrinsics(), scene, _orbit_poses(dim, n_frames), seed,
                    dropout=0.02, mc_every=0)


def precision_c2(n_frames: int = 1000, seed: int = 0xC0FFEE + 2, storage: int = L.KF_STORAGE_F16U16,
                 jtj: int = L.KF_JTJ_SPLIT_BF16, size: int = 512) -> Workload:
    """Precision form: 512^3 over 3 m, FP16 TSDF + uint16 weight, split-BF16 J^T J."""
    dim = 3.0
    rng = np.random.Generator(np.random.PCG64(splitmix64(seed)))
    ground = dim / 2 + 0.6
    spheres, boxes = _objects(rng, dim, 8, 2, ground, max_axis_dist=0.7)
    scene = Scene(planes=[((0.0, 1.0, 0.0), ground)], spheres=spheres, boxes=boxes)
    cfg = GFusionConfig(volumeSize=(size, size, size), volumeDimensions=(dim, dim, dim), mu=0.03,
                        maxWeight=100.0, iterations=(10, 5, 4), storage=storage, jtj=jtj,
                        quirks=L.KF_QUIRKS_TRACKING)
    return Workload(f"c2_precision_{size}", cfg, Intrinsics(), scene, _orbit_poses(dim, n_frames),
                    seed, dropout=0.02, mc_every=100)


def large_c5(n_frames: int = 500, seed: int = 0xC0FFEE + 5, size: int = 768) -> Workload:
    """Large volume: 768^3 over 4 m, room of 4 walls + 20 spheres/boxes, SDF tracking along
    a seeded spline at 5 mm/frame, 5% dropouts and flying pixels."""
    dim = 4.0
    rng = np.random.Generator(np.random.PCG64(splitmix64(seed)))
    floor = 3.6
    walls = [((1.0, 0.0, 0.0), 0.15), ((1.0, 0.0, 0.0), dim - 0.15),
             ((0.0, 0.0, 1.0), 0.15), ((0.0, 0.0, 1.0), dim - 0.15), ((0.0, 1.0, 0.0), floor)]
    spheres, boxes = [], []
    for k in range(20):
        x, z = rng.uniform(0.5, dim - 0.5, size=2)
        if k % 2 == 0:
            r = rng.uniform(0.15, 0.35)
            spheres.append(((x, floor - r - rng.uniform(0, 0.5), z), r))
        else:
            h = rng.uniform(0.1, 0.3, size=3)
            boxes.append(((x - h[0], floor - 2 * h[1], z - h[2]), (x + h[0], floor, z + h[2])))
    scene = Scene(planes=walls, spheres=spheres, boxes=boxes)
    # seeded Catmull-Rom spline through control points in the middle of the room
    ctrl = np.column_stack([rng.uniform(1.3, 2.7, 8), rng.uniform(2.3, 2.6, 8), rng.uniform(1.0, 1.6, 8)])
    ctrl[0] = (2.0, 2.4, 0.9)
    pts = []
    for i in range(1, len(ctrl) - 2):
        p0, p1, p2, p3 = ctrl[i - 1], ctrl[i], ctrl[i + 1], ctrl[i + 2]
        for s in np.linspace(0, 1, 200, endpoint=False):
            pts.append(0.5 * ((2 * p1) + (-p0 + p2) * s + (2 * p0 - 5 * p1 + 4 * p2 - p3) * s * s
                              + (-p0 + 3 * p1 - 3 * p2 + p3) * s ** 3))
    pts = np.array(pts)
    seg = np.linalg.norm(np.diff(pts, axis=0), axis=1)
    arc = np.concatenate([[0], np.cumsum(seg)])
    poses = []
    yaw0 = 0.0
    for k in range(n_frames):
        s = min(0.005 * k, arc[-1])
        p = np.array([np.interp(s, arc, pts[:, j]) for j in range(3)])
        yaw = yaw0 + 0.25 * np.sin(0.004 * k)
        fwd = np.array([np.sin(yaw), 0.12 * np.sin(0.003 * k), np.cos(yaw)])
        T = look_at(p, p + fwd) if k else np.eye(4)
        if k == 0:
            T[:3, 3] = p  # identity rotation: the SDF pose chain starts translation-only
        poses.append(T)
    cfg = GFusionConfig(volumeSize=(size, size, size), volumeDimensions=(dim, dim, dim), mu=0.03,
                        maxWeight=100.0, iterations=(10, 5, 4), storage=L.KF_STORAGE_F16U16,
                        jtj=L.KF_JTJ_FP32, tracking=L.KF_TRACK_SDF, farPlane=4.5,
                        quirks=L.KF_QUIRKS_TRACKING)
    return Workload(f"c5_large_{size}", cfg, Intrinsics(), scene, poses, seed, dropout=0.05,
                    flying_pixels=True, mc_every=0)


def pose_error(A: np.ndarray, B: np.ndarray) -> tuple[float, float]:
    """(translation error in metres, rotation error in degrees) between two poses."""
    dt = float(np.linalg.norm(A[:3, 3] - B[:3, 3]))
    R = A[:3, :3].T @ B[:3, :3]
    c = np.clip((np.trace(R) - 1) / 2, -1.0, 1.0)
    return dt, float(np.degrees(np.arccos(c)))


def ate(poses_a, poses_b) -> float:
    """RMS translation difference (m) between two trajectories."""
    d = [np.linalg.norm(np.asarray(a)[:3, 3] - np.asarray(b)[:3, 3]) for a, b in zip(poses_a, poses_b)]
    return float(np.sqrt(np.mean(np.square(d)))) if d else 0.0


C3_SIZES = (128, 192, 256, 384)


def session_scene(n_frames: int, seed: int, size: int, phase_deg: float = 0.0, deg_per_frame: float = 0.5) -> Workload:
    """One session of the batched and served forms: a seeded scene in a 1.5 m cube (ground
    plane, 6 spheres and 2 boxes near the orbit axis -- C1's three spheres alone leave some
    seeds' tracking ill-conditioned, in the FP64 oracle as on the GPU), an orbit with a
    seeded start angle and direction, FP16 TSDF + uint16 weight, split-BF16 J^T J."""
    w = plain_c1(n_frames, seed=seed)
    rng = np.random.Generator(np.random.PCG64(splitmix64(seed ^ 0x5EED)))
    ground = 1.5 / 2 + 0.6
    spheres, boxes = _objects(rng, 1.5, 6, 2, ground, max_axis_dist=0.7)
    w.scene = Scene(planes=[((0.0, 1.0, 0.0), ground)], spheres=spheres, boxes=boxes)
    w.poses = _orbit_poses(1.5, n_frames, deg_per_frame=deg_per_frame, phase_deg=phase_deg)
    w.config.volumeSize = (size, size, size)
    w.config.storage = L.KF_STORAGE_F16U16
    w.config.jtj = L.KF_JTJ_SPLIT_BF16
    return w


def batched_c3(n_sessions: int = 64, n_frames: int = 300, seed: int = 0xC0FFEE + 3) -> list:
    """Batched form: independent sessions (session_scene), volume size drawn uniformly from
    {128, 192, 256, 384}^3."""
    out = []
    rng = np.random.Generator(np.random.PCG64(splitmix64(seed)))
    for k in range(n_sessions):
        sk = splitmix64(seed + k) & 0xFFFFFFFF
        size = int(rng.choice(C3_SIZES))
        phase = float(rng.uniform(0.0, 360.0))
        step = 0.5 if rng.random() < 0.5 else -0.5
        w = session_scene(n_frames, sk, size, phase, step)
        w.name = f"c3_session{k}_{size}"
        out.append(w)
    return out


@dataclass
class Arrival:
    t: float        # arrival time (s)
    frames: int     # session length
    size: int       # volume side
    scene: int      # index of the pre-rendered sequence it streams


def served_c4(duration_s: float, rate_per_s: float = 20.0, seed: int = 0xC0FFEE + 4,
              n_scenes: int = 16, sizes=tuple(range(128, 513, 32))) -> list:
    """Serving form: Poisson arrivals (rate_per_s), session length U(50, 2000) frames,
    volume side drawn from 128..512 (multiples of 32), each session streaming one of
    n_scenes seeded sequences at 30 Hz.  Arrivals up to duration_s."""
    rng = np.random.Generator(np.random.PCG64(splitmix64(seed)))
    t, out = 0.0, []
    while True:
        t += float(rng.exponential(1.0 / rate_per_s))
        if t > duration_s:
            return out
        out.append(Arrival(t, int(rng.integers(50, 2001)), int(rng.choice(sizes)), int(rng.integers(0, n_scenes))))
