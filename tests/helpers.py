"""Shared helpers for the parity tests: small workloads and comparison utilities."""
from __future__ import annotations

import numpy as np

from oglfusionkinectv2_b200 import GFusionConfig, Intrinsics, synth, _lib as L


def small_workload(n_frames=12, size=64, storage=L.KF_STORAGE_F32F32, quirks=None,
                   jtj=L.KF_JTJ_FP32, tracking=L.KF_TRACK_ICP, seed=0xC0FFEE + 1):
    """C1-like scene (plane + 3 spheres, 1.5 m cube) at a small volume size."""
    w = synth.plain_c1(n_frames, seed=seed)
    c = w.config
    c.volumeSize = (size, size, size)
    c.storage = storage
    c.jtj = jtj
    c.tracking = tracking
    if quirks is not None:
        c.quirks = quirks
    return w


def pixel_boundary_distance(q: np.ndarray) -> np.ndarray:
    """Distance of a coordinate (after the shaders' +0.5) to the nearest truncation step."""
    return np.abs(q - np.rint(q))


def integrate_ambiguous(cfg: GFusionConfig, intr: Intrinsics, pose: np.ndarray, depth_mm: np.ndarray,
                        old_F: np.ndarray, old_W: np.ndarray, idx: np.ndarray, eps=2e-3) -> np.ndarray:
    """For voxels (z, y, x) in idx, True where an FP32 evaluation of integrate.cs may take a
    different branch or pixel than the FP64 oracle: projected coordinate within eps of a
    truncation step or an image bound, or a decision value within eps of its threshold."""
    nx, ny, nz = cfg.volumeSize
    dim = np.array(cfg.volumeDimensions, np.float64)
    z, y, x = idx
    c = np.stack([(x + 0.5) * dim[0] / nx, (y + 0.5) * dim[1] / ny, (z + 0.5) * dim[2] / nz], -1)
    inv = np.linalg.inv(pose)
    p = c @ inv[:3, :3].T + inv[:3, 3]
    amb = np.zeros(len(x), bool)
    pz = p[:, 2]
    amb |= np.abs(pz - 1e-4) < eps
    with np.errstate(divide="ignore", invalid="ignore"):
        u = (intr.fx * p[:, 0] + intr.cx * pz) / pz + 0.5
        v = (intr.fy * p[:, 1] + intr.cy * pz) / pz + 0.5
    amb |= pixel_boundary_distance(u) < eps
    amb |= pixel_boundary_distance(v) < eps
    amb |= (np.abs(u) < eps) | (np.abs(u - (intr.width - 1)) < eps)
    amb |= (np.abs(v) < eps) | (np.abs(v - (intr.height - 1)) < eps)
    ok = (pz >= 1e-4) & (u >= 0) & (u <= intr.width - 1) & (v >= 0) & (v <= intr.height - 1)
    ui = np.clip(u.astype(np.int64), 0, intr.width - 1)
    vi = np.clip(v.astype(np.int64), 0, intr.height - 1)
    d = depth_mm[vi, ui].astype(np.float64) / 1000.0
    diff = (d - pz) * np.sqrt(1 + (p[:, 0] / pz) ** 2 + (p[:, 1] / pz) ** 2)
    mu = cfg.mu
    amb |= ok & (np.abs(diff + mu) < eps * mu)
    sdf = np.minimum(1.0, diff / mu)
    Fo = old_F[z, y, x].astype(np.float64)
    Wo = old_W[z, y, x].astype(np.float64)
    wd = (Wo * Fo + sdf) / (Wo + 1)
    amb |= ok & (np.abs(wd - 0.2) < eps)
    return amb


def rot_deg(A, B) -> float:
    R = A[:3, :3].T @ B[:3, :3]
    return float(np.degrees(np.arccos(np.clip((np.trace(R) - 1) / 2, -1, 1))))


def _trilinear(F: np.ndarray, p: np.ndarray, dim, size) -> np.ndarray:
    """raycast.cs interpVol in FP64 on a decoded volume F[z, y, x] at world points p (n, 3):
    voxel coordinates p * size / dim - 0.5, taps clamped to the volume."""
    nx, ny, nz = size
    q = p * (np.array([nx, ny, nz], np.float64) / np.array(dim, np.float64)) - 0.5
    b = np.floor(q)
    f = q - b
    bi = b.astype(np.int64)
    n = np.array([nx, ny, nz])
    lo = np.clip(bi, 0, n - 1)
    hi = np.clip(np.minimum(bi + 1, n - 1), 0, None)
    def v(ix, iy, iz):
        return F[iz, iy, ix].astype(np.float64)
    x0, y0, z0 = lo[:, 0], lo[:, 1], lo[:, 2]
    x1, y1, z1 = hi[:, 0], hi[:, 1], hi[:, 2]
    fx, fy, fz = f[:, 0], f[:, 1], f[:, 2]
    return (((v(x0, y0, z0) * (1 - fx) + v(x1, y0, z0) * fx) * (1 - fy) +
             (v(x0, y1, z0) * (1 - fx) + v(x1, y1, z0) * fx) * fy) * (1 - fz) +
            ((v(x0, y0, z1) * (1 - fx) + v(x1, y0, z1) * fx) * (1 - fy) +
             (v(x0, y1, z1) * (1 - fx) + v(x1, y1, z1) * fx) * fy) * fz)


def raycast_ambiguous(cfg: GFusionConfig, intr: Intrinsics, pose: np.ndarray, F: np.ndarray,
                      pix: np.ndarray, eps_f=1e-4, eps_t=1e-5, min_den=0.02) -> np.ndarray:
    """For pixels pix = (ys, xs), True where an FP32 evaluation of raycast.cs may take a
    different branch than the FP64 oracle: the march (raycast.cs:181-212, the oracle's
    restatement) re-run in FP64, flagging a sample value within eps_f of 0 (the first
    negative sample) or of 0.8 (the switch to the fine step), a sample position within
    eps_t (relative) of tfar or a tnear/tfar tie, and a hit whose refinement denominator
    f(t0) - f(t1) is below min_den (the refined position is then that sensitive to the
    last bits of the two samples)."""
    ys, xs = pix
    n = len(xs)
    amb = np.zeros(n, bool)
    if n == 0:
        return amb
    dim = np.array(cfg.volumeDimensions, np.float64)
    size = cfg.volumeSize
    step = dim.min() / max(size)
    large = 0.75 * cfg.mu
    o = pose[:3, 3]
    d = np.stack([(xs - intr.cx) / intr.fx, (ys - intr.cy) / intr.fy, np.ones(n)], -1) @ pose[:3, :3].T
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / d
        tb = -inv * o
        tt = inv * (dim - o)
    tmin = np.minimum(tt, tb).max(-1)
    tmax = np.maximum(tt, tb).min(-1)
    tnear = np.maximum(tmin, cfg.nearPlane if hasattr(cfg, "nearPlane") else 0.1)
    tfar = np.minimum(tmax, cfg.farPlane if hasattr(cfg, "farPlane") else 3.0)
    amb |= np.abs(tnear - tfar) <= eps_t * np.maximum(1.0, np.abs(tfar))
    active = tnear < tfar
    t = tnear.copy()
    f_t = np.where(active, _trilinear(F, o + d * t[:, None], dim, size), 0.0)
    amb |= active & (np.abs(f_t) < eps_f) & (f_t != 0)  # an exact 0 (unobserved) is exact in FP32 too
    active &= f_t >= 0
    tbase = t.copy()
    k = np.zeros(n)
    stepsize = np.full(n, large)
    f_tt = np.zeros(n)
    hit = np.zeros(n, bool)
    for _ in range(int(np.ceil(4.0 / step)) + 8):
        run = active & ~hit & (t < tfar)
        if not run.any():
            break
        amb |= run & (np.abs(t - tfar) <= eps_t * np.maximum(1.0, np.abs(tfar)))
        val = np.zeros(n)
        val[run] = _trilinear(F, o + d[run] * t[run, None], dim, size)
        amb |= run & (((np.abs(val) < eps_f) & (val != 0)) | ((stepsize != step) & (np.abs(val - 0.8) < eps_f)))
        neg = run & (val < 0)
        den = f_t - val
        amb |= neg & (den < min_den)
        hit |= neg
        f_tt = np.where(run, val, f_tt)
        go = run & ~neg
        sw = go & (val < 0.8) & (stepsize != step)
        stepsize = np.where(sw, step, stepsize)
        tbase = np.where(sw, t, tbase)
        k = np.where(sw, 0, k)
        f_t = np.where(go, val, f_t)
        k = np.where(go, k + 1, k)
        t = np.where(go, tbase + k * stepsize, t)
    return amb
