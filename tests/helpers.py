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
