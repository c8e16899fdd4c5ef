"""Python mirror of the reference's gFusion and MCubes classes over the C ABI.

Reference: class gFusion (include/gFusion.h:124-624) and class MCubes
(include/mcubes.h:48-168).  Method names follow the reference so that code written
against it reads the same; GL texture/buffer names become numpy arrays copied from the
device.  Poses are 4x4 camera-to-world matrices in ordinary row-major numpy layout;
they cross the ABI column-major (glm layout).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


def _tune_times(t, sweep: bool = True) -> dict:
    names = ["integrate_z8", "integrate_z16", "integrate_z32"] + (["raycast_sweep"] if sweep else []) + \
            ["raycast_rows2", "raycast_rows4", "raycast_rows8"]
    return {n: float(v) for n, v in zip(names, t)}


def _pose_to_c(pose) -> C.Array:
    m = np.asarray(pose, dtype=np.float64).reshape(4, 4)
    return (C.c_double * 16)(*m.flatten(order="F"))


def _pose_from_c(arr) -> np.ndarray:
    return np.array(list(arr), dtype=np.float64).reshape(4, 4, order="F")


@dataclass
class GFusionConfig:
    """gFusionConfig (gFusion.h:42-82) plus the storage / precision / quirk policy."""
    volumeSize: tuple = (256, 256, 256)
    volumeDimensions: tuple = (1.0, 1.0, 1.0)
    mu: float = 0.05
    maxWeight: float = 100.0
    nearPlane: float = 0.1
    farPlane: float = 3.0
    dist_threshold: float = 0.05
    normal_threshold: float = 0.8
    iterations: tuple = (5, 5, 5)  # index 0 = finest level
    storage: int = L.KF_STORAGE_F32F32
    jtj: int = L.KF_JTJ_FP32
    tracking: int = L.KF_TRACK_ICP
    quirks: int = L.KF_QUIRKS_DEFAULT
    integrate_every: int = 1

    def stepSize(self) -> float:
        """gFusionConfig::stepSize (gFusion.h:72-81)."""
        return min(self.volumeDimensions) / max(self.volumeSize)

    def to_c(self) -> L.kf_config:
        c = L.kf_config()
        c.nx, c.ny, c.nz = (int(v) for v in self.volumeSize)
        c.dim_x, c.dim_y, c.dim_z = (float(v) for v in self.volumeDimensions)
        c.mu = self.mu
        c.max_weight = self.maxWeight
        c.near_plane = self.nearPlane
        c.far_plane = self.farPlane
        c.dist_threshold = self.dist_threshold
        c.normal_threshold = self.normal_threshold
        for i in range(3):
            c.iterations[i] = int(self.iterations[i])
        c.storage = self.storage
        c.jtj = self.jtj
        c.tracking = self.tracking
        c.quirks = self.quirks
        c.integrate_every = self.integrate_every
        return c


@dataclass
class Intrinsics:
    fx: float = 365.0
    fy: float = 365.0
    cx: float = 256.0
    cy: float = 212.0
    width: int = 512
    height: int = 424

    def to_c(self) -> L.kf_intrinsics:
        return L.kf_intrinsics(self.fx, self.fy, self.cx, self.cy, self.width, self.height)


def volume_bytes(cfg: GFusionConfig) -> int:
    n = int(np.prod(cfg.volumeSize))
    return n * (4 if cfg.storage == L.KF_STORAGE_F32F32 else 2) * 2


def decode_volume(raw: np.ndarray, cfg: GFusionConfig):
    """Split a raw two-plane volume into (tsdf float32, weight float32) arrays [z, y, x]."""
    nx, ny, nz = cfg.volumeSize
    n = nx * ny * nz
    if cfg.storage == L.KF_STORAGE_F32F32:
        v = raw.view(np.float32)
        F, W = v[:n], v[n:]
    elif cfg.storage == L.KF_STORAGE_F16U16:
        F = raw[:2 * n].view(np.float16).astype(np.float32)
        W = raw[2 * n:].view(np.uint16).astype(np.float32)
    else:
        F = raw[:2 * n].view(np.int16).astype(np.float32) * np.float32(0.00003051944088)
        W = raw[2 * n:].view(np.int16).astype(np.float32)
    return F.reshape(nz, ny, nx), W.reshape(nz, ny, nx)


class GFusion:
    """B200 KinectFusion session with the gFusion method surface."""

    def __init__(self, config: GFusionConfig | None = None, intrinsics: Intrinsics | None = None):
        self.lib = L.load()
        self.configuration = config or GFusionConfig()
        self.intrinsics = intrinsics or Intrinsics()
        self._cc = self.configuration.to_c()
        self._ci = self.intrinsics.to_c()
        h = C.c_void_p()
        L.check(self.lib.kf_create(C.byref(self._cc), C.byref(self._ci), C.byref(h)), "kf_create")
        self._h = h

    # ---- lifecycle --------------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            self.lib.kf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int, what: str) -> None:
        if st != L.KF_OK:
            msg = self.lib.kf_last_error(self._h)
            raise L.KfError(st, what + (": " + msg.decode() if msg else ""))

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def setConfig(self, config: GFusionConfig) -> None:
        self.configuration = config
        self._cc = config.to_c()
        self._check(self.lib.kf_set_config(self._h, C.byref(self._cc)), "kf_set_config")

    # ---- pose / reset -----------------------------------------------------------------
    def Reset(self, pose, deleteFlag: bool = False) -> None:
        self._check(self.lib.kf_reset(self._h, _pose_to_c(pose), int(deleteFlag)), "kf_reset")

    def resetVolume(self) -> None:
        self._check(self.lib.kf_reset_volume(self._h), "kf_reset_volume")

    def resetPose(self, pose) -> None:
        self._check(self.lib.kf_reset_pose(self._h, _pose_to_c(pose)), "kf_reset_pose")

    def setPose(self, pose) -> None:
        self._check(self.lib.kf_set_pose(self._h, _pose_to_c(pose)), "kf_set_pose")

    def getPose(self) -> np.ndarray:
        a = (C.c_double * 16)()
        self._check(self.lib.kf_get_pose(self._h, a), "kf_get_pose")
        return _pose_from_c(a)

    def getTransPose(self) -> np.ndarray:
        return self.getPose()[:3, 3].copy()

    def getCumTwist(self) -> np.ndarray:
        a = (C.c_double * 6)()
        self._check(self.lib.kf_get_cum_twist(self._h, a), "kf_get_cum_twist")
        return np.array(list(a))

    # ---- per-frame operations -----------------------------------------------------------
    def depthToVertex(self, depth) -> None:
        d = np.ascontiguousarray(depth)
        if d.shape != (self.intrinsics.height, self.intrinsics.width):
            raise ValueError(f"depth shape {d.shape}")
        if d.dtype == np.uint16:
            st = self.lib.kf_depth_to_vertex_u16(self._h, d.ctypes.data)
        else:
            d = np.ascontiguousarray(d, dtype=np.float32)
            st = self.lib.kf_depth_to_vertex_f32(self._h, d.ctypes.data)
        self._check(st, "kf_depth_to_vertex")

    def vertexToNormal(self) -> None:
        self._check(self.lib.kf_vertex_to_normal(self._h), "kf_vertex_to_normal")

    def Track(self) -> bool:
        t = C.c_int()
        self._check(self.lib.kf_track_icp(self._h, C.byref(t)), "kf_track_icp")
        return bool(t.value)

    def TrackSDF(self) -> bool:
        t = C.c_int()
        self._check(self.lib.kf_track_sdf(self._h, C.byref(t)), "kf_track_sdf")
        return bool(t.value)

    def recoverPose(self) -> bool:
        t = C.c_int()
        self._check(self.lib.kf_recover_pose(self._h, C.byref(t)), "kf_recover_pose")
        return bool(t.value)

    def integrate(self) -> None:
        self._check(self.lib.kf_integrate(self._h), "kf_integrate")

    def raycast(self) -> None:
        self._check(self.lib.kf_raycast(self._h), "kf_raycast")

    def frameStep(self, depth_u16) -> bool:
        """One iteration of the kinect.cpp:654-695 loop body."""
        d = np.ascontiguousarray(depth_u16, dtype=np.uint16)
        t = C.c_int()
        self._check(self.lib.kf_frame_step_u16(self._h, d.ctypes.data, C.byref(t)), "kf_frame_step_u16")
        return bool(t.value)

    def frameStepAsync(self, depth_u16) -> None:
        """Pipelined frame step (kf_frame_step_u16_async): enqueue this frame and read the
        previous one's result (lastResult()); frameSync() reads the one in flight.  The
        frame array is kept alive until the next call."""
        d = np.ascontiguousarray(depth_u16, dtype=np.uint16)
        if d.shape != (self.intrinsics.height, self.intrinsics.width):
            raise ValueError(f"depth must be {self.intrinsics.height}x{self.intrinsics.width}")
        prev = getattr(self, "_async_frames", [])
        self._check(self.lib.kf_frame_step_u16_async(self._h, d.ctypes.data), "kf_frame_step_u16_async")
        self._async_frames = (prev + [d])[-2:]  # this frame and the one whose step may still run

    def frameSync(self) -> bool:
        t = C.c_int()
        self._check(self.lib.kf_frame_sync(self._h, C.byref(t)), "kf_frame_sync")
        self._async_frames = []
        return bool(t.value)

    def lastResult(self):
        """(pose, tracked) of the last frame result read by the host (no wait)."""
        a = (C.c_double * 16)()
        t = C.c_int()
        self._check(self.lib.kf_get_last_result(self._h, a, C.byref(t)), "kf_get_last_result")
        return _pose_from_c(a), bool(t.value)

    def frameStepDevice(self, device_ptr: int, sync: bool = True):
        t = C.c_int()
        st = self.lib.kf_frame_step_u16_device(self._h, C.c_void_p(device_ptr),
                                               C.byref(t) if sync else None)
        self._check(st, "kf_frame_step_u16_device")
        return bool(t.value) if sync else None

    # ---- accessors ----------------------------------------------------------------------
    def _map(self, fn, level: int, comps: int, dtype=np.float32) -> np.ndarray:
        w, h = self.intrinsics.width >> level, self.intrinsics.height >> level
        out = np.empty((h, w, comps) if comps > 1 else (h, w), dtype=dtype)
        self._check(fn(self._h, level, out.ctypes.data), fn.__name__)
        return out

    def getVerts(self) -> np.ndarray:
        """Raycast vertex map (m_textureReferenceVertex), H x W x 4."""
        v = np.empty((self.intrinsics.height, self.intrinsics.width, 4), np.float32)
        self._check(self.lib.kf_get_raycast(self._h, v.ctypes.data, None), "kf_get_raycast")
        return v

    def getNorms(self) -> np.ndarray:
        n = np.empty((self.intrinsics.height, self.intrinsics.width, 4), np.float32)
        self._check(self.lib.kf_get_raycast(self._h, None, n.ctypes.data), "kf_get_raycast")
        return n

    def setReferenceMaps(self, vertex4, normal4) -> None:
        """Replace the raycast maps Track() associates against (H x W x 4 each, world frame)."""
        v = np.ascontiguousarray(vertex4, np.float32)
        n = np.ascontiguousarray(normal4, np.float32)
        shape = (self.intrinsics.height, self.intrinsics.width, 4)
        if v.shape != shape or n.shape != shape:
            raise ValueError(f"reference maps must be {shape}")
        self._check(self.lib.kf_set_reference_maps(self._h, v.ctypes.data, n.ctypes.data),
                    "kf_set_reference_maps")

    def getVertexMap(self, level: int = 0) -> np.ndarray:
        return self._map(self.lib.kf_get_vertex_map, level, 4)

    def getNormalMap(self, level: int = 0) -> np.ndarray:
        return self._map(self.lib.kf_get_normal_map, level, 4)

    def getDepthImage(self, level: int = 0) -> np.ndarray:
        return self._map(self.lib.kf_get_depth_map, level, 1)

    def getTrackStatus(self, level: int = 0) -> np.ndarray:
        return self._map(self.lib.kf_get_track_status, level, 1, np.int32)

    def getVolumeRaw(self) -> np.ndarray:
        raw = np.empty(volume_bytes(self.configuration), np.uint8)
        self._check(self.lib.kf_copy_volume_to_host(self._h, raw.ctypes.data, raw.nbytes),
                    "kf_copy_volume_to_host")
        return raw

    def setVolumeRaw(self, raw: np.ndarray) -> None:
        raw = np.ascontiguousarray(raw, dtype=np.uint8)
        self._check(self.lib.kf_copy_volume_from_host(self._h, raw.ctypes.data, raw.nbytes),
                    "kf_copy_volume_from_host")

    # ---- depth ingest stages (the capture side of the reference) ---------------------------
    def setDepthUndistortion(self, ir) -> None:
        """Undistort each frame before the pyramid as libfreenect2's Registration does
        (src/interface.cpp:290-313).  ir: (fx, fy, cx, cy, k1, k2, k3, p1, p2) of the IR
        camera, or None to turn it off."""
        if ir is None:
            self._check(self.lib.kf_set_depth_undistortion(self._h, None), "kf_set_depth_undistortion")
            return
        c = L.kf_ir_camera(*[float(v) for v in ir])
        self._check(self.lib.kf_set_depth_undistortion(self._h, C.byref(c)), "kf_set_depth_undistortion")

    def getUndistortionMap(self) -> np.ndarray:
        m = np.empty((self.intrinsics.height, self.intrinsics.width), np.int32)
        self._check(self.lib.kf_get_undistortion_map(self._h, m.ctypes.data), "kf_get_undistortion_map")
        return m

    def setDepthFilter(self, enable: bool) -> None:
        """shaders/filter3D.cs before the pyramid (after the undistortion)."""
        self._check(self.lib.kf_set_depth_filter(self._h, int(bool(enable))), "kf_set_depth_filter")

    # ---- launch shapes and the autotuner -----------------------------------------------
    def setLaunchShape(self, integrate_z_chunk: int, raycast_rows: int) -> None:
        sh = L.kf_launch_shape(int(integrate_z_chunk), int(raycast_rows))
        self._check(self.lib.kf_set_launch_shape(self._h, C.byref(sh)), "kf_set_launch_shape")

    def launchShape(self) -> tuple:
        sh = L.kf_launch_shape()
        self._check(self.lib.kf_get_launch_shape(self._h, C.byref(sh)), "kf_get_launch_shape")
        return sh.integrate_z_chunk, sh.raycast_rows

    def autotune(self, repeats: int = 5):
        """Time every integrate z-chunk and raycast tile shape on the current frame and use
        the fastest.  Returns ((z_chunk, rows), {shape name: mean ms})."""
        sh = L.kf_launch_shape()
        t = (C.c_float * 7)()
        self._check(self.lib.kf_autotune(self._h, int(repeats), C.byref(sh), t), "kf_autotune")
        return (sh.integrate_z_chunk, sh.raycast_rows), _tune_times(t)

    def intensityProjection(self) -> np.ndarray:
        """Volume ray-sum image at the current pose (gFusion::intensityProjection,
        src/gFusion.cpp:1368-1409), H x W x 4: (sum of positive samples, 0, 0, 1)."""
        m = np.empty((self.intrinsics.height, self.intrinsics.width, 4), np.float32)
        self._check(self.lib.kf_intensity_projection(self._h, m.ctypes.data), "kf_intensity_projection")
        return m

    def saveVolume(self, path) -> None:
        """Checkpoint the volume, pose, pose library and reference maps to `path`."""
        self._check(self.lib.kf_save_volume(self._h, os.fsencode(path)), "kf_save_volume")

    def loadVolume(self, path) -> None:
        """Restore a checkpoint written by saveVolume into this (same-sized) session."""
        self._check(self.lib.kf_load_volume(self._h, os.fsencode(path)), "kf_load_volume")

    def selftestBarrierTimeout(self, budget_cycles: int = 2_000_000) -> int:
        """Run the bounded-wait self-test; returns the status (KF_ERR_TIMEOUT expected)."""
        return int(self.lib.kf_selftest_barrier_timeout(self._h, int(budget_cycles)))

    def getVolume(self):
        """(tsdf, weight) float32 arrays indexed [z, y, x]."""
        return decode_volume(self.getVolumeRaw(), self.configuration)

    def getVolumeView(self) -> L.kf_volume_view:
        v = L.kf_volume_view()
        self._check(self.lib.kf_get_volume(self._h, C.byref(v)), "kf_get_volume")
        return v

    def alignmentEnergy(self) -> float:
        f = C.c_float()
        self._check(self.lib.kf_get_alignment_energy(self._h, C.byref(f)), "kf_get_alignment_energy")
        return f.value

    def iterationsRun(self) -> int:
        n = C.c_int()
        self._check(self.lib.kf_get_iterations_run(self._h, C.byref(n)), "kf_get_iterations_run")
        return n.value

    def getReduction(self) -> np.ndarray:
        a = (C.c_float * 32)()
        self._check(self.lib.kf_get_reduction(self._h, a), "kf_get_reduction")
        return np.array(list(a), dtype=np.float32)

    def poseLibrarySize(self) -> int:
        n = C.c_int()
        self._check(self.lib.kf_get_pose_library_size(self._h, C.byref(n)), "kf_get_pose_library_size")
        return n.value

    def getTimes(self) -> np.ndarray:
        """Device ms of the last pyramid, track, integrate, recover and raycast stages and
        of the last marching-cubes extraction."""
        a = (C.c_float * 6)()
        self._check(self.lib.kf_get_stage_times(self._h, a), "kf_get_stage_times")
        return np.array(list(a), dtype=np.float32)

    def stageStats(self):
        """(mean device ms per stage [pyramid, track, integrate, recover, raycast, mc],
        frames) over the timed frame steps (setStageTiming) since resetStageStats()."""
        a = (C.c_double * 6)()
        n = C.c_uint64()
        self._check(self.lib.kf_get_stage_stats(self._h, a, C.byref(n)), "kf_get_stage_stats")
        return np.array(list(a)), n.value

    def setStageTiming(self, every: int) -> None:
        """Record the stage boundaries of every `every`-th frame step (1, 2 or 4; 0 = none)."""
        self._check(self.lib.kf_set_stage_timing(self._h, int(every)), "kf_set_stage_timing")

    def stageTiming(self) -> int:
        e = C.c_int()
        self._check(self.lib.kf_get_stage_timing(self._h, C.byref(e)), "kf_get_stage_timing")
        return e.value

    def resetStageStats(self) -> None:
        self._check(self.lib.kf_reset_stage_stats(self._h), "kf_reset_stage_stats")

    def launchCount(self) -> int:
        n = C.c_uint64()
        self._check(self.lib.kf_get_launch_count(self._h, C.byref(n)), "kf_get_launch_count")
        return n.value

    def stream(self) -> int:
        p = C.c_void_p()
        self._check(self.lib.kf_get_stream(self._h, C.byref(p)), "kf_get_stream")
        return p.value or 0


class GFusionBatch:
    """Batched frame steps over several GFusion sessions (kf_batch_*): one launch per stage
    for all of them; each session's results equal stepping it alone."""

    def __init__(self, max_sessions: int):
        self.lib = L.load()
        h = C.c_void_p()
        L.check(self.lib.kf_batch_create(int(max_sessions), C.byref(h)), "kf_batch_create")
        self._h = h
        self.max_sessions = int(max_sessions)

    def close(self):
        if getattr(self, "_h", None):
            self.lib.kf_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int, what: str):
        if st != L.KF_OK:
            msg = self.lib.kf_batch_last_error(self._h)
            raise L.KfError(st, f"{what}: {msg.decode() if msg else ''}")

    def frameStep(self, sessions, frames) -> np.ndarray:
        """sessions: GFusion list; frames: uint16 H x W arrays (host).  Returns tracked flags."""
        n = len(sessions)
        hs = (C.c_void_p * n)(*[s.handle.value for s in sessions])
        arrs = [np.ascontiguousarray(f, dtype=np.uint16) for f in frames]
        ps = (C.c_void_p * n)(*[a.ctypes.data for a in arrs])
        t = (C.c_int32 * n)()
        self._check(self.lib.kf_batch_frame_step_u16(self._h, hs, ps, n, t), "kf_batch_frame_step_u16")
        return np.array(list(t), dtype=bool)

    def frameStepDevice(self, sessions, device_ptrs) -> np.ndarray:
        """As frameStep, with each frame already in device memory (uint16 pointers)."""
        n = len(sessions)
        hs = (C.c_void_p * n)(*[s.handle.value for s in sessions])
        ps = (C.c_void_p * n)(*[int(p) for p in device_ptrs])
        t = (C.c_int32 * n)()
        self._check(self.lib.kf_batch_frame_step_u16_device(self._h, hs, ps, n, t),
                    "kf_batch_frame_step_u16_device")
        return np.array(list(t), dtype=bool)

    def frameStepDeviceAsync(self, sessions, device_ptrs) -> None:
        """Enqueue a step and read the previous one's results (poses(), tracked()); the
        device runs this step while the caller prepares the next.  sync() finishes it."""
        n = len(sessions)
        hs = (C.c_void_p * n)(*[s.handle.value for s in sessions])
        ps = (C.c_void_p * n)(*[int(p) for p in device_ptrs])
        self._check(self.lib.kf_batch_frame_step_u16_device_async(self._h, hs, ps, n),
                    "kf_batch_frame_step_u16_device_async")

    def sync(self) -> None:
        self._check(self.lib.kf_batch_sync(self._h), "kf_batch_sync")

    def tracked(self, n: int) -> np.ndarray:
        t = (C.c_int32 * n)()
        self._check(self.lib.kf_batch_get_tracked(self._h, n, t), "kf_batch_get_tracked")
        return np.array(list(t), dtype=bool)

    def poses(self, n: int) -> np.ndarray:
        """Camera-to-world poses (n x 4 x 4) of the last step's first n sessions."""
        a = np.empty((n, 16), np.float64)
        self._check(self.lib.kf_batch_get_poses(self._h, n, a.ctypes.data), "kf_batch_get_poses")
        return a.reshape(n, 4, 4).transpose(0, 2, 1).copy()

    def stageTimes(self) -> np.ndarray:
        """Device ms of the last step: pyramid, track, integrate, recover, raycast."""
        a = (C.c_float * 5)()
        self._check(self.lib.kf_batch_get_stage_times(self._h, a), "kf_batch_get_stage_times")
        return np.array(list(a), dtype=np.float32)

    def launchCount(self) -> int:
        n = C.c_uint64()
        self._check(self.lib.kf_batch_get_launch_count(self._h, C.byref(n)), "kf_batch_get_launch_count")
        return int(n.value)

    def setLaunchShape(self, integrate_z_chunk: int, raycast_rows: int) -> None:
        sh = L.kf_launch_shape(int(integrate_z_chunk), int(raycast_rows))
        self._check(self.lib.kf_batch_set_launch_shape(self._h, C.byref(sh)), "kf_batch_set_launch_shape")

    def launchShape(self) -> tuple:
        sh = L.kf_launch_shape()
        self._check(self.lib.kf_batch_get_launch_shape(self._h, C.byref(sh)), "kf_batch_get_launch_shape")
        return sh.integrate_z_chunk, sh.raycast_rows

    def autotune(self, sessions, repeats: int = 3):
        """kf_batch_autotune over this mix of sessions; returns ((z_chunk, rows), times)."""
        n = len(sessions)
        hs = (C.c_void_p * n)(*[s.handle.value for s in sessions])
        sh = L.kf_launch_shape()
        t = (C.c_float * 6)()
        self._check(self.lib.kf_batch_autotune(self._h, hs, n, int(repeats), C.byref(sh), t), "kf_batch_autotune")
        return (sh.integrate_z_chunk, sh.raycast_rows), _tune_times(t, sweep=False)


class GFusionServer:
    """The served form (kf_server_*): resident sessions admitted by slots and device memory,
    frames queued as they arrive, batched steps over the sessions with a waiting frame."""

    def __init__(self, hbm_budget_bytes: int = 0, max_sessions: int = 128, max_batch: int = 64,
                 storage: int = L.KF_STORAGE_F16U16, jtj: int = L.KF_JTJ_SPLIT_BF16):
        self.lib = L.load()
        c = L.ServerConfig()
        L.check(self.lib.kf_server_config_default(C.byref(c)), "kf_server_config_default")
        c.hbm_budget_bytes, c.max_sessions, c.max_batch = int(hbm_budget_bytes), int(max_sessions), int(max_batch)
        c.storage, c.jtj = int(storage), int(jtj)
        h = C.c_void_p()
        L.check(self.lib.kf_server_create(C.byref(c), C.byref(h)), "kf_server_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self.lib.kf_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int, what: str):
        if st != L.KF_OK:
            msg = self.lib.kf_server_last_error(self._h)
            raise L.KfError(st, f"{what}: {msg.decode() if msg else ''}")

    def now(self) -> float:
        return float(self.lib.kf_server_now())

    def open(self, config: "GFusionConfig", intrinsics: "Intrinsics", pose) -> int | None:
        """Admit a session; None when no slot or memory is free (KF_ERR_ADMISSION)."""
        cc = config.to_c()
        ic = intrinsics.to_c()
        sid = C.c_int()
        st = self.lib.kf_server_open(self._h, C.byref(cc), C.byref(ic), _pose_to_c(pose), C.byref(sid))
        if st == L.KF_ERR_ADMISSION:
            return None
        self._check(st, "kf_server_open")
        return sid.value

    def prewarm(self, config: "GFusionConfig", intrinsics: "Intrinsics", count: int) -> int:
        """Create `count` idle sessions of this configuration ahead of admissions."""
        cc, ic, n = config.to_c(), intrinsics.to_c(), C.c_int()
        st = self.lib.kf_server_prewarm(self._h, C.byref(cc), C.byref(ic), int(count), C.byref(n))
        if st not in (L.KF_OK, L.KF_ERR_ADMISSION):
            self._check(st, "kf_server_prewarm")
        return n.value

    def close_session(self, sid: int):
        self._check(self.lib.kf_server_close(self._h, int(sid)), "kf_server_close")

    def submit(self, sid: int, frame: np.ndarray):
        f = np.ascontiguousarray(frame, dtype=np.uint16)
        self._check(self.lib.kf_server_submit(self._h, int(sid), f.ctypes.data), "kf_server_submit")

    def submit_device(self, sid: int, device_ptr: int):
        self._check(self.lib.kf_server_submit_device(self._h, int(sid), C.c_void_p(int(device_ptr))),
                    "kf_server_submit_device")

    def step(self) -> int:
        n = C.c_int()
        self._check(self.lib.kf_server_step(self._h, C.byref(n)), "kf_server_step")
        return n.value

    def step_async(self) -> int:
        """Enqueue a step; returns the frame count of the previous step, whose results are
        now readable (last_step, pose)."""
        n = C.c_int()
        self._check(self.lib.kf_server_step_async(self._h, C.byref(n)), "kf_server_step_async")
        return n.value

    def sync(self) -> int:
        n = C.c_int()
        self._check(self.lib.kf_server_sync(self._h, C.byref(n)), "kf_server_sync")
        return n.value

    def pose(self, sid: int):
        """(camera-to-world pose, tracked, frames done) after the session's last stepped frame."""
        a = (C.c_double * 16)()
        t = C.c_int()
        d = C.c_uint64()
        self._check(self.lib.kf_server_get_pose(self._h, int(sid), a, C.byref(t), C.byref(d)), "kf_server_get_pose")
        return _pose_from_c(a), bool(t.value), int(d.value)

    def last_step(self, max_n: int = 256):
        """(ids, poses n x 4 x 4, tracked) of the sessions in the last step."""
        ids = np.empty(max_n, np.int32)
        poses = np.empty((max_n, 16), np.float64)
        tr = np.empty(max_n, np.int32)
        n = C.c_int()
        self._check(self.lib.kf_server_last_step(self._h, max_n, ids.ctypes.data, poses.ctypes.data,
                                                 tr.ctypes.data, C.byref(n)), "kf_server_last_step")
        k = n.value
        return ids[:k].copy(), poses[:k].reshape(k, 4, 4).transpose(0, 2, 1).copy(), tr[:k].astype(bool)

    def pending(self, sid: int) -> int:
        q = C.c_int()
        self._check(self.lib.kf_server_pending(self._h, int(sid), C.byref(q)), "kf_server_pending")
        return q.value

    def stats(self) -> dict:
        s = L.ServerStats()
        self._check(self.lib.kf_server_stats(self._h, C.byref(s)), "kf_server_stats")
        return {"frames": s.frames, "steps": s.steps, "busy_s": s.busy_s, "p50_ms": s.p50_ms, "p99_ms": s.p99_ms,
                "max_ms": s.max_ms, "bytes_in_use": s.bytes_in_use, "active_sessions": s.active_sessions}

    def reset_stats(self):
        self._check(self.lib.kf_server_reset_stats(self._h), "kf_server_reset_stats")


class MCubes:
    """Marching-cubes extraction of a GFusion volume (mcubes.h:48-168)."""

    def __init__(self, fusion: GFusion | None = None):
        self.fusion = fusion
        self.isoLevel = 0.0
        self.nTriangles = 0

    def setVolumeTexture(self, fusion: GFusion) -> None:
        self.fusion = fusion

    def setIsolevel(self, iso: float) -> None:
        self.isoLevel = float(iso)

    def generateMarchingCubes(self, method: int = L.KF_MC_HISTOPYRAMID) -> int:
        n = C.c_uint32()
        f = self.fusion
        f._check(f.lib.kf_mc_extract(f._h, self.isoLevel, method, C.byref(n)), "kf_mc_extract")
        self.nTriangles = n.value
        return n.value

    def getNumberTriangles(self) -> int:
        """Vertex count, as the reference's getNumberTriangles() (returns m_totalSum)."""
        return 3 * self.nTriangles

    def getVertices(self) -> np.ndarray:
        f = self.fusion
        out = np.empty((3 * self.nTriangles, 4), np.float32)
        f._check(f.lib.kf_mc_copy_vertices(f._h, out.ctypes.data, out.shape[0]), "kf_mc_copy_vertices")
        return out

    def getNormals(self) -> np.ndarray:
        """Face normal of each vertex's triangle (calcNormal, unnormalised, w = 0)."""
        f = self.fusion
        out = np.empty((3 * self.nTriangles, 4), np.float32)
        f._check(f.lib.kf_mc_copy_normals(f._h, out.ctypes.data, out.shape[0]), "kf_mc_copy_normals")
        return out

    def extractMesh(self):
        """Welded mesh of the current volume at the iso level: (positions n x 3 metres,
        unit normals n x 3, triangle indices t x 3)."""
        f = self.fusion
        nv, nt = C.c_uint32(), C.c_uint32()
        f._check(f.lib.kf_mc_extract_mesh(f._h, self.isoLevel, C.byref(nv), C.byref(nt)), "kf_mc_extract_mesh")
        P = np.empty((nv.value, 3), np.float32)
        N = np.empty((nv.value, 3), np.float32)
        I = np.empty((nt.value, 3), np.uint32)
        f._check(f.lib.kf_mc_copy_mesh(f._h, P.ctypes.data, N.ctypes.data, I.ctypes.data, nv.value, nt.value),
                 "kf_mc_copy_mesh")
        return P, N, I

    def exportWeldedMeshPly(self, path: str) -> None:
        f = self.fusion
        f._check(f.lib.kf_mc_export_mesh_ply(f._h, path.encode()), "kf_mc_export_mesh_ply")

    def exportWeldedMeshStl(self, path: str) -> None:
        f = self.fusion
        f._check(f.lib.kf_mc_export_mesh_stl(f._h, path.encode()), "kf_mc_export_mesh_stl")

    def getBaseLevel(self) -> np.ndarray:
        f = self.fusion
        nx, ny, nz = f.configuration.volumeSize
        out = np.empty(nx * ny * nz, np.uint32)
        f._check(f.lib.kf_mc_copy_base_level(f._h, out.ctypes.data, out.size), "kf_mc_copy_base_level")
        return out.reshape(nz, ny, nx)

    def exportMesh(self, path: str) -> None:
        f = self.fusion
        f._check(f.lib.kf_mc_export_stl(f._h, path.encode()), "kf_mc_export_stl")

    def exportPointCloud(self, path: str) -> None:
        f = self.fusion
        f._check(f.lib.kf_mc_export_ply(f._h, path.encode()), "kf_mc_export_ply")


def prefix_sum_device(d_in: int, d_out: int, n: int, stream: int = 0) -> int:
    """Exclusive scan of n uint32 device values; returns the total."""
    lib = L.load()
    tot = C.c_uint32()
    L.check(lib.kf_prefix_sum_u32(C.c_void_p(d_in), C.c_void_p(d_out), n, C.byref(tot),
                                  C.c_void_p(stream)), "kf_prefix_sum_u32")
    return tot.value
