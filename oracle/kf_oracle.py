"""ctypes binding of the FP64 CPU oracle (liboracle_kf.so) — TEST INFRASTRUCTURE.

Only the tests, the smoke check and the CPU-baseline leg of the bench load this module;
the product path never does.  The API mirrors the GPU session so a test can drive both
with the same inputs.  Parity with the reference itself is unpinned (see kf_oracle.h).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_kf.so")

_P = C.c_void_p
_I = C.c_int
_PD = C.POINTER(C.c_double)

_SIG = {
    "or_create": [_P, _P, C.POINTER(_P)], "or_destroy": [_P], "or_set_threads": [_I],
    "or_get_threads": [], "or_reset": [_P, _PD, _I], "or_reset_pose": [_P, _PD],
    "or_set_pose": [_P, _PD], "or_get_pose": [_P, _PD], "or_get_pose_eig": [_P, _PD],
    "or_set_pose_eig": [_P, _PD],
    "or_depth_to_vertex_f32": [_P, _P], "or_depth_to_vertex_u16": [_P, _P],
    "or_vertex_to_normal": [_P], "or_set_depth_undistortion": [_P, _P],
    "or_set_depth_filter": [_P, _I], "or_get_undistortion_map": [_P, _P], "or_track_icp": [_P, C.POINTER(_I)],
    "or_track_sdf": [_P, C.POINTER(_I)], "or_recover_pose": [_P, C.POINTER(_I)],
    "or_get_alignment_energy": [_P, _PD], "or_get_reduction": [_P, _PD],
    "or_icp_reduce_once": [_P, _I, _PD], "or_sdf_reduce_once": [_P, _I, _PD, _PD],
    "or_integrate": [_P], "or_raycast": [_P], "or_intensity_projection": [_P, _P], "or_frame_step_u16": [_P, _P, C.POINTER(_I)],
    "or_get_raycast": [_P, _P, _P], "or_set_raycast": [_P, _P, _P],
    "or_get_vertex_map": [_P, _I, _P], "or_get_normal_map": [_P, _I, _P],
    "or_set_vertex_normal_map": [_P, _I, _P, _P], "or_get_depth_map": [_P, _I, _P],
    "or_get_track_status": [_P, _I, _P], "or_copy_volume_to_host": [_P, _P, C.c_uint64],
    "or_copy_volume_from_host": [_P, _P, C.c_uint64], "or_get_pose_library_size": [_P, C.POINTER(_I)],
    "or_get_cum_twist": [_P, _PD], "or_mc_extract": [_P, C.c_float, _I, C.POINTER(C.c_uint32)],
    "or_mc_copy_vertices": [_P, _P, C.c_uint64], "or_mc_copy_base_level": [_P, _P, C.c_uint64],
    "or_mc_copy_normals": [_P, _P, C.c_uint64],
    "or_mc_extract_mesh": [_P, C.c_float, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)],
    "or_mc_copy_mesh": [_P, _P, _P, _P],
    "or_mc_export_stl": [_P, C.c_char_p], "or_mc_export_ply": [_P, C.c_char_p],
    "or_prefix_sum_u32": [_P, _P, C.c_uint64, C.POINTER(C.c_uint32)],
    "or_euler_xyz": [_PD, _PD], "or_se3_exp": [_PD, _PD], "or_solve_pinv6": [_PD, _PD, _PD],
    "or_solve_icp_guarded6": [_PD, _PD, _PD],
    "or_solve_ldlt6": [_PD, _PD, _PD], "or_mc_tables": [_P, _P, _P, _P, _P],
}

_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"oracle not built: {LIB_PATH} (make -C oracle)")
        lib = C.CDLL(LIB_PATH)
        for name, args in _SIG.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = None if name in ("or_euler_xyz", "or_se3_exp") else _I
        _lib = lib
    return _lib


def _pose_c(pose):
    m = np.asarray(pose, np.float64).reshape(4, 4)
    return (C.c_double * 16)(*m.flatten(order="F"))


def _pose_np(a):
    return np.array(list(a), np.float64).reshape(4, 4, order="F")


def _ok(st, what):
    if st != 0:
        raise RuntimeError(f"oracle {what} failed: {st}")


class Oracle:
    """FP64 oracle session mirroring oglfusionkinectv2_b200.GFusion."""

    def __init__(self, config, intrinsics):
        self.lib = load()
        self.configuration = config
        self.intrinsics = intrinsics
        self._cc = config.to_c()
        self._ci = intrinsics.to_c()
        h = C.c_void_p()
        _ok(self.lib.or_create(C.byref(self._cc), C.byref(self._ci), C.byref(h)), "create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self.lib.or_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def set_threads(n: int = 0):
        load().or_set_threads(n)

    @staticmethod
    def threads() -> int:
        return load().or_get_threads()

    def Reset(self, pose, deleteFlag=False):
        _ok(self.lib.or_reset(self._h, _pose_c(pose), int(deleteFlag)), "reset")

    def resetPose(self, pose):
        _ok(self.lib.or_reset_pose(self._h, _pose_c(pose)), "reset_pose")

    def setPose(self, pose):
        _ok(self.lib.or_set_pose(self._h, _pose_c(pose)), "set_pose")

    def getPose(self):
        a = (C.c_double * 16)()
        _ok(self.lib.or_get_pose(self._h, a), "get_pose")
        return _pose_np(a)

    def getPoseEig(self):
        a = (C.c_double * 16)()
        _ok(self.lib.or_get_pose_eig(self._h, a), "get_pose_eig")
        return _pose_np(a)

    def depthToVertex(self, depth):
        d = np.ascontiguousarray(depth)
        if d.dtype == np.uint16:
            _ok(self.lib.or_depth_to_vertex_u16(self._h, d.ctypes.data), "d2v")
        else:
            d = np.ascontiguousarray(d, np.float32)
            _ok(self.lib.or_depth_to_vertex_f32(self._h, d.ctypes.data), "d2v")

    def vertexToNormal(self):
        _ok(self.lib.or_vertex_to_normal(self._h), "v2n")

    def setDepthUndistortion(self, ir):
        """ir: (fx, fy, cx, cy, k1, k2, k3, p1, p2) of the IR camera, or None (off)."""
        if ir is None:
            _ok(self.lib.or_set_depth_undistortion(self._h, None), "undistortion")
            return
        a = (C.c_float * 9)(*[float(v) for v in ir])
        _ok(self.lib.or_set_depth_undistortion(self._h, a), "undistortion")

    def setDepthFilter(self, enable):
        _ok(self.lib.or_set_depth_filter(self._h, int(bool(enable))), "depth_filter")

    def getUndistortionMap(self):
        w, h = self._wh(0)
        m = np.empty((h, w), np.int32)
        _ok(self.lib.or_get_undistortion_map(self._h, m.ctypes.data), "undistortion_map")
        return m

    def Track(self) -> bool:
        t = C.c_int()
        _ok(self.lib.or_track_icp(self._h, C.byref(t)), "track")
        return bool(t.value)

    def TrackSDF(self) -> bool:
        t = C.c_int()
        _ok(self.lib.or_track_sdf(self._h, C.byref(t)), "track_sdf")
        return bool(t.value)

    def recoverPose(self) -> bool:
        t = C.c_int()
        _ok(self.lib.or_recover_pose(self._h, C.byref(t)), "recover")
        return bool(t.value)

    def integrate(self):
        _ok(self.lib.or_integrate(self._h), "integrate")

    def raycast(self):
        _ok(self.lib.or_raycast(self._h), "raycast")

    def intensityProjection(self):
        w, h = self._wh(0)
        m = np.empty((h, w, 4))
        _ok(self.lib.or_intensity_projection(self._h, m.ctypes.data), "intensity_projection")
        return m

    def frameStep(self, depth_u16) -> bool:
        d = np.ascontiguousarray(depth_u16, np.uint16)
        t = C.c_int()
        _ok(self.lib.or_frame_step_u16(self._h, d.ctypes.data, C.byref(t)), "frame_step")
        return bool(t.value)

    def alignmentEnergy(self) -> float:
        d = C.c_double()
        _ok(self.lib.or_get_alignment_energy(self._h, C.byref(d)), "ae")
        return d.value

    def getReduction(self):
        a = (C.c_double * 32)()
        _ok(self.lib.or_get_reduction(self._h, a), "reduction")
        return np.array(list(a))

    def icpReduceOnce(self, level):
        a = (C.c_double * 32)()
        _ok(self.lib.or_icp_reduce_once(self._h, level, a), "icp_reduce_once")
        return np.array(list(a))

    def _wh(self, level):
        return self.intrinsics.width >> level, self.intrinsics.height >> level

    def getVerts(self):
        w, h = self._wh(0)
        v = np.empty((h, w, 4)); n = np.empty((h, w, 4))
        _ok(self.lib.or_get_raycast(self._h, v.ctypes.data, n.ctypes.data), "get_raycast")
        return v

    def getNorms(self):
        w, h = self._wh(0)
        v = np.empty((h, w, 4)); n = np.empty((h, w, 4))
        _ok(self.lib.or_get_raycast(self._h, v.ctypes.data, n.ctypes.data), "get_raycast")
        return n

    def setRaycast(self, v, n):
        v = np.ascontiguousarray(v, np.float64); n = np.ascontiguousarray(n, np.float64)
        _ok(self.lib.or_set_raycast(self._h, v.ctypes.data, n.ctypes.data), "set_raycast")

    def getVertexMap(self, level=0):
        w, h = self._wh(level)
        v = np.empty((h, w, 4))
        _ok(self.lib.or_get_vertex_map(self._h, level, v.ctypes.data), "vmap")
        return v

    def getNormalMap(self, level=0):
        w, h = self._wh(level)
        v = np.empty((h, w, 4))
        _ok(self.lib.or_get_normal_map(self._h, level, v.ctypes.data), "nmap")
        return v

    def setVertexNormalMap(self, level, v, n):
        v = np.ascontiguousarray(v, np.float64); n = np.ascontiguousarray(n, np.float64)
        _ok(self.lib.or_set_vertex_normal_map(self._h, level, v.ctypes.data, n.ctypes.data), "set_vn")

    def getDepthImage(self, level=0):
        w, h = self._wh(level)
        d = np.empty((h, w))
        _ok(self.lib.or_get_depth_map(self._h, level, d.ctypes.data), "dmap")
        return d

    def getTrackStatus(self, level=0):
        w, h = self._wh(level)
        s = np.empty((h, w), np.int32)
        _ok(self.lib.or_get_track_status(self._h, level, s.ctypes.data), "status")
        return s

    def getVolumeRaw(self):
        from oglfusionkinectv2_b200.gfusion import volume_bytes
        raw = np.empty(volume_bytes(self.configuration), np.uint8)
        _ok(self.lib.or_copy_volume_to_host(self._h, raw.ctypes.data, raw.nbytes), "vol_out")
        return raw

    def setVolumeRaw(self, raw):
        raw = np.ascontiguousarray(raw, np.uint8)
        _ok(self.lib.or_copy_volume_from_host(self._h, raw.ctypes.data, raw.nbytes), "vol_in")

    def getVolume(self):
        from oglfusionkinectv2_b200.gfusion import decode_volume
        return decode_volume(self.getVolumeRaw(), self.configuration)

    def poseLibrarySize(self):
        n = C.c_int()
        _ok(self.lib.or_get_pose_library_size(self._h, C.byref(n)), "lib")
        return n.value

    def getCumTwist(self):
        a = (C.c_double * 6)()
        _ok(self.lib.or_get_cum_twist(self._h, a), "twist")
        return np.array(list(a))

    def mcExtract(self, iso=0.0, method=0) -> int:
        n = C.c_uint32()
        _ok(self.lib.or_mc_extract(self._h, iso, method, C.byref(n)), "mc")
        self._ntri = n.value
        return n.value

    def mcVertices(self):
        out = np.empty((3 * self._ntri, 4), np.float32)
        _ok(self.lib.or_mc_copy_vertices(self._h, out.ctypes.data, out.shape[0]), "mc_verts")
        return out

    def mcNormals(self):
        out = np.empty((3 * self._ntri, 4), np.float32)
        _ok(self.lib.or_mc_copy_normals(self._h, out.ctypes.data, out.shape[0]), "mc_normals")
        return out

    def mcMesh(self, iso=0.0):
        """Welded mesh: (positions n x 3, unit normals n x 3, indices t x 3)."""
        nv, nt = C.c_uint32(), C.c_uint32()
        _ok(self.lib.or_mc_extract_mesh(self._h, iso, C.byref(nv), C.byref(nt)), "mc_mesh")
        P = np.empty((nv.value, 3), np.float32)
        N = np.empty((nv.value, 3), np.float32)
        I = np.empty((nt.value, 3), np.uint32)
        _ok(self.lib.or_mc_copy_mesh(self._h, P.ctypes.data, N.ctypes.data, I.ctypes.data), "mc_mesh_copy")
        return P, N, I

    def mcBaseLevel(self):
        nx, ny, nz = self.configuration.volumeSize
        out = np.empty(nx * ny * nz, np.uint32)
        _ok(self.lib.or_mc_copy_base_level(self._h, out.ctypes.data, out.size), "mc_base")
        return out.reshape(nz, ny, nx)

    def exportMesh(self, path):
        _ok(self.lib.or_mc_export_stl(self._h, path.encode()), "stl")

    def exportPointCloud(self, path):
        _ok(self.lib.or_mc_export_ply(self._h, path.encode()), "ply")


def prefix_sum(arr: np.ndarray):
    a = np.ascontiguousarray(arr, np.uint32)
    out = np.empty_like(a)
    tot = C.c_uint32()
    _ok(load().or_prefix_sum_u32(a.ctypes.data, out.ctypes.data, a.size, C.byref(tot)), "scan")
    return out, tot.value


def euler_xyz(angles):
    a = (C.c_double * 3)(*angles)
    r = (C.c_double * 9)()
    load().or_euler_xyz(a, r)
    return np.array(list(r)).reshape(3, 3, order="F")


def se3_exp(xi):
    a = (C.c_double * 6)(*xi)
    r = (C.c_double * 16)()
    load().or_se3_exp(a, r)
    return _pose_np(r)


def solve_pinv6(Cm, b):
    Cc = (C.c_double * 36)(*np.asarray(Cm, np.float64).flatten())
    bb = (C.c_double * 6)(*b)
    x = (C.c_double * 6)()
    rank = load().or_solve_pinv6(Cc, bb, x)
    return np.array(list(x)), rank


def solve_icp_guarded6(Cm, b):
    """The ICP step with the rank guard: (x, directions kept)."""
    Cc = (C.c_double * 36)(*np.asarray(Cm, np.float64).flatten())
    bb = (C.c_double * 6)(*b)
    x = (C.c_double * 6)()
    kept = load().or_solve_icp_guarded6(Cc, bb, x)
    return np.array(list(x)), kept


def solve_ldlt6(Cm, b):
    Cc = (C.c_double * 36)(*np.asarray(Cm, np.float64).flatten())
    bb = (C.c_double * 6)(*b)
    x = (C.c_double * 6)()
    load().or_solve_ldlt6(Cc, bb, x)
    return np.array(list(x))


def mc_tables():
    edge = np.empty(256, np.uint16); tri = np.empty(4096, np.int8)
    nv = np.empty(256, np.uint8); nt = np.empty(256, np.uint8); off = np.empty(72, np.uint8)
    _ok(load().or_mc_tables(edge.ctypes.data, tri.ctypes.data, nv.ctypes.data, nt.ctypes.data,
                            off.ctypes.data), "tables")
    return edge, tri.reshape(256, 16), nv, nt, off.reshape(12, 6)
