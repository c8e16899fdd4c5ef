// kf_internal.cuh — shared internals of the B200 KinectFusion core (not part of the ABI).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/kf.h"

#define KF_MAX_LIBRARY 64         // pose library entries kept on the device
#define KF_TRACK_THREADS 256      // threads per block of the persistent tracking kernels
#define KF_BATCH_ICP_WAVE 32     // members per cooperative launch of the batched ICP
#define KF_MAX_TRACK_BLOCKS 1024  // upper bound of the persistent grid

// Words of 8 bytes between two ICP reduction sums: 1, so that a warp's atomics on the 32
// sums of a row fall on two 128-byte lines and coalesce (one sum per line measured slower:
// 32 separate L2 requests per block instead of two).
#define KF_ACC_STRIDE 1

// Device-side error word values (KfDevState::error).
#define KF_DEV_ERR_TIMEOUT 1

// Spin-wait budget of the software grid barrier, in SM clock cycles (~0.5 s at 1.9 GHz).
#define KF_BARRIER_SPIN_CYCLES (1000000000LL)

// Device control block: everything the per-frame step keeps resident between kernels.
// Poses are camera-to-world, column-major, FP64.
struct KfDevState {
  // ---- frame result: the bytes the host reads after every frame step ----
  double pose[16];      // m_pose
  int tracked;          // result of the last Track()/TrackSDF()
  int error;            // KF_DEV_ERR_* (sticky until the host clears it)
  int recover_found;    // result of the last recoverPose()
  int counter;          // kinect.cpp frame counter
  // ---- the rest of the resident state ----
  // derived FP32 forms of `pose`, kept in step with it by every writer (kf_store_pose)
  float pose_rows[12];  // rows of [R | t]
  float inv_rows[12];   // rows of [R^T | -R^T t]
  double pose_eig[16];  // m_pose_eig (the SDF tracker's own pose chain)
  double old_pose[16];  // pose at the start of the last tracking call
  double raycast_pose[16];  // pose of the last raycast (projective association, Q4 clear)
  double cum_twist[6];  // m_cumTwist
  double sums[32];      // last reduction row (FP64 sum of the per-block FP32 partials)
  double ae;            // alignment energy of the last iteration
  int lib_size;
  int need_recover;     // frame policy: tracking failed this frame
  int do_integrate;     // frame policy: integrate this frame
  int reset_window;     // kinect.cpp `reset` flag
  int iterations_run;   // ICP/SDF iterations executed by the last tracking call
  // grid barrier counters, each on its own 128-byte line (polled by every block while the
  // reduction atomics land elsewhere)
  alignas(128) unsigned barrier_count;      // grid barrier of the ICP launch
  alignas(128) unsigned sdf_barrier_count;  // grid barrier of the SDF launch
  // ICP reduction rows as fixed-point sums (value * 2^32, exact and order-independent),
  // three buffers used in turn by successive iterations of a launch (KF_ACC_STRIDE words
  // between sums)
  alignas(128) long long icp_acc[3][32][KF_ACC_STRIDE];
  // the persistent raycast sweep's row-segment queue: next segment, warps done (both zero
  // between launches: the sweep's last warp resets them)
  alignas(128) unsigned ray_queue[2];
  double icp_center_cam[3];  // ICP centre at the end of the last frame (camera frame)
  double lib_pose[KF_MAX_LIBRARY][16];  // pose library
};
// Bytes of KfDevState the host reads after a frame step (pose and result flags).
#define KF_STATE_RESULT_BYTES (offsetof(KfDevState, pose_rows))
static_assert(KF_STATE_RESULT_BYTES == 144, "frame result head: pose, tracked, error, recover_found, counter");

// Where the autotuner's timing launches write instead of the session's own buffers.
struct kf_scratch_target {
  void* vol;             // integrate: a copy of the volume
  uint32_t* bricks;      // and of the brick / super-brick flags
  uint32_t* supers;
  float4* out_v;         // raycast: vertex and normal maps
  float4* out_n;
  KfDevState* st_out;    // raycast: the control block that receives raycast_pose
};

struct kf_session {
  kf_config cfg{};
  kf_intrinsics intr{};
  // identity of the session's kernel arguments: uid is unique per created session, layout
  // changes whenever a buffer is (re)allocated or the configuration is set (batched steps
  // cache per-member argument tables)
  uint64_t uid = 0;
  uint64_t layout = 0;
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;

  // per 8^3 brick: bit 0 set when the brick (dilated by one voxel towards +x, +y, +z) may
  // hold a negative TSDF value; set by integrate, cleared by reset, rebuilt on upload
  uint32_t* d_bricks = nullptr;
  int bx = 0, by = 0, bz = 0;
  // per 64^3 super-brick (8^3 bricks; same allocation as d_bricks, after it): KF_BRICK_NEG
  // when some brick in it is NEG
  uint32_t* d_supers = nullptr;
  int sbx = 0, sby = 0, sbz = 0;
  int frames_since_rebuild = 0;  // integrates since the flags were last rebuilt exactly

  // volume: value plane then weight plane
  void* d_vol = nullptr;
  size_t vol_count = 0;
  size_t vol_value_bytes = 0;
  size_t vol_bytes = 0;

  // image pyramid
  int W[3] = {0, 0, 0}, H[3] = {0, 0, 0};
  uint16_t* d_depth_u16 = nullptr;  // upload staging (device)
  float* d_depth_f32_in = nullptr;  // float upload staging (device)
  float* d_depth[3] = {nullptr, nullptr, nullptr};
  float4* d_vertex[3] = {nullptr, nullptr, nullptr};
  float4* d_normal[3] = {nullptr, nullptr, nullptr};
  int32_t* d_status[3] = {nullptr, nullptr, nullptr};
  float4* d_ref_vertex = nullptr;
  float4* d_ref_normal = nullptr;
  float* d_sdf_rows = nullptr;  // persistent trackSDF rows, 8 floats per level-0 pixel
  float* d_partials = nullptr;  // [2][KF_MAX_TRACK_BLOCKS][32] (alternating by iteration)

  KfDevState* d_state = nullptr;
  KfDevState* h_state = nullptr;  // pinned mirror
  uint16_t* h_depth_pinned = nullptr;

  int track_blocks = 0;  // persistent grid of the tracking kernels

  // frame-step CUDA graphs: a ring of instances, each with its own events, so the stage
  // times can be read back without stalling the stream.  An event node costs ~5 us of a
  // ~0.43 ms frame, so only every stage_every-th slot's graph records the frame's start, its
  // four stage boundaries and its end (by default one slot in four); the others hold no
  // event node, and their end is recorded on the stream after the graph.
  static const int kRing = 4;
  cudaGraphExec_t frame_exec[kRing] = {};
  cudaEvent_t ring_ev[kRing][6] = {};
  int ring_pending[kRing] = {};  // slot holds an unread frame
  int ring_stages[kRing] = {};   // slot's graph records the stage boundaries
  int stage_every = 4;           // kf_set_stage_timing: 0 (none), 1, 2 or 4
  // asynchronous frame steps (kf_frame_step_u16_async): each step's result head is copied into
  // the pinned slot of its frame graph and read by the next call
  char* h_heads = nullptr;            // pinned, kRing * KF_STATE_RESULT_BYTES (first use)
  cudaEvent_t head_ev[kRing] = {};
  int async_pend = -1;                // slot of the step whose result is not read yet
  // the frame graphs' inputs: one staging frame per ring slot (slot k's graph reads frame
  // k), so a pipelined step can upload the next frame on copy_stream while one runs
  uint16_t* d_frame_ring = nullptr;   // kRing * W * H
  cudaStream_t copy_stream = nullptr; // created by the first pipelined step
  cudaEvent_t upload_ev[kRing] = {};
  int frame_kernels = 0;         // kernels in one frame graph
  uint64_t frames_run = 0;
  double stage_acc[6] = {0, 0, 0, 0, 0, 0};
  uint64_t stage_frames = 0;
  uint64_t launches = 0;         // kernels launched by this session

  // stage timing of the individual entry points
  cudaEvent_t ev[12] = {};
  float stage_ms[6] = {0, 0, 0, 0, 0, 0};
  bool timing = false;
  bool capturing = false;

  // marching cubes
  uint32_t* d_mc_base = nullptr;  // nx*ny*nz cubes: numTri | cubeIndex << 16
  std::vector<uint32_t*> d_mc_levels;  // level k >= 1, (P >> k)^3
  int mc_P = 0, mc_top = 0;
  float4* d_mc_vertices = nullptr;
  size_t mc_vertex_cap = 0;
  float4* d_mc_normals = nullptr;  // face normal of each soup vertex's triangle (w = 0)
  size_t mc_normal_cap = 0;
  // welded mesh (kf_mc_extract_mesh): one vertex per cut voxel edge, indexed triangles
  uint32_t* d_mesh_mask = nullptr;  // edge bits, 10 voxels x 3 axes per word
  size_t mesh_mask_cap = 0;
  uint32_t* d_mesh_scratch = nullptr;  // triangle counts/offsets, word offsets, scan scratch
  size_t mesh_scratch_cap = 0;
  float* d_mesh_pos = nullptr;  // 3 floats per vertex (metres)
  float* d_mesh_nrm = nullptr;  // 3 floats per vertex (unit)
  uint32_t* d_mesh_idx = nullptr;  // 3 per triangle
  size_t mesh_pos_cap = 0, mesh_nrm_cap = 0, mesh_idx_cap = 0;
  uint32_t mesh_vertices = 0, mesh_triangles = 0;
  int mesh_valid = 0;
  uint32_t mc_triangles = 0;
  int mc_valid = 0;
  uint32_t* d_mc_scratch = nullptr;  // level table / scan path verts, offsets, scan scratch
  size_t mc_scratch_words = 0;       // capacity of d_mc_scratch in bytes
  uint32_t* d_u32_scalar = nullptr;  // one device word for totals
  uint32_t* h_u32_scalar = nullptr;  // pinned

  float4* d_mip = nullptr;  // intensity-projection image, allocated on first use

  // launch shapes (kf_set_launch_shape / kf_autotune); every choice computes the same result
  int int_zc = 16;   // integrate: voxels per thread along z (8, 16, 32)
  int ray_rows = 4;  // raycast: tile rows of 32 pixels (2, 4, 8), or 1: persistent sweep

  // depth ingest before the pyramid (off by default): Kinect-v2 undistortion through a
  // source-index map, and the filter3D.cs validity filter; their output is d_depth_prep
  int undistort = 0;
  int depth_filter = 0;
  int32_t* d_undistort_map = nullptr;
  float* d_depth_prep = nullptr;
};

// ---------------------------------------------------------------------------------------
// error helpers
// A failing call's error is also taken off the runtime's per-thread error state, so that
// a later cudaGetLastError() (after a launch) does not report it again.
#define KF_CUDA_TRY(s, expr)                                                          \
  do {                                                                                \
    cudaError_t e_ = (expr);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      (s)->last_error = std::string(#expr) + ": " + cudaGetErrorString(e_);          \
      cudaGetLastError();                                                             \
      return KF_ERR_CUDA;                                                             \
    }                                                                                 \
  } while (0)

// ---------------------------------------------------------------------------------------
// storage policy: value/weight planes
template <int S>
struct Vox;

template <>
struct Vox<KF_STORAGE_F32F32> {
  typedef float V;
  typedef float Wt;
  static constexpr float kRawToF = 1.0f;
  __device__ static __forceinline__ float raw(const V* f, size_t i) { return __ldg(f + i); }
  __device__ static __forceinline__ float raw_nc(const V* f, size_t i) { return f[i]; }
  __device__ static __forceinline__ float weight(const Wt* w, size_t i) { return w[i]; }
  __device__ static __forceinline__ V encode_value(float F) { return F; }
  __device__ static __forceinline__ Wt encode_weight(float w) { return w; }
};

// A 16-bit integer as float and back without conversion instructions (exact): the integer
// in the low mantissa bits of 2^23, and a non-negative float below 2^16 truncated by an add
// of 2^23 rounded toward zero.
__device__ __forceinline__ float kf_u16_to_float(uint32_t w) { return __int_as_float(0x4B000000 | w) - 8388608.0f; }
__device__ __forceinline__ uint32_t kf_float_to_u16_trunc(float w) {
  return (uint32_t)__float_as_int(__fadd_rz(w, 8388608.0f)) & 0xFFFFu;  // 0 <= w <= 65535
}

template <>
struct Vox<KF_STORAGE_F16U16> {
  typedef __half V;
  typedef uint16_t Wt;
  static constexpr float kRawToF = 1.0f;
  __device__ static __forceinline__ float raw(const V* f, size_t i) { return __half2float(__ldg(f + i)); }
  __device__ static __forceinline__ float raw_nc(const V* f, size_t i) { return __half2float(f[i]); }
  __device__ static __forceinline__ float weight(const Wt* w, size_t i) { return kf_u16_to_float(w[i]); }
  __device__ static __forceinline__ V encode_value(float F) { return __float2half_rn(F); }
  __device__ static __forceinline__ Wt encode_weight(float w) {
    return (uint16_t)kf_float_to_u16_trunc(fminf(fmaxf(w, 0.0f), 65535.0f));
  }
};

template <>
struct Vox<KF_STORAGE_RG16I> {
  typedef int16_t V;
  typedef int16_t Wt;
  // vs() of integrate.cs:42 / raycast.cs:81: float(data.x) * 0.00003051944088f
  static constexpr float kRawToF = 0.00003051944088f;
  __device__ static __forceinline__ float raw(const V* f, size_t i) { return (float)__ldg(f + i); }
  __device__ static __forceinline__ float raw_nc(const V* f, size_t i) { return (float)f[i]; }
  __device__ static __forceinline__ float weight(const Wt* w, size_t i) { return (float)w[i]; }
  // set() of integrate.cs:45-50: int(F * 32766), int(w)
  __device__ static __forceinline__ V encode_value(float F) { return (int16_t)(int)(F * 32766.0f); }
  __device__ static __forceinline__ Wt encode_weight(float w) { return (int16_t)(int)w; }
};

// ---------------------------------------------------------------------------------------
// FP64 pose math (column-major 4x4, glm layout), host and device
__host__ __device__ inline void kf_mat4_mul(const double* a, const double* b, double* out) {
  double r[16];
  for (int c = 0; c < 4; ++c)
    for (int rr = 0; rr < 4; ++rr) {
      double s = 0;
      for (int k = 0; k < 4; ++k) s += a[k * 4 + rr] * b[c * 4 + k];
      r[c * 4 + rr] = s;
    }
  for (int i = 0; i < 16; ++i) out[i] = r[i];
}

// Inverse of a rigid transform [R t; 0 1]: [R^T, -R^T t].
__host__ __device__ inline void kf_rigid_inverse(const double* T, double* out) {
  double r[16];
  for (int c = 0; c < 3; ++c)
    for (int rr = 0; rr < 3; ++rr) r[c * 4 + rr] = T[rr * 4 + c];
  for (int rr = 0; rr < 3; ++rr)
    r[12 + rr] = -(r[rr] * T[12] + r[4 + rr] * T[13] + r[8 + rr] * T[14]);
  r[3] = r[7] = r[11] = 0;
  r[15] = 1;
  for (int i = 0; i < 16; ++i) out[i] = r[i];
}

// glm::eulerAngleXYZ(t1,t2,t3) = Rx(t1) * Ry(t2) * Rz(t3) (used at gFusion.cpp:700),
// written out from the three elementary rotations; column-major 3x3.
__host__ __device__ inline void kf_euler_xyz_from_sincos(double sa, double ca, double sb, double cb, double sc,
                                                         double cc, double* R) {
  // column 0
  R[0] = cb * cc;
  R[1] = ca * sc + sa * sb * cc;
  R[2] = sa * sc - ca * sb * cc;
  // column 1
  R[3] = -cb * sc;
  R[4] = ca * cc - sa * sb * sc;
  R[5] = sa * cc + ca * sb * sc;
  // column 2
  R[6] = sb;
  R[7] = -sa * cb;
  R[8] = ca * cb;
}

__host__ __device__ inline void kf_euler_xyz(double a, double b, double c, double* R) {
  double sa, ca, sb, cb, sc, cc;
  sincos(a, &sa, &ca);
  sincos(b, &sb, &cb);
  sincos(c, &sc, &cc);
  kf_euler_xyz_from_sincos(sa, ca, sb, cb, sc, cc, R);
}

// exp of Twist(xi) (gFusion.cpp:811-833): closed-form SE(3) exponential, xi = (w, v).
__host__ __device__ inline void kf_se3_exp(const double* xi, double* T) {
  const double w0 = xi[0], w1 = xi[1], w2 = xi[2];
  const double th2 = w0 * w0 + w1 * w1 + w2 * w2;
  const double th = sqrt(th2);
  double A, B, C;
  if (th < 1e-6) {
    A = 1 - th2 / 6 + th2 * th2 / 120;
    B = 0.5 - th2 / 24 + th2 * th2 / 720;
    C = 1.0 / 6 - th2 / 120 + th2 * th2 / 5040;
  } else {
    double s, c;
    sincos(th, &s, &c);
    A = s / th;
    B = (1 - c) / th2;
    C = (th - s) / (th2 * th);
  }
  // [w]x column-major
  const double W[9] = {0, w2, -w1, -w2, 0, w0, w1, -w0, 0};
  double W2[9];
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += W[k * 3 + r] * W[c * 3 + k];
      W2[c * 3 + r] = s;
    }
  double R[9], V[9];
  for (int i = 0; i < 9; ++i) {
    double I = (i % 4 == 0) ? 1.0 : 0.0;
    R[i] = I + A * W[i] + B * W2[i];
    V[i] = I + B * W[i] + C * W2[i];
  }
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) T[c * 4 + r] = R[c * 3 + r];
  for (int r = 0; r < 3; ++r) T[12 + r] = V[r] * xi[3] + V[3 + r] * xi[4] + V[6 + r] * xi[5];
  T[3] = T[7] = T[11] = 0;
  T[15] = 1;
}

// Write m_pose and its FP32 forms (used by integrate and raycast).
__host__ __device__ inline void kf_store_pose(KfDevState* st, const double* P) {
  for (int k = 0; k < 16; ++k) st->pose[k] = P[k];
  double I[16];
  kf_rigid_inverse(P, I);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 4; ++c) {
      st->pose_rows[r * 4 + c] = (float)P[c * 4 + r];
      st->inv_rows[r * 4 + c] = (float)I[c * 4 + r];
    }
}

// FP64 Cholesky solve of the 6x6 SPD normal equations.  Returns 0 and x = 0 when a pivot
// is not positive (rank-deficient C, where the reference's JacobiSVD would return the
// minimum-norm solution; an all-zero system gives x = 0 in both).
__host__ __device__ inline int kf_cholesky6(const double* C, const double* b, double* x) {
  double L[36];
  for (int i = 0; i < 36; ++i) L[i] = 0;
  double dmax = 0;
  for (int i = 0; i < 6; ++i) dmax = fmax(dmax, fabs(C[i * 7]));
  const double eps = 1e-13 * dmax;
  for (int j = 0; j < 6; ++j) {
    double d = C[j * 7];
    for (int k = 0; k < j; ++k) d -= L[j * 6 + k] * L[j * 6 + k];
    if (!(d > eps)) {
      for (int i = 0; i < 6; ++i) x[i] = 0;
      return 0;
    }
    double ljj = sqrt(d);
    L[j * 7] = ljj;
    for (int i = j + 1; i < 6; ++i) {
      double v = C[i * 6 + j];
      for (int k = 0; k < j; ++k) v -= L[i * 6 + k] * L[j * 6 + k];
      L[i * 6 + j] = v / ljj;
    }
  }
  double y[6];
  for (int i = 0; i < 6; ++i) {
    double v = b[i];
    for (int k = 0; k < i; ++k) v -= L[i * 6 + k] * y[k];
    y[i] = v / L[i * 7];
  }
  for (int i = 5; i >= 0; --i) {
    double v = y[i];
    for (int k = i + 1; k < 6; ++k) v -= L[k * 6 + i] * x[k];
    x[i] = v / L[i * 7];
  }
  return 1;
}

// LDL^T solve (C.ldlt().solve(b), gFusion.cpp:902), unpivoted; NaN in, NaN out.
__host__ __device__ inline void kf_ldlt6(const double* C, const double* b, double* x) {
  double L[36], D[6];
  for (int i = 0; i < 36; ++i) L[i] = 0;
  for (int j = 0; j < 6; ++j) {
    double d = C[j * 7];
    for (int k = 0; k < j; ++k) d -= L[j * 6 + k] * L[j * 6 + k] * D[k];
    D[j] = d;
    L[j * 7] = 1;
    for (int i = j + 1; i < 6; ++i) {
      double v = C[i * 6 + j];
      for (int k = 0; k < j; ++k) v -= L[i * 6 + k] * L[j * 6 + k] * D[k];
      L[i * 6 + j] = v / d;
    }
  }
  double y[6];
  for (int i = 0; i < 6; ++i) {
    double v = b[i];
    for (int k = 0; k < i; ++k) v -= L[i * 6 + k] * y[k];
    y[i] = v;
  }
  for (int i = 0; i < 6; ++i) y[i] /= D[i];
  for (int i = 5; i >= 0; --i) {
    double v = y[i];
    for (int k = i + 1; k < 6; ++k) v -= L[k * 6 + i] * x[k];
    x[i] = v;
  }
}

// makeJTJ (gFusion.h:472-487): symmetric 6x6 from the 21 upper-triangular sums.
__host__ __device__ inline void kf_make_jtj(const double* v21, double* C) {
  int k = 0;
  for (int i = 0; i < 6; ++i)
    for (int j = i; j < 6; ++j) {
      C[i * 6 + j] = v21[k];
      C[j * 6 + i] = v21[k];
      ++k;
    }
}

// 1 / sqrt(d) to FP64 precision without a divide or square root: an FP32 estimate refined
// by two Newton-Raphson steps for f(y) = 1/y^2 - d, y <- y (3 - d y^2) / 2; each step
// roughly doubles the correct bits (22 -> 44 -> FP64 rounding).  Outside FP32's normal
// range the estimate comes from 1 / sqrt(d) directly.
__device__ __forceinline__ double kf_rsqrt_newton(double d) {
  double y = (d > 1e-30 && d < 1e30) ? (double)rsqrtf((float)d) : 1.0 / sqrt(d);
  const double h = 0.5 * d;
  y = y * fma(-h * y, y, 1.5);
  y = y * fma(-h * y, y, 1.5);
  return y;
}

// sin and cos; below |x| = 0.25 by their Taylor series through x^11 and x^12 (the first
// omitted terms are < 3e-18 relative), which is the whole range of a Gauss-Newton step.
__device__ __forceinline__ void kf_sincos_step(double x, double* s, double* c) {
  if (fabs(x) < 0.25) {
    const double x2 = x * x;
    double ps = -1.0 / 39916800.0;                 // -1/11!
    ps = fma(ps, x2, 1.0 / 362880.0);              //  1/9!
    ps = fma(ps, x2, -1.0 / 5040.0);               // -1/7!
    ps = fma(ps, x2, 1.0 / 120.0);                 //  1/5!
    ps = fma(ps, x2, -1.0 / 6.0);                  // -1/3!
    double pc = 1.0 / 479001600.0;                 //  1/12!
    pc = fma(pc, x2, -1.0 / 3628800.0);            // -1/10!
    pc = fma(pc, x2, 1.0 / 40320.0);               //  1/8!
    pc = fma(pc, x2, -1.0 / 720.0);                // -1/6!
    pc = fma(pc, x2, 1.0 / 24.0);                  //  1/4!
    pc = fma(pc, x2, -0.5);                        // -1/2!
    *s = fma(x * x2, ps, x);
    *c = fma(x2, pc, 1.0);
  } else {
    sincos(x, s, c);
  }
}

// kf_cholesky6 by one thread: C given as the 21 upper-triangular values of reduce.cs rows
// 7..27 (row-major), b as 6 values, both read from shared or global memory.  Returns
// whether C was numerically positive definite (x = 0 otherwise, as kf_cholesky6).  Fully
// unrolled in registers: the dependent chain is six pivots (kf_rsqrt_newton: multiplies,
// no divides) and twelve substitution steps, with no shuffles between lanes (measured
// 11 us per frame faster than a lane-per-row warp factorisation, whose every pivot and
// substitution step waited on a shuffle).
__device__ __forceinline__ bool kf_cholesky6_thread(const double* v21, const double* b, double* x) {
  double L[6][6];  // lower triangle
  double inv[6];
  double dmax = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) dmax = fmax(dmax, fabs(v21[6 * i - (i * (i - 1)) / 2]));
  const double eps = 1e-13 * dmax;
  bool spd = true;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    double dj = v21[6 * j - (j * (j - 1)) / 2];
#pragma unroll
    for (int k = 0; k < j; ++k) dj = fma(-L[j][k], L[j][k], dj);
    spd = spd && (dj > eps);
    const double r = kf_rsqrt_newton(spd ? dj : 1.0);
    inv[j] = r;
    L[j][j] = dj * r;
#pragma unroll
    for (int i = j + 1; i < 6; ++i) {
      double v = v21[6 * j - (j * (j - 1)) / 2 + (i - j)];
#pragma unroll
      for (int k = 0; k < j; ++k) v = fma(-L[i][k], L[j][k], v);
      L[i][j] = v * r;
    }
  }
  double y[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double v = b[i];
#pragma unroll
    for (int k = 0; k < i; ++k) v = fma(-L[i][k], y[k], v);
    y[i] = v * inv[i];
  }
#pragma unroll
  for (int i = 5; i >= 0; --i) {
    double v = y[i];
#pragma unroll
    for (int k = i + 1; k < 6; ++k) v = fma(-L[k][i], x[k], v);
    x[i] = spd ? v * inv[i] : 0.0;
  }
  if (!spd) {
#pragma unroll
    for (int i = 0; i < 6; ++i) x[i] = 0.0;
  }
  return spd;
}

// ---------------------------------------------------------------------------------------
// ICP rank guard (Q22).  The reference solves the 6x6 normal equations with JacobiSVD
// (gFusion.cpp:696-697), which returns the minimum-norm least-squares step, dropping the
// singular values below 6 * machine epsilon of the largest.  That cut sits far below the
// rounding of FP32 sums, so a view of a single plane (rank 3: in-plane motion and rotation
// about the normal are unobservable) yields steps made of rounding noise.  This build uses
// the same rule with the cut at KF_ICP_RANK_TAU of the largest eigenvalue of the
// world-frame C: x = sum_{l_i >= tau l_max} v_i (v_i . b) / l_i.  A full-rank system keeps
// every direction, and x = C^-1 b; well-posed views have l_min / l_max near 1e-3.
#define KF_ICP_RANK_TAU 1e-5

// Cyclic Jacobi eigen-decomposition of a symmetric 6x6 matrix (row-major): A is
// overwritten by its diagonalised form, V receives the eigenvectors in its columns.  At
// most 32 sweeps; stops when the off-diagonal mass is below 1e-30 of the diagonal's.
__device__ inline void kf_jacobi_eigen6(double* A, double* V) {
  #pragma unroll 1
  for (int i = 0; i < 36; ++i) V[i] = (i % 7 == 0) ? 1.0 : 0.0;
  #pragma unroll 1
  for (int sweep = 0; sweep < 32; ++sweep) {
    double off = 0.0, diag = 0.0;
    #pragma unroll 1
    for (int p = 0; p < 6; ++p) {
      diag += A[p * 7] * A[p * 7];
      #pragma unroll 1
      for (int q = p + 1; q < 6; ++q) off += A[p * 6 + q] * A[p * 6 + q];
    }
    if (!(off > 1e-30 * diag)) break;
    #pragma unroll 1
    for (int p = 0; p < 6; ++p)
      #pragma unroll 1
      for (int q = p + 1; q < 6; ++q) {
        const double apq = A[p * 6 + q];
        if (apq == 0.0) continue;
        const double theta = (A[q * 7] - A[p * 7]) / (2.0 * apq);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        #pragma unroll 1
        for (int k = 0; k < 6; ++k) {
          const double akp = A[k * 6 + p], akq = A[k * 6 + q];
          A[k * 6 + p] = c * akp - s * akq;
          A[k * 6 + q] = s * akp + c * akq;
        }
        #pragma unroll 1
        for (int k = 0; k < 6; ++k) {
          const double apk = A[p * 6 + k], aqk = A[q * 6 + k];
          A[p * 6 + k] = c * apk - s * aqk;
          A[q * 6 + k] = s * apk + c * aqk;
        }
        #pragma unroll 1
        for (int k = 0; k < 6; ++k) {
          const double vkp = V[k * 6 + p], vkq = V[k * 6 + q];
          V[k * 6 + p] = c * vkp - s * vkq;
          V[k * 6 + q] = s * vkp + c * vkq;
        }
      }
  }
}

// The rank-guarded step of a world-frame system C x = b (C row-major 6x6), as described
// at KF_ICP_RANK_TAU.  Returns the number of eigen-directions kept.
__device__ inline int kf_icp_guarded_solve(const double* C, const double* b, double* x, double* A,
                                                    double* V) {
  // A, V: 36 doubles of scratch each
  #pragma unroll 1
  for (int i = 0; i < 36; ++i) A[i] = C[i];
  kf_jacobi_eigen6(A, V);
  double lmax = 0.0;
  #pragma unroll 1
  for (int k = 0; k < 6; ++k) lmax = fmax(lmax, A[k * 7]);
  #pragma unroll 1
  for (int i = 0; i < 6; ++i) x[i] = 0.0;
  int kept = 0;
  #pragma unroll 1
  for (int k = 0; k < 6; ++k) {
    const double l = A[k * 7];
    if (!(l > 0.0 && l >= KF_ICP_RANK_TAU * lmax)) continue;
    ++kept;
    double vb = 0.0;
    #pragma unroll 1
    for (int i = 0; i < 6; ++i) vb += V[i * 6 + k] * b[i];
    #pragma unroll 1
    for (int i = 0; i < 6; ++i) x[i] += V[i * 6 + k] * vb / l;
  }
  return kept;
}

// The rank-guarded step from the centred sums about c, in the world frame: b = M^T b',
// C = M^T C' M with M = [[I, -[c]x], [0, I]], then kf_icp_guarded_solve.  It runs only for
// degenerate views; its matrices live in the caller's scratch sm (6 * 36 + 12 doubles,
// shared memory) and its loops are kept rolled, so that this rare path does not raise the
// register pressure of the kernel around it (measured: unrolled, it slowed every ICP
// iteration).
__device__ inline void kf_icp_world_guarded_step(const double* v21c, const double* bc, const double* c, double* out,
                                                 double* sm) {
  const double cx = c[0], cy = c[1], cz = c[2];
  double* Cp = sm;
  double* Mx = sm + 36;
  double* T = sm + 72;
  double* Cw = sm + 108;
  double* bw = sm + 216;
  double* xw = sm + 222;
  kf_make_jtj(v21c, Cp);
  #pragma unroll 1
  for (int k = 0; k < 36; ++k) Mx[k] = (k % 7 == 0) ? 1.0 : 0.0;
  // -[c]x in rows 0..2, columns 3..5
  Mx[0 * 6 + 4] = cz;  Mx[0 * 6 + 5] = -cy;
  Mx[1 * 6 + 3] = -cz; Mx[1 * 6 + 5] = cx;
  Mx[2 * 6 + 3] = cy;  Mx[2 * 6 + 4] = -cx;
  #pragma unroll 1
  for (int r = 0; r < 6; ++r) {
    double v = 0.0;
    #pragma unroll 1
    for (int k = 0; k < 6; ++k) v += Mx[k * 6 + r] * bc[k];
    bw[r] = v;
  }
  #pragma unroll 1
  for (int r = 0; r < 6; ++r)
    #pragma unroll 1
    for (int cc = 0; cc < 6; ++cc) {
      double v = 0.0;
      #pragma unroll 1
      for (int k = 0; k < 6; ++k) v += Cp[r * 6 + k] * Mx[k * 6 + cc];
      T[r * 6 + cc] = v;
    }
  #pragma unroll 1
  for (int r = 0; r < 6; ++r)
    #pragma unroll 1
    for (int cc = 0; cc < 6; ++cc) {
      double v = 0.0;
      #pragma unroll 1
      for (int k = 0; k < 6; ++k) v += Mx[k * 6 + r] * T[k * 6 + cc];
      Cw[r * 6 + cc] = v;
    }
  kf_icp_guarded_solve(Cw, bw, xw, sm + 144, sm + 180);
  #pragma unroll 1
  for (int k = 0; k < 6; ++k) out[k] = xw[k];
}



// The rank guard's check by one thread, in FP32 (run in warp 1 beside warp 0's FP64
// solve): 1 when the world-frame C provably keeps every direction under
// KF_ICP_RANK_TAU, so that the centred system's Cholesky solution is the guarded step.
// v21c: reduce.cs rows 7..27 of the centred J' = [n, (p - c) x n] about c, i.e.
// C' = M^-T C M^-1 with M: t' = t - [c]x w.  Bounds: l_min >= 1 / trace(C^-1),
// l_max <= trace(C), with trace(C) = sum_i m_i^T C' m_i (m_i = M e_i) and
// (C^-1)_ii = |L'^-1 M^-T e_i|^2 for C' = L' L'^T.  A factor of 2 covers FP32's rounding:
// the cut is 1e-5, far above FP32's 6e-8, and a Cholesky too ill-conditioned for FP32 gives
// a large trace (or a non-positive pivot) and fails the check, leaving the decision to the
// exact FP64 path.
__device__ __forceinline__ int kf_icp_rank_check_thread(const double* v21c, const double* c) {
  float A[6][6];
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = i; j < 6; ++j) {
      A[i][j] = (float)v21c[6 * i - (i * (i - 1)) / 2 + (j - i)];
      A[j][i] = A[i][j];
    }
  float L[6][6], id[6];
  bool spd = true;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    float dj = A[j][j];
#pragma unroll
    for (int k = 0; k < j; ++k) dj = fmaf(-L[j][k], L[j][k], dj);
    spd = spd && (dj > 0.0f);
    const float r = rsqrtf(spd ? dj : 1.0f);
    id[j] = r;
    L[j][j] = dj * r;
#pragma unroll
    for (int i = j + 1; i < 6; ++i) {
      float v = A[i][j];
#pragma unroll
      for (int k = 0; k < j; ++k) v = fmaf(-L[i][k], L[j][k], v);
      L[i][j] = v * r;
    }
  }
  if (!spd) return 0;
  const float cx = (float)c[0], cy = (float)c[1], cz = (float)c[2];
  float tinv = 0.0f, tr = 0.0f;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    const int k3 = i < 3 ? i : i - 3;
    // c x e_k3
    const float ck0 = k3 == 0 ? 0.0f : (k3 == 1 ? -cz : cy);
    const float ck1 = k3 == 0 ? cz : (k3 == 1 ? 0.0f : -cx);
    const float ck2 = k3 == 0 ? -cy : (k3 == 1 ? cx : 0.0f);
    float z[6];
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      float v = j == i ? 1.0f : 0.0f;
      if (i < 3 && j >= 3) v = -(j == 3 ? ck0 : (j == 4 ? ck1 : ck2));
#pragma unroll
      for (int k = 0; k < j; ++k) v = fmaf(-L[j][k], z[k], v);
      z[j] = v * id[j];
      tinv = fmaf(z[j], z[j], tinv);
    }
    if (i < 3) {
      tr += A[i][i];
    } else {
      const float m0 = -ck0, m1 = -ck1, m2 = -ck2;
      const float r0 = A[0][0] * m0 + A[0][1] * m1 + A[0][2] * m2;
      const float r1 = A[1][0] * m0 + A[1][1] * m1 + A[1][2] * m2;
      const float r2 = A[2][0] * m0 + A[2][1] * m1 + A[2][2] * m2;
      tr += m0 * r0 + m1 * r1 + m2 * r2 + 2.0f * (m0 * A[0][i] + m1 * A[1][i] + m2 * A[2][i]) + A[i][i];
    }
  }
  return (tinv * tr * (2.0f * (float)KF_ICP_RANK_TAU) <= 1.0f) ? 1 : 0;
}

// ---------------------------------------------------------------------------------------
// Grid barrier for the persistent (cooperatively launched) tracking kernels: every block
// calls kf_grid_sync after writing its partial sums and continues once all have.  Every
// wait is bounded: after KF_BARRIER_SPIN_CYCLES the block records KF_DEV_ERR_TIMEOUT in
// st->error and stops; callers leave their loops when kf_grid_sync returns false, and a
// block that sees another block's error stops too.
__device__ __forceinline__ unsigned kf_ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// The bar.sync before thread 0's gpu-scope release orders every thread's earlier stores
// of the block before it; an acquirer that observes the release sees them.
// Grid barrier over a counter that only grows during a launch (the launcher zeroes it):
// every block adds one and waits until `target` arrivals in total.  One release
// reduction per block and no reset step.  The wait gives up after `budget` clock64 cycles,
// records KF_DEV_ERR_TIMEOUT in *error and returns false; a block that sees an error
// recorded by another block returns false as well.
__device__ inline bool kf_grid_sync_bounded(int* error, unsigned* counter, unsigned target, int* s_flag,
                                            long long budget) {
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(counter) : "memory");
    int ok = 1;
    const long long t0 = clock64();
    while (kf_ld_acquire_gpu(counter) < target) {
      if (*(volatile int*)error) { ok = 0; break; }
      if (clock64() - t0 > budget) {
        atomicExch(error, KF_DEV_ERR_TIMEOUT);
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
    if (*(volatile int*)error) ok = 0;
    *s_flag = ok;
  }
  __syncthreads();
  return *s_flag != 0;
}

// The tracking kernels' barrier: errors go to the session's sticky device error word.
__device__ __forceinline__ bool kf_grid_sync(KfDevState* st, unsigned* counter, unsigned target, int* s_flag) {
  return kf_grid_sync_bounded(&st->error, counter, target, s_flag, KF_BARRIER_SPIN_CYCLES);
}

// A pose passed in by the caller must be finite (NaN or Inf would poison the device state).
inline bool kf_pose_is_finite(const double* p) {
  for (int k = 0; k < 16; ++k)
    if (!std::isfinite(p[k])) return false;
  return true;
}

// ---------------------------------------------------------------------------------------
// batched frame steps (kf_batch.cu): sessions of equal image size, storage and J^T J form
// step together, one launch per stage; per-session arguments live in a device table that
// is rebuilt only when the membership changes.
struct kf_batch {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  int cap = 0;
  std::string last_error;
  std::vector<kf_session*> members;  // membership of the uploaded tables
  std::vector<std::pair<uint64_t, uint64_t>> member_keys;  // (uid, layout) of each member
  // argument tables: pinned host copy and device copy
  char* h_table = nullptr;
  char* d_table = nullptr;
  size_t table_cap = 0, table_used = 0;
  // device pointers into d_table, set by the kf_batch_prepare_* functions
  KfDevState* const* states = nullptr;
  const void* pyr_args = nullptr;
  const void* vn_args = nullptr;
  int vn_pixels = 0, W1 = 0, H1 = 0;
  const void* icp_args = nullptr;
  int icp_blocks = 0;
  // the batched ICP runs in waves of at most KF_BATCH_ICP_WAVE members, each wave one
  // cooperative launch of every block (more blocks per member: 2.66 -> 2.41 ms per 64-session
  // step on the B200); member e of wave w is table entry KF_BATCH_ICP_WAVE * w + e
  const uint32_t* icp_wave_map[(255 + KF_BATCH_ICP_WAVE - 1) / KF_BATCH_ICP_WAVE] = {};
  int icp_waves = 0;
  const void* sdf_args = nullptr;
  const uint32_t* sdf_map = nullptr;
  int sdf_blocks = 0;
  const void* int_args = nullptr;
  const uint32_t* int_prefix = nullptr;
  uint32_t int_blocks = 0;
  const void* ray_args = nullptr;
  // launch shapes of the batched integrate and raycast (kf_batch_set_launch_shape /
  // kf_batch_autotune); the integrate block prefix in the tables depends on int_zc
  int int_zc = 16;
  int ray_rows = 4;
  // Steps use two slots in turn, so that an asynchronous step can be enqueued while the
  // previous one is still running: each slot has its gathered frame results
  // (h_heads + slot * cap * KF_STATE_RESULT_BYTES, pinned), its input pointer list and its
  // stage events.  The device buffers are shared (the stream orders them).
  char* d_heads = nullptr;
  char* h_heads = nullptr;                // pinned, 2 * cap * KF_STATE_RESULT_BYTES
  const uint16_t** h_inputs = nullptr;    // pinned, 2 * cap
  const uint16_t** d_inputs = nullptr;    // device, cap
  cudaEvent_t ev[2][7] = {};  // stage boundaries [0..5], results copied [6]
  // the enqueued step whose results are not read yet (-1: none), and its members
  int pend_slot = -1;
  std::vector<kf_session*> pend_members;
  // the last step whose results were read: its slot and member count
  int last_slot = 0;
  int last_n = 0;
  std::vector<int32_t> last_tracked;
  float stage_ms[5] = {0, 0, 0, 0, 0};
  uint64_t steps = 0;
  uint64_t launches = 0;
  // per-slot CUDA graphs of a device-frame step (input addresses read from the slot's
  // pinned list at replay), valid while the tables and launch shapes they were captured
  // with are (graph_n members); kernels per replay
  cudaGraphExec_t step_exec[2] = {nullptr, nullptr};
  int graph_n[2] = {0, 0};
  uint64_t graph_kernels[2] = {0, 0};
  uint64_t graph_replays = 0;
};

// Reserves `bytes` in the host table (256-byte aligned); returns the matching device
// pointer, or nullptr when the table is full.
inline void* kf_batch_table(kf_batch* b, size_t bytes, void** host) {
  const size_t off = (b->table_used + 255) & ~(size_t)255;
  if (off + bytes > b->table_cap) return nullptr;
  b->table_used = off + bytes;
  *host = b->h_table + off;
  return b->d_table + off;
}

// Splits `total` co-resident blocks of a persistent tracking kernel evenly over the
// batch's members: word = entry << 24 | blocks of the entry << 12 | index.
// The block map of members e0 .. e1-1 over `total` blocks: entry k = (member << 24 | the
// member's block count << 12 | the block's index among them), the members' blocks in order.
inline int kf_batch_block_map_range(kf_batch* b, int total, int e0, int e1, const uint32_t** d_map) {
  const int n = e1 - e0;
  if (n > total || e1 > 255 || total / n > 4095) return KF_ERR_CAPACITY;
  uint32_t* h = nullptr;
  *d_map = static_cast<const uint32_t*>(kf_batch_table(b, (size_t)total * 4, reinterpret_cast<void**>(&h)));
  if (!*d_map) return KF_ERR_CAPACITY;
  int k = 0;
  for (int e = 0; e < n; ++e) {
    const int cnt = total / n + (e < total % n ? 1 : 0);
    for (int i = 0; i < cnt; ++i) h[k++] = (uint32_t)(e0 + e) << 24 | (uint32_t)cnt << 12 | (uint32_t)i;
  }
  return KF_OK;
}

inline int kf_batch_block_map(kf_batch* b, int total, const uint32_t** d_map) {
  return kf_batch_block_map_range(b, total, 0, (int)b->members.size(), d_map);
}

int kf_batch_prepare_pyramid(kf_batch* b);
int kf_batch_prepare_icp(kf_batch* b);
int kf_batch_prepare_sdf(kf_batch* b);
// `over` (one per member, or null): the autotuner's scratch targets (ungated integrate)
int kf_batch_prepare_integrate(kf_batch* b, const kf_scratch_target* over);
int kf_batch_prepare_raycast(kf_batch* b, const kf_scratch_target* over);
int kf_batch_launch_pyramid(kf_batch* b, int n, const uint16_t* const* d_inputs);
int kf_batch_launch_icp(kf_batch* b);
int kf_batch_launch_sdf_recover(kf_batch* b);
int kf_batch_launch_integrate(kf_batch* b);
int kf_batch_launch_raycast(kf_batch* b, int n);

// Zero the barrier counter and the ICP sum buffers of a state block before a tracking launch.
inline cudaError_t kf_clear_icp_words(KfDevState* st, cudaStream_t stream) {
  const size_t b0 = offsetof(KfDevState, barrier_count);
  const size_t b1 = offsetof(KfDevState, icp_acc) + sizeof(st->icp_acc);
  return cudaMemsetAsync(reinterpret_cast<char*>(st) + b0, 0, b1 - b0, stream);
}

// Count kernels launched outside graph capture (captured graphs are counted per replay).
inline void kf_note_launch(kf_session* s, int n = 1) {
  if (!s->capturing) s->launches += (uint64_t)n;
}

// ---------------------------------------------------------------------------------------
// launchers (one per .cu file)
int kf_launch_pyramid(kf_session* s, const uint16_t* d_u16, const float* d_f32);
int kf_launch_depth_ingest(kf_session* s, const uint16_t* d_u16, const float* d_f32);
int kf_launch_undistort_map(kf_session* s, const kf_ir_camera& ir);
int kf_launch_vertex(kf_session* s);
int kf_launch_normal(kf_session* s);
// clear_tracking_words: also zero the barrier counters and ICP sums (frame step)
int kf_launch_vertex_normal(kf_session* s, bool clear_tracking_words = false);
// words_zero: the barrier counter and sum buffers are known to be zero (no memset)
int kf_launch_icp(kf_session* s, int frame_policy, bool words_zero = false);
int kf_launch_sdf(kf_session* s, int recover, int gated, int frame_policy, bool counter_zero = false);
int kf_launch_sdf_policy(kf_session* s);
int kf_launch_integrate(kf_session* s, int gated);
int kf_launch_raycast(kf_session* s);
int kf_launch_integrate_shape(kf_session* s, int gated, int zc, const kf_scratch_target* t);
int kf_launch_raycast_shape(kf_session* s, int rows, const kf_scratch_target* t);
inline bool kf_valid_int_zc(int zc) { return zc == 8 || zc == 16 || zc == 32; }
// raycast shapes: 32 x rows tiles (2, 4, 8), or 1 = the persistent sweep (sessions only)
inline bool kf_valid_ray_rows(int r) { return r == 1 || r == 2 || r == 4 || r == 8; }
inline bool kf_valid_batch_ray_rows(int r) { return r == 2 || r == 4 || r == 8; }
constexpr int kf_tune_int_zc[3] = {8, 16, 32};
constexpr int kf_tune_ray_rows[4] = {1, 2, 4, 8};        // session autotuner
constexpr int kf_tune_batch_ray_rows[3] = {2, 4, 8};     // batch autotuner
// Scratch copies of a session's volume, brick flags and control block plus scratch maps,
// for timing launches without touching the session (kf_capi.cu).
int kf_scratch_alloc(kf_session* s, kf_scratch_target* t);
void kf_scratch_free(kf_scratch_target* t);
// Tuned shapes remembered per (device, volume size, storage, image size) for new sessions.
void kf_tune_cache_put(const kf_session* s, int zc, int rows);
int kf_launch_intensity_projection(kf_session* s, float4* out);
int kf_rebuild_bricks(kf_session* s, cudaStream_t stream);
int kf_reset_bricks(kf_session* s);
int kf_note_integrate(kf_session* s, cudaStream_t stream);
#define KF_BRICK 8
#define KF_SUPER 64
// Brick flags.  A brick B covers the voxels [8B, 8B+8] on each axis (the taps of every
// trilinear sample whose base voxel lies in B); a super-brick S covers [64S, 64S+64].
// NEG: some value there may be negative.  Integrate only ever sets it; an exact rebuild
// (every KF_BRICK_REBUILD_EVERY integrates, and after a volume upload) clears stale bits,
// so a clear bit is a guarantee.
#define KF_BRICK_NEG 1u
#define KF_BRICK_REBUILD_EVERY 16
int kf_mc_run(kf_session* s, float iso, int method, uint32_t* n_tri);
int kf_scan_u32(const uint32_t* d_in, uint32_t* d_out, uint64_t n, uint32_t* d_total,
                cudaStream_t stream, uint32_t* d_scratch, size_t scratch_words);
size_t kf_scan_scratch_words(uint64_t n);
// Co-resident blocks of `kernel` on the session's device: min(per SM, max_per_sm) x SMs
// (with the default 2, capped at KF_MAX_TRACK_BLOCKS for the tracking kernels).
int kf_occupancy_blocks(kf_session* s, const void* kernel, int threads, size_t smem, int max_per_sm = 2);
