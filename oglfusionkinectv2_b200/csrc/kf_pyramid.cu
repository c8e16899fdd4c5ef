// kf_pyramid.cu — depth ingest, mip pyramid, vertex and normal maps.
//
// Reference: gFusion::depthToVertex (src/gFusion.cpp:496-526) with glGenerateMipmap at
// :508 and shaders/depthToVert.cs:33-72; gFusion::vertexToNormal (:528-547) with
// shaders/vertToNorm.cs:9-57.
//
// B200 layout: one kernel turns the uint16 (or float) frame into the three float depth
// levels (2x2 box means, zeros included, level 2 built from level 1 in shared memory);
// a second kernel covers the pixels of all three levels in one grid and writes vertex
// and/or normal float4 maps.  Bytes are tiny (~11 MB per frame), so both are
// latency-bound; fusing the three levels into one launch each is what matters.
#include "kf_internal.cuh"

namespace {

struct PyrArgs {
  const uint16_t* in_u16;
  const float* in_f32;
  float* depth[3];
  int W[3], H[3];
};

// One thread per level-1 pixel; a 32x8 block also produces a 16x4 level-2 tile.
// BATCH: blockIdx.z selects the session's arguments in `many`.
template <bool BATCH>
__global__ void __launch_bounds__(256) depth_mip_kernel(PyrArgs one, const PyrArgs* many,
                                                        const uint16_t* const* inputs) {
  __shared__ float s_l1[8][33];
  PyrArgs a = BATCH ? many[blockIdx.z] : one;
  if (BATCH && inputs) a.in_u16 = inputs[blockIdx.z];  // this step's frame, read in place
  const int x1 = blockIdx.x * 32 + threadIdx.x;
  const int y1 = blockIdx.y * 8 + threadIdx.y;
  float m = 0.0f;
  if (x1 < a.W[1] && y1 < a.H[1]) {
    const int W0 = a.W[0];
    const size_t i0 = (size_t)(2 * y1) * W0 + 2 * x1;
    float d00, d01, d10, d11;
    if (a.in_u16) {
      ushort2 r0 = *reinterpret_cast<const ushort2*>(a.in_u16 + i0);
      ushort2 r1 = *reinterpret_cast<const ushort2*>(a.in_u16 + i0 + W0);
      d00 = r0.x; d01 = r0.y; d10 = r1.x; d11 = r1.y;
    } else {
      float2 r0 = *reinterpret_cast<const float2*>(a.in_f32 + i0);
      float2 r1 = *reinterpret_cast<const float2*>(a.in_f32 + i0 + W0);
      d00 = r0.x; d01 = r0.y; d10 = r1.x; d11 = r1.y;
    }
    *reinterpret_cast<float2*>(a.depth[0] + i0) = make_float2(d00, d01);
    *reinterpret_cast<float2*>(a.depth[0] + i0 + W0) = make_float2(d10, d11);
    m = 0.25f * ((d00 + d01) + (d10 + d11));
    a.depth[1][(size_t)y1 * a.W[1] + x1] = m;
  }
  s_l1[threadIdx.y][threadIdx.x] = m;
  __syncthreads();
  if (threadIdx.x < 16 && threadIdx.y < 4) {
    const int x2 = blockIdx.x * 16 + threadIdx.x;
    const int y2 = blockIdx.y * 4 + threadIdx.y;
    if (x2 < a.W[2] && y2 < a.H[2]) {
      const int tx = 2 * threadIdx.x, ty = 2 * threadIdx.y;
      float v = 0.25f * ((s_l1[ty][tx] + s_l1[ty][tx + 1]) + (s_l1[ty + 1][tx] + s_l1[ty + 1][tx + 1]));
      a.depth[2][(size_t)y2 * a.W[2] + x2] = v;
    }
  }
}

struct VNArgs {
  const float* depth[3];
  float4* vertex[3];
  float4* normal[3];
  int W[3], H[3];
  int start[4];             // pixel offset of each level in the flat grid
  float ifx[3], ify[3];     // invK[0][0], invK[1][1] per level (1/fx_l, 1/fy_l)
  float mcx[3], mcy[3];     // invK[2][0], invK[2][1] per level (-cx_l/fx_l, -cy_l/fy_l)
  int mode;                 // 1 vertex, 2 normal from stored vertex, 3 both from depth
  int down_from_left;       // Q3
  // frame step: the tracking launches that follow start from zeroed barrier counters and
  // ICP sum buffers, which block 0 writes here (in place of two memset nodes)
  KfDevState* clear_state;
};

// (depth / 1000) * rotate(invK, (u, v, 1))  (depthToVert.cs:56)
__device__ __forceinline__ float3 vertex_at(const VNArgs& a, int l, int x, int y) {
  const float d = __ldg(a.depth[l] + (size_t)y * a.W[l] + x) / 1000.0f;
  return make_float3(d * ((float)x * a.ifx[l] + a.mcx[l]), d * ((float)y * a.ify[l] + a.mcy[l]), d);
}

__device__ __forceinline__ float3 neighbour(const VNArgs& a, int l, int x, int y, bool from_depth) {
  // imageLoad returns 0 outside the image; pix.x - 1 at x == 0 wraps to an invalid index
  if (x < 0 || y < 0 || x >= a.W[l] || y >= a.H[l]) return make_float3(0.f, 0.f, 0.f);
  if (from_depth) return vertex_at(a, l, x, y);
  const float4 v = a.vertex[l][(size_t)y * a.W[l] + x];
  return make_float3(v.x, v.y, v.z);
}

template <bool BATCH>
__global__ void __launch_bounds__(256) vertex_normal_kernel(VNArgs one, const VNArgs* many) {
  const VNArgs& a = BATCH ? many[blockIdx.y] : one;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (!BATCH && a.clear_state && blockIdx.x == 0) {
    KfDevState* st = a.clear_state;
    if (threadIdx.x == 0) st->barrier_count = 0u;
    if (threadIdx.x == 1) st->sdf_barrier_count = 0u;
    for (int k = threadIdx.x; k < (int)(sizeof(st->icp_acc) / sizeof(long long)); k += blockDim.x)
      (&st->icp_acc[0][0][0])[k] = 0;
  }
  if (gid >= a.start[3]) return;
  const int l = gid < a.start[1] ? 0 : (gid < a.start[2] ? 1 : 2);
  const int local = gid - a.start[l];
  const int x = local % a.W[l], y = local / a.W[l];
  const size_t i = (size_t)local;
  if (a.mode & 1) {
    const float3 v = vertex_at(a, l, x, y);
    a.vertex[l][i] = make_float4(v.x, v.y, v.z, 0.0f);
  }
  if (a.mode & 2) {
    const bool fd = (a.mode == 3);
    // vertToNorm.cs:23-26: left/right/up clamp on the high side only; "down" takes column
    // x-1 in the reference (Q3)
    const float3 lf = neighbour(a, l, x - 1, y, fd);
    const float3 rt = neighbour(a, l, min(x + 1, a.W[l] - 1), y, fd);
    const float3 up = neighbour(a, l, x, y - 1, fd);
    const float3 dn = neighbour(a, l, a.down_from_left ? x - 1 : x, min(y + 1, a.H[l] - 1), fd);
    float4 n;
    if (lf.z == 0.f || rt.z == 0.f || up.z == 0.f || dn.z == 0.f) {
      n = make_float4(2.f, 0.f, 0.f, 0.f);
    } else {
      const float3 dx = make_float3(rt.x - lf.x, rt.y - lf.y, rt.z - lf.z);
      const float3 dy = make_float3(dn.x - up.x, dn.y - up.y, dn.z - up.z);
      // normalize(cross(dyv, dxv))
      const float cx = dy.y * dx.z - dy.z * dx.y;
      const float cy = dy.z * dx.x - dy.x * dx.z;
      const float cz = dy.x * dx.y - dy.y * dx.x;
      const float inv = 1.0f / sqrtf(cx * cx + cy * cy + cz * cz);
      n = make_float4(cx * inv, cy * inv, cz * inv, 1.0f);
    }
    a.normal[l][i] = n;
  }
}

VNArgs make_vn_args(kf_session* s, int mode) {
  VNArgs a;
  int acc = 0;
  for (int l = 0; l < 3; ++l) {
    a.depth[l] = s->d_depth[l];
    a.vertex[l] = s->d_vertex[l];
    a.normal[l] = s->d_normal[l];
    a.W[l] = s->W[l];
    a.H[l] = s->H[l];
    a.start[l] = acc;
    acc += s->W[l] * s->H[l];
    // getInverseCameraMatrix(m_camPamsDepth / float(1 << l)) in float (gFusion.cpp:517)
    const float sc = (float)(1 << l);
    const float fx = s->intr.fx / sc, fy = s->intr.fy / sc;
    const float cx = s->intr.cx / sc, cy = s->intr.cy / sc;
    a.ifx[l] = 1.0f / fx;
    a.ify[l] = 1.0f / fy;
    a.mcx[l] = -cx / fx;
    a.mcy[l] = -cy / fy;
  }
  a.start[3] = acc;
  a.mode = mode;
  a.clear_state = nullptr;
  a.down_from_left = (s->cfg.quirks & KF_Q3_DOWN_FROM_LEFT) ? 1 : 0;
  return a;
}

PyrArgs make_pyr_args(kf_session* s, const uint16_t* d_u16, const float* d_f32) {
  PyrArgs a;
  a.in_u16 = d_u16;
  a.in_f32 = d_u16 ? nullptr : d_f32;
  for (int l = 0; l < 3; ++l) {
    a.depth[l] = s->d_depth[l];
    a.W[l] = s->W[l];
    a.H[l] = s->H[l];
  }
  return a;
}

// ---- depth ingest before the pyramid ----------------------------------------------------
// Kinect-v2 undistortion: the reference fuses libfreenect2's `undistorted` frame
// (src/interface.cpp:290-313, Registration::apply, libfreenect2 fork at commit 0ee1ee2f).
// Registration maps every undistorted pixel to a raw pixel through the IR camera's
// Brown-Conrady model, evaluated in float, rounds with (int)(m + 0.5f) and marks sources
// outside the image; apply() copies the raw depth through that map (0 where unmapped).
// The map is built once on the device with every operation explicitly rounded (no fused
// multiply-adds), in the expression order of libfreenect2's distort().
__global__ void __launch_bounds__(256) undistort_map_kernel(kf_ir_camera ir, int W, int H, int32_t* map) {
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * 8 + threadIdx.y;
  if (x >= W || y >= H) return;
  const float dx = __fdiv_rn(__fsub_rn((float)x, ir.cx), ir.fx);
  const float dy = __fdiv_rn(__fsub_rn((float)y, ir.cy), ir.fy);
  const float dx2 = __fmul_rn(dx, dx), dy2 = __fmul_rn(dy, dy);
  const float r2 = __fadd_rn(dx2, dy2);
  const float dxdy2 = __fmul_rn(__fmul_rn(2.0f, dx), dy);
  const float kr = __fadd_rn(1.0f, __fmul_rn(__fadd_rn(__fmul_rn(__fadd_rn(__fmul_rn(ir.k3, r2), ir.k2), r2), ir.k1), r2));
  const float mx = __fadd_rn(
      __fmul_rn(ir.fx, __fadd_rn(__fadd_rn(__fmul_rn(dx, kr), __fmul_rn(ir.p2, __fadd_rn(r2, __fmul_rn(2.0f, dx2)))),
                                 __fmul_rn(ir.p1, dxdy2))),
      ir.cx);
  const float my = __fadd_rn(
      __fmul_rn(ir.fy, __fadd_rn(__fadd_rn(__fmul_rn(dy, kr), __fmul_rn(ir.p1, __fadd_rn(r2, __fmul_rn(2.0f, dy2)))),
                                 __fmul_rn(ir.p2, dxdy2))),
      ir.cy);
  const float vx = __fadd_rn(mx, 0.5f), vy = __fadd_rn(my, 0.5f);
  // (int) truncates towards zero: the source is inside the image iff v > -1 and v < size
  int32_t idx = -1;
  if (vx > -1.0f && vx < (float)W && vy > -1.0f && vy < (float)H) idx = __float2int_rz(vy) * W + __float2int_rz(vx);
  map[(size_t)y * W + x] = idx;
}

struct PrepArgs {
  const uint16_t* in_u16;
  const float* in_f32;
  const int32_t* map;  // undistortion map, or null
  float* out;
  int W, H;
  int filter;          // filter3D.cs
};

// filter3D.cs checkPixel (:9-21): a depth is valid when 5 < d < 4000 (millimetres)
__device__ __forceinline__ float check_pixel(float v) { return (v > 5.0f && v < 4000.0f) ? v : 0.0f; }

__device__ __forceinline__ float prep_raw(const PrepArgs& a, int x, int y) {
  if (x < 0 || y < 0 || x >= a.W || y >= a.H) return 0.0f;
  int i = y * a.W + x;
  if (a.map) {
    i = __ldg(a.map + i);
    if (i < 0) return 0.0f;
  }
  return a.in_u16 ? (float)__ldg(a.in_u16 + i) : __ldg(a.in_f32 + i);
}

// One 32x8 tile per block with a one-pixel halo in shared memory (each halo value is an
// undistortion gather).  filter3D.cs:23-86: an interior pixel (1 < x < W-1, 1 < y < H-1)
// keeps its depth when more than 6 of its 3x3 neighbourhood are valid and it is within
// 5 mm of their mean, else 0; the neighbourhood is summed column by column, as the
// shader's loops do.  The shader never writes border pixels; they are 0 here.
__global__ void __launch_bounds__(256) depth_prepare_kernel(PrepArgs a) {
  __shared__ float s_t[10][35];
  const int tid = threadIdx.y * 32 + threadIdx.x;
  const int x0 = blockIdx.x * 32 - 1, y0 = blockIdx.y * 8 - 1;
  for (int k = tid; k < 10 * 34; k += 256) {
    const int ty = k / 34, tx = k - ty * 34;
    const float v = prep_raw(a, x0 + tx, y0 + ty);
    s_t[ty][tx] = a.filter ? check_pixel(v) : v;
  }
  __syncthreads();
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * 8 + threadIdx.y;
  if (x >= a.W || y >= a.H) return;
  float o = s_t[threadIdx.y + 1][threadIdx.x + 1];
  if (a.filter) {
    float r = 0.0f;
    if (x > 1 && x < a.W - 1 && y > 1 && y < a.H - 1) {
      float valid = 9.0f, sum = 0.0f;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const float t = s_t[threadIdx.y + j][threadIdx.x + i];
          if (t == 0.0f) valid = __fsub_rn(valid, 1.0f);
          else sum = __fadd_rn(sum, t);
        }
      const float mean = valid > 6.0f ? __fdiv_rn(sum, valid) : 0.0f;
      if (mean > 0.0f && fabsf(__fsub_rn(o, mean)) < 5.0f) r = o;
    }
    o = r;
  }
  a.out[(size_t)y * a.W + x] = o;
}

}  // namespace

int kf_launch_undistort_map(kf_session* s, const kf_ir_camera& ir) {
  dim3 block(32, 8);
  dim3 grid((s->W[0] + 31) / 32, (s->H[0] + 7) / 8);
  undistort_map_kernel<<<grid, block, 0, s->stream>>>(ir, s->W[0], s->H[0], s->d_undistort_map);
  KF_CUDA_TRY(s, cudaGetLastError());
  kf_note_launch(s);
  return KF_OK;
}

// The pyramid of one frame, through the session's ingest stages when they are on.
int kf_launch_depth_ingest(kf_session* s, const uint16_t* d_u16, const float* d_f32) {
  if (!s->undistort && !s->depth_filter) return kf_launch_pyramid(s, d_u16, d_f32);
  PrepArgs a;
  a.in_u16 = d_u16;
  a.in_f32 = d_u16 ? nullptr : d_f32;
  a.map = s->undistort ? s->d_undistort_map : nullptr;
  a.out = s->d_depth_prep;
  a.W = s->W[0];
  a.H = s->H[0];
  a.filter = s->depth_filter;
  dim3 block(32, 8);
  dim3 grid((a.W + 31) / 32, (a.H + 7) / 8);
  depth_prepare_kernel<<<grid, block, 0, s->stream>>>(a);
  KF_CUDA_TRY(s, cudaGetLastError());
  kf_note_launch(s);
  return kf_launch_pyramid(s, nullptr, s->d_depth_prep);
}

int kf_launch_pyramid(kf_session* s, const uint16_t* d_u16, const float* d_f32) {
  const PyrArgs a = make_pyr_args(s, d_u16, d_f32);
  dim3 block(32, 8);
  dim3 grid((s->W[1] + 31) / 32, (s->H[1] + 7) / 8);
  depth_mip_kernel<false><<<grid, block, 0, s->stream>>>(a, nullptr, nullptr);
  kf_note_launch(s);
  KF_CUDA_TRY(s, cudaGetLastError());
  return KF_OK;
}

static int launch_vn(kf_session* s, int mode, bool clear = false) {
  VNArgs a = make_vn_args(s, mode);
  if (clear) a.clear_state = s->d_state;
  const int threads = 256;
  const int blocks = (a.start[3] + threads - 1) / threads;
  vertex_normal_kernel<false><<<blocks, threads, 0, s->stream>>>(a, nullptr);
  kf_note_launch(s);
  KF_CUDA_TRY(s, cudaGetLastError());
  return KF_OK;
}

int kf_launch_vertex(kf_session* s) { return launch_vn(s, 1); }
int kf_launch_normal(kf_session* s) { return launch_vn(s, 2); }
int kf_launch_vertex_normal(kf_session* s, bool clear_tracking_words) { return launch_vn(s, 3, clear_tracking_words); }

// ---- batched: every member's uint16 upload buffer -> its pyramid, one launch per kernel ----
int kf_batch_prepare_pyramid(kf_batch* b) {
  const int n = (int)b->members.size();
  PyrArgs* hp = nullptr;
  VNArgs* hv = nullptr;
  b->pyr_args = kf_batch_table(b, sizeof(PyrArgs) * n, reinterpret_cast<void**>(&hp));
  b->vn_args = kf_batch_table(b, sizeof(VNArgs) * n, reinterpret_cast<void**>(&hv));
  if (!b->pyr_args || !b->vn_args) return KF_ERR_CAPACITY;
  for (int e = 0; e < n; ++e) {
    kf_session* s = b->members[e];
    hp[e] = make_pyr_args(s, s->d_depth_u16, nullptr);
    hv[e] = make_vn_args(s, 3);
  }
  b->vn_pixels = hv[0].start[3];
  b->W1 = b->members[0]->W[1];
  b->H1 = b->members[0]->H[1];
  return KF_OK;
}

int kf_batch_launch_pyramid(kf_batch* b, int n, const uint16_t* const* d_inputs) {
  dim3 block(32, 8);
  dim3 grid((b->W1 + 31) / 32, (b->H1 + 7) / 8, n);
  depth_mip_kernel<true><<<grid, block, 0, b->stream>>>(PyrArgs{}, static_cast<const PyrArgs*>(b->pyr_args), d_inputs);
  KF_CUDA_TRY(b, cudaGetLastError());
  dim3 g2((b->vn_pixels + 255) / 256, n);
  vertex_normal_kernel<true><<<g2, 256, 0, b->stream>>>(VNArgs{}, static_cast<const VNArgs*>(b->vn_args));
  KF_CUDA_TRY(b, cudaGetLastError());
  b->launches += 2;
  return KF_OK;
}
