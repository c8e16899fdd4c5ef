// kf_icp.cu — projective point-to-plane ICP: track + reduce + solve, all on the device.
//
// Reference: gFusion::Track (src/gFusion.cpp:648-740), gFusion::track (:742-777) with
// shaders/track.cs:47-163, gFusion::reduce (:779-809) with shaders/reduce.cs:27-126,
// getReduction (:1127-1168) and makeJTJ (include/gFusion.h:472-487).
//
// B200 design: ONE cooperative (co-resident) launch runs every pyramid level and every
// Gauss-Newton iteration of a frame.  Per iteration each block associates its pixels
// (same-pixel projective association at level-0 resolution), accumulates the 27 sums of
// reduce.cs, and writes one partial row; the last block to arrive reduces the rows in a
// fixed order in FP64, solves the 6x6 system by FP64 Cholesky, composes the pose in FP64
// and releases the others.  No host round trip per iteration (the reference maps the
// SSBO back every iteration, :1131-1134), no launch per iteration, deterministic sums.
//
// J^T J contraction: KF_JTJ_FP32 uses FMAs; KF_JTJ_SPLIT_BF16 stages each warp's 32
// feature rows f = [J0..J5, e, 0] as bf16 hi + lo pairs and issues
// mma.sync.m16n8k16 (A = [hi; lo]^T rows, B = hi then lo) so that the FP32 accumulator
// holds sum (hi+lo)(hi+lo)^T: every bf16 x bf16 product is exact in FP32, the only
// rounding is the 2^-16 split of each feature and the FP32 accumulation.
#include "kf_internal.cuh"

namespace {

struct IcpArgs {
  const float4* vertex[3];
  const float4* normal[3];
  int32_t* status[3];
  const float4* ref_vertex;
  const float4* ref_normal;
  int W[3], H[3];
  int W0, H0;
  double fx, fy, cx, cy;  // level-0 intrinsics for view = K * inverse(pose) (:747)
  float dist_thresh, normal_thresh;
  int iters[3];
  int q1;                 // reduce only rows y % 8 == 7 (Q1)
  int same_pixel;         // Q4
  int frame_policy;
  int integrate_every;
  float* partials;        // [gridDim.x][32]
  KfDevState* st;
};

// ---- track.cs:53-133 for one pixel ------------------------------------------------------
__device__ __forceinline__ int track_pixel(const IcpArgs& a, int l, int x, int y,
                                           const float* T, const float* V, float* f) {
  const size_t i = (size_t)y * a.W[l] + x;
  const float4 n = __ldg(&a.normal[l][i]);
  if (n.x == 2.0f) return -1;
  const float4 v = __ldg(&a.vertex[l][i]);
  // z == 0 with a valid normal projects (0,0,0) -> 0/0 in track.cs:72 (undefined in
  // GLSL); treated as "outside the image"
  if (v.z == 0.0f) return -2;
  // projectedVertex = Ttrack * vec4(v, 1)
  const float pvx = fmaf(T[0], v.x, fmaf(T[4], v.y, fmaf(T[8], v.z, T[12])));
  const float pvy = fmaf(T[1], v.x, fmaf(T[5], v.y, fmaf(T[9], v.z, T[13])));
  const float pvz = fmaf(T[2], v.x, fmaf(T[6], v.y, fmaf(T[10], v.z, T[14])));
  // projectedPos = view * projectedVertex
  const float ppx = fmaf(V[0], pvx, fmaf(V[4], pvy, fmaf(V[8], pvz, V[12])));
  const float ppy = fmaf(V[1], pvx, fmaf(V[5], pvy, fmaf(V[9], pvz, V[13])));
  const float ppz = fmaf(V[2], pvx, fmaf(V[6], pvy, fmaf(V[10], pvz, V[14])));
  const float px = ppx / ppz + 0.5f, py = ppy / ppz + 0.5f;
  if (!(px >= 0.0f) || px > (float)(a.W0 - 1) || !(py >= 0.0f) || py > (float)(a.H0 - 1))
    return -2;
  const size_t ri = (size_t)(int)py * a.W0 + (int)px;
  const float4 rn = __ldg(&a.ref_normal[ri]);
  if (rn.x == -2.0f) return -3;
  const float4 rv = __ldg(&a.ref_vertex[ri]);
  const float dx = rv.x - pvx, dy = rv.y - pvy, dz = rv.z - pvz;
  // projectedNormal = rotate(Ttrack, normal)
  const float pnx = T[0] * n.x + T[4] * n.y + T[8] * n.z;
  const float pny = T[1] * n.x + T[5] * n.y + T[9] * n.z;
  const float pnz = T[2] * n.x + T[6] * n.y + T[10] * n.z;
  if (sqrtf(dx * dx + dy * dy + dz * dz) > a.dist_thresh) return -4;
  if (pnx * rn.x + pny * rn.y + pnz * rn.z < a.normal_thresh) return -5;
  f[0] = rn.x;
  f[1] = rn.y;
  f[2] = rn.z;
  f[3] = pvy * rn.z - pvz * rn.y;  // cross(projectedVertex, referenceNormal)
  f[4] = pvz * rn.x - pvx * rn.z;
  f[5] = pvx * rn.y - pvy * rn.x;
  f[6] = rn.x * dx + rn.y * dy + rn.z * dz;  // dot(referenceNormal, diff)
  return 1;
}

__device__ __forceinline__ void mma_bf16_16816(float* c, uint32_t a0, uint32_t a1, uint32_t a2,
                                               uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Pose (FP64, shared) -> FP32 Ttrack and view = K * inverse(Pv) in shared memory; Pv is
// the current estimate (Q4, gFusion.cpp:747) or the raycast pose.
__device__ __forceinline__ void make_float_mats(const IcpArgs& a, const double* P, const double* Pv,
                                                float* T, float* V) {
  double inv[16], K[16], view[16];
  kf_rigid_inverse(a.same_pixel ? P : Pv, inv);
  for (int i = 0; i < 16; ++i) K[i] = 0;
  K[0] = a.fx; K[8] = a.cx; K[5] = a.fy; K[9] = a.cy; K[10] = 1; K[15] = 1;
  kf_mat4_mul(K, inv, view);
  for (int i = 0; i < 16; ++i) {
    T[i] = (float)P[i];
    V[i] = (float)view[i];
  }
}

constexpr int kWarps = KF_TRACK_THREADS / 32;

template <int JTJ>
__global__ void __launch_bounds__(KF_TRACK_THREADS) icp_kernel(IcpArgs a) {
  __shared__ double s_pose[16];
  __shared__ double s_old[16];
  __shared__ double s_ray[16];
  __shared__ float s_T[16], s_V[16];
  __shared__ float s_warp[kWarps][64];
  __shared__ double s_red[kWarps][32];
  __shared__ double s_sums[32];
  __shared__ unsigned s_gen;
  __shared__ int s_last, s_flag, s_conv;
  __shared__ __align__(16) __nv_bfloat16 s_hi[JTJ ? kWarps : 1][8][40];
  __shared__ __align__(16) __nv_bfloat16 s_lo[JTJ ? kWarps : 1][8][40];

  KfDevState* st = a.st;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned nb = gridDim.x;

  if (tid < 16) {
    s_pose[tid] = st->pose[tid];
    s_old[tid] = s_pose[tid];
    s_ray[tid] = st->raycast_pose[tid];
  }
  __syncthreads();
  if (tid == 0) make_float_mats(a, s_pose, s_ray, s_T, s_V);
  __syncthreads();

  bool ok = true;
  int iters_run = 0;
  for (int level = 2; level >= 0 && ok; --level) {
    const int Wl = a.W[level], Hl = a.H[level];
    const int P = Wl * Hl;
    for (int it = 0; it < a.iters[level]; ++it) {
      float T[16], V[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) { T[k] = s_T[k]; V[k] = s_V[k]; }

      // ---------------- track + accumulate ----------------
      float acc[JTJ ? 4 : 28];
#pragma unroll
      for (int k = 0; k < (JTJ ? 4 : 28); ++k) acc[k] = 0.0f;
      const int stride = nb * KF_TRACK_THREADS;
      for (int base = (blockIdx.x * kWarps + warp) * 32; base < P; base += stride) {
        const int i = base + lane;
        float f[7] = {0, 0, 0, 0, 0, 0, 0};
        int status = 0;
        if (i < P) {
          const int y = i / Wl, x = i - y * Wl;
          status = track_pixel(a, level, x, y, T, V, f);
          a.status[level][i] = status;
          if (a.q1 && (y & 7) != 7) status = 0;  // only work group 7 reaches the solver
        }
        const bool use = status == 1;
        if constexpr (JTJ == 0) {
          if (use) {
            const float e = f[6];
            acc[0] += e * e;
#pragma unroll
            for (int k = 0; k < 6; ++k) acc[1 + k] += e * f[k];
            int q = 7;
#pragma unroll
            for (int r = 0; r < 6; ++r)
#pragma unroll
              for (int c = r; c < 6; ++c) acc[q++] += f[r] * f[c];
          }
        } else {
          // stage f = [J0..J5, e, 0] as hi/lo bf16, feature-major per warp
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const float v = (use && k < 7) ? f[k] : 0.0f;
            const __nv_bfloat16 hi = __float2bfloat16_rn(v);
            const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
            s_hi[warp][k][lane] = hi;
            s_lo[warp][k][lane] = lo;
          }
          __syncwarp();
          const int g = lane >> 2, t = lane & 3;
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int c0 = 16 * h + 2 * t;
            const uint32_t a0 = *reinterpret_cast<const uint32_t*>(&s_hi[warp][g][c0]);
            const uint32_t a1 = *reinterpret_cast<const uint32_t*>(&s_lo[warp][g][c0]);
            const uint32_t a2 = *reinterpret_cast<const uint32_t*>(&s_hi[warp][g][c0 + 8]);
            const uint32_t a3 = *reinterpret_cast<const uint32_t*>(&s_lo[warp][g][c0 + 8]);
            mma_bf16_16816(acc, a0, a1, a2, a3, a0, a2);  // x B = hi
            mma_bf16_16816(acc, a0, a1, a2, a3, a1, a3);  // x B = lo
          }
          __syncwarp();
        }
      }

      // ---------------- block partial ----------------
      if constexpr (JTJ == 0) {
#pragma unroll
        for (int k = 0; k < 28; ++k) {
          float v = acc[k];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (lane == 0) s_warp[warp][k] = v;
        }
        __syncthreads();
        if (tid < 28) {
          float v = 0.0f;
#pragma unroll
          for (int w = 0; w < kWarps; ++w) v += s_warp[w][tid];
          a.partials[(size_t)blockIdx.x * 32 + tid] = v;
        }
      } else {
        // lane (g, t) holds M[g][2t], M[g][2t+1] as rows g (hi) + g+8 (lo) of the mma
        const int g = lane >> 2, t = lane & 3;
        s_warp[warp][g * 8 + 2 * t] = acc[0] + acc[2];
        s_warp[warp][g * 8 + 2 * t + 1] = acc[1] + acc[3];
        __syncthreads();
        if (tid < 28) {
          int r, c;
          if (tid == 0) { r = 6; c = 6; }
          else if (tid < 7) { r = tid - 1; c = 6; }
          else {
            int q = tid - 7;
            r = 0;
            while (q >= 6 - r) { q -= 6 - r; ++r; }
            c = r + q;
          }
          float v = 0.0f;
#pragma unroll
          for (int w = 0; w < kWarps; ++w) v += s_warp[w][r * 8 + c];
          a.partials[(size_t)blockIdx.x * 32 + tid] = v;
        }
      }

      // ---------------- hand-over: last block reduces + solves ----------------
      if (kf_grid_arrive(st, nb, &s_gen, &s_last)) {
        {
          const int k = tid & 31, r = tid >> 5;
          double v = 0.0;
          if (k < 28)
            for (unsigned b = r; b < nb; b += kWarps) v += (double)__ldcg(&a.partials[(size_t)b * 32 + k]);
          s_red[r][k] = v;
        }
        __syncthreads();
        if (tid < 32) {
          double v = 0.0;
#pragma unroll
          for (int r = 0; r < kWarps; ++r) v += s_red[r][tid];
          s_sums[tid] = v;
        }
        __syncthreads();
        if (tid == 0) {
          // reduce.cs counts every pixel of the (group-7) rows in sums[28]
          const double count = a.q1 ? (double)Wl * (double)(Hl / 8) : (double)P;
          s_sums[28] = count;
          s_sums[29] = s_sums[30] = s_sums[31] = 0.0;
          double b[6], C[36], x[6];
          for (int k = 0; k < 6; ++k) b[k] = s_sums[1 + k];
          kf_make_jtj(&s_sums[7], C);
          const double ae = sqrt(s_sums[0] / count);  // getReduction :1167
          kf_cholesky6(C, b, x);
          // delta = eulerAngleXYZ(x3, x4, x5), delta[3].xyz = x0..2; pose = delta * pose
          double R[9], D[16], Pn[16];
          kf_euler_xyz(x[3], x[4], x[5], R);
          for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) D[c * 4 + r] = R[c * 3 + r];
          D[3] = D[7] = D[11] = 0;
          D[12] = x[0]; D[13] = x[1]; D[14] = x[2]; D[15] = 1;
          kf_mat4_mul(D, s_pose, Pn);
          for (int k = 0; k < 16; ++k) st->iter_pose[k] = Pn[k];
          const double nrm = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + x[3] * x[3] +
                                  x[4] * x[4] + x[5] * x[5]);
          st->iter_conv = (nrm < 1e-5 && nrm != 0.0) ? 1 : 0;
          st->ae = ae;
          for (int k = 0; k < 32; ++k) st->sums[k] = s_sums[k];
        }
        kf_grid_release(st);
      } else {
        ok = kf_grid_wait(st, &s_gen, &s_flag);
      }
      if (!ok) break;
      if (tid < 16) s_pose[tid] = __ldcg(&st->iter_pose[tid]);
      if (tid == 16) s_conv = __ldcg(&st->iter_conv);
      __syncthreads();
      if (tid == 0) make_float_mats(a, s_pose, s_ray, s_T, s_V);
      __syncthreads();
      ++iters_run;
      if (s_conv) break;  // result.norm() < 1e-5 && != 0 leaves this level (:707-708)
    }
  }

  // ---------------- Track() tail (:715-723) + frame policy, block 0 only -----------------
  if (blockIdx.x != 0 || tid != 0 || !ok) return;
  const double ae = iters_run ? __ldcg(&st->ae) : 0.0;
  int tracked;
  if (ae > 0.5 || ae == 0.0) {
    tracked = 0;
    for (int k = 0; k < 16; ++k) st->pose[k] = s_old[k];
  } else {
    tracked = 1;
    for (int k = 0; k < 16; ++k) st->pose[k] = s_pose[k];
    // updatePoseFinder (gFusion.cpp:1570-1594): add when 0.2 m from every library pose
    bool add = true;
    for (int e = 0; e < st->lib_size; ++e) {
      const double dx = st->lib_pose[e][12] - s_pose[12], dy = st->lib_pose[e][13] - s_pose[13],
                   dz = st->lib_pose[e][14] - s_pose[14];
      if (sqrt(dx * dx + dy * dy + dz * dz) < 0.2) { add = false; break; }
    }
    if (add && st->lib_size < KF_MAX_LIBRARY) {
      for (int k = 0; k < 16; ++k) st->lib_pose[st->lib_size][k] = s_pose[k];
      st->lib_size += 1;
    }
  }
  for (int k = 0; k < 16; ++k) st->old_pose[k] = s_old[k];
  st->tracked = tracked;
  st->iterations_run = iters_run;
  if (a.frame_policy) {
    // kinect.cpp:677-689: integrate when tracked (every integrate_every frames) or inside
    // the reset window; recoverPose when not tracked
    const int every = a.integrate_every > 0 ? a.integrate_every : 1;
    const int integ = (tracked && (st->counter % every) == 0) || st->reset_window;
    st->do_integrate = integ;
    if (integ && st->counter > 2) st->reset_window = 0;
    st->need_recover = !tracked;
    st->counter += 1;
  }
}

}  // namespace

int kf_launch_icp(kf_session* s, int frame_policy) {
  IcpArgs a;
  for (int l = 0; l < 3; ++l) {
    a.vertex[l] = s->d_vertex[l];
    a.normal[l] = s->d_normal[l];
    a.status[l] = s->d_status[l];
    a.W[l] = s->W[l];
    a.H[l] = s->H[l];
    a.iters[l] = s->cfg.iterations[l];
  }
  a.ref_vertex = s->d_ref_vertex;
  a.ref_normal = s->d_ref_normal;
  a.W0 = s->W[0];
  a.H0 = s->H[0];
  // getCameraMatrix(m_camPamsDepth) holds float intrinsics (gFusion.h:459-470)
  a.fx = s->intr.fx; a.fy = s->intr.fy; a.cx = s->intr.cx; a.cy = s->intr.cy;
  a.dist_thresh = s->cfg.dist_threshold;
  a.normal_thresh = s->cfg.normal_threshold;
  a.q1 = (s->cfg.quirks & KF_Q1_LAST_GROUP_ONLY) ? 1 : 0;
  a.same_pixel = (s->cfg.quirks & KF_Q4_SAME_PIXEL) ? 1 : 0;
  a.frame_policy = frame_policy;
  a.integrate_every = s->cfg.integrate_every;
  a.partials = s->d_partials;
  a.st = s->d_state;

  const void* fn = (s->cfg.jtj == KF_JTJ_SPLIT_BF16) ? (const void*)icp_kernel<1> : (const void*)icp_kernel<0>;
  int blocks = kf_occupancy_blocks(s, fn, KF_TRACK_THREADS, 0);
  if (blocks <= 0) return KF_ERR_CUDA;
  // barrier words start at zero for every launch
  KF_CUDA_TRY(s, cudaMemsetAsync(&s->d_state->barrier_count, 0, 2 * sizeof(unsigned), s->stream));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(KF_TRACK_THREADS);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (s->cfg.jtj == KF_JTJ_SPLIT_BF16)
    KF_CUDA_TRY(s, cudaLaunchKernelEx(&cfg, icp_kernel<1>, a));
  else
    KF_CUDA_TRY(s, cudaLaunchKernelEx(&cfg, icp_kernel<0>, a));
  kf_note_launch(s);
  return KF_OK;
}
