// kf_icp.cu — projective point-to-plane ICP: track + reduce + solve, all on the device.
//
// Reference: gFusion::Track (src/gFusion.cpp:648-740), gFusion::track (:742-777) with
// shaders/track.cs:47-163, gFusion::reduce (:779-809) with shaders/reduce.cs:27-126,
// getReduction (:1127-1168) and makeJTJ (include/gFusion.h:472-487).
//
// B200 design: ONE cooperative (co-resident) launch runs every pyramid level and every
// Gauss-Newton iteration of a frame.  Per iteration each block associates its pixels
// (same-pixel projective association at level-0 resolution) and adds the 27 sums of
// reduce.cs, plus the valid count and the sum of the points, to the session's rows as
// fixed-point integers (value * 2^32, 64-bit atomics: exact, so the total does not depend
// on the order or on how the pixels were split among blocks); after a grid barrier every
// block reads the rows, solves the 6x6 system in FP64 and composes the pose in FP64.  No
// host round trip per iteration (the reference maps the SSBO back every iteration,
// :1131-1134), no launch per iteration, deterministic sums.  A batched launch gives each
// session its own group of blocks, rows and barrier.

// Conditioning: J = [n, p x n] with world p couples rotation and translation strongly
// (lever arms of metres), so FP32 partial sums lose the small eigen-directions of J^T J.
// The sums are therefore accumulated with the lever arm taken about a centre c (the
// previous iteration's centroid of the valid points): J' = [n, (p - c) x n].  That is an
// exact change of variables: J = M J' with M = [[I, 0], [[c]x, I]], so the world system
// is C = M C' M^T, b = M b', and its solution is t = t' - w x c for the same w.  The
// reported reduction row is the world form, as the reference's.
//
// J^T J contraction: KF_JTJ_FP32 uses FMAs (per-thread FP32 sums, converted per block).
// KF_JTJ_SPLIT_BF16 splits each feature of f = [J'0..J'5, e, 1] into three bf16 terms
// (hi + mid + lo, 24 significant bits), stages them feature-major per warp, and issues four
// mma.sync.m16n8k16 per 16 pixels ([hi; mid] x hi, x mid, x lo, and [lo; q] x hi, q = the
// point's hi and mid terms) with FP32 accumulation: every bf16 x bf16 product is exact in
// FP32 and only the lo*mid and lo*lo terms (~2^-24) are left out.  The constant feature 1
// makes the valid count and the point sums (for the next centre) columns of the same
// products.  Each warp converts its 32-pixel chunk's sums to fixed point, so a chunk
// contributes the same bits whichever block, grid or batch processes it.
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
  KfDevState* st;
};

// A batched launch: the blocks of entry e (one session each) are those whose map word
// names e; every entry runs its own levels, iterations and grid barrier.
struct IcpBatch {
  const IcpArgs* args;        // per entry
  const uint32_t* block_map;  // per block: entry << 24 | blocks of the entry << 12 | index
};

// Fixed-point scale of the reduction sums: |sum| < 2^31 for every row entry (the points
// are within the distance threshold of the raycast surface, inside the volume).
constexpr float kFix = 4294967296.0f;       // 2^32
constexpr double kInvFix = 1.0 / 4294967296.0;

// ---- track.cs:53-133 for one pixel, in two phases -----------------------------------------
// The caller projects its pixels first, then issues every reference gather (normal and
// vertex together, for all of its pixels) and only then finishes them: the gathers are the
// latency of this kernel, and none of them waits for another.
// n, v: the pixel's normal and vertex.  Returns the status for a pixel that stops here, or
// 0 with the transformed vertex pv and the reference index *ri.
__device__ __forceinline__ int track_project(const IcpArgs& a, const float4 n, const float4 v, const float* T,
                                             const float* V, float* pv, int* ri) {
  if (n.x == 2.0f) return -1;
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
  *ri = (int)py * a.W0 + (int)px;
  pv[0] = pvx;
  pv[1] = pvy;
  pv[2] = pvz;
  return 0;
}

// The rest of track.cs for a pixel that track_project passed, with its reference normal rn
// and vertex rv.
__device__ __forceinline__ int track_finish(const IcpArgs& a, const float4 n, const float* pv, const float4 rn,
                                            const float4 rv, const float* T, const float* c, float* f, float* pw) {
  if (rn.x == -2.0f) return -3;
  const float pvx = pv[0], pvy = pv[1], pvz = pv[2];
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
  // cross(projectedVertex - c, referenceNormal): the reference's p x n about centre c
  const float qx = pvx - c[0], qy = pvy - c[1], qz = pvz - c[2];
  f[3] = qy * rn.z - qz * rn.y;
  f[4] = qz * rn.x - qx * rn.z;
  f[5] = qx * rn.y - qy * rn.x;
  f[6] = rn.x * dx + rn.y * dy + rn.z * dz;  // dot(referenceNormal, diff)
  pw[0] = pvx;
  pw[1] = pvy;
  pw[2] = pvz;
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

template <int JTJ, bool BATCH>
__global__ void __launch_bounds__(KF_TRACK_THREADS, 2) icp_kernel(IcpArgs a_one, IcpBatch batch) {
  __shared__ IcpArgs s_args;
  __shared__ double s_pose[16];
  __shared__ double s_old[16];
  __shared__ double s_ray[16];
  __shared__ double s_cd[3];
  __shared__ float s_T[16], s_V[16], s_c[3];
  __shared__ float s_warp[JTJ ? 1 : kWarps][28];
  __shared__ float s_pw[JTJ ? 1 : kWarps][4];
  __shared__ long long s_fix[JTJ ? kWarps : 1][72];
  __shared__ double s_sums[32];
  __shared__ double s_csums[29], s_ccenter[3];  // last centred row (for the tail)
  __shared__ double s_nvalid;                           // its valid-pixel count
  __shared__ double s_gx[8 + 228];                      // the step (+ rank guard's scratch)
  __shared__ int s_fast;                                // the rank check's verdict
  __shared__ int s_flag, s_conv;
  __shared__ __align__(16) __nv_bfloat16 s_hi[JTJ ? kWarps : 1][8][40];
  __shared__ __align__(16) __nv_bfloat16 s_mid[JTJ ? kWarps : 1][8][40];
  __shared__ __align__(16) __nv_bfloat16 s_lo[JTJ ? kWarps : 1][8][40];
  __shared__ __align__(16) __nv_bfloat16 s_q[JTJ ? kWarps : 1][8][40];

  unsigned local, nb;  // this block's index among its entry's blocks, and their number
  if constexpr (BATCH) {
    const uint32_t m = batch.block_map[blockIdx.x];
    local = m & 0xfffu;
    nb = (m >> 12) & 0xfffu;
    const int* src = reinterpret_cast<const int*>(batch.args + (m >> 24));
    for (int k = threadIdx.x; k < (int)(sizeof(IcpArgs) / 4); k += blockDim.x)
      reinterpret_cast<int*>(&s_args)[k] = __ldg(src + k);
    __syncthreads();
  } else {
    local = blockIdx.x;
    nb = gridDim.x;
  }
  const IcpArgs& a = BATCH ? s_args : a_one;

  KfDevState* st = a.st;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  if (tid < 16) {
    s_pose[tid] = st->pose[tid];
    s_old[tid] = s_pose[tid];
    s_ray[tid] = st->raycast_pose[tid];
  }
  __syncthreads();
  if (tid == 0) {
    make_float_mats(a, s_pose, s_ray, s_T, s_V);
    // first centre: last frame's centroid, carried in the camera frame
    const double* cc = st->icp_center_cam;
    for (int r = 0; r < 3; ++r) {
      s_cd[r] = s_pose[r] * cc[0] + s_pose[4 + r] * cc[1] + s_pose[8 + r] * cc[2] + s_pose[12 + r];
      s_c[r] = (float)s_cd[r];
    }
  }
  __syncthreads();

  bool ok = true;
  int iters_run = 0;
  unsigned gi = 0;  // iterations of this launch so far: grid barrier target and sum buffer
  // the first step's vertices and normals of the next iteration, loaded while the current
  // iteration's system is solved (valid when pre_level is the level that runs)
  const float4 none = make_float4(2.0f, 0.f, 0.f, 0.f), zero = make_float4(0.f, 0.f, 0.f, 0.f);
  float4 pn0 = none, pv0 = zero, pn1 = none, pv1 = zero;
  int pre_level = -1;
  for (int level = 2; level >= 0 && ok; --level) {
    const int Wl = a.W[level], Hl = a.H[level];
    const int P = Wl * Hl;
    for (int it = 0; it < a.iters[level]; ++it) {
      // Ttrack and view stay in shared memory (broadcast reads), which leaves the registers
      // for two pixels in flight per thread
      float c[3];
      c[0] = s_c[0]; c[1] = s_c[1]; c[2] = s_c[2];

      // ---------------- track + accumulate ----------------
      long long* accbuf = &a.st->icp_acc[gi % 3u][0][0];
      float acc[JTJ ? 1 : 28];
#pragma unroll
      for (int k = 0; k < (JTJ ? 1 : 28); ++k) acc[k] = 0.0f;
      float pacc[4] = {0.f, 0.f, 0.f, 0.f};  // FP32 path: valid count, sum of world points
      // split-BF16 path: fixed-point sums of M[g][2t], M[g][2t+1] and of q_g (lane g, t)
      long long fx0 = 0, fx1 = 0, fxq = 0;

      // one pixel's row into this thread's sums (FP32) or its 32-pixel chunk (split-BF16)
      auto accumulate = [&](bool use, const float* f, const float* pw) {
        if constexpr (JTJ == 0) {
          if (use) {
            pacc[0] += 1.0f;
            pacc[1] += pw[0];
            pacc[2] += pw[1];
            pacc[3] += pw[2];
            const float e = f[6];
            acc[0] += e * e;
#pragma unroll
            for (int k = 0; k < 6; ++k) acc[1 + k] += e * f[k];
            int q = 7;
#pragma unroll
            for (int r = 0; r < 6; ++r)
#pragma unroll
              for (int cc = r; cc < 6; ++cc) acc[q++] += f[r] * f[cc];
          }
        } else {
          // stage f = [J'0..J'5, e, 1] as hi + mid + lo bf16 and q = [hi(p), mid(p), 0, 0]
          // feature-major per warp (zero for pixels that are not used)
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const float v = use ? (k < 7 ? f[k] : 1.0f) : 0.0f;
            const __nv_bfloat16 hi = __float2bfloat16_rn(v);
            const float r1 = v - __bfloat162float(hi);
            const __nv_bfloat16 mid = __float2bfloat16_rn(r1);
            const __nv_bfloat16 lo = __float2bfloat16_rn(r1 - __bfloat162float(mid));
            s_hi[warp][k][lane] = hi;
            s_mid[warp][k][lane] = mid;
            s_lo[warp][k][lane] = lo;
          }
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const float p = use ? pw[k] : 0.0f;
            const __nv_bfloat16 hi = __float2bfloat16_rn(p);
            s_q[warp][k][lane] = hi;
            s_q[warp][3 + k][lane] = __float2bfloat16_rn(p - __bfloat162float(hi));
          }
          s_q[warp][6][lane] = __float2bfloat16_rn(0.0f);
          s_q[warp][7][lane] = __float2bfloat16_rn(0.0f);
          __syncwarp();
          const int g = lane >> 2, t = lane & 3;
          float cA[4] = {0.f, 0.f, 0.f, 0.f}, cB[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int c0 = 16 * h + 2 * t;
            const uint32_t h0 = *reinterpret_cast<const uint32_t*>(&s_hi[warp][g][c0]);
            const uint32_t h1 = *reinterpret_cast<const uint32_t*>(&s_hi[warp][g][c0 + 8]);
            const uint32_t m0 = *reinterpret_cast<const uint32_t*>(&s_mid[warp][g][c0]);
            const uint32_t m1 = *reinterpret_cast<const uint32_t*>(&s_mid[warp][g][c0 + 8]);
            const uint32_t l0 = *reinterpret_cast<const uint32_t*>(&s_lo[warp][g][c0]);
            const uint32_t l1 = *reinterpret_cast<const uint32_t*>(&s_lo[warp][g][c0 + 8]);
            const uint32_t q0 = *reinterpret_cast<const uint32_t*>(&s_q[warp][g][c0]);
            const uint32_t q1 = *reinterpret_cast<const uint32_t*>(&s_q[warp][g][c0 + 8]);
            // A = [hi; mid] (rows g, g+8); B columns = features of 16 pixels
            mma_bf16_16816(cA, h0, m0, h1, m1, h0, h1);  // x hi
            mma_bf16_16816(cA, h0, m0, h1, m1, m0, m1);  // x mid
            mma_bf16_16816(cA, h0, m0, h1, m1, l0, l1);  // x lo
            mma_bf16_16816(cB, l0, q0, l1, q1, h0, h1);  // [lo; q] x hi
          }
          __syncwarp();
          // this 32-pixel chunk's sums, fixed-point: the same chunk gives the same bits
          // whichever block or launch processes it
          fx0 += __float2ll_rn((cA[0] + cA[2] + cB[0]) * kFix);
          fx1 += __float2ll_rn((cA[1] + cA[3] + cB[1]) * kFix);
          fxq += __float2ll_rn(cB[3] * kFix);  // column 7 (feature 1) of row 8 + g: sum q_g
        }
      };

      // Each warp takes two 32-pixel chunks per step (the chunks of two consecutive grid
      // passes), so two pixels' gathers are in flight per thread, and the step after that
      // one's vertices and normals are loaded meanwhile.
      const int stride = nb * KF_TRACK_THREADS;
      const float4* Nl = a.normal[level];
      const float4* Vl = a.vertex[level];
      const int first = (local * kWarps + warp) * 32;
      float4 n0 = pn0, v0 = pv0, n1 = pn1, v1 = pv1;
      if (pre_level != level) {
        n0 = none; v0 = zero; n1 = none; v1 = zero;
        if (first + lane < P) { n0 = __ldg(Nl + first + lane); v0 = __ldg(Vl + first + lane); }
        if (first + stride + lane < P) { n1 = __ldg(Nl + first + stride + lane); v1 = __ldg(Vl + first + stride + lane); }
      }
      for (int base = first; base < P; base += 2 * stride) {
        const int i0 = base + lane, i1 = base + stride + lane;
        const float4 na = n0, va = v0, nb1 = n1, vb1 = v1;
        n0 = none; v0 = zero; n1 = none; v1 = zero;
        if (i0 + 2 * stride < P) { n0 = __ldg(Nl + i0 + 2 * stride); v0 = __ldg(Vl + i0 + 2 * stride); }
        if (i1 + 2 * stride < P) { n1 = __ldg(Nl + i1 + 2 * stride); v1 = __ldg(Vl + i1 + 2 * stride); }
        float f0[7] = {0, 0, 0, 0, 0, 0, 0}, f1[7] = {0, 0, 0, 0, 0, 0, 0};
        float pw0[3] = {0, 0, 0}, pw1[3] = {0, 0, 0};
        float q0[3], q1[3];
        int st0 = 0, st1 = 0, r0 = 0, r1 = 0;
        if (i0 < P) st0 = track_project(a, na, va, s_T, s_V, q0, &r0);
        if (i1 < P) st1 = track_project(a, nb1, vb1, s_T, s_V, q1, &r1);
        const bool g0 = i0 < P && st0 == 0, g1 = i1 < P && st1 == 0;
        float4 rn0 = zero, rv0 = zero, rn1 = zero, rv1 = zero;
        if (g0) { rn0 = __ldg(&a.ref_normal[r0]); rv0 = __ldg(&a.ref_vertex[r0]); }
        if (g1) { rn1 = __ldg(&a.ref_normal[r1]); rv1 = __ldg(&a.ref_vertex[r1]); }
        if (g0) st0 = track_finish(a, na, q0, rn0, rv0, s_T, c, f0, pw0);
        if (g1) st1 = track_finish(a, nb1, q1, rn1, rv1, s_T, c, f1, pw1);
        if (i0 < P) {
          a.status[level][i0] = st0;
          if (a.q1 && ((i0 / Wl) & 7) != 7) st0 = 0;  // only work group 7 reaches the solver
        }
        if (i1 < P) {
          a.status[level][i1] = st1;
          if (a.q1 && ((i1 / Wl) & 7) != 7) st1 = 0;
        }
        accumulate(st0 == 1, f0, pw0);
        if (base + stride < P) accumulate(st1 == 1, f1, pw1);  // warp-uniform
      }

      // ---------------- block sums -> the entry's fixed-point rows ----------------
      if constexpr (JTJ == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          float v = pacc[k];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (lane == 0) s_pw[warp][k] = v;
        }
#pragma unroll
        for (int k = 0; k < 28; ++k) {
          float v = acc[k];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (lane == 0) s_warp[warp][k] = v;
        }
        __syncthreads();
        if (tid < 32) {
          float v = 0.0f;
#pragma unroll
          for (int w = 0; w < kWarps; ++w) v += tid < 28 ? s_warp[w][tid] : s_pw[w][tid - 28];
          atomicAdd(reinterpret_cast<unsigned long long*>(accbuf + tid), (unsigned long long)__float2ll_rn(v * kFix));
        }
      } else {
        // lane (g, t) holds M[g][2t], M[g][2t+1]; lanes t == 3 also sum q_g
        const int g = lane >> 2, t = lane & 3;
        s_fix[warp][g * 8 + 2 * t] = fx0;
        s_fix[warp][g * 8 + 2 * t + 1] = fx1;
        if (t == 3) s_fix[warp][64 + g] = fxq;
        __syncthreads();
        if (tid < 32) {
          // row layout of reduce.cs: 0 sum e^2, 1..6 sum J e, 7..27 J^T J (upper, row-major);
          // then 28 valid count, 29..31 sum of the points (q = hi(p) + mid(p))
          long long v = 0;
          if (tid < 28) {
            int r, cc;
            if (tid == 0) { r = 6; cc = 6; }
            else if (tid < 7) { r = tid - 1; cc = 6; }
            else {
              int q = tid - 7;
              r = 0;
              while (q >= 6 - r) { q -= 6 - r; ++r; }
              cc = r + q;
            }
#pragma unroll
            for (int w = 0; w < kWarps; ++w) v += s_fix[w][r * 8 + cc];
          } else if (tid == 28) {
#pragma unroll
            for (int w = 0; w < kWarps; ++w) v += s_fix[w][63];
          } else {
#pragma unroll
            for (int w = 0; w < kWarps; ++w) v += s_fix[w][64 + tid - 29] + s_fix[w][64 + tid - 26];
          }
          atomicAdd(reinterpret_cast<unsigned long long*>(accbuf + tid), (unsigned long long)v);
        }
      }
      // the buffer of the next iteration was last read before the previous barrier
      if (local == 0 && tid >= 32 && tid < 64) a.st->icp_acc[(gi + 1u) % 3u][tid - 32][0] = 0;

      // ---------------- grid barrier; then every block solves ----------------
      // Every block reads the same exact sums and solves the same system in FP64, so all
      // blocks hold bit-identical results without a second hand-over, and the solve's code
      // stays warm in every SM's instruction cache.
      ok = kf_grid_sync(st, &st->barrier_count, nb * (gi + 1u), &s_flag);
      if (!ok) break;
      {
        // the next iteration runs this level again unless the level's iterations are used up
        // or this solve converges; the first case is known now, the second is rare
        const int nl = it + 1 < a.iters[level] ? level : level - 1;
        pre_level = nl;
        pn0 = none; pv0 = zero; pn1 = none; pv1 = zero;
        if (nl >= 0) {
          const int Pn = a.W[nl] * a.H[nl];
          const int f0 = (local * kWarps + warp) * 32;
          if (f0 + lane < Pn) { pn0 = __ldg(a.normal[nl] + f0 + lane); pv0 = __ldg(a.vertex[nl] + f0 + lane); }
          if (f0 + stride + lane < Pn) {
            pn1 = __ldg(a.normal[nl] + f0 + stride + lane);
            pv1 = __ldg(a.vertex[nl] + f0 + stride + lane);
          }
        }
      }
      if (tid < 32) s_sums[tid] = (double)__ldcg(accbuf + tid) * kInvFix;
      __syncthreads();
      if (warp == 1) {
        // the rank guard's check (KF_ICP_RANK_TAU), in FP32 by lane 0 beside warp 0's FP64
        // solve (measured 1-2 us per frame faster than the check spread over the warp's lanes)
        if (lane == 0) s_fast = kf_icp_rank_check_thread(&s_sums[7], s_cd);
        asm volatile("bar.sync 1, 64;" ::: "memory");  // warps 0 and 1
      }
      if (warp == 0) {
        // ---- solve in warp 0 ----
        // reduce.cs counts every pixel of the (group-7) rows in sums[28]
        const double count = a.q1 ? (double)Wl * (double)(Hl / 8) : (double)P;
        const double nvalid = s_sums[28];
        const double cx = s_cd[0], cy = s_cd[1], cz = s_cd[2];
        // lane 0 factors and solves; the step reaches the other lanes through shared memory
        double xp[6];
        bool spd = false;
        if (lane == 0) {
          spd = kf_cholesky6_thread(&s_sums[7], &s_sums[1], xp);
#pragma unroll
          for (int k = 0; k < 6; ++k) s_gx[k] = xp[k];
          s_gx[6] = spd ? 1.0 : 0.0;
        }
        __syncwarp();
#pragma unroll
        for (int k = 0; k < 6; ++k) xp[k] = s_gx[k];
        spd = s_gx[6] != 0.0;
        // back to the reference's variables: w = w', t = t' - w x c
        double x[6];
        x[3] = xp[3]; x[4] = xp[4]; x[5] = xp[5];
        x[0] = xp[0] - (x[4] * cz - x[5] * cy);
        x[1] = xp[1] - (x[5] * cx - x[3] * cz);
        x[2] = xp[2] - (x[3] * cy - x[4] * cx);
        asm volatile("bar.sync 1, 64;" ::: "memory");  // warp 1's rank check is in s_fast
        if (!(spd && s_fast)) {
          // a degenerate view (rare): the rank-guarded minimum-norm step of the world-frame
          // system (JacobiSVD::solve, :696-697, with the cut of KF_ICP_RANK_TAU)
          if (lane == 0) kf_icp_world_guarded_step(&s_sums[7], &s_sums[1], s_cd, s_gx, s_gx + 8);
          __syncwarp();
#pragma unroll
          for (int k = 0; k < 6; ++k) x[k] = s_gx[k];
          __syncwarp();
        }
        // delta = eulerAngleXYZ(x3, x4, x5), delta[3].xyz = x0..2 (gFusion.cpp:700-703);
        // lanes 0..2 evaluate the three sincos at once
        double sn, cs;
        kf_sincos_step(lane == 0 ? x[3] : (lane == 1 ? x[4] : x[5]), &sn, &cs);
        const double sa = __shfl_sync(0xffffffffu, sn, 0), ca = __shfl_sync(0xffffffffu, cs, 0);
        const double sb = __shfl_sync(0xffffffffu, sn, 1), cb = __shfl_sync(0xffffffffu, cs, 1);
        const double sc = __shfl_sync(0xffffffffu, sn, 2), cc = __shfl_sync(0xffffffffu, cs, 2);
        double R[9];
        kf_euler_xyz_from_sincos(sa, ca, sb, cb, sc, cc, R);
        // pose = delta * pose, one element per lane (delta column-major: R | x0..2)
        double pn = 0.0;
        if (lane < 16) {
          const int r = lane & 3, col = lane >> 2;
          // row r of delta, selected without indexing registers by lane
          const double d0 = r == 0 ? R[0] : (r == 1 ? R[1] : (r == 2 ? R[2] : 0.0));
          const double d1 = r == 0 ? R[3] : (r == 1 ? R[4] : (r == 2 ? R[5] : 0.0));
          const double d2 = r == 0 ? R[6] : (r == 1 ? R[7] : (r == 2 ? R[8] : 0.0));
          const double d3 = r == 0 ? x[0] : (r == 1 ? x[1] : (r == 2 ? x[2] : 1.0));
          pn += d0 * s_pose[col * 4 + 0];
          pn += d1 * s_pose[col * 4 + 1];
          pn += d2 * s_pose[col * 4 + 2];
          pn += d3 * s_pose[col * 4 + 3];
        }
        // the centred row and its centre; the tail turns the last one into the world form
        if (lane < 28) s_csums[lane] = s_sums[lane];
        if (lane == 28) s_csums[28] = count;
        // the convergence test and the next centre (this iteration's centroid of the valid
        // points) in every lane: one instruction stream, no divergent FP64 square root or
        // division on the hand-over's path
        const double nrm = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + x[3] * x[3] +
                                x[4] * x[4] + x[5] * x[5]);
        if (lane == 29) s_conv = (nrm < 1e-5 && nrm != 0.0) ? 1 : 0;
        if (lane == 31) s_nvalid = nvalid;
        const int ci = lane < 3 ? lane : 2;
        const double centroid = s_sums[29 + ci] / nvalid;  // unused when nvalid == 0
        const double cn = nvalid > 0 ? centroid : s_cd[ci];
        __syncwarp();
        if (lane < 16) {
          s_pose[lane] = pn;
          s_T[lane] = (float)pn;
        }
        if (lane < 3) {
          s_ccenter[lane] = s_cd[lane];
          s_cd[lane] = cn;
          s_c[lane] = (float)cn;
        }
        __syncwarp();
        if (a.same_pixel && lane == 0) make_float_mats(a, s_pose, s_ray, s_T, s_V);
      }
      ++gi;
      __syncthreads();
      ++iters_run;
      if (s_conv) break;  // result.norm() < 1e-5 && != 0 leaves this level (:707-708)
    }
  }

  // ---------------- Track() tail (:715-723) + frame policy, block 0 only -----------------
  if (local != 0 || tid != 0 || !ok) return;
  const double ae = iters_run ? sqrt(s_csums[0] / s_csums[28]) : 0.0;  // getReduction :1167
  st->ae = ae;
  if (iters_run) {
    // the last reduction row in the reference's world form: b = M b', C = M C' M^T,
    // M = [[I, 0], [[c]x, I]]
    const double* cs = s_csums;
    const double cx = s_ccenter[0], cy = s_ccenter[1], cz = s_ccenter[2];
    double Cp[36], Mx[36], MC[36];
    kf_make_jtj(&cs[7], Cp);
    for (int k = 0; k < 36; ++k) Mx[k] = (k % 7 == 0) ? 1.0 : 0.0;
    Mx[3 * 6 + 1] = -cz; Mx[3 * 6 + 2] = cy;
    Mx[4 * 6 + 0] = cz;  Mx[4 * 6 + 2] = -cx;
    Mx[5 * 6 + 0] = -cy; Mx[5 * 6 + 1] = cx;
    st->sums[0] = cs[0];
    for (int r = 0; r < 6; ++r) {
      double v = 0;
      for (int k = 0; k < 6; ++k) v += Mx[r * 6 + k] * cs[1 + k];
      st->sums[1 + r] = v;
    }
    for (int r = 0; r < 6; ++r)
      for (int cc = 0; cc < 6; ++cc) {
        double v = 0;
        for (int k = 0; k < 6; ++k) v += Mx[r * 6 + k] * Cp[k * 6 + cc];
        MC[r * 6 + cc] = v;
      }
    int q = 7;
    for (int r = 0; r < 6; ++r)
      for (int cc = r; cc < 6; ++cc) {
        double v = 0;
        for (int k = 0; k < 6; ++k) v += MC[r * 6 + k] * Mx[cc * 6 + k];
        st->sums[q++] = v;
      }
    st->sums[28] = cs[28];
    st->sums[29] = st->sums[30] = st->sums[31] = 0.0;
  }
  // AE == 0 fails the frame (gFusion.cpp:715-723): in the reference that means no valid
  // pixel.  Here the energy is a fixed-point sum, which rounds residuals of a few microns to
  // exactly 0 (per 32-pixel chunk with split-BF16); with valid pixels the frame is tracked.
  const bool no_energy = ae == 0.0 && !(iters_run && s_nvalid > 0.0);
  int tracked;
  if (ae > 0.5 || no_energy) {
    tracked = 0;
    kf_store_pose(st, s_old);
  } else {
    tracked = 1;
    kf_store_pose(st, s_pose);
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
    // keep the centroid for the next frame, in the camera frame of the tracked pose
    double inv[16];
    kf_rigid_inverse(s_pose, inv);
    for (int r = 0; r < 3; ++r)
      st->icp_center_cam[r] = inv[r] * s_cd[0] + inv[4 + r] * s_cd[1] + inv[8 + r] * s_cd[2] + inv[12 + r];
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

namespace {

IcpArgs make_icp_args(kf_session* s, int frame_policy) {
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
  a.st = s->d_state;
  return a;
}

cudaLaunchConfig_t coop_config(dim3 grid, cudaStream_t stream, cudaLaunchAttribute* attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(KF_TRACK_THREADS);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

}  // namespace

int kf_launch_icp(kf_session* s, int frame_policy, bool words_zero) {
  const IcpArgs a = make_icp_args(s, frame_policy);
  const void* fn = (s->cfg.jtj == KF_JTJ_SPLIT_BF16) ? (const void*)icp_kernel<1, false>
                                                      : (const void*)icp_kernel<0, false>;
  int blocks = kf_occupancy_blocks(s, fn, KF_TRACK_THREADS, 0);
  if (blocks <= 0) return KF_ERR_CUDA;
  // the barrier counter and the sum buffers start at zero for every launch
  if (!words_zero) KF_CUDA_TRY(s, kf_clear_icp_words(s->d_state, s->stream));
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = coop_config(dim3(blocks), s->stream, attr);
  const IcpBatch none = {nullptr, nullptr};
  if (s->cfg.jtj == KF_JTJ_SPLIT_BF16)
    KF_CUDA_TRY(s, cudaLaunchKernelEx(&cfg, icp_kernel<1, false>, a, none));
  else
    KF_CUDA_TRY(s, cudaLaunchKernelEx(&cfg, icp_kernel<0, false>, a, none));
  kf_note_launch(s);
  return KF_OK;
}

// ---- batched: every member's frame-step ICP in one cooperative launch ----
int kf_batch_prepare_icp(kf_batch* b) {
  const int n = (int)b->members.size();
  IcpArgs* h = nullptr;
  b->icp_args = kf_batch_table(b, sizeof(IcpArgs) * n, reinterpret_cast<void**>(&h));
  if (!b->icp_args) return KF_ERR_CAPACITY;
  for (int e = 0; e < n; ++e) h[e] = make_icp_args(b->members[e], 1);
  kf_session* s0 = b->members[0];
  const void* fn = (s0->cfg.jtj == KF_JTJ_SPLIT_BF16) ? (const void*)icp_kernel<1, true>
                                                       : (const void*)icp_kernel<0, true>;
  const int total = kf_occupancy_blocks(s0, fn, KF_TRACK_THREADS, 0);
  if (total <= 0) return KF_ERR_CUDA;
  b->icp_blocks = total;
  b->icp_waves = 0;
  for (int e0 = 0; e0 < n; e0 += KF_BATCH_ICP_WAVE) {
    int rc = kf_batch_block_map_range(b, total, e0, std::min(n, e0 + KF_BATCH_ICP_WAVE), &b->icp_wave_map[b->icp_waves]);
    if (rc) return rc;
    ++b->icp_waves;
  }
  return KF_OK;
}

int kf_batch_launch_icp(kf_batch* b) {
  for (int w = 0; w < b->icp_waves; ++w) {
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = coop_config(dim3(b->icp_blocks), b->stream, attr);
    const IcpBatch batch = {static_cast<const IcpArgs*>(b->icp_args), b->icp_wave_map[w]};
    const IcpArgs none{};
    if (b->members[0]->cfg.jtj == KF_JTJ_SPLIT_BF16)
      KF_CUDA_TRY(b, cudaLaunchKernelEx(&cfg, icp_kernel<1, true>, none, batch));
    else
      KF_CUDA_TRY(b, cudaLaunchKernelEx(&cfg, icp_kernel<0, true>, none, batch));
    b->launches += 1;
  }
  return KF_OK;
}
