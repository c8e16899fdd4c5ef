// kf_sdf.cu — direct SDF tracking (and pose recovery) as one persistent launch.
//
// Reference: gFusion::TrackSDF (src/gFusion.cpp:835-1038), gFusion::trackSDF
// (:1040-1098) with shaders/trackSDF.cs:407-531, gFusion::reduceSDF (:1100-1125) with
// shaders/reduceSDF.cs:28-116, getSDFReduction (:1195-1232), Twist (:811-833) and
// gFusion::recoverPose (:1616-1653).
//
// Per pixel: p = camToWorld * v; the voxel coordinate cvp = p * volSize / volDim - 0.5
// (x and y get -0.5 twice in the reference, trackSDF.cs:429, Q23); D = trilinear SDF()
// with modf (truncation) semantics and zero outside the volume (:193-224); gradient by
// +-1-voxel central differences over 2 * voxel size (:227-237); J = [p x g, g] (the
// dx/dxi table of :459-468 with xi = (w, v)); Huber weight h = 1 if |D| < 0.02 else
// 0.02 / |D|; |D| >= 1 writes a zero row.  The reduction adds D^2 twice (Q6) and reads
// the last column's row left over from an earlier call (Q7).  The solve scales the
// system by 1 / max(C), adds iteration * 0.01 * I, and does result -= LDLT(C)^-1 b in
// FP64; camToWorld = exp(Twist(result)) * m_pose_eig_prev.
//
// B200 design: like kf_icp.cu, one cooperative launch holds every level and iteration;
// after a grid barrier every block reduces the per-block rows in the same fixed order in
// FP64 and solves the same system.  In recover mode the same launch walks the pose library (recoverPose) and
// stops at the first pose that tracks.  The persistent row buffer is only written at
// indices that some level reads back as its stale last column.
#include "kf_internal.cuh"

namespace {

struct SdfArgs {
  const float4* vertex[3];
  int W[3], H[3];
  const void* vol;
  int nx, ny, nz;
  float sx, sy, sz;   // volSize / volDim
  float inv2vs;       // 1 / (2 * volDim.x / volSize.x)
  int iters[3];
  int q1, q6, q7, q23;
  float* rows;        // persistent reduSDFType SSBO: 8 floats per pixel index
  float* partials;
  KfDevState* st;
  int recover;        // walk the pose library (recoverPose)
  const int* gate;    // need_recover flag (frame step)
};

template <int S>
__device__ __forceinline__ float vol_tap(const SdfArgs& a, int x, int y, int z) {
  // imageLoad returns 0 outside the image
  if ((unsigned)x >= (unsigned)a.nx || (unsigned)y >= (unsigned)a.ny || (unsigned)z >= (unsigned)a.nz)
    return 0.0f;
  const typename Vox<S>::V* f = reinterpret_cast<const typename Vox<S>::V*>(a.vol);
  return Vox<S>::raw(f, (size_t)x + (size_t)a.nx * ((size_t)y + (size_t)a.ny * z)) * Vox<S>::kRawToF;
}

// SDF() of trackSDF.cs:193-224
template <int S>
__device__ __forceinline__ float sdf_sample(const SdfArgs& a, float lx, float ly, float lz) {
  const float ix = truncf(lx), iy = truncf(ly), iz = truncf(lz);
  const float x = lx - ix, y = ly - iy, z = lz - iz;
  const int I = (int)ix, J = (int)iy, K = (int)iz;
  const float N0 = vol_tap<S>(a, I, J, K), N1 = vol_tap<S>(a, I, J + 1, K);
  const float N2 = vol_tap<S>(a, I + 1, J, K), N3 = vol_tap<S>(a, I + 1, J + 1, K);
  const float N4 = vol_tap<S>(a, I, J, K + 1), N5 = vol_tap<S>(a, I, J + 1, K + 1);
  const float N6 = vol_tap<S>(a, I + 1, J, K + 1), N7 = vol_tap<S>(a, I + 1, J + 1, K + 1);
  const float a0 = N0 * (1.0f - z) + N4 * z, a1 = N1 * (1.0f - z) + N5 * z;
  const float b0 = N2 * (1.0f - z) + N6 * z, b1 = N3 * (1.0f - z) + N7 * z;
  return (a0 * (1.0f - y) + a1 * y) * (1.0f - x) + (b0 * (1.0f - y) + b1 * y) * x;
}

// trackSDF.cs:413-520 for one pixel: row = (h, D, J0..J5)
template <int S>
__device__ __forceinline__ void sdf_row(const SdfArgs& a, int l, size_t i, const float* T, float* row) {
  const float4 v = __ldg(&a.vertex[l][i]);
  const float px = fmaf(T[0], v.x, fmaf(T[4], v.y, fmaf(T[8], v.z, T[12])));
  const float py = fmaf(T[1], v.x, fmaf(T[5], v.y, fmaf(T[9], v.z, T[13])));
  const float pz = fmaf(T[2], v.x, fmaf(T[6], v.y, fmaf(T[10], v.z, T[14])));
  const float off = a.q23 ? 1.0f : 0.5f;
  const float cx = px * a.sx - off, cy = py * a.sy - off, cz = pz * a.sz - 0.5f;
  const float D = sdf_sample<S>(a, cx, cy, cz);
  const float gx = (sdf_sample<S>(a, cx + 1.0f, cy, cz) - sdf_sample<S>(a, cx - 1.0f, cy, cz)) * a.inv2vs;
  const float gy = (sdf_sample<S>(a, cx, cy + 1.0f, cz) - sdf_sample<S>(a, cx, cy - 1.0f, cz)) * a.inv2vs;
  const float gz = (sdf_sample<S>(a, cx, cy, cz + 1.0f) - sdf_sample<S>(a, cx, cy, cz - 1.0f)) * a.inv2vs;
  if (D < 1.0f && D > -1.0f) {
    const float ad = fabsf(D);
    row[0] = ad < 0.02f ? 1.0f : 0.02f / ad;
    row[1] = D;
    row[2] = py * gz - pz * gy;
    row[3] = pz * gx - px * gz;
    row[4] = px * gy - py * gx;
    row[5] = gx;
    row[6] = gy;
    row[7] = gz;
  } else {
#pragma unroll
    for (int k = 0; k < 8; ++k) row[k] = 0.0f;
  }
}

constexpr int kWarps = KF_TRACK_THREADS / 32;

// A batched launch: the blocks of entry e are those whose map word names e (as in
// kf_icp.cu); every entry runs its own attempts, levels, iterations and barrier.
struct SdfBatch {
  const SdfArgs* args;
  const uint32_t* block_map;  // per block: entry << 24 | blocks of the entry << 12 | index
};

template <int S, bool BATCH>
__global__ void __launch_bounds__(KF_TRACK_THREADS) sdf_kernel(SdfArgs a_one, SdfBatch batch) {
  __shared__ SdfArgs s_args;
  __shared__ double s_prev[16];     // m_pose_eig_prev
  __shared__ double s_result[6];
  __shared__ float s_T[16];
  __shared__ float s_warp[kWarps][28];
  __shared__ double s_red[kWarps][32];
  __shared__ double s_sums[32];
  __shared__ int s_flag, s_conv;

  unsigned local, nb;  // this block's index among its entry's blocks, and their number
  if constexpr (BATCH) {
    const uint32_t m = batch.block_map[blockIdx.x];
    local = m & 0xfffu;
    nb = (m >> 12) & 0xfffu;
    const int* src = reinterpret_cast<const int*>(batch.args + (m >> 24));
    for (int k = threadIdx.x; k < (int)(sizeof(SdfArgs) / 4); k += blockDim.x)
      reinterpret_cast<int*>(&s_args)[k] = __ldg(src + k);
    __syncthreads();
  } else {
    local = blockIdx.x;
    nb = gridDim.x;
  }
  const SdfArgs& a = BATCH ? s_args : a_one;
  KfDevState* st = a.st;
  if (a.gate && *(volatile const int*)a.gate == 0) return;  // uniform over the entry's blocks
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int attempts = a.recover ? st->lib_size : 1;
  if (tid < 16) s_prev[tid] = st->pose_eig[tid];
  __syncthreads();

  bool ok = true, found = false;
  int iters_run = 0;
  unsigned gi = 0;  // iterations of this launch so far: grid barrier target and partials buffer
  for (int attempt = 0; attempt < attempts && ok && !found; ++attempt) {
    if (tid < 6) s_result[tid] = 0.0;
    if (tid < 16) s_T[tid] = (float)s_prev[tid];  // exp(0) * prev
    __syncthreads();
    bool tracked = false;
    for (int level = 2; level >= 0 && ok; --level) {
      const int Wl = a.W[level], Hl = a.H[level];
      const int P = Wl * Hl;
      for (int it = 0; it < a.iters[level]; ++it) {
        float T[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) T[k] = s_T[k];
        float acc[28];
#pragma unroll
        for (int k = 0; k < 28; ++k) acc[k] = 0.0f;
        const float e2 = a.q6 ? 2.0f : 1.0f;
        for (int i = local * KF_TRACK_THREADS + tid; i < P; i += nb * KF_TRACK_THREADS) {
          const int y = i / Wl, x = i - y * Wl;
          float row[8];
          if (a.q7 && x == Wl - 1) {
            // stale row of an earlier call (the reference never writes this column)
#pragma unroll
            for (int k = 0; k < 8; ++k) row[k] = __ldcg(&a.rows[(size_t)i * 8 + k]);
          } else {
            sdf_row<S>(a, level, (size_t)i, T, row);
            if (a.q7 && (((i + 1) % a.W[0]) == 0 || ((i + 1) % a.W[1]) == 0 || ((i + 1) % a.W[2]) == 0)) {
#pragma unroll
              for (int k = 0; k < 8; ++k) a.rows[(size_t)i * 8 + k] = row[k];
            }
          }
          if (a.q1 && (y & 7) != 7) continue;
          const float h = row[0], D = row[1];
          acc[0] += e2 * D * D;
#pragma unroll
          for (int k = 0; k < 6; ++k) acc[1 + k] += h * row[2 + k] * D;
          int q = 7;
#pragma unroll
          for (int r = 0; r < 6; ++r)
#pragma unroll
            for (int c = r; c < 6; ++c) acc[q++] += h * row[2 + r] * row[2 + c];
        }
#pragma unroll
        for (int k = 0; k < 28; ++k) {
          float v = acc[k];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (lane == 0) s_warp[warp][k] = v;
        }
        // two partial buffers, alternating by iteration (see kf_icp.cu)
        float* part = a.partials + (size_t)(gi & 1u) * KF_MAX_TRACK_BLOCKS * 32;
        __syncthreads();
        if (tid < 28) {
          float v = 0.0f;
#pragma unroll
          for (int w = 0; w < kWarps; ++w) v += s_warp[w][tid];
          part[(size_t)local * 32 + tid] = v;
        }

        // grid barrier; then every block reduces the rows in the same fixed order and
        // solves the same system, so every block holds bit-identical results
        ok = kf_grid_sync(st, &st->sdf_barrier_count, nb * (gi + 1u), &s_flag);
        if (!ok) break;
        ++gi;
        {
          const int k = tid & 31, r = tid >> 5;
          double v = 0.0;
          if (k < 28)
            for (unsigned b = r; b < nb; b += kWarps) v += (double)__ldcg(&part[(size_t)b * 32 + k]);
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
          const double count = a.q1 ? (double)Wl * (double)(Hl / 8) : (double)P;
          s_sums[28] = count;
          s_sums[29] = s_sums[30] = s_sums[31] = 0.0;
          double b[6], C[36], dx[6];
          for (int k = 0; k < 6; ++k) b[k] = s_sums[1 + k];
          kf_make_jtj(&s_sums[7], C);
          const double ae = sqrt(s_sums[0] / count);
          double mx = C[0];
          for (int k = 1; k < 36; ++k) mx = fmax(mx, C[k]);  // maxCoeff (:890)
          const double scaling = 1.0 / mx;
          for (int k = 0; k < 36; ++k) C[k] *= scaling;
          for (int k = 0; k < 6; ++k) b[k] *= scaling;
          for (int k = 0; k < 6; ++k) C[k * 7] += (double)it * 0.01;
          kf_ldlt6(C, b, dx);
          double cn = 0.0;
          for (int k = 0; k < 6; ++k) {
            const double prev = s_result[k];
            const double res = prev - dx[k];
            const double ch = res - prev;
            cn += ch * ch;
            s_result[k] = res;
          }
          cn = sqrt(cn);
          double E[16], Tn[16], res[6];
          for (int k = 0; k < 6; ++k) res[k] = s_result[k];
          kf_se3_exp(res, E);
          kf_mat4_mul(E, s_prev, Tn);
          for (int k = 0; k < 16; ++k) s_T[k] = (float)Tn[k];
          s_conv = ((ae != 0.0 && ae < 1e-3) || cn < 1e-3) ? 1 : 0;
          if (local == 0) {
            st->ae = ae;
            for (int k = 0; k < 32; ++k) st->sums[k] = s_sums[k];
          }
        }
        __syncthreads();
        ++iters_run;
        if (s_conv) {
          tracked = true;
          break;  // inner loop only (:906-920)
        }
      }
    }
    if (!ok) break;
    // TrackSDF tail (:991-1012), block 0 writes the state
    if (local == 0 && tid == 0) {
      double res[6], sum = 0.0;
      for (int k = 0; k < 6; ++k) { res[k] = s_result[k]; sum += res[k]; }
      if (isnan(sum))
        for (int k = 0; k < 6; ++k) res[k] = 0.0;
      if (tracked) {
        double E[16], Pn[16];
        kf_se3_exp(res, E);
        kf_mat4_mul(E, s_prev, Pn);
        for (int k = 0; k < 16; ++k) st->pose_eig[k] = Pn[k];
        kf_store_pose(st, Pn);
        for (int k = 0; k < 6; ++k) st->cum_twist[k] += res[k];
      } else {
        // m_pose = oldPose: the pose at entry, i.e. the library pose in recover mode
        if (a.recover)
          kf_store_pose(st, st->lib_pose[attempt]);
      }
      if (!a.recover) st->tracked = tracked ? 1 : 0;  // recoverPose leaves `tracked` alone
      st->iterations_run = iters_run;
    }
    found = tracked;
  }
  if (local == 0 && tid == 0 && ok && a.recover) st->recover_found = found ? 1 : 0;
}

}  // namespace

namespace {

SdfArgs make_sdf_args(kf_session* s, int recover, int gated) {
  SdfArgs a;
  for (int l = 0; l < 3; ++l) {
    a.vertex[l] = s->d_vertex[l];
    a.W[l] = s->W[l];
    a.H[l] = s->H[l];
    a.iters[l] = s->cfg.iterations[l];
  }
  a.vol = s->d_vol;
  a.nx = s->cfg.nx; a.ny = s->cfg.ny; a.nz = s->cfg.nz;
  a.sx = (float)a.nx / s->cfg.dim_x;
  a.sy = (float)a.ny / s->cfg.dim_y;
  a.sz = (float)a.nz / s->cfg.dim_z;
  a.inv2vs = 1.0f / (2.0f * (s->cfg.dim_x / (float)a.nx));
  const uint32_t q = s->cfg.quirks;
  a.q1 = (q & KF_Q1_LAST_GROUP_ONLY) ? 1 : 0;
  a.q6 = (q & KF_Q6_SDF_D2_TWICE) ? 1 : 0;
  a.q7 = (q & KF_Q7_SDF_LAST_COLUMN) ? 1 : 0;
  a.q23 = (q & KF_Q23_SDF_XY_OFFSET) ? 1 : 0;
  a.rows = s->d_sdf_rows;
  a.partials = s->d_partials;
  a.st = s->d_state;
  a.recover = recover;
  a.gate = gated ? &s->d_state->need_recover : nullptr;
  return a;
}

template <bool BATCH>
const void* sdf_fn(int storage) {
  switch (storage) {
    case KF_STORAGE_F32F32: return (const void*)sdf_kernel<KF_STORAGE_F32F32, BATCH>;
    case KF_STORAGE_F16U16: return (const void*)sdf_kernel<KF_STORAGE_F16U16, BATCH>;
    default: return (const void*)sdf_kernel<KF_STORAGE_RG16I, BATCH>;
  }
}

template <bool BATCH>
cudaError_t launch_sdf(int storage, int blocks, cudaStream_t stream, const SdfArgs& a, const SdfBatch& b) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(KF_TRACK_THREADS);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  switch (storage) {
    case KF_STORAGE_F32F32: return cudaLaunchKernelEx(&cfg, sdf_kernel<KF_STORAGE_F32F32, BATCH>, a, b);
    case KF_STORAGE_F16U16: return cudaLaunchKernelEx(&cfg, sdf_kernel<KF_STORAGE_F16U16, BATCH>, a, b);
    default: return cudaLaunchKernelEx(&cfg, sdf_kernel<KF_STORAGE_RG16I, BATCH>, a, b);
  }
}

}  // namespace

int kf_launch_sdf(kf_session* s, int recover, int gated, int frame_policy, bool counter_zero) {
  (void)frame_policy;
  const SdfArgs a = make_sdf_args(s, recover, gated);
  const int blocks = kf_occupancy_blocks(s, sdf_fn<false>(s->cfg.storage), KF_TRACK_THREADS, 0);
  if (blocks <= 0) return KF_ERR_CUDA;
  if (!counter_zero) KF_CUDA_TRY(s, cudaMemsetAsync(&s->d_state->sdf_barrier_count, 0, sizeof(unsigned), s->stream));
  KF_CUDA_TRY(s, launch_sdf<false>(s->cfg.storage, blocks, s->stream, a, SdfBatch{nullptr, nullptr}));
  kf_note_launch(s);
  return KF_OK;
}

// ---- batched: every member's gated recoverPose in one cooperative launch ----
int kf_batch_prepare_sdf(kf_batch* b) {
  const int n = (int)b->members.size();
  SdfArgs* h = nullptr;
  b->sdf_args = kf_batch_table(b, sizeof(SdfArgs) * n, reinterpret_cast<void**>(&h));
  if (!b->sdf_args) return KF_ERR_CAPACITY;
  for (int e = 0; e < n; ++e) h[e] = make_sdf_args(b->members[e], 1, 1);
  kf_session* s0 = b->members[0];
  const int total = kf_occupancy_blocks(s0, sdf_fn<true>(s0->cfg.storage), KF_TRACK_THREADS, 0);
  if (total <= 0) return KF_ERR_CUDA;
  b->sdf_blocks = total;
  return kf_batch_block_map(b, total, &b->sdf_map);
}

int kf_batch_launch_sdf_recover(kf_batch* b) {
  const SdfBatch batch = {static_cast<const SdfArgs*>(b->sdf_args), b->sdf_map};
  KF_CUDA_TRY(b, launch_sdf<true>(b->members[0]->cfg.storage, b->sdf_blocks, b->stream, SdfArgs{}, batch));
  b->launches += 1;
  return KF_OK;
}
