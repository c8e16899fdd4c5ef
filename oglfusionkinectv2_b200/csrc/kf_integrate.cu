// kf_integrate.cu — TSDF fusion of one depth frame.
//
// Reference: gFusion::integrate (src/gFusion.cpp:1234-1287) and shaders/integrate.cs:52-169:
// one thread per (x, y) voxel column marching z; voxel centre ((i + 0.5) * volDim /
// volSize) to camera by inverse(m_pose); skip z < 1e-4, pixels outside the 512x424
// image (:54, Q11) and zero depth; eta = (d - z) * sqrt(1 + (x/z)^2 + (y/z)^2); if
// eta > -mu the running average (w*F + min(1, eta/mu)) / (w + 1) is kept only when it is
// below 0.2, clamped to [-0.1, 0.2] with w = min(w + 1, maxWeight); otherwise (and for
// eta <= -mu) value and weight are zeroed (Q8).
//
// B200 design: a block owns 32 x 8 columns by ZC z (one warp = 32 consecutive x: 64 B
// per plane per z-step for 2-byte storage, fully used sectors); splitting the z-march
// over ZC-voxel chunks (8, 16 or 32, tuned per volume) gives the SMs enough independent
// warps to hide the depth-gather and volume latencies.  A block whose voxel box lies outside one of the five frustum
// half-spaces returns at once, so voxels that cannot project into the image cost nothing;
// inside, every voxel runs the reference's tests.  Per voxel one reciprocal replaces the
// shader's divisions by z (u = fx * x/z + cx + 0.5 is the reference's (fx x + cx z)/z + 0.5
// up to rounding), and the reciprocal, square root and running-average division use the
// hardware approximations (2 ulp; GLSL allows 2.5 ulp for division).  The weight plane is read only where eta > -mu, and a voxel whose
// encoded value and weight do not change is not written back.
#include "kf_internal.cuh"

namespace {

struct IntArgs {
  void* vol;
  size_t count;
  int nx, ny, nz;
  float dimx, dimy, dimz;
  const float* depth;
  int W, H;
  float fx, fy, cx, cy;
  float mu, inv_mu, maxw;
  int band;  // Q8
  const int* gate;
  const KfDevState* st;
  uint32_t* bricks;
  int bx, by, bz;
  uint32_t* supers;
  int sbx, sby, sbz;
};

template <class T>
__device__ __forceinline__ uint32_t bits_of(const T& v) {
  uint32_t b = 0;
  memcpy(&b, &v, sizeof(T));
  return b;
}

// Voxels per thread along z (the block's brick of columns is 32 x 8 x ZC): one of
// KF_INT_ZCHUNKS, chosen per session (default 16, or the autotuner's pick).  Every choice
// computes the same volume.

// True when the box of voxel centres [b0, b1] (index space, inclusive) lies entirely on the
// outside of one of the five half-spaces whose intersection is the set of voxels
// integrate.cs can touch: z >= 1e-4, 0 <= u <= W-1, 0 <= v <= H-1 (u, v the +0.5-rounded
// projection).  Conservative: a box that is not culled is tested voxel by voxel.  Called by
// a whole warp: lane & 7 evaluates one corner, the ballots combine them.
__device__ __forceinline__ bool box_outside_frustum(const IntArgs& a, const float* inv, const int* b0, const int* b1) {
  const float vx = a.dimx / a.nx, vy = a.dimy / a.ny, vz = a.dimz / a.nz;
  const float kx0 = a.cx + 0.5f, kx1 = a.cx + 0.5f - (float)(a.W - 1);
  const float ky0 = a.cy + 0.5f, ky1 = a.cy + 0.5f - (float)(a.H - 1);
  const int c = threadIdx.x & 7;
  const float wx = ((c & 1 ? b1[0] : b0[0]) + 0.5f) * vx;
  const float wy = ((c & 2 ? b1[1] : b0[1]) + 0.5f) * vy;
  const float wz = ((c & 4 ? b1[2] : b0[2]) + 0.5f) * vz;
  const float X = inv[0] * wx + inv[1] * wy + inv[2] * wz + inv[3];
  const float Y = inv[4] * wx + inv[5] * wy + inv[6] * wz + inv[7];
  const float Z = inv[8] * wx + inv[9] * wy + inv[10] * wz + inv[11];
  const unsigned o0 = __ballot_sync(0xffffffffu, Z - 1e-4f < 0.0f);
  const unsigned o1 = __ballot_sync(0xffffffffu, a.fx * X + kx0 * Z < 0.0f);
  const unsigned o2 = __ballot_sync(0xffffffffu, -(a.fx * X + kx1 * Z) < 0.0f);
  const unsigned o3 = __ballot_sync(0xffffffffu, a.fy * Y + ky0 * Z < 0.0f);
  const unsigned o4 = __ballot_sync(0xffffffffu, -(a.fy * Y + ky1 * Z) < 0.0f);
  return (o0 & 0xffu) == 0xffu || (o1 & 0xffu) == 0xffu || (o2 & 0xffu) == 0xffu ||
         (o3 & 0xffu) == 0xffu || (o4 & 0xffu) == 0xffu;
}

// The z-chunk [zb, zb + ZC) of column (x, y); returns which z-bricks received a negative
// value (bit j = brick zb/8 - 1 + j, bit 0 for the dilation of a z % 8 == 0 voxel).
template <int S, int ZC>
__device__ __forceinline__ uint32_t integrate_column(const IntArgs& a, const float* inv, int x, int y, int zb) {
  typedef typename Vox<S>::V V;
  typedef typename Vox<S>::Wt Wt;
  // bits 0..ZC/8: NEG of z-bricks zb/8 - 1 + j; bit 6: NEG of z-super-brick zb/64, bit 7:
  // of zb/64 - 1 (a z % 64 == 0 voxel is that one's +1 layer)
  static_assert(ZC == 8 || ZC == 16 || ZC == 32, "z chunk: 8, 16 or 32 voxels");
  uint32_t flags = 0;

  // getVolumePosition (integrate.cs:16-19; along z as (i + 0.5) * voxel size) and
  // delta = rotate(invTrack, (0,0,vz)): the camera-space position is computed directly at
  // every z % 8 == 0 voxel and stepped by delta in between, so it does not depend on where
  // a chunk starts (every z-chunk size gives the same volume)
  const float cxw = (x + 0.5f) * a.dimx / a.nx;
  const float cyw = (y + 0.5f) * a.dimy / a.ny;
  const float vz = a.dimz / a.nz;
  float pxy[3], dz[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    pxy[r] = fmaf(inv[r * 4 + 0], cxw, fmaf(inv[r * 4 + 1], cyw, inv[r * 4 + 3]));
    dz[r] = __fmul_rn(inv[r * 4 + 2], vz);  // kept rounded: the steps below are plain adds
  }
  V* vf = reinterpret_cast<V*>(a.vol);
  Wt* vw = reinterpret_cast<Wt*>(reinterpret_cast<char*>(a.vol) + a.count * sizeof(V));
  const uint32_t slice = (uint32_t)a.nx * (uint32_t)a.ny;
  uint32_t idx = (uint32_t)x + (uint32_t)a.nx * (uint32_t)y + (uint32_t)zb * slice;
  const float fW1 = (float)(a.W - 1), fH1 = (float)(a.H - 1);
  const float ku = a.cx + 0.5f, kv = a.cy + 0.5f;
  const int zend = min(ZC, a.nz - zb);
  float px, py, pz;
  // one voxel of the march (integrate.cs:63-113); jj: its index in the current brick
  auto voxel = [&](int jj, int jb, int k8) {
    if (pz < 0.0001f) return;
    const float iz = __fdividef(1.0f, pz);  // hardware reciprocal (2 ulp)
    const float rx = px * iz;  // pos.x / pos.z
    const float ry = py * iz;
    // cameraX.x / cameraX.z + 0.5 = fx * x/z + cx + 0.5 (K has no skew, :67)
    const float u = fmaf(a.fx, rx, ku);
    const float v = fmaf(a.fy, ry, kv);
    if (u < 0.0f || u > fW1 || v < 0.0f || v > fH1) return;
    // explicitly rounded: no template instance may fuse the scaling into the subtraction,
    // so every launch shape computes the same bits
    const float d = __fmul_rn(__ldg(a.depth + (uint32_t)(int)v * (uint32_t)a.W + (uint32_t)(int)u), 0.001f);
    if (d == 0.0f) return;
    const float r2 = fmaf(rx, rx, fmaf(ry, ry, 1.0f));
    const float diff = __fmul_rn(__fsub_rn(d, pz), __fmul_rn(r2, rsqrtf(r2)));  // sqrt(r2), r2 >= 1
    if (diff > -a.mu) {
      const float sdf = fminf(1.0f, __fmul_rn(diff, a.inv_mu));
      const V oldv = vf[idx];
      const Wt oldw = vw[idx];
      const float F = __fmul_rn(Vox<S>::raw_nc(&oldv, 0), Vox<S>::kRawToF);
      const float w = Vox<S>::weight(&oldw, 0);
      const float wd = __fdividef(fmaf(w, F, sdf), w + 1.0f);
      float nF, nw;
      if (!a.band) {
        // the reference's earlier update (integrate.cs:115-150)
        nF = fminf(fmaxf(wd, -1.0f), 1.0f);
        nw = fminf(w + 1.0f, a.maxw);
      } else if (wd < 0.2f) {
        nF = fminf(fmaxf(wd, -0.1f), 0.2f);
        nw = fminf(w + 1.0f, a.maxw);
      } else {
        nF = 0.0f;
        nw = 0.0f;
      }
      const V ev = Vox<S>::encode_value(nF);
      const Wt ew = Vox<S>::encode_weight(nw);
      if (bits_of(ev) != bits_of(oldv)) vf[idx] = ev;
      if (bits_of(ew) != bits_of(oldw)) vw[idx] = ew;
      // a non-negative nF never stores a negative value; a brick's first voxel is also
      // the +1 layer of the brick below it (and, at z % 64 == 0, of the super-brick below)
      if (nF < 0.0f) {
        flags |= 1u << jb;
        if (jj == 0) flags |= (1u << (jb - 1)) | (((zb + k8) & 63) == 0 ? 0xc0u : 0x40u);
        else flags |= 0x40u;
      }
    } else {
      vf[idx] = Vox<S>::encode_value(0.0f);
      vw[idx] = Vox<S>::encode_weight(0.0f);
    }
  };
  // One 8-voxel brick of the column at a time: the position is anchored at the brick's first
  // voxel and steps by delta inside it, as integrate.cs:57-62 does, so it does not depend on
  // where a chunk starts.  Whole bricks run unrolled; only a ragged last brick (nz not a
  // multiple of 8) takes the counted loop.
  for (int k8 = 0; k8 < zend; k8 += 8) {
    const float czw = (zb + k8 + 0.5f) * vz;
    px = fmaf(inv[2], czw, pxy[0]);
    py = fmaf(inv[6], czw, pxy[1]);
    pz = fmaf(inv[10], czw, pxy[2]);
    const int jb = (k8 >> 3) + 1;  // this brick's bit in flags
    if (k8 + 8 <= zend) {
#pragma unroll
      for (int jj = 0; jj < 8; ++jj, idx += slice, px += dz[0], py += dz[1], pz += dz[2]) voxel(jj, jb, k8);
    } else {
      for (int jj = 0; jj < zend - k8; ++jj, idx += slice, px += dz[0], py += dz[1], pz += dz[2]) voxel(jj, jb, k8);
    }
  }
  return flags;
}

// A batched launch: flat block b belongs to the entry e with prefix[e] <= b < prefix[e + 1].
struct IntBatch {
  const IntArgs* args;
  const uint32_t* prefix;  // n + 1 entries
  int n;
};

template <int S, bool BATCH, int ZC>
__global__ void __launch_bounds__(256, 6) integrate_kernel(IntArgs a_one, IntBatch batch) {
  __shared__ IntArgs s_args;
  int bxi, byi, bzi;  // this block's position in its volume's block grid
  if constexpr (BATCH) {
    // binary search of the entry (uniform over the block)
    int lo = 0, hi = batch.n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(batch.prefix + mid) <= blockIdx.x) lo = mid; else hi = mid - 1;
    }
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const int* src = reinterpret_cast<const int*>(batch.args + lo);
    for (int k = tid; k < (int)(sizeof(IntArgs) / 4); k += 256) reinterpret_cast<int*>(&s_args)[k] = __ldg(src + k);
    __syncthreads();
    const uint32_t local = blockIdx.x - __ldg(batch.prefix + lo);
    const uint32_t gx = (uint32_t)(s_args.nx + 31) / 32, gy = (uint32_t)(s_args.ny + 7) / 8;
    bxi = (int)(local % gx);
    byi = (int)((local / gx) % gy);
    bzi = (int)(local / (gx * gy));
  } else {
    bxi = blockIdx.x;
    byi = blockIdx.y;
    bzi = blockIdx.z;
  }
  const IntArgs& a = BATCH ? s_args : a_one;
  if (a.gate && *(volatile const int*)a.gate == 0) return;
  float inv[12];  // inverse(m_pose), rows of [R^T | -R^T t] (integrate uses glm::inverse, :1242)
#pragma unroll
  for (int k = 0; k < 12; ++k) inv[k] = a.st->inv_rows[k];
  const int xb = bxi * 32, yb = byi * 8, zb = bzi * ZC;
  // Every warp evaluates the block's frustum test itself (the same inputs give the same
  // answer in every warp), so no warp waits for another: the kernel has no block barrier.
  // One voxel of margin on every side absorbs the rounding of the per-voxel tests.
  {
    const int b0[3] = {xb - 1, yb - 1, zb - 1};
    const int b1[3] = {xb + 32, yb + 8, zb + ZC};
    if (box_outside_frustum(a, inv, b0, b1)) return;
  }
  const int lane = threadIdx.x;
  const int x = xb + lane;
  const int y = yb + threadIdx.y;  // uniform over the warp
  uint32_t flags = 0;  // integrate_column's bits
  if (x < a.nx && y < a.ny) flags = integrate_column<S, ZC>(a, inv, x, y, zb);
  if (!__any_sync(0xffffffffu, flags != 0)) return;
  // Brick flags, merged over the warp: lanes 8c-8..8c-1 write brick column c of the block
  // (c = 1..4) and a lane on a brick's low x face also brick column c-1 (dilation); lane c
  // sets the merged bits of column c in global memory.  Most bricks near surfaces have the
  // bits already, so read first and skip those atomics.
  const int lx = (x >> 3) - (xb >> 3) + 1;
  constexpr int kZBits = ZC / 8 + 1;  // z-bricks a chunk touches, with the dilation one
  const uint32_t zbits = flags & ((1u << kZBits) - 1u);
  uint32_t mine = 0;
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    const uint32_t m = (lx == c ? zbits : 0u) | (lx - 1 == c && (x & 7) == 0 ? zbits : 0u);
    const uint32_t r = __reduce_or_sync(0xffffffffu, m);
    if (lane == c) mine = r;
  }
  if (lane < 5 && mine) {
    const int gx = (xb >> 3) - 1 + lane;
    for (int j = 0; j < kZBits; ++j) {
      if (!((mine >> j) & 1u)) continue;
      const int gz = (zb >> 3) - 1 + j;
      for (int dy = 0; dy < ((y & 7) == 0 ? 2 : 1); ++dy) {
        const int gy = (y >> 3) - dy;
        if (gx >= 0 && gy >= 0 && gz >= 0 && gx < a.bx && gy < a.by && gz < a.bz) {
          uint32_t* w = &a.bricks[(uint32_t)gx + (uint32_t)a.bx * ((uint32_t)gy + (uint32_t)a.by * (uint32_t)gz)];
          if (!(*(volatile uint32_t*)w & KF_BRICK_NEG)) atomicOr(w, KF_BRICK_NEG);
        }
      }
    }
  }
  // super-bricks: own and, on a super-brick's low face, the one below (x, y, z)
  const uint32_t sbits = flags & 0xc0u;
  const uint32_t s_own = __reduce_or_sync(0xffffffffu, sbits);
  const uint32_t s_lowx = __reduce_or_sync(0xffffffffu, (x & 63) == 0 ? sbits : 0u);
  if (lane < 8 && (lane & 1 ? s_own : s_lowx)) {
    const int jx = lane & 1, jy = (lane >> 1) & 1, jz = lane >> 2;
    const uint32_t zsel = jz ? 0x40u : 0x80u;
    const uint32_t src = jx ? s_own : s_lowx;
    if ((src & zsel) && (jy == 1 || (y & 63) == 0)) {
      const int gx = (xb >> 6) - 1 + jx, gy = (y >> 6) - 1 + jy, gz = (zb >> 6) - 1 + jz;
      if (gx >= 0 && gy >= 0 && gz >= 0 && gx < a.sbx && gy < a.sby && gz < a.sbz) {
        uint32_t* w = &a.supers[(uint32_t)gx + (uint32_t)a.sbx * ((uint32_t)gy + (uint32_t)a.sby * (uint32_t)gz)];
        if (!(*(volatile uint32_t*)w & KF_BRICK_NEG)) atomicOr(w, KF_BRICK_NEG);
      }
    }
  }
}

}  // namespace

namespace {

IntArgs make_int_args(kf_session* s, int gated) {
  IntArgs a;
  a.vol = s->d_vol;
  a.count = s->vol_count;
  a.nx = s->cfg.nx; a.ny = s->cfg.ny; a.nz = s->cfg.nz;
  a.dimx = s->cfg.dim_x; a.dimy = s->cfg.dim_y; a.dimz = s->cfg.dim_z;
  a.depth = s->d_depth[0];
  a.W = s->W[0]; a.H = s->H[0];
  a.fx = s->intr.fx; a.fy = s->intr.fy; a.cx = s->intr.cx; a.cy = s->intr.cy;
  a.mu = s->cfg.mu;
  a.inv_mu = 1.0f / s->cfg.mu;
  a.maxw = s->cfg.max_weight;
  a.band = (s->cfg.quirks & KF_Q8_NARROW_BAND) ? 1 : 0;
  a.gate = gated ? &s->d_state->do_integrate : nullptr;
  a.st = s->d_state;
  a.bricks = s->d_bricks;
  a.bx = s->bx; a.by = s->by; a.bz = s->bz;
  a.supers = s->d_supers;
  a.sbx = s->sbx; a.sby = s->sby; a.sbz = s->sbz;
  return a;
}

template <bool BATCH, int ZC>
void launch_int_zc(int storage, dim3 grid, cudaStream_t st, const IntArgs& a, const IntBatch& b) {
  dim3 block(32, 8);
  switch (storage) {
    case KF_STORAGE_F32F32: integrate_kernel<KF_STORAGE_F32F32, BATCH, ZC><<<grid, block, 0, st>>>(a, b); break;
    case KF_STORAGE_F16U16: integrate_kernel<KF_STORAGE_F16U16, BATCH, ZC><<<grid, block, 0, st>>>(a, b); break;
    default: integrate_kernel<KF_STORAGE_RG16I, BATCH, ZC><<<grid, block, 0, st>>>(a, b); break;
  }
}

template <bool BATCH>
void launch_int(int storage, int zc, dim3 grid, cudaStream_t st, const IntArgs& a, const IntBatch& b) {
  if (zc == 8) launch_int_zc<BATCH, 8>(storage, grid, st, a, b);
  else if (zc == 32) launch_int_zc<BATCH, 32>(storage, grid, st, a, b);
  else launch_int_zc<BATCH, 16>(storage, grid, st, a, b);
}

IntArgs retarget(IntArgs a, const kf_scratch_target* t) {
  if (t) {
    a.vol = t->vol;
    a.bricks = t->bricks;
    a.supers = t->supers;
  }
  return a;
}

}  // namespace

int kf_launch_integrate_shape(kf_session* s, int gated, int zc, const kf_scratch_target* t) {
  const IntArgs a = retarget(make_int_args(s, gated), t);
  dim3 grid((a.nx + 31) / 32, (a.ny + 7) / 8, (a.nz + zc - 1) / zc);
  launch_int<false>(s->cfg.storage, zc, grid, s->stream, a, IntBatch{nullptr, nullptr, 0});
  KF_CUDA_TRY(s, cudaGetLastError());
  kf_note_launch(s);
  return KF_OK;
}

int kf_launch_integrate(kf_session* s, int gated) { return kf_launch_integrate_shape(s, gated, s->int_zc, nullptr); }

// ---- batched: every member's gated frame-step integrate in one launch ----
int kf_batch_prepare_integrate(kf_batch* b, const kf_scratch_target* over) {
  const int n = (int)b->members.size();
  IntArgs* h = nullptr;
  uint32_t* hp = nullptr;
  b->int_args = kf_batch_table(b, sizeof(IntArgs) * n, reinterpret_cast<void**>(&h));
  b->int_prefix = static_cast<const uint32_t*>(kf_batch_table(b, 4 * (size_t)(n + 1), reinterpret_cast<void**>(&hp)));
  if (!b->int_args || !b->int_prefix) return KF_ERR_CAPACITY;
  uint64_t total = 0;
  const int zc = b->int_zc;
  for (int e = 0; e < n; ++e) {
    // the autotuner's timing runs ungated into scratch copies
    h[e] = over ? retarget(make_int_args(b->members[e], 0), over + e) : make_int_args(b->members[e], 1);
    hp[e] = (uint32_t)total;
    total += (uint64_t)((h[e].nx + 31) / 32) * ((h[e].ny + 7) / 8) * ((h[e].nz + zc - 1) / zc);
  }
  if (total >= (1ull << 31)) return KF_ERR_CAPACITY;
  hp[n] = (uint32_t)total;
  b->int_blocks = (uint32_t)total;
  return KF_OK;
}

int kf_batch_launch_integrate(kf_batch* b) {
  const IntBatch batch = {static_cast<const IntArgs*>(b->int_args), b->int_prefix, (int)b->members.size()};
  launch_int<true>(b->members[0]->cfg.storage, b->int_zc, dim3(b->int_blocks), b->stream, IntArgs{}, batch);
  KF_CUDA_TRY(b, cudaGetLastError());
  b->launches += 1;
  return KF_OK;
}
