// kf_raycast.cu — surface prediction by ray marching the TSDF.
//
// Reference: gFusion::raycast (src/gFusion.cpp:1289-1366) and shaders/raycast.cs:133-321:
// view = m_pose * invK; ray origin = pose translation, direction = R * K^-1 (u, v, 1)
// (unnormalised: t is camera z); slab test against [0, volDim]^3 clipped to
// [nearPlane, farPlane]; no hit if the first sample is negative; march with largeStep
// until a sample drops below 0.8, then with step = voxel size (stepSize(), Q9), stop at
// the first negative sample; refine t + step * f_tt / (f_t - f_tt); trilinear samples
// (interpVol :69-82, no weight test, border-clamped taps); normal = normalised
// central-difference trilinear gradient (getGradient :229-276), zero when its length is
// zero.  Misses write zero vertex and normal.
//
// B200 design: one thread per pixel, 32-wide tiles so a warp's rays stay coherent and its
// trilinear taps share L1 lines; the value plane alone is read (2 B per tap for the
// 16-bit storages).  The march position is t0 + k * step (one rounding) rather than the
// reference's repeated float addition.  Once the march is in its fine-step phase it
// skips every brick whose negative-value flag is clear (no sample there can be the first
// negative one), keeping the sample positions tb + k * step and re-evaluating the sample
// before a hit for the refinement, so the result is the unskipped march's.
#include "kf_internal.cuh"

namespace {

struct RayArgs {
  const void* vol;
  int nx, ny, nz;
  float sx, sy, sz;         // volSize / volDim
  float gx, gy, gz;         // volDim / volSize * 0.5 (getGradient scale, :273)
  float dimx, dimy, dimz;
  float step, large_step, nearp, farp;
  int max_steps;
  int W, H;
  float ikx, iky, ikcx, ikcy;  // getInverseCameraMatrix: 1/fx, 1/fy, -cx/fx, -cy/fy (float)
  float4* out_v;
  float4* out_n;
  const KfDevState* st;
  KfDevState* st_out;
  const uint32_t* bricks;
  int bx, by, bz;
  const uint32_t* supers;
  int sbx, sby, sbz;
};

// 32 x ROWS pixel tiles (ROWS one of KF_RAY_ROWS, chosen per session: default 4, or the
// autotuner's pick): ray lengths vary a lot, and small blocks keep the SMs evenly loaded to
// the end of the launch (512 x 424 in 32 x 4 tiles gives 1,696 blocks).  Every choice
// computes the same maps.

template <int S>
struct Sampler {
  typedef typename Vox<S>::V V;
  const V* f;
  int nx, ny, nz;
  uint32_t sxy;
  __device__ __forceinline__ float tap(int x, int y, int z) const {
    return Vox<S>::raw(f, (uint32_t)x + (uint32_t)nx * (uint32_t)y + sxy * (uint32_t)z);
  }
  // interpVol (raycast.cs:69-82) before the final * (1/32766); q in voxel coordinates
  // (world * volSize / volDim - 0.5).  The 8 taps share one base offset.
  __device__ __forceinline__ float interp_raw(float qx, float qy, float qz) const {
    const float bx = floorf(qx), by = floorf(qy), bz = floorf(qz);
    const float fx = qx - bx, fy = qy - by, fz = qz - bz;
    const int ix = (int)bx, iy = (int)by, iz = (int)bz;
    const int lx = min(max(ix, 0), nx - 1), ly = min(max(iy, 0), ny - 1), lz = min(max(iz, 0), nz - 1);
    const int ux = max(min(ix + 1, nx - 1), 0), uy = max(min(iy + 1, ny - 1), 0), uz = max(min(iz + 1, nz - 1), 0);
    const uint32_t b = (uint32_t)lx + (uint32_t)nx * (uint32_t)ly + sxy * (uint32_t)lz;
    const uint32_t ox = (uint32_t)(ux - lx), oy = (uint32_t)(uy - ly) * (uint32_t)nx,
                   oz = (uint32_t)(uz - lz) * sxy;
    const float c000 = Vox<S>::raw(f, b), c100 = Vox<S>::raw(f, b + ox);
    const float c010 = Vox<S>::raw(f, b + oy), c110 = Vox<S>::raw(f, b + ox + oy);
    const float c001 = Vox<S>::raw(f, b + oz), c101 = Vox<S>::raw(f, b + ox + oz);
    const float c011 = Vox<S>::raw(f, b + oy + oz), c111 = Vox<S>::raw(f, b + ox + oy + oz);
    return ((c000 * (1 - fx) + c100 * fx) * (1 - fy) + (c010 * (1 - fx) + c110 * fx) * fy) * (1 - fz) +
           ((c001 * (1 - fx) + c101 * fx) * (1 - fy) + (c011 * (1 - fx) + c111 * fx) * fy) * fz;
  }
};

// One pixel of raycast.cs:133-321 for view rows s_view (m_pose * invK): march, refine,
// gradient normal; writes the pixel's vertex and normal.
template <int S>
__device__ __forceinline__ void raycast_pixel(const RayArgs& a, const float* s_view, int x, int y) {
  Sampler<S> smp;
  smp.f = reinterpret_cast<const typename Vox<S>::V*>(a.vol);
  smp.nx = a.nx; smp.ny = a.ny; smp.nz = a.nz;
  smp.sxy = (uint32_t)a.nx * (uint32_t)a.ny;

  const float ox = s_view[3], oy = s_view[7], oz = s_view[11];
  const float fxp = (float)x, fyp = (float)y;
  const float dx = fmaf(s_view[0], fxp, fmaf(s_view[1], fyp, s_view[2]));
  const float dy = fmaf(s_view[4], fxp, fmaf(s_view[5], fyp, s_view[6]));
  const float dzv = fmaf(s_view[8], fxp, fmaf(s_view[9], fyp, s_view[10]));

  // slab test (raycast.cs:141-152)
  const float ix = 1.0f / dx, iy = 1.0f / dy, iz = 1.0f / dzv;
  const float tbx = -1.0f * ix * ox, tby = -1.0f * iy * oy, tbz = -1.0f * iz * oz;
  const float ttx = ix * (a.dimx - ox), tty = iy * (a.dimy - oy), ttz = iz * (a.dimz - oz);
  const float tminx = fminf(ttx, tbx), tminy = fminf(tty, tby), tminz = fminf(ttz, tbz);
  const float tmaxx = fmaxf(ttx, tbx), tmaxy = fmaxf(tty, tby), tmaxz = fmaxf(ttz, tbz);
  const float largest_tmin = fmaxf(fmaxf(tminx, tminy), fmaxf(tminx, tminz));
  const float smallest_tmax = fminf(fminf(tmaxx, tmaxy), fminf(tmaxx, tmaxz));
  const float tnear = fmaxf(largest_tmin, a.nearp);
  const float tfar = fminf(smallest_tmax, a.farp);

  const float scale = Vox<S>::kRawToF;
  float hx = 0.f, hy = 0.f, hz = 0.f, ht = 0.f;
  if (tnear < tfar) {
    float t = tnear, stepsize = a.large_step;
    // the ray in voxel coordinates: q(t) = (o + d t) * volSize / volDim - 0.5
    const float q0x = fmaf(ox, a.sx, -0.5f), q0y = fmaf(oy, a.sy, -0.5f), q0z = fmaf(oz, a.sz, -0.5f);
    const float dqx = dx * a.sx, dqy = dy * a.sy, dqz = dzv * a.sz;
    auto sample = [&](float tt) {
      return smp.interp_raw(fmaf(tt, dqx, q0x), fmaf(tt, dqy, q0y), fmaf(tt, dqz, q0z)) * scale;
    };
    float f_t = sample(t), f_tt = 0.0f;
    if (f_t >= 0.0f) {
      // 1 / ray slope in voxel coordinates, for the brick-exit distances
      const float rdx = 1.0f / dqx, rdy = 1.0f / dqy, rdz = 1.0f / dqz;
      float tb = t;
      int k = 0;
      bool fine = false;       // stepsize == step (the reference never switches back)
      bool prev_known = true;  // f_t holds the sample just before t
      // bounded march: a NaN sample keeps largeStep, so cap the step count
      for (int n = 0; t < tfar && n < a.max_steps; ++n) {
        {
          // empty-space skipping in the fine phase.  A sample's eight taps lie in the brick
          // (and super-brick) of its base voxel; a region without a negative value cannot
          // hold the first negative sample.  Such samples change nothing but f_t, so jump to
          // the first sample past the region; the positions stay tb + k * stepsize, as in
          // the unskipped march.
          const float qx = fmaf(t, dqx, q0x), qy = fmaf(t, dqy, q0y), qz = fmaf(t, dqz, q0z);
          const int vx = min(max((int)floorf(qx), 0), a.nx - 1);
          const int vy = min(max((int)floorf(qy), 0), a.ny - 1);
          const int vz = min(max((int)floorf(qz), 0), a.nz - 1);
          int cell = 0;  // 0: sample it; else the side of the region to skip (64 or 8)
          int cx = 0, cy = 0, cz = 0, ncx = 1, ncy = 1, ncz = 1;
          if (fine) {
            if (!(__ldg(a.supers + (uint32_t)(vx >> 6) +
                        (uint32_t)a.sbx * ((uint32_t)(vy >> 6) + (uint32_t)a.sby * (uint32_t)(vz >> 6))) &
                  KF_BRICK_NEG)) {
              cell = 64;
              cx = vx >> 6; cy = vy >> 6; cz = vz >> 6;
              ncx = a.sbx; ncy = a.sby; ncz = a.sbz;
            } else if (!(__ldg(a.bricks + (uint32_t)(vx >> 3) +
                               (uint32_t)a.bx * ((uint32_t)(vy >> 3) + (uint32_t)a.by * (uint32_t)(vz >> 3))) &
                         KF_BRICK_NEG)) {
              cell = 8;
              cx = vx >> 3; cy = vy >> 3; cz = vz >> 3;
              ncx = a.bx; ncy = a.by; ncz = a.bz;
            }
          }
          if (cell) {
            // the region spans [cell*i, cell*(i+1)) in voxel coordinates; the border ones
            // extend outwards (taps are clamped there)
            const float c = (float)cell;
            float te = tfar;
            if (dqx > 0.0f && cx < ncx - 1) te = fminf(te, (float)(cx + 1) * c * rdx - q0x * rdx);
            if (dqx < 0.0f && cx > 0) te = fminf(te, (float)cx * c * rdx - q0x * rdx);
            if (dqy > 0.0f && cy < ncy - 1) te = fminf(te, (float)(cy + 1) * c * rdy - q0y * rdy);
            if (dqy < 0.0f && cy > 0) te = fminf(te, (float)cy * c * rdy - q0y * rdy);
            if (dqz > 0.0f && cz < ncz - 1) te = fminf(te, (float)(cz + 1) * c * rdz - q0z * rdz);
            if (dqz < 0.0f && cz > 0) te = fminf(te, (float)cz * c * rdz - q0z * rdz);
            const float kf = ceilf((te - tb) / stepsize);
            int kn = kf < 2.0e9f ? (int)kf : k + 1;
            if (kn > k + 1) {
              // te carries rounding; the rounded sample positions are monotone in k on
              // every axis, so if the last skipped sample is still in this region, all of
              // them are.  Otherwise advance by one sample.
              const float tl = fmaf((float)(kn - 1), stepsize, tb);
              const int sh = cell == 64 ? 6 : 3;
              const int jx = min(max((int)floorf(fmaf(tl, dqx, q0x)), 0), a.nx - 1) >> sh;
              const int jy = min(max((int)floorf(fmaf(tl, dqy, q0y)), 0), a.ny - 1) >> sh;
              const int jz = min(max((int)floorf(fmaf(tl, dqz, q0z)), 0), a.nz - 1) >> sh;
              if (jx != cx || jy != cy || jz != cz) kn = k + 1;
            } else {
              kn = k + 1;
            }
            k = kn;
            t = fmaf((float)k, stepsize, tb);
            prev_known = false;
            continue;
          }
        }
        f_tt = sample(t);
        if (f_tt < 0.0f) break;
        if (f_tt < 0.8f && !fine) {
          fine = true;
          stepsize = a.step;
          tb = t;
          k = 0;
        }
        f_t = f_tt;
        prev_known = true;
        ++k;
        t = fmaf((float)k, stepsize, tb);
      }
      if (f_tt < 0.0f) {
        if (!prev_known) f_t = sample(fmaf((float)(k - 1), stepsize, tb));
        t = t + stepsize * f_tt / (f_t - f_tt);
        hx = fmaf(dx, t, ox);
        hy = fmaf(dy, t, oy);
        hz = fmaf(dzv, t, oz);
        ht = t;
      }
    }
  }

  const size_t o = (size_t)y * a.W + x;
  if (ht > 0.0f) {
    a.out_v[o] = make_float4(hx, hy, hz, 1.0f);
    // getGradient (raycast.cs:229-276)
    const float qx = hx * a.sx - 0.5f, qy = hy * a.sy - 0.5f, qz = hz * a.sz - 0.5f;
    const float bx = floorf(qx), by = floorf(qy), bz = floorf(qz);
    const float f3[3] = {qx - bx, qy - by, qz - bz};
    const int bi[3] = {(int)bx, (int)by, (int)bz};
    const int n3[3] = {a.nx, a.ny, a.nz};
    int ll[3], lu[3], ul[3], uu[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      ll[k] = min(max(bi[k] - 1, 0), n3[k] - 1);
      lu[k] = min(max(bi[k], 0), n3[k] - 1);
      ul[k] = max(min(bi[k] + 1, n3[k] - 1), 0);
      uu[k] = max(min(bi[k] + 2, n3[k] - 1), 0);
    }
    float g[3];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      float acc = 0.0f;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int cc[3] = {c & 1, (c >> 1) & 1, (c >> 2) & 1};
        int pa[3], pb[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          if (k == ax) {
            pa[k] = cc[k] ? uu[k] : ul[k];
            pb[k] = cc[k] ? lu[k] : ll[k];
          } else {
            pa[k] = cc[k] ? ul[k] : lu[k];
            pb[k] = pa[k];
          }
        }
        const float w = (cc[0] ? f3[0] : 1.0f - f3[0]) * (cc[1] ? f3[1] : 1.0f - f3[1]) *
                        (cc[2] ? f3[2] : 1.0f - f3[2]);
        acc = fmaf(w, smp.tap(pa[0], pa[1], pa[2]) - smp.tap(pb[0], pb[1], pb[2]), acc);
      }
      g[ax] = acc;
    }
    const float gx = g[0] * a.gx * scale, gy = g[1] * a.gy * scale, gz = g[2] * a.gz * scale;
    const float len = sqrtf(gx * gx + gy * gy + gz * gz);
    if (len == 0.0f)
      a.out_n[o] = make_float4(0.f, 0.f, 0.f, 0.f);
    else
      a.out_n[o] = make_float4(gx / len, gy / len, gz / len, 1.0f);
  } else {
    a.out_v[o] = make_float4(0.f, 0.f, 0.f, 0.f);
    a.out_n[o] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// view = m_pose * invK (gFusion.cpp:1296) from the FP32 pose rows and float invK; thread
// t < 12 writes element t of the 3x4 rows.
__device__ __forceinline__ void raycast_view(const RayArgs& a, float* s_view, int t) {
  const int r = t >> 2, c = t & 3;
  const float* P = a.st->pose_rows;
  float v;
  if (c == 0) v = P[r * 4 + 0] * a.ikx;
  else if (c == 1) v = P[r * 4 + 1] * a.iky;
  else if (c == 2) v = fmaf(P[r * 4 + 0], a.ikcx, fmaf(P[r * 4 + 1], a.ikcy, P[r * 4 + 2]));
  else v = P[r * 4 + 3];
  s_view[r * 4 + c] = v;
}

// BATCH: blockIdx.z selects the session's arguments in `many`.
template <int S, bool BATCH, int ROWS>
__global__ void __launch_bounds__(32 * ROWS) raycast_kernel(RayArgs one, const RayArgs* many) {
  static_assert(ROWS == 2 || ROWS == 4 || ROWS == 8, "raycast tile rows: 2, 4 or 8");
  __shared__ RayArgs s_args;
  __shared__ float s_view[12];  // rows of m_pose * invK: (R K^-1 | t)
  if constexpr (BATCH) {
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const int* src = reinterpret_cast<const int*>(many + blockIdx.z);
    for (int k = tid; k < (int)(sizeof(RayArgs) / 4); k += 32 * ROWS) reinterpret_cast<int*>(&s_args)[k] = __ldg(src + k);
    __syncthreads();
  }
  const RayArgs& a = BATCH ? s_args : one;
  if (threadIdx.y == 0 && threadIdx.x < 12) raycast_view(a, s_view, threadIdx.x);
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.y == 1 && threadIdx.x < 16)
    a.st_out->raycast_pose[threadIdx.x] = a.st->pose[threadIdx.x];
  __syncthreads();
  // each warp takes a compact patch of the 32 x ROWS tile (16 x 2 pixels in 2-row tiles,
  // 8 x 4 otherwise): neighbouring rays march through the same bricks and end at similar
  // depths, so a warp's taps share cache lines and its lanes finish together (measured
  // ~1 % faster than a 32 x 1 row per warp)
  const int t = threadIdx.y * 32 + threadIdx.x, w = t >> 5, l = t & 31;
  int x, y;
  if constexpr (ROWS == 2) {
    x = blockIdx.x * 32 + w * 16 + (l & 15);
    y = blockIdx.y * 2 + (l >> 4);
  } else {
    x = blockIdx.x * 32 + (w & 3) * 8 + (l & 7);
    y = blockIdx.y * ROWS + (w >> 2) * 4 + (l >> 3);
  }
  if (x >= a.W || y >= a.H) return;
  raycast_pixel<S>(a, s_view, x, y);
}

// The same rays as a persistent sweep: one block per resident slot, and every warp takes
// the next row segment of 32 pixels from a device counter until the image is done, so no
// warp waits for another and long rays do not leave SMs idle at the end of the launch.
// The last warp to find the queue empty resets the counter (and its own completion count)
// for the next launch.  Every pixel runs raycast_pixel: the maps are the tiled kernel's.
template <int S>
__global__ void __launch_bounds__(256) raycast_sweep_kernel(RayArgs a, unsigned* queue) {
  __shared__ float s_view[12];
  const int lane = threadIdx.x & 31;
  if (threadIdx.x < 12) raycast_view(a, s_view, threadIdx.x);
  if (blockIdx.x == 0 && threadIdx.x >= 32 && threadIdx.x < 48)
    a.st_out->raycast_pose[threadIdx.x - 32] = a.st->pose[threadIdx.x - 32];
  __syncthreads();
  const int segs_x = (a.W + 31) / 32;
  const unsigned nseg = (unsigned)segs_x * (unsigned)a.H;
  for (;;) {
    unsigned seg = 0;
    if (lane == 0) seg = atomicAdd(queue, 1u);
    seg = __shfl_sync(0xffffffffu, seg, 0);
    if (seg >= nseg) break;
    const int y = (int)(seg / (unsigned)segs_x);
    const int x = (int)(seg % (unsigned)segs_x) * 32 + lane;
    if (x < a.W) raycast_pixel<S>(a, s_view, x, y);
  }
  // every warp drew one ticket past the end; the last of them resets the queue
  if (lane == 0) {
    const unsigned warps = gridDim.x * (blockDim.x / 32);
    if (atomicAdd(queue + 1, 1u) == warps - 1) {
      queue[0] = 0u;
      queue[1] = 0u;
    }
  }
}

// Volume ray-sum image (gFusion::intensityProjection, src/gFusion.cpp:1368-1409, and
// shaders/mip.cs:52-104): the raycast's view, slab test and near/far clipping, then samples
// every largeStep from tnear while t < tfar, summing the positive interpolated values into
// x; the pixel is (sum, 0, 0, 1), misses included (mip.cs's other two branches add zero or
// are unreachable).  Sample positions are tnear + k * largeStep (one rounding, as in the
// raycast).  The reference dispatches it on demand, never from the frame loop; so does this.
template <int S>
__global__ void __launch_bounds__(128) mip_kernel(RayArgs a, float4* out) {
  __shared__ float s_view[12];
  if (threadIdx.y == 0 && threadIdx.x < 12) {
    const int r = threadIdx.x >> 2, c = threadIdx.x & 3;
    const float* P = a.st->pose_rows;
    float v;
    if (c == 0) v = P[r * 4 + 0] * a.ikx;
    else if (c == 1) v = P[r * 4 + 1] * a.iky;
    else if (c == 2) v = fmaf(P[r * 4 + 0], a.ikcx, fmaf(P[r * 4 + 1], a.ikcy, P[r * 4 + 2]));
    else v = P[r * 4 + 3];
    s_view[r * 4 + c] = v;
  }
  __syncthreads();
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= a.W || y >= a.H) return;
  Sampler<S> smp;
  smp.f = reinterpret_cast<const typename Vox<S>::V*>(a.vol);
  smp.nx = a.nx; smp.ny = a.ny; smp.nz = a.nz;
  smp.sxy = (uint32_t)a.nx * (uint32_t)a.ny;

  const float ox = s_view[3], oy = s_view[7], oz = s_view[11];
  const float fxp = (float)x, fyp = (float)y;
  const float dx = fmaf(s_view[0], fxp, fmaf(s_view[1], fyp, s_view[2]));
  const float dy = fmaf(s_view[4], fxp, fmaf(s_view[5], fyp, s_view[6]));
  const float dzv = fmaf(s_view[8], fxp, fmaf(s_view[9], fyp, s_view[10]));
  // slab test (mip.cs:61-77, as raycast.cs:141-152)
  const float ix = 1.0f / dx, iy = 1.0f / dy, iz = 1.0f / dzv;
  const float tbx = -1.0f * ix * ox, tby = -1.0f * iy * oy, tbz = -1.0f * iz * oz;
  const float ttx = ix * (a.dimx - ox), tty = iy * (a.dimy - oy), ttz = iz * (a.dimz - oz);
  const float tminx = fminf(ttx, tbx), tminy = fminf(tty, tby), tminz = fminf(ttz, tbz);
  const float tmaxx = fmaxf(ttx, tbx), tmaxy = fmaxf(tty, tby), tmaxz = fmaxf(ttz, tbz);
  const float largest_tmin = fmaxf(fmaxf(tminx, tminy), fmaxf(tminx, tminz));
  const float smallest_tmax = fminf(fminf(tmaxx, tmaxy), fminf(tmaxx, tmaxz));
  const float tnear = fmaxf(largest_tmin, a.nearp);
  const float tfar = fminf(smallest_tmax, a.farp);

  float sum = 0.0f;
  if (tnear < tfar) {
    const float scale = Vox<S>::kRawToF;
    const float q0x = fmaf(ox, a.sx, -0.5f), q0y = fmaf(oy, a.sy, -0.5f), q0z = fmaf(oz, a.sz, -0.5f);
    const float dqx = dx * a.sx, dqy = dy * a.sy, dqz = dzv * a.sz;
    // bounded: max_steps covers (far - near) / min(step, largeStep) samples
    for (int k = 0; k < a.max_steps; ++k) {
      const float t = fmaf((float)k, a.large_step, tnear);
      if (!(t < tfar)) break;
      const float f = smp.interp_raw(fmaf(t, dqx, q0x), fmaf(t, dqy, q0y), fmaf(t, dqz, q0z)) * scale;
      if (f > 0.0f) sum += f;
    }
  }
  out[(size_t)y * a.W + x] = make_float4(sum, 0.0f, 0.0f, 1.0f);
}

// Exact NEG flags from the volume itself: a brick B is NEG when a value over the voxels
// [8B, 8B+8] (clamped to the volume) is negative, a super-brick when one of its 8^3 bricks
// is (super-bricks are cleared first and set here).  A block takes one row of 32 bricks
// along x at brick (y, z): thread t scans voxel column x0 + t over the brick's 9 x 9 (y, z)
// window (coalesced along x), the extra warp the first columns of the next row (the +1
// layer of the last brick), and thread c merges brick c's 9 columns from shared memory.
constexpr int kRebuildThreads = 256 + 32;

template <int S>
__global__ void __launch_bounds__(kRebuildThreads) rebuild_bricks_kernel(const void* vol, int nx, int ny, int nz,
                                                                          int bx, int by, int bz, uint32_t* bricks,
                                                                          uint32_t* supers, int sbx, int sby) {
  __shared__ uint8_t s_neg[kRebuildThreads];
  const typename Vox<S>::V* f = reinterpret_cast<const typename Vox<S>::V*>(vol);
  const int x = blockIdx.x * 256 + threadIdx.x;
  const int y0 = 8 * blockIdx.y, y1 = min(y0 + 8, ny - 1);
  const int z0 = 8 * blockIdx.z, z1 = min(z0 + 8, nz - 1);
  bool neg = false;
  if (x < nx)
    for (int z = z0; z <= z1 && !neg; ++z) {
      // the plane's (up to) 9 rows are loaded together; the scan stops after a plane
      const uint32_t base = (uint32_t)x + (uint32_t)nx * (uint32_t)ny * (uint32_t)z;
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const int y = min(y0 + k, y1);  // rows past the volume repeat the last one
        neg |= Vox<S>::raw(f, base + (uint32_t)nx * (uint32_t)y) < 0.0f;
      }
    }
  s_neg[threadIdx.x] = neg ? 1 : 0;
  __syncthreads();
  const int c = threadIdx.x;
  const int b = blockIdx.x * 32 + c;
  if (c < 32 && b < bx) {
    uint8_t m = 0;
#pragma unroll
    for (int k = 0; k <= 8; ++k) m |= s_neg[8 * c + k];  // columns past nx - 1 hold 0
    const uint32_t flag = m ? KF_BRICK_NEG : 0u;
    bricks[(uint32_t)b + (uint32_t)bx * ((uint32_t)blockIdx.y + (uint32_t)by * (uint32_t)blockIdx.z)] = flag;
    if (flag) {
      uint32_t* w = &supers[(uint32_t)(b >> 3) +
                            (uint32_t)sbx * ((uint32_t)(blockIdx.y >> 3) + (uint32_t)sby * (uint32_t)(blockIdx.z >> 3))];
      if (!(*(volatile uint32_t*)w & KF_BRICK_NEG)) atomicOr(w, KF_BRICK_NEG);
    }
  }
}

}  // namespace

int kf_rebuild_bricks(kf_session* s, cudaStream_t stream) {
  const uint32_t ns = (uint32_t)s->sbx * s->sby * s->sbz;
  KF_CUDA_TRY(s, cudaMemsetAsync(s->d_supers, 0, ns * sizeof(uint32_t), stream));
  const dim3 grid((s->bx + 31) / 32, s->by, s->bz);
  switch (s->cfg.storage) {
    case KF_STORAGE_F32F32:
      rebuild_bricks_kernel<KF_STORAGE_F32F32><<<grid, kRebuildThreads, 0, stream>>>(
          s->d_vol, s->cfg.nx, s->cfg.ny, s->cfg.nz, s->bx, s->by, s->bz, s->d_bricks, s->d_supers, s->sbx, s->sby);
      break;
    case KF_STORAGE_F16U16:
      rebuild_bricks_kernel<KF_STORAGE_F16U16><<<grid, kRebuildThreads, 0, stream>>>(
          s->d_vol, s->cfg.nx, s->cfg.ny, s->cfg.nz, s->bx, s->by, s->bz, s->d_bricks, s->d_supers, s->sbx, s->sby);
      break;
    default:
      rebuild_bricks_kernel<KF_STORAGE_RG16I><<<grid, kRebuildThreads, 0, stream>>>(
          s->d_vol, s->cfg.nx, s->cfg.ny, s->cfg.nz, s->bx, s->by, s->bz, s->d_bricks, s->d_supers, s->sbx, s->sby);
      break;
  }
  KF_CUDA_TRY(s, cudaGetLastError());
  kf_note_launch(s, 1);
  s->frames_since_rebuild = 0;
  return KF_OK;
}

int kf_note_integrate(kf_session* s, cudaStream_t stream) {
  if (++s->frames_since_rebuild < KF_BRICK_REBUILD_EVERY) return KF_OK;
  return kf_rebuild_bricks(s, stream);
}

int kf_reset_bricks(kf_session* s) {
  // an all-zero volume has no negative value
  const size_t words = (size_t)s->bx * s->by * s->bz + (size_t)s->sbx * s->sby * s->sbz;
  KF_CUDA_TRY(s, cudaMemsetAsync(s->d_bricks, 0, words * 4, s->stream));
  s->frames_since_rebuild = 0;
  return KF_OK;
}

namespace {

RayArgs make_ray_args(kf_session* s) {
  RayArgs a;
  a.vol = s->d_vol;
  a.nx = s->cfg.nx; a.ny = s->cfg.ny; a.nz = s->cfg.nz;
  a.dimx = s->cfg.dim_x; a.dimy = s->cfg.dim_y; a.dimz = s->cfg.dim_z;
  a.sx = (float)a.nx / a.dimx; a.sy = (float)a.ny / a.dimy; a.sz = (float)a.nz / a.dimz;
  a.gx = a.dimx / (float)a.nx * 0.5f; a.gy = a.dimy / (float)a.ny * 0.5f; a.gz = a.dimz / (float)a.nz * 0.5f;
  // stepSize() (gFusion.h:72-81) and largeStep = 0.75 mu (gFusion.cpp:1302)
  const float mind = fminf(fminf(a.dimx, a.dimy), a.dimz);
  const float maxn = (float)max(max(a.nx, a.ny), a.nz);
  a.step = mind / maxn;
  a.large_step = 0.75f * s->cfg.mu;
  a.nearp = s->cfg.near_plane;
  a.farp = s->cfg.far_plane;
  {
    const float smin = fminf(a.step, a.large_step > 0.0f ? a.large_step : a.step);
    const double n = (double)(a.farp - a.nearp) / (double)smin + 16.0;
    a.max_steps = (int)fmin(n, 1.0e8);
  }
  a.W = s->W[0]; a.H = s->H[0];
  a.ikx = 1.0f / s->intr.fx;
  a.iky = 1.0f / s->intr.fy;
  a.ikcx = -s->intr.cx / s->intr.fx;
  a.ikcy = -s->intr.cy / s->intr.fy;
  a.out_v = s->d_ref_vertex;
  a.out_n = s->d_ref_normal;
  a.st = s->d_state;
  a.st_out = s->d_state;
  a.bricks = s->d_bricks;
  a.bx = s->bx; a.by = s->by; a.bz = s->bz;
  a.supers = s->d_supers;
  a.sbx = s->sbx; a.sby = s->sby; a.sbz = s->sbz;
  return a;
}

template <bool BATCH, int ROWS>
void launch_ray_rows(int storage, dim3 grid, cudaStream_t st, const RayArgs& a, const RayArgs* many) {
  dim3 block(32, ROWS);
  switch (storage) {
    case KF_STORAGE_F32F32: raycast_kernel<KF_STORAGE_F32F32, BATCH, ROWS><<<grid, block, 0, st>>>(a, many); break;
    case KF_STORAGE_F16U16: raycast_kernel<KF_STORAGE_F16U16, BATCH, ROWS><<<grid, block, 0, st>>>(a, many); break;
    default: raycast_kernel<KF_STORAGE_RG16I, BATCH, ROWS><<<grid, block, 0, st>>>(a, many); break;
  }
}

template <bool BATCH>
void launch_ray(int storage, int rows, dim3 grid, cudaStream_t st, const RayArgs& a, const RayArgs* many) {
  if (rows == 2) launch_ray_rows<BATCH, 2>(storage, grid, st, a, many);
  else if (rows == 8) launch_ray_rows<BATCH, 8>(storage, grid, st, a, many);
  else launch_ray_rows<BATCH, 4>(storage, grid, st, a, many);
}

RayArgs retarget(RayArgs a, const kf_scratch_target* t) {
  if (t) {
    a.out_v = t->out_v;
    a.out_n = t->out_n;
    a.st_out = t->st_out;
  }
  return a;
}

}  // namespace

int kf_launch_raycast_shape(kf_session* s, int rows, const kf_scratch_target* t) {
  const RayArgs a = retarget(make_ray_args(s), t);
  if (rows == 1) {
    // persistent sweep: every resident slot of 256 threads, the queue in the session state
    const void* fn = s->cfg.storage == KF_STORAGE_F32F32   ? (const void*)raycast_sweep_kernel<KF_STORAGE_F32F32>
                     : s->cfg.storage == KF_STORAGE_F16U16 ? (const void*)raycast_sweep_kernel<KF_STORAGE_F16U16>
                                                           : (const void*)raycast_sweep_kernel<KF_STORAGE_RG16I>;
    const int blocks = kf_occupancy_blocks(s, fn, 256, 0, 64);
    if (blocks <= 0) return KF_ERR_CUDA;
    unsigned* q = s->d_state->ray_queue;
    switch (s->cfg.storage) {
      case KF_STORAGE_F32F32: raycast_sweep_kernel<KF_STORAGE_F32F32><<<blocks, 256, 0, s->stream>>>(a, q); break;
      case KF_STORAGE_F16U16: raycast_sweep_kernel<KF_STORAGE_F16U16><<<blocks, 256, 0, s->stream>>>(a, q); break;
      default: raycast_sweep_kernel<KF_STORAGE_RG16I><<<blocks, 256, 0, s->stream>>>(a, q); break;
    }
    KF_CUDA_TRY(s, cudaGetLastError());
    kf_note_launch(s);
    return KF_OK;
  }
  dim3 grid((a.W + 31) / 32, (a.H + rows - 1) / rows);
  launch_ray<false>(s->cfg.storage, rows, grid, s->stream, a, nullptr);
  KF_CUDA_TRY(s, cudaGetLastError());
  kf_note_launch(s);
  return KF_OK;
}

int kf_launch_raycast(kf_session* s) { return kf_launch_raycast_shape(s, s->ray_rows, nullptr); }

int kf_launch_intensity_projection(kf_session* s, float4* out) {
  const RayArgs a = make_ray_args(s);
  dim3 grid((a.W + 31) / 32, (a.H + 3) / 4);
  dim3 block(32, 4);
  switch (s->cfg.storage) {
    case KF_STORAGE_F32F32: mip_kernel<KF_STORAGE_F32F32><<<grid, block, 0, s->stream>>>(a, out); break;
    case KF_STORAGE_F16U16: mip_kernel<KF_STORAGE_F16U16><<<grid, block, 0, s->stream>>>(a, out); break;
    default: mip_kernel<KF_STORAGE_RG16I><<<grid, block, 0, s->stream>>>(a, out); break;
  }
  KF_CUDA_TRY(s, cudaGetLastError());
  kf_note_launch(s);
  return KF_OK;
}

// ---- batched: every member's raycast in one launch (blockIdx.z = member) ----
int kf_batch_prepare_raycast(kf_batch* b, const kf_scratch_target* over) {
  const int n = (int)b->members.size();
  RayArgs* h = nullptr;
  b->ray_args = kf_batch_table(b, sizeof(RayArgs) * n, reinterpret_cast<void**>(&h));
  if (!b->ray_args) return KF_ERR_CAPACITY;
  for (int e = 0; e < n; ++e) h[e] = retarget(make_ray_args(b->members[e]), over ? over + e : nullptr);
  return KF_OK;
}

int kf_batch_launch_raycast(kf_batch* b, int n) {
  kf_session* s0 = b->members[0];
  const int rows = b->ray_rows;
  dim3 grid((s0->W[0] + 31) / 32, (s0->H[0] + rows - 1) / rows, n);
  launch_ray<true>(s0->cfg.storage, rows, grid, b->stream, RayArgs{}, static_cast<const RayArgs*>(b->ray_args));
  KF_CUDA_TRY(b, cudaGetLastError());
  b->launches += 1;
  return KF_OK;
}
