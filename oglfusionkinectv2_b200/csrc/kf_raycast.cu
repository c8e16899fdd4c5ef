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
// B200 design: one thread per pixel, 32x8 tiles so a warp's rays stay coherent and its
// trilinear taps share L1 lines; the value plane alone is read (2 B per tap for the
// 16-bit storages).  The march position is t0 + k * step (one rounding) rather than the
// reference's repeated float addition.
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
  double fx, fy, cx, cy;
  float4* out_v;
  float4* out_n;
  const KfDevState* st;
  KfDevState* st_out;
};

template <int S>
struct Sampler {
  typedef typename Vox<S>::V V;
  const V* f;
  int nx, ny, nz;
  size_t sxy;
  __device__ __forceinline__ float tap(int x, int y, int z) const {
    return Vox<S>::raw(f, (size_t)x + (size_t)nx * y + sxy * z);
  }
  // interpVol (raycast.cs:69-82) before the final * (1/32766)
  __device__ __forceinline__ float interp_raw(float qx, float qy, float qz) const {
    const float bx = floorf(qx), by = floorf(qy), bz = floorf(qz);
    const float fx = qx - bx, fy = qy - by, fz = qz - bz;
    const int ix = (int)bx, iy = (int)by, iz = (int)bz;
    const int lx = min(max(ix, 0), nx - 1), ly = min(max(iy, 0), ny - 1), lz = min(max(iz, 0), nz - 1);
    const int ux = max(min(ix + 1, nx - 1), 0), uy = max(min(iy + 1, ny - 1), 0), uz = max(min(iz + 1, nz - 1), 0);
    const float c000 = tap(lx, ly, lz), c100 = tap(ux, ly, lz);
    const float c010 = tap(lx, uy, lz), c110 = tap(ux, uy, lz);
    const float c001 = tap(lx, ly, uz), c101 = tap(ux, ly, uz);
    const float c011 = tap(lx, uy, uz), c111 = tap(ux, uy, uz);
    return ((c000 * (1 - fx) + c100 * fx) * (1 - fy) + (c010 * (1 - fx) + c110 * fx) * fy) * (1 - fz) +
           ((c001 * (1 - fx) + c101 * fx) * (1 - fy) + (c011 * (1 - fx) + c111 * fx) * fy) * fz;
  }
};

template <int S>
__global__ void __launch_bounds__(256) raycast_kernel(RayArgs a) {
  __shared__ float s_view[12];  // rows of m_pose * invK: (R K^-1 | t)
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    double P[16], iK[16], Vw[16];
    for (int k = 0; k < 16; ++k) { P[k] = a.st->pose[k]; iK[k] = 0.0; }
    // getInverseCameraMatrix in float (gFusion.h:451-457)
    iK[0] = (double)(1.0f / (float)a.fx);
    iK[8] = (double)(-(float)a.cx / (float)a.fx);
    iK[5] = (double)(1.0f / (float)a.fy);
    iK[9] = (double)(-(float)a.cy / (float)a.fy);
    iK[10] = 1.0; iK[15] = 1.0;
    kf_mat4_mul(P, iK, Vw);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 4; ++c) s_view[r * 4 + c] = (float)Vw[c * 4 + r];
    if (blockIdx.x == 0 && blockIdx.y == 0)
      for (int k = 0; k < 16; ++k) a.st_out->raycast_pose[k] = P[k];
  }
  __syncthreads();
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= a.W || y >= a.H) return;

  Sampler<S> smp;
  smp.f = reinterpret_cast<const typename Vox<S>::V*>(a.vol);
  smp.nx = a.nx; smp.ny = a.ny; smp.nz = a.nz;
  smp.sxy = (size_t)a.nx * a.ny;

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
    auto sample = [&](float tt) {
      const float px = fmaf(dx, tt, ox), py = fmaf(dy, tt, oy), pz = fmaf(dzv, tt, oz);
      return smp.interp_raw(px * a.sx - 0.5f, py * a.sy - 0.5f, pz * a.sz - 0.5f) * scale;
    };
    float f_t = sample(t), f_tt = 0.0f;
    if (f_t >= 0.0f) {
      float tb = t;
      int k = 0;
      // bounded march: a NaN sample keeps largeStep, so cap the step count
      for (int n = 0; t < tfar && n < a.max_steps; ++n) {
        f_tt = sample(t);
        if (f_tt < 0.0f) break;
        if (f_tt < 0.8f && stepsize != a.step) {
          stepsize = a.step;
          tb = t;
          k = 0;
        }
        f_t = f_tt;
        ++k;
        t = fmaf((float)k, stepsize, tb);
      }
      if (f_tt < 0.0f) {
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

}  // namespace

int kf_launch_raycast(kf_session* s) {
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
  a.fx = s->intr.fx; a.fy = s->intr.fy; a.cx = s->intr.cx; a.cy = s->intr.cy;
  a.out_v = s->d_ref_vertex;
  a.out_n = s->d_ref_normal;
  a.st = s->d_state;
  a.st_out = s->d_state;
  dim3 block(32, 8);
  dim3 grid((a.W + 31) / 32, (a.H + 7) / 8);
  switch (s->cfg.storage) {
    case KF_STORAGE_F32F32: raycast_kernel<KF_STORAGE_F32F32><<<grid, block, 0, s->stream>>>(a); break;
    case KF_STORAGE_F16U16: raycast_kernel<KF_STORAGE_F16U16><<<grid, block, 0, s->stream>>>(a); break;
    default: raycast_kernel<KF_STORAGE_RG16I><<<grid, block, 0, s->stream>>>(a); break;
  }
  KF_CUDA_TRY(s, cudaGetLastError());
  kf_note_launch(s);
  return KF_OK;
}
