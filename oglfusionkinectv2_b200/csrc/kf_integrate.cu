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
// B200 design: threads own 32 consecutive x of one y (one warp = 64 B per plane per
// z-step for 2-byte storage, fully used sectors).  Each column first intersects its line
// with the camera frustum analytically (five half-spaces, solved in FP64 with a two-voxel
// margin) so voxels that cannot project into the image are never visited; inside the
// interval every voxel runs the reference's exact tests.  The weight plane is read only
// where eta > -mu, and a voxel whose encoded value and weight do not change is not
// written back (the reference writes it unchanged).  Result bits are the same as
// without these shortcuts.
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
  float mu, maxw;
  int band;  // Q8
  const int* gate;
  const KfDevState* st;
};

template <class T>
__device__ __forceinline__ uint32_t bits_of(const T& v) {
  uint32_t b = 0;
  memcpy(&b, &v, sizeof(T));
  return b;
}

template <int S>
__global__ void __launch_bounds__(256) integrate_kernel(IntArgs a) {
  typedef typename Vox<S>::V V;
  typedef typename Vox<S>::Wt Wt;
  __shared__ float s_inv[12];  // inverse(pose): 3 rows x (R | t), row-major
  if (a.gate && *(volatile const int*)a.gate == 0) return;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    double P[16], I[16];
    for (int k = 0; k < 16; ++k) P[k] = a.st->pose[k];
    kf_rigid_inverse(P, I);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 4; ++c) s_inv[r * 4 + c] = (float)I[c * 4 + r];
  }
  __syncthreads();
  const int x = blockIdx.x * 32 + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= a.nx || y >= a.ny) return;

  // getVolumePosition (integrate.cs:16-19) for z = 0, and delta = rotate(invTrack, (0,0,vz))
  const float cxw = (x + 0.5f) * a.dimx / a.nx;
  const float cyw = (y + 0.5f) * a.dimy / a.ny;
  const float czw = 0.5f * a.dimz / a.nz;
  const float vz = a.dimz / a.nz;
  float p0[3], dz[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    p0[r] = fmaf(s_inv[r * 4 + 0], cxw, fmaf(s_inv[r * 4 + 1], cyw, fmaf(s_inv[r * 4 + 2], czw, s_inv[r * 4 + 3])));
    dz[r] = s_inv[r * 4 + 2] * vz;
  }

  // frustum interval of this column: alpha + beta * z >= 0 for all five constraints
  double lo = 0.0, hi = (double)(a.nz - 1);
  auto clip = [&](double al, double be) {
    const double eps = 1e-5 * (fabs(al) + fabs(be) * a.nz) + 1e-9;
    al += eps;
    if (be > 0) lo = fmax(lo, -al / be);
    else if (be < 0) hi = fmin(hi, -al / be);
    else if (al < 0) hi = -1.0;
  };
  {
    const double X0 = p0[0], Y0 = p0[1], Z0 = p0[2], dX = dz[0], dY = dz[1], dZ = dz[2];
    const double kx0 = (double)a.cx + 0.5, kx1 = (double)a.cx + 0.5 - (a.W - 1);
    const double ky0 = (double)a.cy + 0.5, ky1 = (double)a.cy + 0.5 - (a.H - 1);
    clip(Z0 - 1e-4, dZ);                                             // z >= 1e-4
    clip(a.fx * X0 + kx0 * Z0, a.fx * dX + kx0 * dZ);                 // px >= 0
    clip(-(a.fx * X0 + kx1 * Z0), -(a.fx * dX + kx1 * dZ));           // px <= W - 1
    clip(a.fy * Y0 + ky0 * Z0, a.fy * dY + ky0 * dZ);                 // py >= 0
    clip(-(a.fy * Y0 + ky1 * Z0), -(a.fy * dY + ky1 * dZ));           // py <= H - 1
  }
  if (!(hi >= lo - 2.0)) return;
  const int z0 = max(0, (int)floor(lo) - 2);
  const int z1 = min(a.nz - 1, (int)ceil(hi) + 2);

  V* vf = reinterpret_cast<V*>(a.vol);
  Wt* vw = reinterpret_cast<Wt*>(reinterpret_cast<char*>(a.vol) + a.count * sizeof(V));
  const size_t slice = (size_t)a.nx * a.ny;
  size_t idx = (size_t)x + (size_t)a.nx * y + (size_t)z0 * slice;
  const float fW1 = (float)(a.W - 1), fH1 = (float)(a.H - 1);
  for (int z = z0; z <= z1; ++z, idx += slice) {
    const float fz = (float)z;
    const float px3 = fmaf(fz, dz[0], p0[0]);
    const float py3 = fmaf(fz, dz[1], p0[1]);
    const float pz3 = fmaf(fz, dz[2], p0[2]);
    if (pz3 < 0.0001f) continue;
    const float u = fmaf(a.fx, px3, a.cx * pz3) / pz3 + 0.5f;
    const float v = fmaf(a.fy, py3, a.cy * pz3) / pz3 + 0.5f;
    if (u < 0.0f || u > fW1 || v < 0.0f || v > fH1) continue;
    const float d = __ldg(a.depth + (size_t)(int)v * a.W + (int)u) / 1000.0f;
    if (d == 0.0f) continue;
    const float rx = px3 / pz3, ry = py3 / pz3;
    const float diff = (d - pz3) * sqrtf(1.0f + rx * rx + ry * ry);
    if (diff > -a.mu) {
      const float sdf = fminf(1.0f, diff / a.mu);
      const V oldv = vf[idx];
      const Wt oldw = vw[idx];
      const float F = Vox<S>::raw_nc(&oldv, 0) * Vox<S>::kRawToF;
      const float w = Vox<S>::weight(&oldw, 0);
      const float wd = (w * F + sdf) / (w + 1.0f);
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
    } else {
      vf[idx] = Vox<S>::encode_value(0.0f);
      vw[idx] = Vox<S>::encode_weight(0.0f);
    }
  }
}

}  // namespace

int kf_launch_integrate(kf_session* s, int gated) {
  IntArgs a;
  a.vol = s->d_vol;
  a.count = s->vol_count;
  a.nx = s->cfg.nx; a.ny = s->cfg.ny; a.nz = s->cfg.nz;
  a.dimx = s->cfg.dim_x; a.dimy = s->cfg.dim_y; a.dimz = s->cfg.dim_z;
  a.depth = s->d_depth[0];
  a.W = s->W[0]; a.H = s->H[0];
  a.fx = s->intr.fx; a.fy = s->intr.fy; a.cx = s->intr.cx; a.cy = s->intr.cy;
  a.mu = s->cfg.mu;
  a.maxw = s->cfg.max_weight;
  a.band = (s->cfg.quirks & KF_Q8_NARROW_BAND) ? 1 : 0;
  a.gate = gated ? &s->d_state->do_integrate : nullptr;
  a.st = s->d_state;
  dim3 block(32, 8);
  dim3 grid((a.nx + 31) / 32, (a.ny + 7) / 8);
  switch (s->cfg.storage) {
    case KF_STORAGE_F32F32: integrate_kernel<KF_STORAGE_F32F32><<<grid, block, 0, s->stream>>>(a); break;
    case KF_STORAGE_F16U16: integrate_kernel<KF_STORAGE_F16U16><<<grid, block, 0, s->stream>>>(a); break;
    default: integrate_kernel<KF_STORAGE_RG16I><<<grid, block, 0, s->stream>>>(a); break;
  }
  KF_CUDA_TRY(s, cudaGetLastError());
  kf_note_launch(s);
  return KF_OK;
}
