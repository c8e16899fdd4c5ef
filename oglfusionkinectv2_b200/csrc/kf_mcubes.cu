// kf_mcubes.cu — marching-cubes extraction: histoPyramid path and classic scan path.
//
// Reference: MCubes::histoPyramids (src/mcubes.cpp:206-389) with
// shaders/histoPyramids.cs:42-174 (classifyCubes, constructHPLevel) and
// shaders/traverseHistoPyramids.cs:54-260 (traverseHPLevel); the classic path of
// shaders/marchingCubes.cs:102-305 (classify / compact / generate, dead code in the
// reference) on top of the prefix sum (prefixSum.cs); export mcubes.cpp:391-509.
//
// histoPyramid semantics kept: cube corners in the reference's y/z-swapped order
// {000,100,001,101,010,110,011,111}; "positive found" over the first 7 corners (Q13);
// cubes within 10 voxels of the border left empty (Q15); cubeIndex bits f0,f1,f3,f2,
// f4,f5,f7,f6 -> 1..128; base texel = nrOfTriangles | cubeIndex << 16; level k+1 = 2x2x2
// sum; traversal descends the levels with the reference's running-sum comparison;
// vertices at mix(p0, p1, a) in voxel-index units with a = 0.5 outside [0, 1], w = 0.
// The pyramid is padded to a power of two P >= N with zero counts (the reference only
// supports power-of-two N, Q16).
//
// B200 design: one kernel classifies the 8 cubes of every level-1 cell from its 27
// corner values (each value read once per cell) and writes the base level and level 1;
// each further level is one small reduction; traversal is one thread per triangle over an
// L2-resident pyramid (the levels above the base are 1/8 + 1/64 + ... of the volume).
#include <algorithm>
#include <cstdio>
#include <vector>

#include "kf_internal.cuh"

#define KF_MC_TABLE_QUAL static __device__ const
#include "generated/kf_mc_tables.inc"

namespace {

__constant__ int c_hp_off[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 0, 1}, {1, 0, 1},
                                   {0, 1, 0}, {1, 1, 0}, {0, 1, 1}, {1, 1, 1}};
__constant__ int c_bourke[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                   {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
__constant__ int c_bourke_edge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                         {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

struct McArgs {
  const void* vol;
  int nx, ny, nz;
  float iso;
  int q13, q15;
  uint32_t* base;    // nx*ny*nz
  uint32_t* level1;  // (P/2)^3
  int D1;            // P / 2
};

// getVolumeData (histoPyramids.cs:95-107): the raw int16 for RG16I, the value otherwise
template <int S>
__device__ __forceinline__ float mc_raw(const void* vol, size_t i) {
  return Vox<S>::raw(reinterpret_cast<const typename Vox<S>::V*>(vol), i);
}

template <int S>
__global__ void __launch_bounds__(256) classify_kernel(McArgs a) {
  const int D = a.D1;
  const size_t cell = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= (size_t)D * D * D) return;
  const int cx = (int)(cell % D), cy = (int)((cell / D) % D), cz = (int)(cell / ((size_t)D * D));
  const int x0 = 2 * cx, y0 = 2 * cy, z0 = 2 * cz;
  uint32_t sum = 0;
  if (x0 < a.nx && y0 < a.ny && z0 < a.nz) {
    // the 3x3x3 corner values shared by this cell's 8 cubes
    float v[3][3][3];
#pragma unroll
    for (int dz = 0; dz < 3; ++dz)
#pragma unroll
      for (int dy = 0; dy < 3; ++dy)
#pragma unroll
        for (int dx = 0; dx < 3; ++dx) {
          const int x = x0 + dx, y = y0 + dy, z = z0 + dz;
          v[dz][dy][dx] = (x < a.nx && y < a.ny && z < a.nz)
                              ? mc_raw<S>(a.vol, (size_t)x + (size_t)a.nx * ((size_t)y + (size_t)a.ny * z))
                              : 0.0f;
        }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
      const int x = x0 + ox, y = y0 + oy, z = z0 + oz;
      if (x >= a.nx || y >= a.ny || z >= a.nz) continue;
      bool skip;
      if (a.q15)  // histoPyramids.cs:117
        skip = x <= 10 || x >= a.nx - 10 || y <= 10 || y >= a.ny - 10 || z <= 10 || z >= a.nz - 10;
      else
        skip = x >= a.nx - 1 || y >= a.ny - 1 || z >= a.nz - 1;
      uint32_t texel = 0;
      if (!skip) {
        float f[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) f[c] = v[oz + c_hp_off[c][2]][oy + c_hp_off[c][1]][ox + c_hp_off[c][0]];
        bool pos = false;
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if (c < 7 || !a.q13) pos |= f[c] > 0.0f;
        if (pos) {
          const float iso = a.iso;
          const uint32_t ci = (uint32_t)(f[0] < iso) | ((uint32_t)(f[1] < iso) << 1) | ((uint32_t)(f[3] < iso) << 2) |
                              ((uint32_t)(f[2] < iso) << 3) | ((uint32_t)(f[4] < iso) << 4) |
                              ((uint32_t)(f[5] < iso) << 5) | ((uint32_t)(f[7] < iso) << 6) |
                              ((uint32_t)(f[6] < iso) << 7);
          const uint32_t nt = kf_mc_nr_triangles[ci];
          texel = nt | (ci << 16);
          sum += nt;
        }
      }
      a.base[(size_t)x + (size_t)a.nx * ((size_t)y + (size_t)a.ny * z)] = texel;
    }
  }
  a.level1[cell] = sum;
}

// constructHPLevel (histoPyramids.cs:42-93): level k+1 = 2x2x2 sum of level k
__global__ void __launch_bounds__(256) reduce_level_kernel(const uint32_t* __restrict__ lo, uint32_t* __restrict__ hi,
                                                           int D) {
  const size_t cell = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= (size_t)D * D * D) return;
  const int x = (int)(cell % D), y = (int)((cell / D) % D), z = (int)(cell / ((size_t)D * D));
  const int Dl = 2 * D;
  uint32_t s = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c)
    s += __ldg(lo + (size_t)(2 * x + (c & 1)) + (size_t)Dl * ((size_t)(2 * y + ((c >> 1) & 1)) +
                                                           (size_t)Dl * (2 * z + (c >> 2))));
  hi[cell] = s;
}

struct TravArgs {
  const void* vol;
  int nx, ny, nz;
  float iso;
  const uint32_t* base;
  const uint32_t* const* levels;  // device array: levels[k] for k >= 1
  int P, top;
  uint32_t total;
  float4* out;
};

template <int S>
__global__ void __launch_bounds__(256) traverse_kernel(TravArgs a) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.total) return;
  int cx = 0, cy = 0, cz = 0;
  uint32_t w = 0;
  for (int k = a.top - 1; k >= 0; --k) {  // scanHPLevel (traverseHistoPyramids.cs:54-119)
    uint32_t nb[8];
    if (k == 0) {
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int x = cx + c_hp_off[c][0], y = cy + c_hp_off[c][1], z = cz + c_hp_off[c][2];
        nb[c] = (x < a.nx && y < a.ny && z < a.nz)
                    ? (__ldg(a.base + (size_t)x + (size_t)a.nx * ((size_t)y + (size_t)a.ny * z)) & 0xffffu)
                    : 0u;
      }
    } else {
      const uint32_t* L = a.levels[k];
      const int D = a.P >> k;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int x = cx + c_hp_off[c][0], y = cy + c_hp_off[c][1], z = cz + c_hp_off[c][2];
        nb[c] = __ldg(L + (size_t)x + (size_t)D * ((size_t)y + (size_t)D * z));
      }
    }
    uint32_t acc = w, add = 0;
    int sel = 0;
#pragma unroll
    for (int c = 0; c < 7; ++c) {
      acc += nb[c];
      if (acc <= t) { ++sel; add += nb[c]; }
    }
    cx = (cx + c_hp_off[sel][0]) * 2;
    cy = (cy + c_hp_off[sel][1]) * 2;
    cz = (cz + c_hp_off[sel][2]) * 2;
    w += add;
  }
  cx >>= 1; cy >>= 1; cz >>= 1;
  const size_t cube = (size_t)cx + (size_t)a.nx * ((size_t)cy + (size_t)a.ny * cz);
  const uint32_t ci = __ldg(a.base + cube) >> 16;
  const int j = (int)(t - w);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int edge = kf_mc_tri_table[ci * 16 + 3 * j + k];
    const uint8_t* o = &kf_mc_offsets3[edge * 6];
    const int p0x = cx + o[0], p0y = cy + o[1], p0z = cz + o[2];
    const int p1x = cx + o[3], p1y = cy + o[4], p1z = cz + o[5];
    const float v0 = mc_raw<S>(a.vol, (size_t)p0x + (size_t)a.nx * ((size_t)p0y + (size_t)a.ny * p0z));
    const float v1 = mc_raw<S>(a.vol, (size_t)p1x + (size_t)a.nx * ((size_t)p1y + (size_t)a.ny * p1z));
    float al = (a.iso - v0) / (v1 - v0);
    if (al > 1.0f || al < 0.0f) al = 0.5f;  // traverseHistoPyramids.cs:213-216
    a.out[(size_t)t * 3 + k] = make_float4(p0x * (1.0f - al) + p1x * al, p0y * (1.0f - al) + p1y * al,
                                           p0z * (1.0f - al) + p1z * al, 0.0f);
  }
}

// ---- classic path (marchingCubes.cs) ---------------------------------------------------
struct ScanArgs {
  const void* vol;
  int nx, ny, nz;
  float iso;
  int q13;
  uint32_t* verts;  // numVerts per voxel
  uint32_t* base;   // (numVerts / 3) | cubeIndex << 16, as the histoPyramid base level
  const uint32_t* offsets;
  float4* out;
};

template <int S>
__device__ __forceinline__ void bourke_fields(const ScanArgs& a, int x, int y, int z, float* f) {
  // sampleVolume clamps to gridSize - 1 (marchingCubes.cs:70-78)
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int X = min(x + c_bourke[k][0], a.nx - 1), Y = min(y + c_bourke[k][1], a.ny - 1),
              Z = min(z + c_bourke[k][2], a.nz - 1);
    f[k] = mc_raw<S>(a.vol, (size_t)X + (size_t)a.nx * ((size_t)Y + (size_t)a.ny * Z));
  }
}

template <int S>
__global__ void __launch_bounds__(256) scan_classify_kernel(ScanArgs a) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t n = (size_t)a.nx * a.ny * a.nz;
  if (i >= n) return;
  const int x = (int)(i % a.nx), y = (int)((i / a.nx) % a.ny), z = (int)(i / ((size_t)a.nx * a.ny));
  float f[8];
  bourke_fields<S>(a, x, y, z, f);
  bool pos = false;
#pragma unroll
  for (int k = 0; k < 8; ++k)
    if (k < 7 || !a.q13) pos |= f[k] > 0.0f;
  uint32_t nv = 0, texel = 0;
  if (pos) {
    uint32_t ci = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) ci |= (uint32_t)(f[k] < a.iso) << k;
    nv = kf_mc_num_verts[ci];
    texel = (nv / 3) | (ci << 16);
  }
  a.verts[i] = nv;
  a.base[i] = texel;
}

template <int S>
__global__ void __launch_bounds__(256) scan_generate_kernel(ScanArgs a) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t n = (size_t)a.nx * a.ny * a.nz;
  if (i >= n) return;
  const uint32_t nv = a.verts[i];
  if (!nv) return;
  const int x = (int)(i % a.nx), y = (int)((i / a.nx) % a.ny), z = (int)(i / ((size_t)a.nx * a.ny));
  float f[8];
  bourke_fields<S>(a, x, y, z, f);
  const uint32_t ci = a.base[i] >> 16;
  const uint32_t off = a.offsets[i];
  for (uint32_t v = 0; v < nv; ++v) {
    const int e = kf_mc_tri_table[ci * 16 + v];
    const int p = c_bourke_edge[e][0], q = c_bourke_edge[e][1];
    const float t = (a.iso - f[p]) / (f[q] - f[p]);  // vertexInterp (:81-85)
    const float ax = x + c_bourke[p][0], ay = y + c_bourke[p][1], az = z + c_bourke[p][2];
    const float bx = x + c_bourke[q][0], by = y + c_bourke[q][1], bz = z + c_bourke[q][2];
    a.out[off + v] = make_float4(ax * (1.0f - t) + bx * t, ay * (1.0f - t) + by * t, az * (1.0f - t) + bz * t, 1.0f);
  }
}

// Grows a device buffer to at least `bytes`, by 1.5x steps so that a mesh that grows
// from one extraction to the next does not reallocate (and synchronise) every time.
int ensure(kf_session* s, void** p, size_t* cap, size_t bytes) {
  if (*cap >= bytes && *p) return KF_OK;
  bytes = std::max(bytes, *cap + *cap / 2);
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    s->last_error = "marching cubes: out of device memory";
    return KF_ERR_OUT_OF_MEMORY;
  }
  *cap = bytes;
  return KF_OK;
}

// Bytes for the vertex buffer: the vertices needed now, but at least room for one triangle
// per 64 cubes (fused scenes reach one triangle per 200-600 cubes), so a mesh that grows as
// frames are fused does not reallocate: a reallocation frees and allocates device memory,
// which synchronises the device and takes the driver's locks, whose wait is unbounded on a
// shared machine.
size_t vertex_bytes(size_t ncube, size_t nverts) {
  return std::max<size_t>(16, std::max(nverts, ncube / 64 * 3) * 16);
}

int histopyramid(kf_session* s, float iso, uint32_t* n_tri) {
  const int nx = s->cfg.nx, ny = s->cfg.ny, nz = s->cfg.nz;
  int P = 1, top = 0;
  while (P < std::max(nx, std::max(ny, nz))) { P <<= 1; ++top; }
  if (top < 1) return KF_ERR_INVALID_ARGUMENT;
  const size_t ncube = (size_t)nx * ny * nz;
  if (!s->d_mc_base) {
    if (cudaMalloc((void**)&s->d_mc_base, ncube * 4) != cudaSuccess) {
      cudaGetLastError();
      return KF_ERR_OUT_OF_MEMORY;
    }
  }
  if (s->mc_P != P || (int)s->d_mc_levels.size() != top + 1) {
    for (uint32_t* p : s->d_mc_levels) cudaFree(p);
    s->d_mc_levels.assign(top + 1, nullptr);
    for (int k = 1; k <= top; ++k) {
      const size_t D = (size_t)(P >> k);
      if (cudaMalloc((void**)&s->d_mc_levels[k], D * D * D * 4) != cudaSuccess) {
        cudaGetLastError();
        return KF_ERR_OUT_OF_MEMORY;
      }
    }
    s->mc_P = P;
    s->mc_top = top;
  }
  McArgs a;
  a.vol = s->d_vol;
  a.nx = nx; a.ny = ny; a.nz = nz;
  a.iso = iso;
  a.q13 = (s->cfg.quirks & KF_Q13_MC_FIRST_SEVEN) ? 1 : 0;
  a.q15 = (s->cfg.quirks & KF_Q15_MC_BORDER_SKIP) ? 1 : 0;
  a.base = s->d_mc_base;
  a.level1 = s->d_mc_levels[1];
  a.D1 = P / 2;
  const size_t cells = (size_t)a.D1 * a.D1 * a.D1;
  const int g1 = (int)((cells + 255) / 256);
  switch (s->cfg.storage) {
    case KF_STORAGE_F32F32: classify_kernel<KF_STORAGE_F32F32><<<g1, 256, 0, s->stream>>>(a); break;
    case KF_STORAGE_F16U16: classify_kernel<KF_STORAGE_F16U16><<<g1, 256, 0, s->stream>>>(a); break;
    default: classify_kernel<KF_STORAGE_RG16I><<<g1, 256, 0, s->stream>>>(a); break;
  }
  KF_CUDA_TRY(s, cudaGetLastError());
  kf_note_launch(s);
  for (int k = 2; k <= top; ++k) {
    const int D = P >> k;
    const size_t c = (size_t)D * D * D;
    reduce_level_kernel<<<(int)((c + 255) / 256), 256, 0, s->stream>>>(s->d_mc_levels[k - 1], s->d_mc_levels[k], D);
    KF_CUDA_TRY(s, cudaGetLastError());
    kf_note_launch(s);
  }
  // the top texel holds the triangle count (glGetTexImage at mcubes.cpp:290-300)
  KF_CUDA_TRY(s, cudaMemcpyAsync(s->h_u32_scalar, s->d_mc_levels[top], 4, cudaMemcpyDeviceToHost, s->stream));
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  const uint32_t T = s->h_u32_scalar[0];
  int rc = ensure(s, (void**)&s->d_mc_vertices, &s->mc_vertex_cap, vertex_bytes(ncube, (size_t)T * 3));
  if (rc) return rc;
  // device copy of the level pointer table
  std::vector<uint32_t*> host_levels(s->d_mc_levels);
  uint32_t** d_levels = nullptr;
  rc = ensure(s, (void**)&s->d_mc_scratch, &s->mc_scratch_words, (top + 1) * sizeof(uint32_t*));
  if (rc) return rc;
  d_levels = reinterpret_cast<uint32_t**>(s->d_mc_scratch);
  KF_CUDA_TRY(s, cudaMemcpyAsync(d_levels, host_levels.data(), (top + 1) * sizeof(uint32_t*), cudaMemcpyHostToDevice,
                                 s->stream));
  if (T) {
    TravArgs t;
    t.vol = s->d_vol;
    t.nx = nx; t.ny = ny; t.nz = nz;
    t.iso = iso;
    t.base = s->d_mc_base;
    t.levels = d_levels;
    t.P = P;
    t.top = top;
    t.total = T;
    t.out = s->d_mc_vertices;
    const int g = (int)((T + 255) / 256);
    switch (s->cfg.storage) {
      case KF_STORAGE_F32F32: traverse_kernel<KF_STORAGE_F32F32><<<g, 256, 0, s->stream>>>(t); break;
      case KF_STORAGE_F16U16: traverse_kernel<KF_STORAGE_F16U16><<<g, 256, 0, s->stream>>>(t); break;
      default: traverse_kernel<KF_STORAGE_RG16I><<<g, 256, 0, s->stream>>>(t); break;
    }
    KF_CUDA_TRY(s, cudaGetLastError());
    kf_note_launch(s);
  }
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));  // the pointer table lives in pageable memory
  *n_tri = T;
  return KF_OK;
}

int classic(kf_session* s, float iso, uint32_t* n_tri) {
  const int nx = s->cfg.nx, ny = s->cfg.ny, nz = s->cfg.nz;
  const size_t n = (size_t)nx * ny * nz;
  if (n >= (1ull << 32)) return KF_ERR_INVALID_ARGUMENT;
  if (!s->d_mc_base) {
    if (cudaMalloc((void**)&s->d_mc_base, n * 4) != cudaSuccess) {
      cudaGetLastError();
      return KF_ERR_OUT_OF_MEMORY;
    }
  }
  const size_t sw = kf_scan_scratch_words(n);
  // scratch: verts[n], offsets[n], scan scratch[sw], total[1]
  const size_t words = 2 * n + sw + 1;
  int rc = ensure(s, (void**)&s->d_mc_scratch, &s->mc_scratch_words, words * 4);
  if (rc) return rc;
  uint32_t* verts = s->d_mc_scratch;
  uint32_t* offs = verts + n;
  uint32_t* scr = offs + n;
  uint32_t* d_tot = scr + sw;
  ScanArgs a;
  a.vol = s->d_vol;
  a.nx = nx; a.ny = ny; a.nz = nz;
  a.iso = iso;
  a.q13 = (s->cfg.quirks & KF_Q13_MC_FIRST_SEVEN) ? 1 : 0;
  a.verts = verts;
  a.base = s->d_mc_base;
  a.offsets = offs;
  const int g = (int)((n + 255) / 256);
  switch (s->cfg.storage) {
    case KF_STORAGE_F32F32: scan_classify_kernel<KF_STORAGE_F32F32><<<g, 256, 0, s->stream>>>(a); break;
    case KF_STORAGE_F16U16: scan_classify_kernel<KF_STORAGE_F16U16><<<g, 256, 0, s->stream>>>(a); break;
    default: scan_classify_kernel<KF_STORAGE_RG16I><<<g, 256, 0, s->stream>>>(a); break;
  }
  KF_CUDA_TRY(s, cudaGetLastError());
  kf_note_launch(s);
  rc = kf_scan_u32(verts, offs, n, d_tot, s->stream, scr, sw);
  if (rc) return rc;
  KF_CUDA_TRY(s, cudaMemcpyAsync(s->h_u32_scalar, d_tot, 4, cudaMemcpyDeviceToHost, s->stream));
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  const uint32_t nverts = s->h_u32_scalar[0];
  rc = ensure(s, (void**)&s->d_mc_vertices, &s->mc_vertex_cap, vertex_bytes((size_t)s->cfg.nx * s->cfg.ny * s->cfg.nz, (size_t)nverts));
  if (rc) return rc;
  a.out = s->d_mc_vertices;
  switch (s->cfg.storage) {
    case KF_STORAGE_F32F32: scan_generate_kernel<KF_STORAGE_F32F32><<<g, 256, 0, s->stream>>>(a); break;
    case KF_STORAGE_F16U16: scan_generate_kernel<KF_STORAGE_F16U16><<<g, 256, 0, s->stream>>>(a); break;
    default: scan_generate_kernel<KF_STORAGE_RG16I><<<g, 256, 0, s->stream>>>(a); break;
  }
  KF_CUDA_TRY(s, cudaGetLastError());
  kf_note_launch(s);
  *n_tri = nverts / 3;
  return KF_OK;
}

int copy_vertices_host(kf_session* s, std::vector<float>& v) {
  v.resize((size_t)s->mc_triangles * 3 * 4);
  if (v.empty()) return KF_OK;
  KF_CUDA_TRY(s, cudaMemcpyAsync(v.data(), s->d_mc_vertices, v.size() * 4, cudaMemcpyDeviceToHost, s->stream));
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return KF_OK;
}

}  // namespace

int kf_mc_run(kf_session* s, float iso, int method, uint32_t* n_tri) {
  cudaEvent_t e0 = s->ev[0], e1 = s->ev[1];
  cudaEventRecord(e0, s->stream);
  s->mc_valid = 0;
  int rc = (method == KF_MC_SCAN) ? classic(s, iso, n_tri) : histopyramid(s, iso, n_tri);
  if (rc) return rc;
  cudaEventRecord(e1, s->stream);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(&s->stage_ms[5], e0, e1);
  s->mc_triangles = *n_tri;
  s->mc_valid = 1;
  return KF_OK;
}

extern "C" {

int kf_mc_extract(kf_session* s, float iso, int method, uint32_t* n) {
  if (!s || !n || (method != KF_MC_HISTOPYRAMID && method != KF_MC_SCAN)) return KF_ERR_INVALID_ARGUMENT;
  return kf_mc_run(s, iso, method, n);
}

int kf_mc_copy_vertices(kf_session* s, float* v, uint64_t max_vertices) {
  if (!s || (!v && s->mc_triangles)) return KF_ERR_INVALID_ARGUMENT;
  if (!s->mc_valid) return KF_ERR_STATE;
  const uint64_t n = (uint64_t)s->mc_triangles * 3;
  if (max_vertices < n) return KF_ERR_CAPACITY;
  if (!n) return KF_OK;
  KF_CUDA_TRY(s, cudaMemcpyAsync(v, s->d_mc_vertices, n * 16, cudaMemcpyDeviceToHost, s->stream));
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return KF_OK;
}

int kf_mc_copy_base_level(kf_session* s, uint32_t* base, uint64_t count) {
  if (!s || !base) return KF_ERR_INVALID_ARGUMENT;
  if (!s->mc_valid) return KF_ERR_STATE;
  if (count != (uint64_t)s->cfg.nx * s->cfg.ny * s->cfg.nz) return KF_ERR_INVALID_ARGUMENT;
  KF_CUDA_TRY(s, cudaMemcpyAsync(base, s->d_mc_base, count * 4, cudaMemcpyDeviceToHost, s->stream));
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return KF_OK;
}

int kf_mc_export_stl(kf_session* s, const char* path) {
  // exportMesh (mcubes.cpp:429-509): 80-byte header (zeroed here), uint32 triangle count
  // (4x with Q18), then per triangle normal (1,1,1), three vertices, uint16 0
  if (!s || !path) return KF_ERR_INVALID_ARGUMENT;
  if (!s->mc_valid) return KF_ERR_STATE;
  std::vector<float> v;
  int rc = copy_vertices_host(s, v);
  if (rc) return rc;
  FILE* f = std::fopen(path, "wb");
  if (!f) return KF_ERR_IO;
  char hdr[80];
  std::memset(hdr, 0, sizeof(hdr));
  const uint32_t T = s->mc_triangles;
  const uint32_t count = (s->cfg.quirks & KF_Q18_STL_COUNT_X4) ? 4 * T : T;
  bool ok = std::fwrite(hdr, 1, 80, f) == 80 && std::fwrite(&count, 4, 1, f) == 1;
  std::vector<unsigned char> rec((size_t)T * 50);
  const float nrm[3] = {1.0f, 1.0f, 1.0f};
  const uint16_t attr = 0;
  for (uint32_t t = 0; t < T; ++t) {
    unsigned char* r = &rec[(size_t)t * 50];
    std::memcpy(r, nrm, 12);
    for (int k = 0; k < 3; ++k) std::memcpy(r + 12 + 12 * k, &v[((size_t)t * 3 + k) * 4], 12);
    std::memcpy(r + 48, &attr, 2);
  }
  ok = ok && (T == 0 || std::fwrite(rec.data(), 1, rec.size(), f) == rec.size());
  ok = (std::fclose(f) == 0) && ok;
  return ok ? KF_OK : KF_ERR_IO;
}

int kf_mc_export_ply(kf_session* s, const char* path) {
  // exportPointCloud (mcubes.cpp:391-427): ASCII PLY of the vertex buffer
  if (!s || !path) return KF_ERR_INVALID_ARGUMENT;
  if (!s->mc_valid) return KF_ERR_STATE;
  std::vector<float> v;
  int rc = copy_vertices_host(s, v);
  if (rc) return rc;
  FILE* f = std::fopen(path, "w");
  if (!f) return KF_ERR_IO;
  const unsigned long long n = (unsigned long long)s->mc_triangles * 3;
  std::fprintf(f, "ply\nformat ascii 1.0\nelement vertex %llu\nproperty float x\nproperty float y\n"
               "property float z\nend_header\n", n);
  for (unsigned long long i = 0; i < n; ++i) std::fprintf(f, "%g %g %g\n", v[i * 4], v[i * 4 + 1], v[i * 4 + 2]);
  const bool bad = std::ferror(f);
  return (std::fclose(f) == 0 && !bad) ? KF_OK : KF_ERR_IO;
}

}  // extern "C"
