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
#include <cmath>
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
  float4* nout;  // the triangle's face normal cross(v1 - v0, v2 - v0) per vertex, w = 0
};

__device__ __forceinline__ float4 face_normal(float4 a, float4 b, float4 c) {
  const float ux = b.x - a.x, uy = b.y - a.y, uz = b.z - a.z;
  const float vx = c.x - a.x, vy = c.y - a.y, vz = c.z - a.z;
  return make_float4(uy * vz - uz * vy, uz * vx - ux * vz, ux * vy - uy * vx, 0.0f);
}

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
  float4 vo[3];
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
    vo[k] = make_float4(p0x * (1.0f - al) + p1x * al, p0y * (1.0f - al) + p1y * al,
                        p0z * (1.0f - al) + p1z * al, 0.0f);
    a.out[(size_t)t * 3 + k] = vo[k];
  }
  const float4 fn = face_normal(vo[0], vo[1], vo[2]);
#pragma unroll
  for (int k = 0; k < 3; ++k) a.nout[(size_t)t * 3 + k] = fn;
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
  float4* nout;      // face normal per vertex (w = 0)
  int shader_units;  // Q24: marchingCubes.cs's output convention (see scan_generate_kernel)
  float vsx, vsy, vsz;  // its voxelSize (mCubeConfig, mcubes.h:30-39): 1000 * dim / size
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
  // corner positions: voxel-index units, or with Q24 the shader's p = -1 + gridPos *
  // voxelSize plus the corner's voxelSize offset (launchGenerateTriangles, :205-220)
  float px = (float)x, py = (float)y, pz = (float)z, sx = 1.0f, sy = 1.0f, sz = 1.0f;
  if (a.shader_units) {
    px = -1.0f + (float)x * a.vsx;
    py = -1.0f + (float)y * a.vsy;
    pz = -1.0f + (float)z * a.vsz;
    sx = a.vsx; sy = a.vsy; sz = a.vsz;
  }
  for (uint32_t v = 0; v < nv; v += 3) {
    float4 vo[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int e = kf_mc_tri_table[ci * 16 + v + k];
      const int p = c_bourke_edge[e][0], q = c_bourke_edge[e][1];
      const float t = (a.iso - f[p]) / (f[q] - f[p]);  // vertexInterp (:81-85)
      const float ax = c_bourke[p][0] ? px + sx : px, ay = c_bourke[p][1] ? py + sy : py,
                  az = c_bourke[p][2] ? pz + sz : pz;
      const float bx = c_bourke[q][0] ? px + sx : px, by = c_bourke[q][1] ? py + sy : py,
                  bz = c_bourke[q][2] ? pz + sz : pz;
      vo[k] = make_float4(ax * (1.0f - t) + bx * t, ay * (1.0f - t) + by * t, az * (1.0f - t) + bz * t, 1.0f);
    }
    // calcNormal (:87-93) on the unscaled positions, one per triangle
    const float4 fn = face_normal(vo[0], vo[1], vo[2]);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float4 o = vo[k];
      if (a.shader_units)  // pos[index] of :290-299: / 128 * voxelSize.x, z negated
        o = make_float4((o.x / 128.0f) * a.vsx, (o.y / 128.0f) * a.vsx, -(o.z / 128.0f) * a.vsx, 1.0f);
      a.out[off + v + k] = o;
      a.nout[off + v + k] = fn;
    }
  }
}

// ---- welded mesh: one vertex per cut voxel edge, indexed triangles ----------------------
// Export form (no counterpart in the reference, whose exportMesh writes the triangle soup
// with normal (1,1,1), mcubes.cpp:451-500).  Cubes are the interior cubes [0, n-2]^3 in the
// classic path's Bourke corner order and case table; a triangle vertex lies on a cube edge,
// which belongs to the voxel at its lower end and its axis.  Every edge a triangle uses is
// marked (bit 3 * (v % 10) + axis of word v / 10, so the bits run in voxel order, then axis
// order), the marks are counted per word and prefix-summed: an edge's vertex index is its
// rank among the marked edges, the same whatever the launch.  Positions are world metres
// ((voxel index + 0.5) * dim / size, the voxel centres of integrate.cs:16-19); normals the
// normalised TSDF gradient (central differences at the edge's two voxels, interpolated).
// per Bourke edge (corners c_bourke_edge): the voxel at its lower end (offset from the
// cube's corner 0) and its axis
__constant__ int c_edge_owner[12][4] = {{0, 0, 0, 0}, {1, 0, 0, 1}, {0, 1, 0, 0}, {0, 0, 0, 1},
                                        {0, 0, 1, 0}, {1, 0, 1, 1}, {0, 1, 1, 0}, {0, 0, 1, 1},
                                        {0, 0, 0, 2}, {1, 0, 0, 2}, {1, 1, 0, 2}, {0, 1, 0, 2}};

struct MeshArgs {
  const void* vol;
  int nx, ny, nz;
  float iso;
  int q13;
  uint32_t* mask;            // ceil(nx*ny*nz / 10) words
  uint32_t* tri_count;       // per voxel (cube at its lower corner)
  const uint32_t* tri_off;   // exclusive scan of tri_count
  uint32_t* word_count;      // set bits per mask word
  const uint32_t* word_off;  // exclusive scan of word_count
  float* pos;
  float* nrm;
  uint32_t* idx;
  float dimx, dimy, dimz;
};

template <int S>
__device__ __forceinline__ bool mesh_cube(const MeshArgs& a, int x, int y, int z, uint32_t* ci_out) {
  float f[8];
#pragma unroll
  for (int k = 0; k < 8; ++k)
    f[k] = mc_raw<S>(a.vol, (size_t)(x + c_bourke[k][0]) +
                               (size_t)a.nx * ((size_t)(y + c_bourke[k][1]) + (size_t)a.ny * (z + c_bourke[k][2])));
  bool pos = false;
#pragma unroll
  for (int k = 0; k < 8; ++k)
    if (k < 7 || !a.q13) pos |= f[k] > 0.0f;
  if (!pos) return false;
  uint32_t ci = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) ci |= (uint32_t)(f[k] < a.iso) << k;
  *ci_out = ci;
  return kf_mc_num_verts[ci] != 0;
}

__device__ __forceinline__ void mesh_edge(const MeshArgs& a, int x, int y, int z, int e, uint32_t* word,
                                          uint32_t* bit) {
  const size_t v = (size_t)(x + c_edge_owner[e][0]) +
                   (size_t)a.nx * ((size_t)(y + c_edge_owner[e][1]) + (size_t)a.ny * (z + c_edge_owner[e][2]));
  *word = (uint32_t)(v / 10);
  *bit = (uint32_t)(v % 10) * 3 + (uint32_t)c_edge_owner[e][3];
}

template <int S>
__global__ void __launch_bounds__(256) mesh_mark_kernel(MeshArgs a) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t n = (size_t)a.nx * a.ny * a.nz;
  if (i >= n) return;
  const int x = (int)(i % a.nx), y = (int)((i / a.nx) % a.ny), z = (int)(i / ((size_t)a.nx * a.ny));
  uint32_t nt = 0, ci = 0;
  if (x < a.nx - 1 && y < a.ny - 1 && z < a.nz - 1 && mesh_cube<S>(a, x, y, z, &ci)) {
    const uint32_t nv = kf_mc_num_verts[ci];
    nt = nv / 3;
    for (uint32_t k = 0; k < nv; ++k) {
      uint32_t w, b;
      mesh_edge(a, x, y, z, kf_mc_tri_table[ci * 16 + k], &w, &b);
      atomicOr(a.mask + w, 1u << b);
    }
  }
  a.tri_count[i] = nt;
}

__global__ void __launch_bounds__(256) mesh_popc_kernel(const uint32_t* __restrict__ mask, uint32_t* __restrict__ cnt,
                                                        size_t words) {
  const size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (w < words) cnt[w] = (uint32_t)__popc(mask[w]);
}

template <int S>
__device__ __forceinline__ float mesh_val(const MeshArgs& a, int x, int y, int z) {
  x = min(max(x, 0), a.nx - 1);
  y = min(max(y, 0), a.ny - 1);
  z = min(max(z, 0), a.nz - 1);
  return mc_raw<S>(a.vol, (size_t)x + (size_t)a.nx * ((size_t)y + (size_t)a.ny * z));
}

template <int S>
__global__ void __launch_bounds__(256) mesh_vertex_kernel(MeshArgs a, size_t words) {
  const size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= words) return;
  uint32_t m = a.mask[w];
  uint32_t out = a.word_off[w];
  const float hx = 0.5f * a.nx / a.dimx, hy = 0.5f * a.ny / a.dimy, hz = 0.5f * a.nz / a.dimz;
  while (m) {
    const int b = __ffs(m) - 1;
    m &= m - 1;
    const size_t v = w * 10 + (size_t)(b / 3);
    const int axis = b % 3;
    const int x = (int)(v % a.nx), y = (int)((v / a.nx) % a.ny), z = (int)(v / ((size_t)a.nx * a.ny));
    const int x1 = x + (axis == 0), y1 = y + (axis == 1), z1 = z + (axis == 2);
    const float f0 = mesh_val<S>(a, x, y, z), f1 = mesh_val<S>(a, x1, y1, z1);
    const float t = (a.iso - f0) / (f1 - f0);  // vertexInterp (marchingCubes.cs:81-85)
    const float px = x + t * (x1 - x), py = y + t * (y1 - y), pz = z + t * (z1 - z);
    a.pos[3 * out + 0] = (px + 0.5f) * a.dimx / a.nx;
    a.pos[3 * out + 1] = (py + 0.5f) * a.dimy / a.ny;
    a.pos[3 * out + 2] = (pz + 0.5f) * a.dimz / a.nz;
    // central-difference gradients at both voxels (world units), interpolated
    float g[3];
    {
      const float g0x = (mesh_val<S>(a, x + 1, y, z) - mesh_val<S>(a, x - 1, y, z)) * hx;
      const float g0y = (mesh_val<S>(a, x, y + 1, z) - mesh_val<S>(a, x, y - 1, z)) * hy;
      const float g0z = (mesh_val<S>(a, x, y, z + 1) - mesh_val<S>(a, x, y, z - 1)) * hz;
      const float g1x = (mesh_val<S>(a, x1 + 1, y1, z1) - mesh_val<S>(a, x1 - 1, y1, z1)) * hx;
      const float g1y = (mesh_val<S>(a, x1, y1 + 1, z1) - mesh_val<S>(a, x1, y1 - 1, z1)) * hy;
      const float g1z = (mesh_val<S>(a, x1, y1, z1 + 1) - mesh_val<S>(a, x1, y1, z1 - 1)) * hz;
      g[0] = g0x + t * (g1x - g0x);
      g[1] = g0y + t * (g1y - g0y);
      g[2] = g0z + t * (g1z - g0z);
    }
    const float len = sqrtf(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    const float il = len > 0.0f ? 1.0f / len : 0.0f;
    a.nrm[3 * out + 0] = g[0] * il;
    a.nrm[3 * out + 1] = g[1] * il;
    a.nrm[3 * out + 2] = g[2] * il;
    ++out;
  }
}

template <int S>
__global__ void __launch_bounds__(256) mesh_index_kernel(MeshArgs a) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t n = (size_t)a.nx * a.ny * a.nz;
  if (i >= n || !a.tri_count[i]) return;
  const int x = (int)(i % a.nx), y = (int)((i / a.nx) % a.ny), z = (int)(i / ((size_t)a.nx * a.ny));
  uint32_t ci = 0;
  mesh_cube<S>(a, x, y, z, &ci);
  const uint32_t nv = kf_mc_num_verts[ci];
  const size_t base = (size_t)a.tri_off[i] * 3;
  for (uint32_t k = 0; k < nv; ++k) {
    uint32_t w, b;
    mesh_edge(a, x, y, z, kf_mc_tri_table[ci * 16 + k], &w, &b);
    // table vertices (0, 1, 2) stored as (0, 2, 1): counter-clockwise seen from the positive
    // (free-space) side, so facet normals point along the TSDF gradient
    const uint32_t r = k % 3, slot = k - r + (r == 0 ? 0u : 3u - r);
    a.idx[base + slot] = a.word_off[w] + (uint32_t)__popc(a.mask[w] & ((1u << b) - 1u));
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
  rc = ensure(s, (void**)&s->d_mc_normals, &s->mc_normal_cap, vertex_bytes(ncube, (size_t)T * 3));
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
    t.nout = s->d_mc_normals;
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
  rc = ensure(s, (void**)&s->d_mc_normals, &s->mc_normal_cap, vertex_bytes((size_t)s->cfg.nx * s->cfg.ny * s->cfg.nz, (size_t)nverts));
  if (rc) return rc;
  a.out = s->d_mc_vertices;
  a.nout = s->d_mc_normals;
  a.shader_units = (s->cfg.quirks & KF_Q24_MC_SHADER_UNITS) ? 1 : 0;
  a.vsx = 1000.0f * s->cfg.dim_x / (float)nx;
  a.vsy = 1000.0f * s->cfg.dim_y / (float)ny;
  a.vsz = 1000.0f * s->cfg.dim_z / (float)nz;
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

template <int S>
void launch_mesh_kernels(kf_session* s, const MeshArgs& a, int phase, size_t n, size_t words) {
  const int g = (int)((n + 255) / 256), gw = (int)((words + 255) / 256);
  if (phase == 0) mesh_mark_kernel<S><<<g, 256, 0, s->stream>>>(a);
  else if (phase == 1) mesh_vertex_kernel<S><<<gw, 256, 0, s->stream>>>(a, words);
  else mesh_index_kernel<S><<<g, 256, 0, s->stream>>>(a);
}

int mesh_phase(kf_session* s, const MeshArgs& a, int phase, size_t n, size_t words) {
  switch (s->cfg.storage) {
    case KF_STORAGE_F32F32: launch_mesh_kernels<KF_STORAGE_F32F32>(s, a, phase, n, words); break;
    case KF_STORAGE_F16U16: launch_mesh_kernels<KF_STORAGE_F16U16>(s, a, phase, n, words); break;
    default: launch_mesh_kernels<KF_STORAGE_RG16I>(s, a, phase, n, words); break;
  }
  KF_CUDA_TRY(s, cudaGetLastError());
  kf_note_launch(s);
  return KF_OK;
}

// The welded mesh of the current volume (see MeshArgs).
int extract_mesh(kf_session* s, float iso, uint32_t* nv_out, uint32_t* nt_out) {
  const int nx = s->cfg.nx, ny = s->cfg.ny, nz = s->cfg.nz;
  const size_t n = (size_t)nx * ny * nz;
  if (n >= (1ull << 32)) return KF_ERR_INVALID_ARGUMENT;
  const size_t words = (n + 9) / 10;
  s->mesh_valid = 0;
  int rc = ensure(s, (void**)&s->d_mesh_mask, &s->mesh_mask_cap, words * 4);
  if (rc) return rc;
  const size_t sw = std::max(kf_scan_scratch_words(n), kf_scan_scratch_words(words));
  // tri_count[n], tri_off[n], word_count[words], word_off[words], scan scratch, 2 totals
  rc = ensure(s, (void**)&s->d_mesh_scratch, &s->mesh_scratch_cap, (2 * n + 2 * words + sw + 2) * 4);
  if (rc) return rc;
  MeshArgs a;
  a.vol = s->d_vol;
  a.nx = nx; a.ny = ny; a.nz = nz;
  a.iso = iso;
  a.q13 = (s->cfg.quirks & KF_Q13_MC_FIRST_SEVEN) ? 1 : 0;
  a.mask = s->d_mesh_mask;
  a.tri_count = s->d_mesh_scratch;
  uint32_t* tri_off = a.tri_count + n;
  a.tri_off = tri_off;
  a.word_count = tri_off + n;
  uint32_t* word_off = a.word_count + words;
  a.word_off = word_off;
  uint32_t* scr = word_off + words;
  uint32_t* totals = scr + sw;
  a.dimx = s->cfg.dim_x; a.dimy = s->cfg.dim_y; a.dimz = s->cfg.dim_z;
  a.pos = nullptr; a.nrm = nullptr; a.idx = nullptr;
  KF_CUDA_TRY(s, cudaMemsetAsync(a.mask, 0, words * 4, s->stream));
  if ((rc = mesh_phase(s, a, 0, n, words))) return rc;
  mesh_popc_kernel<<<(int)((words + 255) / 256), 256, 0, s->stream>>>(a.mask, a.word_count, words);
  KF_CUDA_TRY(s, cudaGetLastError());
  kf_note_launch(s);
  if ((rc = kf_scan_u32(a.tri_count, tri_off, n, totals, s->stream, scr, sw))) return rc;
  if ((rc = kf_scan_u32(a.word_count, word_off, words, totals + 1, s->stream, scr, sw))) return rc;
  KF_CUDA_TRY(s, cudaMemcpyAsync(s->h_u32_scalar, totals, 8, cudaMemcpyDeviceToHost, s->stream));
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  const uint32_t T = s->h_u32_scalar[0], NV = s->h_u32_scalar[1];
  if ((uint64_t)T * 3 >= (1ull << 32)) return KF_ERR_CAPACITY;
  if ((rc = ensure(s, (void**)&s->d_mesh_pos, &s->mesh_pos_cap, std::max<size_t>(12, (size_t)NV * 12)))) return rc;
  if ((rc = ensure(s, (void**)&s->d_mesh_nrm, &s->mesh_nrm_cap, std::max<size_t>(12, (size_t)NV * 12)))) return rc;
  if ((rc = ensure(s, (void**)&s->d_mesh_idx, &s->mesh_idx_cap, std::max<size_t>(12, (size_t)T * 12)))) return rc;
  a.pos = s->d_mesh_pos;
  a.nrm = s->d_mesh_nrm;
  a.idx = s->d_mesh_idx;
  if (NV && (rc = mesh_phase(s, a, 1, n, words))) return rc;
  if (T && (rc = mesh_phase(s, a, 2, n, words))) return rc;
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  s->mesh_vertices = NV;
  s->mesh_triangles = T;
  s->mesh_valid = 1;
  *nv_out = NV;
  *nt_out = T;
  return KF_OK;
}

int copy_mesh_host(kf_session* s, std::vector<float>& pos, std::vector<float>& nrm, std::vector<uint32_t>& idx) {
  pos.resize((size_t)s->mesh_vertices * 3);
  nrm.resize((size_t)s->mesh_vertices * 3);
  idx.resize((size_t)s->mesh_triangles * 3);
  if (!pos.empty()) {
    KF_CUDA_TRY(s, cudaMemcpyAsync(pos.data(), s->d_mesh_pos, pos.size() * 4, cudaMemcpyDeviceToHost, s->stream));
    KF_CUDA_TRY(s, cudaMemcpyAsync(nrm.data(), s->d_mesh_nrm, nrm.size() * 4, cudaMemcpyDeviceToHost, s->stream));
  }
  if (!idx.empty())
    KF_CUDA_TRY(s, cudaMemcpyAsync(idx.data(), s->d_mesh_idx, idx.size() * 4, cudaMemcpyDeviceToHost, s->stream));
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

int kf_mc_copy_normals(kf_session* s, float* n4, uint64_t max_vertices) {
  if (!s || (!n4 && s->mc_triangles)) return KF_ERR_INVALID_ARGUMENT;
  if (!s->mc_valid) return KF_ERR_STATE;
  const uint64_t n = (uint64_t)s->mc_triangles * 3;
  if (max_vertices < n) return KF_ERR_CAPACITY;
  if (!n) return KF_OK;
  KF_CUDA_TRY(s, cudaMemcpyAsync(n4, s->d_mc_normals, n * 16, cudaMemcpyDeviceToHost, s->stream));
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

int kf_mc_extract_mesh(kf_session* s, float iso, uint32_t* n_vertices, uint32_t* n_triangles) {
  if (!s || !n_vertices || !n_triangles) return KF_ERR_INVALID_ARGUMENT;
  return extract_mesh(s, iso, n_vertices, n_triangles);
}

int kf_mc_copy_mesh(kf_session* s, float* positions3, float* normals3, uint32_t* indices3, uint64_t max_vertices,
                    uint64_t max_triangles) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  if (!s->mesh_valid) return KF_ERR_STATE;
  const uint64_t nv = s->mesh_vertices, nt = s->mesh_triangles;
  if (max_vertices < nv || max_triangles < nt) return KF_ERR_CAPACITY;
  if ((nv && (!positions3 && !normals3)) || (nt && !indices3 && !positions3 && !normals3)) return KF_ERR_INVALID_ARGUMENT;
  if (nv && positions3) KF_CUDA_TRY(s, cudaMemcpyAsync(positions3, s->d_mesh_pos, nv * 12, cudaMemcpyDeviceToHost, s->stream));
  if (nv && normals3) KF_CUDA_TRY(s, cudaMemcpyAsync(normals3, s->d_mesh_nrm, nv * 12, cudaMemcpyDeviceToHost, s->stream));
  if (nt && indices3) KF_CUDA_TRY(s, cudaMemcpyAsync(indices3, s->d_mesh_idx, nt * 12, cudaMemcpyDeviceToHost, s->stream));
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return KF_OK;
}

int kf_mc_export_mesh_ply(kf_session* s, const char* path) {
  // binary little-endian PLY: vertex x y z nx ny nz (float), face list (uchar, uint32)
  if (!s || !path) return KF_ERR_INVALID_ARGUMENT;
  if (!s->mesh_valid) return KF_ERR_STATE;
  std::vector<float> pos, nrm;
  std::vector<uint32_t> idx;
  int rc = copy_mesh_host(s, pos, nrm, idx);
  if (rc) return rc;
  FILE* f = std::fopen(path, "wb");
  if (!f) return KF_ERR_IO;
  const unsigned long long NV = s->mesh_vertices, NT = s->mesh_triangles;
  std::fprintf(f, "ply\nformat binary_little_endian 1.0\nelement vertex %llu\nproperty float x\nproperty float y\n"
               "property float z\nproperty float nx\nproperty float ny\nproperty float nz\nelement face %llu\n"
               "property list uchar uint vertex_indices\nend_header\n", NV, NT);
  std::vector<float> vrec((size_t)NV * 6);
  for (size_t i = 0; i < NV; ++i)
    for (int k = 0; k < 3; ++k) {
      vrec[i * 6 + k] = pos[i * 3 + k];
      vrec[i * 6 + 3 + k] = nrm[i * 3 + k];
    }
  bool ok = NV == 0 || std::fwrite(vrec.data(), 4, vrec.size(), f) == vrec.size();
  std::vector<unsigned char> frec((size_t)NT * 13);
  for (size_t t = 0; t < NT; ++t) {
    frec[t * 13] = 3;
    std::memcpy(&frec[t * 13 + 1], &idx[t * 3], 12);
  }
  ok = ok && (NT == 0 || std::fwrite(frec.data(), 1, frec.size(), f) == frec.size());
  ok = (std::fclose(f) == 0) && ok;
  return ok ? KF_OK : KF_ERR_IO;
}

int kf_mc_export_mesh_stl(kf_session* s, const char* path) {
  // binary STL of the welded mesh: zeroed 80-byte header, the triangle count, per triangle
  // its unit facet normal (from the vertex positions, counter-clockwise), three vertices
  if (!s || !path) return KF_ERR_INVALID_ARGUMENT;
  if (!s->mesh_valid) return KF_ERR_STATE;
  std::vector<float> pos, nrm;
  std::vector<uint32_t> idx;
  int rc = copy_mesh_host(s, pos, nrm, idx);
  if (rc) return rc;
  FILE* f = std::fopen(path, "wb");
  if (!f) return KF_ERR_IO;
  char hdr[80];
  std::memset(hdr, 0, sizeof(hdr));
  const uint32_t T = s->mesh_triangles;
  bool ok = std::fwrite(hdr, 1, 80, f) == 80 && std::fwrite(&T, 4, 1, f) == 1;
  std::vector<unsigned char> rec((size_t)T * 50);
  const uint16_t attr = 0;
  for (uint32_t t = 0; t < T; ++t) {
    const float* p0 = &pos[(size_t)idx[3 * t] * 3];
    const float* p1 = &pos[(size_t)idx[3 * t + 1] * 3];
    const float* p2 = &pos[(size_t)idx[3 * t + 2] * 3];
    const float ux = p1[0] - p0[0], uy = p1[1] - p0[1], uz = p1[2] - p0[2];
    const float vx = p2[0] - p0[0], vy = p2[1] - p0[1], vz = p2[2] - p0[2];
    float nv[3] = {uy * vz - uz * vy, uz * vx - ux * vz, ux * vy - uy * vx};
    const float len = std::sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
    for (float& c : nv) c = len > 0.0f ? c / len : 0.0f;
    unsigned char* r = &rec[(size_t)t * 50];
    std::memcpy(r, nv, 12);
    std::memcpy(r + 12, p0, 12);
    std::memcpy(r + 24, p1, 12);
    std::memcpy(r + 36, p2, 12);
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
