// kf_scan.cu — exclusive prefix sum of uint32 (reduce-then-scan, any length).
//
// Reference: shaders/prefixSum.cs:28-197 (Blelloch work-efficient scan, 2048 elements
// per work group, one level of group sums, so n <= 2048 * 2048 = 4,194,304 (Q17)) driven
// by MCubes::prefixSum (src/mcubes.cpp:136-204), which returns the total as lastElement +
// lastScanElement.  Same result (exclusive scan, uint32 wrap-around, total = sum of the
// input) for any n < 2^32.
//
// B200 design: tiles of 4096 elements per 256-thread block; a tile is staged through
// shared memory so global loads and stores stay coalesced while every thread scans 16
// consecutive elements in registers, then warp shuffles and one shared-memory pass scan
// the 256 thread totals.  Tile totals go to a scratch array that is scanned by the same
// code recursively (4096^2 = 16.7M elements per level), then added back.  There is no
// inter-block waiting.
#include <cuda.h>

#include <mutex>

#include "kf_internal.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;  // 4096

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread; returns the exclusive prefix and
// the block total in *total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_warp, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t inc = warp_incl_scan(v, lane);
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kThreads / 32 ? s_warp[lane] : 0u;
    const uint32_t wi = warp_incl_scan(w, lane);
    if (lane < kThreads / 32) s_warp[lane] = wi - w;  // exclusive warp offsets
    if (lane == kThreads / 32 - 1) s_warp[kThreads / 32] = wi;
  }
  __syncthreads();
  const uint32_t r = s_warp[warp] + inc - v;
  *total = s_warp[kThreads / 32];
  __syncthreads();
  return r;
}

// Per-tile totals.
__global__ void __launch_bounds__(kThreads) tile_sum_kernel(const uint32_t* __restrict__ in, uint64_t n,
                                                            uint32_t* __restrict__ sums) {
  __shared__ uint32_t s_warp[kThreads / 32 + 1];
  const uint64_t base = (uint64_t)blockIdx.x * kTile;
  uint32_t v = 0;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const uint64_t i = base + (uint64_t)k * kThreads + threadIdx.x;
    if (i < n) v += __ldg(in + i);
  }
  uint32_t total;
  block_excl_scan(v, s_warp, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// Exclusive scan of each tile plus its tile offset (offsets == nullptr: none).
// `in` may equal `out` (the tile totals are scanned in place): each block reads its whole
// tile into shared memory before the barrier and writes it after, and `in` is read with
// ordinary loads (no restrict, no read-only cache path).
__global__ void __launch_bounds__(kThreads) tile_scan_kernel(const uint32_t* in, uint32_t* out,
                                                             uint64_t n, const uint32_t* __restrict__ offsets,
                                                             uint32_t* total_out) {
  __shared__ uint32_t s_tile[kTile + kTile / 32];  // padded against bank conflicts
  __shared__ uint32_t s_warp[kThreads / 32 + 1];
  const uint64_t base = (uint64_t)blockIdx.x * kTile;
  auto pad = [](int j) { return j + (j >> 5); };
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const int j = k * kThreads + threadIdx.x;
    const uint64_t i = base + (uint64_t)j;
    s_tile[pad(j)] = i < n ? in[i] : 0u;
  }
  __syncthreads();
  uint32_t x[kItems];
  uint32_t run = 0;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    x[k] = s_tile[pad(threadIdx.x * kItems + k)];
    const uint32_t t = x[k];
    x[k] = run;
    run += t;
  }
  uint32_t total;
  const uint32_t pre = block_excl_scan(run, s_warp, &total);
  const uint32_t off = (offsets ? offsets[blockIdx.x] : 0u) + pre;
#pragma unroll
  for (int k = 0; k < kItems; ++k) s_tile[pad(threadIdx.x * kItems + k)] = x[k] + off;
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const int j = k * kThreads + threadIdx.x;
    const uint64_t i = base + (uint64_t)j;
    if (i < n) out[i] = s_tile[pad(j)];
  }
  if (total_out && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0)
    *total_out = (offsets ? offsets[blockIdx.x] : 0u) + total;
}

__global__ void zero_word(uint32_t* p) { *p = 0u; }

uint64_t tiles(uint64_t n) { return (n + kTile - 1) / kTile; }

int scan_rec(const uint32_t* d_in, uint32_t* d_out, uint64_t n, uint32_t* d_total, cudaStream_t st,
             uint32_t* scratch, size_t words) {
  const uint64_t nt = tiles(n);
  if (nt <= 1) {
    tile_scan_kernel<<<1, kThreads, 0, st>>>(d_in, d_out, n, nullptr, d_total);
    return cudaGetLastError() == cudaSuccess ? KF_OK : KF_ERR_CUDA;
  }
  if (nt > words) return KF_ERR_CAPACITY;
  uint32_t* sums = scratch;
  tile_sum_kernel<<<(unsigned)nt, kThreads, 0, st>>>(d_in, n, sums);
  if (cudaGetLastError() != cudaSuccess) return KF_ERR_CUDA;
  // exclusive scan of the tile totals in place; the grand total lands in d_total
  int rc = scan_rec(sums, sums, nt, d_total, st, scratch + nt, words - nt);
  if (rc) return rc;
  tile_scan_kernel<<<(unsigned)nt, kThreads, 0, st>>>(d_in, d_out, n, sums, nullptr);
  return cudaGetLastError() == cudaSuccess ? KF_OK : KF_ERR_CUDA;
}

}  // namespace

size_t kf_scan_scratch_words(uint64_t n) {
  size_t w = 0;
  uint64_t m = tiles(n);
  while (m > 1) {
    w += m;
    m = tiles(m);
  }
  return w + 1;
}

int kf_scan_u32(const uint32_t* d_in, uint32_t* d_out, uint64_t n, uint32_t* d_total, cudaStream_t stream,
                uint32_t* d_scratch, size_t scratch_words) {
  if (n == 0) {
    if (d_total) zero_word<<<1, 1, 0, stream>>>(d_total);
    return cudaGetLastError() == cudaSuccess ? KF_OK : KF_ERR_CUDA;
  }
  if (!d_total) return KF_ERR_INVALID_ARGUMENT;
  return scan_rec(d_in, d_out, n, d_total, stream, d_scratch, scratch_words);
}

extern "C" int kf_prefix_sum_u32(const uint32_t* d_in, uint32_t* d_out, uint64_t n, uint32_t* total,
                                 void* cuda_stream) {
  if ((!d_in || !d_out) && n) return KF_ERR_INVALID_ARGUMENT;
  if (n >= (1ull << 32)) return KF_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)cuda_stream;
  const size_t words = kf_scan_scratch_words(n);
  uint32_t* scratch = nullptr;
  if (cudaMallocAsync((void**)&scratch, (words + 1) * sizeof(uint32_t), st) != cudaSuccess) {
    cudaGetLastError();
    return KF_ERR_OUT_OF_MEMORY;
  }
  uint32_t* d_total = scratch + words;
  int rc = kf_scan_u32(d_in, d_out, n, d_total, st, scratch, words);
  uint32_t h = 0;
  if (!rc && total) {
    if (cudaMemcpyAsync(&h, d_total, sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess) rc = KF_ERR_CUDA;
  }
  cudaFreeAsync(scratch, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) rc = KF_ERR_CUDA;
  if (!rc && total) *total = h;
  return rc;
}

// ---- allocation-free variant -----------------------------------------------------------
// Scratch for kf_prefix_sum_u32_noalloc: the tile totals of every scan level plus one
// word for the grand total, for inputs of up to KF_NOALLOC_SCAN_MAX_ELEMENTS elements
// (2^28 elements need 65,536 + 16 tile totals + 1 spare + 1 grand total = 65,554 words;
// the array holds 65,555 words, 262,220 bytes).
// Every GPU that loads this library holds the array until the process exits.
#define KF_NOALLOC_SCAN_MAX_ELEMENTS (1ull << 28)
#define KF_NOALLOC_SCAN_WORDS 65555
static __device__ __align__(256) uint32_t g_noalloc_scan_scratch[KF_NOALLOC_SCAN_WORDS];

namespace {
std::mutex g_noalloc_mu;
// The array's device address per CUDA context, keyed by the context's process-unique id
// (cuCtxGetId): a context created later (a new primary context after cudaDeviceReset, or a
// context a host framework made with cuCtxCreate) never reuses an entry of an earlier one.
struct NoallocEntry {
  unsigned long long ctx_id;
  uint32_t* ptr;
};
constexpr size_t kNoallocMaxEntries = 64;
std::vector<NoallocEntry> g_noalloc_cache;
typedef CUresult (*PFN_ctx_get_current)(CUcontext*);
typedef CUresult (*PFN_ctx_get_id)(CUcontext, unsigned long long*);
PFN_ctx_get_current g_ctx_get_current = nullptr;
PFN_ctx_get_id g_ctx_get_id = nullptr;

// The current context's id through the driver entry points (the library links only the
// CUDA runtime); false when there is no current context.
bool current_ctx_id(unsigned long long* id) {
  if (!g_ctx_get_current || !g_ctx_get_id) {
    void* f0 = nullptr;
    void* f1 = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault) != cudaSuccess || !f0 || !f1) {
      cudaGetLastError();
      return false;
    }
    g_ctx_get_current = reinterpret_cast<PFN_ctx_get_current>(f0);
    g_ctx_get_id = reinterpret_cast<PFN_ctx_get_id>(f1);
  }
  CUcontext ctx = nullptr;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
  return g_ctx_get_id(ctx, id) == CUDA_SUCCESS;
}
}  // namespace

// In host code g_noalloc_scan_scratch only names the symbol; its device address is looked
// up with cudaGetSymbolAddress once per CUDA context (the first call in a context, which
// also makes the runtime's primary context current when none is) and cached by context id.
static int noalloc_scratch(uint32_t** out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  unsigned long long id = 0;
  bool have_id = current_ctx_id(&id);
  if (have_id) {
    for (const NoallocEntry& e : g_noalloc_cache)
      if (e.ctx_id == id) {
        *out = e.ptr;
        return KF_OK;
      }
  }
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scan_scratch);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    return e == cudaErrorNoDevice ? KF_ERR_NO_DEVICE : KF_ERR_CUDA;
  }
  if (!have_id) have_id = current_ctx_id(&id);  // the lookup initialised the primary context
  if (have_id) {
    if (g_noalloc_cache.size() >= kNoallocMaxEntries) g_noalloc_cache.erase(g_noalloc_cache.begin());
    g_noalloc_cache.push_back(NoallocEntry{id, static_cast<uint32_t*>(p)});
  }
  *out = static_cast<uint32_t*>(p);
  return KF_OK;
}

extern "C" int kf_prefix_sum_u32_noalloc(const uint32_t* d_in, uint32_t* d_out, uint64_t n, uint32_t* total,
                                         void* cuda_stream) {
  if ((!d_in || !d_out) && n) return KF_ERR_INVALID_ARGUMENT;
  if (n > KF_NOALLOC_SCAN_MAX_ELEMENTS) return KF_ERR_CAPACITY;
  const size_t words = kf_scan_scratch_words(n);
  if (words + 1 > KF_NOALLOC_SCAN_WORDS) return KF_ERR_CAPACITY;
  uint32_t* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)cuda_stream;
  // nothing in the scratch has to start at zero: every tile total and the grand total are
  // written before they are read
  uint32_t* d_total = scratch + words;
  rc = kf_scan_u32(d_in, d_out, n, d_total, st, scratch, words);
  if (rc || !total) return rc;
  uint32_t h = 0;
  if (cudaMemcpyAsync(&h, d_total, sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    cudaGetLastError();
    return KF_ERR_CUDA;
  }
  *total = h;
  return KF_OK;
}
