// kf_capi.cu — the C ABI (include/kf.h): sessions, state hand-off, frame step, accessors.
//
// Reference: the public members of class gFusion (include/gFusion.h:134-274) and the
// per-frame loop of src/kinect.cpp:654-695.  A session owns its CUDA stream, its device
// buffers and a device control block (KfDevState) that holds the FP64 pose, the pose
// library and the frame-policy flags, so a whole frame runs without a host round trip.
// The first kf_frame_step_* call captures the device part of a frame into a CUDA graph;
// later calls replay it.
#include <algorithm>
#include <array>
#include <cstdio>
#include <map>
#include <mutex>
#include <new>

#include <atomic>

#include "kf_internal.cuh"

namespace {

const double kIdentity[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};

int fail(kf_session* s, int code, const std::string& msg) {
  if (s) s->last_error = msg;
  return code;
}

template <class T>
int dalloc(kf_session* s, T** p, size_t count) {
  *p = nullptr;
  if (count == 0) return KF_OK;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(s, e == cudaErrorMemoryAllocation ? KF_ERR_OUT_OF_MEMORY : KF_ERR_CUDA,
                std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  return KF_OK;
}

int validate(const kf_config* c, const kf_intrinsics* in) {
  if (!c || !in) return KF_ERR_INVALID_ARGUMENT;
  if (c->nx < 4 || c->ny < 4 || c->nz < 4 || c->nx > 4096 || c->ny > 4096 || c->nz > 4096)
    return KF_ERR_INVALID_ARGUMENT;
  // kernels index a volume plane with 32-bit offsets
  if ((uint64_t)c->nx * (uint64_t)c->ny * (uint64_t)c->nz >= (1ull << 31)) return KF_ERR_INVALID_ARGUMENT;
  if (!(c->dim_x > 0) || !(c->dim_y > 0) || !(c->dim_z > 0) || !(c->mu > 0)) return KF_ERR_INVALID_ARGUMENT;
  if (!(c->max_weight > 0) || !(c->far_plane > c->near_plane)) return KF_ERR_INVALID_ARGUMENT;
  if (c->storage < KF_STORAGE_F32F32 || c->storage > KF_STORAGE_RG16I) return KF_ERR_INVALID_ARGUMENT;
  if (c->jtj != KF_JTJ_FP32 && c->jtj != KF_JTJ_SPLIT_BF16) return KF_ERR_INVALID_ARGUMENT;
  if (c->tracking != KF_TRACK_ICP && c->tracking != KF_TRACK_SDF) return KF_ERR_INVALID_ARGUMENT;
  for (int l = 0; l < 3; ++l)
    if (c->iterations[l] < 0 || c->iterations[l] > 1000) return KF_ERR_INVALID_ARGUMENT;
  if (c->storage == KF_STORAGE_F16U16 && c->max_weight > 65535.0f) return KF_ERR_INVALID_ARGUMENT;
  if (c->storage == KF_STORAGE_RG16I && c->max_weight > 32767.0f) return KF_ERR_INVALID_ARGUMENT;
  // three mip levels of exact halves
  if (in->width < 16 || in->height < 16 || (in->width % 4) || (in->height % 4)) return KF_ERR_INVALID_ARGUMENT;
  if (in->width > 8192 || in->height > 8192) return KF_ERR_INVALID_ARGUMENT;
  if (!(in->fx > 0) || !(in->fy > 0)) return KF_ERR_INVALID_ARGUMENT;
  return KF_OK;
}

size_t value_bytes(int storage) { return storage == KF_STORAGE_F32F32 ? 4 : 2; }

void free_mc(kf_session* s) {
  cudaFree(s->d_mc_base);
  s->d_mc_base = nullptr;
  for (uint32_t* p : s->d_mc_levels) cudaFree(p);
  s->d_mc_levels.clear();
  s->mc_P = 0;
  s->mc_top = 0;
  cudaFree(s->d_mc_vertices);
  s->d_mc_vertices = nullptr;
  s->mc_vertex_cap = 0;
  cudaFree(s->d_mc_scratch);
  s->d_mc_scratch = nullptr;
  s->mc_scratch_words = 0;
  cudaFree(s->d_mc_normals);
  s->d_mc_normals = nullptr;
  s->mc_normal_cap = 0;
  s->mc_valid = 0;
  s->mc_triangles = 0;
  cudaFree(s->d_mesh_mask);
  cudaFree(s->d_mesh_scratch);
  cudaFree(s->d_mesh_pos);
  cudaFree(s->d_mesh_nrm);
  cudaFree(s->d_mesh_idx);
  s->d_mesh_mask = s->d_mesh_scratch = s->d_mesh_idx = nullptr;
  s->d_mesh_pos = s->d_mesh_nrm = nullptr;
  s->mesh_mask_cap = s->mesh_scratch_cap = s->mesh_pos_cap = s->mesh_nrm_cap = s->mesh_idx_cap = 0;
  s->mesh_vertices = s->mesh_triangles = 0;
  s->mesh_valid = 0;
}

void drop_graph(kf_session* s) {
  for (int r = 0; r < kf_session::kRing; ++r) {
    if (s->frame_exec[r]) cudaGraphExecDestroy(s->frame_exec[r]);
    s->frame_exec[r] = nullptr;
    s->ring_pending[r] = 0;
  }
}

void free_all(kf_session* s) {
  if (s->stream) cudaStreamSynchronize(s->stream);
  drop_graph(s);
  free_mc(s);
  cudaFree(s->d_vol);
  cudaFree(s->d_bricks);
  cudaFree(s->d_depth_u16);
  cudaFree(s->d_depth_f32_in);
  for (int l = 0; l < 3; ++l) {
    cudaFree(s->d_depth[l]);
    cudaFree(s->d_vertex[l]);
    cudaFree(s->d_normal[l]);
    cudaFree(s->d_status[l]);
  }
  cudaFree(s->d_ref_vertex);
  cudaFree(s->d_ref_normal);
  cudaFree(s->d_sdf_rows);
  cudaFree(s->d_partials);
  cudaFree(s->d_state);
  cudaFree(s->d_u32_scalar);
  cudaFree(s->d_mip);
  cudaFree(s->d_undistort_map);
  cudaFree(s->d_depth_prep);
  if (s->h_heads) cudaFreeHost(s->h_heads);
  for (auto& e : s->head_ev)
    if (e) cudaEventDestroy(e);
  if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
  cudaFree(s->d_frame_ring);
  for (auto& e : s->upload_ev)
    if (e) cudaEventDestroy(e);
  if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
  if (s->h_state) cudaFreeHost(s->h_state);
  if (s->h_depth_pinned) cudaFreeHost(s->h_depth_pinned);
  if (s->h_u32_scalar) cudaFreeHost(s->h_u32_scalar);
  for (auto& e : s->ev)
    if (e) cudaEventDestroy(e);
  for (auto& row : s->ring_ev)
    for (auto& e : row)
      if (e) cudaEventDestroy(e);
  if (s->stream) cudaStreamDestroy(s->stream);
}

// ---- host <-> device control block ------------------------------------------------------
int check_device_error(kf_session* s) {
  if (s->h_state->error) {
    const int err = s->h_state->error;
    s->h_state->error = 0;
    cudaMemsetAsync(&s->d_state->error, 0, sizeof(int), s->stream);
    cudaStreamSynchronize(s->stream);
    return fail(s, KF_ERR_TIMEOUT, "device wait timed out (error " + std::to_string(err) + ")");
  }
  return KF_OK;
}

// Reads the result of the pending asynchronous frame step (waits for that step only) into
// the host mirror, as a synchronous step would have.
int finish_async(kf_session* s) {
  const int p = s->async_pend;
  if (p < 0) return KF_OK;
  s->async_pend = -1;
  KF_CUDA_TRY(s, cudaEventSynchronize(s->head_ev[p]));
  std::memcpy(s->h_state, s->h_heads + (size_t)p * KF_STATE_RESULT_BYTES, KF_STATE_RESULT_BYTES);
  return check_device_error(s);
}

int pull_state(kf_session* s) {
  if (int rc = finish_async(s)) return rc;
  KF_CUDA_TRY(s, cudaMemcpyAsync(s->h_state, s->d_state, sizeof(KfDevState), cudaMemcpyDeviceToHost, s->stream));
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return check_device_error(s);
}

// pose and result flags only (the per-frame result)
int pull_state_head(kf_session* s) {
  if (int rc = finish_async(s)) return rc;
  KF_CUDA_TRY(s, cudaMemcpyAsync(s->h_state, s->d_state, KF_STATE_RESULT_BYTES, cudaMemcpyDeviceToHost, s->stream));
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return check_device_error(s);
}

int push_state(kf_session* s) {
  KF_CUDA_TRY(s, cudaMemcpyAsync(s->d_state, s->h_state, sizeof(KfDevState), cudaMemcpyHostToDevice, s->stream));
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return KF_OK;
}

void set_pose_fields(kf_session* s, const double* pose, bool reset_eig) {
  kf_store_pose(s->h_state, pose);
  if (reset_eig) {
    // resetPose (gFusion.cpp:275-287)
    if (s->cfg.quirks & KF_Q19_EIG_TRANSLATION) {
      std::memcpy(s->h_state->pose_eig, kIdentity, sizeof(kIdentity));
      s->h_state->pose_eig[12] = pose[12];
      s->h_state->pose_eig[13] = pose[13];
      s->h_state->pose_eig[14] = pose[14];
    } else {
      std::memcpy(s->h_state->pose_eig, pose, 16 * sizeof(double));
    }
    for (int k = 0; k < 6; ++k) s->h_state->cum_twist[k] = 0;
  }
}

int alloc_volume(kf_session* s) {
  s->layout += 1;
  cudaFree(s->d_vol);
  s->d_vol = nullptr;
  cudaFree(s->d_bricks);
  s->d_bricks = s->d_supers = nullptr;
  s->bx = (s->cfg.nx + KF_BRICK - 1) / KF_BRICK;
  s->by = (s->cfg.ny + KF_BRICK - 1) / KF_BRICK;
  s->bz = (s->cfg.nz + KF_BRICK - 1) / KF_BRICK;
  s->sbx = (s->cfg.nx + KF_SUPER - 1) / KF_SUPER;
  s->sby = (s->cfg.ny + KF_SUPER - 1) / KF_SUPER;
  s->sbz = (s->cfg.nz + KF_SUPER - 1) / KF_SUPER;
  {
    const size_t nb = (size_t)s->bx * s->by * s->bz, ns = (size_t)s->sbx * s->sby * s->sbz;
    int rc = dalloc(s, &s->d_bricks, nb + ns);
    if (rc) return rc;
    s->d_supers = s->d_bricks + nb;
    if ((rc = kf_reset_bricks(s))) return rc;
  }
  s->vol_count = (size_t)s->cfg.nx * s->cfg.ny * s->cfg.nz;
  s->vol_value_bytes = value_bytes(s->cfg.storage);
  s->vol_bytes = s->vol_count * s->vol_value_bytes * 2;
  char* p = nullptr;
  int rc = dalloc(s, &p, s->vol_bytes);
  if (rc) return rc;
  s->d_vol = p;
  KF_CUDA_TRY(s, cudaMemsetAsync(s->d_vol, 0, s->vol_bytes, s->stream));
  return KF_OK;
}

int record(kf_session* s, int i) {
  if (!s->timing || s->capturing) return KF_OK;
  KF_CUDA_TRY(s, cudaEventRecord(s->ev[i], s->stream));
  return KF_OK;
}

// The input frame of ring slot `slot` (the frame graph of that slot reads it).
uint16_t* slot_frame(kf_session* s, int slot) {
  return s->d_frame_ring + (size_t)slot * s->W[0] * s->H[0];
}

// The device part of one frame of kinect.cpp:654-695 (input already in the slot's frame),
// with events ev[0..5]: start, pyramid, track, integrate, recover, raycast (event record
// nodes in the captured graph, so they can be timed after every replay) when `stages`;
// otherwise the graph holds no event node and run_frame records the frame's end after it.
int enqueue_frame(kf_session* s, cudaEvent_t* ev, int slot, bool stages) {
  int rc;
  auto boundary = [&](int k) {
    return stages ? cudaEventRecordWithFlags(ev[k], s->stream, cudaEventRecordExternal) : cudaSuccess;
  };
  KF_CUDA_TRY(s, boundary(0));
  if ((rc = kf_launch_depth_ingest(s, slot_frame(s, slot), nullptr))) return rc;
  // the vertex/normal launch also zeroes the tracking launches' barrier counters and ICP
  // sums (3.5 us per frame less than two memset nodes); in ICP mode nothing else touches the
  // SDF counter before the recover launch, in SDF mode the tracking launch does
  if ((rc = kf_launch_vertex_normal(s, true))) return rc;
  KF_CUDA_TRY(s, boundary(1));
  const bool sdf_mode = s->cfg.tracking == KF_TRACK_SDF;
  if (sdf_mode) {
    if ((rc = kf_launch_sdf(s, 0, 0, 1, true))) return rc;
    if ((rc = kf_launch_sdf_policy(s))) return rc;
  } else {
    if ((rc = kf_launch_icp(s, 1, true))) return rc;
  }
  KF_CUDA_TRY(s, boundary(2));
  if ((rc = kf_launch_integrate(s, 1))) return rc;
  KF_CUDA_TRY(s, boundary(3));
  if ((rc = kf_launch_sdf(s, 1, 1, 0, !sdf_mode))) return rc;
  KF_CUDA_TRY(s, boundary(4));
  if ((rc = kf_launch_raycast(s))) return rc;
  KF_CUDA_TRY(s, boundary(5));
  return KF_OK;
}

int count_kernels(cudaGraph_t g) {
  size_t n = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return 0;
  std::vector<cudaGraphNode_t> nodes(n);
  if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return 0;
  int k = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
  }
  return k;
}

// Read back the stage times of the frame held by a ring slot (waits for that frame only).
int harvest(kf_session* s, int slot) {
  if (!s->ring_pending[slot]) return KF_OK;
  KF_CUDA_TRY(s, cudaEventSynchronize(s->ring_ev[slot][5]));
  if (s->ring_stages[slot]) {
    for (int i = 0; i < 5; ++i) {
      float ms = 0.0f;
      KF_CUDA_TRY(s, cudaEventElapsedTime(&ms, s->ring_ev[slot][i], s->ring_ev[slot][i + 1]));
      s->stage_ms[i] = ms;
      s->stage_acc[i] += ms;
    }
    s->stage_frames += 1;
  }
  s->ring_pending[slot] = 0;
  return KF_OK;
}

int harvest_all(kf_session* s) {
  // oldest first, so stage_ms ends as the newest frame
  for (int k = 0; k < kf_session::kRing; ++k) {
    const int slot = (int)((s->frames_run + k) % kf_session::kRing);
    int rc = harvest(s, slot);
    if (rc) return rc;
  }
  return KF_OK;
}

int run_frame(kf_session* s) {
  const int slot = (int)(s->frames_run % kf_session::kRing);
  if (!s->frame_exec[slot]) {
    for (int i = 0; i < 6; ++i)
      if (!s->ring_ev[slot][i]) KF_CUDA_TRY(s, cudaEventCreate(&s->ring_ev[slot][i]));
    cudaGraph_t g = nullptr;
    KF_CUDA_TRY(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    s->capturing = true;
    const bool stages = s->stage_every > 0 && slot % s->stage_every == 0;
    int rc = enqueue_frame(s, s->ring_ev[slot], slot, stages);
    s->capturing = false;
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return fail(s, KF_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
    s->frame_kernels = count_kernels(g);
    s->ring_stages[slot] = stages ? 1 : 0;
    e = cudaGraphInstantiate(&s->frame_exec[slot], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      s->frame_exec[slot] = nullptr;
      return fail(s, KF_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
    }
  }
  int rc = harvest(s, slot);  // the frame that used this slot kRing frames ago
  if (rc) return rc;
  KF_CUDA_TRY(s, cudaGraphLaunch(s->frame_exec[slot], s->stream));
  // an untimed frame's end, recorded on the stream outside its graph
  if (!s->ring_stages[slot]) KF_CUDA_TRY(s, cudaEventRecord(s->ring_ev[slot][5], s->stream));
  if ((rc = kf_note_integrate(s, s->stream))) return rc;
  s->ring_pending[slot] = 1;
  s->frames_run += 1;
  s->launches += (uint64_t)s->frame_kernels;
  return KF_OK;
}

int finish_step(kf_session* s, int* tracked) {
  if (!tracked) return KF_OK;
  int rc = pull_state_head(s);
  if (rc) return rc;
  *tracked = s->h_state->tracked;
  return KF_OK;
}

std::mutex g_occ_mu;
std::map<std::pair<const void*, int>, int> g_occ;

// tuned launch shapes by (device, nx, ny, nz, storage, width, height)
typedef std::array<int, 7> TuneKey;
std::mutex g_tune_mu;
std::map<TuneKey, std::pair<int, int>> g_tune;

TuneKey tune_key(const kf_session* s) {
  return TuneKey{s->device, s->cfg.nx, s->cfg.ny, s->cfg.nz, s->cfg.storage, s->intr.width, s->intr.height};
}

void tune_cache_apply(kf_session* s) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(tune_key(s));
  if (it == g_tune.end()) return;
  s->int_zc = it->second.first;
  s->ray_rows = it->second.second;
}

}  // namespace

void kf_tune_cache_put(const kf_session* s, int zc, int rows) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[tune_key(s)] = std::make_pair(zc, rows);
}

void kf_scratch_free(kf_scratch_target* t) {
  cudaFree(t->vol);
  cudaFree(t->bricks);
  cudaFree(t->out_v);
  cudaFree(t->st_out);
  *t = kf_scratch_target{};
}

int kf_scratch_alloc(kf_session* s, kf_scratch_target* t) {
  *t = kf_scratch_target{};
  const size_t px = (size_t)s->W[0] * s->H[0];
  const size_t nflags = (size_t)s->bx * s->by * s->bz + (size_t)s->sbx * s->sby * s->sbz;
  int rc = KF_OK;
  char* vol = nullptr;
  float4* maps = nullptr;
  if ((rc = dalloc(s, &vol, s->vol_bytes)) || (rc = dalloc(s, &t->bricks, nflags)) || (rc = dalloc(s, &maps, 2 * px)) ||
      (rc = dalloc(s, &t->st_out, 1))) {
    t->vol = vol;
    t->out_v = maps;
    kf_scratch_free(t);
    return rc;
  }
  t->vol = vol;
  t->supers = t->bricks + (size_t)s->bx * s->by * s->bz;
  t->out_v = maps;
  t->out_n = maps + px;
  KF_CUDA_TRY(s, cudaMemcpyAsync(t->vol, s->d_vol, s->vol_bytes, cudaMemcpyDeviceToDevice, s->stream));
  KF_CUDA_TRY(s, cudaMemcpyAsync(t->bricks, s->d_bricks, nflags * 4, cudaMemcpyDeviceToDevice, s->stream));
  KF_CUDA_TRY(s, cudaMemcpyAsync(t->st_out, s->d_state, sizeof(KfDevState), cudaMemcpyDeviceToDevice, s->stream));
  return KF_OK;
}

// SDF tracking in the frame step: TrackSDF's result drives the same policy flags as ICP.
__global__ void kf_sdf_policy_kernel(KfDevState* st, int every) {
  const int tracked = st->tracked;
  every = every > 0 ? every : 1;
  const int integ = (tracked && (st->counter % every) == 0) || st->reset_window;
  st->do_integrate = integ;
  if (integ && st->counter > 2) st->reset_window = 0;
  st->need_recover = !tracked;
  st->counter += 1;
}

int kf_launch_sdf_policy(kf_session* s) {
  kf_sdf_policy_kernel<<<1, 1, 0, s->stream>>>(s->d_state, s->cfg.integrate_every);
  KF_CUDA_TRY(s, cudaGetLastError());
  kf_note_launch(s);
  return KF_OK;
}

int kf_occupancy_blocks(kf_session* s, const void* kernel, int threads, size_t smem, int max_per_sm) {
  std::lock_guard<std::mutex> lk(g_occ_mu);
  auto key = std::make_pair(kernel, s->device);
  auto it = g_occ.find(key);
  int per_sm;
  if (it != g_occ.end()) {
    per_sm = it->second;
  } else {
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    if (e != cudaSuccess || per_sm <= 0) {
      s->last_error = std::string("occupancy: ") + cudaGetErrorString(e);
      return 0;
    }
    g_occ[key] = per_sm;
  }
  // the tracking kernels: two co-resident blocks per SM, enough warps to hide the gather
  // latency, few enough partial rows for the single-block FP64 reduction
  const int blocks = std::min(per_sm, max_per_sm) * s->num_sms;
  return max_per_sm == 2 ? std::min(blocks, KF_MAX_TRACK_BLOCKS) : blocks;
}

// =========================================================================================
extern "C" {

int kf_abi_version(void) { return KF_ABI_VERSION; }

const char* kf_status_string(int st) {
  switch (st) {
    case KF_OK: return "ok";
    case KF_ERR_INVALID_ARGUMENT: return "invalid argument";
    case KF_ERR_OUT_OF_MEMORY: return "out of device memory";
    case KF_ERR_CUDA: return "CUDA error";
    case KF_ERR_NO_DEVICE: return "no CUDA device";
    case KF_ERR_TIMEOUT: return "device wait timed out";
    case KF_ERR_STATE: return "call out of order";
    case KF_ERR_IO: return "file error";
    case KF_ERR_CAPACITY: return "capacity exceeded";
    case KF_ERR_ADMISSION: return "admission refused";
    default: return "unknown status";
  }
}

int kf_config_default(kf_config* c) {
  if (!c) return KF_ERR_INVALID_ARGUMENT;
  std::memset(c, 0, sizeof(*c));
  // gFusionConfig() (gFusion.h:56-69)
  c->nx = c->ny = c->nz = 256;
  c->dim_x = c->dim_y = c->dim_z = 1.0f;
  c->mu = 0.05f;
  c->max_weight = 100.0f;
  c->near_plane = 0.1f;
  c->far_plane = 3.0f;
  c->dist_threshold = 0.05f;
  c->normal_threshold = 0.8f;
  c->iterations[0] = c->iterations[1] = c->iterations[2] = 5;
  c->storage = KF_STORAGE_F32F32;
  c->jtj = KF_JTJ_FP32;
  c->tracking = KF_TRACK_ICP;
  c->quirks = KF_QUIRKS_DEFAULT;
  c->integrate_every = 1;
  return KF_OK;
}

int kf_session_device_bytes(const kf_config* cfg, const kf_intrinsics* in, uint64_t* bytes) {
  int rc = validate(cfg, in);
  if (rc) return rc;
  if (!bytes) return KF_ERR_INVALID_ARGUMENT;
  const uint64_t vox = (uint64_t)cfg->nx * cfg->ny * cfg->nz;
  const uint64_t px = (uint64_t)in->width * in->height;
  uint64_t b = vox * value_bytes(cfg->storage) * 2;
  b += (uint64_t)((cfg->nx + KF_BRICK - 1) / KF_BRICK) * ((cfg->ny + KF_BRICK - 1) / KF_BRICK) *
       ((cfg->nz + KF_BRICK - 1) / KF_BRICK) * 4 +
       (uint64_t)((cfg->nx + KF_SUPER - 1) / KF_SUPER) * ((cfg->ny + KF_SUPER - 1) / KF_SUPER) *
       ((cfg->nz + KF_SUPER - 1) / KF_SUPER) * 4;  // brick and super-brick flags
  b += px * (2 + 4) + px * 2 * kf_session::kRing;  // staging, and the frame graphs' inputs
  b += px * (4 + 16 + 16 + 4) * 2;         // three levels (sum < 4/3 of level 0)
  b += px * 32;                            // raycast maps
  b += px * 32;                            // sdf rows
  b += (uint64_t)2 * KF_MAX_TRACK_BLOCKS * 32 * 4 + sizeof(KfDevState);
  *bytes = b;
  return KF_OK;
}

int kf_create(const kf_config* cfg, const kf_intrinsics* intr, kf_session** out) {
  if (!out) return KF_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int rc = validate(cfg, intr);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return KF_ERR_NO_DEVICE;
  }
  kf_session* s = new (std::nothrow) kf_session();
  if (!s) return KF_ERR_OUT_OF_MEMORY;
  static std::atomic<uint64_t> next_uid{1};
  s->uid = next_uid.fetch_add(1);
  s->cfg = *cfg;
  if (s->cfg.integrate_every <= 0) s->cfg.integrate_every = 1;
  s->intr = *intr;
  cudaGetDevice(&s->device);
  cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device);
  tune_cache_apply(s);
  auto bail = [&](int code) {
    free_all(s);
    delete s;
    return code;
  };
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(KF_ERR_CUDA);
  for (auto& e : s->ev)
    if (cudaEventCreate(&e) != cudaSuccess) return bail(KF_ERR_CUDA);
  s->timing = true;
  for (int l = 0; l < 3; ++l) {
    s->W[l] = intr->width >> l;
    s->H[l] = intr->height >> l;
  }
  const size_t px = (size_t)s->W[0] * s->H[0];
  if ((rc = alloc_volume(s))) return bail(rc);
  if ((rc = dalloc(s, &s->d_depth_u16, px))) return bail(rc);
  if ((rc = dalloc(s, &s->d_frame_ring, px * kf_session::kRing))) return bail(rc);
  if ((rc = dalloc(s, &s->d_depth_f32_in, px))) return bail(rc);
  for (int l = 0; l < 3; ++l) {
    const size_t n = (size_t)s->W[l] * s->H[l];
    if ((rc = dalloc(s, &s->d_depth[l], n))) return bail(rc);
    if ((rc = dalloc(s, &s->d_vertex[l], n))) return bail(rc);
    if ((rc = dalloc(s, &s->d_normal[l], n))) return bail(rc);
    if ((rc = dalloc(s, &s->d_status[l], n))) return bail(rc);
    cudaMemsetAsync(s->d_depth[l], 0, n * 4, s->stream);
    cudaMemsetAsync(s->d_vertex[l], 0, n * 16, s->stream);
    cudaMemsetAsync(s->d_normal[l], 0, n * 16, s->stream);
    cudaMemsetAsync(s->d_status[l], 0, n * 4, s->stream);
  }
  if ((rc = dalloc(s, &s->d_ref_vertex, px))) return bail(rc);
  if ((rc = dalloc(s, &s->d_ref_normal, px))) return bail(rc);
  if ((rc = dalloc(s, &s->d_sdf_rows, px * 8))) return bail(rc);
  if ((rc = dalloc(s, &s->d_partials, (size_t)2 * KF_MAX_TRACK_BLOCKS * 32))) return bail(rc);
  if ((rc = dalloc(s, &s->d_state, 1))) return bail(rc);
  if ((rc = dalloc(s, &s->d_u32_scalar, 4))) return bail(rc);
  cudaMemsetAsync(s->d_ref_vertex, 0, px * 16, s->stream);
  cudaMemsetAsync(s->d_ref_normal, 0, px * 16, s->stream);
  cudaMemsetAsync(s->d_sdf_rows, 0, px * 32, s->stream);
  if (cudaMallocHost((void**)&s->h_state, sizeof(KfDevState)) != cudaSuccess) return bail(KF_ERR_OUT_OF_MEMORY);
  if (cudaMallocHost((void**)&s->h_depth_pinned, px * 2) != cudaSuccess) return bail(KF_ERR_OUT_OF_MEMORY);
  if (cudaMallocHost((void**)&s->h_u32_scalar, 16) != cudaSuccess) return bail(KF_ERR_OUT_OF_MEMORY);
  std::memset(s->h_state, 0, sizeof(KfDevState));
  kf_store_pose(s->h_state, kIdentity);
  std::memcpy(s->h_state->pose_eig, kIdentity, sizeof(kIdentity));
  std::memcpy(s->h_state->old_pose, kIdentity, sizeof(kIdentity));
  std::memcpy(s->h_state->raycast_pose, kIdentity, sizeof(kIdentity));
  s->h_state->icp_center_cam[2] = 1.0;  // first ICP centre: 1 m in front of the camera
  s->h_state->reset_window = 1;
  if ((rc = push_state(s))) return bail(rc);
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return bail(KF_ERR_CUDA);
  *out = s;
  return KF_OK;
}

int kf_destroy(kf_session* s) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  free_all(s);
  delete s;
  return KF_OK;
}

const char* kf_last_error(const kf_session* s) { return s ? s->last_error.c_str() : "null session"; }

int kf_reset(kf_session* s, const double pose[16], int delete_flag) {
  if (!s || !pose || !kf_pose_is_finite(pose)) return KF_ERR_INVALID_ARGUMENT;
  int rc;
  if (delete_flag) {
    KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    drop_graph(s);
    if ((rc = alloc_volume(s))) return rc;
  } else {
    KF_CUDA_TRY(s, cudaMemsetAsync(s->d_vol, 0, s->vol_bytes, s->stream));
    if ((rc = kf_reset_bricks(s))) return rc;
  }
  if ((rc = pull_state(s))) return rc;
  s->h_state->lib_size = 0;  // poseLibrary.resize(0)
  // the ICP accumulation centre is carried from frame to frame; a new reconstruction starts
  // from the one a new session has (1 m in front of the camera), so that a reset session
  // computes exactly what a new one does
  s->h_state->icp_center_cam[0] = 0.0;
  s->h_state->icp_center_cam[1] = 0.0;
  s->h_state->icp_center_cam[2] = 1.0;
  set_pose_fields(s, pose, true);
  // the app's "Reset Volume" (kinect.cpp:446-477): reset = true, counter = 0, then a
  // raycast of the empty volume, i.e. zero reference maps
  s->h_state->reset_window = 1;
  s->h_state->counter = 0;
  std::memcpy(s->h_state->raycast_pose, pose, 16 * sizeof(double));
  const size_t px = (size_t)s->W[0] * s->H[0];
  KF_CUDA_TRY(s, cudaMemsetAsync(s->d_ref_vertex, 0, px * 16, s->stream));
  KF_CUDA_TRY(s, cudaMemsetAsync(s->d_ref_normal, 0, px * 16, s->stream));
  free_mc(s);
  return push_state(s);
}

int kf_reset_volume(kf_session* s) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  KF_CUDA_TRY(s, cudaMemsetAsync(s->d_vol, 0, s->vol_bytes, s->stream));
  if (int rc = kf_reset_bricks(s)) return rc;
  return KF_OK;
}

int kf_reset_pose(kf_session* s, const double pose[16]) {
  if (!s || !pose || !kf_pose_is_finite(pose)) return KF_ERR_INVALID_ARGUMENT;
  int rc = pull_state(s);
  if (rc) return rc;
  set_pose_fields(s, pose, true);
  return push_state(s);
}

int kf_set_pose(kf_session* s, const double pose[16]) {
  if (!s || !pose || !kf_pose_is_finite(pose)) return KF_ERR_INVALID_ARGUMENT;
  int rc = pull_state(s);
  if (rc) return rc;
  set_pose_fields(s, pose, false);
  return push_state(s);
}

int kf_get_pose(kf_session* s, double pose[16]) {
  if (!s || !pose) return KF_ERR_INVALID_ARGUMENT;
  int rc = pull_state_head(s);
  if (rc) return rc;
  std::memcpy(pose, s->h_state->pose, 16 * sizeof(double));
  return KF_OK;
}

int kf_set_config(kf_session* s, const kf_config* cfg) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  int rc = validate(cfg, &s->intr);
  if (rc) return rc;
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  const bool realloc = cfg->nx != s->cfg.nx || cfg->ny != s->cfg.ny || cfg->nz != s->cfg.nz ||
                       cfg->storage != s->cfg.storage;
  s->cfg = *cfg;
  s->layout += 1;  // kernel arguments derived from the configuration change
  if (s->cfg.integrate_every <= 0) s->cfg.integrate_every = 1;
  drop_graph(s);
  if (realloc) {
    free_mc(s);
    if ((rc = alloc_volume(s))) return rc;
  }
  return KF_OK;
}

int kf_depth_to_vertex_f32(kf_session* s, const float* host_depth_mm) {
  if (!s || !host_depth_mm) return KF_ERR_INVALID_ARGUMENT;
  const size_t px = (size_t)s->W[0] * s->H[0];
  KF_CUDA_TRY(s, cudaMemcpyAsync(s->d_depth_f32_in, host_depth_mm, px * 4, cudaMemcpyHostToDevice, s->stream));
  int rc = kf_launch_depth_ingest(s, nullptr, s->d_depth_f32_in);
  if (rc) return rc;
  return kf_launch_vertex(s);
}

int kf_depth_to_vertex_u16(kf_session* s, const uint16_t* host_depth_mm) {
  if (!s || !host_depth_mm) return KF_ERR_INVALID_ARGUMENT;
  const size_t px = (size_t)s->W[0] * s->H[0];
  KF_CUDA_TRY(s, cudaMemcpyAsync(s->d_depth_u16, host_depth_mm, px * 2, cudaMemcpyHostToDevice, s->stream));
  int rc = kf_launch_depth_ingest(s, s->d_depth_u16, nullptr);
  if (rc) return rc;
  return kf_launch_vertex(s);
}

int kf_depth_to_vertex_u16_device(kf_session* s, const uint16_t* device_depth_mm) {
  if (!s || !device_depth_mm) return KF_ERR_INVALID_ARGUMENT;
  int rc = kf_launch_depth_ingest(s, device_depth_mm, nullptr);
  if (rc) return rc;
  return kf_launch_vertex(s);
}

int kf_vertex_to_normal(kf_session* s) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  return kf_launch_normal(s);
}

int kf_track_icp(kf_session* s, int* tracked) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  int rc = record(s, 6);
  if (!rc) rc = kf_launch_icp(s, 0);
  if (!rc) rc = record(s, 7);
  if (rc || !tracked) return rc;
  if ((rc = pull_state_head(s))) return rc;
  *tracked = s->h_state->tracked;
  cudaEventElapsedTime(&s->stage_ms[1], s->ev[6], s->ev[7]);
  return KF_OK;
}

int kf_track_sdf(kf_session* s, int* tracked) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  int rc = kf_launch_sdf(s, 0, 0, 0);
  if (rc || !tracked) return rc;
  if ((rc = pull_state(s))) return rc;
  *tracked = s->h_state->tracked;
  return KF_OK;
}

int kf_recover_pose(kf_session* s, int* found) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  int rc = kf_launch_sdf(s, 1, 0, 0);
  if (rc || !found) return rc;
  if ((rc = pull_state(s))) return rc;
  *found = s->h_state->recover_found;
  return KF_OK;
}

int kf_get_alignment_energy(kf_session* s, float* ae) {
  if (!s || !ae) return KF_ERR_INVALID_ARGUMENT;
  int rc = pull_state(s);
  if (rc) return rc;
  *ae = (float)s->h_state->ae;
  return KF_OK;
}

int kf_get_iterations_run(kf_session* s, int* iterations) {
  if (!s || !iterations) return KF_ERR_INVALID_ARGUMENT;
  int rc = pull_state(s);
  if (rc) return rc;
  *iterations = s->h_state->iterations_run;
  return KF_OK;
}

int kf_get_reduction(kf_session* s, float sums[32]) {
  if (!s || !sums) return KF_ERR_INVALID_ARGUMENT;
  int rc = pull_state(s);
  if (rc) return rc;
  for (int k = 0; k < 32; ++k) sums[k] = (float)s->h_state->sums[k];
  return KF_OK;
}

int kf_integrate(kf_session* s) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  int rc = record(s, 8);
  if (!rc) rc = kf_launch_integrate(s, 0);
  if (!rc) rc = record(s, 9);
  if (!rc) rc = kf_note_integrate(s, s->stream);
  return rc;
}

int kf_raycast(kf_session* s) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  int rc = record(s, 10);
  if (!rc) rc = kf_launch_raycast(s);
  if (!rc) rc = record(s, 11);
  return rc;
}

int kf_frame_step_u16(kf_session* s, const uint16_t* host_depth_mm, int* tracked) {
  if (!s || !host_depth_mm) return KF_ERR_INVALID_ARGUMENT;
  const size_t px = (size_t)s->W[0] * s->H[0];
  const int slot = (int)(s->frames_run % kf_session::kRing);  // the graph slot run_frame uses
  KF_CUDA_TRY(s, cudaMemcpyAsync(slot_frame(s, slot), host_depth_mm, px * 2, cudaMemcpyHostToDevice, s->stream));
  int rc = run_frame(s);
  if (rc) return rc;
  return finish_step(s, tracked);
}

int kf_frame_step_u16_async(kf_session* s, const uint16_t* host_depth_mm) {
  if (!s || !host_depth_mm) return KF_ERR_INVALID_ARGUMENT;
  if (!s->h_heads) {
    if (cudaMallocHost((void**)&s->h_heads, (size_t)kf_session::kRing * KF_STATE_RESULT_BYTES) != cudaSuccess) {
      cudaGetLastError();
      s->h_heads = nullptr;
      return fail(s, KF_ERR_OUT_OF_MEMORY, "pinned result ring");
    }
    for (auto& e : s->head_ev) KF_CUDA_TRY(s, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto& e : s->upload_ev) KF_CUDA_TRY(s, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    KF_CUDA_TRY(s, cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
  }
  const size_t px = (size_t)s->W[0] * s->H[0];
  const int slot = (int)(s->frames_run % kf_session::kRing);  // the graph slot run_frame uses
  // the upload overlaps the frame still running: it goes on the copy stream once the last
  // frame of this slot (kRing frames ago) has finished with its input, and the frame waits
  // for it
  if (s->ring_ev[slot][5]) KF_CUDA_TRY(s, cudaStreamWaitEvent(s->copy_stream, s->ring_ev[slot][5], 0));
  KF_CUDA_TRY(s, cudaMemcpyAsync(slot_frame(s, slot), host_depth_mm, px * 2, cudaMemcpyHostToDevice, s->copy_stream));
  KF_CUDA_TRY(s, cudaEventRecord(s->upload_ev[slot], s->copy_stream));
  KF_CUDA_TRY(s, cudaStreamWaitEvent(s->stream, s->upload_ev[slot], 0));
  int rc = run_frame(s);
  if (rc) return rc;
  KF_CUDA_TRY(s, cudaMemcpyAsync(s->h_heads + (size_t)slot * KF_STATE_RESULT_BYTES, s->d_state, KF_STATE_RESULT_BYTES,
                                 cudaMemcpyDeviceToHost, s->stream));
  KF_CUDA_TRY(s, cudaEventRecord(s->head_ev[slot], s->stream));
  // the previous step's result is read now, while this one runs
  rc = finish_async(s);
  s->async_pend = slot;
  return rc;
}

int kf_frame_sync(kf_session* s, int* tracked) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  int rc = finish_async(s);
  if (!rc && tracked) *tracked = s->h_state->tracked;
  return rc;
}

int kf_get_last_result(kf_session* s, double pose[16], int* tracked) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  if (pose) std::memcpy(pose, s->h_state->pose, 16 * sizeof(double));
  if (tracked) *tracked = s->h_state->tracked;
  return KF_OK;
}

int kf_frame_step_u16_device(kf_session* s, const uint16_t* device_depth_mm, int* tracked) {
  if (!s || !device_depth_mm) return KF_ERR_INVALID_ARGUMENT;
  const size_t px = (size_t)s->W[0] * s->H[0];
  const int slot = (int)(s->frames_run % kf_session::kRing);  // the graph slot run_frame uses
  KF_CUDA_TRY(s, cudaMemcpyAsync(slot_frame(s, slot), device_depth_mm, px * 2, cudaMemcpyDeviceToDevice, s->stream));
  int rc = run_frame(s);
  if (rc) return rc;
  return finish_step(s, tracked);
}

static int copy_out(kf_session* s, void* dst, const void* src, size_t bytes) {
  KF_CUDA_TRY(s, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s->stream));
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return KF_OK;
}

int kf_get_raycast(kf_session* s, float* v, float* n) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  const size_t px = (size_t)s->W[0] * s->H[0];
  int rc = KF_OK;
  if (v) rc = copy_out(s, v, s->d_ref_vertex, px * 16);
  if (!rc && n) rc = copy_out(s, n, s->d_ref_normal, px * 16);
  return rc;
}

int kf_set_reference_maps(kf_session* s, const float* v, const float* n) {
  if (!s || !v || !n) return KF_ERR_INVALID_ARGUMENT;
  if (int rc = finish_async(s)) return rc;
  const size_t px = (size_t)s->W[0] * s->H[0];
  KF_CUDA_TRY(s, cudaMemcpyAsync(s->d_ref_vertex, v, px * 16, cudaMemcpyHostToDevice, s->stream));
  KF_CUDA_TRY(s, cudaMemcpyAsync(s->d_ref_normal, n, px * 16, cudaMemcpyHostToDevice, s->stream));
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return KF_OK;
}

int kf_get_vertex_map(kf_session* s, int level, float* v) {
  if (!s || !v || level < 0 || level > 2) return KF_ERR_INVALID_ARGUMENT;
  return copy_out(s, v, s->d_vertex[level], (size_t)s->W[level] * s->H[level] * 16);
}

int kf_get_normal_map(kf_session* s, int level, float* n) {
  if (!s || !n || level < 0 || level > 2) return KF_ERR_INVALID_ARGUMENT;
  return copy_out(s, n, s->d_normal[level], (size_t)s->W[level] * s->H[level] * 16);
}

int kf_get_depth_map(kf_session* s, int level, float* d) {
  if (!s || !d || level < 0 || level > 2) return KF_ERR_INVALID_ARGUMENT;
  return copy_out(s, d, s->d_depth[level], (size_t)s->W[level] * s->H[level] * 4);
}

int kf_get_track_status(kf_session* s, int level, int32_t* st) {
  if (!s || !st || level < 0 || level > 2) return KF_ERR_INVALID_ARGUMENT;
  return copy_out(s, st, s->d_status[level], (size_t)s->W[level] * s->H[level] * 4);
}

int kf_get_volume(kf_session* s, kf_volume_view* v) {
  if (!s || !v) return KF_ERR_INVALID_ARGUMENT;
  v->device_ptr = s->d_vol;
  v->nx = s->cfg.nx; v->ny = s->cfg.ny; v->nz = s->cfg.nz;
  v->storage = s->cfg.storage;
  v->value_bytes = (int64_t)s->vol_value_bytes;
  v->weight_offset_bytes = (int64_t)(s->vol_count * s->vol_value_bytes);
  v->row_pitch_bytes = (int64_t)s->cfg.nx * v->value_bytes;
  v->slice_pitch_bytes = v->row_pitch_bytes * s->cfg.ny;
  return KF_OK;
}

int kf_copy_volume_to_host(kf_session* s, void* dst, uint64_t bytes) {
  if (!s || !dst || bytes != s->vol_bytes) return KF_ERR_INVALID_ARGUMENT;
  return copy_out(s, dst, s->d_vol, bytes);
}

int kf_copy_volume_from_host(kf_session* s, const void* src, uint64_t bytes) {
  if (!s || !src || bytes != s->vol_bytes) return KF_ERR_INVALID_ARGUMENT;
  KF_CUDA_TRY(s, cudaMemcpyAsync(s->d_vol, src, bytes, cudaMemcpyHostToDevice, s->stream));
  int rc = kf_rebuild_bricks(s, s->stream);
  if (rc) return rc;
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return KF_OK;
}

// ---- volume checkpoint -------------------------------------------------------------------
// The reference keeps no volume on disk (gFusion::Reset, src/gFusion.cpp:226-240, only
// reallocates or zero-fills).  A checkpoint here is everything the next frame step reads:
// one JSON header line, then the raw sections in this order: the volume (value plane, then
// weight plane), the device control block (pose, pose library, frame-policy flags), the
// raycast vertex and normal maps and the trackSDF rows.  A session loaded from it steps on
// exactly as the saved one would have.
namespace {

const char kCkptFormat[] = "kf-volume-checkpoint";
const size_t kCkptChunk = (size_t)32 << 20;

struct CkptSection {
  void* dev;
  size_t bytes;
};

void ckpt_sections(kf_session* s, CkptSection out[4]) {
  const size_t px = (size_t)s->W[0] * s->H[0];
  out[0] = {s->d_vol, s->vol_bytes};
  out[1] = {s->d_ref_vertex, px * 16};
  out[2] = {s->d_ref_normal, px * 16};
  out[3] = {s->d_sdf_rows, px * 32};
}

std::string ckpt_header(kf_session* s) {
  const size_t px = (size_t)s->W[0] * s->H[0];
  char buf[2048];
  int n = std::snprintf(
      buf, sizeof(buf),
      "{\"format\":\"%s\",\"version\":1,\"storage\":%d,\"nx\":%d,\"ny\":%d,\"nz\":%d,"
      "\"dim_x\":%.9g,\"dim_y\":%.9g,\"dim_z\":%.9g,\"mu\":%.9g,\"width\":%d,\"height\":%d,"
      "\"volume_bytes\":%llu,\"state_bytes\":%llu,\"map_bytes\":%llu,\"sdf_bytes\":%llu,\"pose\":[",
      kCkptFormat, s->cfg.storage, s->cfg.nx, s->cfg.ny, s->cfg.nz, s->cfg.dim_x, s->cfg.dim_y, s->cfg.dim_z,
      s->cfg.mu, s->W[0], s->H[0], (unsigned long long)s->vol_bytes, (unsigned long long)sizeof(KfDevState),
      (unsigned long long)(px * 16), (unsigned long long)(px * 32));
  std::string h(buf, (size_t)n);
  for (int k = 0; k < 16; ++k) {
    n = std::snprintf(buf, sizeof(buf), "%s%.17g", k ? "," : "", s->h_state->pose[k]);
    h.append(buf, (size_t)n);
  }
  h += "]}\n";
  return h;
}

bool json_number(const std::string& h, const char* key, double* v) {
  const std::string k = std::string("\"") + key + "\":";
  const size_t p = h.find(k);
  if (p == std::string::npos) return false;
  const char* c = h.c_str() + p + k.size();
  char* end = nullptr;
  *v = std::strtod(c, &end);
  return end != c;
}

bool json_string_is(const std::string& h, const char* key, const char* want) {
  const std::string k = std::string("\"") + key + "\":\"" + want + "\"";
  return h.find(k) != std::string::npos;
}

int copy_section_to_file(kf_session* s, std::FILE* f, const void* dev, size_t bytes, std::vector<char>& buf) {
  for (size_t o = 0; o < bytes; o += kCkptChunk) {
    const size_t n = std::min(kCkptChunk, bytes - o);
    KF_CUDA_TRY(s, cudaMemcpyAsync(buf.data(), static_cast<const char*>(dev) + o, n, cudaMemcpyDeviceToHost, s->stream));
    KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    if (std::fwrite(buf.data(), 1, n, f) != n) return fail(s, KF_ERR_IO, "checkpoint write failed");
  }
  return KF_OK;
}

int copy_section_from_file(kf_session* s, std::FILE* f, void* dev, size_t bytes, std::vector<char>& buf) {
  for (size_t o = 0; o < bytes; o += kCkptChunk) {
    const size_t n = std::min(kCkptChunk, bytes - o);
    if (std::fread(buf.data(), 1, n, f) != n) return fail(s, KF_ERR_IO, "checkpoint read failed");
    KF_CUDA_TRY(s, cudaMemcpyAsync(static_cast<char*>(dev) + o, buf.data(), n, cudaMemcpyHostToDevice, s->stream));
    KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  }
  return KF_OK;
}

}  // namespace

int kf_save_volume(kf_session* s, const char* path) {
  if (!s || !path) return KF_ERR_INVALID_ARGUMENT;
  int rc = pull_state(s);
  if (rc) return rc;
  std::FILE* f = std::fopen(path, "wb");
  if (!f) return fail(s, KF_ERR_IO, std::string("cannot open ") + path);
  const std::string h = ckpt_header(s);
  CkptSection sec[4];
  ckpt_sections(s, sec);
  std::vector<char> buf(kCkptChunk);
  if (std::fwrite(h.data(), 1, h.size(), f) != h.size()) rc = fail(s, KF_ERR_IO, "checkpoint write failed");
  if (!rc) rc = copy_section_to_file(s, f, sec[0].dev, sec[0].bytes, buf);
  if (!rc && std::fwrite(s->h_state, 1, sizeof(KfDevState), f) != sizeof(KfDevState))
    rc = fail(s, KF_ERR_IO, "checkpoint write failed");
  for (int k = 1; k < 4 && !rc; ++k) rc = copy_section_to_file(s, f, sec[k].dev, sec[k].bytes, buf);
  if (std::fclose(f) != 0 && !rc) rc = fail(s, KF_ERR_IO, "checkpoint close failed");
  return rc;
}

int kf_load_volume(kf_session* s, const char* path) {
  if (!s || !path) return KF_ERR_INVALID_ARGUMENT;
  std::FILE* f = std::fopen(path, "rb");
  if (!f) return fail(s, KF_ERR_IO, std::string("cannot open ") + path);
  // header line (bounded)
  std::string h;
  for (int c; h.size() < 4096 && (c = std::fgetc(f)) != EOF;) {
    h.push_back((char)c);
    if (c == '\n') break;
  }
  CkptSection sec[4];
  ckpt_sections(s, sec);
  const size_t px = (size_t)s->W[0] * s->H[0];
  double v = 0;
  int rc = KF_OK;
  auto need = [&](const char* key, double want) {
    if (!rc && !(json_number(h, key, &v) && v == want))
      rc = fail(s, KF_ERR_INVALID_ARGUMENT, std::string("checkpoint ") + key + " does not match the session");
  };
  // floats are written with 9 significant digits, which round-trip a float
  auto need_f = [&](const char* key, float want) {
    if (!rc && !(json_number(h, key, &v) && (float)v == want))
      rc = fail(s, KF_ERR_INVALID_ARGUMENT, std::string("checkpoint ") + key + " does not match the session");
  };
  if (h.empty() || h.back() != '\n' || !json_string_is(h, "format", kCkptFormat))
    rc = fail(s, KF_ERR_INVALID_ARGUMENT, "not a volume checkpoint");
  need("version", 1);
  need("storage", s->cfg.storage);
  need("nx", s->cfg.nx);
  need("ny", s->cfg.ny);
  need("nz", s->cfg.nz);
  need("width", s->W[0]);
  need("height", s->H[0]);
  // the TSDF's meaning depends on the volume's metric size and truncation distance
  need_f("dim_x", s->cfg.dim_x);
  need_f("dim_y", s->cfg.dim_y);
  need_f("dim_z", s->cfg.dim_z);
  need_f("mu", s->cfg.mu);
  need("volume_bytes", (double)s->vol_bytes);
  need("state_bytes", (double)sizeof(KfDevState));  // the control block of this library build
  need("map_bytes", (double)(px * 16));
  need("sdf_bytes", (double)(px * 32));
  // the whole payload must be there before the session is touched
  if (!rc) {
    const long long payload = (long long)(s->vol_bytes + sizeof(KfDevState) + px * 64);
    const long long at = (long long)h.size();
    if (std::fseek(f, 0, SEEK_END) != 0 || (long long)std::ftell(f) != at + payload ||
        std::fseek(f, (long)at, SEEK_SET) != 0)
      rc = fail(s, KF_ERR_IO, "checkpoint has the wrong size");
  }
  if (rc) {
    std::fclose(f);
    return rc;
  }
  // the control block is read and checked before anything is written to the device
  std::vector<char> state(sizeof(KfDevState));
  std::vector<char> buf(kCkptChunk);
  if (std::fseek(f, (long)(h.size() + s->vol_bytes), SEEK_SET) != 0 ||
      std::fread(state.data(), 1, state.size(), f) != state.size() ||
      std::fseek(f, (long)h.size(), SEEK_SET) != 0)
    rc = fail(s, KF_ERR_IO, "checkpoint read failed");
  KfDevState* st = reinterpret_cast<KfDevState*>(state.data());
  if (!rc && (!kf_pose_is_finite(st->pose) || st->lib_size < 0 || st->lib_size > KF_MAX_LIBRARY))
    rc = fail(s, KF_ERR_INVALID_ARGUMENT, "checkpoint control block is invalid");
  if (!rc) {
    KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    free_mc(s);  // a mesh of the old volume
    rc = copy_section_from_file(s, f, sec[0].dev, sec[0].bytes, buf);
  }
  if (!rc && std::fseek(f, (long)sizeof(KfDevState), SEEK_CUR) != 0) rc = fail(s, KF_ERR_IO, "checkpoint read failed");
  for (int k = 1; k < 4 && !rc; ++k) rc = copy_section_from_file(s, f, sec[k].dev, sec[k].bytes, buf);
  std::fclose(f);
  if (rc) return rc;
  std::memcpy(s->h_state, st, sizeof(KfDevState));
  s->h_state->error = 0;
  if ((rc = push_state(s))) return rc;
  if ((rc = kf_rebuild_bricks(s, s->stream))) return rc;
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  return KF_OK;
}

// ---- depth ingest: Kinect-v2 undistortion and filter3D.cs -----------------------------------
namespace {
int ensure_depth_prep(kf_session* s) {
  if (s->d_depth_prep) return KF_OK;
  return dalloc(s, &s->d_depth_prep, (size_t)s->W[0] * s->H[0]);
}
}  // namespace

int kf_set_depth_undistortion(kf_session* s, const kf_ir_camera* ir) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  if (ir) {
    const float v[9] = {ir->fx, ir->fy, ir->cx, ir->cy, ir->k1, ir->k2, ir->k3, ir->p1, ir->p2};
    for (float f : v)
      if (!std::isfinite(f)) return KF_ERR_INVALID_ARGUMENT;
    if (!(ir->fx > 0) || !(ir->fy > 0)) return KF_ERR_INVALID_ARGUMENT;
  }
  // the captured frame graphs hold the old ingest
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  drop_graph(s);
  if (!ir) {
    s->undistort = 0;
    return KF_OK;
  }
  int rc = ensure_depth_prep(s);
  if (rc) return rc;
  if (!s->d_undistort_map && (rc = dalloc(s, &s->d_undistort_map, (size_t)s->W[0] * s->H[0]))) return rc;
  if ((rc = kf_launch_undistort_map(s, *ir))) return rc;
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  s->undistort = 1;
  return KF_OK;
}

int kf_set_depth_filter(kf_session* s, int enable) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  drop_graph(s);
  if (enable) {
    int rc = ensure_depth_prep(s);
    if (rc) return rc;
  }
  s->depth_filter = enable ? 1 : 0;
  return KF_OK;
}

int kf_get_undistortion_map(kf_session* s, int32_t* map) {
  if (!s || !map) return KF_ERR_INVALID_ARGUMENT;
  if (!s->undistort) return fail(s, KF_ERR_STATE, "undistortion is off");
  return copy_out(s, map, s->d_undistort_map, (size_t)s->W[0] * s->H[0] * sizeof(int32_t));
}

// ---- intensity projection (gFusion::intensityProjection, src/gFusion.cpp:1368-1409) ------
int kf_intensity_projection(kf_session* s, float* rgba) {
  if (!s || !rgba) return KF_ERR_INVALID_ARGUMENT;
  const size_t px = (size_t)s->W[0] * s->H[0];
  int rc;
  if (!s->d_mip && (rc = dalloc(s, &s->d_mip, px))) return rc;
  if ((rc = kf_launch_intensity_projection(s, s->d_mip))) return rc;
  return copy_out(s, rgba, s->d_mip, px * 16);
}

// ---- bounded-wait self-test ------------------------------------------------------------------
namespace {
// Block 0 waits at a two-block barrier that block 1 never reaches, so its bounded wait
// must give up and record KF_DEV_ERR_TIMEOUT in the session's device error word.
__global__ void barrier_timeout_selftest_kernel(unsigned* counter, int* error, long long budget) {
  __shared__ int s_flag;
  if (blockIdx.x != 0) return;
  kf_grid_sync_bounded(error, counter, 2u, &s_flag, budget);
}
}  // namespace

int kf_selftest_barrier_timeout(kf_session* s, long long budget_cycles) {
  if (!s || budget_cycles < 1000 || budget_cycles > KF_BARRIER_SPIN_CYCLES) return KF_ERR_INVALID_ARGUMENT;
  KF_CUDA_TRY(s, cudaMemsetAsync(s->d_u32_scalar, 0, sizeof(uint32_t), s->stream));
  barrier_timeout_selftest_kernel<<<2, 32, 0, s->stream>>>(s->d_u32_scalar, &s->d_state->error, budget_cycles);
  KF_CUDA_TRY(s, cudaGetLastError());
  kf_note_launch(s);
  // the host side of every tracking call: read the sticky error word, report and clear it
  return pull_state_head(s);
}

int kf_get_cum_twist(kf_session* s, double t[6]) {
  if (!s || !t) return KF_ERR_INVALID_ARGUMENT;
  int rc = pull_state(s);
  if (rc) return rc;
  std::memcpy(t, s->h_state->cum_twist, 6 * sizeof(double));
  return KF_OK;
}

int kf_get_pose_library_size(kf_session* s, int* n) {
  if (!s || !n) return KF_ERR_INVALID_ARGUMENT;
  int rc = pull_state(s);
  if (rc) return rc;
  *n = s->h_state->lib_size;
  return KF_OK;
}

int kf_set_stage_timing(kf_session* s, int every) {
  if (!s || !(every == 0 || every == 1 || every == 2 || every == 4)) return KF_ERR_INVALID_ARGUMENT;
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  int rc = harvest_all(s);  // the frames already run keep their stage times
  if (rc) return rc;
  drop_graph(s);  // the captured frames hold the old event layout
  s->stage_every = every;
  return KF_OK;
}

int kf_get_stage_timing(kf_session* s, int* every) {
  if (!s || !every) return KF_ERR_INVALID_ARGUMENT;
  *every = s->stage_every;
  return KF_OK;
}

int kf_get_stage_times(kf_session* s, float ms[6]) {
  if (!s || !ms) return KF_ERR_INVALID_ARGUMENT;
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  int rc = harvest_all(s);
  if (rc) return rc;
  for (int i = 0; i < 6; ++i) ms[i] = s->stage_ms[i];
  return KF_OK;
}

int kf_get_stage_stats(kf_session* s, double mean_ms[6], uint64_t* frames) {
  if (!s || !mean_ms || !frames) return KF_ERR_INVALID_ARGUMENT;
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  int rc = harvest_all(s);
  if (rc) return rc;
  *frames = s->stage_frames;
  for (int i = 0; i < 6; ++i) mean_ms[i] = s->stage_frames ? s->stage_acc[i] / (double)s->stage_frames : 0.0;
  return KF_OK;
}

int kf_reset_stage_stats(kf_session* s) {
  if (!s) return KF_ERR_INVALID_ARGUMENT;
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  int rc = harvest_all(s);
  if (rc) return rc;
  for (int i = 0; i < 6; ++i) s->stage_acc[i] = 0.0;
  s->stage_frames = 0;
  return KF_OK;
}

int kf_get_launch_count(kf_session* s, uint64_t* launches) {
  if (!s || !launches) return KF_ERR_INVALID_ARGUMENT;
  *launches = s->launches;
  return KF_OK;
}

int kf_get_stream(kf_session* s, void** stream) {
  if (!s || !stream) return KF_ERR_INVALID_ARGUMENT;
  *stream = (void*)s->stream;
  return KF_OK;
}

// ---- launch shapes and the autotuner ------------------------------------------------------
int kf_set_launch_shape(kf_session* s, const kf_launch_shape* shape) {
  if (!s || !shape || !kf_valid_int_zc(shape->integrate_z_chunk) || !kf_valid_ray_rows(shape->raycast_rows))
    return KF_ERR_INVALID_ARGUMENT;
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  drop_graph(s);  // the captured frames hold the old shapes
  s->int_zc = shape->integrate_z_chunk;
  s->ray_rows = shape->raycast_rows;
  return KF_OK;
}

int kf_get_launch_shape(kf_session* s, kf_launch_shape* shape) {
  if (!s || !shape) return KF_ERR_INVALID_ARGUMENT;
  std::memset(shape, 0, sizeof(*shape));
  shape->integrate_z_chunk = s->int_zc;
  shape->raycast_rows = s->ray_rows;
  return KF_OK;
}

int kf_autotune(kf_session* s, int repeats, kf_launch_shape* chosen, float* times_ms) {
  if (!s || repeats < 1 || repeats > 1000) return KF_ERR_INVALID_ARGUMENT;
  KF_CUDA_TRY(s, cudaStreamSynchronize(s->stream));
  kf_scratch_target t;
  int rc = kf_scratch_alloc(s, &t);
  if (rc) return rc;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) rc = fail(s, KF_ERR_CUDA, "autotune events");
  // each candidate: one untimed launch, then `repeats` timed launches; two rounds over all
  // candidates, the better mean kept (clock and cache drift even out).  Integrate
  // candidates run back to back (in the frame loop only ICP, which touches a few MB, runs
  // between two integrates); each raycast candidate launch follows an untimed integrate,
  // as in the frame loop, whose volume traffic leaves L2 as a frame's raycast finds it
  // (raycasts back to back would find the previous one's bricks in L2 and favour other
  // shapes).
  float best[7] = {1e30f, 1e30f, 1e30f, 1e30f, 1e30f, 1e30f, 1e30f};
  auto elapsed = [&](float* ms) {
    if (cudaEventRecord(e1, s->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(ms, e0, e1) != cudaSuccess)
      return fail(s, KF_ERR_CUDA, "autotune timing failed");
    return (int)KF_OK;
  };
  for (int round = 0; round < 2 && !rc; ++round)
    for (int c = 0; c < 7 && !rc; ++c) {
      const bool ray = c >= 3;
      const int v = ray ? kf_tune_ray_rows[c - 3] : kf_tune_int_zc[c];
      auto launch = [&]() {
        return ray ? kf_launch_raycast_shape(s, v, &t) : kf_launch_integrate_shape(s, 0, v, &t);
      };
      if ((rc = launch())) break;
      float total = 0.0f;
      if (!ray) {
        if (cudaEventRecord(e0, s->stream) != cudaSuccess) { rc = fail(s, KF_ERR_CUDA, "autotune timing failed"); break; }
        for (int r = 0; r < repeats && !rc; ++r) rc = launch();
        if (rc || (rc = elapsed(&total))) break;
      } else {
        for (int r = 0; r < repeats && !rc; ++r) {
          if ((rc = kf_launch_integrate_shape(s, 0, s->int_zc, &t))) break;
          if (cudaEventRecord(e0, s->stream) != cudaSuccess) { rc = fail(s, KF_ERR_CUDA, "autotune timing failed"); break; }
          float ms = 0.0f;
          if ((rc = launch()) || (rc = elapsed(&ms))) break;
          total += ms;
        }
        if (rc) break;
      }
      best[c] = std::min(best[c], total / (float)repeats);
    }
  cudaStreamSynchronize(s->stream);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  kf_scratch_free(&t);
  if (rc) return rc;
  int zi = 1, ri = 5;  // the defaults (z-chunk 16, 32 x 4 tiles) win ties
  for (int c = 0; c < 3; ++c)
    if (best[c] < best[zi]) zi = c;
  for (int c = 3; c < 7; ++c)
    if (best[c] < best[ri]) ri = c;
  kf_launch_shape sh{};
  sh.integrate_z_chunk = kf_tune_int_zc[zi];
  sh.raycast_rows = kf_tune_ray_rows[ri - 3];
  if ((rc = kf_set_launch_shape(s, &sh))) return rc;
  kf_tune_cache_put(s, sh.integrate_z_chunk, sh.raycast_rows);
  if (chosen) *chosen = sh;
  if (times_ms) std::memcpy(times_ms, best, sizeof(best));
  return KF_OK;
}

}  // extern "C"
