// kf_batch.cu — batched frame steps: many sessions, one launch per stage.
//
// Reference: the per-frame body of kinect.cpp:654-695 (pyramid, Track, integrate when
// tracked or in the reset window, recoverPose when not tracked, raycast), run for every
// member session.  The reference has one session; this is the batched form.
//
// B200 design: a batch step launches each stage once for all members — the pyramid and
// raycast grids carry the member in blockIdx.z, integrate walks a flat grid of every
// member's voxel blocks (a prefix table maps a block to its member), and the tracking
// kernels split the co-resident grid into one group of blocks per member, each with its
// own barrier and fixed-point reduction rows.  Per-member arguments live in one device
// table, rebuilt only when the membership changes.  A member's results are bit-identical
// to stepping it alone: every kernel computes a member exactly as in its single-session
// launch, and the ICP sums are exact integers whatever the block split.
#include <algorithm>
#include <cstring>

#include "kf_internal.cuh"

namespace {

// Zero each member's tracking words (barrier counters and ICP sum buffers).
__global__ void batch_clear_kernel(KfDevState* const* states) {
  KfDevState* st = states[blockIdx.x];
  if (threadIdx.x == 0) {
    st->barrier_count = 0;
    st->sdf_barrier_count = 0;
  }
  for (int k = threadIdx.x; k < 3 * 32; k += blockDim.x) st->icp_acc[k / 32][k % 32][0] = 0;
}

// Gather each member's frame result (the first KF_STATE_RESULT_BYTES of its state).
__global__ void batch_gather_kernel(KfDevState* const* states, char* heads) {
  const char* src = reinterpret_cast<const char*>(states[blockIdx.x]);
  for (int k = threadIdx.x; k < (int)(KF_STATE_RESULT_BYTES / 4); k += blockDim.x)
    reinterpret_cast<int*>(heads + (size_t)blockIdx.x * KF_STATE_RESULT_BYTES)[k] = reinterpret_cast<const int*>(src)[k];
}

int bfail(kf_batch* b, int code, const std::string& msg) {
  b->last_error = msg;
  return code;
}

int check_members(kf_batch* b, kf_session* const* ss, int n) {
  kf_session* s0 = ss[0];
  for (int e = 0; e < n; ++e) {
    kf_session* s = ss[e];
    if (!s) return bfail(b, KF_ERR_INVALID_ARGUMENT, "null session");
    if (s->device != b->device) return bfail(b, KF_ERR_INVALID_ARGUMENT, "session on another device");
    if (s->W[0] != s0->W[0] || s->H[0] != s0->H[0])
      return bfail(b, KF_ERR_INVALID_ARGUMENT, "sessions of one batch step need the same image size");
    if (s->cfg.storage != s0->cfg.storage || s->cfg.jtj != s0->cfg.jtj)
      return bfail(b, KF_ERR_INVALID_ARGUMENT, "sessions of one batch step need the same storage and J^T J form");
    if (s->cfg.tracking != KF_TRACK_ICP) return bfail(b, KF_ERR_INVALID_ARGUMENT, "batched frame steps track by ICP");
    if (s->undistort || s->depth_filter)
      return bfail(b, KF_ERR_INVALID_ARGUMENT, "batched frame steps read raw depth (undistortion and filter off)");
    for (int f = 0; f < e; ++f)
      if (ss[f] == s) return bfail(b, KF_ERR_INVALID_ARGUMENT, "a session appears twice in one batch step");
  }
  return KF_OK;
}

bool same_members(const kf_batch* b, kf_session* const* ss, int n) {
  if ((int)b->members.size() != n) return false;
  for (int e = 0; e < n; ++e)
    if (b->members[e] != ss[e] || b->member_keys[e] != std::make_pair(ss[e]->uid, ss[e]->layout)) return false;
  return true;
}

// The step graphs bake in the tables' launch configuration and shapes: dropped whenever
// those change.
void drop_graphs(kf_batch* b) {
  for (int k = 0; k < 2; ++k) {
    if (b->step_exec[k]) cudaGraphExecDestroy(b->step_exec[k]);
    b->step_exec[k] = nullptr;
    b->graph_n[k] = 0;
    b->graph_kernels[k] = 0;
  }
}

int rebuild_tables(kf_batch* b, kf_session* const* ss, int n) {
  drop_graphs(b);
  b->members.assign(ss, ss + n);
  b->member_keys.resize(n);
  for (int e = 0; e < n; ++e) b->member_keys[e] = std::make_pair(ss[e]->uid, ss[e]->layout);
  b->table_used = 0;
  KfDevState** hs = nullptr;
  b->states = static_cast<KfDevState* const*>(kf_batch_table(b, sizeof(KfDevState*) * n, reinterpret_cast<void**>(&hs)));
  if (!b->states) return bfail(b, KF_ERR_CAPACITY, "batch table full");
  for (int e = 0; e < n; ++e) hs[e] = ss[e]->d_state;
  int rc;
  if ((rc = kf_batch_prepare_pyramid(b)) || (rc = kf_batch_prepare_icp(b)) ||
      (rc = kf_batch_prepare_integrate(b, nullptr)) || (rc = kf_batch_prepare_sdf(b)) ||
      (rc = kf_batch_prepare_raycast(b, nullptr))) {
    b->members.clear();
    b->member_keys.clear();
    return bfail(b, rc, "batch tables: too many sessions for the table or the co-resident grid");
  }
  KF_CUDA_TRY(b, cudaMemcpyAsync(b->d_table, b->h_table, b->table_used, cudaMemcpyHostToDevice, b->stream));
  return KF_OK;
}

// Reads the results of the pending step (waits for it): each member's frame result into
// its host state, the stage times, the tracked flags; a member's device timeout is
// reported and cleared.
int harvest(kf_batch* b) {
  const int slot = b->pend_slot;
  if (slot < 0) return KF_OK;
  b->pend_slot = -1;
  KF_CUDA_TRY(b, cudaEventSynchronize(b->ev[slot][6]));  // this step's results are copied
  for (int i = 0; i < 5; ++i) KF_CUDA_TRY(b, cudaEventElapsedTime(&b->stage_ms[i], b->ev[slot][i], b->ev[slot][i + 1]));
  const int n = (int)b->pend_members.size();
  const char* heads = b->h_heads + (size_t)slot * b->cap * KF_STATE_RESULT_BYTES;
  b->last_slot = slot;
  b->last_n = n;
  b->last_tracked.assign(n, 0);
  int first_err = KF_OK;
  for (int e = 0; e < n; ++e) {
    kf_session* s = b->pend_members[e];
    std::memcpy(s->h_state, heads + (size_t)e * KF_STATE_RESULT_BYTES, KF_STATE_RESULT_BYTES);
    b->last_tracked[e] = s->h_state->tracked;
    if (s->h_state->error) {
      const int err = s->h_state->error;
      s->h_state->error = 0;
      KF_CUDA_TRY(b, cudaMemsetAsync(&s->d_state->error, 0, sizeof(int), b->stream));
      s->last_error = "device wait timed out (error " + std::to_string(err) + ")";
      if (!first_err) first_err = bfail(b, KF_ERR_TIMEOUT, "session " + std::to_string(e) + ": " + s->last_error);
    }
  }
  if (first_err) KF_CUDA_TRY(b, cudaStreamSynchronize(b->stream));
  return first_err;
}

// Enqueues one step into the next slot (the previous step may still be running).
int enqueue_step(kf_batch* b, kf_session* const* ss, const uint16_t* const* depth, int n, cudaMemcpyKind kind) {
  if (!b || !ss || !depth || n <= 0) return KF_ERR_INVALID_ARGUMENT;
  if (n > b->cap) return bfail(b, KF_ERR_CAPACITY, "more sessions than the batch was created for");
  int rc = check_members(b, ss, n);
  if (rc) return rc;
  for (int e = 0; e < n; ++e)
    if (!depth[e]) return bfail(b, KF_ERR_INVALID_ARGUMENT, "null depth frame");
  int cur = 0;
  KF_CUDA_TRY(b, cudaGetDevice(&cur));
  if (cur != b->device) KF_CUDA_TRY(b, cudaSetDevice(b->device));
  // a destroyed session's address may come back for a new one, and a session may
  // reallocate its buffers: the tables are keyed by (address, uid, layout).  The host
  // table is rewritten only once the pending step (whose copy may read it) is done.
  if (!same_members(b, ss, n)) {
    if ((rc = harvest(b))) return rc;
    KF_CUDA_TRY(b, cudaStreamSynchronize(b->stream));
    if ((rc = rebuild_tables(b, ss, n))) return rc;
  }
  // a member's own stream may still hold work (an asynchronous frame step)
  for (int e = 0; e < n; ++e)
    if (cudaStreamQuery(ss[e]->stream) != cudaSuccess) KF_CUDA_TRY(b, cudaStreamSynchronize(ss[e]->stream));
  const int slot = (int)(b->steps & 1u);
  cudaEvent_t* ev = b->ev[slot];
  const uint16_t* const* inputs = nullptr;
  if (kind == cudaMemcpyHostToDevice) {
    const size_t px = (size_t)ss[0]->W[0] * ss[0]->H[0];
    for (int e = 0; e < n; ++e)
      KF_CUDA_TRY(b, cudaMemcpyAsync(ss[e]->d_depth_u16, depth[e], px * 2, kind, b->stream));
  } else {
    // device frames are read in place: one small upload of their addresses (in the step)
    const uint16_t** hin = b->h_inputs + (size_t)slot * b->cap;
    for (int e = 0; e < n; ++e) hin[e] = depth[e];
    inputs = b->d_inputs;
  }
  // the device part of the step: stages with their events, then every member's frame
  // result gathered and copied to the slot's pinned heads (external event records, so that
  // a captured step's events are recorded, and readable from the host, on every replay)
  // events recorded while capturing must be external records to be seen from the host;
  // outside capture the flag is not allowed
  unsigned rec_flags = cudaEventRecordDefault;
  auto body = [&]() -> int {
    int r;
    if (inputs) KF_CUDA_TRY(b, cudaMemcpyAsync(b->d_inputs, b->h_inputs + (size_t)slot * b->cap,
                                               n * sizeof(uint16_t*), cudaMemcpyHostToDevice, b->stream));
    KF_CUDA_TRY(b, cudaEventRecordWithFlags(ev[0], b->stream, rec_flags));
    batch_clear_kernel<<<n, 128, 0, b->stream>>>(b->states);
    KF_CUDA_TRY(b, cudaGetLastError());
    if ((r = kf_batch_launch_pyramid(b, n, inputs))) return r;
    KF_CUDA_TRY(b, cudaEventRecordWithFlags(ev[1], b->stream, rec_flags));
    if ((r = kf_batch_launch_icp(b))) return r;
    KF_CUDA_TRY(b, cudaEventRecordWithFlags(ev[2], b->stream, rec_flags));
    if ((r = kf_batch_launch_integrate(b))) return r;
    KF_CUDA_TRY(b, cudaEventRecordWithFlags(ev[3], b->stream, rec_flags));
    if ((r = kf_batch_launch_sdf_recover(b))) return r;
    KF_CUDA_TRY(b, cudaEventRecordWithFlags(ev[4], b->stream, rec_flags));
    if ((r = kf_batch_launch_raycast(b, n))) return r;
    KF_CUDA_TRY(b, cudaEventRecordWithFlags(ev[5], b->stream, rec_flags));
    batch_gather_kernel<<<n, 64, 0, b->stream>>>(b->states, b->d_heads);
    KF_CUDA_TRY(b, cudaGetLastError());
    b->launches += 2;
    KF_CUDA_TRY(b, cudaMemcpyAsync(b->h_heads + (size_t)slot * b->cap * KF_STATE_RESULT_BYTES, b->d_heads,
                                   (size_t)n * KF_STATE_RESULT_BYTES, cudaMemcpyDeviceToHost, b->stream));
    KF_CUDA_TRY(b, cudaEventRecordWithFlags(ev[6], b->stream, rec_flags));
    return KF_OK;
  };
  if (inputs) {
    // device frames: the step is a CUDA graph per slot, captured on its first use with
    // these tables and replayed (the input addresses are read from the slot's pinned list)
    if (!b->step_exec[slot] || b->graph_n[slot] != n) {
      if (b->step_exec[slot]) cudaGraphExecDestroy(b->step_exec[slot]);
      b->step_exec[slot] = nullptr;
      const uint64_t l0 = b->launches;
      KF_CUDA_TRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      rec_flags = cudaEventRecordExternal;
      rc = body();
      rec_flags = cudaEventRecordDefault;
      cudaGraph_t g = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
      if (rc || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return rc ? rc : bfail(b, KF_ERR_CUDA, std::string("batch step capture: ") + cudaGetErrorString(ce));
      }
      const cudaError_t ie = cudaGraphInstantiate(&b->step_exec[slot], g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess) {
        b->step_exec[slot] = nullptr;
        return bfail(b, KF_ERR_CUDA, std::string("batch step graph: ") + cudaGetErrorString(ie));
      }
      b->graph_n[slot] = n;
      b->graph_kernels[slot] = b->launches - l0;
      b->launches = l0;
    }
    KF_CUDA_TRY(b, cudaGraphLaunch(b->step_exec[slot], b->stream));
    b->launches += b->graph_kernels[slot];
    b->graph_replays += 1;
  } else if ((rc = body())) {
    return rc;
  }
  // every KF_BRICK_REBUILD_EVERY integrates a member's skip flags are rebuilt exactly
  for (int e = 0; e < n; ++e)
    if ((rc = kf_note_integrate(ss[e], b->stream))) return bfail(b, rc, "brick flag rebuild: " + ss[e]->last_error);
  b->steps += 1;
  // the previous step's results are read now, while this one runs
  const int prev = harvest(b);
  b->pend_slot = slot;
  b->pend_members.assign(ss, ss + n);
  return prev;
}

int batch_step(kf_batch* b, kf_session* const* ss, const uint16_t* const* depth, int n, int32_t* tracked,
               cudaMemcpyKind kind) {
  int rc = enqueue_step(b, ss, depth, n, kind);
  if (rc) {
    harvest(b);
    return rc;
  }
  if ((rc = harvest(b))) return rc;
  if (tracked)
    for (int e = 0; e < n; ++e) tracked[e] = b->last_tracked[e];
  return KF_OK;
}

void free_batch(kf_batch* b) {
  drop_graphs(b);
  cudaFree(b->d_table);
  cudaFreeHost(b->h_table);
  cudaFree(b->d_heads);
  cudaFreeHost(b->h_heads);
  cudaFree(b->d_inputs);
  cudaFreeHost(b->h_inputs);
  for (auto& row : b->ev)
    for (auto& e : row)
      if (e) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
}

}  // namespace

extern "C" {

int kf_batch_create(int max_sessions, kf_batch** out) {
  if (!out || max_sessions <= 0 || max_sessions > KF_BATCH_MAX_SESSIONS) return KF_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return KF_ERR_NO_DEVICE;
  }
  kf_batch* b = new (std::nothrow) kf_batch();
  if (!b) return KF_ERR_OUT_OF_MEMORY;
  b->cap = max_sessions;
  auto bail = [&](int code) {
    free_batch(b);
    delete b;
    return code;
  };
  if (cudaGetDevice(&b->device) != cudaSuccess) return bail(KF_ERR_CUDA);
  if (cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess)
    return bail(KF_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(KF_ERR_CUDA);
  for (auto& row : b->ev)
    for (auto& e : row)
      if (cudaEventCreate(&e) != cudaSuccess) return bail(KF_ERR_CUDA);
  // per member: seven argument records (< 2 KB) and two block maps of the co-resident grid
  b->table_cap = 64 * 1024 + (size_t)max_sessions * 2048;
  if (cudaMallocHost((void**)&b->h_table, b->table_cap) != cudaSuccess) return bail(KF_ERR_OUT_OF_MEMORY);
  if (cudaMalloc((void**)&b->d_table, b->table_cap) != cudaSuccess) return bail(KF_ERR_OUT_OF_MEMORY);
  const size_t hb = (size_t)max_sessions * KF_STATE_RESULT_BYTES;
  if (cudaMallocHost((void**)&b->h_heads, 2 * hb) != cudaSuccess) return bail(KF_ERR_OUT_OF_MEMORY);
  if (cudaMalloc((void**)&b->d_heads, hb) != cudaSuccess) return bail(KF_ERR_OUT_OF_MEMORY);
  if (cudaMallocHost((void**)&b->h_inputs, 2 * max_sessions * sizeof(uint16_t*)) != cudaSuccess)
    return bail(KF_ERR_OUT_OF_MEMORY);
  if (cudaMalloc((void**)&b->d_inputs, max_sessions * sizeof(uint16_t*)) != cudaSuccess)
    return bail(KF_ERR_OUT_OF_MEMORY);
  *out = b;
  return KF_OK;
}

int kf_batch_destroy(kf_batch* b) {
  if (!b) return KF_ERR_INVALID_ARGUMENT;
  harvest(b);
  cudaStreamSynchronize(b->stream);
  free_batch(b);
  delete b;
  return KF_OK;
}

const char* kf_batch_last_error(const kf_batch* b) { return b ? b->last_error.c_str() : "null batch"; }

int kf_batch_frame_step_u16(kf_batch* b, kf_session* const* sessions, const uint16_t* const* host_depth_mm, int n,
                            int32_t* tracked) {
  return batch_step(b, sessions, host_depth_mm, n, tracked, cudaMemcpyHostToDevice);
}

int kf_batch_frame_step_u16_device(kf_batch* b, kf_session* const* sessions, const uint16_t* const* device_depth_mm,
                                   int n, int32_t* tracked) {
  return batch_step(b, sessions, device_depth_mm, n, tracked, cudaMemcpyDeviceToDevice);
}

int kf_batch_get_stage_times(kf_batch* b, float* ms) {
  if (!b || !ms) return KF_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < 5; ++i) ms[i] = b->stage_ms[i];
  return KF_OK;
}

int kf_batch_frame_step_u16_device_async(kf_batch* b, kf_session* const* sessions,
                                         const uint16_t* const* device_depth_mm, int n) {
  return enqueue_step(b, sessions, device_depth_mm, n, cudaMemcpyDeviceToDevice);
}

int kf_batch_sync(kf_batch* b) {
  if (!b) return KF_ERR_INVALID_ARGUMENT;
  return harvest(b);
}

int kf_batch_get_poses(kf_batch* b, int n, double* poses) {
  if (!b || !poses || n < 0) return KF_ERR_INVALID_ARGUMENT;
  if (n > b->last_n) return bfail(b, KF_ERR_INVALID_ARGUMENT, "more poses than the last step had sessions");
  const char* heads = b->h_heads + (size_t)b->last_slot * b->cap * KF_STATE_RESULT_BYTES;
  for (int e = 0; e < n; ++e)
    std::memcpy(poses + 16 * e, heads + (size_t)e * KF_STATE_RESULT_BYTES, 16 * sizeof(double));
  return KF_OK;
}

int kf_batch_get_tracked(kf_batch* b, int n, int32_t* tracked) {
  if (!b || !tracked || n < 0) return KF_ERR_INVALID_ARGUMENT;
  if (n > b->last_n) return bfail(b, KF_ERR_INVALID_ARGUMENT, "more flags than the last step had sessions");
  for (int e = 0; e < n; ++e) tracked[e] = b->last_tracked[e];
  return KF_OK;
}

int kf_batch_get_launch_count(kf_batch* b, uint64_t* n) {
  if (!b || !n) return KF_ERR_INVALID_ARGUMENT;
  *n = b->launches;
  return KF_OK;
}

int kf_batch_set_launch_shape(kf_batch* b, const kf_launch_shape* shape) {
  if (!b || !shape || !kf_valid_int_zc(shape->integrate_z_chunk) || !kf_valid_batch_ray_rows(shape->raycast_rows))
    return KF_ERR_INVALID_ARGUMENT;
  if (int rc = harvest(b)) return rc;
  KF_CUDA_TRY(b, cudaStreamSynchronize(b->stream));
  b->int_zc = shape->integrate_z_chunk;
  b->ray_rows = shape->raycast_rows;
  // the integrate block prefix depends on the z-chunk: rebuild the tables at the next step
  b->members.clear();
  b->member_keys.clear();
  return KF_OK;
}

int kf_batch_get_launch_shape(kf_batch* b, kf_launch_shape* shape) {
  if (!b || !shape) return KF_ERR_INVALID_ARGUMENT;
  std::memset(shape, 0, sizeof(*shape));
  shape->integrate_z_chunk = b->int_zc;
  shape->raycast_rows = b->ray_rows;
  return KF_OK;
}

int kf_batch_autotune(kf_batch* b, kf_session* const* ss, int n, int repeats, kf_launch_shape* chosen,
                      float* times_ms) {
  if (!b || !ss || n < 1 || n > b->cap || repeats < 1 || repeats > 1000) return KF_ERR_INVALID_ARGUMENT;
  int rc = check_members(b, ss, n);
  if (rc) return rc;
  int cur = 0;
  KF_CUDA_TRY(b, cudaGetDevice(&cur));
  if (cur != b->device) KF_CUDA_TRY(b, cudaSetDevice(b->device));
  if ((rc = harvest(b))) return rc;
  KF_CUDA_TRY(b, cudaStreamSynchronize(b->stream));
  std::vector<kf_scratch_target> t(n);
  for (int e = 0; e < n && !rc; ++e) {
    if (cudaStreamSynchronize(ss[e]->stream) != cudaSuccess) {
      rc = bfail(b, KF_ERR_CUDA, "autotune: a member's stream failed");
      break;
    }
    if ((rc = kf_scratch_alloc(ss[e], &t[e]))) {
      bfail(b, rc, "autotune scratch: " + ss[e]->last_error);
      break;
    }
    if (cudaStreamSynchronize(ss[e]->stream) != cudaSuccess) rc = bfail(b, KF_ERR_CUDA, "autotune scratch copy");
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (!rc && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
    rc = bfail(b, KF_ERR_CUDA, "autotune events");
  // the tables are rebuilt here with scratch targets, one candidate at a time
  b->members.assign(ss, ss + n);
  b->member_keys.clear();
  const int zc0 = b->int_zc, rows0 = b->ray_rows;
  float best[6] = {1e30f, 1e30f, 1e30f, 1e30f, 1e30f, 1e30f};
  for (int round = 0; round < 2 && !rc; ++round)
    for (int c = 0; c < 6 && !rc; ++c) {
      const bool ray = c >= 3;
      if (cudaStreamSynchronize(b->stream) != cudaSuccess) { rc = bfail(b, KF_ERR_CUDA, "autotune"); break; }
      b->table_used = 0;
      if (ray) {
        b->ray_rows = kf_tune_batch_ray_rows[c - 3];
        rc = kf_batch_prepare_raycast(b, t.data());
      } else {
        b->int_zc = kf_tune_int_zc[c];
        rc = kf_batch_prepare_integrate(b, t.data());
      }
      if (rc) { bfail(b, rc, "autotune tables"); break; }
      if (cudaMemcpyAsync(b->d_table, b->h_table, b->table_used, cudaMemcpyHostToDevice, b->stream) != cudaSuccess) {
        rc = bfail(b, KF_ERR_CUDA, "autotune tables");
        break;
      }
      auto launch = [&]() { return ray ? kf_batch_launch_raycast(b, n) : kf_batch_launch_integrate(b); };
      if ((rc = launch())) break;
      if (cudaEventRecord(e0, b->stream) != cudaSuccess) { rc = bfail(b, KF_ERR_CUDA, "autotune timing"); break; }
      for (int r = 0; r < repeats && !rc; ++r) rc = launch();
      if (rc) break;
      float ms = 0.0f;
      if (cudaEventRecord(e1, b->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
          cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
        rc = bfail(b, KF_ERR_CUDA, "autotune timing");
        break;
      }
      best[c] = std::min(best[c], ms / (float)repeats);
    }
  cudaStreamSynchronize(b->stream);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  for (auto& x : t) kf_scratch_free(&x);
  // the next step rebuilds the real tables
  b->members.clear();
  b->member_keys.clear();
  b->int_zc = zc0;
  b->ray_rows = rows0;
  if (rc) return rc;
  int zi = 1, ri = 4;  // the defaults win ties
  for (int c = 0; c < 3; ++c)
    if (best[c] < best[zi]) zi = c;
  for (int c = 3; c < 6; ++c)
    if (best[c] < best[ri]) ri = c;
  b->int_zc = kf_tune_int_zc[zi];
  b->ray_rows = kf_tune_batch_ray_rows[ri - 3];
  if (chosen) kf_batch_get_launch_shape(b, chosen);
  if (times_ms) std::memcpy(times_ms, best, sizeof(best));
  return KF_OK;
}

}  // extern "C"
