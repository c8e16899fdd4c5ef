// kf_server.cu — the served form: a request loop over resident sessions.
//
// No counterpart in the reference (its app runs one live session, kinect.cpp:654-695).
// Sessions are admitted while a slot and the device-memory budget allow (each session's
// footprint from kf_session_device_bytes: 4 bytes per FP16+u16 voxel plus its image
// pyramid), keep their volumes, pyramids and poses resident, and queue depth frames as
// they arrive.  Each kf_server_step runs one batched frame step (kf_batch) over the
// sessions that have a frame waiting, oldest waiting frame first, up to the batch size:
// continuous batching, so sessions that arrive while others are on the GPU join the
// next step.  Every frame's latency (arrival to pose available on the host) is recorded
// for the p50/p99 report.  Closed sessions are kept, reset, for the next admission of the
// same volume size (device allocation and release synchronise the GPU, which would stall
// every resident session), and released only when the memory budget needs the room.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>

#include "kf_internal.cuh"

namespace {

double now_s() {
  using clk = std::chrono::steady_clock;
  static const clk::time_point t0 = clk::now();
  return std::chrono::duration<double>(clk::now() - t0).count();
}

struct Frame {
  const uint16_t* d_depth;  // device frame (the session's staging ring or the caller's)
  double t_arrival;
};

struct Slot {
  kf_session* s = nullptr;
  uint64_t bytes = 0;
  std::deque<Frame> queue;
  uint16_t* d_ring = nullptr;  // staging for host-submitted frames
  int ring_next = 0;
  uint64_t done = 0;
  int tracked = 0;
  double pose[16];
  int ring_in_flight = 0;  // host-submitted frames of this session in the step in flight
};

}  // namespace

struct kf_server {
  kf_server_config cfg{};
  std::string last_error;
  std::vector<Slot> slots;   // index = session id; s == nullptr when free
  std::vector<Slot> idle;    // closed sessions kept for reuse (their bytes stay counted)
  uint64_t bytes_in_use = 0;
  kf_batch* batch = nullptr;
  cudaStream_t copy_stream = nullptr;
  std::vector<float> latency_ms;
  uint64_t frames = 0, steps = 0;
  double busy_s = 0.0;
  std::vector<kf_session*> step_sessions;
  std::vector<const uint16_t*> step_frames;
  std::vector<int> step_ids;
  std::vector<int32_t> step_tracked;
  std::vector<double> step_poses;
  int last_n = 0;
  // the asynchronous step in flight (kf_server_step_async): its sessions' ids, their frames'
  // arrival times and whether each frame came from the session's staging ring
  std::vector<int> fl_ids;
  std::vector<double> fl_arrival;
  std::vector<char> fl_ring;
  bool in_flight = false;
};

namespace {

constexpr int kRing = 8;  // host-submitted frames a session may have queued

int sfail(kf_server* v, int code, const std::string& msg) {
  v->last_error = msg;
  return code;
}

Slot* slot_of(kf_server* v, int id) {
  if (!v || id < 0 || id >= (int)v->slots.size() || !v->slots[id].s) return nullptr;
  return &v->slots[id];
}

}  // namespace

extern "C" {

int kf_server_config_default(kf_server_config* c) {
  if (!c) return KF_ERR_INVALID_ARGUMENT;
  std::memset(c, 0, sizeof(*c));
  c->hbm_budget_bytes = 0;  // free device memory at creation, minus 8 GiB
  c->max_sessions = 128;
  c->max_batch = 64;
  c->storage = KF_STORAGE_F16U16;
  c->jtj = KF_JTJ_SPLIT_BF16;
  return KF_OK;
}

int kf_server_create(const kf_server_config* cfg, kf_server** out) {
  if (!cfg || !out) return KF_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (cfg->max_sessions <= 0 || cfg->max_batch <= 0 || cfg->max_batch > KF_BATCH_MAX_SESSIONS)
    return KF_ERR_INVALID_ARGUMENT;
  kf_server* v = new (std::nothrow) kf_server();
  if (!v) return KF_ERR_OUT_OF_MEMORY;
  v->cfg = *cfg;
  if (!v->cfg.hbm_budget_bytes) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      cudaGetLastError();
      delete v;
      return KF_ERR_NO_DEVICE;
    }
    const size_t reserve = (size_t)8 << 30;
    v->cfg.hbm_budget_bytes = free_b > reserve ? free_b - reserve : 0;
  }
  int rc = kf_batch_create(cfg->max_batch, &v->batch);
  if (rc) {
    delete v;
    return rc;
  }
  if (cudaStreamCreateWithFlags(&v->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
    kf_batch_destroy(v->batch);
    delete v;
    return KF_ERR_CUDA;
  }
  v->slots.resize(cfg->max_sessions);
  *out = v;
  return KF_OK;
}

int kf_server_destroy(kf_server* v) {
  if (!v) return KF_ERR_INVALID_ARGUMENT;
  if (v->in_flight && v->batch) kf_batch_sync(v->batch);
  for (auto& sl : v->slots) {
    if (sl.s) kf_destroy(sl.s);
    cudaFree(sl.d_ring);
  }
  for (auto& sl : v->idle) {
    kf_destroy(sl.s);
    cudaFree(sl.d_ring);
  }
  if (v->batch) kf_batch_destroy(v->batch);
  if (v->copy_stream) cudaStreamDestroy(v->copy_stream);
  delete v;
  return KF_OK;
}

const char* kf_server_last_error(const kf_server* v) { return v ? v->last_error.c_str() : "null server"; }

double kf_server_now(void) { return now_s(); }

int kf_server_open(kf_server* v, const kf_config* cfg, const kf_intrinsics* intr, const double pose[16], int* id) {
  if (!v || !cfg || !intr || !pose || !id || !kf_pose_is_finite(pose)) return KF_ERR_INVALID_ARGUMENT;
  kf_config c = *cfg;
  c.storage = v->cfg.storage;
  c.jtj = v->cfg.jtj;
  c.tracking = KF_TRACK_ICP;
  uint64_t need = 0;
  int rc = kf_session_device_bytes(&c, intr, &need);
  if (rc) return sfail(v, rc, "invalid session configuration");
  need += (uint64_t)kRing * intr->width * intr->height * 2;
  int free_slot = -1;
  for (int k = 0; k < (int)v->slots.size(); ++k)
    if (!v->slots[k].s) { free_slot = k; break; }
  if (free_slot < 0) return sfail(v, KF_ERR_ADMISSION, "no free session slot");
  Slot& sl = v->slots[free_slot];
  // a kept session of the same volume and image size is reset instead of allocating
  for (size_t k = 0; k < v->idle.size(); ++k) {
    kf_session* is = v->idle[k].s;
    if (is->cfg.nx == c.nx && is->cfg.ny == c.ny && is->cfg.nz == c.nz && is->intr.width == intr->width &&
        is->intr.height == intr->height && std::memcmp(&is->intr, intr, sizeof(*intr)) == 0) {
      sl = v->idle[k];
      v->idle.erase(v->idle.begin() + k);
      // a fresh session also starts with zero trackSDF rows (read back by Q7)
      if (cudaMemsetAsync(sl.s->d_sdf_rows, 0, (size_t)sl.s->W[0] * sl.s->H[0] * 8 * sizeof(float), sl.s->stream) !=
          cudaSuccess)
        rc = KF_ERR_CUDA;
      if (rc || (rc = kf_set_config(sl.s, &c)) || (rc = kf_reset(sl.s, pose, 0))) {
        v->bytes_in_use -= sl.bytes;
        kf_destroy(sl.s);
        cudaFree(sl.d_ring);
        sl = Slot();
        return sfail(v, rc, "session reuse failed");
      }
      sl.queue.clear();
      sl.ring_next = 0;
      sl.done = 0;
      sl.tracked = 0;
      std::memcpy(sl.pose, pose, sizeof(sl.pose));
      *id = free_slot;
      return KF_OK;
    }
  }
  // release kept sessions (oldest first) until the new one fits the budget
  while (v->bytes_in_use + need > v->cfg.hbm_budget_bytes && !v->idle.empty()) {
    Slot& old = v->idle.front();
    v->bytes_in_use -= old.bytes;
    kf_destroy(old.s);
    cudaFree(old.d_ring);
    v->idle.erase(v->idle.begin());
  }
  if (v->bytes_in_use + need > v->cfg.hbm_budget_bytes) return sfail(v, KF_ERR_ADMISSION, "device memory budget full");
  rc = kf_create(&c, intr, &sl.s);
  if (rc) {
    sl.s = nullptr;
    return sfail(v, rc == KF_ERR_OUT_OF_MEMORY ? KF_ERR_ADMISSION : rc, "session creation failed");
  }
  if (cudaMalloc((void**)&sl.d_ring, (size_t)kRing * intr->width * intr->height * 2) != cudaSuccess) {
    cudaGetLastError();
    kf_destroy(sl.s);
    sl.s = nullptr;
    return sfail(v, KF_ERR_ADMISSION, "session staging allocation failed");
  }
  if ((rc = kf_reset(sl.s, pose, 0))) {
    kf_destroy(sl.s);
    cudaFree(sl.d_ring);
    sl = Slot();
    return sfail(v, rc, "session reset failed");
  }
  sl.bytes = need;
  sl.queue.clear();
  sl.ring_next = 0;
  sl.done = 0;
  sl.tracked = 0;
  std::memcpy(sl.pose, pose, sizeof(sl.pose));
  v->bytes_in_use += need;
  *id = free_slot;
  return KF_OK;
}

int kf_server_prewarm(kf_server* v, const kf_config* cfg, const kf_intrinsics* intr, int count, int* created) {
  if (!v || !cfg || !intr || count < 0) return KF_ERR_INVALID_ARGUMENT;
  if (created) *created = 0;
  kf_config c = *cfg;
  c.storage = v->cfg.storage;
  c.jtj = v->cfg.jtj;
  c.tracking = KF_TRACK_ICP;
  uint64_t need = 0;
  int rc = kf_session_device_bytes(&c, intr, &need);
  if (rc) return sfail(v, rc, "invalid session configuration");
  need += (uint64_t)kRing * intr->width * intr->height * 2;
  const double identity[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  for (int k = 0; k < count; ++k) {
    if (v->bytes_in_use + need > v->cfg.hbm_budget_bytes) return sfail(v, KF_ERR_ADMISSION, "device memory budget full");
    Slot sl;
    if ((rc = kf_create(&c, intr, &sl.s))) return sfail(v, rc, "session creation failed");
    if (cudaMalloc((void**)&sl.d_ring, (size_t)kRing * intr->width * intr->height * 2) != cudaSuccess ||
        (rc = kf_reset(sl.s, identity, 0))) {
      cudaGetLastError();
      kf_destroy(sl.s);
      cudaFree(sl.d_ring);
      return sfail(v, rc ? rc : KF_ERR_OUT_OF_MEMORY, "session creation failed");
    }
    sl.bytes = need;
    v->bytes_in_use += need;
    v->idle.push_back(sl);
    if (created) *created += 1;
  }
  return KF_OK;
}

int kf_server_close(kf_server* v, int id) {
  Slot* sl = slot_of(v, id);
  if (!sl) return KF_ERR_INVALID_ARGUMENT;
  if (v->in_flight && std::find(v->fl_ids.begin(), v->fl_ids.end(), id) != v->fl_ids.end()) {
    // the session is in the step in flight: finish that step first (its results are then
    // what kf_server_last_step describes)
    int n = 0;
    if (int rc = kf_server_sync(v, &n)) return rc;
  }
  sl->queue.clear();
  v->idle.push_back(*sl);  // kept for reuse; its bytes stay counted
  *sl = Slot();
  return KF_OK;
}

int kf_server_submit(kf_server* v, int id, const uint16_t* host_depth_mm) {
  Slot* sl = slot_of(v, id);
  if (!sl || !host_depth_mm) return KF_ERR_INVALID_ARGUMENT;
  int host_queued = sl->ring_in_flight;  // a frame in flight still occupies its ring slot
  for (const Frame& f : sl->queue)
    if (f.d_depth >= sl->d_ring && f.d_depth < sl->d_ring + (size_t)kRing * sl->s->W[0] * sl->s->H[0]) ++host_queued;
  if (host_queued >= kRing) return sfail(v, KF_ERR_CAPACITY, "session frame queue full");
  const size_t px = (size_t)sl->s->W[0] * sl->s->H[0];
  uint16_t* dst = sl->d_ring + (size_t)sl->ring_next * px;
  sl->ring_next = (sl->ring_next + 1) % kRing;
  if (cudaMemcpyAsync(dst, host_depth_mm, px * 2, cudaMemcpyHostToDevice, v->copy_stream) != cudaSuccess) {
    cudaGetLastError();
    return sfail(v, KF_ERR_CUDA, "frame upload failed");
  }
  sl->queue.push_back(Frame{dst, now_s()});
  return KF_OK;
}

int kf_server_submit_device(kf_server* v, int id, const uint16_t* device_depth_mm) {
  Slot* sl = slot_of(v, id);
  if (!sl || !device_depth_mm) return KF_ERR_INVALID_ARGUMENT;
  sl->queue.push_back(Frame{device_depth_mm, now_s()});
  return KF_OK;
}

}  // extern "C"

namespace {

// Records the results of the step in flight (its poses and flags are the batch's last
// read step): per-frame latency, the sessions' poses and counts.
void complete_in_flight(kf_server* v, int* n_done) {
  const int n = (int)v->fl_ids.size();
  const double t = now_s();
  v->step_ids = v->fl_ids;
  v->step_tracked.resize(n);
  v->step_poses.resize((size_t)16 * n);
  kf_batch_get_poses(v->batch, n, v->step_poses.data());
  kf_batch_get_tracked(v->batch, n, v->step_tracked.data());
  float ms[5] = {0, 0, 0, 0, 0};
  kf_batch_get_stage_times(v->batch, ms);
  v->busy_s += (ms[0] + ms[1] + ms[2] + ms[3] + ms[4]) / 1000.0;
  for (int e = 0; e < n; ++e) {
    Slot& sl = v->slots[v->fl_ids[e]];
    v->latency_ms.push_back((float)(1000.0 * (t - v->fl_arrival[e])));
    if (v->fl_ring[e]) sl.ring_in_flight -= 1;
    sl.done += 1;
    sl.tracked = v->step_tracked[e];
    std::memcpy(sl.pose, &v->step_poses[(size_t)16 * e], sizeof(sl.pose));
  }
  v->last_n = n;
  v->frames += (uint64_t)n;
  v->steps += 1;
  v->in_flight = false;
  v->fl_ids.clear();
  if (n_done) *n_done = n;
}

// One batched step over the sessions with a waiting frame (oldest waiting frame first, up
// to max_batch).  async: the step is enqueued and the previous one completed (when no frame
// waits, the step in flight is waited for); otherwise the step is run to completion.
int server_step(kf_server* v, bool async, int* n_done) {
  if (!v) return KF_ERR_INVALID_ARGUMENT;
  if (n_done) *n_done = 0;
  // sessions with a waiting frame, oldest waiting frame first
  std::vector<int> ids;
  for (int k = 0; k < (int)v->slots.size(); ++k)
    if (v->slots[k].s && !v->slots[k].queue.empty()) ids.push_back(k);
  if (ids.empty()) {
    if (v->in_flight) {
      if (int rc = kf_batch_sync(v->batch)) {
        v->in_flight = false;
        return sfail(v, rc, std::string("batch step: ") + kf_batch_last_error(v->batch));
      }
      complete_in_flight(v, n_done);
    } else {
      v->last_n = 0;
    }
    return KF_OK;
  }
  std::stable_sort(ids.begin(), ids.end(), [&](int a, int b) {
    return v->slots[a].queue.front().t_arrival < v->slots[b].queue.front().t_arrival;
  });
  if ((int)ids.size() > v->cfg.max_batch) ids.resize(v->cfg.max_batch);
  // a stable member order keeps the batch's argument tables (and its step graphs) from being
  // rebuilt when the same sessions step again
  std::sort(ids.begin(), ids.end());
  const int n = (int)ids.size();
  v->step_sessions.resize(n);
  v->step_frames.resize(n);
  std::vector<double> arrival(n);
  std::vector<char> ring(n);
  for (int e = 0; e < n; ++e) {
    Slot& sl = v->slots[ids[e]];
    const Frame f = sl.queue.front();
    sl.queue.pop_front();
    v->step_sessions[e] = sl.s;
    v->step_frames[e] = f.d_depth;
    arrival[e] = f.t_arrival;
    ring[e] = f.d_depth >= sl.d_ring && f.d_depth < sl.d_ring + (size_t)kRing * sl.s->W[0] * sl.s->H[0];
    if (ring[e]) sl.ring_in_flight += 1;
  }
  if (cudaStreamSynchronize(v->copy_stream) != cudaSuccess) return sfail(v, KF_ERR_CUDA, "frame upload failed");
  // enqueue this step; the batch completes the previous one (its results are then readable)
  const int rc = kf_batch_frame_step_u16_device_async(v->batch, v->step_sessions.data(), v->step_frames.data(), n);
  const bool had = v->in_flight;
  if (had && !rc) complete_in_flight(v, n_done);
  v->fl_ids = ids;
  v->fl_arrival = arrival;
  v->fl_ring = ring;
  v->in_flight = true;
  if (rc) {
    v->in_flight = false;
    v->fl_ids.clear();
    return sfail(v, rc, std::string("batch step: ") + kf_batch_last_error(v->batch));
  }
  if (!async) {
    // synchronous: wait for this step and return its results
    if (int r = kf_batch_sync(v->batch)) {
      v->in_flight = false;
      return sfail(v, r, std::string("batch step: ") + kf_batch_last_error(v->batch));
    }
    int done_now = 0;
    complete_in_flight(v, &done_now);
    if (n_done) *n_done += done_now;
  }
  return KF_OK;
}

}  // namespace

extern "C" {

int kf_server_step(kf_server* v, int* n_done) { return server_step(v, false, n_done); }

int kf_server_step_async(kf_server* v, int* n_done) { return server_step(v, true, n_done); }

int kf_server_sync(kf_server* v, int* n_done) {
  if (!v) return KF_ERR_INVALID_ARGUMENT;
  if (n_done) *n_done = 0;
  if (!v->in_flight) return KF_OK;
  if (int rc = kf_batch_sync(v->batch)) {
    v->in_flight = false;
    return sfail(v, rc, std::string("batch step: ") + kf_batch_last_error(v->batch));
  }
  complete_in_flight(v, n_done);
  return KF_OK;
}

int kf_server_get_pose(kf_server* v, int id, double pose[16], int* tracked, uint64_t* frames_done) {
  Slot* sl = slot_of(v, id);
  if (!sl) return KF_ERR_INVALID_ARGUMENT;
  if (pose) std::memcpy(pose, sl->pose, sizeof(sl->pose));
  if (tracked) *tracked = sl->tracked;
  if (frames_done) *frames_done = sl->done;
  return KF_OK;
}

int kf_server_last_step(kf_server* v, int max_n, int* ids, double* poses, int32_t* tracked, int* n) {
  if (!v || !n || max_n < 0) return KF_ERR_INVALID_ARGUMENT;
  const int k = std::min(max_n, v->last_n);
  for (int e = 0; e < k; ++e) {
    if (ids) ids[e] = v->step_ids[e];
    if (poses) std::memcpy(poses + 16 * e, &v->step_poses[(size_t)16 * e], 16 * sizeof(double));
    if (tracked) tracked[e] = v->step_tracked[e];
  }
  *n = k;
  return KF_OK;
}

int kf_server_pending(kf_server* v, int id, int* queued) {
  Slot* sl = slot_of(v, id);
  if (!sl || !queued) return KF_ERR_INVALID_ARGUMENT;
  *queued = (int)sl->queue.size();
  return KF_OK;
}

int kf_server_stats(kf_server* v, kf_server_stats_t* st) {
  if (!v || !st) return KF_ERR_INVALID_ARGUMENT;
  std::memset(st, 0, sizeof(*st));
  st->frames = v->frames;
  st->steps = v->steps;
  st->busy_s = v->busy_s;
  st->bytes_in_use = v->bytes_in_use;
  int active = 0;
  for (const auto& sl : v->slots)
    if (sl.s) ++active;
  st->active_sessions = active;
  if (!v->latency_ms.empty()) {
    std::vector<float> l = v->latency_ms;
    auto pct = [&](double p) {
      const size_t k = std::min(l.size() - 1, (size_t)(p * (l.size() - 1) + 0.5));
      std::nth_element(l.begin(), l.begin() + k, l.end());
      return (double)l[k];
    };
    st->p50_ms = pct(0.50);
    st->p99_ms = pct(0.99);
    st->max_ms = (double)*std::max_element(l.begin(), l.end());
  }
  return KF_OK;
}

int kf_server_reset_stats(kf_server* v) {
  if (!v) return KF_ERR_INVALID_ARGUMENT;
  v->latency_ms.clear();
  v->frames = v->steps = 0;
  v->busy_s = 0.0;
  return KF_OK;
}

}  // extern "C"
