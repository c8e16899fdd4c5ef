// kf_gfusion.hpp — header-only C++ classes over the C ABI (kf.h) with the method names of
// the reference's gFusion (include/gFusion.h:124-624) and MCubes (include/mcubes.h:48-168).
//
// Differences a caller sees: GL texture/buffer names become host copies (std::vector) or a
// device view (kf_volume_view); errors throw kf::Error carrying the kf status code and the
// library's message instead of the reference's exit(); poses are column-major float[16]
// (glm layout) or double[16].
#ifndef KF_GFUSION_HPP
#define KF_GFUSION_HPP

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "kf.h"

namespace kf {

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string& what)
      : std::runtime_error(what + ": " + kf_status_string(status)), status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

using Pose = std::array<double, 16>;  // camera-to-world, column-major

inline Pose identity() { return {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1}; }

inline Pose from_float(const float* m) {
  Pose p;
  for (int i = 0; i < 16; ++i) p[i] = m[i];
  return p;
}

// gFusionConfig (gFusion.h:42-82) with the defaults of its constructor.
inline kf_config default_config() {
  kf_config c;
  kf_config_default(&c);
  return c;
}

class GFusion {
 public:
  GFusion(const kf_config& cfg, const kf_intrinsics& intr) : intr_(intr) {
    check(kf_create(&cfg, &intr, &s_), "kf_create");
  }
  ~GFusion() {
    if (s_) kf_destroy(s_);
  }
  GFusion(const GFusion&) = delete;
  GFusion& operator=(const GFusion&) = delete;

  // ---- configuration / reset ----
  void setConfig(const kf_config& c) { check(kf_set_config(s_, &c), "kf_set_config"); }
  void Reset(const Pose& pose, bool deleteFlag) { check(kf_reset(s_, pose.data(), deleteFlag), "kf_reset"); }
  void resetVolume() { check(kf_reset_volume(s_), "kf_reset_volume"); }
  void resetPose(const Pose& pose) { check(kf_reset_pose(s_, pose.data()), "kf_reset_pose"); }
  Pose getPose() {
    Pose p;
    check(kf_get_pose(s_, p.data()), "kf_get_pose");
    return p;
  }
  void setPose(const Pose& p) { check(kf_set_pose(s_, p.data()), "kf_set_pose"); }

  // ---- per frame ----
  void depthToVertex(const float* depthArray) {
    check(kf_depth_to_vertex_f32(s_, depthArray), "kf_depth_to_vertex_f32");
  }
  void depthToVertex(const uint16_t* depthMm) { check(kf_depth_to_vertex_u16(s_, depthMm), "kf_depth_to_vertex_u16"); }
  void vertexToNormal() { check(kf_vertex_to_normal(s_), "kf_vertex_to_normal"); }
  // depth ingest before the pyramid: libfreenect2-style undistortion, filter3D.cs
  void setDepthUndistortion(const kf_ir_camera* ir) {
    check(kf_set_depth_undistortion(s_, ir), "kf_set_depth_undistortion");
  }
  void setDepthFilter(bool enable) { check(kf_set_depth_filter(s_, enable ? 1 : 0), "kf_set_depth_filter"); }
  bool Track() {
    int t = 0;
    check(kf_track_icp(s_, &t), "kf_track_icp");
    return t != 0;
  }
  bool TrackSDF() {
    int t = 0;
    check(kf_track_sdf(s_, &t), "kf_track_sdf");
    return t != 0;
  }
  bool recoverPose() {
    int f = 0;
    check(kf_recover_pose(s_, &f), "kf_recover_pose");
    return f != 0;
  }
  void integrate() { check(kf_integrate(s_), "kf_integrate"); }
  void raycast() { check(kf_raycast(s_), "kf_raycast"); }
  // the body of the reference's main loop (kinect.cpp:654-695)
  bool frameStep(const uint16_t* depthMm) {
    int t = 0;
    check(kf_frame_step_u16(s_, depthMm, &t), "kf_frame_step_u16");
    return t != 0;
  }
  // pipelined loop body: enqueues this frame (depthMm must stay unchanged until the next
  // call) and reads the previous frame's result, returned by lastResult(); frameSync()
  // reads the frame still in flight
  void frameStepAsync(const uint16_t* depthMm) {
    check(kf_frame_step_u16_async(s_, depthMm), "kf_frame_step_u16_async");
  }
  bool frameSync() {
    int t = 0;
    check(kf_frame_sync(s_, &t), "kf_frame_sync");
    return t != 0;
  }
  std::pair<Pose, bool> lastResult() {
    Pose p;
    int t = 0;
    check(kf_get_last_result(s_, p.data(), &t), "kf_get_last_result");
    return {p, t != 0};
  }
  // launch shapes for this volume and GPU (results do not depend on them)
  kf_launch_shape autotune(int repeats = 5) {
    kf_launch_shape sh{};
    check(kf_autotune(s_, repeats, &sh, nullptr), "kf_autotune");
    return sh;
  }

  // ---- accessors (the reference returns GL names; these return data) ----
  std::vector<float> getVerts() { return raycast_map(true); }
  std::vector<float> getNorms() { return raycast_map(false); }
  kf_volume_view getVolume() {
    kf_volume_view v;
    check(kf_get_volume(s_, &v), "kf_get_volume");
    return v;
  }
  std::array<double, 6> getCumTwist() {
    std::array<double, 6> t;
    check(kf_get_cum_twist(s_, t.data()), "kf_get_cum_twist");
    return t;
  }
  std::array<double, 3> getTransPose() {
    Pose p = getPose();
    return {p[12], p[13], p[14]};
  }
  // intensityProjection (gFusion.cpp:1368-1409): W*H RGBA floats, (ray sum, 0, 0, 1)
  std::vector<float> intensityProjection() {
    std::vector<float> m((size_t)intr_.width * intr_.height * 4);
    check(kf_intensity_projection(s_, m.data()), "kf_intensity_projection");
    return m;
  }
  // volume checkpoint: the session steps on from a loaded file exactly as it would have
  void saveVolume(const std::string& path) { check(kf_save_volume(s_, path.c_str()), "kf_save_volume"); }
  void loadVolume(const std::string& path) { check(kf_load_volume(s_, path.c_str()), "kf_load_volume"); }
  std::array<float, 6> getTimes() {
    std::array<float, 6> t;
    check(kf_get_stage_times(s_, t.data()), "kf_get_stage_times");
    return t;
  }
  // which frame steps record their stage boundaries (every 1, 2 or 4; 0 = none)
  void setStageTiming(int every) { check(kf_set_stage_timing(s_, every), "kf_set_stage_timing"); }
  kf_session* handle() { return s_; }

 private:
  std::vector<float> raycast_map(bool vertex) {
    std::vector<float> m((size_t)intr_.width * intr_.height * 4);
    check(kf_get_raycast(s_, vertex ? m.data() : nullptr, vertex ? nullptr : m.data()), "kf_get_raycast");
    return m;
  }
  void check(int st, const char* what) {
    if (st != KF_OK) throw Error(st, std::string(what) + (s_ ? std::string(" (") + kf_last_error(s_) + ")" : ""));
  }
  kf_session* s_ = nullptr;
  kf_intrinsics intr_;
};

class MCubes {
 public:
  explicit MCubes(GFusion& f) : f_(&f) {}
  void setVolumeTexture(GFusion& f) { f_ = &f; }
  void setIsolevel(float iso) { iso_ = iso; }
  void generateMarchingCubes(int method = KF_MC_HISTOPYRAMID) {
    int st = kf_mc_extract(f_->handle(), iso_, method, &ntri_);
    if (st) throw Error(st, "kf_mc_extract");
  }
  int getNumberTriangles() const { return (int)(3 * ntri_); }  // m_totalSum: vertices
  std::vector<float> getPositions() {
    std::vector<float> v((size_t)ntri_ * 12);
    int st = kf_mc_copy_vertices(f_->handle(), v.data(), (uint64_t)ntri_ * 3);
    if (st) throw Error(st, "kf_mc_copy_vertices");
    return v;
  }
  void exportMesh(const std::string& path) {
    int st = kf_mc_export_stl(f_->handle(), path.c_str());
    if (st) throw Error(st, "kf_mc_export_stl");
  }
  void exportPointCloud(const std::string& path) {
    int st = kf_mc_export_ply(f_->handle(), path.c_str());
    if (st) throw Error(st, "kf_mc_export_ply");
  }

 private:
  GFusion* f_;
  float iso_ = 0.0f;
  uint32_t ntri_ = 0;
};

}  // namespace kf

#endif  // KF_GFUSION_HPP
