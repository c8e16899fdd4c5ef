/*
 * kf_oracle.h — FP64 CPU oracle for the KinectFusion hot path (test infrastructure).
 *
 * THIS IS TEST INFRASTRUCTURE, NOT PRODUCT CODE.  It restates, in scalar FP64 C++ with
 * OpenMP, the GLSL compute shaders and the gFusion / MCubes host logic of
 * philipNoonan/oglFusionKinectV2 (file:line citations at each function in
 * kf_oracle.cpp).  Only the tests, the smoke check and the CPU-baseline leg of the bench
 * may load it, and only as the checker or the timed CPU baseline.
 *
 * Parity status: the reference cannot be built or run on this machine (OpenGL 4.3 GLSL
 * compute shaders; no graphics stack, no Eigen/glm) and it ships no tests, golden vectors
 * or fixtures.  This oracle is therefore "parity unpinned" against the reference's own
 * outputs: it is pinned only by analytic known-answer tests (tests/test_oracle_kat.py)
 * and by the marching-cubes table consistency facts.
 *
 * The API mirrors include/kf.h so that the tests can drive both sides with one script.
 * Volumes use the same byte layout as the CUDA path (KF_STORAGE_*), so a volume can be
 * copied between the two and compared byte for byte.
 */
#ifndef KF_ORACLE_H
#define KF_ORACLE_H
#include <stdint.h>
#include "../include/kf.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_session or_session;

int or_create(const kf_config* cfg, const kf_intrinsics* intr, or_session** out);
int or_destroy(or_session* s);
int or_set_threads(int n);  /* OpenMP threads (0 = all) */
int or_get_threads(void);

int or_reset(or_session* s, const double pose[16], int delete_flag);
int or_reset_pose(or_session* s, const double pose[16]);
int or_set_pose(or_session* s, const double pose[16]);
int or_get_pose(or_session* s, double pose[16]);
int or_get_pose_eig(or_session* s, double pose[16]);
int or_set_pose_eig(or_session* s, const double pose[16]);

int or_depth_to_vertex_f32(or_session* s, const float* depth_mm);
int or_depth_to_vertex_u16(or_session* s, const uint16_t* depth_mm);
int or_vertex_to_normal(or_session* s);
/* Depth ingest before the pyramid: libfreenect2 Registration undistortion with the IR
 * camera (fx, fy, cx, cy, k1, k2, k3, p1, p2; NULL turns it off) and filter3D.cs. */
int or_set_depth_undistortion(or_session* s, const float ir[9]);
int or_set_depth_filter(or_session* s, int enable);
int or_get_undistortion_map(or_session* s, int32_t* map);

int or_track_icp(or_session* s, int* tracked);
int or_track_sdf(or_session* s, int* tracked);
int or_recover_pose(or_session* s, int* found);
int or_get_alignment_energy(or_session* s, double* ae);
int or_get_reduction(or_session* s, double sums[32]);
/* One ICP iteration at `level` with the current pose: track + reduce only. */
int or_icp_reduce_once(or_session* s, int level, double sums[32]);
/* One trackSDF + reduceSDF at `level` for the given camera-to-world pose. */
int or_sdf_reduce_once(or_session* s, int level, const double cam_to_world[16], double sums[32]);

int or_integrate(or_session* s);
int or_raycast(or_session* s);
/* intensityProjection (gFusion.cpp:1368-1409, mip.cs): W*H*4 doubles, (sum, 0, 0, 1). */
int or_intensity_projection(or_session* s, double* rgba);
int or_frame_step_u16(or_session* s, const uint16_t* depth_mm, int* tracked);

int or_get_raycast(or_session* s, double* vertex4, double* normal4);
int or_set_raycast(or_session* s, const double* vertex4, const double* normal4);
int or_get_vertex_map(or_session* s, int level, double* vertex4);
int or_get_normal_map(or_session* s, int level, double* normal4);
int or_set_vertex_normal_map(or_session* s, int level, const double* vertex4,
                             const double* normal4);
int or_get_depth_map(or_session* s, int level, double* depth_mm);
int or_get_track_status(or_session* s, int level, int32_t* status);
int or_copy_volume_to_host(or_session* s, void* dst, uint64_t bytes);
int or_copy_volume_from_host(or_session* s, const void* src, uint64_t bytes);
int or_get_pose_library_size(or_session* s, int* n);
int or_get_cum_twist(or_session* s, double twist[6]);

int or_mc_extract(or_session* s, float iso, int method, uint32_t* n_triangles);
int or_mc_copy_vertices(or_session* s, float* vertex4, uint64_t max_vertices);
int or_mc_copy_normals(or_session* s, float* n, uint64_t max_vertices);
int or_mc_extract_mesh(or_session* s, float iso, uint32_t* nv, uint32_t* nt);
int or_mc_copy_mesh(or_session* s, float* pos, float* nrm, uint32_t* idx);
int or_mc_copy_base_level(or_session* s, uint32_t* base, uint64_t count);
int or_mc_export_stl(or_session* s, const char* path);
int or_mc_export_ply(or_session* s, const char* path);

/* Exclusive scan (uint32 wrap-around), *total = sum of the input. */
int or_prefix_sum_u32(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* total);

/* Pose helpers, exposed for unit tests. */
void or_euler_xyz(const double angles[3], double R[9]);        /* Rx*Ry*Rz, column-major */
void or_se3_exp(const double xi[6], double T[16]);             /* xi = (w, v)            */
int or_solve_pinv6(const double C[36], const double b[6], double x[6]);
int or_solve_icp_guarded6(const double C[36], const double b[6], double x[6]);
int or_solve_ldlt6(const double C[36], const double b[6], double x[6]);

/* Marching-cubes tables as seen by the build (table self-consistency test). */
int or_mc_tables(uint16_t edge[256], int8_t tri[256 * 16], uint8_t nverts[256],
                 uint8_t ntri[256], uint8_t offsets3[72]);

#ifdef __cplusplus
}
#endif
#endif
