/*
 * kf.h — C ABI of the B200 KinectFusion core.
 *
 * This is the drop-in boundary for the compute path of philipNoonan/oglFusionKinectV2:
 * the `gFusion` class (include/gFusion.h:124-624, src/gFusion.cpp) and the `MCubes`
 * class (include/mcubes.h:48-168, src/mcubes.cpp).  Every entry point below names the
 * reference member it replaces.  The reference has no FFI of its own (it is one
 * in-process C++ class used by src/kinect.cpp), so these are the calls such a binding
 * would make: plain pointers and sizes, POD structs, int status codes, no exceptions and
 * no process exit across the boundary (the reference calls exit() on shader errors,
 * src/gFusion.cpp:69-72, src/mcubes.cpp:32-35; here that is KF_ERR_*).
 *
 * Conventions
 *   - Poses are camera-to-world 4x4 matrices, column-major (glm layout, the reference's
 *     m_pose), passed as double[16].  The device keeps the pose in FP64.
 *   - The volume covers world [0, dim]^3 (raycast.cs:141-143); voxel (x,y,z) has its
 *     centre at ((x+0.5)*dim_x/nx, ...) (integrate.cs:16-19) and linear index
 *     x + nx*(y + ny*z) in each of its two planes (values, then weights).
 *   - Maps are row-major W x H (level l: (W>>l) x (H>>l)) of float4 (RGBA32F textures).
 *   - Every call is enqueued on the session's own CUDA stream; calls that return data to
 *     the host synchronise that stream first.  One session is used by one host thread.
 */
#ifndef KF_H
#define KF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KF_ABI_VERSION 2

#if defined(KF_BUILDING_LIBRARY) && defined(__GNUC__)
#define KF_API __attribute__((visibility("default")))
#else
#define KF_API
#endif

/* ---- status codes ------------------------------------------------------------------ */
#define KF_OK 0
#define KF_ERR_INVALID_ARGUMENT (-1)
#define KF_ERR_OUT_OF_MEMORY (-2)
#define KF_ERR_CUDA (-3)
#define KF_ERR_NO_DEVICE (-4)
#define KF_ERR_TIMEOUT (-5)       /* a bounded device-side wait gave up */
#define KF_ERR_STATE (-6)         /* call out of order (e.g. export before extract) */
#define KF_ERR_IO (-7)            /* file could not be written */
#define KF_ERR_CAPACITY (-8)      /* output larger than the caller's buffer / static limit */
#define KF_ERR_ADMISSION (-9)     /* not enough free device memory for a new session */

/* ---- volume storage (gFusion.cpp:223 uses GL_RG16I) --------------------------------- */
#define KF_STORAGE_F32F32 0 /* float TSDF + float weight, 8 B/voxel                     */
#define KF_STORAGE_F16U16 1 /* half TSDF + uint16 weight, 4 B/voxel (FP32 update math)  */
#define KF_STORAGE_RG16I 2  /* int16 TSDF*32766 + int16 weight, 4 B/voxel (reference)   */

/* ---- J^T J contraction ----------------------------------------------------------- */
#define KF_JTJ_FP32 0       /* FP32 FMAs on the CUDA cores                                */
#define KF_JTJ_SPLIT_BF16 1 /* split-BF16 (hi+lo) tensor-core mma, FP32 accumulation      */

/* ---- tracking mode (kinect.h:143-144 trackDepthToPoint / trackDepthToVolume) ------- */
#define KF_TRACK_ICP 0
#define KF_TRACK_SDF 1

/* ---- reference behaviours that can be reproduced ("faithful") or fixed ("clean") -----
 * Each bit, when set, reproduces the reference behaviour named beside it.            */
#define KF_Q1_LAST_GROUP_ONLY (1u << 0)  /* getReduction keeps only rows y%8==7,        \
                                            gFusion.cpp:1143-1149, 1206-1212             */
#define KF_Q3_DOWN_FROM_LEFT (1u << 1)   /* vertToNorm "down" reads column x-1,          \
                                            vertToNorm.cs:26                             */
#define KF_Q6_SDF_D2_TWICE (1u << 2)     /* reduceSDF adds D^2 twice, reduceSDF.cs:52,60 */
#define KF_Q7_SDF_LAST_COLUMN (1u << 3)  /* trackSDF skips x=W-1, the reduction reads   \
                                            the stale row, trackSDF.cs:413               */
#define KF_Q13_MC_FIRST_SEVEN (1u << 4)  /* MC "positive found" ignores corner 7,        \
                                            histoPyramids.cs:140                          */
#define KF_Q15_MC_BORDER_SKIP (1u << 5)  /* MC classify skips cubes within 10 of the     \
                                            border, histoPyramids.cs:117-120              */
#define KF_Q18_STL_COUNT_X4 (1u << 6)    /* STL header count = 4x triangles,             \
                                            mcubes.cpp:451-457                            */
#define KF_Q23_SDF_XY_OFFSET (1u << 7)   /* trackSDF subtracts 0.5 twice from x and y of \
                                            the voxel coordinate, trackSDF.cs:429         */
#define KF_Q8_NARROW_BAND (1u << 9)     /* integrate keeps a value only while the running \
                                            average is below 0.2, clamped to [-0.1, 0.2]; \
                                            clear: the reference's earlier update, clamp  \
                                            to [-1, 1] (integrate.cs:80-113 vs 115-150)   */
#define KF_Q4_SAME_PIXEL (1u << 10)      /* ICP projects with the current estimate, so   \
                                            the association is the same pixel; clear:    \
                                            project with the raycast (previous) pose,    \
                                            gFusion.cpp:747-755                          */
#define KF_Q19_EIG_TRANSLATION (1u << 8) /* resetPose seeds the SDF pose chain with the     \
                                            translation only, gFusion.cpp:275-287         */
#define KF_Q24_MC_SHADER_UNITS (1u << 11) /* the scan (classic) marching-cubes path writes  \
                                            marchingCubes.cs's units: corners at           \
                                            -1 + gridPos * voxelSize, vertex / 128 *       \
                                            voxelSize.x with z negated, w = 1, voxelSize = \
                                            1000 * dim / size (mcubes.h:30-39); clear:     \
                                            voxel-index units (marchingCubes.cs:205-299)   */
/* Exactly the reference's behaviour. */
#define KF_QUIRKS_REFERENCE                                                                  \
  (KF_Q1_LAST_GROUP_ONLY | KF_Q3_DOWN_FROM_LEFT | KF_Q4_SAME_PIXEL | KF_Q6_SDF_D2_TWICE |      \
   KF_Q7_SDF_LAST_COLUMN | KF_Q8_NARROW_BAND | KF_Q13_MC_FIRST_SEVEN | KF_Q15_MC_BORDER_SKIP |  \
   KF_Q19_EIG_TRANSLATION | KF_Q23_SDF_XY_OFFSET)
/* Default: the reference, with the J^T J reduction over the whole image (Q1 cleared). */
#define KF_QUIRKS_DEFAULT (KF_QUIRKS_REFERENCE & ~KF_Q1_LAST_GROUP_ONLY)
/* Default with projective association from the raycast pose and the reference's earlier
 * [-1, 1] TSDF update (Q4, Q8 cleared): with a truncation of a few voxels the reference's
 * 0.2*mu band is thinner than a voxel and same-pixel association biases every step. */
#define KF_QUIRKS_TRACKING (KF_QUIRKS_DEFAULT & ~(KF_Q4_SAME_PIXEL | KF_Q8_NARROW_BAND))

/* ---- marching-cubes method ---------------------------------------------------------- */
#define KF_MC_HISTOPYRAMID 0 /* histoPyramids.cs + traverseHistoPyramids.cs (live path)   */
#define KF_MC_SCAN 1         /* marchingCubes.cs classify/compact/generate + prefix sum   */

/* gFusionConfig (include/gFusion.h:42-82) plus the storage/precision/quirk policy. */
typedef struct kf_config {
  int32_t nx, ny, nz;         /* volumeSize, voxels                                        */
  float dim_x, dim_y, dim_z;  /* volumeDimensions, metres                                  */
  float mu;                   /* truncation, metres                                        */
  float max_weight;           /* maxWeight                                                 */
  float near_plane, far_plane;/* raycast clip, metres                                      */
  float dist_threshold;       /* ICP gating distance, metres                               */
  float normal_threshold;     /* ICP gating normal dot                                     */
  int32_t iterations[3];      /* per pyramid level, index 0 = finest (gFusion.cpp:661-666) */
  int32_t storage;            /* KF_STORAGE_*                                              */
  int32_t jtj;                /* KF_JTJ_*                                                  */
  int32_t tracking;           /* KF_TRACK_*                                                */
  uint32_t quirks;            /* KF_Q*                                                     */
  int32_t integrate_every;    /* counter % integrate_every == 0 (kinect.cpp:677, 1)        */
  int32_t reserved[7];
} kf_config;

/* Depth camera intrinsics; setCameraParams(vec4(fx, fy, cx, cy)) (gFusion.h:184-188). */
typedef struct kf_intrinsics {
  float fx, fy, cx, cy;
  int32_t width, height; /* 512 x 424 for the Kinect v2 (gFusion.h:555-556) */
} kf_intrinsics;

/* Non-owning view of the TSDF volume (replaces getVolume() -> GL texture name).
 * The volume is two planes: nx*ny*nz TSDF values (x fastest), then as many weights.
 * F32F32: float + float; F16U16: IEEE half + uint16; RG16I: int16 (TSDF*32766) + int16. */
typedef struct kf_volume_view {
  void* device_ptr;            /* value plane, for reading; valid until kf_reset(.., 1)  */
                               /* or kf_destroy.  New contents go in through            */
                               /* kf_copy_volume_from_host, which also refreshes the    */
                               /* per-8^3-brick summary that kf_raycast skips by.       */
  int32_t nx, ny, nz;
  int32_t storage;             /* KF_STORAGE_*                                           */
  int64_t value_bytes;         /* bytes per value (and per weight): 4 or 2              */
  int64_t weight_offset_bytes; /* weight plane = device_ptr + weight_offset_bytes       */
  int64_t row_pitch_bytes;     /* nx * value_bytes                                      */
  int64_t slice_pitch_bytes;   /* nx * ny * value_bytes                                 */
} kf_volume_view;

typedef struct kf_session kf_session;

/* ---- library --------------------------------------------------------------------- */
KF_API int kf_abi_version(void);
KF_API const char* kf_status_string(int status);
/* gFusionConfig() defaults (gFusion.h:56-69) with storage F32F32, FP32 J^T J, ICP. */
KF_API int kf_config_default(kf_config* cfg);

/* ---- lifecycle: initTextures/initVolume/allocateBuffers (gFusion.cpp:200-383) ------ */
KF_API int kf_create(const kf_config* cfg, const kf_intrinsics* intr, kf_session** out);
KF_API int kf_destroy(kf_session* s);
KF_API const char* kf_last_error(const kf_session* s);
/* Bytes a session with this config holds on the device (admission control). */
KF_API int kf_session_device_bytes(const kf_config* cfg, const kf_intrinsics* intr, uint64_t* bytes);

/* Reset(pose, deleteFlag) (gFusion.cpp:226-240): zero or reallocate the volume, clear
 * the pose library, resetPose(pose). */
KF_API int kf_reset(kf_session* s, const double pose[16], int delete_flag);
KF_API int kf_reset_volume(kf_session* s);                 /* resetVolume, gFusion.cpp:242-273 */
KF_API int kf_reset_pose(kf_session* s, const double pose[16]); /* resetPose, :275-287 */
KF_API int kf_set_pose(kf_session* s, const double pose[16]);   /* setPose, gFusion.h:177-180 */
KF_API int kf_get_pose(kf_session* s, double pose[16]);         /* getPose, gFusion.h:173-176 */
KF_API int kf_set_config(kf_session* s, const kf_config* cfg);  /* setConfig (same volume size) */

/* ---- depth ingest: depthToVertex (gFusion.cpp:496-526) ------------------------------
 * Uploads one depth frame, builds the 3-level mip pyramid (2x2 box mean including zeros,
 * glGenerateMipmap at :508) and the vertex maps.  _f32 takes millimetres as float (the
 * reference's input); _u16 takes uint16 millimetres; _device reads a device pointer. */
KF_API int kf_depth_to_vertex_f32(kf_session* s, const float* host_depth_mm);
KF_API int kf_depth_to_vertex_u16(kf_session* s, const uint16_t* host_depth_mm);
KF_API int kf_depth_to_vertex_u16_device(kf_session* s, const uint16_t* device_depth_mm);
KF_API int kf_vertex_to_normal(kf_session* s); /* vertexToNormal, gFusion.cpp:528-547 */

/* ---- depth ingest stages before the pyramid (both off by default) --------------------
 * IR (depth) camera of the Kinect v2 as libfreenect2 describes it
 * (Freenect2Device::IrCameraParams), set by the reference from its calibration file
 * (src/interface.cpp:239-272, src/kinect.cpp:82-160). */
typedef struct kf_ir_camera {
  float fx, fy, cx, cy;
  float k1, k2, k3; /* radial distortion */
  float p1, p2;     /* tangential distortion */
} kf_ir_camera;
/* Undistort every frame before the pyramid, as libfreenect2's Registration::apply makes
 * the `undistorted` depth the reference fuses (src/interface.cpp:290-313; libfreenect2
 * fork at commit 0ee1ee2f): each pixel takes the raw depth at its distorted position
 * (Brown-Conrady model in float, rounded as (int)(m + 0.5f)), 0 where that falls outside
 * the image.  NULL turns it off.  Applies to every kf_depth_to_vertex_* and frame step of
 * this session (not to batched steps, which refuse such sessions). */
KF_API int kf_set_depth_undistortion(kf_session* s, const kf_ir_camera* ir);
/* The undistortion map: W*H source pixel indices, -1 where unmapped (KF_ERR_STATE if off). */
KF_API int kf_get_undistortion_map(kf_session* s, int32_t* map);
/* shaders/filter3D.cs (shipped by the reference, never dispatched): an interior pixel keeps
 * its depth when more than 6 of its 3x3 neighbours are in (5, 4000) mm and it is within
 * 5 mm of their mean, else 0; border pixels become 0.  Runs after the undistortion. */
KF_API int kf_set_depth_filter(kf_session* s, int enable);

/* ---- tracking ------------------------------------------------------------------------ */
/* Track() (gFusion.cpp:648-740): coarse-to-fine projective point-to-plane ICP with the
 * 27-term reduction, an on-device FP64 solve and pose update.  *tracked may be NULL (then
 * the call does not synchronise). */
KF_API int kf_track_icp(kf_session* s, int* tracked);
/* TrackSDF() (gFusion.cpp:835-1038): direct SDF tracking, LM-damped, SE(3) exponential. */
KF_API int kf_track_sdf(kf_session* s, int* tracked);
/* recoverPose() (gFusion.cpp:1616-1653): TrackSDF from each pose of the pose library. */
KF_API int kf_recover_pose(kf_session* s, int* found);
/* Alignment energy and the 32-float reduction row of the last ICP / SDF iteration
 * (getReduction / getSDFReduction, gFusion.cpp:1127-1168, 1195-1232). */
KF_API int kf_get_alignment_energy(kf_session* s, float* ae);
/* Gauss-Newton iterations the last Track()/TrackSDF() executed (early exits included). */
KF_API int kf_get_iterations_run(kf_session* s, int* iterations);
KF_API int kf_get_reduction(kf_session* s, float sums[32]);

/* ---- volume ------------------------------------------------------------------------- */
KF_API int kf_integrate(kf_session* s); /* integrate(), gFusion.cpp:1234-1287 */
KF_API int kf_raycast(kf_session* s);   /* raycast(),   gFusion.cpp:1289-1366 */

/* One frame of src/kinect.cpp:654-695: depthToVertex, vertexToNormal, Track (or
 * TrackSDF), integrate when tracked (or inside the reset window), recoverPose when not
 * tracked, raycast.  Replayed from a CUDA graph after the first call. */
KF_API int kf_frame_step_u16(kf_session* s, const uint16_t* host_depth_mm, int* tracked);
KF_API int kf_frame_step_u16_device(kf_session* s, const uint16_t* device_depth_mm, int* tracked);
/* Pipelined frame steps: enqueues the upload of this frame (read from host_depth_mm until the
 * step completes: keep the buffer unchanged until the next call), the frame and a copy of its
 * result (pose and flags, 144 B), then reads the PREVIOUS asynchronous step's result, waiting
 * for that step only; the device runs this frame while the caller prepares the next.  The
 * previous step's error status is this call's return value: when that is not KF_OK, THIS
 * frame has still been enqueued and will be stepped, so a caller must not submit it again
 * (a failure to enqueue, e.g. KF_ERR_INVALID_ARGUMENT, is returned before anything is
 * enqueued and leaves the previous step unread).  kf_get_last_result returns the
 * last result read (no wait); kf_frame_sync waits for and reads the step still in flight.
 * Every synchronous call of the session reads it first.  A session stepped this way is not
 * put in a batch until kf_frame_sync. */
KF_API int kf_frame_step_u16_async(kf_session* s, const uint16_t* host_depth_mm);
KF_API int kf_frame_sync(kf_session* s, int* tracked);
KF_API int kf_get_last_result(kf_session* s, double pose[16], int* tracked);

/* ---- accessors (getVerts/getNorms/getDepthImage/getVolume/getTrackImage) ------------- */
KF_API int kf_get_raycast(kf_session* s, float* vertex4, float* normal4);            /* W*H*4 each */
/* Replace the maps Track() associates against (m_textureReferenceVertex/Normal, written by
 * raycast(), gFusion.cpp:1289-1366) with the caller's W*H*4 world-frame vertex and normal
 * maps (w = 1 where valid, 0 elsewhere), e.g. a model rendered elsewhere; the pose they were
 * made from stays the last raycast's.  No counterpart in the reference, which tracks only
 * against its own raycast. */
KF_API int kf_set_reference_maps(kf_session* s, const float* vertex4, const float* normal4);
KF_API int kf_get_vertex_map(kf_session* s, int level, float* vertex4);
KF_API int kf_get_normal_map(kf_session* s, int level, float* normal4);
KF_API int kf_get_depth_map(kf_session* s, int level, float* depth_mm);
KF_API int kf_get_track_status(kf_session* s, int level, int32_t* status); /* trackOutput.result */
KF_API int kf_get_volume(kf_session* s, kf_volume_view* view);
KF_API int kf_copy_volume_to_host(kf_session* s, void* dst, uint64_t bytes);
KF_API int kf_copy_volume_from_host(kf_session* s, const void* src, uint64_t bytes);
KF_API int kf_get_cum_twist(kf_session* s, double twist[6]); /* getCumTwist, gFusion.h:260-265 */
/* Volume ray-sum image (intensityProjection, gFusion.cpp:1368-1409, shaders/mip.cs) at
 * the current pose: per pixel (sum of the positive trilinear TSDF samples taken every
 * 0.75 mu between the slab entry/near plane and exit/far plane, 0, 0, 1); W*H*4 floats.
 * Its device image (W*H*16 bytes) is allocated on the first call and kept. */
KF_API int kf_intensity_projection(kf_session* s, float* rgba);
/* Volume checkpoint (the reference keeps none; Reset, gFusion.cpp:226-240, only clears).
 * The file is one JSON header line (format "kf-volume-checkpoint", sizes, metric volume
 * size, mu, pose) followed by the raw volume, the session's device control block (pose,
 * pose library, frame policy), the raycast maps and the trackSDF rows: a session loaded
 * from it steps on exactly as the saved one would have.  Loading requires the same
 * storage, volume size, metric size, mu and image size and a file written by this library
 * build (KF_ERR_INVALID_ARGUMENT otherwise, KF_ERR_IO for a short or unreadable file; the
 * session is left untouched by both).  File errors are KF_ERR_IO. */
KF_API int kf_save_volume(kf_session* s, const char* path);
KF_API int kf_load_volume(kf_session* s, const char* path);
/* Self-test of the bounded device waits: one block waits at a two-block grid barrier that
 * the other block never reaches; after budget_cycles (1e3 .. 1e9 SM clocks) the wait gives
 * up, records the timeout in the session's device error word and the kernel ends.  Returns
 * KF_ERR_TIMEOUT, exactly as a tracking call whose barrier timed out would, and clears the
 * error word; the session stays usable. */
KF_API int kf_selftest_barrier_timeout(kf_session* s, long long budget_cycles);
KF_API int kf_get_pose_library_size(kf_session* s, int* n);
/* Device times in milliseconds of the last call of each stage, in the order
 * pyramid, track, integrate, recover, raycast, mc (for frame steps: the last timed frame). */
KF_API int kf_get_stage_times(kf_session* s, float ms[6]);
/* Mean device milliseconds per stage (same order) over the timed frames of the
 * kf_frame_step_* calls since the last kf_reset_stage_stats (*frames: how many); read from
 * the frame graphs' events without stalling the stream. */
KF_API int kf_get_stage_stats(kf_session* s, double mean_ms[6], uint64_t* frames);
KF_API int kf_reset_stage_stats(kf_session* s);
/* Which frame steps record their stage boundaries: every `every`-th (1, 2 or 4; 0 = none;
 * default 4).  Each boundary is an event node in the frame's CUDA graph, ~5 us apiece on a
 * B200, so timing every frame costs ~5 % of a 512^3 frame step.  No counterpart in the
 * reference, whose stage timers are never assigned (gFusion.h:598-604). */
KF_API int kf_set_stage_timing(kf_session* s, int every);
KF_API int kf_get_stage_timing(kf_session* s, int* every);
/* Kernels this session has launched (a frame step counts every kernel of its graph). */
KF_API int kf_get_launch_count(kf_session* s, uint64_t* launches);
KF_API int kf_get_stream(kf_session* s, void** cuda_stream);

/* ---- launch shapes and the autotuner (no counterpart in the reference, whose shaders
 * fix their work-group sizes, e.g. integrate.cs local_size 32x32, raycast.cs 32x32) -----
 * Every shape computes bit-identical results; only the time differs. */
typedef struct kf_launch_shape {
  int32_t integrate_z_chunk; /* voxels per thread along z: 8, 16 (default) or 32 */
  int32_t raycast_rows;      /* raycast tile of 32 x rows pixels: 2, 4 (default) or 8;  */
                             /* 1 = persistent sweep, every warp taking the next 32-pixel */
                             /* row segment from a queue (sessions only, not batches)     */
  int32_t reserved[6];
} kf_launch_shape;
KF_API int kf_set_launch_shape(kf_session* s, const kf_launch_shape* shape);
KF_API int kf_get_launch_shape(kf_session* s, kf_launch_shape* shape);
/* Times every integrate z-chunk and raycast shape on the session's current depth frame,
 * pose and volume (repeats launches each, twice over, into scratch copies: the session's
 * volume, maps and pose are untouched; needs one more volume's worth of device memory
 * meanwhile), then uses the fastest.  times_ms (optional, 7 floats) receives the mean time
 * of integrate with z-chunk 8, 16, 32 and raycast with rows 1 (sweep), 2, 4, 8.  Sessions
 * created later with the same device, volume size, storage and image size start with the
 * shape chosen here. */
KF_API int kf_autotune(kf_session* s, int repeats, kf_launch_shape* chosen, float* times_ms);

/* ---- batched frame steps (the batched and served forms; no counterpart in the reference,
 * whose app runs one session) -----------------------------------------------------------
 * A batch steps several sessions' frames together, one launch per stage for all of them
 * (the per-frame body of kinect.cpp:654-695 for each).  Sessions of one step must share
 * the image size, storage and J^T J form and track by ICP; volume sizes and every other
 * setting may differ.  Each session's results are bit-identical to stepping it alone
 * (kf_frame_step_u16).  The step synchronises its stream; the sessions' poses and flags
 * are readable afterwards (kf_get_pose, ...).  Per-member tables are rebuilt when the set
 * or order of sessions changes.  A batch is used by one host thread at a time. */
#define KF_BATCH_MAX_SESSIONS 255
typedef struct kf_batch kf_batch;
KF_API int kf_batch_create(int max_sessions, kf_batch** out);
KF_API int kf_batch_destroy(kf_batch* b);
KF_API const char* kf_batch_last_error(const kf_batch* b);
/* host_depth_mm[i]: session i's 512x424-style uint16 frame (pinned memory copies fastest);
 * tracked[i] (may be NULL) receives the session's tracking result. */
KF_API int kf_batch_frame_step_u16(kf_batch* b, kf_session* const* sessions,
                                   const uint16_t* const* host_depth_mm, int n, int32_t* tracked);
KF_API int kf_batch_frame_step_u16_device(kf_batch* b, kf_session* const* sessions,
                                          const uint16_t* const* device_depth_mm, int n,
                                          int32_t* tracked);
/* The poses (camera-to-world, column-major) of the last step's first n sessions, in step
 * order, without another device round trip. */
KF_API int kf_batch_get_poses(kf_batch* b, int n, double* poses16);
/* Device ms of the last step's stages: pyramid, track, integrate, recover, raycast. */
KF_API int kf_batch_get_stage_times(kf_batch* b, float* ms5);
KF_API int kf_batch_get_launch_count(kf_batch* b, uint64_t* launches);
/* Asynchronous batched step (device-resident frames): enqueues the step and returns once
 * the PREVIOUS step's results are read (waiting for that one only), so the device runs one
 * step while the host prepares the next.  After it, kf_batch_get_poses / kf_batch_get_tracked
 * describe the previous step; its error status (e.g. KF_ERR_TIMEOUT of a member) is this
 * call's return value.  kf_batch_sync waits for and reads the step still in flight.  Until
 * then the step's sessions must not be used on their own.  Every other batch call finishes
 * the step in flight first. */
KF_API int kf_batch_frame_step_u16_device_async(kf_batch* b, kf_session* const* sessions,
                                                const uint16_t* const* device_depth_mm, int n);
KF_API int kf_batch_sync(kf_batch* b);
/* Tracked flags of the last step whose results were read (as kf_batch_get_poses). */
KF_API int kf_batch_get_tracked(kf_batch* b, int n, int32_t* tracked);
/* Launch shapes of the batched integrate and raycast (one shape per batch launch). */
KF_API int kf_batch_set_launch_shape(kf_batch* b, const kf_launch_shape* shape);
KF_API int kf_batch_get_launch_shape(kf_batch* b, kf_launch_shape* shape);
/* kf_autotune for the batched launches over these sessions (the mix of one step): each
 * candidate shape times one batched integrate and raycast over all of them, into scratch
 * copies (one more copy of every member's volume meanwhile); the batch then uses the
 * fastest.  times_ms (optional, 6 floats): integrate with z-chunk 8, 16, 32 and raycast
 * with rows 2, 4, 8 (a batch has no sweep shape). */
KF_API int kf_batch_autotune(kf_batch* b, kf_session* const* sessions, int n, int repeats,
                             kf_launch_shape* chosen, float* times_ms);

/* ---- served form (no counterpart in the reference) --------------------------------------
 * A request loop over resident sessions: kf_server_open admits a session while a slot and
 * the device-memory budget allow (KF_ERR_ADMISSION otherwise: retry after a close), frames
 * are queued with their arrival time as they come, and each kf_server_step runs one
 * batched frame step over the sessions with a waiting frame (oldest waiting frame first,
 * up to max_batch): continuous batching.  Frame latency = arrival to pose on the host.
 * All sessions use the server's storage and J^T J form and track by ICP. */
typedef struct kf_server_config {
  uint64_t hbm_budget_bytes; /* admission budget; 0 = free device memory at creation - 8 GiB */
  int32_t max_sessions;      /* resident session slots                                     */
  int32_t max_batch;         /* sessions per batched step (<= KF_BATCH_MAX_SESSIONS)       */
  int32_t storage;           /* KF_STORAGE_* of every session (default F16U16)             */
  int32_t jtj;               /* KF_JTJ_* of every session (default split-BF16)             */
  int32_t reserved[8];
} kf_server_config;
typedef struct kf_server_stats_t {
  uint64_t frames;           /* frames stepped since the last reset                         */
  uint64_t steps;            /* batched steps                                               */
  double busy_s;             /* seconds spent in batched steps                              */
  double p50_ms, p99_ms, max_ms; /* frame latency (arrival -> pose on the host)             */
  uint64_t bytes_in_use;     /* admitted sessions' device bytes                             */
  int32_t active_sessions;
  int32_t reserved[7];
} kf_server_stats_t;
typedef struct kf_server kf_server;
KF_API int kf_server_config_default(kf_server_config* cfg);
KF_API int kf_server_create(const kf_server_config* cfg, kf_server** out);
KF_API int kf_server_destroy(kf_server* v);
KF_API const char* kf_server_last_error(const kf_server* v);
KF_API double kf_server_now(void); /* the server's clock (seconds, monotonic) */
/* cfg's storage, jtj and tracking are replaced by the server's form. */
KF_API int kf_server_open(kf_server* v, const kf_config* cfg, const kf_intrinsics* intr,
                          const double pose[16], int* session_id);
/* Create `count` sessions of this configuration ahead of admissions (kept, like closed
 * sessions, for the next admissions of the same volume size); *created receives how many
 * fit the budget. */
KF_API int kf_server_prewarm(kf_server* v, const kf_config* cfg, const kf_intrinsics* intr,
                             int count, int* created);
/* The session's slot is freed at once; its device memory is kept for the next admission of
 * the same volume size, and released when the budget needs it (or at kf_server_destroy). */
KF_API int kf_server_close(kf_server* v, int session_id);
/* Queue a frame; it arrives now.  Host frames are copied (up to 8 waiting per session);
 * device frames are read in place and must stay valid until the step that uses them. */
KF_API int kf_server_submit(kf_server* v, int session_id, const uint16_t* host_depth_mm);
KF_API int kf_server_submit_device(kf_server* v, int session_id, const uint16_t* device_depth_mm);
KF_API int kf_server_step(kf_server* v, int* frames_done);
/* Asynchronous served step: enqueues a batched step over the sessions with a waiting frame
 * and returns once the PREVIOUS step's results are on the host (waiting for that step
 * only), so the host admits sessions and queues frames while the device runs.  After it,
 * kf_server_last_step / kf_server_get_pose describe the previous step, whose frame count
 * is *frames_done; when no frame is waiting, the step in flight is waited for instead.
 * kf_server_sync completes the step in flight; kf_server_step does so first, and so does
 * kf_server_close of a session in that step (its results are then the last step's).  A
 * frame's latency runs from its arrival to the call that returns its pose. */
KF_API int kf_server_step_async(kf_server* v, int* frames_done);
KF_API int kf_server_sync(kf_server* v, int* frames_done);
KF_API int kf_server_get_pose(kf_server* v, int session_id, double pose16[16], int* tracked,
                              uint64_t* frames_done);
/* The sessions of the last kf_server_step (up to max_n): ids, poses (16 doubles each,
 * column-major) and tracked flags, in step order; *n receives the count. */
KF_API int kf_server_last_step(kf_server* v, int max_n, int* session_ids, double* poses16,
                               int32_t* tracked, int* n);
KF_API int kf_server_pending(kf_server* v, int session_id, int* queued);
KF_API int kf_server_stats(kf_server* v, kf_server_stats_t* stats);
KF_API int kf_server_reset_stats(kf_server* v);

/* ---- marching cubes (MCubes, mcubes.cpp:206-509) ---------------------------------------
 * kf_mc_extract = setIsolevel + generateMarchingCubes; *n_triangles is the triangle count
 * (getNumberTriangles() returns 3x that).  Vertices are float4 in voxel-index units,
 * w = 0 (traverseHistoPyramids.cs:218-241). */
KF_API int kf_mc_extract(kf_session* s, float iso, int method, uint32_t* n_triangles);
KF_API int kf_mc_copy_vertices(kf_session* s, float* vertex4, uint64_t max_vertices);
/* Per vertex of the last extraction, its triangle's face normal cross(v1 - v0, v2 - v0),
 * unnormalised, w = 0: calcNormal of marchingCubes.cs:87-93, written to norm[] at :290-299
 * (in the units the positions were computed in, before the Q24 output scaling); the
 * histoPyramid path, which writes no normals in the reference, gets the same. */
KF_API int kf_mc_copy_normals(kf_session* s, float* normal4, uint64_t max_vertices);
/* Base level: numTri | cubeIndex << 16 per cube (RG16UI, histoPyramids.cs:170). */
KF_API int kf_mc_copy_base_level(kf_session* s, uint32_t* base, uint64_t count);
KF_API int kf_mc_export_stl(kf_session* s, const char* path);  /* exportMesh, :429-509 */
KF_API int kf_mc_export_ply(kf_session* s, const char* path);  /* exportPointCloud, :391-427 */

/* Welded mesh for export (no counterpart in the reference: exportMesh writes the triangle
 * soup with the normal (1,1,1), mcubes.cpp:451-500).  Extracted on the device from the
 * current volume with the classic path's corner order and case table (marchingCubes.cs)
 * over the interior cubes: one vertex per cut voxel edge that a triangle uses, numbered in
 * voxel order then axis (x, y, z), so the numbering does not depend on the launch;
 * positions in world metres ((voxel index + 0.5) * dim / size, integrate.cs:16-19);
 * normals the unit TSDF gradient (central differences at the edge's two voxels,
 * interpolated); triangles as three vertex indices, counter-clockwise seen from the
 * positive (free-space) side, so facet normals follow the gradient. */
KF_API int kf_mc_extract_mesh(kf_session* s, float iso, uint32_t* n_vertices, uint32_t* n_triangles);
/* Copies of the last welded mesh (any pointer may be NULL): 3 floats per vertex position
 * and normal, 3 indices per triangle. */
KF_API int kf_mc_copy_mesh(kf_session* s, float* positions3, float* normals3, uint32_t* indices3,
                           uint64_t max_vertices, uint64_t max_triangles);
/* Binary little-endian PLY (vertex x y z nx ny nz, face lists) and binary STL (zeroed
 * header, true triangle count, unit facet normals) of the last welded mesh. */
KF_API int kf_mc_export_mesh_ply(kf_session* s, const char* path);
KF_API int kf_mc_export_mesh_stl(kf_session* s, const char* path);

/* ---- prefix sum (prefixSum.cs, MCubes::prefixSum mcubes.cpp:136-204) --------------------
 * Exclusive scan of n uint32 device values on `stream` (0 = legacy default); *total, if
 * not NULL, receives sum(in) (lastElement + lastScanElement).  Any n up to 2^32-1. */
KF_API int kf_prefix_sum_u32(const uint32_t* d_in, uint32_t* d_out, uint64_t n, uint32_t* total,
                      void* cuda_stream);

/* Allocation-free prefix sum.  No counterpart in the reference: it exists for callers that
 * must not allocate device memory, such as a frame loop running under a fixed memory
 * budget or inside a host framework that owns every device allocation, where the
 * cudaMalloc of kf_prefix_sum_u32's scratch is not allowed.  Same result as
 * kf_prefix_sum_u32; the scratch is a 262,220-byte array compiled into the library,
 * which every GPU that loads the library keeps until the process exits.
 *   - n may be at most 2^28 (268,435,456) elements; larger n returns KF_ERR_CAPACITY.
 *   - The first call in a CUDA context looks up the array's device address (a host-side
 *     step, done once per context with that context current, and again in every new
 *     context: a primary context re-created after cudaDeviceReset, or one a framework
 *     made with cuCtxCreate); make that first call before any stream capture.
 *   - All calls on a device share the one array: calls whose work overlaps on the GPU
 *     (different streams, or host threads) race and corrupt each other's results.
 *     Serialise them, e.g. on one stream.
 *   - No cudaMalloc/cudaFree or allocating library call is made; if total is not NULL the
 *     call copies it back and synchronises the stream. */
KF_API int kf_prefix_sum_u32_noalloc(const uint32_t* d_in, uint32_t* d_out, uint64_t n,
                                     uint32_t* total, void* cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* KF_H */
