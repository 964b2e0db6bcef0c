/*
 * kf_api.h -- C ABI of the B200 KinectFusion per-frame pipeline (libkfb200.so).
 *
 * A uint16 depth frame goes in; the camera pose, the TSDF volume and the per-level raycast
 * vertex/normal maps come out.  Everything behind this header is hand-written sm_100a CUDA
 * driven by C++ host code; nothing here carries a C++ or torch type.
 *
 * Conventions (all inherited from the reference so that its callers' data drops in):
 *   - Depth maps are row-major float[h][w] in metres.
 *   - Vertex / normal maps are row-major float[h][w][4] = (x, y, z, tag) with tag -1 for a valid
 *     element and -2 for an invalid one (project/src/device_helper.cuh:9-10, :37-44).
 *   - Matrices are column-major, the memory order of glm::mat3 / glm::mat4 (element (row r,
 *     col c) at flat[c*dim + r]; test/example_test.cpp:36-50 pins this).
 *   - A pose is camera->world (project/src/sensor.h:30-34).
 *   - The TSDF is x-fastest, then y, then z.  Format KF_TSDF_F32F32 keeps distance and weight
 *     in two float arrays; KF_TSDF_F16U16 keeps an fp16 distance array and a uint16 weight array
 *     with KF_WEIGHT_SCALE fixed-point steps per unit of weight.  kf_get_tsdf /
 *     kf_set_tsdf convert to and from the reference's interleaved float2 .bin layout
 *     (project/src/voxel_grid.cpp:43-80).
 *   - Every call returns a kf_status; nothing throws across this boundary.  Where the
 *     reference throws std::runtime_error on a shape mismatch (e.g.
 *     project/src/measurement.cu:144-147) this ABI returns KF_ERR_SHAPE.
 *   - Stream arguments are cudaStream_t passed as void* (NULL = legacy default stream).
 *     Stage calls are asynchronous unless elapsed_ms is non-NULL, in which case they record
 *     events around the launch, synchronize and store the elapsed time, as every
 *     reference kernel:: wrapper does (project/src/measurement.cuh:11).
 */
#ifndef KF_API_H
#define KF_API_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KF_API_VERSION 1
#define KF_MAX_LEVELS 3
/* fixed-point steps per unit of weight in the uint16 weight array of KF_TSDF_F16U16; the
 * weight saturates at 65535 / 1024 (just under 64, the configurations' max weight) */
#define KF_WEIGHT_SCALE 1024.0f

typedef enum kf_status {
    KF_OK = 0,
    KF_ERR_ARG = 1,         /* null pointer, bad enum, unsupported size */
    KF_ERR_SHAPE = 2,       /* map sizes disagree (reference: std::runtime_error) */
    KF_ERR_CUDA = 3,        /* a CUDA runtime call failed */
    KF_ERR_NONFINITE = 4,   /* ICP solution not finite: pose kept, frame not fused
                               (reference: project/src/icp.cpp:67-73 throws) */
    KF_ERR_OOM_BUDGET = 5,  /* admission refused: the session does not fit the HBM budget */
    KF_ERR_TIMEOUT = 6,     /* a bounded device-side wait expired; the context stays usable */
    KF_ERR_STATE = 7,       /* call not valid in the object's current state */
    KF_ERR_CAPACITY = 8,    /* no free slot */
    KF_ERR_TOO_LARGE = 9    /* problem larger than the fixed scratch of a no-allocation entry point */
} kf_status;

typedef enum kf_tsdf_format {
    KF_TSDF_F32F32 = 0,     /* float distance + float weight, 8 B/voxel (reference layout) */
    KF_TSDF_F16U16 = 1      /* fp16 distance + uint16 weight, 4 B/voxel */
} kf_tsdf_format;

/*
 * Session configuration.  One struct replaces the reference's KinectFusionConfig
 * (project/src/kinect_fusion.h:17-36), IcpConfig (project/src/icp.h:11-20) and the
 * compile-time constants the reference hard-codes:
 *   bilateral sigma_s / sigma_r / window  (project/src/measurement.cu:11-12, :38)
 *   min / max sensor range 0.4 / 6.0 m     (project/src/tsdf.cuh:11-12)
 *   raycast steps 1.99 mu / 0.1 mu          (project/src/raycast.cu:75-76)
 *   principal point 319.5 / 239.5          (project/src/sensor.h:14)
 *   frustum bounds 640 x 480                (project/src/tsdf.cu:40)
 * kf_config_default() fills the reference's values (project/src/main.cpp:11-59, the
 * dataset configuration) so that a default session behaves like the reference.
 */
typedef struct kf_config {
    int width, height;           /* frame size; divisible by 2^(levels-1) */
    float fx, fy, cx, cy;        /* level-0 intrinsics (reference: fx = fy = field_of_view) */
    float depth_scale;           /* raw uint16 -> metres */
    int unmirror;                /* flip columns on conversion (reference: use_kinect) */
    int levels;                  /* pyramid levels, 1..3 (reference: iters_per_layer.size()) */
    int iters[KF_MAX_LEVELS];    /* ICP iterations per level, index 0 = finest */
    float dist_thresh;           /* correspondence distance rejection, metres */
    float angle_thresh;          /* correspondence normal-angle rejection, radians */
    float stop_angle;            /* early stop: rotation chord threshold */
    float stop_dist;             /* early stop: translation threshold, metres */
    float bilateral_sigma_s;     /* pixels */
    float bilateral_sigma_r;     /* metres; the downsample gate is 3 * sigma_r */
    int bilateral_radius;        /* window = 2 * radius + 1 */
    int volume_n;                /* voxels per side */
    float volume_width;          /* cube edge in metres, centred at the world origin */
    float mu;                    /* truncation distance in metres */
    float max_weight;            /* 0 = no clamp (reference behaviour) */
    int tsdf_format;             /* kf_tsdf_format */
    float min_depth, max_depth;  /* sensor range used by fusion and raycast */
    float step_large, step_small;/* raycast steps in units of mu */
    int compat_trunc8;           /* process only what the reference's dims/8 grids cover */
    int keep_on_miss;            /* rays that miss the volume keep the previous map contents
                                    (reference: project/src/raycast.cu:61-73 returns early) */
    int export_icp_mask;         /* record per-pixel correspondence masks of the last iteration */
    float initial_pose[16];      /* camera->world, column-major */
    /* Visualization volume: the reference's second voxel grid (project/src/kinect_fusion.cpp:19,
     * :179-203), which it fuses every frame at the frame's pose and raycasts for display only.
     * vis_volume_n = 0: none.  Else an n^3 grid (n a multiple of 8, format tsdf_format) over a
     * cube of vis_volume_width metres, truncation vis_mu metres; kf_render raycasts it. */
    int vis_volume_n;
    float vis_volume_width;
    float vis_mu;
} kf_config;

/* A TSDF volume in device memory, for the per-stage calls. */
typedef struct kf_volume {
    void* f;                     /* distance array: float or __half, n^3, x fastest */
    void* w;                     /* weight array: float or uint16, n^3 */
    int n;
    float width;                 /* metres */
    float mu;                    /* metres */
    int format;                  /* kf_tsdf_format */
    float max_weight;            /* 0 = no clamp */
} kf_volume;

/* Per-frame results beyond the pose. */
typedef struct kf_frame_stats {
    int frame;                   /* index of the frame just processed (0 = first) */
    int status;                  /* kf_status of that frame */
    int icp_iters[KF_MAX_LEVELS];/* ICP iterations run per level (0 for frame 0) */
} kf_frame_stats;

/* ------------------------------------------------------------------------------------------ */
/* library                                                                                    */
/* ------------------------------------------------------------------------------------------ */
int kf_api_version(void);
const char* kf_status_string(int status);
/* Fill the reference's defaults (project/src/main.cpp:11-59 dataset config, 640x480). */
void kf_config_default(kf_config* cfg);
/* Bytes of device memory a session with this configuration holds. */
kf_status kf_session_footprint(const kf_config* cfg, size_t* bytes);

/* ------------------------------------------------------------------------------------------ */
/* session: the reference's KinectFusion class (project/src/kinect_fusion.h:38-48)          */
/* ------------------------------------------------------------------------------------------ */
typedef struct kf_session kf_session;

/* Allocate buffers and the volume, initialise the grid to {f = 2, w = 0}
 * (reference constructor, project/src/kinect_fusion.cpp:13-42). */
kf_status kf_session_create(const kf_config* cfg, kf_session** out);
kf_status kf_session_destroy(kf_session* s);
/* Back to frame 0: grid re-initialised, pose = initial_pose. */
kf_status kf_session_reset(kf_session* s);
/* One frame.  Frame 0 converts and fuses only (initializeTracking,
 * project/src/kinect_fusion.cpp:75-94); later frames run preprocessing, raycast at the
 * previous pose, ICP and fusion (project/src/kinect_fusion.cpp:48-72).
 * depth: w*h uint16 in host memory (is_device_ptr = 0) or device memory (1).
 * pose_out (may be NULL): the new camera->world pose, column-major.
 * The call synchronizes the stream before returning. */
kf_status kf_process_frame(kf_session* s, const uint16_t* depth, int is_device_ptr,
                           void* stream, float pose_out[16]);
/* Streaming form of kf_process_frame: submit queues a frame (host memory, or device memory
 * when is_device_ptr = 1) and returns without waiting; wait returns the oldest submitted
 * frame's pose and statistics (and its status), blocking until that frame is done.  Up to
 * KF_MAX_FRAMES_IN_FLIGHT frames may be submitted and not yet waited for (KF_ERR_CAPACITY
 * beyond); a host frame must stay unchanged until its wait returns.  Submitting frame k + 1
 * before waiting for frame k hides the host's share of a frame (the call overhead, the copy
 * set-up, the wake-up after the result) behind the device's work on frame k; the frames run
 * in order on the stream, with the same results as kf_process_frame.  kf_process_frame
 * returns KF_ERR_STATE while submitted frames are outstanding; kf_session_reset drops them.
 * No counterpart in the reference (its frame loop is synchronous,
 * project/src/kinect_fusion.cpp:55-72). */
#define KF_MAX_FRAMES_IN_FLIGHT 4
kf_status kf_process_frame_submit(kf_session* s, const uint16_t* depth, int is_device_ptr, void* stream);
kf_status kf_process_frame_wait(kf_session* s, float pose_out[16], kf_frame_stats* stats);
/* Enqueue one frame from device memory without synchronizing (for graph-replay drivers);
 * results are valid once the stream reaches this point. */
kf_status kf_process_frame_async(kf_session* s, const uint16_t* depth_device, void* stream);
kf_status kf_get_pose(kf_session* s, float pose[16]);
kf_status kf_set_pose(kf_session* s, const float pose[16]);
kf_status kf_get_frame_stats(kf_session* s, kf_frame_stats* out);
/* Map taps.  dst is host memory when to_host = 1, else device memory.  level in
 * [0, levels); kf_get_depth with level = -1 returns the unfiltered metres map that fusion
 * reads. */
kf_status kf_get_depth(kf_session* s, int level, float* dst, int to_host);
kf_status kf_get_vertex(kf_session* s, int level, float* dst, int to_host);
kf_status kf_get_raycast(kf_session* s, int level, float* vertex, float* normal, int to_host);
kf_status kf_get_icp_mask(kf_session* s, int level, uint8_t* dst, int to_host);
/* TSDF readback / load.  layout 0: native arrays (f array then w array, each n^3);
 * layout 1: reference interleaved float2 {f, w} (.bin layout). */
kf_status kf_get_tsdf(kf_session* s, void* dst, size_t dst_bytes, int layout, int to_host);
kf_status kf_set_tsdf(kf_session* s, const void* src, size_t src_bytes, int layout, int from_host);
kf_status kf_get_volume(kf_session* s, kf_volume* out);
/* The visualization volume (KF_ERR_STATE when the session has none), as kf_get_tsdf /
 * kf_get_volume do for the tracking volume. */
kf_status kf_get_vis_tsdf(kf_session* s, void* dst, size_t dst_bytes, int layout, int to_host);
kf_status kf_get_vis_volume(kf_session* s, kf_volume* out);

/* ------------------------------------------------------------------------------------------ */
/* stages: the reference's kernel:: wrappers, on device pointers                            */
/* ------------------------------------------------------------------------------------------ */
/* kernel::convertToDepthMeters, project/src/measurement.cuh:12 */
kf_status kf_convert_to_depth_meters(const uint16_t* raw, int w, int h, float* out, int out_w,
                                     int out_h, float scale, int unmirror, void* stream,
                                     float* elapsed_ms);
/* kernel::applyBilateralFilter, project/src/measurement.cuh:13 (sigma/window are the
 * reference's compile-time constants, passed here) */
kf_status kf_apply_bilateral_filter(const float* in, int w, int h, float* out, int out_w,
                                    int out_h, float sigma_s, float sigma_r, int radius,
                                    void* stream, float* elapsed_ms);
/* kernel::downSample, project/src/measurement.cuh:14 */
kf_status kf_down_sample(const float* in, int w, int h, float* out, int out_w, int out_h,
                         float sigma_r, void* stream, float* elapsed_ms);
/* kernel::createVertexMap, project/src/measurement.cuh:15 (inv_cam_k column-major 3x3) */
kf_status kf_create_vertex_map(const float* depth, int w, int h, float* vertex, int out_w,
                               int out_h, const float inv_cam_k[9], void* stream,
                               float* elapsed_ms);
/* kernel::createNormalMap, project/src/measurement.cuh:16 */
kf_status kf_create_normal_map(const float* vertex, int w, int h, float* normal, int out_w,
                               int out_h, void* stream, float* elapsed_ms);
/* kernel::initializeGrid, project/src/tsdf.cuh:15 (value {f = 2, w = 0}) */
kf_status kf_initialize_grid(const kf_volume* vol, void* stream, float* elapsed_ms);
/* kernel::fuse, project/src/tsdf.cuh:16.  cam_k: level-0 intrinsics, column-major;
 * w, h: the frustum bounds (the reference hard-codes 640 x 480). */
kf_status kf_fuse(const float* depth_m, int w, int h, const float cam_k[9], const kf_volume* vol,
                  const float pose[16], float min_depth, float max_depth, void* stream,
                  float* elapsed_ms);
/* kernel::raycast, project/src/raycast.cuh:11.  inv_cam_k: the level's inverse intrinsics. */
kf_status kf_raycast(const kf_volume* vol, const float pose[16], const float inv_cam_k[9],
                     float* vertex, int w, int h, float* normal, int nw, int nh,
                     float min_depth, float max_depth, float step_large, float step_small,
                     void* stream, float* elapsed_ms);
/* kernel::constructIcpResiduals, project/src/icp.cuh:34-37.  Writes the reference's
 * row-major A (w*h x 6) and b (w*h), zero rows for rejected pixels. */
kf_status kf_construct_icp_residuals(const float* vertex, const float* target_vertex,
                                     const float* target_normal, int w, int h,
                                     const float prev_rot[9], const float prev_transl[3],
                                     const float cur_rot[9], const float cur_transl[3],
                                     const float cam_k[9], float distance_thresh,
                                     float angle_thresh, float* mat_a, float* vec_b,
                                     void* stream, float* elapsed_ms);
/* LinearLeastSquares::solve, project/src/linear_least_squares.h:19: x = argmin |A x - b|
 * over n rows (A row-major n x 6 and b on the device).  The normal equations are reduced
 * in FP32 with compensated block sums and combined and solved (Cholesky) in FP64 on the
 * device; only the 6 floats of x come back. */
kf_status kf_solve_linear_least_squares(const float* mat_a, const float* vec_b, int n,
                                        float x_out[6], void* stream);
/* Row limit of kf_solve_linear_least_squares_noalloc (2^20: a 1280 x 720 frame fits). */
#define KF_LLS_NOALLOC_MAX_ROWS 1048576
/* kf_solve_linear_least_squares without any device allocation.  No counterpart in the
 * reference: its LinearLeastSquares::solve (project/src/linear_least_squares.cpp:23-44)
 * allocates, and so does kf_solve_linear_least_squares, which grows a process-wide scratch
 * with cudaFree + cudaMalloc when a larger n arrives.  Some callers cannot allow that: a
 * tracking loop that shares the device with other sessions (cudaFree waits for the whole
 * device, stalling their frames) and a process whose device memory is all reserved up
 * front by a caching allocator or an HBM budget (an unplanned allocation can fail with out
 * of memory in mid-sequence).  This entry point runs the same two kernels, with the same
 * block count, on a scratch that is a fixed 110,640-byte array in the library's device
 * image; its result is bit-identical to kf_solve_linear_least_squares.
 *   - n above KF_LLS_NOALLOC_MAX_ROWS returns KF_ERR_TOO_LARGE before touching the device.
 *   - The first call on each device does a one-time set-up with that device current (it
 *     looks up the scratch's device address, which may load the library's device code):
 *     make it before any latency-critical work.
 *   - Nothing has to start at zero: each call writes every scratch value it reads.
 *   - All calls on one device share the one scratch, so calls that overlap (two host
 *     threads, or two streams in flight) race and give wrong results: serialise them.
 *   - Like kf_solve_linear_least_squares it returns x to the host and synchronises
 *     `stream`. */
kf_status kf_solve_linear_least_squares_noalloc(const float* mat_a, const float* vec_b, int n,
                                                float x_out[6], void* stream);
/* ICP::computePose, project/src/icp.h:35-36.  Coarse-to-fine point-to-plane ICP of the
 * vertex pyramid against the predicted (world-frame) pyramid, starting at pose; each map
 * pointer array holds `levels` device pointers.  One cooperative device launch runs every
 * iteration, solve and early-stop test.  iters_out (may be NULL) gets iterations per level. */
kf_status kf_compute_pose(const float* const* vertex, const float* const* target_vertex,
                          const float* const* target_normal, int w, int h, int levels,
                          const kf_config* cfg, const float pose[16], float pose_out[16],
                          int iters_out[KF_MAX_LEVELS], void* stream);
/* poseError, project/src/general_helper.h:9: out[0] = chord between the two rotations
 * applied to normalize(1,1,1); out[1] = translation distance.  Host-side helper. */
kf_status kf_pose_error(const float pose_1[16], const float pose_2[16], float out[2]);

/* ------------------------------------------------------------------------------------------ */
/* files: TSDF in the reference's .bin layout, session checkpoints                            */
/* ------------------------------------------------------------------------------------------ */
/* VoxelGrid::saveVoxelGrid / loadVoxelGrid (project/src/voxel_grid.cpp:43-80): n^3 interleaved
 * float {f, w}, x fastest, no header.  Loading a file of another size is KF_ERR_SHAPE.  F16U16
 * sessions convert to and from float. */
kf_status kf_save_tsdf_file(kf_session* s, const char* path);
kf_status kf_load_tsdf_file(kf_session* s, const char* path);
/* The same for the visualization volume, the grid the reference's KinectFusion::saveTSDF /
 * loadTSDF write and read (project/src/kinect_fusion.cpp:327-335); KF_ERR_STATE without one. */
kf_status kf_save_vis_tsdf_file(kf_session* s, const char* path);
kf_status kf_load_vis_tsdf_file(kf_session* s, const char* path);
/* Checkpoint: the .bin TSDF at `path` plus `path`.pose (text: frame count and the
 * column-major camera->world pose).  After a load the session resumes tracking as frame
 * `frames` of its sequence.  No counterpart in the reference beyond the .bin file. */
kf_status kf_session_checkpoint_save(kf_session* s, const char* path);
kf_status kf_session_checkpoint_load(kf_session* s, const char* path);

/* ------------------------------------------------------------------------------------------ */
/* headless display: the reference's window-content kernels (project/src/display.cu:9-105)    */
/* into RGBA8 images in device memory (row-major, bytes r, g, b, 255 per pixel)              */
/* ------------------------------------------------------------------------------------------ */
#define KF_RENDER_NORMALS 0   /* normalMapToWindowContent: rotated normal * 255 as r, g, b */
#define KF_RENDER_SHADING 1   /* shadingToWindowContent: |normal . ray| * 255 as grey */
/* kernel::normalMapToWindowContent (project/src/display.cu:143-154); normal: float4 map,
 * inv_rot: the inverse sensor rotation (column-major 3x3). */
kf_status kf_normal_map_to_rgba(const float* normal, int w, int h, const float inv_rot[9],
                                uint8_t* rgba, void* stream, float* elapsed_ms);
/* kernel::shadingToWindowContent (project/src/display.cu:156-167); pose: camera->world,
 * inv_cam_k: level-0 inverse intrinsics. */
kf_status kf_shading_to_rgba(const float* normal, int w, int h, const float pose[16],
                             const float inv_cam_k[9], uint8_t* rgba, void* stream,
                             float* elapsed_ms);
/* kernel::oneFloatChannelToWindowContent (project/src/display.cu:117-128): value * scale. */
kf_status kf_float_channel_to_rgba(const float* src, int w, int h, float scale, uint8_t* rgba,
                                   void* stream, float* elapsed_ms);
/* KinectFusion::visualizeCurrentModel (project/src/kinect_fusion.cpp:185-203), headless: raycast
 * the session's visualization volume (the tracking volume when it has none) at level 0 from
 * `pose` (NULL: the current pose; the reference's static view passes the initial pose) into the
 * session's own render maps, then the display kernel of `mode` into rgba (w * h * 4 bytes; host
 * memory when to_host = 1).  Tracking maps are not touched.  Synchronizes `stream`. */
kf_status kf_render(kf_session* s, int mode, const float pose[16], uint8_t* rgba, int to_host,
                    void* stream);

/* ------------------------------------------------------------------------------------------ */
/* datasets: TUM RGB-D sequences (RgbdDataset, project/src/rgbd_dataset.h:12-27)              */
/* ------------------------------------------------------------------------------------------ */
typedef struct kf_tum kf_tum;
/* RgbdDataset::load (project/src/rgbd_dataset.cpp:6-76): groundtruth.txt and depth.txt (three
 * comment lines each); every depth image is paired with the nearest ground-truth pose. */
kf_status kf_tum_open(const char* dir, kf_tum** out);
kf_status kf_tum_close(kf_tum* d);
kf_status kf_tum_count(const kf_tum* d, int* count);
/* Frame `index`: the 16-bit depth PNG decoded into depth (w * h, KF_ERR_SHAPE if the image
 * size differs; NULL to skip) and its ground-truth pose (column-major camera->world, the
 * reference's mat4_cast(quaternion) with the translation; NULL to skip). */
kf_status kf_tum_frame(const kf_tum* d, int index, uint16_t* depth, int w, int h, float pose[16]);
/* RgbdDataset::getInitialPoseInverse (project/src/rgbd_dataset.cpp:89-92). */
kf_status kf_tum_initial_pose_inverse(const kf_tum* d, float out[16]);
/* DepthMap::update(path) (project/src/depth_map.cpp:17-28): a 16-bit greyscale PNG. */
kf_status kf_png16_read(const char* path, uint16_t* dst, int w, int h);

/* ------------------------------------------------------------------------------------------ */
/* batch: many independent sessions of uneven sizes, one persistent launch per stage,        */
/* replayed from a captured CUDA graph                                                        */
/* ------------------------------------------------------------------------------------------ */
typedef struct kf_batch kf_batch;

kf_status kf_batch_create(const kf_config* cfgs, int n, kf_batch** out);
kf_status kf_batch_destroy(kf_batch* b);
/* One frame for every session whose entry in `depth` is non-NULL (host pointers when
 * is_device_ptr = 0).  Sessions with a NULL entry sit this step out.  poses_out (may be
 * NULL): n * 16 floats.  Synchronizes before returning. */
kf_status kf_batch_step(kf_batch* b, const uint16_t* const* depth, int is_device_ptr,
                        void* stream, float* poses_out);
/* Enqueue a step whose frames are already in each session's device input buffer. */
kf_status kf_batch_step_async(kf_batch* b, const int* active, void* stream);
/* Device address of session i's uint16 input frame buffer (w*h elements). */
kf_status kf_batch_input_buffer(kf_batch* b, int i, uint16_t** dev_ptr);
kf_status kf_batch_session(kf_batch* b, int i, kf_session** out);
/* Tune the batch's launch shapes on its own live steps.  The shapes are the persistent grid of
 * every stage, the raycast kernel's form (3 or 4 blocks per SM), the number of march iterations
 * a lane takes before it hands a long ray to a warp, the ray tile (8 x 4, 16 x 2 or 4 x 8
 * pixels per warp) and how fusion splits its queue entries; none of them changes a result, bit
 * for bit.  After this call each kf_batch_step runs one candidate shape and its stage times
 * (device events) are recorded; a walk over the parameters, one at a time, keeps the fastest
 * candidate of each (by the step's device time), and after the last step of the walk the
 * batch keeps the chosen shape.
 * cache_path (may be NULL): a JSON file of chosen shapes keyed by the batch's session mix
 * (frame sizes, volumes, formats, counts) and the device's SM count; if it holds an entry for
 * this mix, that shape is applied at once and no step is spent tuning, else the walk's result
 * is added to it.  kf_batch_step_async steps do not advance the walk.  The reference has no
 * counterpart (its launch shapes are fixed 8 x 8 blocks). */
kf_status kf_batch_autotune_start(kf_batch* b, const char* cache_path);
/* Steps the walk still needs (0 when done or not started) and a JSON report: the mix key, the
 * source of the shape ("tuned" or "cache") and the shape, with each parameter's winning step
 * time (ms) when tuned. */
kf_status kf_batch_autotune_status(kf_batch* b, int* steps_left, char* report, size_t report_bytes);

/* ------------------------------------------------------------------------------------------ */
/* server: continuous batching of concurrent sessions with HBM-budget admission              */
/* ------------------------------------------------------------------------------------------ */
typedef struct kf_server kf_server;

typedef struct kf_server_stats {
    long long frames_done;
    long long sessions_admitted;
    long long sessions_refused;
    long long steps;
    int active_sessions;
    int max_active_sessions;
    size_t hbm_in_use;
    size_t hbm_budget;
    double p50_ms, p99_ms, max_ms;   /* submit -> result ready */
} kf_server_stats;

/* max_slots: most sessions resident at once; hbm_budget: bytes all sessions may hold. */
kf_status kf_server_create(int max_slots, size_t hbm_budget, kf_server** out);
kf_status kf_server_destroy(kf_server* srv);
/* Admit a session: KF_ERR_OOM_BUDGET when it does not fit the budget, KF_ERR_CAPACITY when
 * every slot is taken.  *id identifies it in later calls. */
kf_status kf_server_open(kf_server* srv, const kf_config* cfg, int* id);
kf_status kf_server_close(kf_server* srv, int id);
/* Queue one frame (host memory, copied before return).  A session holds at most one
 * queued frame; a second submit before the first is served returns KF_ERR_STATE. */
kf_status kf_server_submit(kf_server* srv, int id, const uint16_t* depth, double t_submit_ms);
/* Run one batched step over every session with a queued frame; returns how many frames it
 * served in *served.  Frames that arrive while a step runs join the next one. */
kf_status kf_server_step(kf_server* srv, int* served);
/* Result of the session's last served frame. */
kf_status kf_server_result(kf_server* srv, int id, float pose[16], kf_frame_stats* stats);
kf_status kf_server_get_session(kf_server* srv, int id, kf_session** out);
kf_status kf_server_stats_get(kf_server* srv, kf_server_stats* out);
/* Capacity planning: allocate device arenas for `count` sessions shaped like cfg (and pinned
 * staging for as many slots) into the server's pool, so that opening such sessions later
 * allocates nothing.  Cached arenas count against the HBM budget; KF_ERR_OOM_BUDGET when
 * they would not fit. */
kf_status kf_server_reserve(kf_server* srv, const kf_config* cfg, int count);
/* Start a new statistics window: latencies, frame, step and session counters restart from
 * zero (after a warm-up, say); sessions and their state are untouched. */
kf_status kf_server_stats_reset(kf_server* srv);
/* Clock used for latency accounting (milliseconds, monotonic). */
double kf_now_ms(void);

/* ------------------------------------------------------------------------------------------ */
/* instrumentation (the reference times every kernel:: call with a blocking event pair,       */
/* project/src/cuda_event.cpp:14-29; here events sit between the stage launches of a step,    */
/* inside the captured graph, and nothing blocks)                                              */
/* ------------------------------------------------------------------------------------------ */
/* Record events between the stages of every step (re-captures the step graph). */
kf_status kf_session_set_profiling(kf_session* s, int on);
/* Device durations (ms) of the last completed step: preprocess, raycast, ICP, fusion.  The
 * preprocess runs on a graph branch beside the raycast, so the raycast figure spans both. */
kf_status kf_session_stage_times(kf_session* s, float ms[4]);
/* Debug modes of a session (flags, 0 = off).  KF_DEBUG_RAY_TRACE makes every raycast record,
 * per pixel, the decisions its march took: how many samples it took before leaving large steps
 * and how (a sample below 0.99, or a negative one that backs off by mu), how many it took in
 * all and how it ended (bits 40.., 8..39, 4..5 and 0..1 of a uint64; 0 for a ray that never
 * marched).  Two implementations of the reference's march (project/src/raycast.cu:75-117) that
 * give a pixel the same trace took the same samples in the same order, so their hits can only
 * differ by arithmetic rounding; a different trace means a sample near 0.99 or 0 decided
 * otherwise.  No counterpart in the reference (a parity aid). */
#define KF_DEBUG_RAY_TRACE 1
/* KF_DEBUG_NO_GRAPH launches every step's kernels one by one instead of replaying the captured
 * graph, each stage inside an NVTX range (kf.preprocess, kf.raycast, kf.icp, kf.fusion), so a
 * profiler can select a stage's launches.  Results are the same; steps are slower. */
#define KF_DEBUG_NO_GRAPH 2
/* KF_DEBUG_COUNTERS makes the raycast count its work in every step (kernels built with the
 * counts; the plain kernels run otherwise): kf_session_debug_counts / kf_batch_debug_counts
 * return, for the last step, [0] rays that marched, [1] samples evaluated during large steps,
 * [2] during small steps, [3] cell skips, [4] samples the skips jumped over, [5] gradient
 * samples, [6] rays handed to the long-ray warp kernel, [7] that kernel's warp rounds.  The
 * counts cost time; results are the same. */
#define KF_DEBUG_COUNTERS 4
#define KF_RAY_COUNTS 8
kf_status kf_session_set_debug(kf_session* s, int flags);
/* The same for every session of a batch (KF_DEBUG_NO_GRAPH and KF_DEBUG_COUNTERS apply to the
 * batch's steps). */
kf_status kf_batch_set_debug(kf_batch* b, int flags);
/* The raycast work counts of the last step (n entries, at most KF_RAY_COUNTS; KF_ERR_STATE
 * unless KF_DEBUG_COUNTERS is on).  For a session of a batch the counts are the whole step's. */
kf_status kf_session_debug_counts(kf_session* s, uint64_t* out, int n);
kf_status kf_batch_debug_counts(kf_batch* b, uint64_t* out, int n);
/* The traces of the last raycast at `level` (w * h uint64; host memory when to_host = 1).
 * KF_ERR_STATE unless KF_DEBUG_RAY_TRACE is on. */
kf_status kf_get_ray_trace(kf_session* s, int level, uint64_t* dst, int to_host);
kf_status kf_batch_set_profiling(kf_batch* b, int on);
kf_status kf_batch_stage_times(kf_batch* b, float ms[4]);
/* Self-test of the bounded device-side waits: a cooperative launch whose barrier is never
 * completed must give up after timeout_ms and report KF_ERR_TIMEOUT, leaving the context
 * usable.  waited_ms (may be NULL) gets the wall time the launch took. */
kf_status kf_selftest_bounded_wait(int timeout_ms, int* waited_ms);
/* Read bandwidth of this device (GB/s) over a buffer of `bytes` (16 MiB .. 4 GiB, a multiple of
 * 16), read `rounds` times (1 .. 1000) by a grid of 8 blocks per SM after one untimed round.  A
 * buffer under the L2's size measures the L2; the raycaster's gather rate is read against it.
 * Allocates and frees its buffer.  No counterpart in the reference (a measurement aid). */
kf_status kf_measure_read_bandwidth(size_t bytes, int rounds, double* gbs);

#ifdef __cplusplus
}
#endif

#endif /* KF_API_H */
