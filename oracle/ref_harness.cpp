// TEST INFRASTRUCTURE ONLY: a C ABI over the reference's own compute code, compiled where it
// lies (project/src/*.cu, icp.cpp, linear_least_squares.cpp, voxel_grid.cpp, ...) by
// oracle/Makefile into oracle/_ref/libkfref.so.  The tests and the bench's reference arm drive
// it; nothing in the CUDA library links it.
//
// The reference's frame loop is KinectFusion::startTracking (project/src/kinect_fusion.cpp:
// 44-73), which also runs an SDL/OpenGL window (not built here) and reads depth PNGs through
// stb_image (an empty submodule of the reference).  Its TUM sequence reader, RgbdDataset, is
// built and exported below on its own (host only).
// This file restates that loop's compute calls in the same order with the reference's own
// classes and kernel wrappers:
//   first frame  initializeTracking   (kinect_fusion.cpp:75-95): convert, fuse
//   every frame  depthFrameToVertexPyramid (:115-135): convert, bilateral, vertex map, then
//                per coarser level downSample + createVertexMap;
//                raycastTsdf (:137-144) at every level; computePose (:146-160) through
//                ICP::computePose; fuseCurrentDepthToTSDF (:176-180); with a visualization
//                grid also visualizeCurrentModel's raycast (:182-189) into the level-0 maps.
// Frames come from memory through DepthMap::update(void*) (project/src/depth_map.cpp:28-33).
// ICP::computePose throws when the solve is not finite (project/src/icp.cpp:63-69); the
// reference program would end there, the harness reports status 1 and keeps the pose.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "cuda_grid_map.h"
#include "depth_map.h"
#include "general_helper.h"
#include "grid_map_pyramid.h"
#include "icp.h"
#include "rgbd_dataset.h"
#include "sensor.h"
#include "voxel_grid.h"

// the kernel wrappers (project/src/measurement.cuh:10-16, raycast.cuh:8-11, tsdf.cuh:9-16);
// their headers also pull in the window class, so the declarations are repeated here
namespace kernel {
float convertToDepthMeters(const DepthMap& raw_depth_map, const CudaGridMap& raw_depth_map_meters, float scale,
                           bool unmirror);
float applyBilateralFilter(const CudaGridMap& raw_depth_map_meters, const CudaGridMap& filtered_depth_map);
float downSample(const CudaGridMap& depth_map, const CudaGridMap& depth_map_downsampled);
float createVertexMap(const CudaGridMap& depth_map, const CudaGridMap& vertex_map, const glm::mat3& inv_cam_k);
float createNormalMap(const CudaGridMap& vertex_map, const CudaGridMap& normal_map);
float raycast(const VoxelGridStruct& voxel_grid, const Sensor& sensor, const CudaGridMap& output_vertex,
              const CudaGridMap& output_normal, int level);
float initializeGrid(const VoxelGridStruct& voxel_grid, const Voxel& value);
float fuse(const CudaGridMap& raw_depth_map_meters, const VoxelGridStruct& voxel_grid, const Sensor& sensor);
float constructIcpResiduals(CudaGridMap& vertex_map, CudaGridMap& target_vertex_map, CudaGridMap& target_normal_map,
                            glm::mat3 prev_rot_mat, glm::vec3 prev_transl_vec, glm::mat3 curr_rot_mat_estimate,
                            glm::vec3 current_transl_vec_estimate, glm::mat3 sensor_intrinsics,
                            float distance_thresh, float angle_thresh, float* mat_A, float* vec_b);
}  // namespace kernel

namespace {

constexpr int kW = 640, kH = 480, kLevels = 3;   // the reference's fixed frame (sensor.h:14-16)

struct Times {
    double preprocess = 0, raycast = 0, icp_residuals = 0, icp_solve = 0, fuse = 0, vis = 0;
};

struct Harness {
    const cudaChannelFormatDesc half_desc = cudaCreateChannelDesc(16, 0, 0, 0, cudaChannelFormatKindFloat);
    const cudaChannelFormatDesc single_desc = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    const cudaChannelFormatDesc vec4_desc = cudaCreateChannelDesc(32, 32, 32, 32, cudaChannelFormatKindFloat);

    float depth_scale;
    bool unmirror = false;
    Sensor sensor;
    VoxelGrid grid;
    std::unique_ptr<VoxelGrid> vis;
    IcpConfig icp_config;
    ICP icp;
    DepthMap raw;
    CudaGridMap meters;
    GridMapPyramid<CudaGridMap> depth, vertex, pred_vertex, pred_normal;
    CudaGridMap normal_scratch;
    Times t;
    int frames = 0;

    Harness(int n, float width, float mue_scale, float fov, float scale, const IcpConfig& ic, int vis_n,
            float vis_width, float vis_mue_scale)
        : depth_scale(scale), sensor(fov), grid(width, n, mue_scale), icp_config(ic), icp(ic),
          raw(kW, kH, half_desc), meters(kW, kH, single_desc), depth(kW, kH, kLevels, single_desc),
          vertex(kW, kH, kLevels, vec4_desc), pred_vertex(kW, kH, kLevels, vec4_desc),
          pred_normal(kW, kH, kLevels, vec4_desc), normal_scratch(kW, kH, vec4_desc) {
        kernel::initializeGrid(grid.getStruct(), Voxel());
        if (vis_n > 0) {
            vis = std::make_unique<VoxelGrid>(vis_width, vis_n, vis_mue_scale);
            kernel::initializeGrid(vis->getStruct(), Voxel());
        }
    }

    void preprocess() {   // depthFrameToVertexPyramid
        t.preprocess += kernel::convertToDepthMeters(raw, meters, depth_scale, unmirror);
        t.preprocess += kernel::applyBilateralFilter(meters, depth[0]);
        t.preprocess += kernel::createVertexMap(depth[0], vertex[0], sensor.getInverseIntr(0));
        for (int i = 1; i < kLevels; ++i) {
            t.preprocess += kernel::downSample(depth[i - 1], depth[i]);
            t.preprocess += kernel::createVertexMap(depth[i], vertex[i], sensor.getInverseIntr(i));
        }
    }
    void raycast_all() {   // raycastTsdf
        for (int i = 0; i < kLevels; ++i)
            t.raycast += kernel::raycast(grid.getStruct(), sensor, pred_vertex[i], pred_normal[i], i);
    }
    int compute_pose() {   // computePose
        try {
            RigidTransform3D p = icp.computePose(vertex, pred_vertex, pred_normal, sensor);
            sensor.setPose(p.getTransformation());
            auto e = icp.getExecutionTimes();
            t.icp_residuals += e[0];
            t.icp_solve += e[1];
            return 0;
        } catch (const std::exception&) {
            return 1;
        }
    }
    void fuse() {   // fuseCurrentDepthToTSDF
        t.fuse += kernel::fuse(meters, grid.getStruct(), sensor);
        if (vis) t.vis += kernel::fuse(meters, vis->getStruct(), sensor);
    }
    void visualize() {   // visualizeCurrentModel's raycast (the moving sensor's view)
        if (vis) t.vis += kernel::raycast(vis->getStruct(), sensor, pred_vertex[0], pred_normal[0], 0);
    }
};

bool copy_map(const CudaGridMap& m, void* dst, size_t elem) {
    const auto d = m.getGridDims();
    return cudaMemcpy2DFromArray(dst, d[0] * elem, m.getCudaArray(), 0, 0, d[0] * elem, d[1],
                                 cudaMemcpyDeviceToHost) == cudaSuccess;
}

bool clear_map(const CudaGridMap& m, size_t elem) {
    const auto d = m.getGridDims();
    std::vector<unsigned char> z(size_t(d[0]) * d[1] * elem, 0);
    return cudaMemcpy2DToArray(m.getCudaArray(), 0, 0, z.data(), d[0] * elem, d[0] * elem, d[1],
                               cudaMemcpyHostToDevice) == cudaSuccess;
}

bool copy_volume(const VoxelGridStruct& g, float* host, bool to_device) {
    cudaMemcpy3DParms p = {};
    const cudaPitchedPtr hp = make_cudaPitchedPtr(host, size_t(g.n) * 2 * sizeof(float), g.n, g.n);
    if (to_device) {
        p.srcPtr = hp;
        p.dstArray = g.cuda_array;
        p.kind = cudaMemcpyHostToDevice;
    } else {
        p.srcArray = g.cuda_array;
        p.dstPtr = hp;
        p.kind = cudaMemcpyDeviceToHost;
    }
    p.extent = make_cudaExtent(g.n, g.n, g.n);
    return cudaMemcpy3D(&p) == cudaSuccess;
}

glm::mat4 to_mat4(const float* cm) {   // column-major 16 floats
    glm::mat4 m;
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) m[c][r] = cm[c * 4 + r];
    return m;
}

void from_mat4(const glm::mat4& m, float* cm) {
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) cm[c * 4 + r] = m[c][r];
}

int cuda_status() { return cudaGetLastError() == cudaSuccess ? 0 : 2; }

}  // namespace

extern "C" {

// Status codes: 0 ok, 1 ICP solve not finite (pose kept), 2 CUDA error, 3 bad argument.

// iters[l]: ICP iterations of level l (0 = finest), the reference's iters_per_layer.
void* kfref_create(int n, float width, float mue_scale, float fov, float depth_scale, const int* iters,
                   float dist_thresh, float angle_thresh, float stop_angle, float stop_dist, int vis_n,
                   float vis_width, float vis_mue_scale) {
    if (n <= 0 || n % 8 || !iters || (vis_n > 0 && vis_n % 8)) return nullptr;
    IcpConfig ic;
    ic.iters_per_layer = {unsigned(iters[0]), unsigned(iters[1]), unsigned(iters[2])};
    ic.width = kW;
    ic.height = kH;
    ic.distance_thresh = dist_thresh;
    ic.angle_thresh = angle_thresh;
    ic.iteration_stop_thresh_angle = stop_angle;
    ic.iteration_stop_thresh_distance = stop_dist;
    try {
        auto* h = new Harness(n, width, mue_scale, fov, depth_scale, ic, vis_n, vis_width, vis_mue_scale);
        if (cudaDeviceSynchronize() != cudaSuccess) {
            delete h;
            return nullptr;
        }
        return h;
    } catch (const std::exception&) {
        return nullptr;
    }
}

void kfref_destroy(void* p) { delete static_cast<Harness*>(p); }

int kfref_set_pose(void* p, const float* pose_cm) {
    if (!p || !pose_cm) return 3;
    static_cast<Harness*>(p)->sensor.setPose(to_mat4(pose_cm));
    return 0;
}

int kfref_get_pose(void* p, float* pose_cm) {
    if (!p || !pose_cm) return 3;
    from_mat4(static_cast<Harness*>(p)->sensor.getPose(), pose_cm);
    return 0;
}

// upload one raw frame (uint16, 640 x 480) the way DepthMap::update(void*) does
int kfref_upload(void* p, const uint16_t* raw) {
    if (!p || !raw) return 3;
    static_cast<Harness*>(p)->raw.update(const_cast<uint16_t*>(raw));
    return cuda_status();
}

// the stages, each on the current frame / pose
int kfref_convert(void* p) {   // convertToDepthMeters alone (the first frame's preprocess)
    if (!p) return 3;
    auto* h = static_cast<Harness*>(p);
    h->t.preprocess += kernel::convertToDepthMeters(h->raw, h->meters, h->depth_scale, h->unmirror);
    return cuda_status();
}
int kfref_preprocess(void* p) {
    if (!p) return 3;
    static_cast<Harness*>(p)->preprocess();
    return cuda_status();
}
int kfref_raycast(void* p) {
    if (!p) return 3;
    static_cast<Harness*>(p)->raycast_all();
    return cuda_status();
}
int kfref_compute_pose(void* p) {
    if (!p) return 3;
    const int s = static_cast<Harness*>(p)->compute_pose();
    const int c = cuda_status();
    return c ? c : s;
}
int kfref_fuse(void* p) {
    if (!p) return 3;
    static_cast<Harness*>(p)->fuse();
    return cuda_status();
}
int kfref_visualize(void* p) {
    if (!p) return 3;
    static_cast<Harness*>(p)->visualize();
    return cuda_status();
}

// the reference's frame loop: frame 0 as initializeTracking, later frames as one iteration
// of startTracking's loop
int kfref_process_frame(void* p, const uint16_t* raw) {
    if (!p || !raw) return 3;
    auto* h = static_cast<Harness*>(p);
    h->raw.update(const_cast<uint16_t*>(raw));
    int s = 0;
    if (h->frames == 0) {
        h->t.preprocess += kernel::convertToDepthMeters(h->raw, h->meters, h->depth_scale, h->unmirror);
        h->fuse();
    } else {
        h->preprocess();
        h->raycast_all();
        s = h->compute_pose();
        h->fuse();
        h->visualize();
    }
    ++h->frames;
    const int c = cuda_status();
    return c ? c : s;
}

// wall-clock seconds of nframes iterations of the frame loop over the given frames (cycled),
// each uploading its frame from host memory; statuses of the frames in status (may be NULL)
int kfref_time_frames(void* p, const uint16_t* frames, int nframes_avail, int nframes, double* seconds,
                      int* status) {
    if (!p || !frames || nframes_avail <= 0 || nframes < 0 || !seconds) return 3;
    const size_t px = size_t(kW) * kH;
    cudaDeviceSynchronize();
    const auto t0 = std::chrono::steady_clock::now();
    int worst = 0;
    for (int i = 0; i < nframes; ++i) {
        const int s = kfref_process_frame(p, frames + px * size_t(i % nframes_avail));
        if (status) status[i] = s;
        if (s == 2 || s == 3) return s;
        worst = s > worst ? s : worst;
    }
    cudaDeviceSynchronize();
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return cuda_status();
}

// the reference's own per-stage CUDA-event / host times (ms, summed since creation):
// preprocess, raycast, ICP residuals, ICP solve, fuse, visualization
int kfref_stage_times(void* p, double* ms6) {
    if (!p || !ms6) return 3;
    const Times& t = static_cast<Harness*>(p)->t;
    const double v[6] = {t.preprocess, t.raycast, t.icp_residuals, t.icp_solve, t.fuse, t.vis};
    std::memcpy(ms6, v, sizeof(v));
    return 0;
}

int kfref_frames(void* p) { return p ? static_cast<Harness*>(p)->frames : -1; }
int kfref_set_frames(void* p, int f) {
    if (!p || f < 0) return 3;
    static_cast<Harness*>(p)->frames = f;
    return 0;
}

// maps: which 0 converted metres (float), 1 filtered depth (float), 2 vertex map (float4),
// 3 raycast vertex map (float4), 4 raycast normal map (float4), 5 the level's createNormalMap
// of map 2 (float4; computed on request)
int kfref_get_map(void* p, int which, int level, float* out) {
    if (!p || !out || level < 0 || level >= kLevels || which < 0 || which > 5) return 3;
    auto* h = static_cast<Harness*>(p);
    switch (which) {
        case 0: return level == 0 && copy_map(h->meters, out, 4) ? 0 : 3;
        case 1: return copy_map(h->depth[level], out, 4) ? 0 : 2;
        case 2: return copy_map(h->vertex[level], out, 16) ? 0 : 2;
        case 3: return copy_map(h->pred_vertex[level], out, 16) ? 0 : 2;
        case 4: return copy_map(h->pred_normal[level], out, 16) ? 0 : 2;
        default: {
            if (level != 0) return 3;   // the scratch map is level-0 sized
            kernel::createNormalMap(h->vertex[0], h->normal_scratch);
            return copy_map(h->normal_scratch, out, 16) ? cuda_status() : 2;
        }
    }
}

// zero the raycast maps of every level (rays that return early leave them as they were,
// project/src/raycast.cu:61-73)
int kfref_clear_raycast_maps(void* p) {
    if (!p) return 3;
    auto* h = static_cast<Harness*>(p);
    for (int l = 0; l < kLevels; ++l)
        if (!clear_map(h->pred_vertex[l], 16) || !clear_map(h->pred_normal[l], 16)) return 2;
    return 0;
}

// the volume as interleaved (distance, weight) floats, x fastest (VoxelGrid::saveVoxelGrid's
// layout, project/src/voxel_grid.cpp:43-60); vis selects the visualization grid
int kfref_get_tsdf(void* p, int vis, float* out) {
    if (!p || !out) return 3;
    auto* h = static_cast<Harness*>(p);
    if (vis && !h->vis) return 3;
    return copy_volume(vis ? h->vis->getStruct() : h->grid.getStruct(), out, false) ? 0 : 2;
}
int kfref_set_tsdf(void* p, int vis, const float* in) {
    if (!p || !in) return 3;
    auto* h = static_cast<Harness*>(p);
    if (vis && !h->vis) return 3;
    return copy_volume(vis ? h->vis->getStruct() : h->grid.getStruct(), const_cast<float*>(in), true) ? 0 : 2;
}

// kernel::constructIcpResiduals at one level against the raycast maps (project/src/icp.cu:
// 88-105): A (w * h x 6, row-major) and b (w * h) for the given previous and current poses
int kfref_icp_residuals(void* p, int level, const float* prev_cm, const float* cur_cm, float dist_thresh,
                        float angle_thresh, float* A, float* b) {
    if (!p || level < 0 || level >= kLevels || !prev_cm || !cur_cm || !A || !b) return 3;
    auto* h = static_cast<Harness*>(p);
    const RigidTransform3D prev(to_mat4(prev_cm)), cur(to_mat4(cur_cm));
    const auto d = h->vertex[level].getGridDims();
    const size_t n = size_t(d[0]) * d[1];
    float *dA = nullptr, *db = nullptr;
    if (cudaMalloc(&dA, n * 6 * sizeof(float)) != cudaSuccess) return 2;
    if (cudaMalloc(&db, n * sizeof(float)) != cudaSuccess) {
        cudaFree(dA);
        return 2;
    }
    kernel::constructIcpResiduals(h->vertex[level], h->pred_vertex[level], h->pred_normal[level], prev.rot_mat,
                                  prev.transl_vec, cur.rot_mat, cur.transl_vec, h->sensor.getIntr(level),
                                  dist_thresh, angle_thresh, dA, db);
    const bool ok = cudaMemcpy(A, dA, n * 6 * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess &&
                    cudaMemcpy(b, db, n * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess;
    cudaFree(dA);
    cudaFree(db);
    return ok ? cuda_status() : 2;
}

// poseError (project/src/general_helper.cpp:11-21), the reference's own host function: the
// chord between the two rotations' images of normalize(1, 1, 1) and the distance between the
// translations of two column-major poses.  Host only: it needs no device.
int kfref_pose_error(const float* pose1_cm, const float* pose2_cm, float* out2) {
    if (!pose1_cm || !pose2_cm || !out2) return 3;
    const std::pair<float, float> e = poseError(to_mat4(pose1_cm), to_mat4(pose2_cm));
    out2[0] = e.first;
    out2[1] = e.second;
    return 0;
}

// RgbdDataset (project/src/rgbd_dataset.cpp:6-96), the reference's own TUM RGB-D reader: load
// a sequence directory (groundtruth.txt, depth.txt), then walk its frames in order, each the
// depth image's path and the ground-truth pose of the nearest timestamp found by the
// reference's forward search.  Host only.  The reference indexes the first frame without a
// check, so a directory without both files or without frames is refused here first.
void* kfref_tum_open(const char* dir) {
    if (!dir) return nullptr;
    const std::string root(dir);
    std::ifstream gt(root + "/groundtruth.txt"), dl(root + "/depth.txt");
    if (!gt || !dl) return nullptr;
    std::string line;
    int depth_lines = 0;
    while (std::getline(dl, line)) ++depth_lines;
    if (depth_lines <= 3) return nullptr;
    auto* d = new RgbdDataset;
    d->load(root);
    return d;
}

void kfref_tum_close(void* d) { delete static_cast<RgbdDataset*>(d); }

// the next frame: its pose (getCurrentPose) and its path (getNextDepthImagePath); 1 while
// frames remain, 0 once the sequence is finished, 3 when the path does not fit path_len
int kfref_tum_next(void* p, char* path, int path_len, float* pose_cm) {
    auto* d = static_cast<RgbdDataset*>(p);
    if (!d || !path || path_len <= 0 || !pose_cm) return 3;
    if (d->isFinished()) return 0;
    from_mat4(d->getCurrentPose(), pose_cm);
    const std::string s = d->getNextDepthImagePath();
    if (int(s.size()) >= path_len) return 3;
    std::memcpy(path, s.c_str(), s.size() + 1);
    return 1;
}

int kfref_tum_initial_pose_inverse(void* p, float* out_cm) {
    auto* d = static_cast<RgbdDataset*>(p);
    if (!d || !out_cm) return 3;
    from_mat4(d->getInitialPoseInverse(), out_cm);
    return 0;
}

// Sensor (project/src/sensor.h:10-52), the reference's own camera: the level's intrinsics
// (fov on the diagonal, its fixed principal points 319.5 / 159.5 / 79.5 and 239.5 / 119.5 /
// 59.5) and their glm::inverse, both column-major 3 x 3.  Host only.
int kfref_sensor_intrinsics(float fov, int level, float* k_cm, float* inv_k_cm) {
    if (level < 0 || level >= kLevels || !k_cm || !inv_k_cm) return 3;
    const Sensor sensor(fov);
    const glm::mat3 k = sensor.getIntr(level), ik = sensor.getInverseIntr(level);
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) {
            k_cm[c * 3 + r] = k[c][r];
            inv_k_cm[c * 3 + r] = ik[c][r];
        }
    return 0;
}

}  // extern "C"
