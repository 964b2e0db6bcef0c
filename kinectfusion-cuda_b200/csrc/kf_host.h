// kf_host.h -- host-side interface between the C ABI layer and the kernel files.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kf_device.cuh"

namespace kf {

// Table sizes the kernels read from device memory, so that a captured graph stays valid
// when the work lists change (sessions opening and closing).
struct Tables {
    int S;                   // slot capacity (length of the session / step / range arrays)
    int n_pre;               // preprocessing tiles
    int n_ray;               // raycast tiles
    int n_itiles[kMaxLevels];// ICP tiles per level
    int icp_off[kMaxLevels]; // offset of each level's tiles in the ICP tile array
    int max_levels;
    int ray_budget;          // march iterations a lane takes before handing its ray to a warp
    int ray_tw;              // ray tile width (a warp's 32 rays are ray_tw x 32 / ray_tw pixels)
    int fuse_split;          // 0: fusion takes queue entries by the rule of fuse_split(); 1, 2, 4:
                             // whole, in halves or in quarters
    long long fuse_total;    // fusion segments over all slots
    long long vis_fuse_total;  // the same over the slots' visualization volumes
};

struct LongRay;   // march state of a ray handed from a lane to a warp (k_raycast.cu)
int serial_budget(int ray_tiles);   // ray_budget for a step with this many ray tiles
bool many_ray_tiles(int ray_tiles); // a step large enough for the raycast's long-budget, 4-block form

// raw pointers the kernels take
struct EngineView {
    const SessionDev* sess;
    const StepDev* step;
    OutDev* out;
    const Tables* tb;
    const PreTile* pre;
    const RayTile* ray;
    const IcpTile* itiles;
    const IcpRange* iranges;     // [level * S + s]
    const long long* fuse_prefix;// S + 1 entries, in segments
    const long long* vis_fuse_prefix;   // the same for the visualization volumes
    float* partials;             // ICP tile partials, kIcpPartialStride floats per tile
    float* partials2;            // a second set: a single session's odd passes (see icp_kernel)
    int4* icp_sched;             // per slot: {level of the next ICP pass or -1, first tile, tiles, 0}
    float* icp_mats;             // per slot: 24 floats phase A reads (R, t, K_l R_prev^T, t_prev)
    GridSync* sync;
    unsigned int* counters;      // [0] raycast tiles, [4] fusion blocks queued, [5] fusion
                                 // items taken, [6] long rays queued, [7] long rays taken,
                                 // [8], [9] the visualization volumes' [4], [5]
    LongRay* longq;              // long-ray queue
    int longq_cap;
    unsigned int* fuseq;         // fusion queue: global unit index of each block that can update
    int fuseq_cap;
    unsigned int* vis_fuseq;     // the visualization volumes' fusion queue
    int vis_fuseq_cap;
    unsigned long long* ray_counts;   // debug mode: the raycast's work counts (null: not counted)
};

constexpr int kPreTileSize = 32;
constexpr int kRayTileW = 8;   // default ray tile width; one warp per 32-ray tile
constexpr int kIcpThreads = 256;
constexpr int kIcpPxPerThread = 8;
constexpr int kIcpTilePx = kIcpThreads * kIcpPxPerThread;   // rows per block of the LLS stage
constexpr int kIcpTilesPerBlock = 4;  // ICP tiles per session-level per group
// A session-level's ICP tiles form kIcpGroups groups (group g: tiles g, g + G, g + 2 G, ...);
// each group is accumulated by one block into one partial, and the partials are combined in
// group order.  G is a constant -- not the launch's grid -- so that a session's arithmetic is
// the same in any grid, batch or tuning.
constexpr int kIcpGroups = 148;
constexpr int kIcpMinTile = kIcpThreads * 4;   // smallest ICP tile: 4 pixels per thread
constexpr int kIcpPartialStride = 56; // floats per ICP tile partial: 27 (sum, compensation) pairs + pad
constexpr int kIcpMaxPasses = 64;     // hard cap on ICP passes per frame

// launch helpers (each returns the CUDA error of its launch)
cudaError_t launch_preprocess(const EngineView& v, int grid, cudaStream_t st);
// many: a step of more than kManyRayTiles ray tiles (serial_budget's rule)
cudaError_t launch_raycast(const EngineView& v, int grid, cudaStream_t st, bool many);
int serial_budget_many();   // the lane budget of the raycast's many-tile form
int ray_count_slots();      // entries of the raycast's debug work counts
// single: an engine of one slot (the kernel keeps that session's state per block)
cudaError_t launch_icp(const EngineView& v, int grid, cudaStream_t st, bool single);
cudaError_t launch_fuse(const EngineView& v, int grid, cudaStream_t st);
// the same for the sessions' visualization volumes (cull, fuse and bounds)
cudaError_t launch_fuse_vis(const EngineView& v, int grid, cudaStream_t st);
// bounds = key(2), the initial distance; rebuild recomputes them exactly from a loaded volume
cudaError_t launch_init_bricks(int* bmin, int* bdil, int* sdil, int n, cudaStream_t st);
cudaError_t launch_rebuild_bricks(const void* f, int fmt, int n, int* bmin, int* bdil, int* sdil, cudaStream_t st);
int icp_max_grid(int num_sms);
int long_ray_bytes();
cudaError_t launch_barrier_selftest(GridSync* g, unsigned long long timeout_ns, int* result, cudaStream_t st);
cudaError_t launch_read_probe(const float4* buf, long long n4, int rounds, float* sink, int grid, cudaStream_t st);
__host__ __device__ int fuse_units(int n);   // 32 x 8 x 8 voxel blocks of an n^3 volume

cudaError_t launch_init_volume(void* f, void* w, long long nvox, int fmt, cudaStream_t st);
cudaError_t launch_export_interleaved(const void* f, const void* w, long long nvox, int fmt, float* dst, cudaStream_t st);
cudaError_t launch_import_interleaved(const float* src, void* f, void* w, long long nvox, int fmt, cudaStream_t st);

// stage kernels (per-stage C ABI)
cudaError_t stage_convert(const uint16_t* raw, float* out, int w, int h, float scale, int unmirror, cudaStream_t st);
cudaError_t stage_bilateral(const float* in, float* out, int w, int h, float ss, float sr, int r, cudaStream_t st);
cudaError_t stage_down_sample(const float* in, float* out, int wo, int ho, float sr, cudaStream_t st);
cudaError_t stage_vertex(const float* d, float4* v, int w, int h, const float* ik, cudaStream_t st);
cudaError_t stage_normal(const float4* v, float4* n, int w, int h, cudaStream_t st);
// bounds (optional): a session whose brick bounds the march may use to skip
cudaError_t stage_raycast(const kf_volume* vol, const float* pose, const float* ik, float4* vtx, float4* nrm, int w,
                          int h, float min_d, float max_d, float step_l, float step_s, cudaStream_t st,
                          const SessionDev* bounds = nullptr);
// headless display (project/src/display.cu): RGBA8 images
constexpr int kDisplayNormals = 0, kDisplayShading = 1, kDisplayFloat = 2;
struct DispMats {
    float r[9];    // normals: inverse sensor rotation; shading: sensor rotation (column-major)
    float ik[9];   // shading: inverse intrinsics (column-major)
};
cudaError_t stage_display(int mode, const void* src, int w, int h, const DispMats& m, float scale, unsigned int* out,
                          cudaStream_t st);
cudaError_t stage_fuse(const float* depth, int w, int h, const float* k, const kf_volume* vol, const float* pose,
                       float min_d, float max_d, const float* xs, const float* zs, cudaStream_t st);
cudaError_t stage_icp_residuals(const float4* vmap, const float4* tv, const float4* tn, int w, int h,
                                const float* Rp, const float* tp, const float* Rc, const float* tc, const float* k,
                                float dist, float angle, float* A, float* b, cudaStream_t st);
// LinearLeastSquares::solve: partials of the normal equations then an FP64 combine + solve
int lls_num_blocks(int n);
cudaError_t stage_lls(const float* A, const float* b, int n, float* partials, double* x_dev, int nblocks,
                      cudaStream_t st);

// host math shared by the API layer
void voxel_axes(int n, float width, float* xs, float* zs);
void level_intrinsics(const kf_config& c, int level, float k[9], float ik[9]);

}  // namespace kf
