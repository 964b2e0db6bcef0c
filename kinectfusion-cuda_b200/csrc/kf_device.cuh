// kf_device.cuh -- device-side layout of sessions in HBM and the helpers every kernel shares.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cuda/atomic>

#include "../../include/kf_api.h"

namespace kf {

constexpr int kMaxLevels = KF_MAX_LEVELS;
constexpr float kValid = -1.0f;     // project/src/device_helper.cuh:9
constexpr float kInvalid = -2.0f;   // project/src/device_helper.cuh:10
constexpr float kMinDepth = 0.01f;  // project/src/device_helper.cuh:11
constexpr int kMaxBilateralRadius = 7;

// one pyramid level of one session
struct LevelDev {
    int w, h;        // map size (W >> l, H >> l)
    int cw, ch;      // extent the 8x8-block stages write (compat_trunc8), else w, h
    int icw, ich;    // extent of the ICP residual grid (compat_trunc8), else w, h
    float fx, fy, cx, cy;   // K_l
    float ik[9];            // K_l^-1, column-major
};

// device-resident pose state of one session (updated by the ICP kernel, never by the host
// during a frame)
struct PoseDev {
    double R[9], t[3];      // ICP estimate, camera->world, column-major R
    double Rp[9], tp[3];    // pose of the previous frame
    float Rpf[9], tpf[3];   // float copy of the previous pose (raycast, correspondence)
    float iRf[9], itf[3];   // inverse of the frame's final pose (world->camera) for fusion
    int iters[kMaxLevels];  // ICP iterations run per level in the current frame
    int level;              // level of the next ICP pass (-1 once ICP is finished)
    int it;                 // iteration index within that level
    int cont;               // 1 while this session takes part in the next ICP pass
    int status;             // kf_status of the current frame
    int frame;              // frames processed so far
    int fuse_ok;            // 1 when this frame's fusion runs
};

// a session's visualization volume (n = 0: none): a second TSDF in the session's format, fused
// at the frame's pose from the same depth map, never raycast by the frame step
struct VisDev {
    int n, nb, ns;          // voxels, bricks and super-bricks per axis
    float vol_w, mu;
    void* tf;
    void* tw;
    const float* xs;
    const float* zs;
    int* bmin;
    int* bdil;
    int* sdil;
};

// everything a kernel needs about one session; an array of these lives in device memory
struct SessionDev {
    int W, H, L;
    float depth_scale;
    int unmirror, trunc8;
    float bil_inv_ss, bil_inv_sr, down_thr;
    int bil_r;
    LevelDev lv[kMaxLevels];
    // maps
    const uint16_t* raw;   // input frame (w*h uint16)
    float* depth_m;        // unfiltered metres (fusion input)
    float* dmax16;         // per 16x16-pixel tile of depth_m: largest valid depth (0: none)
    int t16w, t16h;        // tiles per row / column
    float* depth[kMaxLevels];
    float4* vmap[kMaxLevels];
    float4* pv[kMaxLevels];   // predicted (raycast) vertices, world frame
    float4* pn[kMaxLevels];   // predicted normals, world frame
    uint8_t* mask[kMaxLevels];// ICP correspondence masks (null unless exported)
    // debug mode only (null otherwise): per-pixel march decision traces of the last raycast,
    // see ray_trace_code in k_raycast.cu
    unsigned long long* trace[kMaxLevels];
    // volume
    int n, fmt;
    float vol_w, res, mu, max_w;
    void* tf;              // distance array (float or __half)
    void* tw;              // weight array (float or uint16)
    const float* xs;       // voxel-centre x (= y) coordinates, n floats
    const float* zs;       // voxel-centre z coordinates accumulated as the reference does
    // 8^3-voxel bricks: a lower bound of the brick's distances (order-preserving int keys,
    // kept by fusion with atomic minima) and the same widened to the 2 x 2 x 2 bricks a
    // trilinear sample can touch, which the raycaster reads to skip samples
    int* bmin;
    int* bdil;
    int* sdil;             // the same for 32^3 super-bricks (bricks [4s, 4s + 4] per axis)
    int nb;                // bricks per axis (n / 8)
    int ns;                // super-bricks per axis (ceil(nb / 4))
    float min_d, max_d, step_l, step_s;
    int keep_on_miss;
    // ICP
    int iters[kMaxLevels];
    float dist_th, angle_th, stop_a, stop_d;
    float angle_cos;       // cos(angle_th): the normal test compares cosines
    PoseDev* pose;
    VisDev vis;
};

// per-step control, written by the host: which sessions take part and which are on their
// first frame (fusion only, project/src/kinect_fusion.cpp:75-94)
struct StepDev {
    int active;
    int first;
};

// per-session result block copied back to the host after a step
struct OutDev {
    float pose[16];
    int iters[kMaxLevels];
    int status;
    int frame;
    int pad[3];
};

// work items
struct PreTile { int s, x0, y0; };                 // 32x32 level-0 tile
struct RayTile { int s, level, x0, y0; };          // ray tile
struct IcpTile { int s, p0, np; };                 // pixel range of one level's ICP grid
struct IcpRange { int begin, end; };               // tiles of one session at one level

// bounded grid barrier for cooperative launches: a monotonically increasing arrival counter
// plus an abort flag.  A wait that exceeds the limit sets abort and reports failure, so no
// block spins forever.
struct GridSync {
    unsigned int count;
    unsigned int abort;
    unsigned int timeouts;
    unsigned int pad;
};

// ------------------------------------------------------------------------------------------
// helpers
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ bool depth_valid(float d) {   // project/src/device_helper.cuh:14-17
    return d > kMinDepth && isfinite(d);
}

// isValid with cudaBoundaryModeZero (project/src/device_helper.cuh:37-44)
__device__ __forceinline__ bool map_valid(const float4* m, int w, int h, int i, int j) {
    if (i < 0 || j < 0 || i >= w || j >= h) return false;
    return __ldg(&m[size_t(j) * w + i].w) == kValid;
}

struct F3 { float x, y, z; };
__device__ __forceinline__ F3 f3(float4 v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 operator*(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
// column-major 3x3 times vector
__device__ __forceinline__ F3 mv3(const float* m, F3 v) {
    return {m[0] * v.x + m[3] * v.y + m[6] * v.z, m[1] * v.x + m[4] * v.y + m[7] * v.z,
            m[2] * v.x + m[5] * v.y + m[8] * v.z};
}

// device_helper::computeNormal (project/src/device_helper.cuh:81-110): normalised
// cross(v(i+1,j) - v, v(i,j+1) - v) when the three vertices are valid; a degenerate cross
// product gives NaN components with a valid tag, as in the reference.
__device__ __forceinline__ float4 compute_normal(const float4* m, int w, int h, int i, int j) {
    if (map_valid(m, w, h, i, j) && map_valid(m, w, h, i + 1, j) && map_valid(m, w, h, i, j + 1)) {
        const F3 c = f3(__ldg(&m[size_t(j) * w + i]));
        const F3 r = f3(__ldg(&m[size_t(j) * w + i + 1]));
        const F3 d = f3(__ldg(&m[size_t(j + 1) * w + i]));
        F3 n = cross3(r - c, d - c);
        const float s = rsqrtf(dot3(n, n));
        n = n * s;
        return make_float4(n.x, n.y, n.z, kValid);
    }
    return make_float4(0.f, 0.f, 0.f, kInvalid);
}

// uint16 -> fp16 value -> float (project/src/measurement.cu:19-21: __half2float of an
// unsigned short converts the value with round-to-nearest-even)
__device__ __forceinline__ float raw_to_half_value(uint16_t u) {
    return __half2float(__ushort2half_rn(u));
}

// distance loads for the two voxel formats
__device__ __forceinline__ float load_f(const float* f, size_t i) { return __ldg(f + i); }
__device__ __forceinline__ float load_f(const __half* f, size_t i) { return __half2float(__ldg(f + i)); }

// The base voxel of a trilinear sample at texel coordinates (x, y, z) (already uvw * n - 0.5):
// the low taps clamped to [0, n-1], the fractional weights, and whether the high tap is the
// next voxel along each axis or the same one (index below 0, or at n-1 and above, where
// clamping makes both taps equal).
struct TexelBase {
    float ax, ay, az;
    int x0, y0, z0;
    bool hx, hy, hz;
};

__device__ __forceinline__ TexelBase texel_base(int n, float x, float y, float z) {
    TexelBase b;
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    b.ax = x - fx;
    b.ay = y - fy;
    b.az = z - fz;
    const int ix = int(fx), iy = int(fy), iz = int(fz);
    b.x0 = min(max(ix, 0), n - 1);
    b.y0 = min(max(iy, 0), n - 1);
    b.z0 = min(max(iz, 0), n - 1);
    b.hx = unsigned(ix) < unsigned(n - 1);
    b.hy = unsigned(iy) < unsigned(n - 1);
    b.hz = unsigned(iz) < unsigned(n - 1);
    return b;
}

// trilinear sample of the distance array from its base voxel: what tex3D<float2>(...).x
// returns with normalized coordinates, linear filtering and clamp addressing
// (project/src/voxel_grid.cpp:24-33), computed with exact float weights.  n^3 < 2^32, so the
// offsets are 32-bit.
template <class TF>
__device__ __forceinline__ float trilinear_at(const TF* f, int n, const TexelBase& b) {
    const unsigned int un = unsigned(n);
    const TF* p00 = f + ((unsigned(b.z0) * un + unsigned(b.y0)) * un + unsigned(b.x0));
    const int dx = b.hx ? 1 : 0;
    const unsigned int dy = b.hy ? un : 0u;
    const unsigned int dz = b.hz ? un * un : 0u;
    const TF* p10 = p00 + dy;
    const TF* p01 = p00 + dz;
    const TF* p11 = p01 + dy;
    const float v000 = load_f(p00, 0), v100 = load_f(p00, dx);
    const float v010 = load_f(p10, 0), v110 = load_f(p10, dx);
    const float v001 = load_f(p01, 0), v101 = load_f(p01, dx);
    const float v011 = load_f(p11, 0), v111 = load_f(p11, dx);
    // each lerp a (1 - w) + b w as one rounded product and one fused multiply-add, spelled
    // out so every kernel that samples the volume rounds identically
    const float bx = __fsub_rn(1.f, b.ax), by = __fsub_rn(1.f, b.ay), bz = __fsub_rn(1.f, b.az);
    const float c00 = __fmaf_rn(v100, b.ax, __fmul_rn(v000, bx));
    const float c10 = __fmaf_rn(v110, b.ax, __fmul_rn(v010, bx));
    const float c01 = __fmaf_rn(v101, b.ax, __fmul_rn(v001, bx));
    const float c11 = __fmaf_rn(v111, b.ax, __fmul_rn(v011, bx));
    const float c0 = __fmaf_rn(c10, b.ay, __fmul_rn(c00, by));
    const float c1 = __fmaf_rn(c11, b.ay, __fmul_rn(c01, by));
    return __fmaf_rn(c1, b.az, __fmul_rn(c0, bz));
}

// trilinear sample at texel coordinates (x, y, z)
template <class TF>
__device__ __forceinline__ float trilinear(const TF* f, int n, float x, float y, float z) {
    return trilinear_at(f, n, texel_base(n, x, y, z));
}

// globaltimer (ns) for bounded waits
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;   // 2 s

// Grid-wide barrier for a cooperative launch.  `epoch` counts barriers passed by this
// block.  Returns false (in every thread of the block) when the wait timed out or another
// block aborted; callers then leave the kernel.
__device__ __forceinline__ bool grid_barrier(GridSync* g, unsigned int nblocks, unsigned int& epoch,
                                             unsigned long long timeout_ns = kBarrierTimeoutNs) {
    __syncthreads();
    int ok = 1;
    if (threadIdx.x == 0) {
        ++epoch;
        const unsigned int target = epoch * nblocks;
        // arrival releases the block's writes (the __syncthreads above orders them before
        // thread 0's), the acquiring load that sees every arrival makes the others' visible
        cuda::atomic_ref<unsigned int, cuda::thread_scope_device> cnt(g->count);
        cnt.fetch_add(1u, cuda::memory_order_release);
        const unsigned long long t0 = global_ns();
        unsigned int spins = 0;
        while (true) {
            const unsigned int c = cnt.load(cuda::memory_order_acquire);
            if (c >= target) break;
            if (*((volatile unsigned int*)&g->abort)) { ok = 0; break; }
            if ((++spins & 255u) == 0u && global_ns() - t0 > timeout_ns) {
                atomicExch(&g->abort, 1u);
                atomicAdd(&g->timeouts, 1u);
                ok = 0;
                break;
            }
            __nanosleep(32);
        }
    }
    return __syncthreads_and(threadIdx.x == 0 ? ok : 1) != 0;
}

}  // namespace kf
