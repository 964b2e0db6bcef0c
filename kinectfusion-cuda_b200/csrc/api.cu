// api.cu -- the C ABI (include/kf_api.h): sessions, per-stage calls, batches and the server.
//
// Host orchestration replaces KinectFusion (project/src/kinect_fusion.cpp), ICP
// (project/src/icp.cpp) and LinearLeastSquares (project/src/linear_least_squares.cpp).
// An Engine owns a set of session slots and the four per-step launches (preprocess,
// raycast, ICP, fusion) over all of them; the launches plus the result copy are captured
// once into a CUDA graph and replayed every step.  Work lists and per-session parameters
// live in device memory, so sessions can join and leave without re-capturing.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "kf_host.h"

using namespace kf;

namespace {

// NVTX range over a host call or a stage's launches (a no-op unless a tool such as ncu
// injects NVTX; `ncu --nvtx --nvtx-include kf.raycast/` then selects that stage's kernels)
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

thread_local cudaError_t g_last_cuda = cudaSuccess;

#define KF_CK(expr)                                  \
    do {                                             \
        cudaError_t e_ = (expr);                     \
        if (e_ != cudaSuccess) {                     \
            g_last_cuda = e_;                        \
            return KF_ERR_CUDA;                      \
        }                                            \
    } while (0)

#define KF_TRY(expr)                                 \
    do {                                             \
        kf_status s_ = (expr);                       \
        if (s_ != KF_OK) return s_;                  \
    } while (0)

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

// ---- configuration ----

kf_status validate(const kf_config& c) {
    if (c.width <= 0 || c.height <= 0) return KF_ERR_ARG;
    if (c.levels < 1 || c.levels > KF_MAX_LEVELS) return KF_ERR_ARG;
    const int div = 1 << (c.levels - 1);
    // GridMapPyramid::checkGridDimensions (project/src/grid_map_pyramid.h:63-72)
    if (c.width % div || c.height % div) return KF_ERR_SHAPE;
    if (c.compat_trunc8 && (c.width % 8 || c.height % 8)) return KF_ERR_SHAPE;
    if (c.volume_n < 8 || c.volume_n % 8) return KF_ERR_ARG;
    if (!(c.volume_width > 0.f) || !(c.mu > 0.f)) return KF_ERR_ARG;
    if (c.tsdf_format != KF_TSDF_F32F32 && c.tsdf_format != KF_TSDF_F16U16) return KF_ERR_ARG;
    if (c.bilateral_radius < 0 || c.bilateral_radius > kMaxBilateralRadius) return KF_ERR_ARG;
    if (!(c.bilateral_sigma_s > 0.f) || !(c.bilateral_sigma_r > 0.f)) return KF_ERR_ARG;
    // large steps must exceed small ones (the reference tells the two phases apart by them)
    if (!(c.step_small > 0.f) || !(c.step_large > c.step_small)) return KF_ERR_ARG;
    // a march step must still advance t in float at the far end of the range
    if (!(c.min_depth >= 0.f) || !(c.max_depth > c.min_depth) || !(c.max_depth < 1000.f)) return KF_ERR_ARG;
    if (!(c.mu * c.step_small > c.max_depth * 1e-6f)) return KF_ERR_ARG;
    if (c.vis_volume_n != 0 &&
        (c.vis_volume_n < 8 || c.vis_volume_n % 8 || !(c.vis_volume_width > 0.f) || !(c.vis_mu > 0.f)))
        return KF_ERR_ARG;
    int total = 0;
    for (int l = 0; l < c.levels; ++l) {
        if (c.iters[l] < 0) return KF_ERR_ARG;
        total += c.iters[l];
    }
    if (total > kIcpMaxPasses) return KF_ERR_ARG;
    return KF_OK;
}

size_t level_px(const kf_config& c, int l) { return size_t(c.width >> l) * size_t(c.height >> l); }

size_t footprint(const kf_config& c) {
    const size_t n3 = size_t(c.volume_n) * c.volume_n * c.volume_n;
    size_t b = n3 * (c.tsdf_format == KF_TSDF_F16U16 ? 4 : 8);
    b += size_t(c.width) * c.height * (2 + 4);
    for (int l = 0; l < c.levels; ++l) {
        b += level_px(c, l) * (4 + 16 * 3);
        if (c.export_icp_mask) b += level_px(c, l);
    }
    b += sizeof(float) * 2 * c.volume_n + sizeof(PoseDev);
    // brick bounds (bmin, bdil), super-brick bounds, depth-tile maxima
    const size_t nb = size_t(c.volume_n / 8), ns = (nb + 3) / 4;
    b += nb * nb * nb * 2 * sizeof(int) + ns * ns * ns * sizeof(int);
    b += sizeof(float) * size_t((c.width + 15) / 16) * ((c.height + 15) / 16);
    if (c.vis_volume_n) {   // the visualization volume: grid, axes, brick and super-brick bounds
        const size_t vn = size_t(c.vis_volume_n), vnb = vn / 8, vns = (vnb + 3) / 4;
        b += vn * vn * vn * (c.tsdf_format == KF_TSDF_F16U16 ? 4 : 8) + sizeof(float) * 2 * vn;
        b += vnb * vnb * vnb * 2 * sizeof(int) + vns * vns * vns * sizeof(int);
    }
    return b;
}

int cover8(int dim, int trunc) { return trunc ? (dim / 8) * 8 : dim; }
int cover_icp(int dim, int trunc) {
    if (!trunc) return dim;
    const int t = std::min(dim - 1, 8);
    if (t <= 0) return dim;
    return (dim / t) * t;
}

void pose16_to_double(const float* p, double* R, double* t) {
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) R[c * 3 + r] = p[c * 4 + r];
    for (int r = 0; r < 3; ++r) t[r] = p[12 + r];
}

// initial device pose state: estimate = previous = pose, float mirrors, inverse
PoseDev make_pose_dev(const float* pose16) {
    PoseDev P;
    std::memset(&P, 0, sizeof(P));
    pose16_to_double(pose16, P.Rp, P.tp);
    std::memcpy(P.R, P.Rp, sizeof(P.R));
    std::memcpy(P.t, P.tp, sizeof(P.t));
    for (int q = 0; q < 9; ++q) P.Rpf[q] = float(P.Rp[q]);
    for (int q = 0; q < 3; ++q) P.tpf[q] = float(P.tp[q]);
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) P.iRf[c * 3 + r] = float(P.Rp[r * 3 + c]);
    for (int r = 0; r < 3; ++r)
        P.itf[r] = float(-(P.Rp[r * 3 + 0] * P.tp[0] + P.Rp[r * 3 + 1] * P.tp[1] + P.Rp[r * 3 + 2] * P.tp[2]));
    P.level = -1;
    P.fuse_ok = 1;
    return P;
}

// ---- one session's device resources ----

// Device arenas a server keeps after its sessions close, for the next sessions to reuse: a
// session opening or closing then allocates and frees nothing (cudaFree waits for the whole
// device, which would stall every other session's frames).
struct ArenaPool {
    std::mutex mu;
    std::vector<std::pair<char*, size_t>> free;
    size_t cached = 0;   // bytes held in `free` (read without the lock only as an estimate)

    // the smallest cached arena of at least `need` bytes and at most about twice that
    char* take(size_t need, size_t& cap) {
        std::lock_guard<std::mutex> g(mu);
        int best = -1;
        for (int i = 0; i < int(free.size()); ++i)
            if (free[i].second >= need && free[i].second <= 2 * need + (16u << 20) &&
                (best < 0 || free[i].second < free[best].second))
                best = i;
        if (best < 0) return nullptr;
        char* p = free[best].first;
        cap = free[best].second;
        free.erase(free.begin() + best);
        cached -= cap;
        return p;
    }
    void put(char* p, size_t cap) {
        std::lock_guard<std::mutex> g(mu);
        free.emplace_back(p, cap);
        cached += cap;
    }
    // free cached arenas, largest first, until at most `keep` bytes stay cached
    void trim(size_t keep) {
        std::lock_guard<std::mutex> g(mu);
        while (cached > keep && !free.empty()) {
            int big = 0;
            for (int i = 1; i < int(free.size()); ++i)
                if (free[i].second > free[big].second) big = i;
            cudaFree(free[big].first);
            cached -= free[big].second;
            free.erase(free.begin() + big);
        }
    }
};

struct Slot {
    bool used = false;
    kf_config cfg{};
    SessionDev d{};
    std::vector<void*> allocs;    // buffers outside the arena
    char* arena = nullptr;        // one device allocation holding the session's buffers
    size_t arena_cap = 0, arena_used = 0;
    ArenaPool* pool = nullptr;    // set by a server: arenas come from and go back to it
    size_t bytes = 0;
    int frames = 0;
    kf_frame_stats stats{};
    float pose[16]{};
    bool external = false;   // maps supplied by the caller (kf_compute_pose)
    float4* render_v = nullptr;          // kf_render's own level-0 maps and image (lazily)
    float4* render_n = nullptr;
    unsigned int* render_rgba = nullptr;

    // reserve (and zero, on st) one arena for buffers of `need` bytes in all
    cudaError_t begin_arena(size_t need, cudaStream_t st) {
        if (pool) arena = pool->take(need, arena_cap);
        if (!arena) {
            cudaError_t e = cudaMalloc(&arena, need);
            if (e != cudaSuccess) { arena = nullptr; return e; }
            arena_cap = need;
        }
        arena_used = 0;
        zero_stream = st;
        return cudaMemsetAsync(arena, 0, need, st);
    }
    cudaStream_t zero_stream = nullptr;
    void* alloc(size_t nbytes, cudaError_t& err) {
        const size_t off = (arena_used + 255) & ~size_t(255);
        if (arena && off + nbytes <= arena_cap) {
            arena_used = off + nbytes;
            bytes += nbytes;
            err = cudaSuccess;
            return arena + off;
        }
        void* p = nullptr;
        err = cudaMalloc(&p, nbytes);
        if (err != cudaSuccess) return nullptr;
        allocs.push_back(p);
        bytes += nbytes;
        err = cudaMemsetAsync(p, 0, nbytes, zero_stream);
        return p;
    }
    void release() {
        for (void* p : allocs) cudaFree(p);
        allocs.clear();
        if (arena) {
            if (pool) pool->put(arena, arena_cap);
            else cudaFree(arena);
        }
        arena = nullptr;
        arena_cap = arena_used = 0;
        render_v = render_n = nullptr;
        render_rgba = nullptr;
        bytes = 0;
        used = false;
        external = false;
        frames = 0;
    }
};

// level geometry (shared by full sessions and external-map ICP runs)
void fill_levels(SessionDev& d, const kf_config& c) {
    d.W = c.width;
    d.H = c.height;
    d.L = c.levels;
    for (int l = 0; l < KF_MAX_LEVELS; ++l) {
        LevelDev& Lv = d.lv[l];
        std::memset(&Lv, 0, sizeof(Lv));
        if (l >= c.levels) continue;
        Lv.w = c.width >> l;
        Lv.h = c.height >> l;
        Lv.cw = cover8(Lv.w, c.compat_trunc8);
        Lv.ch = cover8(Lv.h, c.compat_trunc8);
        Lv.icw = cover_icp(Lv.w, c.compat_trunc8);
        Lv.ich = cover_icp(Lv.h, c.compat_trunc8);
        float k[9], ik[9];
        level_intrinsics(c, l, k, ik);
        Lv.fx = k[0]; Lv.fy = k[4]; Lv.cx = k[6]; Lv.cy = k[7];
        std::memcpy(Lv.ik, ik, sizeof(ik));
    }
    d.iters[0] = d.iters[1] = d.iters[2] = 0;
    for (int l = 0; l < c.levels; ++l) d.iters[l] = c.iters[l];
    d.dist_th = c.dist_thresh;
    d.angle_th = c.angle_thresh;
    d.angle_cos = float(std::cos(double(c.angle_thresh)));
    d.stop_a = c.stop_angle;
    d.stop_d = c.stop_dist;
}

// allocate and initialise a session's buffers; all device work on st, synchronised before
// returning (so a server can build a session while other sessions' steps run)
kf_status slot_create(Slot& s, const kf_config& c, cudaStream_t st = nullptr) {
    KF_TRY(validate(c));
    s.release();
    s.cfg = c;
    SessionDev& d = s.d;
    std::memset(&d, 0, sizeof(d));
    fill_levels(d, c);
    d.depth_scale = c.depth_scale;
    d.unmirror = c.unmirror;
    d.trunc8 = c.compat_trunc8;
    d.bil_inv_ss = 1.0f / (c.bilateral_sigma_s * c.bilateral_sigma_s);
    d.bil_inv_sr = 1.0f / (c.bilateral_sigma_r * c.bilateral_sigma_r);
    d.down_thr = 3.0f * c.bilateral_sigma_r;
    d.bil_r = c.bilateral_radius;
    cudaError_t err = s.begin_arena(footprint(c) + (64u << 10), st);   // + alignment of ~30 buffers
    if (err != cudaSuccess) { g_last_cuda = err; s.release(); return KF_ERR_CUDA; }
#define KF_ALLOC(ptr, type, bytes)                                   \
    do {                                                             \
        ptr = static_cast<type>(s.alloc((bytes), err));              \
        if (err != cudaSuccess) { g_last_cuda = err; s.release(); return KF_ERR_CUDA; } \
    } while (0)
    const size_t px = size_t(c.width) * c.height;
    uint16_t* raw;
    KF_ALLOC(raw, uint16_t*, px * 2);
    d.raw = raw;
    KF_ALLOC(d.depth_m, float*, px * 4);
    d.t16w = (c.width + 15) / 16;
    d.t16h = (c.height + 15) / 16;
    KF_ALLOC(d.dmax16, float*, sizeof(float) * size_t(d.t16w) * d.t16h);
    for (int l = 0; l < c.levels; ++l) {
        const size_t np = level_px(c, l);
        KF_ALLOC(d.depth[l], float*, np * 4);
        KF_ALLOC(d.vmap[l], float4*, np * 16);
        KF_ALLOC(d.pv[l], float4*, np * 16);
        KF_ALLOC(d.pn[l], float4*, np * 16);
        if (c.export_icp_mask) KF_ALLOC(d.mask[l], uint8_t*, np);
    }
    d.n = c.volume_n;
    d.fmt = c.tsdf_format;
    d.vol_w = c.volume_width;
    d.res = c.volume_width / float(c.volume_n - 1);
    d.mu = c.mu;
    d.max_w = c.max_weight;
    const size_t n3 = size_t(c.volume_n) * c.volume_n * c.volume_n;
    const size_t es = c.tsdf_format == KF_TSDF_F16U16 ? 2 : 4;
    KF_ALLOC(d.tf, void*, n3 * es);
    KF_ALLOC(d.tw, void*, n3 * es);
    float* xs;
    float* zs;
    KF_ALLOC(xs, float*, sizeof(float) * c.volume_n);
    KF_ALLOC(zs, float*, sizeof(float) * c.volume_n);
    std::vector<float> hx(c.volume_n), hz(c.volume_n);   // alive until the stream sync below
    voxel_axes(c.volume_n, c.volume_width, hx.data(), hz.data());
    err = cudaMemcpyAsync(xs, hx.data(), sizeof(float) * c.volume_n, cudaMemcpyHostToDevice, st);
    if (err == cudaSuccess) err = cudaMemcpyAsync(zs, hz.data(), sizeof(float) * c.volume_n, cudaMemcpyHostToDevice, st);
    if (err != cudaSuccess) { g_last_cuda = err; s.release(); return KF_ERR_CUDA; }
    d.xs = xs;
    d.zs = zs;
    d.min_d = c.min_depth;
    d.max_d = c.max_depth;
    d.step_l = c.step_large;
    d.step_s = c.step_small;
    d.keep_on_miss = c.keep_on_miss;
    KF_ALLOC(d.pose, PoseDev*, sizeof(PoseDev));
    d.nb = c.volume_n / 8;
    d.ns = (d.nb + 3) / 4;
    const long long nbricks = (long long)d.nb * d.nb * d.nb, nsuper = (long long)d.ns * d.ns * d.ns;
    KF_ALLOC(d.bmin, int*, sizeof(int) * size_t(nbricks));
    KF_ALLOC(d.bdil, int*, sizeof(int) * size_t(nbricks));
    KF_ALLOC(d.sdil, int*, sizeof(int) * size_t(nsuper));
    std::vector<float> vhx, vhz;   // alive until the stream sync below
    if (c.vis_volume_n) {
        VisDev& V = d.vis;
        V.n = c.vis_volume_n;
        V.nb = V.n / 8;
        V.ns = (V.nb + 3) / 4;
        V.vol_w = c.vis_volume_width;
        V.mu = c.vis_mu;
        const size_t vn3 = size_t(V.n) * V.n * V.n;
        KF_ALLOC(V.tf, void*, vn3 * es);
        KF_ALLOC(V.tw, void*, vn3 * es);
        float* vxs;
        float* vzs;
        KF_ALLOC(vxs, float*, sizeof(float) * V.n);
        KF_ALLOC(vzs, float*, sizeof(float) * V.n);
        vhx.resize(V.n);
        vhz.resize(V.n);
        voxel_axes(V.n, V.vol_w, vhx.data(), vhz.data());
        err = cudaMemcpyAsync(vxs, vhx.data(), sizeof(float) * V.n, cudaMemcpyHostToDevice, st);
        if (err == cudaSuccess) err = cudaMemcpyAsync(vzs, vhz.data(), sizeof(float) * V.n, cudaMemcpyHostToDevice, st);
        if (err != cudaSuccess) { g_last_cuda = err; s.release(); return KF_ERR_CUDA; }
        V.xs = vxs;
        V.zs = vzs;
        const size_t vnb3 = size_t(V.nb) * V.nb * V.nb, vns3 = size_t(V.ns) * V.ns * V.ns;
        KF_ALLOC(V.bmin, int*, sizeof(int) * vnb3);
        KF_ALLOC(V.bdil, int*, sizeof(int) * vnb3);
        KF_ALLOC(V.sdil, int*, sizeof(int) * vns3);
    }
#undef KF_ALLOC
    // grid {f = 2, w = 0} and pose = initial_pose (project/src/kinect_fusion.cpp:33-36, :80)
    err = launch_init_volume(d.tf, d.tw, (long long)n3, d.fmt, st);
    if (err == cudaSuccess) err = launch_init_bricks(d.bmin, d.bdil, d.sdil, c.volume_n, st);
    if (err == cudaSuccess && d.vis.n) {
        const long long vn3 = (long long)d.vis.n * d.vis.n * d.vis.n;
        err = launch_init_volume(d.vis.tf, d.vis.tw, vn3, d.fmt, st);
        if (err == cudaSuccess) err = launch_init_bricks(d.vis.bmin, d.vis.bdil, d.vis.sdil, d.vis.n, st);
    }
    const PoseDev P = make_pose_dev(c.initial_pose);
    if (err == cudaSuccess) err = cudaMemcpyAsync(d.pose, &P, sizeof(P), cudaMemcpyHostToDevice, st);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    if (err != cudaSuccess) { g_last_cuda = err; s.release(); return KF_ERR_CUDA; }
    s.used = true;
    s.frames = 0;
    std::memcpy(s.pose, c.initial_pose, sizeof(s.pose));
    s.stats = kf_frame_stats{};
    s.stats.frame = -1;
    return KF_OK;
}

kf_status slot_reset(Slot& s) {
    const kf_config& c = s.cfg;
    const size_t n3 = size_t(c.volume_n) * c.volume_n * c.volume_n;
    KF_CK(launch_init_volume(s.d.tf, s.d.tw, (long long)n3, s.d.fmt, 0));
    KF_CK(launch_init_bricks(s.d.bmin, s.d.bdil, s.d.sdil, c.volume_n, 0));
    if (s.d.vis.n) {
        const long long vn3 = (long long)s.d.vis.n * s.d.vis.n * s.d.vis.n;
        KF_CK(launch_init_volume(s.d.vis.tf, s.d.vis.tw, vn3, s.d.fmt, 0));
        KF_CK(launch_init_bricks(s.d.vis.bmin, s.d.vis.bdil, s.d.vis.sdil, s.d.vis.n, 0));
    }
    PoseDev P = make_pose_dev(c.initial_pose);
    KF_CK(cudaMemcpy(s.d.pose, &P, sizeof(P), cudaMemcpyHostToDevice));
    KF_CK(cudaDeviceSynchronize());
    s.frames = 0;
    std::memcpy(s.pose, c.initial_pose, sizeof(s.pose));
    s.stats = kf_frame_stats{};
    s.stats.frame = -1;
    return KF_OK;
}

// ---- engine: slots + launches ----

template <class T>
kf_status grow(T*& ptr, int& cap, int need) {
    if (need <= cap && ptr) return KF_OK;
    int nc = std::max(need, std::max(16, cap * 2));
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;   // a failed allocation leaves an empty buffer, never a stale capacity
    KF_CK(cudaMalloc(&ptr, sizeof(T) * size_t(nc)));
    KF_CK(cudaMemset(ptr, 0, sizeof(T) * size_t(nc)));
    cap = nc;
    return KF_OK;
}

// The long-ray queue holds 1 / kLongRayShare of a step's rays (about 2 % of a frame's rays take
// the long-ray path; more than the queue holds finish in their lane, several times slower), and
// at least a quarter of them up to kLongRayFloor entries, so that a small step (one session)
// has room for a scene with many more grazing rays.
constexpr int kLongRayShare = 16;
constexpr long long kLongRayFloor = 1 << 18;
long long long_ray_entries(long long rays) {
    return std::max(std::max(1024LL, rays / kLongRayShare), std::min(rays / 4, kLongRayFloor));
}

// Launch shapes of a step.  Every value gives the same results bit for bit -- they only change
// which block or lane does which part of the work -- so they can be tuned on live steps.
struct Shape {
    int grid_pre = 0, grid_ray = 0, grid_fuse = 0, grid_icp = 0;
    int ray_form = 0;     // 0: by the ray-tile count (many_ray_tiles); 3 or 4: the raycast kernel's
                          // form with that many blocks per SM
    int ray_budget = 0;   // 0: by the ray-tile count (serial_budget); else march iterations a lane
                          // takes before queueing its ray for a warp
    int ray_tw = kRayTileW;   // ray tile width (32 / ray_tw rows)
    int fuse_split = 0;   // 0: by the queue length (fuse_split); 1, 2, 4: entries whole, halves, quarters
    bool operator==(const Shape& o) const {
        return grid_pre == o.grid_pre && grid_ray == o.grid_ray && grid_fuse == o.grid_fuse &&
               grid_icp == o.grid_icp && ray_form == o.ray_form &&
               ray_budget == o.ray_budget && ray_tw == o.ray_tw && fuse_split == o.fuse_split;
    }
    bool operator!=(const Shape& o) const { return !(*this == o); }
};

// The autotuner's walk over the shapes: coordinate descent, one parameter at a time, each
// candidate run on kReps live steps and timed by the device time of those steps (the stage
// events from the fork to the end of fusion; the smallest time counts); the winner of each
// parameter is kept for the next.  The whole step is the objective because the stages share
// the GPU: the preprocess runs on a branch beside the raycast, and a preprocess grid that
// finishes its own branch sooner can delay the raycast.
struct Tuner {
    static constexpr int kReps = 2;
    struct Param {
        const char* name;
        int Shape::*field;
        std::vector<int> cand;
    };
    bool active = false;
    bool done = false;
    bool was_profiling = false;
    std::string cache_path, key;
    std::vector<Param> params;
    int pi = 0, ci = 0, rep = 0;
    std::vector<float> best;      // per candidate of the current parameter
    Shape base;                   // the shape the walk has settled on so far
    std::string report;           // JSON of the chosen shape and the step times behind it
    int steps_left() const {
        if (!active) return 0;
        int n = (int(params[pi].cand.size()) - ci) * kReps - rep;
        for (size_t q = pi + 1; q < params.size(); ++q) n += int(params[q].cand.size()) * kReps;
        return n;
    }
};

struct Engine {
    int sms = 148;
    int cap = 0;
    std::vector<Slot> slots;
    // device
    SessionDev* d_sess = nullptr;
    StepDev* d_step = nullptr;
    OutDev* d_out = nullptr;
    Tables* d_tb = nullptr;
    PreTile* d_pre = nullptr;
    RayTile* d_ray = nullptr;
    IcpTile* d_itiles = nullptr;
    IcpRange* d_iranges = nullptr;
    long long* d_fprefix = nullptr;
    long long* d_vfprefix = nullptr;   // the same three over the visualization volumes
    float* d_partials = nullptr;
    int4* d_icp_sched = nullptr;
    float* d_icp_mats = nullptr;
    // one block [OutDev x cap | GridSync | counters]: a step clears the wait record and the
    // counters with one memset, and a caller that reads the results copies them with one copy
    GridSync* d_sync = nullptr;
    unsigned int* d_ctr = nullptr;
    static constexpr int kCounters = 12;
    size_t out_bytes() const { return sizeof(OutDev) * cap + sizeof(GridSync); }
    int cap_pre = 0, cap_ray = 0, cap_it = 0, cap_part = 0;
    // long-ray queue of the raycaster (bytes; entries = bytes / long_ray_bytes())
    char* d_longq = nullptr;
    int cap_longq = 0;
    // fusion queue (one entry per block of every slot at most), and the visualization volumes'
    unsigned int* d_fuseq = nullptr;
    int cap_fuseq = 0;
    unsigned int* d_vfuseq = nullptr;
    int cap_vfuseq = 0;
    bool has_vis = false;      // some slot has a visualization volume: the step fuses it too
    unsigned long long* d_ray_counts = nullptr;   // debug mode KF_DEBUG_COUNTERS: raycast work counts
    bool count_rays = false;
    // work-list entries reserved ahead for sessions not open yet (reserve_work)
    long long res_pre = 0, res_ray = 0, res_it = 0, res_fq = 0, res_vfq = 0;
    // pinned host
    StepDev* h_step = nullptr;
    OutDev* h_out = nullptr;
    GridSync* h_sync = nullptr;
    Tables tb{};
    bool tables_dirty = true;
    bool step_dirty = true;
    Shape shape;
    Tuner tuner;
    // graph
    bool use_graph = true;
    bool graph_dirty = true;
    cudaGraphExec_t gexec = nullptr;
    cudaStream_t cap_stream = nullptr;
    // the preprocess of a frame runs on a branch beside its raycast (which reads the previous
    // frame's volume and pose only): fork and join events and the branch's stream
    cudaStream_t aux_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // frames from host memory: their copies run on h2d_stream while the step's raycast (which
    // needs only the previous frames) runs; the preprocess branch of the graph waits for
    // ev_input (an external event wait node), recorded after every step's copies
    bool input_wait = true;
    bool capturing = false;   // record() runs inside a stream capture (the wait becomes a node)
    bool ray_many = false;    // the raycast kernel's 4-block form (shape.ray_form, else the tile-count rule)
    cudaStream_t h2d_stream = nullptr;
    cudaEvent_t ev_input = nullptr, ev_prev = nullptr;
    bool stages[4] = {true, true, true, true};
    // per-stage timing: events between the launches (also inside the captured graph)
    bool profile = false;
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};

    kf_status init(int capacity) {
        if (capacity <= 0 || capacity > 1024) return KF_ERR_ARG;   // ICP kernel keeps 1024 slots in smem
        cap = capacity;
        slots.resize(capacity);
        int dev = 0;
        KF_CK(cudaGetDevice(&dev));
        KF_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        KF_CK(cudaMalloc(&d_sess, sizeof(SessionDev) * capacity));
        KF_CK(cudaMemset(d_sess, 0, sizeof(SessionDev) * capacity));
        KF_CK(cudaMalloc(&d_step, sizeof(StepDev) * capacity));
        KF_CK(cudaMemset(d_step, 0, sizeof(StepDev) * capacity));
        static_assert(sizeof(OutDev) % 16 == 0 && sizeof(GridSync) % 16 == 0, "result block layout");
        KF_CK(cudaMalloc(&d_out, out_bytes() + sizeof(unsigned int) * kCounters));
        KF_CK(cudaMemset(d_out, 0, out_bytes() + sizeof(unsigned int) * kCounters));
        d_sync = reinterpret_cast<GridSync*>(d_out + capacity);
        d_ctr = reinterpret_cast<unsigned int*>(d_sync + 1);
        KF_CK(cudaMalloc(&d_tb, sizeof(Tables)));
        KF_CK(cudaMalloc(&d_iranges, sizeof(IcpRange) * KF_MAX_LEVELS * capacity));
        KF_CK(cudaMemset(d_iranges, 0, sizeof(IcpRange) * KF_MAX_LEVELS * capacity));
        KF_CK(cudaMalloc(&d_fprefix, sizeof(long long) * (capacity + 1)));
        KF_CK(cudaMalloc(&d_vfprefix, sizeof(long long) * (capacity + 1)));
        KF_CK(cudaMalloc(&d_icp_sched, sizeof(int4) * capacity));
        KF_CK(cudaMemset(d_icp_sched, 0, sizeof(int4) * capacity));
        KF_CK(cudaMalloc(&d_icp_mats, sizeof(float) * 24 * capacity));
        KF_CK(cudaMemset(d_icp_mats, 0, sizeof(float) * 24 * capacity));
        KF_CK(cudaMallocHost(&h_step, sizeof(StepDev) * capacity));
        KF_CK(cudaMallocHost(&h_out, out_bytes()));
        h_sync = reinterpret_cast<GridSync*>(h_out + capacity);
        std::memset(h_step, 0, sizeof(StepDev) * capacity);
        std::memset(h_out, 0, out_bytes());
        KF_CK(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking));
        KF_CK(cudaStreamCreateWithFlags(&aux_stream, cudaStreamNonBlocking));
        KF_CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        KF_CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        KF_CK(cudaStreamCreateWithFlags(&h2d_stream, cudaStreamNonBlocking));
        KF_CK(cudaEventCreateWithFlags(&ev_input, cudaEventDisableTiming));
        KF_CK(cudaEventCreateWithFlags(&ev_prev, cudaEventDisableTiming));
        // persistent grids (the autotuner may replace them)
        shape.grid_pre = sms * 4;
        shape.grid_ray = sms * 6;
        shape.grid_fuse = sms * 4;
        shape.grid_icp = icp_max_grid(sms);
        return KF_OK;
    }

    // the stream a step's frame copies go on: h2d_stream, after the work already queued on st
    // (earlier steps read the same input buffers; a device frame may come from work on st).  The
    // step's raycast needs only earlier frames and starts at once; its preprocess branch waits
    // for ev_input, and the step ends after that branch, so later work on st (a caller
    // refilling its frame buffer) stays ordered after the copy.
    kf_status begin_inputs(cudaStream_t st, cudaStream_t* cs) {
        KF_CK(cudaEventRecord(ev_prev, st));
        KF_CK(cudaStreamWaitEvent(h2d_stream, ev_prev, 0));
        *cs = h2d_stream;
        return KF_OK;
    }
    kf_status end_inputs(cudaStream_t cs) {
        KF_CK(cudaEventRecord(ev_input, cs));
        return KF_OK;
    }

    kf_status set_profile(bool on) {
        if (on)
            for (cudaEvent_t& e : ev)
                if (!e) KF_CK(cudaEventCreate(&e));
        if (profile != on) graph_dirty = true;
        profile = on;
        return KF_OK;
    }

    // switch to launch shape `to` for the next steps (callers hold the engine, stream idle)
    void set_shape(const Shape& to) {
        if (to == shape) return;
        if (to.ray_tw != shape.ray_tw || to.ray_budget != shape.ray_budget || to.fuse_split != shape.fuse_split ||
            to.ray_form != shape.ray_form)
            tables_dirty = true;
        shape = to;
        graph_dirty = true;
    }

    // durations of the four stages of the last completed step (ms); the preprocess runs beside
    // the raycast, so the raycast's figure spans both branches (from the fork to the join)
    kf_status stage_times(float* ms) {
        if (!profile) return KF_ERR_STATE;
        KF_CK(cudaEventElapsedTime(&ms[0], ev[0], ev[1]));
        KF_CK(cudaEventElapsedTime(&ms[1], ev[0], ev[2]));
        KF_CK(cudaEventElapsedTime(&ms[2], ev[2], ev[3]));
        KF_CK(cudaEventElapsedTime(&ms[3], ev[3], ev[4]));
        return KF_OK;
    }

    void destroy() {
        if (gexec) cudaGraphExecDestroy(gexec);
        gexec = nullptr;
        for (Slot& s : slots) if (!s.external) s.release();
        for (cudaEvent_t& e : ev)
            if (e) cudaEventDestroy(e);
        cudaFree(d_sess); cudaFree(d_step); cudaFree(d_out); cudaFree(d_tb); cudaFree(d_pre); cudaFree(d_ray);
        cudaFree(d_itiles); cudaFree(d_iranges); cudaFree(d_fprefix);
        cudaFree(d_vfprefix); cudaFree(d_vfuseq);
        cudaFree(d_ray_counts);
        cudaFree(d_partials);
        cudaFree(d_icp_sched);
        cudaFree(d_icp_mats);
        cudaFree(d_longq);
        cudaFree(d_fuseq);
        cudaFreeHost(h_step); cudaFreeHost(h_out);
        if (cap_stream) cudaStreamDestroy(cap_stream);
        if (aux_stream) cudaStreamDestroy(aux_stream);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (h2d_stream) cudaStreamDestroy(h2d_stream);
        if (ev_input) cudaEventDestroy(ev_input);
        if (ev_prev) cudaEventDestroy(ev_prev);
    }

    EngineView view() const {
        EngineView v;
        v.sess = d_sess; v.step = d_step; v.out = d_out; v.tb = d_tb; v.pre = d_pre; v.ray = d_ray;
        v.itiles = d_itiles; v.iranges = d_iranges; v.fuse_prefix = d_fprefix;
        v.partials = d_partials;
        v.partials2 = d_partials ? d_partials + cap_part / 2 : nullptr;   // two equal halves
        v.icp_sched = d_icp_sched;
        v.icp_mats = d_icp_mats;
        v.sync = d_sync; v.counters = d_ctr;
        v.longq = reinterpret_cast<LongRay*>(d_longq);
        v.longq_cap = cap_longq / long_ray_bytes();
        v.fuseq = d_fuseq;
        v.fuseq_cap = cap_fuseq;
        v.vis_fuse_prefix = d_vfprefix;
        v.vis_fuseq = d_vfuseq;
        v.vis_fuseq_cap = cap_vfuseq;
        v.ray_counts = count_rays ? d_ray_counts : nullptr;
        return v;
    }

    // Grow the work-list buffers for `count` more sessions like c on top of the current
    // tables, ahead of time (a server's capacity planning): growing them while serving frees
    // and reallocates device memory and re-instantiates the step graph.
    kf_status reserve_work(const kf_config& c, int count) {
        SessionDev d{};
        fill_levels(d, c);
        long long pre = 0, ray = 0, itiles = 0;
        pre = (long long)((c.width + kPreTileSize - 1) / kPreTileSize) * ((c.height + kPreTileSize - 1) / kPreTileSize);
        for (int l = 0; l < c.levels; ++l) {
            const LevelDev& Lv = d.lv[l];
            // tiles of the narrowest shape the tuner tries (4 x 8) bound every shape's count
            ray += (long long)((Lv.cw + 3) / 4) * ((Lv.ch + 7) / 8);
            itiles += (long long)kIcpGroups * kIcpTilesPerBlock + 1;   // at most that many per level
        }
        // reservations add up: every kind reserved so far may be open at once
        const long long k = count;
        res_pre += k * pre;
        res_ray += k * ray;
        res_it += k * itiles;
        res_fq += k * fuse_units(c.volume_n);
        res_vfq += k * (c.vis_volume_n ? fuse_units(c.vis_volume_n) : 0);
        const long long need_pre = tb.n_pre + res_pre, need_ray = tb.n_ray + res_ray;
        long long cur_it = 0;
        for (int l = 0; l < KF_MAX_LEVELS; ++l) cur_it += tb.n_itiles[l];
        const long long need_it = cur_it + res_it;
        const long long need_fq = tb.fuse_total + res_fq;
        const long long need_vfq = tb.vis_fuse_total + res_vfq;
        if (need_pre > INT32_MAX || long_ray_entries(need_ray * 32) > INT32_MAX / long_ray_bytes() ||
            need_it * kIcpPartialStride > INT32_MAX || need_fq > (1 << 29) || need_vfq > (1 << 29))
            return KF_ERR_CAPACITY;
        const int old_pre = cap_pre, old_ray = cap_ray, old_it = cap_it, old_part = cap_part, old_lq = cap_longq,
                  old_fq = cap_fuseq;
        KF_TRY(grow(d_pre, cap_pre, int(need_pre)));
        KF_TRY(grow(d_ray, cap_ray, int(need_ray)));
        KF_TRY(grow(d_itiles, cap_it, int(need_it)));
        KF_TRY(grow(d_partials, cap_part, 2 * int(need_it) * kIcpPartialStride));
        KF_TRY(grow(d_longq, cap_longq, int(long_ray_entries(need_ray * 32)) * long_ray_bytes()));
        KF_TRY(grow(d_fuseq, cap_fuseq, int(need_fq)));
        const int old_vfq = cap_vfuseq;
        if (need_vfq > 0) KF_TRY(grow(d_vfuseq, cap_vfuseq, int(need_vfq)));
        if (old_pre != cap_pre || old_ray != cap_ray || old_it != cap_it || old_part != cap_part || old_lq != cap_longq ||
            old_fq != cap_fuseq || old_vfq != cap_vfuseq) {
            graph_dirty = true;
            tables_dirty = true;
        }
        return KF_OK;
    }

    // rebuild and upload work lists (synchronous; callers hold the engine)
    kf_status build_tables() {
        std::vector<PreTile> pre;
        std::vector<RayTile> ray;
        std::vector<IcpTile> it[KF_MAX_LEVELS];
        std::vector<IcpRange> ranges(size_t(KF_MAX_LEVELS) * cap, IcpRange{0, 0});
        std::vector<long long> fprefix(cap + 1, 0), vfprefix(cap + 1, 0);
        std::vector<SessionDev> sess(cap);
        int max_levels = 1;
        for (int s = 0; s < cap; ++s) {
            const Slot& sl = slots[s];
            fprefix[s + 1] = fprefix[s];
            vfprefix[s + 1] = vfprefix[s];
            if (!sl.used) { std::memset(&sess[s], 0, sizeof(SessionDev)); continue; }
            sess[s] = sl.d;
            const kf_config& c = sl.cfg;
            max_levels = std::max(max_levels, c.levels);
            if (!sl.external) {
                for (int y = 0; y < c.height; y += kPreTileSize)
                    for (int x = 0; x < c.width; x += kPreTileSize) pre.push_back(PreTile{s, x, y});
                for (int l = 0; l < c.levels; ++l) {
                    const LevelDev& Lv = sl.d.lv[l];
                    const int tw = shape.ray_tw, th = 32 / shape.ray_tw;
                    for (int y = 0; y < Lv.ch; y += th)
                        for (int x = 0; x < Lv.cw; x += tw) ray.push_back(RayTile{s, l, x, y});
                }
                fprefix[s + 1] += fuse_units(c.volume_n);
                if (sl.d.vis.n) vfprefix[s + 1] += fuse_units(sl.d.vis.n);
            }
            for (int l = 0; l < c.levels; ++l) {
                const LevelDev& Lv = sl.d.lv[l];
                const int np = Lv.icw * Lv.ich;
                // up to a few tiles per ICP block per session-level (the grid's blocks take them
                // round robin, which evens out tiles of mostly invalid pixels), each at least
                // one pipelined step of the block (kIcpMinTile pixels): small levels get few
                // tiles, so a pass over many sessions stores few partials
                const int per_block = std::max(1, std::min(kIcpTilesPerBlock, np / (kIcpGroups * kIcpMinTile)));
                const int ntiles = kIcpGroups * per_block;
                int tile = (np + ntiles - 1) / ntiles;
                tile = std::max(kIcpMinTile, (tile + 31) / 32 * 32);
                IcpRange rg;
                rg.begin = int(it[l].size());
                for (int p0 = 0; p0 < np; p0 += tile) it[l].push_back(IcpTile{s, p0, std::min(tile, np - p0)});
                rg.end = int(it[l].size());
                ranges[size_t(l) * cap + s] = rg;
            }
        }
        // concatenate ICP levels; ranges become absolute
        std::vector<IcpTile> all;
        int off[KF_MAX_LEVELS];
        for (int l = 0; l < KF_MAX_LEVELS; ++l) {
            off[l] = int(all.size());
            all.insert(all.end(), it[l].begin(), it[l].end());
            for (int s = 0; s < cap; ++s) {
                IcpRange& rg = ranges[size_t(l) * cap + s];
                rg.begin += off[l];
                rg.end += off[l];
            }
        }
        const int old_pre = cap_pre, old_ray = cap_ray, old_it = cap_it, old_part = cap_part, old_lq = cap_longq,
                  old_fq = cap_fuseq;
        // fusion queue entries are 32-bit and each is taken in 4 parts counted in 32 bits
        if (fprefix[cap] > (long long)(1 << 29) || vfprefix[cap] > (long long)(1 << 29)) return KF_ERR_CAPACITY;
        KF_TRY(grow(d_fuseq, cap_fuseq, std::max<int>(1, int(fprefix[cap]))));
        const int old_vfq = cap_vfuseq;
        KF_TRY(grow(d_vfuseq, cap_vfuseq, std::max<int>(1, int(vfprefix[cap]))));
        if (old_vfq != cap_vfuseq) graph_dirty = true;
        const bool vis = vfprefix[cap] > 0;
        if (vis != has_vis) graph_dirty = true;   // the step launches the visualization fusion or not
        has_vis = vis;
        KF_TRY(grow(d_pre, cap_pre, std::max<int>(1, int(pre.size()))));
        KF_TRY(grow(d_ray, cap_ray, std::max<int>(1, int(ray.size()))));
        KF_TRY(grow(d_itiles, cap_it, std::max<int>(1, int(all.size()))));
        KF_TRY(grow(d_partials, cap_part, 2 * std::max<int>(1, int(all.size())) * kIcpPartialStride));
        if (long_ray_entries((long long)ray.size() * 32) > INT32_MAX / long_ray_bytes()) return KF_ERR_CAPACITY;
        KF_TRY(grow(d_longq, cap_longq, int(long_ray_entries((long long)ray.size() * 32)) * long_ray_bytes()));
        if (old_pre != cap_pre || old_ray != cap_ray || old_it != cap_it || old_part != cap_part || old_lq != cap_longq ||
            old_fq != cap_fuseq)
            graph_dirty = true;
        if (!pre.empty()) KF_CK(cudaMemcpy(d_pre, pre.data(), sizeof(PreTile) * pre.size(), cudaMemcpyHostToDevice));
        if (!ray.empty()) KF_CK(cudaMemcpy(d_ray, ray.data(), sizeof(RayTile) * ray.size(), cudaMemcpyHostToDevice));
        if (!all.empty()) KF_CK(cudaMemcpy(d_itiles, all.data(), sizeof(IcpTile) * all.size(), cudaMemcpyHostToDevice));
        KF_CK(cudaMemcpy(d_iranges, ranges.data(), sizeof(IcpRange) * ranges.size(), cudaMemcpyHostToDevice));
        KF_CK(cudaMemcpy(d_fprefix, fprefix.data(), sizeof(long long) * fprefix.size(), cudaMemcpyHostToDevice));
        KF_CK(cudaMemcpy(d_vfprefix, vfprefix.data(), sizeof(long long) * vfprefix.size(), cudaMemcpyHostToDevice));
        KF_CK(cudaMemcpy(d_sess, sess.data(), sizeof(SessionDev) * cap, cudaMemcpyHostToDevice));
        tb.S = cap;
        tb.n_pre = int(pre.size());
        tb.n_ray = int(ray.size());
        tb.ray_budget = shape.ray_budget ? shape.ray_budget : serial_budget(tb.n_ray);
        tb.ray_tw = shape.ray_tw;
        tb.fuse_split = shape.fuse_split;
        const bool many = shape.ray_form ? shape.ray_form == 4 : many_ray_tiles(tb.n_ray);
        if (ray_many != many) graph_dirty = true;
        ray_many = many;
        for (int l = 0; l < KF_MAX_LEVELS; ++l) {
            tb.n_itiles[l] = int(it[l].size());
            tb.icp_off[l] = off[l];
        }
        tb.max_levels = max_levels;
        tb.fuse_total = fprefix[cap];
        tb.vis_fuse_total = vfprefix[cap];
        KF_CK(cudaMemcpy(d_tb, &tb, sizeof(Tables), cudaMemcpyHostToDevice));
        tables_dirty = false;
        return KF_OK;
    }

    // the per-step sequence
    kf_status record(cudaStream_t st) {
        const EngineView v = view();
        KF_CK(cudaMemsetAsync(d_sync, 0, sizeof(GridSync) + sizeof(unsigned int) * kCounters, st));
        if (count_rays) KF_CK(cudaMemsetAsync(d_ray_counts, 0, sizeof(unsigned long long) * ray_count_slots(), st));
        if (profile) KF_CK(cudaEventRecordWithFlags(ev[0], st, cudaEventRecordExternal));
        const bool fork = stages[0] && stages[1];
        if (fork) {
            // preprocess on a branch beside the raycast; ICP waits for both
            KF_CK(cudaEventRecord(ev_fork, st));
            KF_CK(cudaStreamWaitEvent(aux_stream, ev_fork, 0));
            if (input_wait) KF_CK(cudaStreamWaitEvent(aux_stream, ev_input, capturing ? cudaEventWaitExternal : 0));
            NvtxRange r("kf.preprocess");
            KF_CK(launch_preprocess(v, shape.grid_pre, aux_stream));
            if (profile) KF_CK(cudaEventRecordWithFlags(ev[1], aux_stream, cudaEventRecordExternal));
            KF_CK(cudaEventRecord(ev_join, aux_stream));
        } else {
            if (stages[0] && input_wait) KF_CK(cudaStreamWaitEvent(st, ev_input, capturing ? cudaEventWaitExternal : 0));
            NvtxRange r("kf.preprocess");
            if (stages[0]) KF_CK(launch_preprocess(v, shape.grid_pre, st));
            if (profile) KF_CK(cudaEventRecordWithFlags(ev[1], st, cudaEventRecordExternal));
        }
        {
            NvtxRange r("kf.raycast");
            if (stages[1]) KF_CK(launch_raycast(v, shape.grid_ray, st, ray_many));
        }
        if (fork) KF_CK(cudaStreamWaitEvent(st, ev_join, 0));
        if (profile) KF_CK(cudaEventRecordWithFlags(ev[2], st, cudaEventRecordExternal));
        {
            NvtxRange r("kf.icp");
            if (stages[2]) KF_CK(launch_icp(v, shape.grid_icp, st, cap == 1));
        }
        if (profile) KF_CK(cudaEventRecordWithFlags(ev[3], st, cudaEventRecordExternal));
        {
            NvtxRange r("kf.fusion");
            if (stages[3]) KF_CK(launch_fuse(v, shape.grid_fuse, st));
        }
        if (has_vis && stages[3]) {
            // the visualization volumes (the reference's second grid), after the tracking fusion
            // and in the same stage time
            NvtxRange r("kf.fusion_vis");
            KF_CK(launch_fuse_vis(v, shape.grid_fuse, st));
        }
        if (profile) KF_CK(cudaEventRecordWithFlags(ev[4], st, cudaEventRecordExternal));
        return KF_OK;
    }

    // the step's results (every slot's OutDev and the wait record) into pinned memory, for
    // collect() once the stream is idle; steps whose results stay on the device skip it
    kf_status fetch(cudaStream_t st) {
        KF_CK(cudaMemcpyAsync(h_out, d_out, out_bytes(), cudaMemcpyDeviceToHost, st));
        return KF_OK;
    }

    kf_status capture() {
        if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
        cudaGraph_t g = nullptr;
        KF_CK(cudaStreamBeginCapture(cap_stream, cudaStreamCaptureModeThreadLocal));
        capturing = true;
        kf_status rs = record(cap_stream);
        capturing = false;
        cudaError_t e = cudaStreamEndCapture(cap_stream, &g);
        if (rs != KF_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            use_graph = false;   // e.g. a cooperative launch that cannot be captured
            return KF_OK;
        }
        e = cudaGraphInstantiate(&gexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            cudaGetLastError();
            gexec = nullptr;
            use_graph = false;
            return KF_OK;
        }
        graph_dirty = false;
        return KF_OK;
    }

    kf_status enqueue(cudaStream_t st) {
        if (tables_dirty) {
            KF_CK(cudaStreamSynchronize(st));
            KF_TRY(build_tables());
        }
        if (step_dirty) {
            KF_CK(cudaMemcpyAsync(d_step, h_step, sizeof(StepDev) * cap, cudaMemcpyHostToDevice, st));
            step_dirty = false;
        }
        if (use_graph) {
            if (graph_dirty || !gexec) KF_TRY(capture());
            if (use_graph) {
                KF_CK(cudaGraphLaunch(gexec, st));
                return KF_OK;
            }
        }
        return record(st);
    }

    // set h_step; waits for in-flight work before touching pinned memory the stream may read
    kf_status set_step(const std::vector<StepDev>& want, cudaStream_t st) {
        bool same = true;
        for (int s = 0; s < cap; ++s)
            if (h_step[s].active != want[s].active || h_step[s].first != want[s].first) same = false;
        if (same && !step_dirty) return KF_OK;
        KF_CK(cudaStreamSynchronize(st));
        for (int s = 0; s < cap; ++s) h_step[s] = want[s];
        step_dirty = true;
        return KF_OK;
    }

    // after the stream finished: pull per-session results
    kf_status collect(const std::vector<StepDev>& want) {
        kf_status worst = KF_OK;
        const bool timed_out = h_sync->abort != 0;
        for (int s = 0; s < cap; ++s) {
            if (!want[s].active) continue;
            Slot& sl = slots[s];
            const OutDev& o = h_out[s];
            std::memcpy(sl.pose, o.pose, sizeof(sl.pose));
            sl.stats.frame = sl.frames;
            sl.stats.status = timed_out ? KF_ERR_TIMEOUT : o.status;
            for (int l = 0; l < KF_MAX_LEVELS; ++l) sl.stats.icp_iters[l] = o.iters[l];
            sl.frames += 1;
            if (sl.stats.status != KF_OK && worst == KF_OK) worst = kf_status(sl.stats.status);
        }
        return worst;
    }
};

// the batch autotuner's step hooks (defined with the batch API below)
kf_status tuner_before_step(Engine& e);
kf_status tuner_after_step(Engine& e);

kf_status record_ms(cudaStream_t st, cudaEvent_t a, cudaEvent_t b, float* ms) {
    KF_CK(cudaEventRecord(b, st));
    KF_CK(cudaEventSynchronize(b));
    KF_CK(cudaEventElapsedTime(ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return KF_OK;
}

// event pair around a stage call when the caller asks for its time (the reference's
// kernel:: wrappers all return elapsed milliseconds)
struct StageTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    float* ms;
    cudaStream_t st;
    StageTimer(float* m, cudaStream_t s) : ms(m), st(s) {
        if (ms) {
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, st);
        }
    }
    kf_status finish(cudaError_t launch) {
        if (launch != cudaSuccess) {
            g_last_cuda = launch;
            if (ms) { cudaEventDestroy(a); cudaEventDestroy(b); }
            return KF_ERR_CUDA;
        }
        if (!ms) return KF_OK;
        return record_ms(st, a, b, ms);
    }
};

}  // namespace

// ------------------------------------------------------------------------------------------
// shared host math
// ------------------------------------------------------------------------------------------
namespace kf {

void voxel_axes(int n, float width, float* xs, float* zs) {
    // project/src/tsdf.cu:27-31: x = -w/2 + i * res; z accumulated "+= resolution" in float
    const float res = width / float(n - 1);
    const float base = -width * 0.5f;
    for (int i = 0; i < n; ++i) xs[i] = base + float(i) * res;
    float z = base + (-res);
    for (int k = 0; k < n; ++k) {
        z = z + res;
        zs[k] = z;
    }
}

void level_intrinsics(const kf_config& c, int level, float k[9], float ik[9]) {
    // Sensor (project/src/sensor.h:14-19): f / 2^l, principal point (c + 0.5) / 2^l - 0.5
    const float s = 1.0f / float(1 << level);
    const float fx = c.fx * s, fy = c.fy * s;
    const float cx = (c.cx + 0.5f) * s - 0.5f, cy = (c.cy + 0.5f) * s - 0.5f;
    const float m[9] = {fx, 0.f, 0.f, 0.f, fy, 0.f, cx, cy, 1.f};
    std::memcpy(k, m, sizeof(m));
    // adjugate / determinant (glm::inverse of the 3x3)
    const float a = m[0], b = m[3], cc = m[6], d = m[1], e = m[4], f = m[7], g = m[2], h = m[5], i = m[8];
    const float det = a * (e * i - f * h) - b * (d * i - f * g) + cc * (d * h - e * g);
    const float od = 1.0f / det;
    ik[0] = (e * i - f * h) * od;  ik[3] = -(b * i - cc * h) * od; ik[6] = (b * f - cc * e) * od;
    ik[1] = -(d * i - f * g) * od; ik[4] = (a * i - cc * g) * od;  ik[7] = -(a * f - cc * d) * od;
    ik[2] = (d * h - e * g) * od;  ik[5] = -(a * h - b * g) * od;  ik[8] = (a * e - b * d) * od;
}

}  // namespace kf

// ------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------
// a session is a slot of an engine: its own (kf_session_create) or a batch's / server's
// frames of one session queued by kf_process_frame_submit and not yet collected by
// kf_process_frame_wait: each has its own pinned copy of the step's result and an event
struct FrameRing {
    static constexpr int kDepth = KF_MAX_FRAMES_IN_FLIGHT;
    // a frame's result block and the step's wait record, laid out as on the device when the
    // session is its engine's last slot (one copy)
    struct Entry { OutDev out; GridSync sync; };
    Entry* res = nullptr;                  // kDepth pinned entries
    cudaEvent_t done[kDepth] = {};
    int head = 0, count = 0;               // oldest in-flight entry, entries in flight
    kf_status init() {
        KF_CK(cudaMallocHost(&res, sizeof(Entry) * kDepth));
        for (cudaEvent_t& e : done) KF_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        return KF_OK;
    }
    void destroy() {
        if (res) cudaFreeHost(res);
        res = nullptr;
        for (cudaEvent_t& e : done)
            if (e) cudaEventDestroy(e);
    }
};

struct kf_session {
    Engine* eng = nullptr;
    int slot = 0;
    bool owns = false;
    FrameRing* ring = nullptr;   // created by the first kf_process_frame_submit
    Slot& sl() { return eng->slots[slot]; }
};

struct kf_batch {
    Engine eng;
    int n = 0;
    std::vector<kf_session*> views;
};

extern "C" {

int kf_api_version(void) { return KF_API_VERSION; }

const char* kf_status_string(int s) {
    switch (s) {
        case KF_OK: return "ok";
        case KF_ERR_ARG: return "invalid argument";
        case KF_ERR_SHAPE: return "map sizes do not match";
        case KF_ERR_CUDA: return cudaGetErrorString(g_last_cuda);
        case KF_ERR_NONFINITE: return "ICP solution not finite";
        case KF_ERR_OOM_BUDGET: return "session does not fit the HBM budget";
        case KF_ERR_TIMEOUT: return "device wait timed out";
        case KF_ERR_STATE: return "call not valid in this state";
        case KF_ERR_CAPACITY: return "no free slot";
        case KF_ERR_TOO_LARGE: return "problem larger than the fixed scratch of a no-allocation entry point";
        default: return "unknown status";
    }
}

void kf_config_default(kf_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    const float pi = 3.14159265358979323846f;
    // project/src/main.cpp:11-59 (dataset configuration)
    c->width = 640;
    c->height = 480;
    c->fx = c->fy = 525.0f;
    c->cx = 319.5f;                 // project/src/sensor.h:14
    c->cy = 239.5f;
    c->depth_scale = 1.0f / 5000.0f;
    c->unmirror = 0;
    c->levels = 3;
    c->iters[0] = 10; c->iters[1] = 5; c->iters[2] = 3;
    c->dist_thresh = 0.4f;
    c->angle_thresh = 4.0f * pi / 18.0f;
    c->stop_angle = 0.1f * pi / 180.0f;    // glm::radians(0.1f)
    c->stop_dist = 0.01f;
    c->bilateral_sigma_s = 4.0f;    // project/src/measurement.cu:11-12, :38
    c->bilateral_sigma_r = 0.25f;
    c->bilateral_radius = 3;
    c->volume_n = 256;              // fusion volume: 8 m, 256^3, mu = 3 voxels
    c->volume_width = 8.0f;
    c->mu = 3.0f * (8.0f / 255.0f);
    c->max_weight = 0.0f;
    c->tsdf_format = KF_TSDF_F32F32;
    c->min_depth = 0.4f;            // project/src/tsdf.cuh:11-12
    c->max_depth = 6.0f;
    c->step_large = 1.99f;          // project/src/raycast.cu:75-76
    c->step_small = 0.1f;
    c->compat_trunc8 = 0;
    c->keep_on_miss = 1;
    c->export_icp_mask = 0;
    for (int i = 0; i < 16; ++i) c->initial_pose[i] = (i % 5 == 0) ? 1.0f : 0.0f;
    // visualization grid: 512^3 over 5 m, mu = 2 voxels (project/src/main.cpp:25-26,
    // project/src/kinect_fusion.cpp:19)
    c->vis_volume_n = 512;
    c->vis_volume_width = 5.0f;
    c->vis_mu = 2.0f * (5.0f / 511.0f);
}

kf_status kf_session_footprint(const kf_config* cfg, size_t* bytes) {
    if (!cfg || !bytes) return KF_ERR_ARG;
    KF_TRY(validate(*cfg));
    *bytes = footprint(*cfg);
    return KF_OK;
}

kf_status kf_session_create(const kf_config* cfg, kf_session** out) {
    NvtxRange nvtx_("kf_session_create");
    if (!cfg || !out) return KF_ERR_ARG;
    KF_TRY(validate(*cfg));
    kf_session* s = new (std::nothrow) kf_session;
    if (!s) return KF_ERR_ARG;
    s->eng = new (std::nothrow) Engine;
    if (!s->eng) { delete s; return KF_ERR_ARG; }
    s->owns = true;
    kf_status st = s->eng->init(1);
    if (st == KF_OK) st = slot_create(s->eng->slots[0], *cfg);
    if (st != KF_OK) { s->eng->destroy(); delete s->eng; delete s; return st; }
    s->eng->tables_dirty = true;
    *out = s;
    return KF_OK;
}

kf_status kf_session_destroy(kf_session* s) {
    if (!s) return KF_ERR_ARG;
    if (!s->owns) return KF_ERR_STATE;   // batch / server members go with their owner
    cudaDeviceSynchronize();
    if (s->ring) {
        s->ring->destroy();
        delete s->ring;
    }
    s->eng->destroy();
    delete s->eng;
    delete s;
    return KF_OK;
}

kf_status kf_session_reset(kf_session* s) {
    if (!s) return KF_ERR_ARG;
    KF_CK(cudaDeviceSynchronize());
    if (s->ring) s->ring->head = s->ring->count = 0;   // results of submitted frames are dropped
    return slot_reset(s->sl());
}

static kf_status session_enqueue(kf_session* s, const uint16_t* depth, int is_dev, cudaStream_t st) {
    Slot& sl = s->sl();
    const size_t bytes = size_t(sl.cfg.width) * sl.cfg.height * 2;
    std::vector<StepDev> want(s->eng->cap, StepDev{0, 0});
    want[s->slot] = StepDev{1, sl.frames == 0 ? 1 : 0};
    KF_TRY(s->eng->set_step(want, st));
    Engine& e = *s->eng;
    cudaStream_t cs = st;
    KF_TRY(e.begin_inputs(st, &cs));
    KF_CK(cudaMemcpyAsync(const_cast<uint16_t*>(sl.d.raw), depth, bytes,
                          is_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, cs));
    KF_TRY(e.end_inputs(cs));
    return e.enqueue(st);
}

kf_status kf_process_frame(kf_session* s, const uint16_t* depth, int is_device_ptr, void* stream, float pose_out[16]) {
    NvtxRange nvtx_("kf_process_frame");
    if (!s || !depth) return KF_ERR_ARG;
    if (s->ring && s->ring->count) return KF_ERR_STATE;   // collect submitted frames first
    cudaStream_t st = as_stream(stream);
    KF_TRY(session_enqueue(s, depth, is_device_ptr, st));
    KF_TRY(s->eng->fetch(st));
    KF_CK(cudaStreamSynchronize(st));
    std::vector<StepDev> want(s->eng->cap, StepDev{0, 0});
    want[s->slot] = StepDev{1, 0};
    kf_status r = s->eng->collect(want);
    if (pose_out) std::memcpy(pose_out, s->sl().pose, sizeof(float) * 16);
    return r;
}

kf_status kf_process_frame_submit(kf_session* s, const uint16_t* depth, int is_device_ptr, void* stream) {
    NvtxRange nvtx_("kf_process_frame_submit");
    if (!s || !depth) return KF_ERR_ARG;
    if (!s->owns) return KF_ERR_STATE;   // a batch's or server's session steps with its owner
    if (!s->ring) {
        FrameRing* r = new (std::nothrow) FrameRing;
        if (!r) return KF_ERR_ARG;
        const kf_status st = r->init();
        if (st != KF_OK) { r->destroy(); delete r; return st; }
        s->ring = r;
    }
    FrameRing& r = *s->ring;
    if (r.count == FrameRing::kDepth) return KF_ERR_CAPACITY;
    cudaStream_t st = as_stream(stream);
    const int frame_no = s->sl().frames;
    KF_TRY(session_enqueue(s, depth, is_device_ptr, st));
    // this frame's result, read back before a later frame's step overwrites it on the device
    const int k = (r.head + r.count) % FrameRing::kDepth;
    static_assert(sizeof(FrameRing::Entry) == sizeof(OutDev) + sizeof(GridSync), "ring entry layout");
    if (s->slot == s->eng->cap - 1) {
        KF_CK(cudaMemcpyAsync(&r.res[k], s->eng->d_out + s->slot, sizeof(FrameRing::Entry), cudaMemcpyDeviceToHost, st));
    } else {
        KF_CK(cudaMemcpyAsync(&r.res[k].out, s->eng->d_out + s->slot, sizeof(OutDev), cudaMemcpyDeviceToHost, st));
        KF_CK(cudaMemcpyAsync(&r.res[k].sync, s->eng->d_sync, sizeof(GridSync), cudaMemcpyDeviceToHost, st));
    }
    KF_CK(cudaEventRecord(r.done[k], st));
    r.count += 1;
    s->sl().frames = frame_no + 1;
    return KF_OK;
}

kf_status kf_process_frame_wait(kf_session* s, float pose_out[16], kf_frame_stats* stats_out) {
    NvtxRange nvtx_("kf_process_frame_wait");
    if (!s) return KF_ERR_ARG;
    if (!s->ring || s->ring->count == 0) return KF_ERR_STATE;
    FrameRing& r = *s->ring;
    const int k = r.head;
    KF_CK(cudaEventSynchronize(r.done[k]));
    const OutDev& o = r.res[k].out;
    Slot& sl = s->sl();
    kf_frame_stats fs{};
    fs.frame = o.frame - 1;
    fs.status = r.res[k].sync.abort != 0 ? KF_ERR_TIMEOUT : o.status;
    for (int l = 0; l < KF_MAX_LEVELS; ++l) fs.icp_iters[l] = o.iters[l];
    r.head = (r.head + 1) % FrameRing::kDepth;
    r.count -= 1;
    sl.stats = fs;
    std::memcpy(sl.pose, o.pose, sizeof(sl.pose));
    if (pose_out) std::memcpy(pose_out, o.pose, sizeof(float) * 16);
    if (stats_out) *stats_out = fs;
    return kf_status(fs.status);
}

kf_status kf_process_frame_async(kf_session* s, const uint16_t* depth_device, void* stream) {
    NvtxRange nvtx_("kf_process_frame_async");
    if (!s || !depth_device) return KF_ERR_ARG;
    cudaStream_t st = as_stream(stream);
    KF_TRY(session_enqueue(s, depth_device, 1, st));
    // results stay on the device; the frame counter advances here
    s->sl().frames += 1;
    return KF_OK;
}

kf_status kf_get_pose(kf_session* s, float pose[16]) {
    if (!s || !pose) return KF_ERR_ARG;
    // read the device state (also valid after async frames once the stream is idle)
    PoseDev P;
    KF_CK(cudaMemcpy(&P, s->sl().d.pose, sizeof(P), cudaMemcpyDeviceToHost));
    for (int i = 0; i < 16; ++i) pose[i] = 0.f;
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) pose[c * 4 + r] = float(P.Rp[c * 3 + r]);
    for (int r = 0; r < 3; ++r) pose[12 + r] = float(P.tp[r]);
    pose[15] = 1.f;
    return KF_OK;
}

kf_status kf_set_pose(kf_session* s, const float pose[16]) {
    if (!s || !pose) return KF_ERR_ARG;
    KF_CK(cudaDeviceSynchronize());
    PoseDev old;
    KF_CK(cudaMemcpy(&old, s->sl().d.pose, sizeof(old), cudaMemcpyDeviceToHost));
    PoseDev P = make_pose_dev(pose);
    P.frame = old.frame;
    KF_CK(cudaMemcpy(s->sl().d.pose, &P, sizeof(P), cudaMemcpyHostToDevice));
    std::memcpy(s->sl().pose, pose, sizeof(float) * 16);
    return KF_OK;
}

kf_status kf_get_frame_stats(kf_session* s, kf_frame_stats* out) {
    if (!s || !out) return KF_ERR_ARG;
    *out = s->sl().stats;
    return KF_OK;
}

static kf_status copy_out(void* dst, const void* src, size_t bytes, int to_host) {
    KF_CK(cudaDeviceSynchronize());
    KF_CK(cudaMemcpy(dst, src, bytes, to_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice));
    return KF_OK;
}

kf_status kf_get_depth(kf_session* s, int level, float* dst, int to_host) {
    if (!s || !dst) return KF_ERR_ARG;
    const Slot& sl = s->sl();
    if (level == -1) return copy_out(dst, sl.d.depth_m, size_t(sl.cfg.width) * sl.cfg.height * 4, to_host);
    if (level < 0 || level >= sl.cfg.levels) return KF_ERR_ARG;
    return copy_out(dst, sl.d.depth[level], level_px(sl.cfg, level) * 4, to_host);
}

kf_status kf_get_vertex(kf_session* s, int level, float* dst, int to_host) {
    if (!s || !dst) return KF_ERR_ARG;
    const Slot& sl = s->sl();
    if (level < 0 || level >= sl.cfg.levels) return KF_ERR_ARG;
    return copy_out(dst, sl.d.vmap[level], level_px(sl.cfg, level) * 16, to_host);
}

kf_status kf_get_raycast(kf_session* s, int level, float* vertex, float* normal, int to_host) {
    if (!s) return KF_ERR_ARG;
    const Slot& sl = s->sl();
    if (level < 0 || level >= sl.cfg.levels) return KF_ERR_ARG;
    if (vertex) KF_TRY(copy_out(vertex, sl.d.pv[level], level_px(sl.cfg, level) * 16, to_host));
    if (normal) KF_TRY(copy_out(normal, sl.d.pn[level], level_px(sl.cfg, level) * 16, to_host));
    return KF_OK;
}

kf_status kf_get_icp_mask(kf_session* s, int level, uint8_t* dst, int to_host) {
    if (!s || !dst) return KF_ERR_ARG;
    const Slot& sl = s->sl();
    if (level < 0 || level >= sl.cfg.levels || !sl.d.mask[level]) return KF_ERR_STATE;
    return copy_out(dst, sl.d.mask[level], level_px(sl.cfg, level), to_host);
}

// a grid (distance and weight arrays of n^3) to dst in layout 0 (native) or 1 (.bin float2)
static kf_status copy_grid_out(const void* tf, const void* tw, int n, int fmt, void* dst, size_t dst_bytes, int layout,
                               int to_host) {
    const size_t n3 = size_t(n) * n * n;
    const size_t es = fmt == KF_TSDF_F16U16 ? 2 : 4;
    KF_CK(cudaDeviceSynchronize());
    const cudaMemcpyKind kind = to_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (layout == 0) {
        if (dst_bytes < 2 * n3 * es) return KF_ERR_SHAPE;
        KF_CK(cudaMemcpy(dst, tf, n3 * es, kind));
        KF_CK(cudaMemcpy(static_cast<char*>(dst) + n3 * es, tw, n3 * es, kind));
        return KF_OK;
    }
    if (layout != 1) return KF_ERR_ARG;
    if (dst_bytes < n3 * 8) return KF_ERR_SHAPE;
    float* tmp = nullptr;
    if (to_host) KF_CK(cudaMalloc(&tmp, n3 * 8));
    float* target = to_host ? tmp : static_cast<float*>(dst);
    cudaError_t e = launch_export_interleaved(tf, tw, (long long)n3, fmt, target, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess && to_host) e = cudaMemcpy(dst, tmp, n3 * 8, cudaMemcpyDeviceToHost);
    if (tmp) cudaFree(tmp);
    KF_CK(e);
    return KF_OK;
}

kf_status kf_get_vis_tsdf(kf_session* s, void* dst, size_t dst_bytes, int layout, int to_host) {
    if (!s || !dst) return KF_ERR_ARG;
    const Slot& sl = s->sl();
    if (!sl.d.vis.n) return KF_ERR_STATE;
    return copy_grid_out(sl.d.vis.tf, sl.d.vis.tw, sl.d.vis.n, sl.d.fmt, dst, dst_bytes, layout, to_host);
}

kf_status kf_get_tsdf(kf_session* s, void* dst, size_t dst_bytes, int layout, int to_host) {
    if (!s || !dst) return KF_ERR_ARG;
    const Slot& sl = s->sl();
    return copy_grid_out(sl.d.tf, sl.d.tw, sl.cfg.volume_n, sl.d.fmt, dst, dst_bytes, layout, to_host);
}

// a grid (distance and weight arrays of n^3, with its brick bounds) from src in layout 0
// (native) or 1 (.bin float2)
static kf_status copy_grid_in(void* tf, void* tw, int n, int fmt, int* bmin, int* bdil, int* sdil, const void* src,
                              size_t src_bytes, int layout, int from_host) {
    const size_t n3 = size_t(n) * n * n;
    const size_t es = fmt == KF_TSDF_F16U16 ? 2 : 4;
    KF_CK(cudaDeviceSynchronize());
    const cudaMemcpyKind kind = from_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    if (layout == 0) {
        if (src_bytes < 2 * n3 * es) return KF_ERR_SHAPE;
        KF_CK(cudaMemcpy(tf, src, n3 * es, kind));
        KF_CK(cudaMemcpy(tw, static_cast<const char*>(src) + n3 * es, n3 * es, kind));
    } else {
        if (layout != 1) return KF_ERR_ARG;
        if (src_bytes < n3 * 8) return KF_ERR_SHAPE;
        float* tmp = nullptr;
        const float* from = static_cast<const float*>(src);
        if (from_host) {
            KF_CK(cudaMalloc(&tmp, n3 * 8));
            KF_CK(cudaMemcpy(tmp, src, n3 * 8, cudaMemcpyHostToDevice));
            from = tmp;
        }
        cudaError_t e = launch_import_interleaved(from, tf, tw, (long long)n3, fmt, 0);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (tmp) cudaFree(tmp);
        KF_CK(e);
    }
    // the raycaster's brick minima follow the new volume
    KF_CK(launch_rebuild_bricks(tf, fmt, n, bmin, bdil, sdil, 0));
    KF_CK(cudaDeviceSynchronize());
    return KF_OK;
}

kf_status kf_set_tsdf(kf_session* s, const void* src, size_t src_bytes, int layout, int from_host) {
    if (!s || !src) return KF_ERR_ARG;
    Slot& sl = s->sl();
    return copy_grid_in(sl.d.tf, sl.d.tw, sl.cfg.volume_n, sl.d.fmt, sl.d.bmin, sl.d.bdil, sl.d.sdil, src, src_bytes,
                        layout, from_host);
}

// ---- files: the reference's .bin TSDF layout, and checkpoints (TSDF + pose + frame index) ----

// n^3 interleaved float {f, w} (VoxelGrid::saveVoxelGrid, project/src/voxel_grid.cpp:43-62)
static kf_status save_grid_file(const void* tf, const void* tw, int n, int fmt, const char* path) {
    const size_t n3 = size_t(n) * n * n;
    std::vector<float> host(n3 * 2);
    KF_TRY(copy_grid_out(tf, tw, n, fmt, host.data(), n3 * 8, 1, 1));
    FILE* f = std::fopen(path, "wb");
    if (!f) return KF_ERR_ARG;
    const size_t wrote = std::fwrite(host.data(), 1, n3 * 8, f);
    const int closed = std::fclose(f);
    return wrote == n3 * 8 && closed == 0 ? KF_OK : KF_ERR_ARG;
}

// VoxelGrid::loadVoxelGrid (project/src/voxel_grid.cpp:64-80); a file of another size is
// KF_ERR_SHAPE
static kf_status load_grid_file(void* tf, void* tw, int n, int fmt, int* bmin, int* bdil, int* sdil, const char* path) {
    const size_t n3 = size_t(n) * n * n;
    FILE* f = std::fopen(path, "rb");
    if (!f) return KF_ERR_ARG;
    std::vector<float> host(n3 * 2);
    const size_t got = std::fread(host.data(), 1, n3 * 8, f);
    const bool extra = std::fgetc(f) != EOF;
    std::fclose(f);
    if (got != n3 * 8 || extra) return KF_ERR_SHAPE;
    return copy_grid_in(tf, tw, n, fmt, bmin, bdil, sdil, host.data(), n3 * 8, 1, 1);
}

kf_status kf_save_tsdf_file(kf_session* s, const char* path) {
    if (!s || !path) return KF_ERR_ARG;
    const Slot& sl = s->sl();
    return save_grid_file(sl.d.tf, sl.d.tw, sl.cfg.volume_n, sl.d.fmt, path);
}

kf_status kf_load_tsdf_file(kf_session* s, const char* path) {
    if (!s || !path) return KF_ERR_ARG;
    Slot& sl = s->sl();
    return load_grid_file(sl.d.tf, sl.d.tw, sl.cfg.volume_n, sl.d.fmt, sl.d.bmin, sl.d.bdil, sl.d.sdil, path);
}

kf_status kf_save_vis_tsdf_file(kf_session* s, const char* path) {
    if (!s || !path) return KF_ERR_ARG;
    const Slot& sl = s->sl();
    if (!sl.d.vis.n) return KF_ERR_STATE;
    return save_grid_file(sl.d.vis.tf, sl.d.vis.tw, sl.d.vis.n, sl.d.fmt, path);
}

kf_status kf_load_vis_tsdf_file(kf_session* s, const char* path) {
    if (!s || !path) return KF_ERR_ARG;
    Slot& sl = s->sl();
    if (!sl.d.vis.n) return KF_ERR_STATE;
    return load_grid_file(sl.d.vis.tf, sl.d.vis.tw, sl.d.vis.n, sl.d.fmt, sl.d.vis.bmin, sl.d.vis.bdil, sl.d.vis.sdil,
                          path);
}

kf_status kf_session_checkpoint_save(kf_session* s, const char* path) {
    if (!s || !path) return KF_ERR_ARG;
    KF_TRY(kf_save_tsdf_file(s, path));
    float pose[16];
    KF_TRY(kf_get_pose(s, pose));
    const std::string side = std::string(path) + ".pose";
    FILE* f = std::fopen(side.c_str(), "w");
    if (!f) return KF_ERR_ARG;
    std::fprintf(f, "kinectfusion-b200 checkpoint 1\nframes %d\npose", s->sl().frames);
    for (int i = 0; i < 16; ++i) std::fprintf(f, " %.9g", double(pose[i]));
    std::fprintf(f, "\n");
    return std::fclose(f) == 0 ? KF_OK : KF_ERR_ARG;
}

kf_status kf_session_checkpoint_load(kf_session* s, const char* path) {
    if (!s || !path) return KF_ERR_ARG;
    const std::string side = std::string(path) + ".pose";
    FILE* f = std::fopen(side.c_str(), "r");
    if (!f) return KF_ERR_ARG;
    int frames = -1;
    float pose[16];
    char head[64] = {0};
    bool ok = std::fscanf(f, "%63[^\n]\nframes %d\npose", head, &frames) == 2 &&
              std::strcmp(head, "kinectfusion-b200 checkpoint 1") == 0 && frames >= 0;
    for (int i = 0; ok && i < 16; ++i) ok = std::fscanf(f, " %f", &pose[i]) == 1;
    std::fclose(f);
    if (!ok) return KF_ERR_ARG;
    KF_TRY(kf_load_tsdf_file(s, path));
    KF_TRY(kf_set_pose(s, pose));
    // resume: the next frame is frame `frames` (tracking, not the first-frame fusion only)
    Slot& sl = s->sl();
    sl.frames = frames;
    std::memcpy(sl.pose, pose, sizeof(pose));
    PoseDev P;
    KF_CK(cudaMemcpy(&P, sl.d.pose, sizeof(P), cudaMemcpyDeviceToHost));
    P.frame = frames;
    KF_CK(cudaMemcpy(sl.d.pose, &P, sizeof(P), cudaMemcpyHostToDevice));
    return KF_OK;
}

// ---- headless display (project/src/display.cu) ----

static kf_status display(int mode, const void* src, int w, int h, const DispMats& m, float scale, uint8_t* rgba,
                         void* stream, float* elapsed_ms) {
    if (!src || !rgba || w <= 0 || h <= 0) return KF_ERR_ARG;
    StageTimer t(elapsed_ms, as_stream(stream));
    return t.finish(stage_display(mode, src, w, h, m, scale, reinterpret_cast<unsigned int*>(rgba), as_stream(stream)));
}

kf_status kf_normal_map_to_rgba(const float* normal, int w, int h, const float inv_rot[9], uint8_t* rgba, void* stream,
                                float* elapsed_ms) {
    if (!inv_rot) return KF_ERR_ARG;
    DispMats m{};
    std::memcpy(m.r, inv_rot, sizeof(m.r));
    return display(kDisplayNormals, normal, w, h, m, 0.f, rgba, stream, elapsed_ms);
}

kf_status kf_shading_to_rgba(const float* normal, int w, int h, const float pose[16], const float inv_cam_k[9],
                             uint8_t* rgba, void* stream, float* elapsed_ms) {
    if (!pose || !inv_cam_k) return KF_ERR_ARG;
    DispMats m{};
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) m.r[c * 3 + r] = pose[c * 4 + r];
    std::memcpy(m.ik, inv_cam_k, sizeof(m.ik));
    return display(kDisplayShading, normal, w, h, m, 0.f, rgba, stream, elapsed_ms);
}

kf_status kf_float_channel_to_rgba(const float* src, int w, int h, float scale, uint8_t* rgba, void* stream,
                                   float* elapsed_ms) {
    DispMats m{};
    return display(kDisplayFloat, src, w, h, m, scale, rgba, stream, elapsed_ms);
}

kf_status kf_render(kf_session* s, int mode, const float pose_in[16], uint8_t* rgba, int to_host, void* stream) {
    NvtxRange nvtx_("kf_render");
    if (!s || !rgba || (mode != KF_RENDER_NORMALS && mode != KF_RENDER_SHADING)) return KF_ERR_ARG;
    Slot& sl = s->sl();
    if (sl.external) return KF_ERR_STATE;
    const kf_config& c = sl.cfg;
    const int w = c.width, h = c.height;
    cudaStream_t st = as_stream(stream);
    if (!sl.render_v) {
        cudaError_t err = cudaSuccess;
        sl.render_v = static_cast<float4*>(sl.alloc(size_t(w) * h * 16, err));
        if (err == cudaSuccess) sl.render_n = static_cast<float4*>(sl.alloc(size_t(w) * h * 16, err));
        if (err == cudaSuccess) sl.render_rgba = static_cast<unsigned int*>(sl.alloc(size_t(w) * h * 4, err));
        if (err != cudaSuccess) { g_last_cuda = err; sl.render_v = sl.render_n = nullptr; return KF_ERR_CUDA; }
    }
    float pose[16];
    if (pose_in) std::memcpy(pose, pose_in, sizeof(pose));
    else KF_TRY(kf_get_pose(s, pose));
    float k[9], ik[9];
    level_intrinsics(c, 0, k, ik);
    // the reference raycasts its visualization grid at level 0 into the predicted maps, then
    // displays (KinectFusion::visualizeCurrentModel, project/src/kinect_fusion.cpp:185-203); the
    // tracking maps are left alone here, and a session without a visualization volume renders
    // its tracking volume
    kf_volume vol;
    SessionDev bounds = sl.d;   // the brick bounds the march may skip by
    if (sl.d.vis.n) {
        KF_TRY(kf_get_vis_volume(s, &vol));
        bounds.bdil = sl.d.vis.bdil;
        bounds.sdil = sl.d.vis.sdil;
        bounds.nb = sl.d.vis.nb;
        bounds.ns = sl.d.vis.ns;
    } else {
        KF_TRY(kf_get_volume(s, &vol));
    }
    KF_CK(cudaStreamSynchronize(st));
    KF_CK(cudaMemsetAsync(sl.render_v, 0, size_t(w) * h * 16, st));
    KF_CK(cudaMemsetAsync(sl.render_n, 0, size_t(w) * h * 16, st));
    KF_CK(stage_raycast(&vol, pose, ik, sl.render_v, sl.render_n, w, h, c.min_depth, c.max_depth, c.step_large,
                        c.step_small, st, &bounds));
    DispMats m{};
    if (mode == KF_RENDER_NORMALS) {
        for (int cc = 0; cc < 3; ++cc)
            for (int r = 0; r < 3; ++r) m.r[cc * 3 + r] = pose[r * 4 + cc];   // inverse rotation R^T
    } else {
        for (int cc = 0; cc < 3; ++cc)
            for (int r = 0; r < 3; ++r) m.r[cc * 3 + r] = pose[cc * 4 + r];
        std::memcpy(m.ik, ik, sizeof(ik));
    }
    KF_CK(stage_display(mode == KF_RENDER_NORMALS ? kDisplayNormals : kDisplayShading, sl.render_n, w, h, m, 0.f,
                        sl.render_rgba, st));
    KF_CK(cudaMemcpyAsync(rgba, sl.render_rgba, size_t(w) * h * 4,
                          to_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, st));
    KF_CK(cudaStreamSynchronize(st));
    return KF_OK;
}

kf_status kf_get_volume(kf_session* s, kf_volume* out) {
    if (!s || !out) return KF_ERR_ARG;
    const Slot& sl = s->sl();
    out->f = sl.d.tf;
    out->w = sl.d.tw;
    out->n = sl.cfg.volume_n;
    out->width = sl.cfg.volume_width;
    out->mu = sl.cfg.mu;
    out->format = sl.cfg.tsdf_format;
    out->max_weight = sl.cfg.max_weight;
    return KF_OK;
}

kf_status kf_get_vis_volume(kf_session* s, kf_volume* out) {
    if (!s || !out) return KF_ERR_ARG;
    const Slot& sl = s->sl();
    if (!sl.d.vis.n) return KF_ERR_STATE;
    out->f = sl.d.vis.tf;
    out->w = sl.d.vis.tw;
    out->n = sl.d.vis.n;
    out->width = sl.d.vis.vol_w;
    out->mu = sl.d.vis.mu;
    out->format = sl.cfg.tsdf_format;
    out->max_weight = sl.cfg.max_weight;
    return KF_OK;
}

// ---- stages ----

kf_status kf_convert_to_depth_meters(const uint16_t* raw, int w, int h, float* out, int out_w, int out_h, float scale,
                                     int unmirror, void* stream, float* elapsed_ms) {
    if (!raw || !out || w <= 0 || h <= 0) return KF_ERR_ARG;
    if (w != out_w || h != out_h) return KF_ERR_SHAPE;
    StageTimer t(elapsed_ms, as_stream(stream));
    return t.finish(stage_convert(raw, out, w, h, scale, unmirror, as_stream(stream)));
}

kf_status kf_apply_bilateral_filter(const float* in, int w, int h, float* out, int out_w, int out_h, float sigma_s,
                                    float sigma_r, int radius, void* stream, float* elapsed_ms) {
    if (!in || !out || w <= 0 || h <= 0 || radius < 0 || radius > kMaxBilateralRadius) return KF_ERR_ARG;
    if (w != out_w || h != out_h) return KF_ERR_SHAPE;
    StageTimer t(elapsed_ms, as_stream(stream));
    return t.finish(stage_bilateral(in, out, w, h, sigma_s, sigma_r, radius, as_stream(stream)));
}

kf_status kf_down_sample(const float* in, int w, int h, float* out, int out_w, int out_h, float sigma_r, void* stream,
                         float* elapsed_ms) {
    if (!in || !out || out_w <= 0 || out_h <= 0) return KF_ERR_ARG;
    // project/src/measurement.cu:186-189
    if (w / out_w != 2 || h / out_h != 2) return KF_ERR_SHAPE;
    StageTimer t(elapsed_ms, as_stream(stream));
    return t.finish(stage_down_sample(in, out, out_w, out_h, sigma_r, as_stream(stream)));
}

kf_status kf_create_vertex_map(const float* depth, int w, int h, float* vertex, int out_w, int out_h,
                               const float inv_cam_k[9], void* stream, float* elapsed_ms) {
    if (!depth || !vertex || !inv_cam_k || w <= 0 || h <= 0) return KF_ERR_ARG;
    if (w != out_w || h != out_h) return KF_ERR_SHAPE;
    StageTimer t(elapsed_ms, as_stream(stream));
    return t.finish(stage_vertex(depth, reinterpret_cast<float4*>(vertex), w, h, inv_cam_k, as_stream(stream)));
}

kf_status kf_create_normal_map(const float* vertex, int w, int h, float* normal, int out_w, int out_h, void* stream,
                               float* elapsed_ms) {
    if (!vertex || !normal || w <= 0 || h <= 0) return KF_ERR_ARG;
    if (w != out_w || h != out_h) return KF_ERR_SHAPE;
    StageTimer t(elapsed_ms, as_stream(stream));
    return t.finish(stage_normal(reinterpret_cast<const float4*>(vertex), reinterpret_cast<float4*>(normal), w, h,
                                 as_stream(stream)));
}

static kf_status check_volume(const kf_volume* v) {
    if (!v || !v->f || !v->w || v->n < 8 || v->n % 8) return KF_ERR_ARG;
    if (v->format != KF_TSDF_F32F32 && v->format != KF_TSDF_F16U16) return KF_ERR_ARG;
    if (!(v->width > 0.f) || !(v->mu > 0.f)) return KF_ERR_ARG;
    return KF_OK;
}

kf_status kf_initialize_grid(const kf_volume* vol, void* stream, float* elapsed_ms) {
    KF_TRY(check_volume(vol));
    const long long n3 = (long long)vol->n * vol->n * vol->n;
    StageTimer t(elapsed_ms, as_stream(stream));
    return t.finish(launch_init_volume(vol->f, vol->w, n3, vol->format, as_stream(stream)));
}

kf_status kf_fuse(const float* depth_m, int w, int h, const float cam_k[9], const kf_volume* vol, const float pose[16],
                  float min_depth, float max_depth, void* stream, float* elapsed_ms) {
    NvtxRange nvtx_("kf_fuse");
    if (!depth_m || !cam_k || !pose || w <= 0 || h <= 0) return KF_ERR_ARG;
    KF_TRY(check_volume(vol));
    std::vector<float> xs(vol->n), zs(vol->n);
    voxel_axes(vol->n, vol->width, xs.data(), zs.data());
    float* d_ax = nullptr;
    KF_CK(cudaMalloc(&d_ax, sizeof(float) * 2 * vol->n));
    cudaStream_t st = as_stream(stream);
    cudaError_t e = cudaMemcpyAsync(d_ax, xs.data(), sizeof(float) * vol->n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_ax + vol->n, zs.data(), sizeof(float) * vol->n, cudaMemcpyHostToDevice, st);
    StageTimer t(elapsed_ms, st);
    if (e == cudaSuccess) e = stage_fuse(depth_m, w, h, cam_k, vol, pose, min_depth, max_depth, d_ax, d_ax + vol->n, st);
    kf_status r = t.finish(e);
    cudaStreamSynchronize(st);
    cudaFree(d_ax);
    return r;
}

kf_status kf_raycast(const kf_volume* vol, const float pose[16], const float inv_cam_k[9], float* vertex, int w, int h,
                     float* normal, int nw, int nh, float min_depth, float max_depth, float step_large,
                     float step_small, void* stream, float* elapsed_ms) {
    NvtxRange nvtx_("kf_raycast");
    if (!pose || !inv_cam_k || !vertex || !normal || w <= 0 || h <= 0) return KF_ERR_ARG;
    KF_TRY(check_volume(vol));
    if (w != nw || h != nh) return KF_ERR_SHAPE;   // project/src/raycast.cu:155-158
    if (!(step_large > step_small) || !(max_depth > min_depth) || !(max_depth < 1000.f) ||
        !(vol->mu * step_small > max_depth * 1e-6f))
        return KF_ERR_ARG;
    StageTimer t(elapsed_ms, as_stream(stream));
    return t.finish(stage_raycast(vol, pose, inv_cam_k, reinterpret_cast<float4*>(vertex),
                                  reinterpret_cast<float4*>(normal), w, h, min_depth, max_depth, step_large,
                                  step_small, as_stream(stream)));
}

kf_status kf_construct_icp_residuals(const float* vertex, const float* target_vertex, const float* target_normal, int w,
                                     int h, const float prev_rot[9], const float prev_transl[3], const float cur_rot[9],
                                     const float cur_transl[3], const float cam_k[9], float distance_thresh,
                                     float angle_thresh, float* mat_a, float* vec_b, void* stream, float* elapsed_ms) {
    if (!vertex || !target_vertex || !target_normal || !prev_rot || !prev_transl || !cur_rot || !cur_transl ||
        !cam_k || !mat_a || !vec_b || w <= 0 || h <= 0)
        return KF_ERR_ARG;
    StageTimer t(elapsed_ms, as_stream(stream));
    return t.finish(stage_icp_residuals(reinterpret_cast<const float4*>(vertex),
                                        reinterpret_cast<const float4*>(target_vertex),
                                        reinterpret_cast<const float4*>(target_normal), w, h, prev_rot, prev_transl,
                                        cur_rot, cur_transl, cam_k, distance_thresh, angle_thresh, mat_a, vec_b,
                                        as_stream(stream)));
}

// scratch of kf_solve_linear_least_squares: block partials + the FP64 solution, kept per
// process and per device ordinal (a call finds the scratch of the device current at the
// call), grown on demand
namespace {
constexpr int kLlsMaxDevices = 64;
struct LlsScratch {
    float* partials = nullptr;
    int cap = 0;
    double* x = nullptr;
};
std::mutex g_lls_mu;
LlsScratch g_lls[kLlsMaxDevices];
}  // namespace

kf_status kf_solve_linear_least_squares(const float* mat_a, const float* vec_b, int n, float x_out[6], void* stream) {
    if (!mat_a || !vec_b || !x_out || n <= 0) return KF_ERR_ARG;
    int dev = -1;
    KF_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kLlsMaxDevices) return KF_ERR_ARG;
    std::lock_guard<std::mutex> lk(g_lls_mu);
    LlsScratch& sc = g_lls[dev];
    const int nb = lls_num_blocks(n);
    if (nb > sc.cap || !sc.partials) {
        if (sc.partials) cudaFree(sc.partials);
        sc.partials = nullptr;
        sc.cap = 0;
        KF_CK(cudaMalloc(&sc.partials, sizeof(float) * 54 * size_t(nb)));
        sc.cap = nb;
    }
    if (!sc.x) KF_CK(cudaMalloc(&sc.x, sizeof(double) * 6));
    cudaStream_t st = as_stream(stream);
    KF_CK(stage_lls(mat_a, vec_b, n, sc.partials, sc.x, nb, st));
    double x[6];
    KF_CK(cudaMemcpyAsync(x, sc.x, sizeof(x), cudaMemcpyDeviceToHost, st));
    KF_CK(cudaStreamSynchronize(st));
    for (int q = 0; q < 6; ++q) x_out[q] = float(x[q]);
    for (int q = 0; q < 6; ++q)
        if (!std::isfinite(x[q])) return KF_ERR_NONFINITE;
    return KF_OK;
}

kf_status kf_compute_pose(const float* const* vertex, const float* const* target_vertex,
                          const float* const* target_normal, int w, int h, int levels, const kf_config* cfg,
                          const float pose[16], float pose_out[16], int iters_out[KF_MAX_LEVELS], void* stream) {
    NvtxRange nvtx_("kf_compute_pose");
    if (!vertex || !target_vertex || !target_normal || !cfg || !pose || !pose_out) return KF_ERR_ARG;
    if (levels < 1 || levels > KF_MAX_LEVELS) return KF_ERR_ARG;
    kf_config c = *cfg;
    c.width = w;
    c.height = h;
    c.levels = levels;
    c.export_icp_mask = 0;
    const int div = 1 << (levels - 1);
    if (w % div || h % div) return KF_ERR_SHAPE;
    int total = 0;
    for (int l = 0; l < levels; ++l) total += std::max(0, c.iters[l]);
    if (total > kIcpMaxPasses) return KF_ERR_ARG;
    for (int l = 0; l < levels; ++l)
        if (!vertex[l] || !target_vertex[l] || !target_normal[l]) return KF_ERR_ARG;
    Engine eng;
    kf_status st = eng.init(1);
    if (st != KF_OK) { eng.destroy(); return st; }
    Slot& sl = eng.slots[0];
    sl.cfg = c;
    sl.used = true;
    sl.external = true;
    std::memset(&sl.d, 0, sizeof(sl.d));
    fill_levels(sl.d, c);
    for (int l = 0; l < levels; ++l) {
        sl.d.vmap[l] = reinterpret_cast<float4*>(const_cast<float*>(vertex[l]));
        sl.d.pv[l] = reinterpret_cast<float4*>(const_cast<float*>(target_vertex[l]));
        sl.d.pn[l] = reinterpret_cast<float4*>(const_cast<float*>(target_normal[l]));
    }
    PoseDev* d_pose = nullptr;
    cudaStream_t s = as_stream(stream);
    auto fail = [&](cudaError_t e) {
        g_last_cuda = e;
        if (d_pose) cudaFree(d_pose);
        eng.destroy();
        return KF_ERR_CUDA;
    };
    cudaError_t e = cudaMalloc(&d_pose, sizeof(PoseDev));
    if (e != cudaSuccess) return fail(e);
    PoseDev P = make_pose_dev(pose);
    e = cudaMemcpy(d_pose, &P, sizeof(P), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(e);
    sl.d.pose = d_pose;
    st = eng.build_tables();
    if (st != KF_OK) { cudaFree(d_pose); eng.destroy(); return st; }
    StepDev step{1, 0};
    e = cudaMemcpy(eng.d_step, &step, sizeof(step), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemsetAsync(eng.d_sync, 0, sizeof(GridSync), s);
    if (e == cudaSuccess) e = launch_icp(eng.view(), eng.shape.grid_icp, s, eng.cap == 1);
    if (e == cudaSuccess) e = cudaMemcpyAsync(eng.h_out, eng.d_out, eng.out_bytes(), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(e);
    std::memcpy(pose_out, eng.h_out[0].pose, sizeof(float) * 16);
    if (iters_out)
        for (int l = 0; l < KF_MAX_LEVELS; ++l) iters_out[l] = eng.h_out[0].iters[l];
    kf_status r = eng.h_sync->abort ? KF_ERR_TIMEOUT : kf_status(eng.h_out[0].status);
    cudaFree(d_pose);
    eng.destroy();
    return r;
}

kf_status kf_pose_error(const float p1[16], const float p2[16], float out[2]) {
    if (!p1 || !p2 || !out) return KF_ERR_ARG;
    // project/src/general_helper.cpp:11-21 in float
    const float inv = 1.0f / std::sqrt(3.0f);
    const float v[3] = {inv, inv, inv};
    float a[3], b[3];
    for (int r = 0; r < 3; ++r) {
        a[r] = p1[r] * v[0] + p1[4 + r] * v[1] + p1[8 + r] * v[2];
        b[r] = p2[r] * v[0] + p2[4 + r] * v[1] + p2[8 + r] * v[2];
    }
    out[0] = std::sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
    out[1] = std::sqrt((p1[12] - p2[12]) * (p1[12] - p2[12]) + (p1[13] - p2[13]) * (p1[13] - p2[13]) +
                       (p1[14] - p2[14]) * (p1[14] - p2[14]));
    return KF_OK;
}

// ---- batch ----

kf_status kf_batch_create(const kf_config* cfgs, int n, kf_batch** out) {
    if (!cfgs || n <= 0 || !out) return KF_ERR_ARG;
    for (int i = 0; i < n; ++i) KF_TRY(validate(cfgs[i]));
    kf_batch* b = new (std::nothrow) kf_batch;
    if (!b) return KF_ERR_ARG;
    b->n = n;
    kf_status st = b->eng.init(n);
    for (int i = 0; i < n && st == KF_OK; ++i) st = slot_create(b->eng.slots[i], cfgs[i]);
    if (st != KF_OK) { b->eng.destroy(); delete b; return st; }
    b->eng.tables_dirty = true;
    *out = b;
    return KF_OK;
}

kf_status kf_batch_destroy(kf_batch* b) {
    if (!b) return KF_ERR_ARG;
    cudaDeviceSynchronize();
    for (kf_session* v : b->views) delete v;
    b->eng.destroy();
    delete b;
    return KF_OK;
}

kf_status kf_batch_step(kf_batch* b, const uint16_t* const* depth, int is_device_ptr, void* stream, float* poses_out) {
    NvtxRange nvtx_("kf_batch_step");
    if (!b || !depth) return KF_ERR_ARG;
    cudaStream_t st = as_stream(stream);
    std::vector<StepDev> want(b->n);
    for (int i = 0; i < b->n; ++i) {
        Slot& sl = b->eng.slots[i];
        want[i] = StepDev{depth[i] ? 1 : 0, sl.frames == 0 ? 1 : 0};
    }
    KF_TRY(b->eng.set_step(want, st));
    KF_TRY(tuner_before_step(b->eng));
    cudaStream_t cs = st;
    KF_TRY(b->eng.begin_inputs(st, &cs));
    for (int i = 0; i < b->n; ++i) {
        if (!depth[i]) continue;
        Slot& sl = b->eng.slots[i];
        KF_CK(cudaMemcpyAsync(const_cast<uint16_t*>(sl.d.raw), depth[i], size_t(sl.cfg.width) * sl.cfg.height * 2,
                              is_device_ptr ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, cs));
    }
    KF_TRY(b->eng.end_inputs(cs));
    KF_TRY(b->eng.enqueue(st));
    KF_TRY(b->eng.fetch(st));
    KF_CK(cudaStreamSynchronize(st));
    kf_status r = b->eng.collect(want);
    KF_TRY(tuner_after_step(b->eng));
    if (poses_out)
        for (int i = 0; i < b->n; ++i) std::memcpy(poses_out + 16 * size_t(i), b->eng.slots[i].pose, sizeof(float) * 16);
    return r;
}

kf_status kf_batch_step_async(kf_batch* b, const int* active, void* stream) {
    NvtxRange nvtx_("kf_batch_step_async");
    if (!b || !active) return KF_ERR_ARG;
    cudaStream_t st = as_stream(stream);
    std::vector<StepDev> want(b->n);
    for (int i = 0; i < b->n; ++i) want[i] = StepDev{active[i] ? 1 : 0, b->eng.slots[i].frames == 0 ? 1 : 0};
    KF_TRY(b->eng.set_step(want, st));
    KF_TRY(b->eng.enqueue(st));
    for (int i = 0; i < b->n; ++i)
        if (active[i]) b->eng.slots[i].frames += 1;
    return KF_OK;
}

kf_status kf_batch_input_buffer(kf_batch* b, int i, uint16_t** dev_ptr) {
    if (!b || !dev_ptr || i < 0 || i >= b->n) return KF_ERR_ARG;
    *dev_ptr = const_cast<uint16_t*>(b->eng.slots[i].d.raw);
    return KF_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// batch views and autotuning
// ------------------------------------------------------------------------------------------
namespace {

// the batch's session mix: what the tuned shapes depend on (frame sizes, volumes, formats,
// how many of each) and the device's SM count
std::string mix_key(const Engine& e) {
    std::vector<std::string> kinds;
    for (const Slot& sl : e.slots) {
        if (!sl.used) continue;
        char buf[96];
        std::snprintf(buf, sizeof(buf), "%dx%d/%d/%s/L%d", sl.cfg.width, sl.cfg.height, sl.cfg.volume_n,
                      sl.cfg.tsdf_format == KF_TSDF_F16U16 ? "f16u16" : "f32f32", sl.cfg.levels);
        kinds.emplace_back(buf);
    }
    std::sort(kinds.begin(), kinds.end());
    std::string key = std::to_string(e.sms) + "sm";
    for (size_t i = 0; i < kinds.size();) {
        size_t j = i;
        while (j < kinds.size() && kinds[j] == kinds[i]) ++j;
        key += " " + kinds[i] + "*" + std::to_string(j - i);
        i = j;
    }
    return key;
}

const char* const kShapeFields[] = {"grid_pre", "grid_ray", "grid_fuse", "grid_icp",
                                    "ray_form", "ray_budget", "ray_tw", "fuse_split"};
int Shape::* const kShapeMembers[] = {&Shape::grid_pre, &Shape::grid_ray, &Shape::grid_fuse, &Shape::grid_icp,
                                      &Shape::ray_form, &Shape::ray_budget, &Shape::ray_tw, &Shape::fuse_split};
constexpr int kShapeFieldCount = 8;

std::string shape_json(const Shape& sh) {
    std::string j = "{";
    for (int q = 0; q < kShapeFieldCount; ++q) {
        j += std::string(q ? ", " : "") + "\"" + kShapeFields[q] + "\": " + std::to_string(sh.*kShapeMembers[q]);
    }
    return j + "}";
}

// The cache file is a JSON object with one line per session mix:
//   "<mix key>": {"grid_pre": 592, "grid_ray": 888, ...},
// Returns true and fills `out` when `key` has an entry.
bool cache_lookup(const std::string& path, const std::string& key, Shape& out) {
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return false;
    char line[1024];
    bool found = false;
    const std::string head = "\"" + key + "\": {";
    while (!found && std::fgets(line, sizeof(line), f)) {
        const char* p = std::strstr(line, head.c_str());
        if (!p) continue;
        Shape sh = out;
        int got = 0;
        for (int q = 0; q < kShapeFieldCount; ++q) {
            const std::string name = "\"" + std::string(kShapeFields[q]) + "\": ";
            const char* v = std::strstr(p + head.size(), name.c_str());
            int x = 0;
            if (v && std::sscanf(v + name.size(), "%d", &x) == 1) {
                sh.*kShapeMembers[q] = x;
                ++got;
            }
        }
        if (got == kShapeFieldCount) {
            out = sh;
            found = true;
        }
    }
    std::fclose(f);
    return found;
}

// add or replace the entry of `key` (other mixes' entries are kept)
bool cache_store(const std::string& path, const std::string& key, const Shape& sh) {
    std::vector<std::string> entries;
    const std::string head = "\"" + key + "\": {";
    if (FILE* f = std::fopen(path.c_str(), "r")) {
        char line[1024];
        while (std::fgets(line, sizeof(line), f)) {
            std::string l(line);
            while (!l.empty() && (l.back() == '\n' || l.back() == ',' || l.back() == ' ')) l.pop_back();
            if (l.find("\": {") == std::string::npos || l.find(head) != std::string::npos) continue;
            size_t start = l.find('"');
            entries.push_back(l.substr(start));
        }
        std::fclose(f);
    }
    entries.push_back("\"" + key + "\": " + shape_json(sh));
    const std::string tmp = path + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "w");
    if (!f) return false;
    std::fprintf(f, "{\n");
    for (size_t i = 0; i < entries.size(); ++i)
        std::fprintf(f, "  %s%s\n", entries[i].c_str(), i + 1 < entries.size() ? "," : "");
    std::fprintf(f, "}\n");
    if (std::fclose(f) != 0) return false;
    return std::rename(tmp.c_str(), path.c_str()) == 0;
}

// the candidates the walk tries, in order (grids as multiples of the SM count)
std::vector<Tuner::Param> tuner_params(int sms) {
    std::vector<Tuner::Param> p;
    p.push_back({"grid_ray", &Shape::grid_ray, {2 * sms, 4 * sms, 6 * sms, 8 * sms, 12 * sms, 16 * sms}});
    p.push_back({"ray_form", &Shape::ray_form, {3, 4}});
    p.push_back({"ray_budget", &Shape::ray_budget, {24, 32, 40, 48, 64, 96}});
    p.push_back({"ray_tw", &Shape::ray_tw, {8, 16, 4}});
    p.push_back({"grid_pre", &Shape::grid_pre, {1 * sms, 2 * sms, 4 * sms, 8 * sms}});
    p.push_back({"grid_icp", &Shape::grid_icp, {sms, 2 * sms}});
    p.push_back({"grid_fuse", &Shape::grid_fuse, {2 * sms, 4 * sms, 6 * sms, 8 * sms}});
    p.push_back({"fuse_split", &Shape::fuse_split, {1, 2, 4}});
    return p;
}

// before a batch step: the shape of the tuner's current candidate
kf_status tuner_before_step(Engine& e) {
    Tuner& t = e.tuner;
    if (!t.active) return KF_OK;
    Shape sh = t.base;
    sh.*(t.params[t.pi].field) = t.params[t.pi].cand[t.ci];
    e.set_shape(sh);
    return KF_OK;
}

// after a batch step finished: record its stage time for the candidate and move on
kf_status tuner_after_step(Engine& e) {
    Tuner& t = e.tuner;
    if (!t.active) return KF_OK;
    float ms[4];
    KF_TRY(e.stage_times(ms));
    const Tuner::Param& p = t.params[t.pi];
    t.best[t.ci] = std::min(t.best[t.ci], ms[1] + ms[2] + ms[3]);   // fork to the end of fusion
    if (++t.rep < Tuner::kReps) return KF_OK;
    t.rep = 0;
    if (++t.ci < int(p.cand.size())) return KF_OK;
    // the parameter's winner
    int w = 0;
    for (int c = 1; c < int(p.cand.size()); ++c)
        if (t.best[c] < t.best[w]) w = c;
    t.base.*(p.field) = p.cand[w];
    char buf[96];
    std::snprintf(buf, sizeof(buf), "%s\"%s\": [%d, %.5f]", t.report.size() > 1 ? ", " : "", p.name, p.cand[w],
                  t.best[w]);
    t.report += buf;
    t.ci = 0;
    if (++t.pi < int(t.params.size())) {
        t.best.assign(t.params[t.pi].cand.size(), 1e30f);
        return KF_OK;
    }
    // done: keep the walk's shape and remember it
    t.active = false;
    t.done = true;
    e.set_shape(t.base);
    KF_TRY(e.set_profile(t.was_profiling));
    t.report = "{\"mix\": \"" + t.key + "\", \"source\": \"tuned\", \"shape\": " + shape_json(t.base) +
               ", \"step_ms\": " + t.report + "}}";
    if (!t.cache_path.empty()) cache_store(t.cache_path, t.key, t.base);
    return KF_OK;
}

}  // namespace

extern "C" {

kf_status kf_batch_session(kf_batch* b, int i, kf_session** out) {
    if (!b || !out || i < 0 || i >= b->n) return KF_ERR_ARG;
    if (b->views.empty()) {
        b->views.resize(b->n, nullptr);
    }
    if (!b->views[i]) {
        kf_session* v = new (std::nothrow) kf_session;
        if (!v) return KF_ERR_ARG;
        v->eng = &b->eng;
        v->slot = i;
        v->owns = false;
        b->views[i] = v;
    }
    *out = b->views[i];
    return KF_OK;
}

kf_status kf_batch_autotune_start(kf_batch* b, const char* cache_path) {
    NvtxRange nvtx_("kf_batch_autotune_start");
    if (!b) return KF_ERR_ARG;
    Engine& e = b->eng;
    Tuner& t = e.tuner;
    KF_CK(cudaDeviceSynchronize());
    t = Tuner{};
    t.key = mix_key(e);
    t.cache_path = cache_path ? cache_path : "";
    Shape cached = e.shape;
    if (!t.cache_path.empty() && cache_lookup(t.cache_path, t.key, cached)) {
        e.set_shape(cached);
        t.base = cached;
        t.done = true;
        t.report = "{\"mix\": \"" + t.key + "\", \"source\": \"cache\", \"shape\": " + shape_json(cached) + "}";
        return KF_OK;
    }
    t.params = tuner_params(e.sms);
    t.base = e.shape;
    t.best.assign(t.params[0].cand.size(), 1e30f);
    t.was_profiling = e.profile;
    KF_TRY(e.set_profile(true));
    t.report = "{";
    t.active = true;
    return KF_OK;
}

kf_status kf_batch_autotune_status(kf_batch* b, int* steps_left, char* report, size_t report_bytes) {
    if (!b) return KF_ERR_ARG;
    const Tuner& t = b->eng.tuner;
    if (steps_left) *steps_left = t.steps_left();
    if (report && report_bytes) {
        const std::string r = t.done ? t.report : t.active ? std::string("{\"source\": \"tuning\"}") : std::string("{}");
        std::strncpy(report, r.c_str(), report_bytes - 1);
        report[report_bytes - 1] = 0;
    }
    return KF_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// server: continuous batching with HBM-budget admission
// ------------------------------------------------------------------------------------------
namespace {

struct ServerSlot {
    int id = -1;                  // session id, -1 = free
    uint16_t* stage[2] = {nullptr, nullptr};   // pinned staging buffers (kept across sessions)
    size_t stage_bytes = 0;       // frame bytes of the current session
    size_t stage_cap = 0;         // bytes each staging buffer holds
    bool reserved = false;        // being opened or closed: not free, not yet serving
    int pending = -1;             // staged buffer waiting for a step
    int inflight = -1;            // staged buffer a running step reads
    double t_submit[2] = {0, 0};
    bool has_result = false;
};

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct kf_server {
    Engine eng;
    ArenaPool pool;      // device arenas of closed sessions, reused by the next ones
    int max_slots = 0;
    size_t budget = 0, in_use = 0;
    std::vector<ServerSlot> hs;
    std::vector<kf_session*> views;
    std::mutex q_mu;     // queue state (submit / step bookkeeping)
    std::mutex gpu_mu;   // engine: steps, open, close
    cudaStream_t stream = nullptr;
    int next_id = 1;
    std::vector<double> lat;
    long long frames_done = 0, admitted = 0, refused = 0, steps = 0;
    int max_active = 0;

    int find(int id) const {
        for (int i = 0; i < max_slots; ++i)
            if (hs[i].id == id) return i;
        return -1;
    }
};

extern "C" {

double kf_now_ms(void) { return now_ms(); }

kf_status kf_server_create(int max_slots, size_t hbm_budget, kf_server** out) {
    if (max_slots <= 0 || !out) return KF_ERR_ARG;
    kf_server* s = new (std::nothrow) kf_server;
    if (!s) return KF_ERR_ARG;
    s->max_slots = max_slots;
    s->budget = hbm_budget;
    s->hs.resize(max_slots);
    s->views.resize(max_slots, nullptr);
    kf_status st = s->eng.init(max_slots);
    if (st == KF_OK && cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) st = KF_ERR_CUDA;
    if (st != KF_OK) { s->eng.destroy(); delete s; return st; }
    *out = s;
    return KF_OK;
}

kf_status kf_server_destroy(kf_server* s) {
    if (!s) return KF_ERR_ARG;
    std::lock_guard<std::mutex> g(s->gpu_mu);
    cudaDeviceSynchronize();
    for (ServerSlot& h : s->hs)
        for (int b = 0; b < 2; ++b)
            if (h.stage[b]) cudaFreeHost(h.stage[b]);
    for (kf_session* v : s->views) delete v;
    s->eng.destroy();
    s->pool.trim(0);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return KF_OK;
}

kf_status kf_server_open(kf_server* s, const kf_config* cfg, int* id) {
    NvtxRange nvtx_("kf_server_open");
    if (!s || !cfg || !id) return KF_ERR_ARG;
    KF_TRY(validate(*cfg));
    const size_t need = footprint(*cfg) + size_t(cfg->width) * cfg->height * 2 * 2;
    int slot = -1;
    size_t keep_cached = 0;
    {
        std::lock_guard<std::mutex> q(s->q_mu);
        if (s->in_use + need > s->budget) {
            s->refused++;
            return KF_ERR_OOM_BUDGET;
        }
        for (int i = 0; i < s->max_slots; ++i)
            if (s->hs[i].id < 0 && !s->hs[i].reserved) { slot = i; break; }
        if (slot < 0) {
            s->refused++;
            return KF_ERR_CAPACITY;
        }
        s->hs[slot].reserved = true;
        s->in_use += need;   // held while the session is built
        keep_cached = s->budget - s->in_use;
    }
    // Build the session outside the GPU lock, on a stream of its own, so that the other
    // sessions' steps go on meanwhile.  Cached arenas count against the budget too.
    if (s->pool.cached > keep_cached) s->pool.trim(keep_cached);
    ServerSlot& h = s->hs[slot];   // reserved: no other thread touches it until registered
    Slot tmp;
    tmp.pool = &s->pool;
    cudaStream_t st = nullptr;
    kf_status r = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess ? KF_OK : KF_ERR_CUDA;
    if (r == KF_OK) r = slot_create(tmp, *cfg, st);
    if (st) cudaStreamDestroy(st);
    const size_t frame_bytes = size_t(cfg->width) * cfg->height * 2;
    if (r == KF_OK && h.stage_cap < frame_bytes) {
        for (int b = 0; b < 2; ++b) {
            if (h.stage[b]) cudaFreeHost(h.stage[b]);
            h.stage[b] = nullptr;
        }
        h.stage_cap = 0;
        for (int b = 0; b < 2 && r == KF_OK; ++b)
            if (cudaMallocHost(&h.stage[b], frame_bytes) != cudaSuccess) r = KF_ERR_CUDA;
        if (r == KF_OK) h.stage_cap = frame_bytes;
    }
    if (r != KF_OK) {
        tmp.release();
        std::lock_guard<std::mutex> q(s->q_mu);
        h.reserved = false;
        s->in_use -= need;
        return r;
    }
    {
        std::lock_guard<std::mutex> g(s->gpu_mu);
        std::swap(s->eng.slots[slot], tmp);   // tmp receives the empty slot
        s->eng.tables_dirty = true;
    }
    tmp.release();
    {
        std::lock_guard<std::mutex> q(s->q_mu);
        h.stage_bytes = frame_bytes;
        h.pending = h.inflight = -1;
        h.has_result = false;
        h.id = s->next_id++;
        h.reserved = false;
        s->in_use = s->in_use - need + s->eng.slots[slot].bytes + 2 * frame_bytes;
        s->admitted++;
        *id = h.id;
    }
    return KF_OK;
}

kf_status kf_server_reserve(kf_server* s, const kf_config* cfg, int count) {
    if (!s || !cfg || count < 0) return KF_ERR_ARG;
    KF_TRY(validate(*cfg));
    const size_t arena = footprint(*cfg) + (64u << 10);   // what slot_create reserves
    const size_t frame_bytes = size_t(cfg->width) * cfg->height * 2;
    {
        std::lock_guard<std::mutex> q(s->q_mu);
        if (s->in_use + s->pool.cached + size_t(count) * arena > s->budget) return KF_ERR_OOM_BUDGET;
    }
    for (int k = 0; k < count; ++k) {
        char* p = nullptr;
        KF_CK(cudaMalloc(&p, arena));
        s->pool.put(p, arena);
    }
    {
        // the engine's work lists, sized for these sessions on top of the current ones
        std::lock_guard<std::mutex> g(s->gpu_mu);
        KF_CK(cudaStreamSynchronize(s->stream));
        KF_TRY(s->eng.reserve_work(*cfg, count));
    }
    // staging for up to `count` free slots that have none large enough
    int staged = 0;
    for (int i = 0; i < s->max_slots && staged < count; ++i) {
        ServerSlot& h = s->hs[i];
        {
            std::lock_guard<std::mutex> q(s->q_mu);
            if (h.id >= 0 || h.reserved) continue;
            h.reserved = true;
        }
        kf_status r = KF_OK;
        if (h.stage_cap < frame_bytes) {
            for (int b = 0; b < 2; ++b) {
                if (h.stage[b]) cudaFreeHost(h.stage[b]);
                h.stage[b] = nullptr;
            }
            h.stage_cap = 0;
            for (int b = 0; b < 2 && r == KF_OK; ++b)
                if (cudaMallocHost(&h.stage[b], frame_bytes) != cudaSuccess) r = KF_ERR_CUDA;
            if (r == KF_OK) h.stage_cap = frame_bytes;
        }
        {
            std::lock_guard<std::mutex> q(s->q_mu);
            h.reserved = false;
        }
        if (r != KF_OK) return r;
        ++staged;
    }
    return KF_OK;
}

kf_status kf_server_close(kf_server* s, int id) {
    NvtxRange nvtx_("kf_server_close");
    if (!s) return KF_ERR_ARG;
    int slot;
    {
        std::lock_guard<std::mutex> q(s->q_mu);
        slot = s->find(id);
        if (slot < 0) return KF_ERR_ARG;
        s->hs[slot].id = -1;
        s->hs[slot].pending = -1;
        s->hs[slot].reserved = true;   // not reusable until its memory is back
    }
    Slot tmp;
    {
        std::lock_guard<std::mutex> g(s->gpu_mu);   // no step is running while it is held
        KF_CK(cudaStreamSynchronize(s->stream));
        std::swap(s->eng.slots[slot], tmp);
        s->eng.tables_dirty = true;
    }
    const size_t freed = tmp.bytes + 2 * s->hs[slot].stage_bytes;
    tmp.release();   // the arena goes back to the pool; the staging stays with the slot
    {
        std::lock_guard<std::mutex> q(s->q_mu);
        s->in_use -= freed;
        s->hs[slot].reserved = false;
    }
    return KF_OK;
}

kf_status kf_server_submit(kf_server* s, int id, const uint16_t* depth, double t_submit_ms) {
    if (!s || !depth) return KF_ERR_ARG;
    std::lock_guard<std::mutex> q(s->q_mu);
    const int slot = s->find(id);
    if (slot < 0) return KF_ERR_ARG;
    ServerSlot& h = s->hs[slot];
    if (h.pending >= 0) return KF_ERR_STATE;
    const int b = h.inflight == 0 ? 1 : 0;
    std::memcpy(h.stage[b], depth, h.stage_bytes);
    h.t_submit[b] = t_submit_ms;
    h.pending = b;
    return KF_OK;
}

kf_status kf_server_step(kf_server* s, int* served) {
    NvtxRange nvtx_("kf_server_step");
    if (!s) return KF_ERR_ARG;
    std::lock_guard<std::mutex> g(s->gpu_mu);
    const int cap = s->max_slots;
    std::vector<StepDev> want(cap, StepDev{0, 0});
    int n = 0;
    {
        std::lock_guard<std::mutex> q(s->q_mu);
        for (int i = 0; i < cap; ++i) {
            ServerSlot& h = s->hs[i];
            if (h.id < 0 || h.pending < 0) continue;
            h.inflight = h.pending;
            h.pending = -1;
            want[i] = StepDev{1, s->eng.slots[i].frames == 0 ? 1 : 0};
            ++n;
        }
    }
    if (served) *served = n;
    if (n == 0) return KF_OK;
    cudaStream_t st = s->stream;
    KF_TRY(s->eng.set_step(want, st));
    cudaStream_t cs = st;
    KF_TRY(s->eng.begin_inputs(st, &cs));
    for (int i = 0; i < cap; ++i) {
        if (!want[i].active) continue;
        const ServerSlot& h = s->hs[i];
        KF_CK(cudaMemcpyAsync(const_cast<uint16_t*>(s->eng.slots[i].d.raw), h.stage[h.inflight], h.stage_bytes,
                              cudaMemcpyHostToDevice, cs));
    }
    KF_TRY(s->eng.end_inputs(cs));
    KF_TRY(s->eng.enqueue(st));
    KF_TRY(s->eng.fetch(st));
    KF_CK(cudaStreamSynchronize(st));
    kf_status r = s->eng.collect(want);
    const double t = now_ms();
    {
        std::lock_guard<std::mutex> q(s->q_mu);
        for (int i = 0; i < cap; ++i) {
            if (!want[i].active) continue;
            ServerSlot& h = s->hs[i];
            s->lat.push_back(t - h.t_submit[h.inflight]);
            h.inflight = -1;
            h.has_result = true;
        }
        s->frames_done += n;
        s->steps++;
        s->max_active = std::max(s->max_active, n);
    }
    return r;
}

kf_status kf_server_result(kf_server* s, int id, float pose[16], kf_frame_stats* stats) {
    if (!s) return KF_ERR_ARG;
    std::lock_guard<std::mutex> g(s->gpu_mu);
    const int slot = s->find(id);
    if (slot < 0) return KF_ERR_ARG;
    if (!s->hs[slot].has_result) return KF_ERR_STATE;
    if (pose) std::memcpy(pose, s->eng.slots[slot].pose, sizeof(float) * 16);
    if (stats) *stats = s->eng.slots[slot].stats;
    return KF_OK;
}

kf_status kf_server_get_session(kf_server* s, int id, kf_session** out) {
    if (!s || !out) return KF_ERR_ARG;
    std::lock_guard<std::mutex> g(s->gpu_mu);
    const int slot = s->find(id);
    if (slot < 0) return KF_ERR_ARG;
    if (!s->views[slot]) {
        kf_session* v = new (std::nothrow) kf_session;
        if (!v) return KF_ERR_ARG;
        v->eng = &s->eng;
        v->slot = slot;
        v->owns = false;
        s->views[slot] = v;
    }
    *out = s->views[slot];
    return KF_OK;
}

kf_status kf_server_stats_reset(kf_server* s) {
    if (!s) return KF_ERR_ARG;
    std::lock_guard<std::mutex> q(s->q_mu);
    s->lat.clear();
    s->frames_done = s->admitted = s->refused = s->steps = 0;
    int active = 0;
    for (const ServerSlot& h : s->hs)
        if (h.id >= 0) ++active;
    s->max_active = active;
    return KF_OK;
}

kf_status kf_server_stats_get(kf_server* s, kf_server_stats* out) {
    if (!s || !out) return KF_ERR_ARG;
    std::lock_guard<std::mutex> q(s->q_mu);
    std::memset(out, 0, sizeof(*out));
    out->frames_done = s->frames_done;
    out->sessions_admitted = s->admitted;
    out->sessions_refused = s->refused;
    out->steps = s->steps;
    int active = 0;
    for (const ServerSlot& h : s->hs)
        if (h.id >= 0) ++active;
    out->active_sessions = active;
    out->max_active_sessions = s->max_active;
    out->hbm_in_use = s->in_use;
    out->hbm_budget = s->budget;
    if (!s->lat.empty()) {
        std::vector<double> v = s->lat;
        std::sort(v.begin(), v.end());
        auto pct = [&v](double p) {
            const size_t i = std::min(v.size() - 1, size_t(p * double(v.size() - 1) + 0.5));
            return v[i];
        };
        out->p50_ms = pct(0.50);
        out->p99_ms = pct(0.99);
        out->max_ms = v.back();
    }
    return KF_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// instrumentation
// ------------------------------------------------------------------------------------------
extern "C" {

kf_status kf_session_set_profiling(kf_session* s, int on) {
    if (!s) return KF_ERR_ARG;
    return s->eng->set_profile(on != 0);
}

kf_status kf_session_stage_times(kf_session* s, float ms[4]) {
    if (!s || !ms) return KF_ERR_ARG;
    return s->eng->stage_times(ms);
}

// debug modes of one slot's session (traces) and of its engine (plain launches)
static kf_status slot_set_debug(Engine& e, Slot& sl, int flags) {
    if (sl.external) return KF_ERR_STATE;
    const bool want = (flags & KF_DEBUG_RAY_TRACE) != 0;
    for (int l = 0; l < sl.cfg.levels; ++l) {
        if (want && !sl.d.trace[l]) {
            void* p = nullptr;
            const size_t bytes = level_px(sl.cfg, l) * sizeof(unsigned long long);
            KF_CK(cudaMalloc(&p, bytes));
            sl.allocs.push_back(p);
            KF_CK(cudaMemset(p, 0, bytes));
            sl.d.trace[l] = static_cast<unsigned long long*>(p);
        } else if (!want && sl.d.trace[l]) {
            // the buffer stays with the slot (freed with it); the kernels stop writing it
            sl.d.trace[l] = nullptr;
        }
    }
    e.tables_dirty = true;   // the session record on the device carries the pointers
    const bool graph = (flags & KF_DEBUG_NO_GRAPH) == 0;
    if (graph != e.use_graph) {
        e.use_graph = graph;
        e.graph_dirty = true;
    }
    const bool count = (flags & KF_DEBUG_COUNTERS) != 0;
    if (count && !e.d_ray_counts) {
        KF_CK(cudaMalloc(&e.d_ray_counts, sizeof(unsigned long long) * ray_count_slots()));
        KF_CK(cudaMemset(e.d_ray_counts, 0, sizeof(unsigned long long) * ray_count_slots()));
    }
    if (count != e.count_rays) {
        e.count_rays = count;
        e.graph_dirty = true;   // the step launches the counting or the plain kernels
    }
    return KF_OK;
}

static kf_status engine_counts(Engine& e, uint64_t* out, int n) {
    if (!out || n <= 0) return KF_ERR_ARG;
    if (!e.count_rays || !e.d_ray_counts) return KF_ERR_STATE;
    std::vector<unsigned long long> c(ray_count_slots());
    KF_CK(cudaDeviceSynchronize());
    KF_CK(cudaMemcpy(c.data(), e.d_ray_counts, sizeof(unsigned long long) * c.size(), cudaMemcpyDeviceToHost));
    for (int k = 0; k < n; ++k) out[k] = k < int(c.size()) ? c[k] : 0;
    return KF_OK;
}

kf_status kf_session_set_debug(kf_session* s, int flags) {
    if (!s || (flags & ~(KF_DEBUG_RAY_TRACE | KF_DEBUG_NO_GRAPH | KF_DEBUG_COUNTERS))) return KF_ERR_ARG;
    KF_CK(cudaDeviceSynchronize());
    return slot_set_debug(*s->eng, s->sl(), flags);
}

kf_status kf_batch_set_debug(kf_batch* b, int flags) {
    if (!b || (flags & ~(KF_DEBUG_RAY_TRACE | KF_DEBUG_NO_GRAPH | KF_DEBUG_COUNTERS))) return KF_ERR_ARG;
    KF_CK(cudaDeviceSynchronize());
    for (Slot& sl : b->eng.slots)
        if (sl.used) KF_TRY(slot_set_debug(b->eng, sl, flags));
    return KF_OK;
}

kf_status kf_session_debug_counts(kf_session* s, uint64_t* out, int n) {
    if (!s) return KF_ERR_ARG;
    return engine_counts(*s->eng, out, n);
}

kf_status kf_batch_debug_counts(kf_batch* b, uint64_t* out, int n) {
    if (!b) return KF_ERR_ARG;
    return engine_counts(b->eng, out, n);
}

kf_status kf_get_ray_trace(kf_session* s, int level, uint64_t* dst, int to_host) {
    if (!s || !dst) return KF_ERR_ARG;
    const Slot& sl = s->sl();
    if (level < 0 || level >= sl.cfg.levels) return KF_ERR_ARG;
    if (!sl.d.trace[level]) return KF_ERR_STATE;
    return copy_out(dst, sl.d.trace[level], level_px(sl.cfg, level) * sizeof(uint64_t), to_host);
}

kf_status kf_batch_set_profiling(kf_batch* b, int on) {
    if (!b) return KF_ERR_ARG;
    return b->eng.set_profile(on != 0);
}

kf_status kf_batch_stage_times(kf_batch* b, float ms[4]) {
    if (!b || !ms) return KF_ERR_ARG;
    return b->eng.stage_times(ms);
}

kf_status kf_selftest_bounded_wait(int timeout_ms, int* waited_ms) {
    if (timeout_ms <= 0 || timeout_ms > 5000) return KF_ERR_ARG;
    GridSync* g = nullptr;
    int* res = nullptr;
    KF_CK(cudaMalloc(&g, sizeof(GridSync)));
    cudaError_t e = cudaMalloc(&res, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(g, 0, sizeof(GridSync));
    if (e == cudaSuccess) e = cudaMemset(res, 0xff, sizeof(int));
    const double t0 = now_ms();
    if (e == cudaSuccess) e = launch_barrier_selftest(g, (unsigned long long)timeout_ms * 1000000ull, res, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    const double t1 = now_ms();
    int h_res = -1;
    GridSync h_g{};
    if (e == cudaSuccess) e = cudaMemcpy(&h_res, res, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&h_g, g, sizeof(GridSync), cudaMemcpyDeviceToHost);
    cudaFree(g);
    cudaFree(res);
    KF_CK(e);
    if (waited_ms) *waited_ms = int(t1 - t0 + 0.5);
    if (h_res == 0 && h_g.abort && h_g.timeouts == 1) return KF_ERR_TIMEOUT;
    return h_res == 1 ? KF_OK : KF_ERR_STATE;
}

kf_status kf_measure_read_bandwidth(size_t bytes, int rounds, double* gbs) {
    if (!gbs || bytes < (size_t(16) << 20) || bytes > (size_t(4) << 30) || bytes % 16 || rounds < 1 || rounds > 1000)
        return KF_ERR_ARG;
    int dev = 0, sms = 0;
    KF_CK(cudaGetDevice(&dev));
    KF_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int grid = sms * 8;
    float4* buf = nullptr;
    float* sink = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaMalloc(&buf, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&sink, sizeof(float) * grid);
    if (e == cudaSuccess) e = cudaMemset(buf, 0, bytes);
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    const long long n4 = (long long)(bytes / 16);
    if (e == cudaSuccess) e = launch_read_probe(buf, n4, 1, sink, grid, 0);   // warm: the buffer into L2
    if (e == cudaSuccess) e = cudaEventRecord(a, 0);
    if (e == cudaSuccess) e = launch_read_probe(buf, n4, rounds, sink, grid, 0);
    if (e == cudaSuccess) e = cudaEventRecord(b, 0);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    cudaFree(buf);
    cudaFree(sink);
    KF_CK(e);
    *gbs = ms > 0.f ? double(bytes) * rounds / (double(ms) * 1e-3) / 1e9 : 0.0;
    return KF_OK;
}

}  // extern "C"
