// k_tsdf.cu -- TSDF volume: initialisation, projective fusion, brick minima, layout conversion.
//
// Reference: initializeGridKernel (project/src/tsdf.cu:7-18) and fuseKernel
// (project/src/tsdf.cu:20-75), which walks one (x, y) voxel column per thread through a
// cudaArray surface with 4-byte reads and writes.  Here the volume is two linear arrays in
// HBM (distance, weight; x fastest) and a warp owns a 32 x VEC-voxel segment of an x row:
// 4 voxels per lane for float/float, 8 for fp16/uint16, moved with 16-byte vectors.
//   - A segment whose two end voxels project outside the view frustum on the same side is
//     skipped whole: depth and image coordinates are monotone along the row, so no voxel
//     between them can pass the reference's frustum test.
//   - A lane projects its voxels, issues all their depth-map gathers together, and touches
//     the volume only when one of them updates.
//   - Every updated voxel marks its 8^3 brick (and the brick whose one-voxel apron it is)
//     dirty; a second kernel refreshes those bricks' minimum distance for the raycaster.
// Segments of every session of a batch are handed to persistent warps through one atomic
// counter.
#include "kf_host.h"

namespace kf {

int fuse_vec(int fmt) { return fmt == KF_TSDF_F16U16 ? 8 : 4; }
int fuse_segs_per_row(int n, int fmt) {
    const int span = 32 * fuse_vec(fmt);
    return (n + span - 1) / span;
}

// per-warp fusion context (shared memory): the session's camera and volume for the segment
struct FuseCtx {
    float iR[9], it[3];          // world -> camera
    float fx, fy, cx, cy, min_d, max_d, mu, max_w;
    const float* depth;          // unfiltered metres map
    const float* dmax;           // per 16x16 tile: largest valid depth (null: not available)
    int t16w, t16h;
    int w, h, n, nb;
    void* F;
    void* W;
    const float* xs;
    const float* zs;
    uint8_t* dirty;              // null: no brick bookkeeping (stage calls)
};

// running weighted average (project/src/tsdf.cu:56-69); max_w > 0 clamps the weight
__device__ __forceinline__ void fuse_update(float& F, float& Wt, float fn, float wn, float max_w) {
    F = (F * Wt + fn * wn) / (Wt + wn);
    float w1 = Wt + wn;
    if (max_w > 0.0f) w1 = fminf(w1, max_w);
    Wt = w1;
}

__device__ __forceinline__ void mark_dirty(const FuseCtx& c, int x0, int j, int k) {
    const int nb = c.nb;
    const int bx = x0 >> 3, by = j >> 3, bz = k >> 3;
    const int bx0 = ((x0 & 7) == 0 && bx > 0) ? bx - 1 : bx;
    const int by0 = ((j & 7) == 0 && by > 0) ? by - 1 : by;
    const int bz0 = ((k & 7) == 0 && bz > 0) ? bz - 1 : bz;
    for (int zz = bz0; zz <= bz; ++zz)
        for (int yy = by0; yy <= by; ++yy)
            for (int xx = bx0; xx <= bx; ++xx) c.dirty[(size_t(zz) * nb + yy) * nb + xx] = 1;
}

// One segment of row (j, k): voxels [seg * 32 * VEC, (seg + 1) * 32 * VEC) of the row.
template <int VEC, class TF, class TW>
__device__ __forceinline__ void fuse_segment(const FuseCtx& c, int j, int k, int seg, int lane) {
    const int n = c.n;
    const float y = __ldg(c.xs + j), z = __ldg(c.zs + k);
    // row-constant part of the world -> camera transform
    const F3 b{c.iR[3] * y + c.iR[6] * z + c.it[0], c.iR[4] * y + c.iR[7] * z + c.it[1],
               c.iR[5] * y + c.iR[8] * z + c.it[2]};
    // warp-uniform frustum test of the segment's end voxels
    {
        const int s0 = seg * 32 * VEC, s1 = min(n, (seg + 1) * 32 * VEC) - 1;
        const float xa = __ldg(c.xs + s0), xb = __ldg(c.xs + s1);
        const float za = c.iR[2] * xa + b.z, zb = c.iR[2] * xb + b.z;
        if (fmaxf(za, zb) < c.min_d - 1e-4f || fminf(za, zb) >= c.max_d + 1e-4f) return;
        if (fminf(za, zb) > 1e-3f) {
            const float pxa = (c.fx * (c.iR[0] * xa + b.x) + c.cx * za) / za;
            const float pxb = (c.fx * (c.iR[0] * xb + b.x) + c.cx * zb) / zb;
            if (fmaxf(pxa, pxb) < -0.01f || fminf(pxa, pxb) > float(c.w) + 0.01f) return;
            const float pya = (c.fy * (c.iR[1] * xa + b.y) + c.cy * za) / za;
            const float pyb = (c.fy * (c.iR[1] * xb + b.y) + c.cy * zb) / zb;
            if (fmaxf(pya, pyb) < -0.01f || fminf(pya, pyb) > float(c.h) + 0.01f) return;
            if (c.dmax) {
                // The voxels project onto the image segment between the two end pixels, so
                // onto its bounding box of 16x16 tiles.  With D the largest valid depth there,
                // a voxel either meets no valid depth or has diff <= D - z: nothing updates
                // when D = 0 or when every voxel lies more than mu behind D.
                const int tx0 = min(max(int(fminf(pxa, pxb) - 0.01f), 0), c.w - 1) >> 4;
                const int tx1 = min(max(int(fmaxf(pxa, pxb) + 0.01f), 0), c.w - 1) >> 4;
                const int ty0 = min(max(int(fminf(pya, pyb) - 0.01f), 0), c.h - 1) >> 4;
                const int ty1 = min(max(int(fmaxf(pya, pyb) + 0.01f), 0), c.h - 1) >> 4;
                const int nx = tx1 - tx0 + 1, ntile = nx * (ty1 - ty0 + 1);
                if (ntile <= 256) {
                    float dm = 0.0f;
                    for (int q = lane; q < ntile; q += 32)
                        dm = fmaxf(dm, __ldg(c.dmax + size_t(ty0 + q / nx) * c.t16w + tx0 + q % nx));
#pragma unroll
                    for (int off = 16; off >= 1; off >>= 1) dm = fmaxf(dm, __shfl_xor_sync(0xffffffffu, dm, off));
                    if (dm == 0.0f || fminf(za, zb) > dm + c.mu + 1e-4f) return;
                }
            }
        }
    }
    const int x0 = seg * 32 * VEC + lane * VEC;
    if (x0 >= n) return;
    float xv[VEC];
#pragma unroll
    for (int q = 0; q < VEC; q += 4) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(c.xs + x0 + q));
        xv[q] = t.x; xv[q + 1] = t.y; xv[q + 2] = t.z; xv[q + 3] = t.w;
    }
    // project (fuseKernel steps 1-2, project/src/tsdf.cu:33-44)
    int pix[VEC];
    float pz[VEC];
    unsigned int cand = 0;
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
        const float ex = c.iR[0] * xv[v] + b.x, ey = c.iR[1] * xv[v] + b.y, ez = c.iR[2] * xv[v] + b.z;
        const float iz = 1.0f / ez;
        const float px = (c.fx * ex + c.cx * ez) * iz;
        const float py = (c.fy * ey + c.cy * ez) * iz;
        pz[v] = ez;
        pix[v] = 0;
        if (ez >= c.min_d && ez < c.max_d && px >= 0.0f && px < float(c.w) && py >= 0.0f && py < float(c.h)) {
            pix[v] = int(py) * c.w + int(px);
            cand |= 1u << v;
        }
    }
    if (!cand) return;
    // nearest-pixel depth (step 3), all gathers in flight together
    float d[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) d[v] = (cand & (1u << v)) ? __ldg(c.depth + pix[v]) : 0.0f;
    float fn[VEC], wn[VEC];
    unsigned int upd = 0;
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
        fn[v] = 0.f;
        wn[v] = 0.f;
        if (!(cand & (1u << v)) || !depth_valid(d[v])) continue;
        const float diff = d[v] - pz[v];
        if (diff >= -c.mu) {   // step 4
            fn[v] = fminf(1.0f, diff / c.mu);
            wn[v] = 1.0f / d[v];
            upd |= 1u << v;
        }
    }
    if (!upd) return;
    // step 5: read-modify-write of the voxels that update
    const size_t base = (size_t(k) * n + j) * n + x0;
    if constexpr (VEC == 4) {
        float4* fp = reinterpret_cast<float4*>(static_cast<float*>(c.F) + base);
        float4* wp = reinterpret_cast<float4*>(static_cast<float*>(c.W) + base);
        const float4 fq = *fp, wq = *wp;
        float fa[4] = {fq.x, fq.y, fq.z, fq.w}, wa[4] = {wq.x, wq.y, wq.z, wq.w};
#pragma unroll
        for (int v = 0; v < 4; ++v)
            if (upd & (1u << v)) fuse_update(fa[v], wa[v], fn[v], wn[v], c.max_w);
        *fp = make_float4(fa[0], fa[1], fa[2], fa[3]);
        *wp = make_float4(wa[0], wa[1], wa[2], wa[3]);
    } else {
        uint4* fp = reinterpret_cast<uint4*>(static_cast<__half*>(c.F) + base);
        uint4* wp = reinterpret_cast<uint4*>(static_cast<uint16_t*>(c.W) + base);
        uint4 fq = *fp, wq = *wp;
        __half* fh = reinterpret_cast<__half*>(&fq);
        uint16_t* wh = reinterpret_cast<uint16_t*>(&wq);
#pragma unroll
        for (int v = 0; v < 8; ++v)
            if (upd & (1u << v)) {
                float f0 = __half2float(fh[v]);
                float w0 = float(wh[v]) * (1.0f / KF_WEIGHT_SCALE);
                fuse_update(f0, w0, fn[v], wn[v], c.max_w);
                fh[v] = __float2half_rn(f0);
                wh[v] = uint16_t(fminf(rintf(w0 * KF_WEIGHT_SCALE), 65535.0f));
            }
        *fp = fq;
        *wp = wq;
    }
    if (c.dirty) mark_dirty(c, x0, j, k);
}

template <int VEC, class TF, class TW>
__device__ __forceinline__ void fuse_segment_index(const FuseCtx& c, long long seg_local, int lane) {
    const int spr = (c.n + 32 * VEC - 1) / (32 * VEC);
    const long long row = seg_local / spr;
    const int seg = int(seg_local - row * spr);
    fuse_segment<VEC, TF, TW>(c, int(row % c.n), int(row / c.n), seg, lane);
}

__device__ void load_ctx(const SessionDev* S, FuseCtx& c) {
    const PoseDev* P = S->pose;
    for (int q = 0; q < 9; ++q) c.iR[q] = P->iRf[q];
    for (int q = 0; q < 3; ++q) c.it[q] = P->itf[q];
    c.fx = S->lv[0].fx; c.fy = S->lv[0].fy; c.cx = S->lv[0].cx; c.cy = S->lv[0].cy;
    c.min_d = S->min_d; c.max_d = S->max_d; c.mu = S->mu; c.max_w = S->max_w;
    c.depth = S->depth_m;
    c.dmax = S->dmax16;
    c.t16w = S->t16w; c.t16h = S->t16h;
    c.w = S->W; c.h = S->H; c.n = S->n; c.nb = S->nb;
    c.F = S->tf; c.W = S->tw; c.xs = S->xs; c.zs = S->zs; c.dirty = S->dirty;
}

constexpr int kFuseChunk = 4;   // segments a warp takes per atomic
constexpr int kFuseWarps = 8;

__global__ void __launch_bounds__(256, 4) fuse_kernel(EngineView v) {
    __shared__ FuseCtx ctx[kFuseWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long total = v.tb->fuse_total;
    const int S_cap = v.tb->S;
    unsigned long long* ctr = reinterpret_cast<unsigned long long*>(v.counters + 2);
    FuseCtx& c = ctx[warp];
    int cur_s = -1;
    bool live = false;
    while (true) {
        unsigned long long g0 = 0;
        if (lane == 0) g0 = atomicAdd(ctr, (unsigned long long)kFuseChunk);
        g0 = __shfl_sync(0xffffffffu, g0, 0);
        if ((long long)g0 >= total) break;
        for (int q = 0; q < kFuseChunk; ++q) {
            const long long g = (long long)g0 + q;
            if (g >= total) break;
            int lo = 0, hi = S_cap;   // session of segment g (warp-uniform binary search)
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (__ldg(v.fuse_prefix + mid) <= g) lo = mid; else hi = mid;
            }
            if (lo != cur_s) {
                cur_s = lo;
                const SessionDev* S = &v.sess[lo];
                live = v.step[lo].active && S->pose->fuse_ok;
                __syncwarp();
                if (live && lane == 0) load_ctx(S, c);
                __syncwarp();
            }
            if (!live) continue;
            const long long local = g - __ldg(v.fuse_prefix + lo);
            if (v.sess[lo].fmt == KF_TSDF_F16U16)
                fuse_segment_index<8, __half, uint16_t>(c, local, lane);
            else
                fuse_segment_index<4, float, float>(c, local, lane);
        }
    }
}

cudaError_t launch_fuse(const EngineView& v, int grid, cudaStream_t st) {
    fuse_kernel<<<grid, 256, 0, st>>>(v);
    return cudaGetLastError();
}

// ---- brick minima ----

// min over the 9 x 9 x 9 voxels [8b, 8b + 8] (clamped) of brick (bx, by, bz); one warp
template <class TF>
__device__ __forceinline__ float brick_min(const TF* f, int n, int bx, int by, int bz, int lane) {
    float m = 3.0e38f;
    for (int q = lane; q < 729; q += 32) {
        const int dx = q % 9, dy = (q / 9) % 9, dz = q / 81;
        const int x = min(bx * 8 + dx, n - 1), y = min(by * 8 + dy, n - 1), z = min(bz * 8 + dz, n - 1);
        m = fminf(m, load_f(f, (size_t(z) * n + y) * n + x));
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, off));
    return m;
}

// persistent warps take 32 bricks at a time, recompute the dirty ones, clear their flags
__global__ void __launch_bounds__(256) brick_kernel(EngineView v) {
    const int lane = threadIdx.x & 31;
    const long long total = v.tb->brick_total;
    const int S_cap = v.tb->S;
    unsigned long long* ctr = reinterpret_cast<unsigned long long*>(v.counters + 4);
    while (true) {
        unsigned long long g0 = 0;
        if (lane == 0) g0 = atomicAdd(ctr, 32ull);
        g0 = __shfl_sync(0xffffffffu, g0, 0);
        if ((long long)g0 >= total) break;
        const long long g = (long long)g0 + lane;
        int s = -1;
        long long local = 0;
        bool dirty = false;
        if (g < total) {
            int lo = 0, hi = S_cap;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (__ldg(v.brick_prefix + mid) <= g) lo = mid; else hi = mid;
            }
            s = lo;
            local = g - __ldg(v.brick_prefix + lo);
            const SessionDev* S = &v.sess[s];
            dirty = v.step[s].active && S->dirty[local] != 0;
        }
        unsigned int mask = __ballot_sync(0xffffffffu, dirty);
        while (mask) {
            const int src = __ffs(mask) - 1;
            mask &= mask - 1;
            const int ss = __shfl_sync(0xffffffffu, s, src);
            const long long bl = __shfl_sync(0xffffffffu, local, src);
            const SessionDev* S = &v.sess[ss];
            const int nb = S->nb;
            const int bx = int(bl % nb), by = int((bl / nb) % nb), bz = int(bl / ((long long)nb * nb));
            const float m = S->fmt == KF_TSDF_F16U16
                                ? brick_min(static_cast<const __half*>(S->tf), S->n, bx, by, bz, lane)
                                : brick_min(static_cast<const float*>(S->tf), S->n, bx, by, bz, lane);
            if (lane == 0) {
                S->bmin[bl] = m;
                S->dirty[bl] = 0;
            }
        }
    }
}

cudaError_t launch_bricks(const EngineView& v, int grid, cudaStream_t st) {
    brick_kernel<<<grid, 256, 0, st>>>(v);
    return cudaGetLastError();
}

__global__ void init_bricks_kernel(float* bmin, uint8_t* dirty, long long nbricks) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nbricks; i += (long long)gridDim.x * blockDim.x) {
        bmin[i] = 2.0f;
        dirty[i] = 0;
    }
}

cudaError_t launch_init_bricks(float* bmin, uint8_t* dirty, long long nbricks, cudaStream_t st) {
    init_bricks_kernel<<<148 * 4, 256, 0, st>>>(bmin, dirty, nbricks);
    return cudaGetLastError();
}

template <class TF>
__global__ void rebuild_bricks_kernel(const TF* f, int n, float* bmin) {
    const int nb = n / 8;
    const long long total = (long long)nb * nb * nb;
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long b = warp; b < total; b += nwarps) {
        const float m = brick_min(f, n, int(b % nb), int((b / nb) % nb), int(b / ((long long)nb * nb)), lane);
        if (lane == 0) bmin[b] = m;
    }
}

cudaError_t launch_rebuild_bricks(const void* f, int fmt, int n, float* bmin, cudaStream_t st) {
    if (fmt == KF_TSDF_F16U16)
        rebuild_bricks_kernel<<<148 * 8, 256, 0, st>>>(static_cast<const __half*>(f), n, bmin);
    else
        rebuild_bricks_kernel<<<148 * 8, 256, 0, st>>>(static_cast<const float*>(f), n, bmin);
    return cudaGetLastError();
}

// ---- stage fusion on a caller volume (kernel::fuse) ----

template <int VEC, class TF, class TW>
__global__ void __launch_bounds__(256) fuse_stage_kernel(FuseCtx c) {
    const long long spr = (c.n + 32 * VEC - 1) / (32 * VEC);
    const long long total = (long long)c.n * c.n * spr;
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long g = warp; g < total; g += nwarps) fuse_segment_index<VEC, TF, TW>(c, g, lane);
}

cudaError_t stage_fuse(const float* depth, int w, int h, const float* k, const kf_volume* vol, const float* pose,
                       float min_d, float max_d, const float* xs, const float* zs, cudaStream_t st) {
    FuseCtx c;
    c.depth = depth;
    c.dmax = nullptr;
    c.t16w = c.t16h = 0;
    c.w = w;
    c.h = h;
    c.fx = k[0]; c.fy = k[4]; c.cx = k[6]; c.cy = k[7];
    c.min_d = min_d; c.max_d = max_d; c.mu = vol->mu; c.max_w = vol->max_weight;
    c.n = vol->n;
    c.nb = vol->n / 8;
    c.F = vol->f;
    c.W = vol->w;
    c.xs = xs;
    c.zs = zs;
    c.dirty = nullptr;
    // inverse of the rigid pose: R^T, -R^T t
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 3; ++row) c.iR[col * 3 + row] = pose[row * 4 + col];
    for (int row = 0; row < 3; ++row)
        c.it[row] = -(c.iR[row] * pose[12] + c.iR[3 + row] * pose[13] + c.iR[6 + row] * pose[14]);
    const int grid = 148 * 8;
    if (vol->format == KF_TSDF_F16U16)
        fuse_stage_kernel<8, __half, uint16_t><<<grid, 256, 0, st>>>(c);
    else
        fuse_stage_kernel<4, float, float><<<grid, 256, 0, st>>>(c);
    return cudaGetLastError();
}

// ---- initialisation {f = 2, w = 0} (project/src/voxel_grid.h:8-15) and layout conversion ----

__global__ void init_f32_kernel(float4* f, float4* w, long long nvec) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvec; i += (long long)gridDim.x * blockDim.x) {
        f[i] = make_float4(2.f, 2.f, 2.f, 2.f);
        w[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}
__global__ void init_f16_kernel(uint4* f, uint4* w, long long nvec) {
    const __half two = __float2half_rn(2.0f);
    const unsigned short tb = *reinterpret_cast<const unsigned short*>(&two);
    const unsigned int pair = (unsigned int)tb | ((unsigned int)tb << 16);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvec; i += (long long)gridDim.x * blockDim.x) {
        f[i] = make_uint4(pair, pair, pair, pair);
        w[i] = make_uint4(0u, 0u, 0u, 0u);
    }
}
__global__ void init_tail_kernel(void* f, void* w, long long start, long long nvox, int fmt) {
    for (long long i = start + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvox; i += (long long)gridDim.x * blockDim.x) {
        if (fmt == KF_TSDF_F16U16) {
            static_cast<__half*>(f)[i] = __float2half_rn(2.0f);
            static_cast<uint16_t*>(w)[i] = 0;
        } else {
            static_cast<float*>(f)[i] = 2.0f;
            static_cast<float*>(w)[i] = 0.0f;
        }
    }
}

cudaError_t launch_init_volume(void* f, void* w, long long nvox, int fmt, cudaStream_t st) {
    const int per = fmt == KF_TSDF_F16U16 ? 8 : 4;
    const long long nvec = nvox / per;
    const int grid = 148 * 8;
    if (nvec > 0) {
        if (fmt == KF_TSDF_F16U16)
            init_f16_kernel<<<grid, 256, 0, st>>>(static_cast<uint4*>(f), static_cast<uint4*>(w), nvec);
        else
            init_f32_kernel<<<grid, 256, 0, st>>>(static_cast<float4*>(f), static_cast<float4*>(w), nvec);
    }
    if (nvec * per < nvox) init_tail_kernel<<<1, 256, 0, st>>>(f, w, nvec * per, nvox, fmt);
    return cudaGetLastError();
}

__global__ void export_kernel(const void* f, const void* w, long long nvox, int fmt, float2* dst) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvox; i += (long long)gridDim.x * blockDim.x) {
        float a, b;
        if (fmt == KF_TSDF_F16U16) {
            a = __half2float(static_cast<const __half*>(f)[i]);
            b = float(static_cast<const uint16_t*>(w)[i]) * (1.0f / KF_WEIGHT_SCALE);
        } else {
            a = static_cast<const float*>(f)[i];
            b = static_cast<const float*>(w)[i];
        }
        dst[i] = make_float2(a, b);
    }
}

__global__ void import_kernel(const float2* src, void* f, void* w, long long nvox, int fmt) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvox; i += (long long)gridDim.x * blockDim.x) {
        const float2 v = src[i];
        if (fmt == KF_TSDF_F16U16) {
            static_cast<__half*>(f)[i] = __float2half_rn(v.x);
            static_cast<uint16_t*>(w)[i] = uint16_t(fminf(fmaxf(rintf(v.y * KF_WEIGHT_SCALE), 0.0f), 65535.0f));
        } else {
            static_cast<float*>(f)[i] = v.x;
            static_cast<float*>(w)[i] = v.y;
        }
    }
}

cudaError_t launch_export_interleaved(const void* f, const void* w, long long nvox, int fmt, float* dst, cudaStream_t st) {
    export_kernel<<<148 * 8, 256, 0, st>>>(f, w, nvox, fmt, reinterpret_cast<float2*>(dst));
    return cudaGetLastError();
}
cudaError_t launch_import_interleaved(const float* src, void* f, void* w, long long nvox, int fmt, cudaStream_t st) {
    import_kernel<<<148 * 8, 256, 0, st>>>(reinterpret_cast<const float2*>(src), f, w, nvox, fmt);
    return cudaGetLastError();
}

}  // namespace kf
