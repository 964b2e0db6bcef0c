// k_tsdf.cu -- TSDF volume: initialisation, projective fusion, brick bounds, layout conversion.
//
// Reference: initializeGridKernel (project/src/tsdf.cu:7-18) and fuseKernel
// (project/src/tsdf.cu:20-75), which walks one (x, y) voxel column per thread through a
// cudaArray surface with 4-byte reads and writes, projecting every voxel of the volume.
//
// Here the volume is two linear arrays in HBM (distance, weight; x fastest), cut into
// 32 x 8 x 8 voxel blocks.  Two launches per frame:
//   - fuse_cull_kernel tests every block of every session as a whole, one block per thread,
//     from its 8 projected corners (the projection of a box in front of the camera lies
//     inside its corners' bounding box): outside the depth range or the image, no valid depth
//     under it, or every voxel more than mu behind the farthest valid depth under it -- then
//     no voxel of it can update.  The surviving blocks (a few percent of a 512^3 volume) are
//     appended to a queue with one atomic per warp.
//   - fuse_kernel's persistent warps take queue entries whole, or in halves or quarters when
//     there are few, and walk the rows four at a time, each lane four consecutive voxels along
//     x, so the warp reads and writes the volume as 16-byte vectors in 128-byte rows.
// Each 8^3 brick keeps a lower bound of its distances (an atomic minimum of every value
// fusion stores), widened to the 2 x 2 x 2 bricks a trilinear sample can touch and to 32^3
// super-bricks; fusion lowers the widened bounds itself whenever a brick's bound falls, so no
// pass recomputes them.  The raycaster skips samples whose bound proves they cannot matter.
#include "kf_host.h"

namespace kf {

__host__ __device__ int fuse_units(int n) { return ((n + 31) / 32) * ((n + 7) / 8) * ((n + 7) / 8); }

// order-preserving int key of a float (atomicMin on floats of either sign)
__device__ __forceinline__ int fkey(float x) {
    const int i = __float_as_int(x);
    return i >= 0 ? i : (i ^ 0x7fffffff);
}

// per-warp fusion context (shared memory): the session's camera and volume
struct FuseCtx {
    float iR[9], it[3];          // world -> camera
    float fx, fy, cx, cy, min_d, max_d, mu, max_w;
    const float* depth;          // unfiltered metres map
    const float* dmax;           // per 16x16 tile: largest valid depth (null: not available)
    int t16w, t16h;
    int w, h, n, nb, fmt;
    void* F;
    void* W;
    const float* xs;
    const float* zs;
    int* bmin;                   // brick lower bounds (null: none kept)
    int* bdil;                   // their widenings to the bricks and super-bricks around them
    int* sdil;
    int ns;
};

// A brick's lower bound fell to key k: the widened bounds of every brick and super-brick whose
// neighbourhood holds the brick fall with it -- bdil of bricks b - {0,1}^3 (a brick's bdil
// covers {b, b+1}^3) and sdil of super-bricks s with 4 s <= b <= 4 s + 4 per axis.  Bounds only
// ever fall (atomic minima), so these running minima are exactly the minima over each
// neighbourhood.  Most calls find the bound already at or below k and stop at one load.
__device__ __forceinline__ void lower_brick_bound(const FuseCtx& c, int bx, int by, int bz, int k) {
    const int nb = c.nb;
    int* pb = c.bmin + (size_t(bz) * nb + by) * nb + bx;
    if (k >= __ldcg(pb)) return;          // a stale read is never below the bound
    if (k >= atomicMin(pb, k)) return;    // another warp lowered it as far already
#pragma unroll
    for (int d = 0; d < 8; ++d) {
        const int x = bx - (d & 1), y = by - ((d >> 1) & 1), z = bz - (d >> 2);
        if (x >= 0 && y >= 0 && z >= 0) atomicMin(c.bdil + (size_t(z) * nb + y) * nb + x, k);
    }
    const int ns = c.ns;
#pragma unroll
    for (int d = 0; d < 8; ++d) {
        // super-brick b / 4 per axis, and b / 4 - 1 when b is the last brick of its range too
        const int x = (bx >> 2) - (d & 1), y = (by >> 2) - ((d >> 1) & 1), z = (bz >> 2) - (d >> 2);
        const bool ok = ((d & 1) == 0 || ((bx & 3) == 0 && bx > 0)) && (((d >> 1) & 1) == 0 || ((by & 3) == 0 && by > 0)) &&
                        ((d >> 2) == 0 || ((bz & 3) == 0 && bz > 0));
        if (ok && x < ns && y < ns && z < ns) atomicMin(c.sdil + (size_t(z) * ns + y) * ns + x, k);
    }
}

// running weighted average (project/src/tsdf.cu:56-69, built with -use_fast_math: the
// division is the approximate one); max_w > 0 clamps the weight
__device__ __forceinline__ void fuse_update(float& F, float& Wt, float fn, float wn, float max_w) {
    F = __fdividef(__fmaf_rn(F, Wt, __fmul_rn(fn, wn)), __fadd_rn(Wt, wn));
    float w1 = __fadd_rn(Wt, wn);
    if (max_w > 0.0f) w1 = fminf(w1, max_w);
    Wt = w1;
}

// true when no voxel of the block [x0, x0+32) x [j0, j0+8) x [k0, k0+8) can update; one
// thread tests one block
__device__ __forceinline__ bool block_culled(const FuseCtx& c, int x0, int j0, int k0) {
    const int n = c.n;
    const float xa = __ldg(c.xs + x0), xb = __ldg(c.xs + min(x0 + 31, n - 1));
    const float ya = __ldg(c.xs + j0), yb = __ldg(c.xs + min(j0 + 7, n - 1));
    const float za = __ldg(c.zs + k0), zb = __ldg(c.zs + min(k0 + 7, n - 1));
    float ex[8], ey[8], ez[8];
    float zmin = 3.0e38f, zmax = -3.0e38f;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const float x = (q & 1) ? xb : xa, y = (q & 2) ? yb : ya, z = (q & 4) ? zb : za;
        // same operation order as the per-voxel projection below
        const float bx = c.iR[3] * y + c.iR[6] * z + c.it[0];
        const float by = c.iR[4] * y + c.iR[7] * z + c.it[1];
        const float bz = c.iR[5] * y + c.iR[8] * z + c.it[2];
        ex[q] = c.iR[0] * x + bx;
        ey[q] = c.iR[1] * x + by;
        ez[q] = c.iR[2] * x + bz;
        zmin = fminf(zmin, ez[q]);
        zmax = fmaxf(zmax, ez[q]);
    }
    if (zmax < c.min_d - 1e-4f || zmin >= c.max_d + 1e-4f) return true;
    if (!(zmin > 1e-3f)) return false;   // a corner behind the camera: no image bound
    float pxmin = 3.0e38f, pxmax = -3.0e38f, pymin = 3.0e38f, pymax = -3.0e38f;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        // approximate division (a few 1e-4 px at most): the bounds below keep 0.01 px margins
        const float px = __fdividef(c.fx * ex[q] + c.cx * ez[q], ez[q]);
        const float py = __fdividef(c.fy * ey[q] + c.cy * ez[q], ez[q]);
        pxmin = fminf(pxmin, px);
        pxmax = fmaxf(pxmax, px);
        pymin = fminf(pymin, py);
        pymax = fmaxf(pymax, py);
    }
    if (pxmax < -0.01f || pxmin > float(c.w) + 0.01f || pymax < -0.01f || pymin > float(c.h) + 0.01f) return true;
    if (!c.dmax) return false;
    const int tx0 = min(max(int(pxmin - 0.01f), 0), c.w - 1) >> 4;
    const int tx1 = min(max(int(pxmax + 0.01f), 0), c.w - 1) >> 4;
    const int ty0 = min(max(int(pymin - 0.01f), 0), c.h - 1) >> 4;
    const int ty1 = min(max(int(pymax + 0.01f), 0), c.h - 1) >> 4;
    if ((tx1 - tx0 + 1) * (ty1 - ty0 + 1) > 512) return false;
    float dm = 0.0f;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) dm = fmaxf(dm, __ldg(c.dmax + size_t(ty) * c.t16w + tx));
    // every voxel meets either an invalid depth or d - z <= dm - zmin < -mu
    return dm == 0.0f || zmin > dm + c.mu + 1e-4f;
}

// block coordinates of fusion unit u of an n^3 volume (units: 32 x 8 x 8 blocks, x fastest)
__device__ __forceinline__ void unit_origin(int n, int u, int& x0, int& j0, int& k0) {
    const int ux = (n + 31) >> 5, uy = (n + 7) >> 3;
    x0 = (u % ux) * 32;
    j0 = ((u / ux) % uy) * 8;
    k0 = (u / (ux * uy)) * 8;
}

// four consecutive voxels of a row as one vector: 16 bytes of f32, 8 bytes of f16 or u16
__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ uint2 ld4(const __half* p) { return *reinterpret_cast<const uint2*>(p); }
__device__ __forceinline__ uint2 ld4(const uint16_t* p) { return *reinterpret_cast<const uint2*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ void st4(__half* p, uint2 v) { *reinterpret_cast<uint2*>(p) = v; }
__device__ __forceinline__ void st4(uint16_t* p, uint2 v) { *reinterpret_cast<uint2*>(p) = v; }
// component q of a 4-vector (q a compile-time constant after unrolling)
__device__ __forceinline__ float& comp(float4& v, int q) { return q == 0 ? v.x : q == 1 ? v.y : q == 2 ? v.z : v.w; }

// fuseKernel (project/src/tsdf.cu:28-74) for rows [r_begin, r_end) of one block (row r is
// y = j0 + r % 8, z = k0 + r / 8; n is a multiple of 8, so every block has 64 rows).  A warp
// takes four rows per step: lanes 8 q .. 8 q + 7 row r0 + q, each lane four consecutive voxels
// along x, so the warp reads and writes the volume as four 128-byte rows of 16-byte (f32) or
// 8-byte (f16, u16) vectors.  A vector whose voxels all stay unchanged is not touched; voxels
// that stay unchanged inside a written vector are written back with their own bits.
template <class TF, class TW>
__device__ __forceinline__ void fuse_block(const FuseCtx& c, int x0, int j0, int k0, int r_begin, int r_end, int lane) {
    const int n = c.n;
    const int sub = lane >> 3;
    const int x = x0 + 4 * (lane & 7);   // the first of this lane's four voxels
    const bool lane_in = x < n;            // n % 8 == 0: all four voxels or none
    float xv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) xv[q] = __ldg(c.xs + min(x + q, n - 1));
    const int rows = min(r_end, 64);
    int kmin = 0x7fffffff;   // key of the smallest distance this lane stores
    TF* F = static_cast<TF*>(c.F);
    TW* Wa = static_cast<TW*>(c.W);
    for (int r0 = r_begin; r0 < rows; r0 += 4) {
        const int r = r0 + sub;
        const bool row_in = lane_in && r < rows;
        const int j = j0 + (r & 7), k = k0 + (r >> 3);
        int pix[4];
        float pz[4], d[4];
        unsigned int cand = 0;
        // The f16+u16 form (the batched one) prefetches the lane's volume vectors to L2 while
        // the row is projected and its depths gathered, so a row that updates reads them from
        // L2 instead of DRAM: +0.6 % for 32 sessions.  In the f32 form (one session's quarter
        // blocks) it gained nothing: there the longer-lived address cost 0.5 %.
        if (sizeof(TF) == 2 && row_in) {
            const size_t at = (size_t(k) * n + j) * n + x;
            asm volatile("prefetch.global.L2 [%0];" :: "l"(F + at));
            asm volatile("prefetch.global.L2 [%0];" :: "l"(Wa + at));
        }
        // project (steps 1-2)
        if (row_in) {
            const float y = __ldg(c.xs + j), z = __ldg(c.zs + k);
            const float bx = c.iR[3] * y + c.iR[6] * z + c.it[0];
            const float by = c.iR[4] * y + c.iR[7] * z + c.it[1];
            const float bz = c.iR[5] * y + c.iR[8] * z + c.it[2];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float ex = c.iR[0] * xv[q] + bx, ey = c.iR[1] * xv[q] + by, ez = c.iR[2] * xv[q] + bz;
                // pixel /= pixel.z: the reference's build divides approximately, but rounded
                // division here keeps the per-frame pose within 2e-6 rad of the FP64 oracle
                // (1e-4 with the approximate one: voxels near a pixel edge change pixel)
                const float iz = 1.0f / ez;
                const float px = (c.fx * ex + c.cx * ez) * iz;
                const float py = (c.fy * ey + c.cy * ez) * iz;
                pz[q] = ez;
                pix[q] = 0;
                if (ez >= c.min_d && ez < c.max_d && px >= 0.0f && px < float(c.w) && py >= 0.0f && py < float(c.h)) {
                    pix[q] = int(py) * c.w + int(px);
                    cand |= 1u << q;
                }
            }
        }
        // nearest-pixel depth (step 3), four gathers in flight
#pragma unroll
        for (int q = 0; q < 4; ++q) d[q] = (cand & (1u << q)) ? __ldg(c.depth + pix[q]) : 0.0f;
        float fn[4], wn[4];
        unsigned int upd = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            fn[q] = wn[q] = 0.f;
            if (!(cand & (1u << q)) || !depth_valid(d[q])) continue;
            const float diff = d[q] - pz[q];
            if (diff >= -c.mu) {   // step 4 (the reference divides with -use_fast_math)
                fn[q] = fminf(1.0f, __fdividef(diff, c.mu));
                wn[q] = __fdividef(1.0f, d[q]);   // its 1 / depth is the fast reciprocal too
                upd |= 1u << q;
            }
        }
        if (!__any_sync(0xffffffffu, upd != 0)) continue;
        if (!upd) continue;
        // step 5: one vector read-modify-write of the lane's four voxels
        const size_t idx = (size_t(k) * n + j) * n + x;
        if constexpr (sizeof(TF) == 4) {
            float4 fv = ld4(F + idx), wv = ld4(Wa + idx);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (!(upd & (1u << q))) continue;
                float f0 = comp(fv, q), w0 = comp(wv, q);
                fuse_update(f0, w0, fn[q], wn[q], c.max_w);
                comp(fv, q) = f0;
                comp(wv, q) = w0;
                kmin = min(kmin, fkey(f0));
            }
            st4(F + idx, fv);
            st4(Wa + idx, wv);
        } else {
            uint2 fv = ld4(F + idx), wv = ld4(Wa + idx);
            // All four voxels are decoded and encoded again, the unchanged ones exactly: an fp16
            // value survives float and back, and a weight u / 1024 survives the scaling by a
            // power of two.  The weight steps u < 2^16 become floats as the float 2^23 + u
            // (bits 0x4B000000 | u) less 2^23, and return as the low bits of x + 2^23, whose
            // round-to-nearest-even addition is rintf(x) for 0 <= x < 2^22: exact, without
            // conversion instructions.
            static_assert(KF_WEIGHT_SCALE == 1024.0f, "weights are steps of 1 / 1024");
            const float2 f01 = __half22float2(*reinterpret_cast<const __half2*>(&fv.x));
            const float2 f23 = __half22float2(*reinterpret_cast<const __half2*>(&fv.y));
            float f[4] = {f01.x, f01.y, f23.x, f23.y}, w[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const unsigned int bits = __byte_perm(q < 2 ? wv.x : wv.y, 0x4B000000u, (q & 1) ? 0x7632 : 0x7610);
                w[q] = __fmul_rn(__fsub_rn(__uint_as_float(bits), 8388608.0f), 1.0f / KF_WEIGHT_SCALE);
                if (upd & (1u << q)) fuse_update(f[q], w[q], fn[q], wn[q], c.max_w);
            }
            const __half2 h01 = __floats2half2_rn(f[0], f[1]), h23 = __floats2half2_rn(f[2], f[3]);
            fv.x = *reinterpret_cast<const unsigned int*>(&h01);
            fv.y = *reinterpret_cast<const unsigned int*>(&h23);
            unsigned int wb[4];
#pragma unroll
            for (int q = 0; q < 4; ++q)
                wb[q] = __float_as_uint(__fadd_rn(fminf(__fmul_rn(w[q], KF_WEIGHT_SCALE), 65535.0f), 8388608.0f));
            wv.x = __byte_perm(wb[0], wb[1], 0x5410);
            wv.y = __byte_perm(wb[2], wb[3], 0x5410);
            const float2 r01 = __half22float2(h01), r23 = __half22float2(h23);
            const float r[4] = {r01.x, r01.y, r23.x, r23.y};
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (upd & (1u << q)) kmin = min(kmin, fkey(r[q]));
            st4(F + idx, fv);
            st4(Wa + idx, wv);
        }
    }
    if (c.bmin) {
        // a lane's voxels sit in brick (x >> 3, j0 >> 3, k0 >> 3): reduce over the lanes of the
        // same brick (lane pairs along x, the four row groups), one atomic per brick
        kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, 1));
        kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, 8));
        kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, 16));
        if ((lane & 0x19) == 0 && kmin != 0x7fffffff && lane_in) lower_brick_bound(c, x >> 3, j0 >> 3, k0 >> 3, kmin);
    }
}

__device__ __forceinline__ void fuse_rows(const FuseCtx& c, int x0, int j0, int k0, int r_begin, int r_end, int lane) {
    if (c.fmt == KF_TSDF_F16U16)
        fuse_block<__half, uint16_t>(c, x0, j0, k0, r_begin, r_end, lane);
    else
        fuse_block<float, float>(c, x0, j0, k0, r_begin, r_end, lane);
}

// the fusion context of a session's tracking volume, or of its visualization volume (kVis):
// the same depth map and pose, the other grid
template <bool kVis>
__device__ void load_ctx(const SessionDev* S, FuseCtx& c) {
    const PoseDev* P = S->pose;
    for (int q = 0; q < 9; ++q) c.iR[q] = P->iRf[q];
    for (int q = 0; q < 3; ++q) c.it[q] = P->itf[q];
    c.fx = S->lv[0].fx; c.fy = S->lv[0].fy; c.cx = S->lv[0].cx; c.cy = S->lv[0].cy;
    c.min_d = S->min_d; c.max_d = S->max_d; c.max_w = S->max_w;
    c.depth = S->depth_m;
    c.dmax = S->dmax16;
    c.t16w = S->t16w; c.t16h = S->t16h;
    c.w = S->W; c.h = S->H; c.fmt = S->fmt;
    if (kVis) {
        const VisDev& V = S->vis;
        c.mu = V.mu; c.n = V.n; c.nb = V.nb; c.ns = V.ns;
        c.F = V.tf; c.W = V.tw; c.xs = V.xs; c.zs = V.zs; c.bmin = V.bmin; c.bdil = V.bdil; c.sdil = V.sdil;
    } else {
        c.mu = S->mu; c.n = S->n; c.nb = S->nb; c.ns = S->ns;
        c.F = S->tf; c.W = S->tw; c.xs = S->xs; c.zs = S->zs; c.bmin = S->bmin; c.bdil = S->bdil; c.sdil = S->sdil;
    }
}

// which tables a fusion launch walks: the tracking volumes' or the visualization volumes'
template <bool kVis> struct FuseLists;
template <> struct FuseLists<false> {
    static __device__ long long total(const EngineView& v) { return v.tb->fuse_total; }
    static __device__ const long long* prefix(const EngineView& v) { return v.fuse_prefix; }
    static __device__ unsigned int* queue(const EngineView& v) { return v.fuseq; }
    static __device__ int queue_cap(const EngineView& v) { return v.fuseq_cap; }
    static constexpr int kQueued = 4, kTaken = 5;   // counters
};
template <> struct FuseLists<true> {
    static __device__ long long total(const EngineView& v) { return v.tb->vis_fuse_total; }
    static __device__ const long long* prefix(const EngineView& v) { return v.vis_fuse_prefix; }
    static __device__ unsigned int* queue(const EngineView& v) { return v.vis_fuseq; }
    static __device__ int queue_cap(const EngineView& v) { return v.vis_fuseq_cap; }
    static constexpr int kQueued = 8, kTaken = 9;
};

// session of global fusion unit g (binary search over the per-slot prefix)
__device__ __forceinline__ int unit_session(const long long* prefix, long long g, int S_cap) {
    int lo = 0, hi = S_cap;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(prefix + mid) <= g) lo = mid; else hi = mid;
    }
    return lo;
}

// one thread per block of every stepping session: append the blocks that can update to the
// queue (counters[4] = entries; [8] for the visualization volumes), one atomic per warp
template <bool kVis>
__global__ void __launch_bounds__(256, 4) fuse_cull_kernel(EngineView v) {
    using Lists = FuseLists<kVis>;
    const long long total = Lists::total(v);
    const long long* prefix = Lists::prefix(v);
    unsigned int* queue = Lists::queue(v);
    const int queue_cap = Lists::queue_cap(v);
    const int S_cap = v.tb->S;
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x;
    FuseCtx c;
    int cur_s = -1;
    bool live = false;
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < total; base += stride) {
        const long long g = base + lane;
        bool keep = false;
        if (g < total) {
            const int s = unit_session(prefix, g, S_cap);
            if (s != cur_s) {
                cur_s = s;
                const SessionDev* S = &v.sess[s];
                live = v.step[s].active && S->pose->fuse_ok;
                if (live) load_ctx<kVis>(S, c);
            }
            if (live) {
                int x0, j0, k0;
                unit_origin(c.n, int(g - __ldg(prefix + s)), x0, j0, k0);
                keep = !block_culled(c, x0, j0, k0);
            }
        }
        const unsigned int m = __ballot_sync(0xffffffffu, keep);
        if (m == 0) continue;
        unsigned int slot = 0;
        if (lane == 0) slot = atomicAdd(&v.counters[Lists::kQueued], unsigned(__popc(m)));
        slot = __shfl_sync(0xffffffffu, slot, 0);
        const unsigned int at = slot + __popc(m & ((1u << lane) - 1u));
        if (keep && at < unsigned(queue_cap)) queue[at] = unsigned(g);   // capacity >= all blocks
    }
}

constexpr int kFuseWarps = 8;

// Queue entries are taken whole (64 rows) when there are at least eight per warp of the grid
// (a batch), in halves from four per warp, and in quarters below that (a single session's
// frame), so every warp has work and few entries pay the per-entry set-up.  Which warp fuses
// which rows changes no voxel's arithmetic.
__device__ __forceinline__ int fuse_split(unsigned int blocks) {
    const unsigned int warps = gridDim.x * kFuseWarps;
    return blocks >= 8u * warps ? 1 : blocks >= 4u * warps ? 2 : 4;
}

template <bool kVis>
__global__ void __launch_bounds__(256, 4) fuse_kernel(EngineView v) {
    using Lists = FuseLists<kVis>;
    __shared__ FuseCtx ctx[kFuseWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int S_cap = v.tb->S;
    const long long* prefix = Lists::prefix(v);
    const unsigned int* queue = Lists::queue(v);
    const unsigned int blocks = min(__ldcg(&v.counters[Lists::kQueued]), unsigned(Lists::queue_cap(v)));
    const int split = v.tb->fuse_split ? v.tb->fuse_split : fuse_split(blocks), rows = 64 / split;
    const unsigned int items = blocks * unsigned(split);
    FuseCtx& c = ctx[warp];
    int cur_s = -1;
    while (true) {
        unsigned int i = 0;
        if (lane == 0) i = atomicAdd(&v.counters[Lists::kTaken], 1u);
        i = __shfl_sync(0xffffffffu, i, 0);
        if (i >= items) break;
        const long long g = __ldcg(queue + i / unsigned(split));
        const int part = int(i % unsigned(split));
        const int s = unit_session(prefix, g, S_cap);
        if (s != cur_s) {
            cur_s = s;
            __syncwarp();
            if (lane == 0) load_ctx<kVis>(&v.sess[s], c);
            __syncwarp();
        }
        int x0, j0, k0;
        unit_origin(c.n, int(g - __ldg(prefix + s)), x0, j0, k0);
        fuse_rows(c, x0, j0, k0, part * rows, (part + 1) * rows, lane);
    }
}

cudaError_t launch_fuse(const EngineView& v, int grid, cudaStream_t st) {
    const int cull_grid = grid;   // grid-stride over all blocks of all sessions
    fuse_cull_kernel<false><<<cull_grid, 256, 0, st>>>(v);
    fuse_kernel<false><<<grid, 256, 0, st>>>(v);
    return cudaGetLastError();
}

cudaError_t launch_fuse_vis(const EngineView& v, int grid, cudaStream_t st) {
    fuse_cull_kernel<true><<<grid, 256, 0, st>>>(v);
    fuse_kernel<true><<<grid, 256, 0, st>>>(v);
    return cudaGetLastError();
}

// ---- brick bounds ----
//
// bmin: lower bound of each 8^3 brick's distances (fusion's atomic minima).
// bdil: bmin widened to bricks {b, b+1}^3 (clamped), every brick a trilinear sample whose base
//       voxel lies in brick b can touch; the raycaster's brick-level skip test reads it.
// sdil: the same for 32^3 super-bricks: the minimum of bmin over bricks [4s, 4s + 4] per axis.
//       The raycaster reads the two small arrays (sdil stays in L1) to skip samples.
// Fusion keeps bdil and sdil equal to these minima as it lowers bmin (lower_brick_bound); the
// kernels below compute them from scratch after a volume is loaded.

__device__ __forceinline__ int large_key() { return __float_as_int(0.991f); }

// bdil[b] = min of bmin over bricks {b, b+1}^3 (clamped); nb^3 < 2^31, so 32-bit indices
__device__ __forceinline__ void dilate_brick(const int* __restrict__ m, int* bdil, int nb, int b) {
    const int bx = b % nb, byz = b / nb, by = byz % nb, bz = byz / nb;
    const int dx = bx + 1 < nb ? 1 : 0, dy = by + 1 < nb ? nb : 0, dz = bz + 1 < nb ? nb * nb : 0;
    const int* p = m + b;
    int k = min(min(__ldg(p), __ldg(p + dx)), min(__ldg(p + dy), __ldg(p + dy + dx)));
    k = min(k, min(min(__ldg(p + dz), __ldg(p + dz + dx)), min(__ldg(p + dz + dy), __ldg(p + dz + dy + dx))));
    bdil[b] = k;
}

// sdil of super-brick (sx, sy, sz): min of bmin over bricks [4s, 4s + 4] per axis (clamped),
// one warp
__device__ __forceinline__ int superbrick_bound(const int* bmin, int nb, int sx, int sy, int sz, int lane) {
    const int x0 = 4 * sx, y0 = 4 * sy, z0 = 4 * sz;
    int k = 0x7fffffff;
    for (int q = lane; q < 125; q += 32) {
        const int x = min(x0 + q % 5, nb - 1), y = min(y0 + (q / 5) % 5, nb - 1), z = min(z0 + q / 25, nb - 1);
        k = min(k, __ldg(bmin + (size_t(z) * nb + y) * nb + x));
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) k = min(k, __shfl_xor_sync(0xffffffffu, k, off));
    return k;
}

__global__ void fill_key_kernel(int* a, long long count, int key) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x)
        a[i] = key;
}

cudaError_t launch_init_bricks(int* bmin, int* bdil, int* sdil, int n, cudaStream_t st) {
    const int nb = n / 8, ns = (nb + 3) / 4;
    const long long nbricks = (long long)nb * nb * nb, nsuper = (long long)ns * ns * ns;
    const int k2 = 0x40000000;   // key of 2.0f (bits of a positive float)
    fill_key_kernel<<<148 * 4, 256, 0, st>>>(bmin, nbricks, k2);
    fill_key_kernel<<<148 * 4, 256, 0, st>>>(bdil, nbricks, k2);
    fill_key_kernel<<<148, 256, 0, st>>>(sdil, nsuper, k2);
    return cudaGetLastError();
}

// exact minimum over each brick's own 8^3 voxels (after a volume load), one warp per brick
template <class TF>
__global__ void rebuild_bricks_kernel(const TF* f, int n, int* bmin) {
    const int nb = n / 8;
    const long long total = (long long)nb * nb * nb;
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long b = warp; b < total; b += nwarps) {
        const int bx = int(b % nb), by = int((b / nb) % nb), bz = int(b / ((long long)nb * nb));
        float m = 3.0e38f;
        for (int q = lane; q < 512; q += 32) {
            const int x = bx * 8 + (q & 7), y = by * 8 + ((q >> 3) & 7), z = bz * 8 + (q >> 6);
            m = fminf(m, load_f(f, (size_t(z) * n + y) * n + x));
        }
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, off));
        if (lane == 0) bmin[b] = fkey(m);
    }
}

__global__ void dilate_one_kernel(const int* bmin, int* bdil, int nb) {
    const long long total = (long long)nb * nb * nb;
    for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < total; b += (long long)gridDim.x * blockDim.x)
        dilate_brick(bmin, bdil, nb, int(b));
}

__global__ void superbrick_one_kernel(const int* bmin, int* sdil, int nb) {
    const int ns = (nb + 3) / 4;
    const long long total = (long long)ns * ns * ns;
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long b = warp; b < total; b += nwarps) {
        const int k = superbrick_bound(bmin, nb, int(b % ns), int((b / ns) % ns), int(b / ((long long)ns * ns)), lane);
        if (lane == 0) sdil[b] = k;
    }
}

cudaError_t launch_rebuild_bricks(const void* f, int fmt, int n, int* bmin, int* bdil, int* sdil, cudaStream_t st) {
    if (fmt == KF_TSDF_F16U16)
        rebuild_bricks_kernel<<<148 * 8, 256, 0, st>>>(static_cast<const __half*>(f), n, bmin);
    else
        rebuild_bricks_kernel<<<148 * 8, 256, 0, st>>>(static_cast<const float*>(f), n, bmin);
    dilate_one_kernel<<<148 * 4, 256, 0, st>>>(bmin, bdil, n / 8);
    superbrick_one_kernel<<<148 * 4, 256, 0, st>>>(bmin, sdil, n / 8);
    return cudaGetLastError();
}

// ---- stage fusion on a caller volume (kernel::fuse) ----

__global__ void __launch_bounds__(256) fuse_stage_kernel(FuseCtx c) {
    const int total = fuse_units(c.n);
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    // each warp tests 32 consecutive blocks (one per lane), then fuses the survivors together
    for (int base = warp * 32; base < total; base += nwarps * 32) {
        const int u = base + lane;
        int x0 = 0, j0 = 0, k0 = 0;
        bool keep = false;
        if (u < total) {
            unit_origin(c.n, u, x0, j0, k0);
            keep = !block_culled(c, x0, j0, k0);
        }
        unsigned int m = __ballot_sync(0xffffffffu, keep);
        while (m) {
            const int q = __ffs(m) - 1;
            m &= m - 1;
            const int bx = __shfl_sync(0xffffffffu, x0, q), by = __shfl_sync(0xffffffffu, j0, q),
                      bz = __shfl_sync(0xffffffffu, k0, q);
            fuse_rows(c, bx, by, bz, 0, 64, lane);
        }
    }
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
    c.fmt = vol->format;
    c.F = vol->f;
    c.W = vol->w;
    c.xs = xs;
    c.zs = zs;
    c.bmin = nullptr;
    // inverse of the rigid pose: R^T, -R^T t
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 3; ++row) c.iR[col * 3 + row] = pose[row * 4 + col];
    for (int row = 0; row < 3; ++row)
        c.it[row] = -(c.iR[row] * pose[12] + c.iR[3 + row] * pose[13] + c.iR[6 + row] * pose[14]);
    fuse_stage_kernel<<<148 * 8, 256, 0, st>>>(c);
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
