// k_tsdf.cu -- TSDF volume: initialisation, projective fusion, layout conversion.
//
// Reference: initializeGridKernel (project/src/tsdf.cu:7-18) and fuseKernel
// (project/src/tsdf.cu:20-75), which walks one (x, y) voxel column per thread through a
// cudaArray surface with 4-byte reads and writes.  Here the volume is two linear arrays in
// HBM (distance, weight; x fastest), so a warp streams a 32 x VEC-voxel segment of an x row
// with 16-byte vector loads and stores per lane: 4 voxels per lane for float/float, 8 for
// fp16/uint16.  A lane projects its voxels first and touches HBM only when one of them
// updates; segments are handed out to persistent warps through an atomic counter, over all
// sessions of a batch in one launch.
#include "kf_host.h"

namespace kf {

int fuse_vec(int fmt) { return fmt == KF_TSDF_F16U16 ? 8 : 4; }
int fuse_segs_per_row(int n, int fmt) {
    const int span = 32 * fuse_vec(fmt);
    return (n + span - 1) / span;
}

// the fuseKernel update of one voxel (project/src/tsdf.cu:33-70); returns false when the
// voxel is left alone.  pe: voxel centre in camera coordinates.
__device__ __forceinline__ bool fuse_voxel(F3 pe, const float* __restrict__ depth, int w, int h, float fx, float fy,
                                           float cx, float cy, float min_d, float max_d, float mu, float& fn,
                                           float& wn) {
    const float iz = 1.0f / pe.z;
    const float px = (fx * pe.x + cx * pe.z) * iz;
    const float py = (fy * pe.y + cy * pe.z) * iz;
    if (!(pe.z >= min_d && pe.z < max_d && px >= 0.0f && px < float(w) && py >= 0.0f && py < float(h)))
        return false;
    const float d = __ldg(depth + size_t(int(py)) * w + int(px));
    if (!depth_valid(d)) return false;
    const float diff = d - pe.z;
    if (!(diff >= -mu)) return false;
    fn = fminf(1.0f, diff / mu);
    wn = 1.0f / d;
    return true;
}

struct FuseCtx {
    const float* depth;
    int w, h;
    float fx, fy, cx, cy, min_d, max_d, mu, max_w;
    float iR[9], it[3];
};

// running weighted average (project/src/tsdf.cu:56-69); max_w > 0 clamps the weight
__device__ __forceinline__ void fuse_update(float& F, float& Wt, float fn, float wn, float max_w) {
    F = (F * Wt + fn * wn) / (Wt + wn);
    float w1 = Wt + wn;
    if (max_w > 0.0f) w1 = fminf(w1, max_w);
    Wt = w1;
}

// One lane's VEC voxels starting at x0 of row (j, k).  Arrays are float (VEC = 4) or
// __half / uint16 (VEC = 8).
template <int VEC, class TF, class TW>
__device__ __forceinline__ void fuse_lane(const FuseCtx& c, TF* __restrict__ F, TW* __restrict__ Wt,
                                          const float* __restrict__ xs, float y, float z, size_t row_base, int x0,
                                          int n) {
    if (x0 >= n) return;
    // row-constant part of the world->camera transform
    const F3 b{c.iR[3] * y + c.iR[6] * z + c.it[0], c.iR[4] * y + c.iR[7] * z + c.it[1],
               c.iR[5] * y + c.iR[8] * z + c.it[2]};
    float xv[VEC];
    if constexpr (VEC == 4) {
        const float4 q = __ldg(reinterpret_cast<const float4*>(xs + x0));
        xv[0] = q.x; xv[1] = q.y; xv[2] = q.z; xv[3] = q.w;
    } else {
        const float4 q0 = __ldg(reinterpret_cast<const float4*>(xs + x0));
        const float4 q1 = __ldg(reinterpret_cast<const float4*>(xs + x0 + 4));
        xv[0] = q0.x; xv[1] = q0.y; xv[2] = q0.z; xv[3] = q0.w;
        xv[4] = q1.x; xv[5] = q1.y; xv[6] = q1.z; xv[7] = q1.w;
    }
    float fn[VEC], wn[VEC];
    unsigned int upd = 0;
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
        const F3 pe{c.iR[0] * xv[v] + b.x, c.iR[1] * xv[v] + b.y, c.iR[2] * xv[v] + b.z};
        if (fuse_voxel(pe, c.depth, c.w, c.h, c.fx, c.fy, c.cx, c.cy, c.min_d, c.max_d, c.mu, fn[v], wn[v]))
            upd |= 1u << v;
    }
    if (!upd) return;
    const size_t base = row_base + x0;
    if constexpr (VEC == 4) {
        float4* fp = reinterpret_cast<float4*>(F + base);
        float4* wp = reinterpret_cast<float4*>(Wt + base);
        float4 fq = *fp, wq = *wp;
        float fa[4] = {fq.x, fq.y, fq.z, fq.w}, wa[4] = {wq.x, wq.y, wq.z, wq.w};
#pragma unroll
        for (int v = 0; v < 4; ++v)
            if (upd & (1u << v)) fuse_update(fa[v], wa[v], fn[v], wn[v], c.max_w);
        *fp = make_float4(fa[0], fa[1], fa[2], fa[3]);
        *wp = make_float4(wa[0], wa[1], wa[2], wa[3]);
    } else {
        uint4* fp = reinterpret_cast<uint4*>(F + base);
        uint4* wp = reinterpret_cast<uint4*>(Wt + base);
        uint4 fq = *fp, wq = *wp;
        __half* fh = reinterpret_cast<__half*>(&fq);
        uint16_t* wh = reinterpret_cast<uint16_t*>(&wq);
        const float wscale = KF_WEIGHT_SCALE, inv_wscale = 1.0f / KF_WEIGHT_SCALE;
#pragma unroll
        for (int v = 0; v < 8; ++v)
            if (upd & (1u << v)) {
                float f0 = __half2float(fh[v]);
                float w0 = float(wh[v]) * inv_wscale;
                fuse_update(f0, w0, fn[v], wn[v], c.max_w);
                fh[v] = __float2half_rn(f0);
                wh[v] = uint16_t(fminf(rintf(w0 * wscale), 65535.0f));
            }
        *fp = fq;
        *wp = wq;
    }
}

template <int VEC, class TF, class TW>
__device__ __forceinline__ void fuse_segment(const SessionDev* S, const FuseCtx& c, long long seg_local, int lane) {
    const int n = S->n;
    const int spr = (n + 32 * VEC - 1) / (32 * VEC);
    const long long row = seg_local / spr;
    const int seg = int(seg_local - row * spr);
    const int j = int(row % n), k = int(row / n);
    const float y = __ldg(S->xs + j), z = __ldg(S->zs + k);
    const int x0 = seg * 32 * VEC + lane * VEC;
    fuse_lane<VEC>(c, static_cast<TF*>(S->tf), static_cast<TW*>(S->tw), S->xs, y, z, size_t(row) * n, x0, n);
}

__device__ __forceinline__ void make_ctx(const SessionDev* S, FuseCtx& c) {
    c.depth = S->depth_m;
    c.w = S->W;
    c.h = S->H;
    c.fx = S->lv[0].fx; c.fy = S->lv[0].fy; c.cx = S->lv[0].cx; c.cy = S->lv[0].cy;
    c.min_d = S->min_d; c.max_d = S->max_d; c.mu = S->mu; c.max_w = S->max_w;
#pragma unroll
    for (int q = 0; q < 9; ++q) c.iR[q] = S->pose->iRf[q];
#pragma unroll
    for (int q = 0; q < 3; ++q) c.it[q] = S->pose->itf[q];
}

constexpr int kFuseChunk = 4;   // segments a warp takes per atomic

__global__ void __launch_bounds__(256) fuse_kernel(EngineView v) {
    const int lane = threadIdx.x & 31;
    const long long total = v.tb->fuse_total;
    const int S_cap = v.tb->S;
    unsigned long long* ctr = reinterpret_cast<unsigned long long*>(v.counters + 2);
    int cur_s = -1;
    bool live = false;
    FuseCtx c;
    while (true) {
        unsigned long long g0 = 0;
        if (lane == 0) g0 = atomicAdd(ctr, (unsigned long long)kFuseChunk);
        g0 = __shfl_sync(0xffffffffu, g0, 0);
        if ((long long)g0 >= total) break;
        for (int q = 0; q < kFuseChunk; ++q) {
            const long long g = (long long)g0 + q;
            if (g >= total) break;
            // session of segment g: binary search of the prefix (warp-uniform)
            int lo = 0, hi = S_cap;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (__ldg(v.fuse_prefix + mid) <= g) lo = mid; else hi = mid;
            }
            const int s = lo;
            const SessionDev* S = &v.sess[s];
            if (s != cur_s) {
                cur_s = s;
                const StepDev st = v.step[s];
                live = st.active && S->pose->fuse_ok;
                if (live) make_ctx(S, c);
            }
            if (!live) continue;
            const long long local = g - __ldg(v.fuse_prefix + s);
            if (S->fmt == KF_TSDF_F16U16)
                fuse_segment<8, __half, uint16_t>(S, c, local, lane);
            else
                fuse_segment<4, float, float>(S, c, local, lane);
        }
    }
}

cudaError_t launch_fuse(const EngineView& v, int grid, cudaStream_t st) {
    fuse_kernel<<<grid, 256, 0, st>>>(v);
    return cudaGetLastError();
}

// ---- stage fusion on a caller volume (kernel::fuse) ----

template <int VEC, class TF, class TW>
__global__ void fuse_stage_kernel(FuseCtx c, TF* F, TW* Wt, const float* xs, const float* zs, int n) {
    const long long spr = (n + 32 * VEC - 1) / (32 * VEC);
    const long long total = (long long)n * n * spr;
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long g = warp; g < total; g += nwarps) {
        const long long row = g / spr;
        const int seg = int(g - row * spr);
        const int j = int(row % n), k = int(row / n);
        fuse_lane<VEC>(c, F, Wt, xs, __ldg(xs + j), __ldg(zs + k), size_t(row) * n, seg * 32 * VEC + lane * VEC, n);
    }
}

cudaError_t stage_fuse(const float* depth, int w, int h, const float* k, const kf_volume* vol, const float* pose,
                       float min_d, float max_d, const float* xs, const float* zs, cudaStream_t st) {
    FuseCtx c;
    c.depth = depth;
    c.w = w;
    c.h = h;
    c.fx = k[0]; c.fy = k[4]; c.cx = k[6]; c.cy = k[7];
    c.min_d = min_d; c.max_d = max_d; c.mu = vol->mu; c.max_w = vol->max_weight;
    // inverse of the rigid pose: R^T, -R^T t
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 3; ++row) c.iR[col * 3 + row] = pose[row * 4 + col];
    for (int row = 0; row < 3; ++row)
        c.it[row] = -(c.iR[row] * pose[12] + c.iR[3 + row] * pose[13] + c.iR[6 + row] * pose[14]);
    const int grid = 148 * 8;
    if (vol->format == KF_TSDF_F16U16)
        fuse_stage_kernel<8, __half, uint16_t><<<grid, 256, 0, st>>>(c, static_cast<__half*>(vol->f),
                                                                   static_cast<uint16_t*>(vol->w), xs, zs, vol->n);
    else
        fuse_stage_kernel<4, float, float><<<grid, 256, 0, st>>>(c, static_cast<float*>(vol->f),
                                                               static_cast<float*>(vol->w), xs, zs, vol->n);
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
