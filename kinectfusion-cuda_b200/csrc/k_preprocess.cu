// k_preprocess.cu -- depth preprocessing: uint16 -> metres, bilateral filter, 3-level
// pyramid and vertex maps.
//
// Reference: project/src/measurement.cu (convertToDepthMetersKernel :14-31,
// applyBilateralFilterKernel :33-66, downSampleKernel :68-102, createVertexMapKernel
// :104-126, createNormalMapKernel :128-135), driven by
// KinectFusion::depthFrameToVertexPyramid (project/src/kinect_fusion.cpp:116-135) as seven
// synchronous launches.  Here one block owns a 32x32 level-0 tile: it converts the tile plus
// its filter halo into shared memory once, filters from there, and produces the 16x16 and
// 8x8 tiles of levels 1 and 2 and all vertex maps without touching HBM again.  All sessions'
// tiles form one work list, so a single launch serves a whole batch.
//
// This file is compiled with the float semantics of the reference's Release build (FastMath,
// project/project.vcxproj:139: denormals flushed, fast division and square root; see
// build.py), and each core below performs the reference's operations in the reference's
// order, so the converted, filtered and down-sampled depth maps and the vertex maps are
// bit-identical to those of the reference's own kernels.
#include "kf_host.h"

namespace kf {

// ---- per-pixel cores shared by the fused kernel and the stage kernels ----

// applyBilateralFilterKernel body (project/src/measurement.cu:45-65): x outer, y inner,
// exp(-dx2/ss^2 - dr2/sr^2) with the fast exponential the reference's fast-math build
// selects, then acc / norm.  rd(x, y) returns the clamped neighbour.
template <class Reader>
__device__ __forceinline__ float bilateral_core(Reader rd, int R, float inv_ss, float inv_sr) {
    const float center = rd(0, 0);
    float norm = 0.f, acc = 0.f;
    for (int x = -R; x <= R; ++x) {
        for (int y = -R; y <= R; ++y) {
            const float cur = rd(x, y);
            const float s = float(x * x + y * y);
            float r = center - cur;
            r *= r;
            const float e = __expf(-s * inv_ss - r * inv_sr);
            norm += e;
            acc += e * cur;
        }
    }
    return acc / norm;
}

// The same for a radius known at compile time (the configurations' 2 and the reference's 3):
// the taps unroll with constant offsets into the tile; the arithmetic is the loop's above,
// operation for operation.
template <int kR, class Reader>
__device__ __forceinline__ float bilateral_fixed(Reader rd, float inv_ss, float inv_sr) {
    const float center = rd(0, 0);
    float norm = 0.f, acc = 0.f;
#pragma unroll
    for (int x = -kR; x <= kR; ++x) {
#pragma unroll
        for (int y = -kR; y <= kR; ++y) {
            const float cur = rd(x, y);
            const float s = float(x * x + y * y);
            float r = center - cur;
            r *= r;
            const float e = __expf(-s * inv_ss - r * inv_sr);
            norm += e;
            acc += e * cur;
        }
    }
    return acc / norm;
}

// downSampleKernel body (project/src/measurement.cu:73-101)
__device__ __forceinline__ float downsample_core(float f1, float f2, float f3, float f4, float thr) {
    float acc = f1;
    int count = 1;
    if (fabsf(f1 - f2) <= thr) { acc += f2; ++count; }
    if (fabsf(f1 - f3) <= thr) { acc += f3; ++count; }
    if (fabsf(f1 - f4) <= thr) { acc += f4; ++count; }
    return acc / float(count);
}

// createVertexMapKernel body (project/src/measurement.cu:109-125)
__device__ __forceinline__ float4 vertex_core(float d, int i, int j, const float* ik) {
    if (depth_valid(d)) {
        F3 p = mv3(ik, F3{float(i) + 0.5f, float(j) + 0.5f, 1.0f});
        p = p * d;
        return make_float4(p.x, p.y, p.z, kValid);
    }
    return make_float4(0.f, 0.f, 0.f, kInvalid);
}

// ---- fused, batched kernel ----

// One tile.  kR: the bilateral radius when it is known at compile time (2 or 3: the halo's
// pitch and the filter's offsets are constants), 0 for any other radius.
template <int kR>
__device__ __forceinline__ void preprocess_tile(const EngineView& v, const PreTile T, float* smem, unsigned int* qmax) {
    const int tid = threadIdx.x;
    {
        const SessionDev* S = &v.sess[T.s];
        const int W = S->W, H = S->H, R = kR ? kR : S->bil_r, L = S->L;
        const int pitch = kPreTileSize + 2 * R;
        float* reg = smem;                           // converted metres, tile + halo
        float* l0 = smem + pitch * pitch;            // filtered level 0, 32 x 32
        float* l1 = l0 + kPreTileSize * kPreTileSize;// level 1, 16 x 16
        const float scale = S->depth_scale;
        const uint16_t* raw = S->raw;

        // 1. convert the tile and its clamp-to-edge halo (convertToDepthMetersKernel); the
        //    interior is also the unfiltered metres map fusion reads, and its per-16x16
        //    largest valid depth lets fusion skip row segments that cannot update
        if (tid < 4) qmax[tid] = 0u;
        __syncthreads();
        for (int idx = tid; idx < pitch * pitch; idx += blockDim.x) {
            const int rx = idx % pitch, ry = idx / pitch;
            const int gx = min(max(T.x0 - R + rx, 0), W - 1);
            const int gy = min(max(T.y0 - R + ry, 0), H - 1);
            const int src = S->unmirror ? (W - 1 - gx) : gx;
            const float d = raw_to_half_value(__ldg(raw + size_t(gy) * W + src)) * scale;
            reg[idx] = d;
            const int ix = T.x0 - R + rx, iy = T.y0 - R + ry;
            if (rx >= R && rx < R + kPreTileSize && ry >= R && ry < R + kPreTileSize && ix < W && iy < H) {
                S->depth_m[size_t(iy) * W + ix] = d;
                if (depth_valid(d)) atomicMax(&qmax[((ry - R) >> 4) * 2 + ((rx - R) >> 4)], __float_as_uint(d));
            }
        }
        __syncthreads();
        if (tid < 4) {
            const int tx = (T.x0 >> 4) + (tid & 1), ty = (T.y0 >> 4) + (tid >> 1);
            if (tx < S->t16w && ty < S->t16h) S->dmax16[size_t(ty) * S->t16w + tx] = __uint_as_float(qmax[tid]);
        }

        // 2. bilateral filter + level-0 vertex map
        const LevelDev& L0 = S->lv[0];
        for (int k = tid; k < kPreTileSize * kPreTileSize; k += blockDim.x) {
            const int lx = k % kPreTileSize, ly = k / kPreTileSize;
            const int gx = T.x0 + lx, gy = T.y0 + ly;
            float d = 0.f;
            if (gx < L0.cw && gy < L0.ch) {
                const float* c = reg + (ly + R) * pitch + (lx + R);
                if constexpr (kR > 0)
                    d = bilateral_fixed<kR>([c](int x, int y) { return c[y * (kPreTileSize + 2 * kR) + x]; },
                                            S->bil_inv_ss, S->bil_inv_sr);
                else
                    d = bilateral_core([c, pitch](int x, int y) { return c[y * pitch + x]; }, R, S->bil_inv_ss,
                                       S->bil_inv_sr);
                S->depth[0][size_t(gy) * W + gx] = d;
                S->vmap[0][size_t(gy) * W + gx] = vertex_core(d, gx, gy, L0.ik);
            }
            l0[k] = d;
        }
        if (L > 1) {
            __syncthreads();
            // 3. level 1 (downSampleKernel + createVertexMapKernel)
            const LevelDev& L1 = S->lv[1];
            {
                const int lx = tid % 16, ly = tid / 16;
                const int gx = T.x0 / 2 + lx, gy = T.y0 / 2 + ly;
                float d = 0.f;
                if (gx < L1.cw && gy < L1.ch) {
                    const float* b = l0 + (2 * ly) * kPreTileSize + 2 * lx;
                    d = downsample_core(b[0], b[1], b[kPreTileSize], b[kPreTileSize + 1], S->down_thr);
                    S->depth[1][size_t(gy) * L1.w + gx] = d;
                    S->vmap[1][size_t(gy) * L1.w + gx] = vertex_core(d, gx, gy, L1.ik);
                }
                l1[tid] = d;
            }
            if (L > 2) {
                __syncthreads();
                // 4. level 2
                const LevelDev& L2 = S->lv[2];
                if (tid < 64) {
                    const int lx = tid % 8, ly = tid / 8;
                    const int gx = T.x0 / 4 + lx, gy = T.y0 / 4 + ly;
                    if (gx < L2.cw && gy < L2.ch) {
                        const float* b = l1 + (2 * ly) * 16 + 2 * lx;
                        const float d = downsample_core(b[0], b[1], b[16], b[17], S->down_thr);
                        S->depth[2][size_t(gy) * L2.w + gx] = d;
                        S->vmap[2][size_t(gy) * L2.w + gx] = vertex_core(d, gx, gy, L2.ik);
                    }
                }
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) preprocess_kernel(EngineView v) {
    extern __shared__ float smem[];
    __shared__ unsigned int qmax[4];   // largest valid depth of each 16x16 quadrant (float bits)
    const int ntiles = v.tb->n_pre;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const PreTile T = v.pre[t];
        if (!v.step[T.s].active) continue;   // block-uniform
        const int R = v.sess[T.s].bil_r;
        if (R == 2)
            preprocess_tile<2>(v, T, smem, qmax);
        else if (R == 3)
            preprocess_tile<3>(v, T, smem, qmax);
        else
            preprocess_tile<0>(v, T, smem, qmax);
    }
}

cudaError_t launch_preprocess(const EngineView& v, int grid, cudaStream_t st) {
    const int pitch = kPreTileSize + 2 * kMaxBilateralRadius;
    const size_t smem = sizeof(float) * (pitch * pitch + kPreTileSize * kPreTileSize + 256);
    preprocess_kernel<<<grid, 256, smem, st>>>(v);
    return cudaGetLastError();
}

// ---- stage kernels (one thread per pixel, mirroring the reference's kernel:: calls) ----

__global__ void convert_kernel(const uint16_t* raw, float* out, int w, int h, float scale, int unmirror) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= w || j >= h) return;
    const float d = raw_to_half_value(raw[size_t(j) * w + i]) * scale;
    const int io = unmirror ? (w - 1 - i) : i;
    out[size_t(j) * w + io] = d;
}

__global__ void bilateral_kernel(const float* in, float* out, int w, int h, float inv_ss, float inv_sr, int R) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= w || j >= h) return;
    out[size_t(j) * w + i] = bilateral_core(
        [in, w, h, i, j](int x, int y) {
            const int xx = min(max(i + x, 0), w - 1), yy = min(max(j + y, 0), h - 1);
            return __ldg(in + size_t(yy) * w + xx);
        },
        R, inv_ss, inv_sr);
}

__global__ void downsample_kernel(const float* in, float* out, int wo, int ho, float thr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= wo || j >= ho) return;
    const int wi = 2 * wo;
    const float* b = in + size_t(2 * j) * wi + 2 * i;
    out[size_t(j) * wo + i] = downsample_core(b[0], b[1], b[wi], b[wi + 1], thr);
}

struct Ik { float m[9]; };

__global__ void vertex_kernel(const float* d, float4* vm, int w, int h, Ik ik) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= w || j >= h) return;
    vm[size_t(j) * w + i] = vertex_core(d[size_t(j) * w + i], i, j, ik.m);
}

__global__ void normal_kernel(const float4* vm, float4* nm, int w, int h) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= w || j >= h) return;
    nm[size_t(j) * w + i] = compute_normal(vm, w, h, i, j);
}

static dim3 grid2(int w, int h) { return dim3((w + 15) / 16, (h + 15) / 16); }

cudaError_t stage_convert(const uint16_t* raw, float* out, int w, int h, float scale, int unmirror, cudaStream_t st) {
    convert_kernel<<<grid2(w, h), dim3(16, 16), 0, st>>>(raw, out, w, h, scale, unmirror);
    return cudaGetLastError();
}
cudaError_t stage_bilateral(const float* in, float* out, int w, int h, float ss, float sr, int r, cudaStream_t st) {
    bilateral_kernel<<<grid2(w, h), dim3(16, 16), 0, st>>>(in, out, w, h, 1.0f / (ss * ss), 1.0f / (sr * sr), r);
    return cudaGetLastError();
}
cudaError_t stage_down_sample(const float* in, float* out, int wo, int ho, float sr, cudaStream_t st) {
    downsample_kernel<<<grid2(wo, ho), dim3(16, 16), 0, st>>>(in, out, wo, ho, 3.0f * sr);
    return cudaGetLastError();
}
cudaError_t stage_vertex(const float* d, float4* v, int w, int h, const float* ik, cudaStream_t st) {
    Ik k;
    for (int q = 0; q < 9; ++q) k.m[q] = ik[q];
    vertex_kernel<<<grid2(w, h), dim3(16, 16), 0, st>>>(d, v, w, h, k);
    return cudaGetLastError();
}
cudaError_t stage_normal(const float4* v, float4* n, int w, int h, cudaStream_t st) {
    normal_kernel<<<grid2(w, h), dim3(16, 16), 0, st>>>(v, n, w, h);
    return cudaGetLastError();
}

}  // namespace kf
