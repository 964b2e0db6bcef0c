// k_raycast.cu -- predicted vertex / normal maps by ray marching the TSDF.
//
// Reference: raycastKernel (project/src/raycast.cu:44-145) with intersectBBox (:7-27) and
// computeGradient (:29-42), called once per pyramid level at the previous frame's pose
// (project/src/kinect_fusion.cpp:137-144).  The reference samples a cudaArray through the
// texture unit; here the distance array stays in linear HBM (x fastest), so fusion can stream
// it with 16-byte vectors, and the march does its own trilinear interpolation with the
// reference's texel mapping (uvw * n - 0.5, clamp).  The slice of the volume near the
// surface a frame's rays touch stays resident in the 126 MB L2.  Rays of all levels and all
// sessions form one tile list that persistent blocks pull from an atomic counter.
#include "kf_host.h"

namespace kf {

constexpr int kMaxMarchSamples = 1 << 16;

// one ray of raycastKernel; returns after writing (or deliberately not writing) its pixel
template <class TF>
__device__ __forceinline__ void march_ray(const SessionDev* __restrict__ S, const LevelDev& Lv, const float* Rw,
                                          F3 o, const TF* __restrict__ f, int level, int i, int j) {
    const int w = Lv.w;
    float4* ov = S->pv[level] + size_t(j) * w + i;
    float4* on = S->pn[level] + size_t(j) * w + i;
    const int n = S->n;
    const float width = S->vol_w, mu = S->mu;

    // direction = (R * K^-1) (i + .5, j + .5, 1), not normalised: t is camera depth
    const F3 pix{float(i) + 0.5f, float(j) + 0.5f, 1.0f};
    const F3 dir = mv3(Rw, pix);
    const F3 inv{1.0f / dir.x, 1.0f / dir.y, 1.0f / dir.z};
    const float half = width * 0.5f;
    // intersectBBox
    const float t0x = (-half - o.x) * inv.x, t1x = (half - o.x) * inv.x;
    const float t0y = (-half - o.y) * inv.y, t1y = (half - o.y) * inv.y;
    const float t0z = (-half - o.z) * inv.z, t1z = (half - o.z) * inv.z;
    float tmin = fminf(t0x, t1x), tmax = fmaxf(t0x, t1x);
    tmin = fmaxf(tmin, fminf(t0y, t1y));
    tmax = fminf(tmax, fmaxf(t0y, t1y));
    tmin = fmaxf(tmin, fminf(t0z, t1z));
    tmax = fminf(tmax, fmaxf(t0z, t1z));
    if (tmax < tmin) { tmin = -1.0f; tmax = -1.0f; }
    bool early = tmax < 0.0f;
    float near_d = 0.f, far_d = 0.f;
    if (!early) {
        near_d = fmaxf(S->min_d, tmin);
        far_d = fminf(S->max_d, tmax);
        early = near_d >= far_d;
    }
    if (early) {
        if (!S->keep_on_miss) {
            *ov = make_float4(0.f, 0.f, 0.f, kInvalid);
            *on = make_float4(0.f, 0.f, 0.f, kInvalid);
        }
        return;
    }
    // texel coordinate of world point p: (p / width + 0.5) * n - 0.5
    const float sc = float(n) / width, off = 0.5f * float(n) - 0.5f;
    const float large = mu * S->step_l, small = mu * S->step_s;
    const float* __restrict__ bmin = S->bmin;
    const int nb = S->nb;
    // the ray in texel space, for brick exits: x(t) = tox + tdx t
    const float tox = o.x * sc + off, toy = o.y * sc + off, toz = o.z * sc + off;
    const float tdx = dir.x * sc, tdy = dir.y * sc, tdz = dir.z * sc;
    float inc = large, prev = 0.f, precise = 0.f;
    float prev_t = 0.f;       // position of the last non-negative sample
    bool prev_known = true;   // false when that sample was skipped (its value not computed)
    int guard = 0;            // hard bound on samples per ray, whatever the configuration
    float t = near_d;
    while (t < far_d && guard < kMaxMarchSamples) {
        const float x = (o.x + dir.x * t) * sc + off;
        const float y = (o.y + dir.y * t) * sc + off;
        const float z = (o.z + dir.z * t) * sc + off;
        if (bmin) {
            // A brick whose minimum is >= 0.991 (large steps) or >= 0.001 (small steps) holds
            // no sample that changes the march: the value stays >= 0.99 resp. >= 0, so the
            // reference would only step on.  Skip this sample and every later one inside the
            // brick (0.01 texel inside its faces), advancing t exactly as the reference does.
            const int ix = min(max(int(floorf(x)), 0), n - 1) >> 3;
            const int iy = min(max(int(floorf(y)), 0), n - 1) >> 3;
            const int iz = min(max(int(floorf(z)), 0), n - 1) >> 3;
            const float m = __ldg(bmin + (size_t(iz) * nb + iy) * nb + ix);
            if (m >= (inc == large ? 0.991f : 0.001f)) {
                float t_safe = far_d;
                if (tdx > 0.f && ix < nb - 1) t_safe = fminf(t_safe, (float(8 * ix + 8) - 0.01f - tox) / tdx);
                if (tdx < 0.f && ix > 0) t_safe = fminf(t_safe, (float(8 * ix) + 0.01f - tox) / tdx);
                if (tdy > 0.f && iy < nb - 1) t_safe = fminf(t_safe, (float(8 * iy + 8) - 0.01f - toy) / tdy);
                if (tdy < 0.f && iy > 0) t_safe = fminf(t_safe, (float(8 * iy) + 0.01f - toy) / tdy);
                if (tdz > 0.f && iz < nb - 1) t_safe = fminf(t_safe, (float(8 * iz + 8) - 0.01f - toz) / tdz);
                if (tdz < 0.f && iz > 0) t_safe = fminf(t_safe, (float(8 * iz) + 0.01f - toz) / tdz);
                do {
                    prev_t = t;
                    t += inc;
                    ++guard;
                } while (t < t_safe && t < far_d && guard < kMaxMarchSamples);
                prev_known = false;
                continue;
            }
        }
        const float tsdf = trilinear(f, n, x, y, z);
        ++guard;
        if (tsdf < 0.0f) {
            if (t != near_d) {
                if (inc == large) {   // went through the surface with a large step: back off
                    t -= mu;
                    inc = small;
                    t += inc;
                    continue;
                }
                if (!prev_known) {
                    const float ax = (o.x + dir.x * prev_t) * sc + off;
                    const float ay = (o.y + dir.y * prev_t) * sc + off;
                    const float az = (o.z + dir.z * prev_t) * sc + off;
                    prev = trilinear(f, n, ax, ay, az);
                }
                precise = t - inc * prev / (tsdf - prev);   // the reference's zero-crossing formula
            }
            break;
        } else if (tsdf < 0.99f) {
            inc = small;
        }
        prev = tsdf;
        prev_known = true;
        prev_t = t;
        t += inc;
    }
    if (precise != 0.0f) {
        const F3 vtx{o.x + dir.x * precise, o.y + dir.y * precise, o.z + dir.z * precise};
        // computeGradient: central differences mu / 2 apart, in uvw units
        const float r = mu * 0.5f / width;
        const float rt = r * float(n);
        const float x = vtx.x * sc + off, y = vtx.y * sc + off, z = vtx.z * sc + off;
        const float fx0 = trilinear(f, n, x + rt, y, z), fy0 = trilinear(f, n, x, y + rt, z);
        const float fz0 = trilinear(f, n, x, y, z + rt);
        const float fx = trilinear(f, n, x - rt, y, z), fy = trilinear(f, n, x, y - rt, z);
        const float fz = trilinear(f, n, x, y, z - rt);
        F3 g{(fx - fx0) / r, (fy - fy0) / r, (fz - fz0) / r};
        const float gn = sqrtf(dot3(g, g));
        if (depth_valid(gn)) {
            g = F3{g.x / gn, g.y / gn, g.z / gn};
            *ov = make_float4(vtx.x, vtx.y, vtx.z, kValid);
            *on = make_float4(g.x, g.y, g.z, kValid);
            return;
        }
    }
    *ov = make_float4(0.f, 0.f, 0.f, kInvalid);
    *on = make_float4(0.f, 0.f, 0.f, kInvalid);
}

__global__ void __launch_bounds__(256) raycast_kernel(EngineView v) {
    __shared__ int s_tile;
    __shared__ float s_m[9];
    __shared__ float s_o[3];
    const int tid = threadIdx.x;
    const int ntiles = v.tb->n_ray;
    // lane layout: each warp owns an 8 x 4 patch of the 16 x 16 tile
    const int warp = tid >> 5, lane = tid & 31;
    const int lx = (warp & 1) * 8 + (lane & 7), ly = (warp >> 1) * 4 + (lane >> 3);
    while (true) {
        if (tid == 0) s_tile = int(atomicAdd(&v.counters[0], 1u));
        __syncthreads();
        const int t = s_tile;
        if (t >= ntiles) break;
        const RayTile T = v.ray[t];
        const StepDev st = v.step[T.s];
        if (st.active && !st.first) {
            const SessionDev* S = &v.sess[T.s];
            const LevelDev& Lv = S->lv[T.level];
            if (tid < 9) {
                // R_prev * K_l^-1 (the reference forms mat3(pose) * invK per ray)
                const int col = tid / 3, row = tid % 3;
                const float* R = S->pose->Rpf;
                s_m[tid] = R[row] * Lv.ik[col * 3 + 0] + R[3 + row] * Lv.ik[col * 3 + 1] + R[6 + row] * Lv.ik[col * 3 + 2];
            } else if (tid < 12) {
                s_o[tid - 9] = S->pose->tpf[tid - 9];
            }
            __syncthreads();
            const int i = T.x0 + lx, j = T.y0 + ly;
            if (i < Lv.cw && j < Lv.ch) {
                const F3 o{s_o[0], s_o[1], s_o[2]};
                if (S->fmt == KF_TSDF_F16U16)
                    march_ray(S, Lv, s_m, o, static_cast<const __half*>(S->tf), T.level, i, j);
                else
                    march_ray(S, Lv, s_m, o, static_cast<const float*>(S->tf), T.level, i, j);
            }
        }
        __syncthreads();
    }
}

cudaError_t launch_raycast(const EngineView& v, int grid, cudaStream_t st) {
    raycast_kernel<<<grid, 256, 0, st>>>(v);
    return cudaGetLastError();
}

// ---- stage kernel: kernel::raycast on a caller volume ----

struct RayStage {
    float m[9];
    float o[3];
};

template <class TF>
__global__ void raycast_stage_kernel(SessionDev S, RayStage rs, int w, int h) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= w || j >= h) return;
    march_ray(&S, S.lv[0], rs.m, F3{rs.o[0], rs.o[1], rs.o[2]}, static_cast<const TF*>(S.tf), 0, i, j);
}

cudaError_t stage_raycast(const kf_volume* vol, const float* pose, const float* ik, float4* vtx, float4* nrm, int w,
                          int h, float min_d, float max_d, float step_l, float step_s, cudaStream_t st) {
    SessionDev S{};
    S.n = vol->n;
    S.fmt = vol->format;
    S.vol_w = vol->width;
    S.mu = vol->mu;
    S.tf = vol->f;
    S.tw = vol->w;
    S.min_d = min_d;
    S.max_d = max_d;
    S.step_l = step_l;
    S.step_s = step_s;
    S.keep_on_miss = 1;
    S.pv[0] = vtx;
    S.pn[0] = nrm;
    S.lv[0].w = w;
    S.lv[0].h = h;
    S.lv[0].cw = w;
    S.lv[0].ch = h;
    RayStage rs;
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 3; ++row)
            rs.m[col * 3 + row] = pose[row] * ik[col * 3 + 0] + pose[4 + row] * ik[col * 3 + 1] + pose[8 + row] * ik[col * 3 + 2];
    rs.o[0] = pose[12];
    rs.o[1] = pose[13];
    rs.o[2] = pose[14];
    dim3 blk(8, 8), grd((w + 7) / 8, (h + 7) / 8);
    if (vol->format == KF_TSDF_F16U16)
        raycast_stage_kernel<__half><<<grd, blk, 0, st>>>(S, rs, w, h);
    else
        raycast_stage_kernel<float><<<grd, blk, 0, st>>>(S, rs, w, h);
    return cudaGetLastError();
}

}  // namespace kf
