// k_icp.cu -- projective point-to-plane ICP on the device.
//
// Reference: constructIcpResidualsKernel (project/src/icp.cu:7-82) writes an N x 6 matrix A
// and a vector b to HBM, cuBLAS forms A^T A and A^T b, two copies bring them to the host,
// Eigen solves a float LLT and the host updates the pose, per iteration
// (project/src/icp.cpp:25-87, project/src/linear_least_squares.cpp:23-44).
//
// Here one cooperative launch runs the whole coarse-to-fine loop for every session of a
// batch.  Each pass:
//   A. every block takes pixel tiles of sessions still iterating, associates and rejects
//      pixels as the reference does, and accumulates the 27 distinct entries of A^T A / A^T b
//      (21 + 6) in FP32; a warp-shuffle reduce-scatter with two-sum compensation and a
//      compensated combine across warps give one (sum, compensation) pair per entry per tile;
//   B. one block per session adds its tiles' pairs in FP64, solves the 6x6 system by FP64
//      Cholesky, updates the FP64 pose and applies the reference's early-stop test;
// separated by bounded grid barriers.  Nothing returns to the host until the frame is done.
#include <mutex>

#include <cmath>

#include "kf_host.h"

namespace kf {

// ---- loads of data other blocks of the same launch wrote (bypass L1) ----
__device__ __forceinline__ float ldcg(const float* p) { return __ldcg(p); }
__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ int ldcg(const int* p) { return __ldcg(p); }

// ---- the reference's correspondence and rejection tests (project/src/icp.cuh:40-48, 72-85),
// in the forms its -use_fast_math build evaluates or cheaper equivalents ----
// floor(x / z) of computeCorrespondence with the approximate division of that build
__device__ __forceinline__ int corr_coord(float x, float z) {
    return int(floorf(__fdividef(x, z)));   // cvt.rzi: NaN -> 0, as in the reference
}
// areVerticesTooFarAway: |e| > d  <=>  e.e > d^2 (NaN compares false either way)
__device__ __forceinline__ bool too_far(F3 e, float dist_th) { return dot3(e, e) > dist_th * dist_th; }
// areNormalsTooDifferent: acos(c) > a  <=>  c < cos(a) for c in [-1, 1]; outside [-1, 1] and
// for NaN acos is NaN, the comparison is false and the pair passes, as in the reference
__device__ __forceinline__ bool too_different(float c, float cos_th) { return c < cos_th && c >= -1.0f; }

// ---- per-pixel residual: constructIcpResidualsKernel body with computeCorrespondence,
// areVerticesTooFarAway, areNormalsTooDifferent and computeAndFillA/B
// (project/src/icp.cu:20-81, project/src/icp.cuh:40-95) ----
__device__ __forceinline__ bool icp_pixel(const float4* __restrict__ vm, const float4* __restrict__ tv,
                                          const float4* __restrict__ tn, int w, int h, int u, int v, const float* R,
                                          const float* t, const float* M, const float* tp, float dist_th,
                                          float cos_th, float a[6], float& b) {
    const float4 vc = __ldg(vm + size_t(v) * w + u);
    if (vc.w != kValid) return false;
    const F3 s = mv3(R, f3(vc)) + F3{t[0], t[1], t[2]};
    // (K * R_prev^T) * (s - t_prev), then floor(x / z), floor(y / z)
    const F3 pt = mv3(M, s - F3{tp[0], tp[1], tp[2]});
    const int uc = corr_coord(pt.x, pt.z);
    const int vcor = corr_coord(pt.y, pt.z);
    if (uc < 0 || vcor < 0 || uc >= w || vcor >= h) return false;
    const float4 d4 = __ldg(tv + size_t(vcor) * w + uc);
    const float4 n4 = __ldg(tn + size_t(vcor) * w + uc);
    if (d4.w != kValid || n4.w != kValid) return false;
    const F3 d = f3(d4);
    const F3 e = s - d;
    if (too_far(e, dist_th)) return false;
    const float4 ns = compute_normal(vm, w, h, u, v);
    if (ns.w == kInvalid) return false;
    F3 nr = mv3(R, f3(ns));
    nr = nr * rsqrtf(dot3(nr, nr));
    const F3 n = f3(n4);
    if (too_different(dot3(nr, n), cos_th)) return false;
    a[0] = n.y * s.z - n.z * s.y;
    a[1] = n.z * s.x - n.x * s.z;
    a[2] = n.x * s.y - n.y * s.x;
    a[3] = n.x;
    a[4] = n.y;
    a[5] = n.z;
    b = n.x * d.x + n.y * d.y + n.z * d.z - n.x * s.x - n.y * s.y - n.z * s.z;
    return true;
}

// U pixels of a tile per thread and step (p0, p0 + 256, ...), with the same arithmetic as
// icp_pixel: the source vertices and their right and lower neighbours (for the normal) of all
// U pixels are loaded together, then all correspondences are gathered together, so up to
// 5 U loads are in flight per thread instead of one dependent chain per pixel.  Rejection
// tests are conjunctive, so evaluating them in a different order gives the same mask and
// rows; products are accumulated in pixel order.
struct IcpMats { const float* R; const float* t; const float* M; const float* tp; };

template <int U, class Acc>
__device__ __forceinline__ void icp_multi(const float4* __restrict__ vm, const float4* __restrict__ tv,
                                        const float4* __restrict__ tn, int w, int h, int icw, int p0, int pend,
                                        const IcpMats& m, float dist_th, float cos_th, uint8_t* mask, Acc&& accumulate) {
    int u[U], vv[U];
    bool in[U];
    float4 vc[U], vr[U], vd[U];
    const float4 none = make_float4(0.f, 0.f, 0.f, kInvalid);
#pragma unroll
    for (int q = 0; q < U; ++q) {
        const int p = p0 + q * kIcpThreads;
        in[q] = p < pend;
        u[q] = p % icw;
        vv[q] = p / icw;
        const size_t i = size_t(vv[q]) * w + u[q];
        vc[q] = in[q] ? __ldg(vm + i) : none;
        vr[q] = in[q] && u[q] + 1 < w ? __ldg(vm + i + 1) : none;
        vd[q] = in[q] && vv[q] + 1 < h ? __ldg(vm + i + w) : none;
    }
    F3 s[U];
    int uc[U], vcor[U];
    bool ok[U];
#pragma unroll
    for (int q = 0; q < U; ++q) {
        ok[q] = in[q] && vc[q].w == kValid;
        uc[q] = vcor[q] = 0;
        if (ok[q]) {
            s[q] = mv3(m.R, f3(vc[q])) + F3{m.t[0], m.t[1], m.t[2]};
            const F3 pt = mv3(m.M, s[q] - F3{m.tp[0], m.tp[1], m.tp[2]});
            uc[q] = corr_coord(pt.x, pt.z);
            vcor[q] = corr_coord(pt.y, pt.z);
            ok[q] = !(uc[q] < 0 || vcor[q] < 0 || uc[q] >= w || vcor[q] >= h);
        }
    }
    float4 d4[U], n4[U];
#pragma unroll
    for (int q = 0; q < U; ++q) {
        d4[q] = ok[q] ? __ldg(tv + size_t(vcor[q]) * w + uc[q]) : none;
        n4[q] = ok[q] ? __ldg(tn + size_t(vcor[q]) * w + uc[q]) : none;
    }
#pragma unroll
    for (int q = 0; q < U; ++q) {
        bool good = ok[q] && d4[q].w == kValid && n4[q].w == kValid;
        float a[6], b = 0.f;
        if (good) {
            const F3 d = f3(d4[q]);
            const F3 e = s[q] - d;
            good = !too_far(e, dist_th);
            // computeNormal: the vertex, its right and its lower neighbour valid
            good = good && vr[q].w == kValid && vd[q].w == kValid;
            if (good) {
                const F3 c = f3(vc[q]);
                F3 nn = cross3(f3(vr[q]) - c, f3(vd[q]) - c);
                nn = nn * rsqrtf(dot3(nn, nn));
                F3 nr = mv3(m.R, nn);
                nr = nr * rsqrtf(dot3(nr, nr));
                const F3 n = f3(n4[q]);
                good = !too_different(dot3(nr, n), cos_th);
                if (good) {
                    const F3 sv = s[q];
                    a[0] = n.y * sv.z - n.z * sv.y;
                    a[1] = n.z * sv.x - n.x * sv.z;
                    a[2] = n.x * sv.y - n.y * sv.x;
                    a[3] = n.x;
                    a[4] = n.y;
                    a[5] = n.z;
                    b = n.x * d.x + n.y * d.y + n.z * d.z - n.x * sv.x - n.y * sv.y - n.z * sv.z;
                }
            }
        }
        if (in[q] && mask) mask[size_t(vv[q]) * w + u[q]] = good ? 1 : 0;
        if (good) accumulate(a, b);
    }
}

// the 27 distinct products: upper triangle of A^T A row by row, then A^T b
__device__ __forceinline__ void accumulate_products(float acc[32], const float a[6], float b) {
    int k = 0;
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int c = r; c < 6; ++c) acc[k++] += a[r] * a[c];
#pragma unroll
    for (int r = 0; r < 6; ++r) acc[21 + r] += a[r] * b;
}

__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = a + b;
    const float bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

// Reduce 32 slots across the warp.  Each step halves the slots a lane keeps and exchanges the
// other half with its partner, adding with two-sum; lane l ends with the warp total of slot l
// as (sum, compensation).
__device__ __forceinline__ void warp_reduce_scatter(float (&v)[32], float (&c)[32], int lane) {
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        const bool up = (lane & off) != 0;
#pragma unroll
        for (int i = 0; i < off; ++i) {
            const float sv = up ? v[i] : v[i + off];
            const float sc = up ? c[i] : c[i + off];
            const float kv = up ? v[i + off] : v[i];
            const float kc = up ? c[i + off] : c[i];
            const float rv = __shfl_xor_sync(0xffffffffu, sv, off);
            const float rc = __shfl_xor_sync(0xffffffffu, sc, off);
            float s, e;
            two_sum(kv, rv, s, e);
            v[i] = s;
            c[i] = kc + rc + e;
        }
    }
}

// Block reduction of each thread's 27 partial sums to 27 compensated pairs stored at out
// (54 floats).  red: shared scratch of 8 * 32 * 2 floats.  Must be called by all threads.
__device__ __forceinline__ void block_reduce_store(float (&acc)[32], float* red, float* out) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float c[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) c[i] = 0.f;
    warp_reduce_scatter(acc, c, lane);
    red[(warp * 32 + lane) * 2 + 0] = acc[0];
    red[(warp * 32 + lane) * 2 + 1] = c[0];
    __syncthreads();
    if (tid < 27) {
        float s = red[tid * 2 + 0], cc = red[tid * 2 + 1];
        const int nw = blockDim.x >> 5;
        for (int w = 1; w < nw; ++w) {
            float t, e;
            two_sum(s, red[(w * 32 + tid) * 2 + 0], t, e);
            cc += red[(w * 32 + tid) * 2 + 1] + e;
            s = t;
        }
        __stcg(out + 2 * tid + 0, s);
        __stcg(out + 2 * tid + 1, cc);
    }
    __syncthreads();
}

// ---- FP64 solve and pose algebra (thread-level) ----

// Cholesky (LLT) solve of the 6x6 normal equations (the reference: Eigen LLT<float>,
// project/src/linear_least_squares.cpp:41).  Returns false for a non-positive pivot.  Fully
// unrolled so the factor stays in registers; each pivot costs one reciprocal square root and
// the substitutions multiply by it.
__device__ __forceinline__ bool cholesky6(const double (&ata)[36], const double (&atb)[6], double (&x)[6]) {
    double L[6][6], inv[6];
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        double d = ata[j * 6 + j];
#pragma unroll
        for (int k = 0; k < j; ++k) d -= L[j][k] * L[j][k];
        if (!(d > 0.0)) return false;
        inv[j] = rsqrt(d);
#pragma unroll
        for (int i = j + 1; i < 6; ++i) {
            double t = ata[i * 6 + j];
#pragma unroll
            for (int k = 0; k < j; ++k) t -= L[i][k] * L[j][k];
            L[i][j] = t * inv[j];
        }
    }
    double y[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double t = atb[i];
#pragma unroll
        for (int k = 0; k < i; ++k) t -= L[i][k] * y[k];
        y[i] = t * inv[i];
    }
#pragma unroll
    for (int i = 5; i >= 0; --i) {
        double t = y[i];
#pragma unroll
        for (int k = i + 1; k < 6; ++k) t -= L[k][i] * x[k];
        x[i] = t * inv[i];
    }
    bool fin = true;
#pragma unroll
    for (int i = 0; i < 6; ++i) fin = fin && isfinite(x[i]);
    return fin;
}

// glm::orientate3(vec3(beta, alpha, gamma)) of project/src/icp.cpp:82: the Euler composition
// Y * X * Z, i.e. R_y(gamma) R_x(beta) R_z(alpha); column-major out, from the sines and
// cosines of beta (x), gamma (y) and alpha (z)
__device__ __forceinline__ void euler_yxz_sc(double sx, double cx, double sy, double cy, double sz, double cz,
                                             double (&m)[9]) {
    m[0] = cy * cz + sy * sx * sz;  m[1] = cx * sz;  m[2] = -sy * cz + cy * sx * sz;
    m[3] = -cy * sz + sy * sx * cz; m[4] = cx * cz;  m[5] = sy * sz + cy * sx * cz;
    m[6] = sy * cx;                 m[7] = -sx;      m[8] = cy * cx;
}

__device__ __forceinline__ void m3d_vec(const double* m, const double* v, double* o) {
    for (int r = 0; r < 3; ++r) o[r] = m[r] * v[0] + m[3 + r] * v[1] + m[6 + r] * v[2];
}

// the 24 floats phase A of the next pass reads for a session at level Lv: the estimate
// (R, t), M = K_l * R_prev^T and t_prev
__device__ void publish_mats(float* m, const double* R, const double* t, const double* Rp, const float* tpf,
                             const LevelDev& Lv) {
    for (int q = 0; q < 9; ++q) m[q] = float(R[q]);
    for (int q = 0; q < 3; ++q) m[9 + q] = float(t[q]);
    // K = [fx 0 cx; 0 fy cy; 0 0 1];  M = K * Rp^T;  (Rp^T)(r, c) = Rp(c, r) = Rp[r * 3 + c]
    for (int col = 0; col < 3; ++col) {
        // column col of Rp^T = row col of Rp = (Rp[col], Rp[3 + col], Rp[6 + col])
        const double a0 = Rp[col], a1 = Rp[3 + col], a2 = Rp[6 + col];
        m[12 + col * 3 + 0] = float(double(Lv.fx) * a0 + double(Lv.cx) * a2);
        m[12 + col * 3 + 1] = float(double(Lv.fy) * a1 + double(Lv.cy) * a2);
        m[12 + col * 3 + 2] = float(a2);
    }
    for (int q = 0; q < 3; ++q) m[21 + q] = tpf[q];
}

// first ICP level with iterations at or below `from`
__device__ __forceinline__ int next_level(const SessionDev* S, int from) {
    int l = from;
    while (l >= 0 && S->iters[l] <= 0) --l;
    return l;
}

// schedule entry of a session: the level of its next pass and that level's tiles
__device__ __forceinline__ int4 sched_entry(const EngineView& v, int s, int level) {
    if (level < 0) return make_int4(-1, 0, 0, 0);
    const IcpRange rg = v.iranges[level * v.tb->S + s];
    return make_int4(level, rg.begin, rg.end - rg.begin, 0);
}

// Where a session's ICP iteration state lives: in the session's pose block and the engine's
// schedule and matrix arrays (one owner block updates them and a grid barrier publishes
// them), or in a block's shared memory (every block updates its own copy, identically).
struct IcpStateRef {
    double* R;
    double* t;
    int* it;
    int* iters;
    int* level;
    int* cont;
    int* status;
    float* mats;   // the 24 floats phase A reads
    int4* sched;   // the schedule entry of the next pass
};

__device__ __forceinline__ IcpStateRef global_state(const EngineView& v, int s) {
    PoseDev* P = v.sess[s].pose;
    return IcpStateRef{P->R, P->t, &P->it, P->iters, &P->level, &P->cont, &P->status,
                       v.icp_mats + size_t(s) * 24, v.icp_sched + s};
}

struct IcpLocal {
    double R[9], t[3];
    int it, level, cont, status;
    int iters[kMaxLevels];
    float mats[24];
    int4 sched;
};

__device__ __forceinline__ IcpStateRef local_state(IcpLocal& L) {
    return IcpStateRef{L.R, L.t, &L.it, L.iters, &L.level, &L.cont, &L.status, L.mats, &L.sched};
}

// phase 0 for one session (one thread); every slot gets a schedule entry
__device__ void icp_begin(const EngineView& v, int s, const IcpStateRef& ref) {
    const SessionDev* S = &v.sess[s];
    const StepDev st = v.step[s];
    if (!st.active) {   // empty or idle slot: its state is not touched
        *ref.sched = make_int4(-1, 0, 0, 0);
        return;
    }
    const PoseDev* P = S->pose;
    *ref.status = KF_OK;
    for (int l = 0; l < kMaxLevels; ++l) ref.iters[l] = 0;
    *ref.it = 0;
    int level = -1;
    if (!st.first) {
        for (int q = 0; q < 9; ++q) ref.R[q] = P->Rp[q];
        for (int q = 0; q < 3; ++q) ref.t[q] = P->tp[q];
        level = next_level(S, S->L - 1);
        if (level >= 0) publish_mats(ref.mats, P->Rp, P->tp, P->Rp, P->tpf, S->lv[level]);
    }
    *ref.level = level;
    *ref.cont = level >= 0 ? 1 : 0;
    *ref.sched = sched_entry(v, s, level);
    // no fence here: thread 0 writes all of this, and the grid barrier that follows fences
    // thread 0's writes before it arrives
}

// phase B for one session: FP64 combine of the tile pairs, solve, update, stop test
// (ICP::computePose loop body, project/src/icp.cpp:36-54).  All threads of the block call it.
// sm: 19 * 28 doubles of shared scratch.  Warp 0 runs the solve redundantly on every lane
// (identical values), so the three sines and cosines are computed on three lanes at once and
// no lane waits on another through memory; lane 0 stores the results.
template <bool kLocal>
__device__ void icp_solve(const EngineView& v, int s, int level, int begin, int cnt, double* sm,
                          const float* parts, IcpLocal* loc) {
    const IcpStateRef ref = kLocal ? local_state(*loc) : global_state(v, s);
    const SessionDev* S = &v.sess[s];
    const PoseDev* P = S->pose;
    const int tid = threadIdx.x, lane = tid & 31;
    // warp 0 fetches everything the update needs while the block sums the tiles
    double R0[9], t0[3], Rp[9];
    int it0 = 0, done0 = 0, S_cap = 0, siters[kMaxLevels];
    float stop_a = 0.f, stop_d = 0.f, tpf[3], lfx[kMaxLevels], lfy[kMaxLevels], lcx[kMaxLevels], lcy[kMaxLevels];
    IcpRange rng[kMaxLevels];
    if (tid < 32) {
#pragma unroll
        // the state was written by this block's thread 0 (ordered by the block barriers)
        for (int q = 0; q < 9; ++q) { R0[q] = ref.R[q]; Rp[q] = ldcg(&P->Rp[q]); }
#pragma unroll
        for (int q = 0; q < 3; ++q) { t0[q] = ref.t[q]; tpf[q] = ldcg(&P->tpf[q]); }
        it0 = *ref.it;
        done0 = ref.iters[level];
        S_cap = v.tb->S;
        stop_a = S->stop_a;
        stop_d = S->stop_d;
#pragma unroll
        for (int l = 0; l < kMaxLevels; ++l) {
            siters[l] = S->iters[l];
            lfx[l] = S->lv[l].fx; lfy[l] = S->lv[l].fy; lcx[l] = S->lv[l].cx; lcy[l] = S->lv[l].cy;
        }
#pragma unroll
        for (int l = 0; l < kMaxLevels; ++l) rng[l] = v.iranges[l * S_cap + s];
    }
    // partial pairs as float4 (two entries each): thread (g, q) adds, in FP64 and in tile
    // order, entries 2q and 2q + 1 of tiles g, g + 18, g + 36, ...; 9 tiles' loads in flight,
    // so up to 162 partials (a grid of one block per SM) arrive in one round trip
    constexpr int kGroups = kIcpThreads / 14;   // 18
    const int q = tid % 14, g = tid / 14;
    if (g < kGroups) {
        const float4* src = reinterpret_cast<const float4*>(parts + size_t(begin) * kIcpPartialStride) + q;
        double a0 = 0.0, a1 = 0.0;
        for (int t = g; t < cnt; t += 9 * kGroups) {
            float4 p[9];
#pragma unroll
            for (int u = 0; u < 9; ++u) {
                const float4* a = src + size_t(t + kGroups * u) * (kIcpPartialStride / 4);
                p[u] = t + kGroups * u < cnt ? __ldcg(a) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < 9; ++u)
                if (t + kGroups * u < cnt) {
                    a0 += double(p[u].x) + double(p[u].y);
                    a1 += double(p[u].z) + double(p[u].w);
                }
        }
        sm[g * 28 + 2 * q] = a0;
        sm[g * 28 + 2 * q + 1] = a1;
    }
    __syncthreads();
    if (tid < 27) {
        double a = 0.0;
        for (int r = 0; r < kGroups; ++r) a += sm[r * 28 + tid];
        sm[kGroups * 28 + tid] = a;
    }
    __syncthreads();
    if (tid >= 32) return;
    const double* tot = sm + kGroups * 28;
    double ata[36], atb[6];
    {
        int k = 0;
#pragma unroll
        for (int r = 0; r < 6; ++r)
#pragma unroll
            for (int c = r; c < 6; ++c) { ata[r * 6 + c] = tot[k]; ata[c * 6 + r] = tot[k]; ++k; }
#pragma unroll
        for (int r = 0; r < 6; ++r) atb[r] = tot[21 + r];
    }
    double x[6];
    const bool solved = cholesky6(ata, atb, x);   // warp-uniform
    if (!solved) {
        if (lane == 0) {
            // the reference throws (project/src/icp.cpp:67-73): keep the previous pose, no fusion
            *ref.status = KF_ERR_NONFINITE;
            *ref.level = -1;
            *ref.cont = 0;
            *ref.sched = make_int4(-1, 0, 0, 0);   // published by the barrier's fence
        }
        return;
    }
    // sin / cos of beta (x[0]), gamma (x[1]), alpha (x[2]) on lanes 0, 1, 2
    double sn = 0.0, cs = 1.0;
    if (lane < 3) sincos(x[lane], &sn, &cs);
    const double sx = __shfl_sync(0xffffffffu, sn, 0), cx = __shfl_sync(0xffffffffu, cs, 0);
    const double sy = __shfl_sync(0xffffffffu, sn, 1), cy = __shfl_sync(0xffffffffu, cs, 1);
    const double sz = __shfl_sync(0xffffffffu, sn, 2), cz = __shfl_sync(0xffffffffu, cs, 2);
    double dR[9], R1[9], t1[3];
    euler_yxz_sc(sx, cx, sy, cy, sz, cz, dR);
    // R <- dR^T R, t <- dR^T t + dt (ICP::updatePose, project/src/icp.cpp:85-86)
    double dRt[9];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 3; ++r) dRt[c * 3 + r] = dR[r * 3 + c];
#pragma unroll
    for (int c = 0; c < 3; ++c) m3d_vec(dRt, R0 + 3 * c, R1 + 3 * c);
    double nt[3];
    m3d_vec(dRt, t0, nt);
#pragma unroll
    for (int r = 0; r < 3; ++r) t1[r] = nt[r] + x[3 + r];
    // poseError(previous estimate, new estimate) (project/src/general_helper.cpp:11-21)
    const double iv = 0.57735026918962576451;
    double a0[3], a1[3], vv[3] = {iv, iv, iv};
    m3d_vec(R0, vv, a0);
    m3d_vec(R1, vv, a1);
    const double ang = sqrt((a0[0] - a1[0]) * (a0[0] - a1[0]) + (a0[1] - a1[1]) * (a0[1] - a1[1]) +
                            (a0[2] - a1[2]) * (a0[2] - a1[2]));
    const double dist = sqrt((t0[0] - t1[0]) * (t0[0] - t1[0]) + (t0[1] - t1[1]) * (t0[1] - t1[1]) +
                             (t0[2] - t1[2]) * (t0[2] - t1[2]));
    int it = it0 + 1;
    int lvl = level;
    if ((ang < double(stop_a) && dist < double(stop_d)) || it >= siters[level]) {
        lvl = level - 1;   // next level with iterations (next_level)
        while (lvl >= 0 && siters[lvl] <= 0) --lvl;
        it = 0;
    }
    if (lane != 0) return;
#pragma unroll
    for (int r = 0; r < 9; ++r) ref.R[r] = R1[r];
#pragma unroll
    for (int r = 0; r < 3; ++r) ref.t[r] = t1[r];
    ref.iters[level] = done0 + 1;
    *ref.it = it;
    *ref.level = lvl;
    *ref.cont = lvl >= 0 ? 1 : 0;
    if (lvl >= 0) {
        float* m = ref.mats;
#pragma unroll
        for (int r = 0; r < 9; ++r) m[r] = float(R1[r]);
#pragma unroll
        for (int r = 0; r < 3; ++r) m[9 + r] = float(t1[r]);
        // M = K_l * Rp^T (as publish_mats)
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            const double b0 = Rp[col], b1 = Rp[3 + col], b2 = Rp[6 + col];
            m[12 + col * 3 + 0] = float(double(lfx[lvl]) * b0 + double(lcx[lvl]) * b2);
            m[12 + col * 3 + 1] = float(double(lfy[lvl]) * b1 + double(lcy[lvl]) * b2);
            m[12 + col * 3 + 2] = float(b2);
        }
#pragma unroll
        for (int r = 0; r < 3; ++r) m[21 + r] = tpf[r];
        *ref.sched = make_int4(lvl, rng[lvl].begin, rng[lvl].end - rng[lvl].begin, 0);
    } else {
        *ref.sched = make_int4(-1, 0, 0, 0);
    }
    // lane 0 of warp 0 is thread 0, whose writes the grid barrier after phase B fences
}

// phase C for one session (one thread): the frame's pose becomes the previous pose; the
// inverse feeds fusion; the result block goes to the host.
__device__ void icp_finish(const SessionDev* S, const StepDev st, OutDev* out) {
    if (!st.active) return;
    PoseDev* P = S->pose;
    const bool ok = P->status == KF_OK;
    if (ok && !st.first) {
        for (int q = 0; q < 9; ++q) P->Rp[q] = P->R[q];
        for (int q = 0; q < 3; ++q) P->tp[q] = P->t[q];
    }
    for (int q = 0; q < 9; ++q) P->Rpf[q] = float(P->Rp[q]);
    for (int q = 0; q < 3; ++q) P->tpf[q] = float(P->tp[q]);
    // inverse: R^T, -R^T t
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) P->iRf[c * 3 + r] = float(P->Rp[r * 3 + c]);
    for (int r = 0; r < 3; ++r)
        P->itf[r] = float(-(P->Rp[r * 3 + 0] * P->tp[0] + P->Rp[r * 3 + 1] * P->tp[1] + P->Rp[r * 3 + 2] * P->tp[2]));
    P->fuse_ok = ok ? 1 : 0;
    P->frame += 1;
    for (int q = 0; q < 16; ++q) out->pose[q] = 0.f;
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) out->pose[c * 4 + r] = P->Rpf[c * 3 + r];
    for (int r = 0; r < 3; ++r) out->pose[12 + r] = P->tpf[r];
    out->pose[15] = 1.f;
    for (int l = 0; l < kMaxLevels; ++l) out->iters[l] = P->iters[l];
    out->status = P->status;
    out->frame = P->frame;
    __threadfence();
}

// In-place inclusive scan of a[0..n) in shared memory by the whole block (n <= 1024).
__device__ void block_inclusive_scan(int* a, int n, int* warp_tot) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nthreads = blockDim.x;
    const int per = (n + nthreads - 1) / nthreads;
    const int lo = min(n, tid * per), hi = min(n, lo + per);
    int run = 0;
    for (int i = lo; i < hi; ++i) run += a[i];
    int incl = run;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += y;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (tid == 0) {
        int acc = 0;
        for (int w = 0; w < (nthreads >> 5); ++w) { const int x = warp_tot[w]; warp_tot[w] = acc; acc += x; }
    }
    __syncthreads();
    int base = warp_tot[warp] + incl - run;   // exclusive prefix of this thread's chunk
    for (int i = lo; i < hi; ++i) { base += a[i]; a[i] = base; }
    __syncthreads();
}

// ---- the persistent cooperative kernel ----

constexpr int kIcpMaxSessionsSmem = 1024;
constexpr int kIcpPixelsPerStep = 4;   // pixels a thread carries through one pipelined step

// Phase A of one group: tiles g, g + G, ... of a session at one level, accumulated by the whole
// block in tile order (each thread its pixels p0 + tid, p0 + tid + 256, ... of each tile), then
// reduced to one compensated partial at `out`.  The partial depends on the group's tiles only,
// not on which block or launch computes it.
__device__ __forceinline__ void icp_group(const EngineView& v, int s, int lvl, int tile0, int ntiles, int g, int G,
                                          const float* mats, float* red, float* out) {
    float acc[32];
#pragma unroll
    for (int q = 0; q < 32; ++q) acc[q] = 0.f;
    const SessionDev* S = &v.sess[s];
    const LevelDev& Lv = S->lv[lvl];
    const float4* vm = S->vmap[lvl];
    const float4* tv = S->pv[lvl];
    const float4* tn = S->pn[lvl];
    uint8_t* mask = S->mask[lvl];
    const float dist = S->dist_th, ang = S->angle_cos;
    const IcpMats m{mats, mats + 9, mats + 12, mats + 21};
    for (int j = g; j < ntiles; j += G) {
        const IcpTile T = v.itiles[tile0 + j];
        const int pend = T.p0 + T.np;
#pragma unroll 1
        for (int p = T.p0 + threadIdx.x; p < pend; p += kIcpPixelsPerStep * kIcpThreads)
            icp_multi<kIcpPixelsPerStep>(vm, tv, tn, Lv.w, Lv.h, Lv.icw, p, pend, m, dist, ang, mask,
                                         [&](const float (&a)[6], float b) { accumulate_products(acc, a, b); });
    }
    block_reduce_store(acc, red, out);
}

// thread 0: the block-local state goes back to the session's pose block
__device__ void store_local_state(PoseDev* P, const IcpLocal& L, bool first) {
    if (!first) {   // a first frame has no estimate (fusion only)
        for (int q = 0; q < 9; ++q) P->R[q] = L.R[q];
        for (int q = 0; q < 3; ++q) P->t[q] = L.t[q];
    }
    for (int l = 0; l < kMaxLevels; ++l) P->iters[l] = L.iters[l];
    P->it = L.it;
    P->level = L.level;
    P->cont = L.cont;
    P->status = L.status;
}

// A batch's launch holds two blocks per SM (128 registers; the solve, run once per session
// and pass, spills a little): twice the warps to hide phase A's gathers.  A single session's
// keeps one block per SM, the solve in registers: every block runs it on every pass.
template <bool local>
__global__ void __launch_bounds__(kIcpThreads, local ? 1 : 2) icp_kernel(EngineView v) {
    __shared__ float red[8 * 32 * 2];
    __shared__ double dsm[(kIcpThreads / 14 + 1) * 28];
    __shared__ float mats[24];
    __shared__ int s_pre[kIcpMaxSessionsSmem + 1];   // groups of sessions before s in this pass
    __shared__ short s_lvl[kIcpMaxSessionsSmem];
    __shared__ int s_beg[kIcpMaxSessionsSmem];
    __shared__ int s_cnt[kIcpMaxSessionsSmem];       // tiles of session s at its level
    __shared__ int s_wtot[kIcpThreads / 32];
    __shared__ IcpLocal loc;
    const int tid = threadIdx.x;
    const unsigned int nb = gridDim.x;
    unsigned int epoch = 0;
    const int S_cap = v.tb->S;
    // local (an engine of one session): every block runs the session's solve itself (the same arithmetic on the
    // same partials, so every block's copy of the state is identical) and goes straight on to
    // the next pass -- one grid barrier per pass instead of two.  The partials of consecutive
    // passes go to alternate buffers, since a block may start writing the next pass's
    // partials while another still sums this pass's; a block two passes on has passed a
    // barrier that every block reaches only after its solve.

    if (local) {
        if (tid == 0) icp_begin(v, 0, local_state(loc));
        __syncthreads();
    } else {
        for (int s = blockIdx.x; s < S_cap; s += gridDim.x)
            if (tid == 0) icp_begin(v, s, global_state(v, s));
        if (!grid_barrier(v.sync, nb, epoch)) return;
    }

    for (int pass = 0; pass < kIcpMaxPasses; ++pass) {
        float* const parts = (local && (pass & 1)) ? v.partials2 : v.partials;
        // which sessions iterate in this pass, at which level, with which tiles and groups
        for (int s = tid; s < S_cap; s += blockDim.x) {
            const int4 e = local ? loc.sched : __ldcg(v.icp_sched + s);
            s_lvl[s] = short(e.x);
            s_beg[s] = e.y;
            s_cnt[s] = e.z;
            s_pre[s + 1] = e.x >= 0 ? min(e.z, kIcpGroups) : 0;
        }
        if (tid == 0) s_pre[0] = 0;
        __syncthreads();
        if (!local) block_inclusive_scan(s_pre + 1, S_cap, s_wtot);   // one slot: s_pre[1] is its own count
        const int total = s_pre[S_cap];
        if (total == 0) break;   // block-uniform: every block reads the same schedule

        // phase A: the groups of every iterating session, round robin over the grid; group g of
        // session s stores its partial in slot g of the session's tiles
        {
            int cur_s = -1;
            for (int vt = blockIdx.x; vt < total; vt += gridDim.x) {
                int lo = 0, hi = S_cap;
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (s_pre[mid] <= vt) lo = mid; else hi = mid;
                }
                const int s = lo, lvl = s_lvl[s], g = vt - s_pre[s];
                if (s != cur_s) {
                    cur_s = s;
                    __syncthreads();   // the previous group's threads are done with mats
                    if (tid < 24) mats[tid] = local ? loc.mats[tid] : ldcg(v.icp_mats + size_t(s) * 24 + tid);
                    __syncthreads();
                }
                icp_group(v, s, lvl, s_beg[s], s_cnt[s], g, kIcpGroups, mats, red,
                                 parts + size_t(s_beg[s] + g) * kIcpPartialStride);
            }
        }
        if (!grid_barrier(v.sync, nb, epoch)) return;

        if constexpr (local) {
            // phase B in every block, on its own copy of the state
            if (s_lvl[0] >= 0) icp_solve<true>(v, 0, s_lvl[0], s_beg[0], s_pre[1], dsm, parts, &loc);
            __syncthreads();
        } else {
            // phase B: the block that owns a session solves it
            for (int s = blockIdx.x; s < S_cap; s += gridDim.x) {
                if (s_lvl[s] < 0) continue;
                icp_solve<false>(v, s, s_lvl[s], s_beg[s], s_pre[s + 1] - s_pre[s], dsm, parts, nullptr);
                __syncthreads();
            }
            if (!grid_barrier(v.sync, nb, epoch)) return;
        }
    }

    if constexpr (local) {
        // block 0 stores the state the rest of the frame and the host read
        if (blockIdx.x == 0 && tid == 0 && v.step[0].active) {
            store_local_state(v.sess[0].pose, loc, v.step[0].first != 0);
            icp_finish(&v.sess[0], v.step[0], v.out);
        }
    } else {
        for (int s = blockIdx.x; s < S_cap; s += gridDim.x)
            if (tid == 0) icp_finish(&v.sess[s], v.step[s], v.out + s);
    }
}

int icp_max_grid(int num_sms) { return 2 * num_sms; }

// Bounded-wait self test: a two-block cooperative launch in which block 1 never arrives at
// the barrier block 0 waits on.  The wait gives up after timeout_ns, sets the abort flag and
// records the outcome; nothing spins past the limit.
__global__ void barrier_selftest_kernel(GridSync* g, unsigned long long timeout_ns, int* result) {
    unsigned int epoch = 0;
    if (blockIdx.x == 0) {
        const bool ok = grid_barrier(g, gridDim.x, epoch, timeout_ns);
        if (threadIdx.x == 0) *result = ok ? 1 : 0;
    }
}

cudaError_t launch_barrier_selftest(GridSync* g, unsigned long long timeout_ns, int* result, cudaStream_t st) {
    void* args[] = {&g, &timeout_ns, &result};
    return cudaLaunchCooperativeKernel((const void*)barrier_selftest_kernel, dim3(2), dim3(32), args, 0, st);
}

cudaError_t launch_icp(const EngineView& v, int grid, cudaStream_t st, bool single) {
    void* args[] = {const_cast<EngineView*>(&v)};
    const void* k = single ? (const void*)icp_kernel<true> : (const void*)icp_kernel<false>;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (single) grid = std::min(grid, sms);   // one co-resident block per SM
    return cudaLaunchCooperativeKernel(k, dim3(grid), dim3(kIcpThreads), args, 0, st);
}

// ---- stage: kernel::constructIcpResiduals (A rows and b to HBM, as the reference) ----

struct IcpStageMats { float R[9], t[3], M[9], tp[3]; };

__global__ void icp_rows_kernel(const float4* vm, const float4* tv, const float4* tn, int w, int h, IcpStageMats m,
                                float dist, float cos_th, float* A, float* b) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x, vv = blockIdx.y * blockDim.y + threadIdx.y;
    if (u >= w || vv >= h) return;
    float a[6], bb;
    const bool ok = icp_pixel(vm, tv, tn, w, h, u, vv, m.R, m.t, m.M, m.tp, dist, cos_th, a, bb);
    const size_t idx = size_t(vv) * w + u;
    for (int q = 0; q < 6; ++q) A[idx * 6 + q] = ok ? a[q] : 0.f;
    b[idx] = ok ? bb : 0.f;
}

cudaError_t stage_icp_residuals(const float4* vmap, const float4* tv, const float4* tn, int w, int h,
                                const float* Rp, const float* tp, const float* Rc, const float* tc, const float* k,
                                float dist, float angle, float* A, float* b, cudaStream_t st) {
    IcpStageMats m;
    for (int q = 0; q < 9; ++q) m.R[q] = Rc[q];
    for (int q = 0; q < 3; ++q) { m.t[q] = tc[q]; m.tp[q] = tp[q]; }
    // M = K * Rp^T with K the caller's full 3x3 (column-major)
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 3; ++row) {
            float acc = 0.f;
            for (int q = 0; q < 3; ++q) acc += k[q * 3 + row] * Rp[q * 3 + col];   // K(row,q) * Rp^T(q,col) = K(row,q) * Rp(col,q)
            m.M[col * 3 + row] = acc;
        }
    dim3 blk(16, 16), grd((w + 15) / 16, (h + 15) / 16);
    const float cos_th = float(std::cos(double(angle)));
    icp_rows_kernel<<<grd, blk, 0, st>>>(vmap, tv, tn, w, h, m, dist, cos_th, A, b);
    return cudaGetLastError();
}

// ---- stage: LinearLeastSquares::solve on A (n x 6, row-major) and b in device memory ----

int lls_num_blocks(int n) {
    const int per = kIcpTilePx;
    int nb = (n + per - 1) / per;
    if (nb < 1) nb = 1;
    if (nb > 148 * 4) nb = 148 * 4;
    return nb;
}

__global__ void __launch_bounds__(kIcpThreads) lls_partials_kernel(const float* A, const float* b, int n,
                                                                   float* partials) {
    __shared__ float red[8 * 32 * 2];
    float acc[32];
#pragma unroll
    for (int q = 0; q < 32; ++q) acc[q] = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float a[6];
        for (int q = 0; q < 6; ++q) a[q] = A[size_t(i) * 6 + q];
        accumulate_products(acc, a, b[i]);
    }
    block_reduce_store(acc, red, partials + size_t(blockIdx.x) * 54);
}

__global__ void lls_solve_kernel(const float* partials, int nblocks, double* x_out) {
    __shared__ double sm[8 * 27];
    const int tid = threadIdx.x;
    if (tid < 8 * 27) {
        const int k = tid % 27, g = tid / 27;
        double acc = 0.0;
        for (int t = g; t < nblocks; t += 8) acc += double(partials[size_t(t) * 54 + 2 * k]) + double(partials[size_t(t) * 54 + 2 * k + 1]);
        sm[g * 27 + k] = acc;
    }
    __syncthreads();
    if (tid == 0) {
        double tot[27];
        for (int k = 0; k < 27; ++k) {
            double a = 0.0;
            for (int g = 0; g < 8; ++g) a += sm[g * 27 + k];
            tot[k] = a;
        }
        double ata[36], atb[6], x[6];
        int k = 0;
        for (int r = 0; r < 6; ++r)
            for (int c = r; c < 6; ++c) { ata[r * 6 + c] = tot[k]; ata[c * 6 + r] = tot[k]; ++k; }
        for (int r = 0; r < 6; ++r) atb[r] = tot[21 + r];
        if (!cholesky6(ata, atb, x))
            for (int q = 0; q < 6; ++q) x[q] = __longlong_as_double(0x7ff8000000000000ll);
        for (int q = 0; q < 6; ++q) x_out[q] = x[q];
    }
}

cudaError_t stage_lls(const float* A, const float* b, int n, float* partials, double* x_dev, int nblocks,
                      cudaStream_t st) {
    lls_partials_kernel<<<nblocks, kIcpThreads, 0, st>>>(A, b, n, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    lls_solve_kernel<<<1, 256, 0, st>>>(partials, nblocks, x_dev);
    return cudaGetLastError();
}

}  // namespace kf

// ---- kf_solve_linear_least_squares_noalloc: the same two kernels on a fixed scratch ----
//
// The scratch is this file's static device array: the partial sums of up to 512 blocks
// (KF_LLS_NOALLOC_MAX_ROWS rows / 2048 rows per block, 54 floats each) followed by the FP64
// solution (6 doubles), 110,640 bytes, part of the library's device image.  For
// n <= KF_LLS_NOALLOC_MAX_ROWS, lls_num_blocks(n) is the same block count the allocating
// entry point uses, so both reduce in the same order.  Each call writes every partial slot
// it reads and the solution before reading them: nothing has to start at zero.  One scratch
// per device, shared by all calls on it: overlapping calls race.

namespace {
constexpr int kNaMaxBlocks = KF_LLS_NOALLOC_MAX_ROWS / kf::kIcpTilePx;
constexpr int kNaXOffset = kNaMaxBlocks * 54;        // in floats; the solution follows the partials
constexpr int kNaFloats = kNaXOffset + 2 * 6;        // 6 doubles
constexpr int kNaMaxDevices = 64;
static_assert(kNaMaxBlocks * kf::kIcpTilePx == KF_LLS_NOALLOC_MAX_ROWS, "row limit is a whole number of blocks");
static_assert(kNaMaxBlocks <= 148 * 4, "lls_num_blocks does not clamp below the limit");
static_assert(kNaXOffset % 2 == 0, "the FP64 solution is 8-byte aligned");
static_assert(sizeof(float) * kNaFloats == 110640, "scratch size stated in kf_api.h");

std::mutex g_na_mu;                        // guards the one-time set-up only
float* g_na_base[kNaMaxDevices] = {};      // device address of the scratch, per device ordinal
}  // namespace

static __device__ __align__(256) float g_lls_noalloc_scratch[kNaFloats];

extern "C" kf_status kf_solve_linear_least_squares_noalloc(const float* mat_a, const float* vec_b, int n,
                                                           float x_out[6], void* stream) {
    if (!mat_a || !vec_b || !x_out || n <= 0) return KF_ERR_ARG;
    if (n > KF_LLS_NOALLOC_MAX_ROWS) return KF_ERR_TOO_LARGE;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return KF_ERR_CUDA;
    if (dev < 0 || dev >= kNaMaxDevices) return KF_ERR_ARG;
    float* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_na_mu);
        if (!g_na_base[dev]) {
            // set-up, once per device, with that device current
            float* ptr = nullptr;
            if (cudaGetSymbolAddress((void**)&ptr, g_lls_noalloc_scratch) != cudaSuccess || !ptr) return KF_ERR_CUDA;
            g_na_base[dev] = ptr;
        }
        base = g_na_base[dev];
    }
    const int nb = kf::lls_num_blocks(n);
    if (nb > kNaMaxBlocks) return KF_ERR_TOO_LARGE;
    double* x_dev = reinterpret_cast<double*>(base + kNaXOffset);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (kf::stage_lls(mat_a, vec_b, n, base, x_dev, nb, st) != cudaSuccess) return KF_ERR_CUDA;
    double x[6];
    if (cudaMemcpyAsync(x, x_dev, sizeof(x), cudaMemcpyDeviceToHost, st) != cudaSuccess) return KF_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return KF_ERR_CUDA;
    for (int q = 0; q < 6; ++q) x_out[q] = float(x[q]);
    for (int q = 0; q < 6; ++q)
        if (!isfinite(x[q])) return KF_ERR_NONFINITE;
    return KF_OK;
}
