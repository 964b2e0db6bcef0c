// k_raycast.cu -- predicted vertex / normal maps by ray marching the TSDF.
//
// Reference: raycastKernel (project/src/raycast.cu:44-145) with intersectBBox (:7-27) and
// computeGradient (:29-42), called once per pyramid level at the previous frame's pose
// (project/src/kinect_fusion.cpp:137-144).  The reference samples a cudaArray through the
// texture unit; here the distance array stays in linear HBM (x fastest), so fusion can stream
// it, and the march does its own trilinear interpolation with the reference's texel mapping
// (uvw * n - 0.5, clamp).  The march takes the reference's samples in the reference's order,
// with one difference in arithmetic: the reference forms each position by adding the step to
// the last one (t <- t + inc, project/src/raycast.cu:78), so float rounding drifts along a ray
// (up to ~1e-4 m over a grazing ray of a thousand small steps, which moves its hit by up to a
// millimetre); here sample k of a phase is at base + k * inc with a single rounding, where base
// is the near distance, the sample that left large steps, or t - mu after a back-off.  That is
// the FP64 march's position to within a rounding, and any sample's position is known without
// the ones before it.  Three things make the march fast:
//   - Skipping: a sample whose eight taps lie in cells (32^3 super-bricks, then 8^3 bricks)
//     whose distance lower bound proves it cannot change the march (>= 0.991 during large
//     steps, >= 0.001 during small steps) is not evaluated, nor is any later sample in the
//     same cell; the march jumps to the first sample index past the cell.  A skip that starts
//     in a skippable super-brick continues through up to three more skippable super-bricks
//     along the ray (a run; longer runs let one lane hold its warp too long).  Rays that pass
//     within mu of a surface without crossing it keep 0.1 mu steps to the far plane (the
//     reference never returns to large steps); super-bricks let them cross free space 94 steps
//     at a time.
//   - Load balance: each warp pulls 8 x 4-ray tiles from an atomic counter, and a lane marches
//     at most 40 iterations (64 in steps of many sessions); longer rays are queued with their
//     exact march state.
//   - Long rays: a second kernel marches each queued ray with a whole warp, 32 consecutive
//     samples per round (64 after a round in which nothing changed), taking the first sample
//     (in order) that changes the state.
#include "kf_host.h"

namespace kf {

constexpr int kMaxMarchSamples = 1 << 16;
// loop iterations a lane marches before queueing the ray: a short budget keeps the tail of a
// single session's frame short; steps of many sessions hand off fewer rays with a longer one
constexpr int kSerialBudgetSingle = 40;
constexpr int kSerialBudgetMany = 64;
constexpr int kManyRayTiles = 25000;   // more ray tiles than this in a step: kSerialBudgetMany
// skippable super-bricks one skip may cross: 4 cuts the raycast's thread instructions by a
// third and is 8 % faster for 32 sessions; longer runs hold a lane's warp too long (a single
// session is 4 % slower at 8, 7 % at 16)
constexpr int kRunCells = 4;

bool many_ray_tiles(int ray_tiles) { return ray_tiles > kManyRayTiles; }
int serial_budget_many() { return kSerialBudgetMany; }
int serial_budget(int ray_tiles) { return many_ray_tiles(ray_tiles) ? kSerialBudgetMany : kSerialBudgetSingle; }

struct RayGeo {
    F3 o, dir;
    float sc, off;                            // texel coordinate = (o + dir t) * sc + off
    float tox, toy, toz, tdx, tdy, tdz;       // the same as an affine function of t
    float itdx, itdy, itdz;
};

// march state: everything the reference's loop carries from one sample to the next
struct RayState {
    float t;          // position of the next sample: base + idx * inc, one rounding
    float base;       // start of the current phase of the march
    float prev, prev_t, near_d, far_d;
    int idx;          // index of the next sample within the phase
    int small;        // 0 while stepping by 1.99 mu, 1 once stepping by 0.1 mu
    int prev_known;   // 0 when the last non-negative sample was skipped (value not computed)
    int guard;        // samples taken (hard bound)
    int sw;           // (samples taken when large steps ended) << 2 | how: 1 below 0.99, 2 negative
};

// position of sample k of the phase that starts at base
__device__ __forceinline__ float march_pos(float base, int k, float inc) { return __fmaf_rn(float(k), inc, base); }

// enter small steps: the next sample is base + inc (the sample that left large steps, or
// t - mu after a back-off, is the new base)
__device__ __forceinline__ void begin_small(RayState& st, float base, float small) {
    st.small = 1;
    st.base = base;
    st.idx = 1;
    st.t = march_pos(base, 1, small);
}

// The march's decision trace of one ray (written only in debug mode), so that a test can tell
// rays whose march took the same decisions as another implementation's from rays where a sample
// near 0.99 or 0 decided differently:
//   bits 40..  samples taken when the march left large steps (0: it never did)
//   bits  8..39 samples taken when the march ended (skipped samples count as taken)
//   bits  4..5  how it left large steps: 1 a sample in [0, 0.99), 2 a negative one (back-off)
//   bits  0..1  how it ended: 0 past the far plane or the sample bound, 1 negative first
//               sample, 2 refined hit
// A ray that returns before marching has trace 0.
__device__ __forceinline__ unsigned long long ray_trace_code(const RayState& st, float precise) {
    const int end = precise != 0.0f ? 2 : (st.t < st.far_d && st.guard < kMaxMarchSamples ? 1 : 0);
    return (static_cast<unsigned long long>(st.sw >> 2) << 40) | (static_cast<unsigned long long>(st.guard) << 8) |
           static_cast<unsigned long long>((st.sw & 3) << 4) | static_cast<unsigned long long>(end);
}

// Work counts of the march, kept only by the kernels' counting instantiation (debug mode
// KF_DEBUG_COUNTERS); the production instantiation compiles every count away.
enum RayCount {
    kCntRays = 0,        // rays that marched
    kCntEvalLarge,       // samples evaluated (trilinear) during large steps
    kCntEvalSmall,       // samples evaluated during small steps
    kCntSkips,           // cell skips (each jumps over one or more samples)
    kCntSkipped,         // samples jumped over by the skips
    kCntGrad,            // gradient samples of hits (six per refined hit)
    kCntQueued,          // rays handed from a lane to the long-ray warp kernel
    kCntRounds,          // warp rounds of the long-ray kernel (32 or 64 samples each)
    kRayCounts
};

template <bool kOn> struct MarchCount {
    __device__ __forceinline__ void add(int, unsigned int) {}
    __device__ __forceinline__ void flush(unsigned long long*) {}
};
template <> struct MarchCount<true> {
    unsigned int c[kRayCounts] = {};
    __device__ __forceinline__ void add(int k, unsigned int x) { c[k] += x; }
    __device__ __forceinline__ void flush(unsigned long long* dst) {
        if (!dst) return;
#pragma unroll
        for (int k = 0; k < kRayCounts; ++k)
            if (c[k]) atomicAdd(dst + k, static_cast<unsigned long long>(c[k]));
    }
};

// a ray handed from a lane to a warp: where it is, its exact march state and its geometry (so
// the warp neither reloads the pose nor divides again)
struct __align__(16) LongRay {
    int s, level, i, j;
    RayState st;
    RayGeo g;
};

__device__ __forceinline__ void ray_matrix(const SessionDev* S, const LevelDev& Lv, float* m, F3& o) {
    // R_prev * K_l^-1 (the reference forms mat3(pose) * invK per ray), each product and sum
    // rounded on its own -- the same arithmetic as the host's for the stage raycast, so that a
    // stage raycast of a session's volume at its pose takes the session's rays bit for bit
    const float* R = S->pose->Rpf;
#pragma unroll
    for (int col = 0; col < 3; ++col)
#pragma unroll
        for (int row = 0; row < 3; ++row)
            m[col * 3 + row] = __fadd_rn(__fadd_rn(__fmul_rn(R[row], Lv.ik[col * 3 + 0]),
                                                   __fmul_rn(R[3 + row], Lv.ik[col * 3 + 1])),
                                         __fmul_rn(R[6 + row], Lv.ik[col * 3 + 2]));
    o = F3{S->pose->tpf[0], S->pose->tpf[1], S->pose->tpf[2]};
}

// ray through pixel (i, j): direction (R K^-1)(i + .5, j + .5, 1), not normalised, so t is
// camera depth
__device__ __forceinline__ void make_geo(const SessionDev* S, const float* m, F3 o, int i, int j, RayGeo& g) {
    g.o = o;
    g.dir = mv3(m, F3{float(i) + 0.5f, float(j) + 0.5f, 1.0f});
    g.sc = float(S->n) / S->vol_w;
    g.off = 0.5f * float(S->n) - 0.5f;
    g.tox = o.x * g.sc + g.off; g.toy = o.y * g.sc + g.off; g.toz = o.z * g.sc + g.off;
    g.tdx = g.dir.x * g.sc; g.tdy = g.dir.y * g.sc; g.tdz = g.dir.z * g.sc;
    // only the skips' cell exits use these, 0.01 texel inside the faces: the fast reciprocal's
    // 2 ulp cannot move a skip across a sample
    g.itdx = __fdividef(1.0f, g.tdx); g.itdy = __fdividef(1.0f, g.tdy); g.itdz = __fdividef(1.0f, g.tdz);
}

// texel coordinate of the sample at t, (o + dir t) * sc + off, with its roundings spelled out
// (two fused multiply-adds): a sample's value must not depend on which kernel, or which
// branch of the march, evaluates it, since its comparison with 0.99 or 0 decides the march
__device__ __forceinline__ void texel(const RayGeo& g, float t, float& x, float& y, float& z) {
    x = __fmaf_rn(__fmaf_rn(g.dir.x, t, g.o.x), g.sc, g.off);
    y = __fmaf_rn(__fmaf_rn(g.dir.y, t, g.o.y), g.sc, g.off);
    z = __fmaf_rn(__fmaf_rn(g.dir.z, t, g.o.z), g.sc, g.off);
}

template <class TF>
__device__ __forceinline__ float sample_at(const SessionDev* S, const RayGeo& g, const TF* f, float t) {
    float x, y, z;
    texel(g, t, x, y, z);
    return trilinear(f, S->n, x, y, z);
}

// intersectBBox and the [min, max] depth clip; false when the reference returns before
// marching (such rays keep the previous map contents unless keep_on_miss is off)
__device__ __forceinline__ bool ray_start(const SessionDev* S, const RayGeo& g, RayState& st) {
    const F3 inv{1.0f / g.dir.x, 1.0f / g.dir.y, 1.0f / g.dir.z};
    const float half = S->vol_w * 0.5f;
    const F3 o = g.o;
    const float t0x = (-half - o.x) * inv.x, t1x = (half - o.x) * inv.x;
    const float t0y = (-half - o.y) * inv.y, t1y = (half - o.y) * inv.y;
    const float t0z = (-half - o.z) * inv.z, t1z = (half - o.z) * inv.z;
    float tmin = fminf(t0x, t1x), tmax = fmaxf(t0x, t1x);
    tmin = fmaxf(tmin, fminf(t0y, t1y));
    tmax = fminf(tmax, fmaxf(t0y, t1y));
    tmin = fmaxf(tmin, fminf(t0z, t1z));
    tmax = fminf(tmax, fmaxf(t0z, t1z));
    if (tmax < tmin) { tmin = -1.0f; tmax = -1.0f; }
    if (tmax < 0.0f) return false;
    const float near_d = fmaxf(S->min_d, tmin), far_d = fminf(S->max_d, tmax);
    if (near_d >= far_d) return false;
    st.t = near_d;
    st.base = near_d;
    st.idx = 0;
    st.near_d = near_d;
    st.far_d = far_d;
    st.prev = 0.f;
    st.prev_t = 0.f;
    st.small = 0;
    st.prev_known = 1;
    st.guard = 0;
    st.sw = 0;
    return true;
}

// t at which the base voxel of the march leaves the voxel box [lo, hi) per axis (0.01 texel
// inside its faces); faces on the volume's edge do not bound (coordinates clamp there).  The
// margin absorbs the rounding of the affine form to + td t: a skip that stops early only
// evaluates samples it could have skipped; it never passes a sample outside the box.
__device__ __forceinline__ float box_exit(const RayGeo& g, int n, int lox, int hix, int loy, int hiy, int loz, int hiz,
                                          float t_far) {
    float t = t_far;
    if (g.tdx > 0.f && hix < n) t = fminf(t, (float(hix) - 0.01f - g.tox) * g.itdx);
    if (g.tdx < 0.f && lox > 0) t = fminf(t, (float(lox) + 0.01f - g.tox) * g.itdx);
    if (g.tdy > 0.f && hiy < n) t = fminf(t, (float(hiy) - 0.01f - g.toy) * g.itdy);
    if (g.tdy < 0.f && loy > 0) t = fminf(t, (float(loy) + 0.01f - g.toy) * g.itdy);
    if (g.tdz > 0.f && hiz < n) t = fminf(t, (float(hiz) - 0.01f - g.toz) * g.itdz);
    if (g.tdz < 0.f && loz > 0) t = fminf(t, (float(loz) + 0.01f - g.toz) * g.itdz);
    return t;
}

// The run of consecutive skippable super-bricks the ray is in, from super-brick s (skippable):
// the t before which every sample's base voxel lies in the run.  Per axis, tc is the t at
// which the ray crosses the cell's face ahead and tm the t at which it comes within 0.01 texel
// of it (faces on the volume's edge do not bound: coordinates clamp there).  The ray leaves a
// cell through the face it crosses first; the run continues into the neighbour across that
// face when the neighbour is skippable and the crossing is clean -- every other coordinate
// still 0.01 texel inside the cell's faces ahead at that t, so a rounded sample near the
// crossing lies in one of the two cells and in no third one.  The run ends at the last cell's
// margined exit, exactly where a skip of that cell alone would end.  At most kRunCells cells.
__device__ __forceinline__ void cell_face(float to, float td, float itd, int s, int n, float t_far, float& tc,
                                          float& tm) {
    // the face of super-brick s ahead along one axis: crossing t and margined t
    tc = tm = t_far;
    if (td > 0.f && 32 * (s + 1) < n) {
        const float face = float(32 * (s + 1));
        tc = (face - to) * itd;
        tm = (face - 0.01f - to) * itd;
    } else if (td < 0.f && s > 0) {
        const float face = float(32 * s);
        tc = (face - to) * itd;
        tm = (face + 0.01f - to) * itd;
    }
}

__device__ __forceinline__ float superbrick_run_exit(const SessionDev* S, const RayGeo& g, int thr, int sx, int sy,
                                                     int sz, float t_far) {
    const int n = S->n, ns = S->ns;
    float tcx, tmx, tcy, tmy, tcz, tmz;
    cell_face(g.tox, g.tdx, g.itdx, sx, n, t_far, tcx, tmx);
    cell_face(g.toy, g.tdy, g.itdy, sy, n, t_far, tcy, tmy);
    cell_face(g.toz, g.tdz, g.itdz, sz, n, t_far, tcz, tmz);
    for (int step = 0; step < kRunCells - 1; ++step) {
        if (tcx <= tcy && tcx <= tcz) {          // leaves through the x face
            if (!(tcx < t_far) || tmy < tcx || tmz < tcx) break;
            const int nx = sx + (g.tdx > 0.f ? 1 : -1);
            if (__ldg(S->sdil + (sz * ns + sy) * ns + nx) < thr) break;
            sx = nx;
            cell_face(g.tox, g.tdx, g.itdx, sx, n, t_far, tcx, tmx);
        } else if (tcy <= tcz) {                 // the y face
            if (!(tcy < t_far) || tmx < tcy || tmz < tcy) break;
            const int ny = sy + (g.tdy > 0.f ? 1 : -1);
            if (__ldg(S->sdil + (sz * ns + ny) * ns + sx) < thr) break;
            sy = ny;
            cell_face(g.toy, g.tdy, g.itdy, sy, n, t_far, tcy, tmy);
        } else {                                 // the z face
            if (!(tcz < t_far) || tmx < tcz || tmy < tcz) break;
            const int nz = sz + (g.tdz > 0.f ? 1 : -1);
            if (__ldg(S->sdil + (nz * ns + sy) * ns + sx) < thr) break;
            sz = nz;
            cell_face(g.toz, g.tdz, g.itdz, sz, n, t_far, tcz, tmz);
        }
    }
    return fminf(fminf(tmx, tmy), tmz);
}

// a read-only load the compiler keeps where it is written (not sunk into a branch)
__device__ __forceinline__ int ld_keep(const int* p) {
    int v;
    asm volatile("ld.global.nc.s32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

// Samples whose base voxel lies in a cell whose distance lower bound is at or above the
// current threshold (0.991 during large steps, 0.001 during small steps) cannot change the
// march.  If the sample at st.t, with base voxel (vx, vy, vz), is such a sample, advance st past
// every following sample in the same cell -- the run of skippable 32^3 super-bricks along the
// ray when its super-brick qualifies, else its 8^3 brick -- to the first sample index whose
// position is at or past the cell's (run's) exit, and return true.  kEager issues the brick
// bound's load beside the super-brick bound's (an evaluated sample needs both): one L1/L2 round
// trip instead of two where latency bounds the march (a single session's raycast, the long
// rays: +0.9 % for one session); where instruction issue bounds it (the 64-register form for
// many ray tiles) the load after a failed super-brick test only is cheaper (0.8 %).
template <bool kEager>
__device__ __forceinline__ bool skip_cell(const SessionDev* S, const RayGeo& g, RayState& st, int vx, int vy, int vz,
                                          float inc) {
    const int n = S->n;
    // order-preserving int keys of the two thresholds
    const int thr = st.small ? __float_as_int(0.001f) : __float_as_int(0.991f);
    const int sx = vx >> 5, sy = vy >> 5, sz = vz >> 5;
    const int ns = S->ns, nb = S->nb;   // (n / 8)^3 bricks: 32-bit indices
    float exit_t;
    if constexpr (kEager) {
        const int bx = vx >> 3, by = vy >> 3, bz = vz >> 3;
        const int skey = ld_keep(S->sdil + (sz * ns + sy) * ns + sx);
        const int bkey = ld_keep(S->bdil + (bz * nb + by) * nb + bx);
        if (skey >= thr) {
            exit_t = superbrick_run_exit(S, g, thr, sx, sy, sz, st.far_d);
        } else {
            if (bkey < thr) return false;
            exit_t = box_exit(g, n, bx * 8, bx * 8 + 8, by * 8, by * 8 + 8, bz * 8, bz * 8 + 8, st.far_d);
        }
    } else {
        if (__ldg(S->sdil + (sz * ns + sy) * ns + sx) >= thr) {
            exit_t = superbrick_run_exit(S, g, thr, sx, sy, sz, st.far_d);
        } else {
            const int bx = vx >> 3, by = vy >> 3, bz = vz >> 3;
            if (__ldg(S->bdil + (bz * nb + by) * nb + bx) < thr) return false;
            exit_t = box_exit(g, n, bx * 8, bx * 8 + 8, by * 8, by * 8 + 8, bz * 8, bz * 8 + 8, st.far_d);
        }
    }
    // skip this sample and every later one whose base voxel stays in the box: the next sample
    // is the first index k > idx with base + k inc >= lim (positions increase with k), or the
    // last index the sample bound allows
    const float lim = fminf(exit_t, st.far_d);
    const int k_lo = st.idx + 1, k_hi = st.idx + (kMaxMarchSamples - st.guard);
    int k = k_lo;
    const float est = __fdividef(lim - st.base, inc);   // within an index or two of the answer
    if (est > float(k_lo)) k = int(fminf(est, float(k_hi)));
    while (k > k_lo && !(march_pos(st.base, k - 1, inc) < lim)) --k;
    while (k < k_hi && march_pos(st.base, k, inc) < lim) ++k;
    st.guard += k - st.idx;
    st.idx = k;
    st.prev_t = march_pos(st.base, k - 1, inc);
    st.t = march_pos(st.base, k, inc);
    st.prev_known = 0;
    return true;
}

// The reference's march loop for one lane (project/src/raycast.cu:75-117).  Returns 1 when
// the ray is finished (precise = refined hit distance, 0 for none) and 0 when `budget`
// iterations ran out with the ray still marching (state kept in st).
template <class TF, class Cnt, bool kEager>
__device__ int march_serial(const SessionDev* S, const RayGeo& g, const TF* f, RayState& st, int budget,
                            float& precise, Cnt& cnt) {
    const int n = S->n;
    const float mu = S->mu, large = mu * S->step_l, small = mu * S->step_s;
    const int* __restrict__ bdil = S->bdil;
    int iters = 0;
    while (st.t < st.far_d && st.guard < kMaxMarchSamples) {
        if (iters++ >= budget) return 0;
        const float inc = st.small ? small : large;
        float x, y, z;
        texel(g, st.t, x, y, z);
        const TexelBase tb = texel_base(n, x, y, z);
        const int g0 = st.guard;
        if (bdil && skip_cell<kEager>(S, g, st, tb.x0, tb.y0, tb.z0, inc)) {
            cnt.add(kCntSkips, 1u);
            cnt.add(kCntSkipped, unsigned(st.guard - g0));
            continue;
        }
        const float tsdf = trilinear_at(f, n, tb);
        cnt.add(st.small ? kCntEvalSmall : kCntEvalLarge, 1u);
        ++st.guard;
        if (tsdf < 0.0f) {
            if (st.t != st.near_d) {
                if (!st.small) {   // went through the surface with a large step: back off by mu
                    st.sw = (st.guard << 2) | 2;
                    begin_small(st, __fsub_rn(st.t, mu), small);
                    continue;
                }
                if (!st.prev_known) {
                    float px, py, pz;
                    texel(g, st.prev_t, px, py, pz);
                    st.prev = trilinear(f, n, px, py, pz);
                }
                precise = st.t - small * st.prev / (tsdf - st.prev);   // the reference's formula
            }
            return 1;
        }
        st.prev = tsdf;
        st.prev_known = 1;
        st.prev_t = st.t;
        if (!st.small && tsdf < 0.99f) {   // the region of uncertainty: small steps from here
            st.sw = (st.guard << 2) | 1;
            begin_small(st, st.t, small);
        } else {
            ++st.idx;
            st.t = march_pos(st.base, st.idx, inc);
        }
    }
    return 1;
}

// The same loop for one ray, carried by all 32 lanes of a warp (every lane holds the same
// g and st): each round lane k evaluates the sample k indices ahead, and the first sample
// that changes the state -- a negative value, or below 0.99 during large steps -- is applied.
// A round that follows a round without any such sample takes two sets, samples k and 32 + k
// (such rays are in a long run of samples that change nothing, a grazing ray in small steps
// for instance); the first event in sample order is applied all the same.
template <class TF, class Cnt>
__device__ void march_coop(const SessionDev* S, const RayGeo& g, const TF* f, RayState& st, int lane,
                           float& precise, Cnt& cnt) {
    const float mu = S->mu, large = mu * S->step_l, small = mu * S->step_s;
    const unsigned int full = 0xffffffffu;
    bool wide = false;   // the last round changed nothing
    while (st.t < st.far_d && st.guard < kMaxMarchSamples) {
        const float inc = st.small ? small : large;
        if (S->bdil) {
            float x, y, z;
            texel(g, st.t, x, y, z);
            const TexelBase tb = texel_base(S->n, x, y, z);
            const int g0 = st.guard;
            if (skip_cell<true>(S, g, st, tb.x0, tb.y0, tb.z0, inc)) {   // every lane takes the same steps
                if (lane == 0) {
                    cnt.add(kCntSkips, 1u);
                    cnt.add(kCntSkipped, unsigned(st.guard - g0));
                }
                wide = false;
                continue;
            }
        }
        float tk[2], fk[2];
        bool valid[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int n = 32 * j + lane;   // sample n of the round
            tk[j] = march_pos(st.base, st.idx + n, inc);
            valid[j] = (j == 0 || wide) && tk[j] < st.far_d && st.guard + n < kMaxMarchSamples;
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            fk[j] = valid[j] ? sample_at(S, g, f, tk[j]) : 0.0f;
            if (valid[j]) cnt.add(st.small ? kCntEvalSmall : kCntEvalLarge, 1u);
        }
        if (lane == 0) cnt.add(kCntRounds, 1u);
        unsigned int evm[2], valm[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            evm[j] = __ballot_sync(full, valid[j] && (fk[j] < 0.0f || (!st.small && fk[j] < 0.99f)));
            valm[j] = __ballot_sync(full, valid[j]);   // valid samples form a prefix in n
        }
        if (!evm[0] && !evm[1]) {
            if (!valm[0]) break;
            const int js = valm[1] ? 1 : 0;
            const int last = 31 - __clz(js ? valm[1] : valm[0]);
            st.prev = __shfl_sync(full, js ? fk[1] : fk[0], last);
            st.prev_t = __shfl_sync(full, js ? tk[1] : tk[0], last);
            st.prev_known = 1;
            st.guard += 32 * js + last + 1;
            st.idx += 32 * js + last + 1;
            st.t = march_pos(st.base, st.idx, inc);
            wide = true;
            continue;
        }
        wide = false;
        const int js = evm[0] ? 0 : 1;
        const float tj = js ? tk[1] : tk[0], fj = js ? fk[1] : fk[0];
        const int e = __ffs(js ? evm[1] : evm[0]) - 1;
        const float te = __shfl_sync(full, tj, e), fe = __shfl_sync(full, fj, e);
        // the sample before the event: lane e - 1 of the same set, or the first set's last lane
        const float tb = __shfl_sync(full, tj, max(e - 1, 0)), fb = __shfl_sync(full, fj, max(e - 1, 0));
        const float tb0 = __shfl_sync(full, tk[0], 31), fb0 = __shfl_sync(full, fk[0], 31);
        const int ne = 32 * js + e;
        if (ne > 0) {
            st.prev = e > 0 ? fb : fb0;
            st.prev_t = e > 0 ? tb : tb0;
            st.prev_known = 1;
        }
        st.guard += ne + 1;
        if (fe < 0.0f) {
            if (te != st.near_d) {
                if (!st.small) {
                    st.sw = (st.guard << 2) | 2;
                    begin_small(st, __fsub_rn(te, mu), small);
                    continue;
                }
                if (!st.prev_known) st.prev = sample_at(S, g, f, st.prev_t);
                precise = te - small * st.prev / (fe - st.prev);
            }
            return;
        }
        st.sw = (st.guard << 2) | 1;   // 0 <= fe < 0.99 during large steps (only they are events)
        st.prev = fe;
        st.prev_t = te;
        st.prev_known = 1;
        begin_small(st, te, small);
    }
}

// computeGradient (project/src/raycast.cu:29-42) at the hit: texel coordinates of the hit
// and the offset of the six central-difference samples (mu / 2 apart, in uvw units)
struct HitGeo {
    F3 vtx;
    float x, y, z, rt, r;
};

__device__ __forceinline__ HitGeo hit_geo(const SessionDev* S, const RayGeo& g, float precise) {
    HitGeo h;
    h.vtx = F3{__fmaf_rn(g.dir.x, precise, g.o.x), __fmaf_rn(g.dir.y, precise, g.o.y),
               __fmaf_rn(g.dir.z, precise, g.o.z)};
    h.r = S->mu * 0.5f / S->vol_w;
    h.rt = h.r * float(S->n);
    h.x = __fmaf_rn(h.vtx.x, g.sc, g.off);
    h.y = __fmaf_rn(h.vtx.y, g.sc, g.off);
    h.z = __fmaf_rn(h.vtx.z, g.sc, g.off);
    return h;
}

// gradient sample q of computeGradient: q = 0, 1, 2 at +rt along x, y, z; 3, 4, 5 at -rt
template <class TF>
__device__ __forceinline__ float grad_sample(const TF* f, int n, const HitGeo& h, int q) {
    const float d = q < 3 ? h.rt : -h.rt;
    const int a = q < 3 ? q : q - 3;
    return trilinear(f, n, a == 0 ? __fadd_rn(h.x, d) : h.x, a == 1 ? __fadd_rn(h.y, d) : h.y,
                     a == 2 ? __fadd_rn(h.z, d) : h.z);
}

// the normal from the six samples and the map writes (project/src/raycast.cu:120-144)
__device__ __forceinline__ void write_hit(const SessionDev* S, int level, int i, int j, bool hit, const HitGeo& h,
                                          const float (&v)[6]) {
    const int w = S->lv[level].w;
    float4* ov = S->pv[level] + size_t(j) * w + i;
    float4* on = S->pn[level] + size_t(j) * w + i;
    if (hit) {
        F3 gr{(v[3] - v[0]) / h.r, (v[4] - v[1]) / h.r, (v[5] - v[2]) / h.r};
        const float gn = sqrtf(dot3(gr, gr));
        if (depth_valid(gn)) {
            gr = F3{gr.x / gn, gr.y / gn, gr.z / gn};
            *ov = make_float4(h.vtx.x, h.vtx.y, h.vtx.z, kValid);
            *on = make_float4(gr.x, gr.y, gr.z, kValid);
            return;
        }
    }
    *ov = make_float4(0.f, 0.f, 0.f, kInvalid);
    *on = make_float4(0.f, 0.f, 0.f, kInvalid);
}

__device__ __forceinline__ void write_trace(const SessionDev* S, int level, int i, int j, unsigned long long code) {
    unsigned long long* tr = S->trace[level];
    if (tr) tr[size_t(j) * S->lv[level].w + i] = code;
}

template <class TF, class Cnt>
__device__ void finish_ray(const SessionDev* S, const RayGeo& g, const TF* f, int level, int i, int j, float precise,
                           const RayState& st, Cnt& cnt) {
    write_trace(S, level, i, j, ray_trace_code(st, precise));
    const HitGeo h = hit_geo(S, g, precise);
    float v[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (precise != 0.0f) {
        cnt.add(kCntGrad, 6u);
#pragma unroll
        for (int q = 0; q < 6; ++q) v[q] = grad_sample(f, S->n, h, q);
    }
    write_hit(S, level, i, j, precise != 0.0f, h, v);
}

// the same for a ray carried by a whole warp: lanes 0-5 take one gradient sample each, lane 0
// writes
template <class TF, class Cnt>
__device__ void finish_ray_warp(const SessionDev* S, const RayGeo& g, const TF* f, int level, int i, int j,
                                float precise, int lane, const RayState& st, Cnt& cnt) {
    if (lane == 0) write_trace(S, level, i, j, ray_trace_code(st, precise));
    const HitGeo h = hit_geo(S, g, precise);
    float mine = 0.f;
    if (precise != 0.0f && lane < 6) {
        mine = grad_sample(f, S->n, h, lane);
        cnt.add(kCntGrad, 1u);
    }
    float v[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) v[q] = __shfl_sync(0xffffffffu, mine, q);
    if (lane == 0) write_hit(S, level, i, j, precise != 0.0f, h, v);
}

__device__ __forceinline__ void write_miss(const SessionDev* S, int level, int i, int j) {
    write_trace(S, level, i, j, 0ull);
    if (S->keep_on_miss) return;
    const int w = S->lv[level].w;
    S->pv[level][size_t(j) * w + i] = make_float4(0.f, 0.f, 0.f, kInvalid);
    S->pn[level][size_t(j) * w + i] = make_float4(0.f, 0.f, 0.f, kInvalid);
}

template <class TF, class Cnt, bool kEager>
__device__ void serial_ray(const EngineView& v, const SessionDev* S, int s, const float* m, F3 o, int level, int i,
                           int j, int budget, Cnt& cnt) {
    const TF* f = static_cast<const TF*>(S->tf);
    RayGeo g;
    make_geo(S, m, o, i, j, g);
    RayState st;
    if (!ray_start(S, g, st)) {
        write_miss(S, level, i, j);
        return;
    }
    cnt.add(kCntRays, 1u);
    float precise = 0.0f;
    if (!march_serial<TF, Cnt, kEager>(S, g, f, st, budget, precise, cnt)) {
        const unsigned int slot = atomicAdd(&v.counters[6], 1u);
        if (slot < unsigned(v.longq_cap)) {
            v.longq[slot] = LongRay{s, level, i, j, st, g};
            cnt.add(kCntQueued, 1u);
            return;
        }
        march_serial<TF, Cnt, kEager>(S, g, f, st, 0x7fffffff, precise, cnt);   // queue full: finish here
    }
    finish_ray(S, g, f, level, i, j, precise, st, cnt);
}

// Each warp pulls 8 x 4-ray tiles on its own (no block-wide barrier).  Steps of many ray tiles
// run four blocks per SM (64 registers: more warps to hide the gathers behind); a single
// session's step runs three (80 registers: fewer instructions per sample, a shorter tail).
template <int kBlocksPerSm, bool kCount>
__global__ void __launch_bounds__(256, kBlocksPerSm) raycast_kernel(EngineView v) {
    MarchCount<kCount> cnt;
    const int lane = threadIdx.x & 31;
    const int ntiles = v.tb->n_ray;
    const int budget = v.tb->ray_budget;
    const int tw = v.tb->ray_tw;
    const int lx = lane % tw, ly = lane / tw;
    while (true) {
        int t = 0;
        if (lane == 0) t = int(atomicAdd(&v.counters[0], 1u));
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= ntiles) break;
        const RayTile T = v.ray[t];
        const StepDev st = v.step[T.s];
        if (!st.active || st.first) continue;
        const SessionDev* S = &v.sess[T.s];
        const LevelDev& Lv = S->lv[T.level];
        const int i = T.x0 + lx, j = T.y0 + ly;
        if (i >= Lv.cw || j >= Lv.ch) continue;
        float m[9];
        F3 o;
        ray_matrix(S, Lv, m, o);
        if (S->fmt == KF_TSDF_F16U16)
            serial_ray<__half, MarchCount<kCount>, kBlocksPerSm == 3>(v, S, T.s, m, o, T.level, i, j, budget, cnt);
        else
            serial_ray<float, MarchCount<kCount>, kBlocksPerSm == 3>(v, S, T.s, m, o, T.level, i, j, budget, cnt);
    }
    cnt.flush(v.ray_counts);
}

template <class TF, class Cnt>
__device__ void coop_ray(const SessionDev* S, const LongRay& L, int lane, Cnt& cnt) {
    const TF* f = static_cast<const TF*>(S->tf);
    const RayGeo g = L.g;
    RayState st = L.st;
    float precise = 0.0f;
    march_coop(S, g, f, st, lane, precise, cnt);
    finish_ray_warp(S, g, f, L.level, L.i, L.j, precise, lane, st, cnt);
}

// the queued long rays, one warp each
template <bool kCount>
__global__ void __launch_bounds__(256) raycast_long_kernel(EngineView v) {
    MarchCount<kCount> cnt;
    const int lane = threadIdx.x & 31;
    const int count = min(int(v.counters[6]), v.longq_cap);
    while (true) {
        int idx = 0;
        if (lane == 0) idx = int(atomicAdd(&v.counters[7], 1u));
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (idx >= count) break;
        const LongRay L = v.longq[idx];
        const SessionDev* S = &v.sess[L.s];
        if (S->fmt == KF_TSDF_F16U16)
            coop_ray<__half>(S, L, lane, cnt);
        else
            coop_ray<float>(S, L, lane, cnt);
    }
    cnt.flush(v.ray_counts);
}

int long_ray_bytes() { return int(sizeof(LongRay)); }

cudaError_t launch_raycast(const EngineView& v, int grid, cudaStream_t st, bool many) {
    const bool count = v.ray_counts != nullptr;
    if (count) {
        if (many) raycast_kernel<4, true><<<grid, 256, 0, st>>>(v);
        else raycast_kernel<3, true><<<grid, 256, 0, st>>>(v);
    } else {
        if (many) raycast_kernel<4, false><<<grid, 256, 0, st>>>(v);
        else raycast_kernel<3, false><<<grid, 256, 0, st>>>(v);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (count) raycast_long_kernel<true><<<grid, 256, 0, st>>>(v);
    else raycast_long_kernel<false><<<grid, 256, 0, st>>>(v);
    return cudaGetLastError();
}

int ray_count_slots() { return kRayCounts; }

// ---- stage kernel: kernel::raycast on a caller volume ----

struct RayStage {
    float m[9];
    float o[3];
};

template <class TF>
__global__ void raycast_stage_kernel(SessionDev S, RayStage rs, int w, int h) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= w || j >= h) return;
    const TF* f = static_cast<const TF*>(S.tf);
    RayGeo g;
    make_geo(&S, rs.m, F3{rs.o[0], rs.o[1], rs.o[2]}, i, j, g);
    RayState st;
    if (!ray_start(&S, g, st)) {
        write_miss(&S, 0, i, j);
        return;
    }
    float precise = 0.0f;
    MarchCount<false> cnt;
    march_serial<TF, MarchCount<false>, false>(&S, g, f, st, 0x7fffffff, precise, cnt);
    finish_ray(&S, g, f, 0, i, j, precise, st, cnt);
}

cudaError_t stage_raycast(const kf_volume* vol, const float* pose, const float* ik, float4* vtx, float4* nrm, int w,
                          int h, float min_d, float max_d, float step_l, float step_s, cudaStream_t st,
                          const SessionDev* bounds) {
    SessionDev S{};
    if (bounds) {   // a session's brick bounds: the same samples, skipping exactly as the pipeline
        S.bdil = bounds->bdil;
        S.sdil = bounds->sdil;
        S.nb = bounds->nb;
        S.ns = bounds->ns;
    }
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
    // R * K^-1 with every product and sum rounded on its own (ray_matrix's arithmetic)
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 3; ++row) {
            const volatile float a = pose[row] * ik[col * 3 + 0], b = pose[4 + row] * ik[col * 3 + 1],
                                 c = pose[8 + row] * ik[col * 3 + 2];
            const volatile float ab = a + b;
            rs.m[col * 3 + row] = ab + c;
        }
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
