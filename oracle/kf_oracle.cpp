// kf_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the per-frame KinectFusion path of isikmustafa/kinectfusion-cuda
// (project/src).  It is the reference the tests compare the CUDA library in kinectfusion-cuda_b200/ with, and the
// timed CPU baseline of bench.py; the product never links, loads or calls it.  Only tests/,
// __graft_entry__.smoke() and bench.py's CPU legs load it.
//
// Every function names the reference file:line it restates.  The code is templated on the
// scalar type: the float instantiation follows the reference's float arithmetic (without
// the fast-math approximations, which have no CPU counterpart); the double instantiation is
// the FP64 accuracy oracle.  Two parts of the algorithm are defined in float for both
// instantiations because the reference defines them that way: the uint16 -> fp16 depth
// rounding (project/src/measurement.cu:19-21) and the voxel-centre coordinates, which the
// reference accumulates in float along z (project/src/tsdf.cu:27-31).
//
// Pinned against the reference's own known-answer tests (test/icp_tests.cpp,
// test/transformation_tests.cpp, test/cuda_grid_map_tests.cpp): see
// tests/test_oracle_golden.py.  Stages no reference test covers (bilateral filter,
// downsample, vertex map, fusion, raycast) are pinned by hand-derived known answers there.
// The one third-party semantic on the path, glm::orientate3 (project/src/icp.cpp:82), is
// restated from its documented convention (rotation Y * X * Z) and is not pinned by any
// reference test.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "../include/kf_api.h"

namespace {

// ------------------------------------------------------------------------------------------
// small linear algebra in the memory order of glm (column-major)
// ------------------------------------------------------------------------------------------
template <class T> struct V3 { T x, y, z; };
template <class T> struct V4 { T x, y, z, w; };

template <class T> inline V3<T> add(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> sub(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> scale(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
template <class T> inline T length(V3<T> a) { return std::sqrt(dot(a, a)); }
// v * (1 / sqrt(dot(v, v))): a zero vector becomes NaN, as in the reference.
template <class T> inline V3<T> normalize(V3<T> a) { return scale(a, T(1) / std::sqrt(dot(a, a))); }

// 3x3, c[col][row]
template <class T> struct M3 { T c[3][3]; };

template <class T> inline V3<T> mul(const M3<T>& m, V3<T> v) {
    return {m.c[0][0] * v.x + m.c[1][0] * v.y + m.c[2][0] * v.z,
            m.c[0][1] * v.x + m.c[1][1] * v.y + m.c[2][1] * v.z,
            m.c[0][2] * v.x + m.c[1][2] * v.y + m.c[2][2] * v.z};
}
template <class T> inline M3<T> mul(const M3<T>& a, const M3<T>& b) {
    M3<T> r;
    for (int col = 0; col < 3; ++col) {
        V3<T> bc{b.c[col][0], b.c[col][1], b.c[col][2]};
        V3<T> v = mul(a, bc);
        r.c[col][0] = v.x; r.c[col][1] = v.y; r.c[col][2] = v.z;
    }
    return r;
}
template <class T> inline M3<T> transpose(const M3<T>& m) {
    M3<T> r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.c[i][j] = m.c[j][i];
    return r;
}
// Adjugate / determinant inverse (the generic 3x3 inverse glm::inverse computes,
// used for the inverse intrinsics, project/src/sensor.h:17-19).
template <class T> inline M3<T> inverse(const M3<T>& m) {
    const T a = m.c[0][0], b = m.c[1][0], c = m.c[2][0];
    const T d = m.c[0][1], e = m.c[1][1], f = m.c[2][1];
    const T g = m.c[0][2], h = m.c[1][2], i = m.c[2][2];
    const T det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
    const T od = T(1) / det;
    M3<T> r;  // r(row, col) = cof(col, row) / det
    r.c[0][0] = (e * i - f * h) * od;  r.c[1][0] = -(b * i - c * h) * od; r.c[2][0] = (b * f - c * e) * od;
    r.c[0][1] = -(d * i - f * g) * od; r.c[1][1] = (a * i - c * g) * od;  r.c[2][1] = -(a * f - c * d) * od;
    r.c[0][2] = (d * h - e * g) * od;  r.c[1][2] = -(a * h - b * g) * od; r.c[2][2] = (a * e - b * d) * od;
    return r;
}
template <class T> inline M3<T> from_flat9(const float* f) {
    M3<T> m;
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 3; ++row) m.c[col][row] = T(f[col * 3 + row]);
    return m;
}

// rigid pose camera->world: x_world = R x_cam + t (project/src/rigid_transform_3d.h:5-23)
template <class T> struct Pose { M3<T> R; V3<T> t; };

template <class T> inline Pose<T> pose_from16(const float* p) {
    Pose<T> r;
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 3; ++row) r.R.c[col][row] = T(p[col * 4 + row]);
    r.t = {T(p[12]), T(p[13]), T(p[14])};
    return r;
}
template <class T> inline void pose_to16(const Pose<T>& P, float* p) {
    for (int i = 0; i < 16; ++i) p[i] = 0.0f;
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 3; ++row) p[col * 4 + row] = float(P.R.c[col][row]);
    p[12] = float(P.t.x); p[13] = float(P.t.y); p[14] = float(P.t.z); p[15] = 1.0f;
}
template <class T> inline Pose<T> pose_inverse(const Pose<T>& P) {
    Pose<T> r;
    r.R = transpose(P.R);
    V3<T> mt = mul(r.R, P.t);
    r.t = {-mt.x, -mt.y, -mt.z};
    return r;
}
template <class T> inline V3<T> pose_apply(const Pose<T>& P, V3<T> p) { return add(mul(P.R, p), P.t); }

// intrinsics of level l: f / 2^l and (c + 0.5) / 2^l - 0.5 (project/src/sensor.h:14-16
// writes these for 640 x 480 as literals)
template <class T> inline M3<T> intrinsics(const kf_config& c, int level) {
    const float s = 1.0f / float(1 << level);
    M3<T> k{};
    k.c[0][0] = T(c.fx * s);
    k.c[1][1] = T(c.fy * s);
    k.c[2][0] = T((c.cx + 0.5f) * s - 0.5f);
    k.c[2][1] = T((c.cy + 0.5f) * s - 0.5f);
    k.c[2][2] = T(1);
    return k;
}

constexpr float kValid = -1.0f;     // project/src/device_helper.cuh:9
constexpr float kInvalid = -2.0f;   // project/src/device_helper.cuh:10
constexpr float kMinDepth = 0.01f;  // project/src/device_helper.cuh:11

// project/src/device_helper.cuh:14-17
template <class T> inline bool depth_valid(T d) { return d > T(kMinDepth) && std::isfinite(d); }

// The float -> int conversion the GPU performs (cvt.rzi.s32.f32): NaN -> 0, saturating.
template <class T> inline int to_int_device(T x) {
    if (std::isnan(x)) return 0;
    if (x >= T(2147483647.0)) return 2147483647;
    if (x <= T(-2147483648.0)) return (-2147483647 - 1);
    return int(x);
}

// Value conversion uint16 -> fp16 (round to nearest even, 11 significant bits, inf above
// 65504): what __half2float(unsigned short) does through __half's integral constructor
// (project/src/measurement.cu:19-21).
inline float u16_to_half_value(uint16_t u) {
    if (u < 2048) return float(u);
    const int e = 31 - __builtin_clz(uint32_t(u));  // 11..15
    const int shift = e - 10;
    uint32_t q = uint32_t(u) >> shift;
    const uint32_t rem = uint32_t(u) & ((1u << shift) - 1u);
    const uint32_t half = 1u << (shift - 1);
    if (rem > half || (rem == half && (q & 1u))) ++q;
    const uint32_t v = q << shift;
    if (v > 65504u) return std::numeric_limits<float>::infinity();
    return float(v);
}

// the reference's launch grids cover (dim / 8) * 8 elements (project/src/measurement.cu:151)
inline int cover8(int dim, int trunc) { return trunc ? (dim / 8) * 8 : dim; }
// the ICP grid: threads = min(dim - 1, 8), blocks = dim / threads (project/src/icp.cu:94-95)
inline int cover_icp(int dim, int trunc) {
    if (!trunc) return dim;
    int t = std::min(dim - 1, 8);
    if (t <= 0) return dim;
    return (dim / t) * t;
}

// ------------------------------------------------------------------------------------------
// stages
// ------------------------------------------------------------------------------------------

// kernel::convertToDepthMeters, project/src/measurement.cu:14-31
template <class T>
void convert(const uint16_t* raw, T* out, int w, int h, int cw, int ch, float scale, int unmirror) {
    for (int j = 0; j < ch; ++j)
        for (int i = 0; i < cw; ++i) {
            const float hv = u16_to_half_value(raw[size_t(j) * w + i]);
            const T d = T(hv) * T(scale);
            const int io = unmirror ? (w - 1 - i) : i;
            out[size_t(j) * w + io] = d;
        }
}

// kernel::applyBilateralFilter, project/src/measurement.cu:33-66 (exp(-dx2/ss^2 - dr2/sr^2),
// clamp-to-edge reads, x-outer / y-inner accumulation, acc / norm)
template <class T>
void bilateral(const T* in, T* out, int w, int h, int cw, int ch, float sigma_s, float sigma_r,
               int radius) {
    const T inv_ss = T(1) / (T(sigma_s) * T(sigma_s));
    const T inv_sr = T(1) / (T(sigma_r) * T(sigma_r));
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ch; ++j)
        for (int i = 0; i < cw; ++i) {
            const T center = in[size_t(j) * w + i];
            T norm = 0, acc = 0;
            for (int x = -radius; x <= radius; ++x) {
                const int ii = std::min(std::max(i + x, 0), w - 1);
                for (int y = -radius; y <= radius; ++y) {
                    const int jj = std::min(std::max(j + y, 0), h - 1);
                    const T cur = in[size_t(jj) * w + ii];
                    const T s = T(x * x + y * y);
                    T r = center - cur;
                    r *= r;
                    const T f = std::exp(-s * inv_ss - r * inv_sr);
                    norm += f;
                    acc += f * cur;
                }
            }
            out[size_t(j) * w + i] = acc / norm;
        }
}

// kernel::downSample, project/src/measurement.cu:68-102 (top-left pixel plus the 2x2
// neighbours within 3 sigma_r of it; no validity test)
template <class T>
void down_sample(const T* in, T* out, int w_out, int h_out, int cw, int ch, float sigma_r) {
    const int w_in = 2 * w_out;
    const T thr = T(3.0f * sigma_r);
    for (int j = 0; j < ch; ++j)
        for (int i = 0; i < cw; ++i) {
            const T f1 = in[size_t(2 * j) * w_in + 2 * i];
            const T f2 = in[size_t(2 * j) * w_in + 2 * i + 1];
            const T f3 = in[size_t(2 * j + 1) * w_in + 2 * i];
            const T f4 = in[size_t(2 * j + 1) * w_in + 2 * i + 1];
            T acc = f1;
            int count = 1;
            if (std::fabs(f1 - f2) <= thr) { acc += f2; ++count; }
            if (std::fabs(f1 - f3) <= thr) { acc += f3; ++count; }
            if (std::fabs(f1 - f4) <= thr) { acc += f4; ++count; }
            out[size_t(j) * w_out + i] = acc / T(count);
        }
}

// kernel::createVertexMap, project/src/measurement.cu:104-126
template <class T>
void vertex_map(const T* depth, V4<T>* vmap, int w, int cw, int ch, const M3<T>& inv_k) {
    for (int j = 0; j < ch; ++j)
        for (int i = 0; i < cw; ++i) {
            const T d = depth[size_t(j) * w + i];
            V4<T>& o = vmap[size_t(j) * w + i];
            if (depth_valid(d)) {
                V3<T> p{T(float(i) + 0.5f), T(float(j) + 0.5f), T(1)};
                p = mul(inv_k, p);
                p = scale(p, d);
                o = {p.x, p.y, p.z, T(kValid)};
            } else {
                o = {T(0), T(0), T(0), T(kInvalid)};
            }
        }
}

// device_helper::isValid with cudaBoundaryModeZero, project/src/device_helper.cuh:37-44
template <class T> inline bool map_valid(const V4<T>* m, int w, int h, int i, int j) {
    if (i < 0 || j < 0 || i >= w || j >= h) return false;
    return m[size_t(j) * w + i].w == T(kValid);
}

// device_helper::computeNormal, project/src/device_helper.cuh:81-110
template <class T> inline V4<T> compute_normal(const V4<T>* m, int w, int h, int i, int j) {
    if (map_valid(m, w, h, i, j) && map_valid(m, w, h, i + 1, j) && map_valid(m, w, h, i, j + 1)) {
        const V4<T>& c = m[size_t(j) * w + i];
        const V4<T>& r = m[size_t(j) * w + i + 1];
        const V4<T>& d = m[size_t(j + 1) * w + i];
        V3<T> n = normalize(cross(sub(V3<T>{r.x, r.y, r.z}, V3<T>{c.x, c.y, c.z}),
                                  sub(V3<T>{d.x, d.y, d.z}, V3<T>{c.x, c.y, c.z})));
        return {n.x, n.y, n.z, T(kValid)};
    }
    return {T(0), T(0), T(0), T(kInvalid)};
}

// kernel::createNormalMap, project/src/measurement.cu:128-135
template <class T> void normal_map(const V4<T>* vmap, V4<T>* nmap, int w, int h, int cw, int ch) {
    for (int j = 0; j < ch; ++j)
        for (int i = 0; i < cw; ++i) nmap[size_t(j) * w + i] = compute_normal(vmap, w, h, i, j);
}

// ---- volume ----

template <class T> struct Volume {
    int n = 0;
    float width = 0, res = 0, mu = 0, max_w = 0;
    const T* f = nullptr;   // distance
    T* fw = nullptr;        // writable distance
    T* w = nullptr;         // weight
};

// trilinear tex3D<float2>(...).x with normalized coordinates, linear filtering and clamp
// addressing: texel coordinate uvw * n - 0.5, taps clamped to [0, n-1]
// (project/src/voxel_grid.cpp:24-33, project/src/raycast.cu:86-87).  tex9bit rounds the
// interpolation weights to the 8 fractional bits the texture unit keeps.
template <class T> inline T sample(const T* f, int n, T u, T v, T w, int tex9bit) {
    const T x = u * T(n) - T(0.5), y = v * T(n) - T(0.5), z = w * T(n) - T(0.5);
    const T fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
    T ax = x - fx, ay = y - fy, az = z - fz;
    if (tex9bit) {
        ax = std::nearbyint(ax * T(256)) / T(256);
        ay = std::nearbyint(ay * T(256)) / T(256);
        az = std::nearbyint(az * T(256)) / T(256);
    }
    auto clampi = [n](long long i) { return int(std::min<long long>(std::max<long long>(i, 0), n - 1)); };
    const long long ix = (long long)fx, iy = (long long)fy, iz = (long long)fz;
    const int x0 = clampi(ix), x1 = clampi(ix + 1), y0 = clampi(iy), y1 = clampi(iy + 1);
    const int z0 = clampi(iz), z1 = clampi(iz + 1);
    auto at = [f, n](int a, int b, int c) { return f[(size_t(c) * n + b) * n + a]; };
    const T c00 = at(x0, y0, z0) * (T(1) - ax) + at(x1, y0, z0) * ax;
    const T c10 = at(x0, y1, z0) * (T(1) - ax) + at(x1, y1, z0) * ax;
    const T c01 = at(x0, y0, z1) * (T(1) - ax) + at(x1, y0, z1) * ax;
    const T c11 = at(x0, y1, z1) * (T(1) - ax) + at(x1, y1, z1) * ax;
    const T c0 = c00 * (T(1) - ay) + c10 * ay;
    const T c1 = c01 * (T(1) - ay) + c11 * ay;
    return c0 * (T(1) - az) + c1 * az;
}

template <class T> inline V3<T> to_uvw(V3<T> p, T width) {
    return {p.x / width + T(0.5), p.y / width + T(0.5), p.z / width + T(0.5)};
}

// intersectBBox, project/src/raycast.cu:7-27
template <class T> inline void intersect_bbox(V3<T> o, V3<T> inv_dir, T lo, T hi, T& tn, T& tf) {
    const T t0x = (lo - o.x) * inv_dir.x, t1x = (hi - o.x) * inv_dir.x;
    const T t0y = (lo - o.y) * inv_dir.y, t1y = (hi - o.y) * inv_dir.y;
    const T t0z = (lo - o.z) * inv_dir.z, t1z = (hi - o.z) * inv_dir.z;
    T tmin = std::fmin(t0x, t1x), tmax = std::fmax(t0x, t1x);
    tmin = std::fmax(tmin, std::fmin(t0y, t1y));
    tmax = std::fmin(tmax, std::fmax(t0y, t1y));
    tmin = std::fmax(tmin, std::fmin(t0z, t1z));
    tmax = std::fmin(tmax, std::fmax(t0z, t1z));
    if (tmax < tmin) { tn = T(-1); tf = T(-1); return; }
    tn = tmin; tf = tmax;
}

// computeGradient, project/src/raycast.cu:29-42
template <class T> inline V3<T> gradient(V3<T> p, const T* f, int n, T width, T mu, int tex9bit) {
    const T r = mu * T(0.5) / width;
    const V3<T> u = to_uvw(p, width);
    const T fx0 = sample(f, n, u.x + r, u.y, u.z, tex9bit);
    const T fy0 = sample(f, n, u.x, u.y + r, u.z, tex9bit);
    const T fz0 = sample(f, n, u.x, u.y, u.z + r, tex9bit);
    const T fx = sample(f, n, u.x - r, u.y, u.z, tex9bit);
    const T fy = sample(f, n, u.x, u.y - r, u.z, tex9bit);
    const T fz = sample(f, n, u.x, u.y, u.z - r, tex9bit);
    return {(fx - fx0) / r, (fy - fy0) / r, (fz - fz0) / r};
}

struct RaycastParams {
    float min_d, max_d, step_l, step_s;
    int keep_on_miss, tex9bit;
    // 0: sample positions by the reference's repeated additions t <- t + inc
    //    (project/src/raycast.cu:78), whose float rounding drifts along a ray;
    // 1: the CUDA library's positions, t_k = base + k * inc with one rounding (base: the near
    //    distance, the sample that left large steps, or t - mu after a back-off), which follow
    //    the FP64 march to within a rounding.  In FP64 both agree to ~1e-16.
    int exact_positions = 0;
};

// raycastKernel, project/src/raycast.cu:44-145.  Returns the number of TSDF samples taken
// (march samples plus six per gradient), the unit of the raycast's algorithmic traffic.
// The march's decision trace of one ray, in the encoding the CUDA library's debug mode writes
// (so a test can tell pixels whose march took the same decisions from pixels where a sample
// near 0.99 or 0 decided differently):
//   bits 40..  samples taken when the march left large steps (0: it never did)
//   bits  8..39 samples taken when the march ended
//   bits  4..5  how it left large steps: 1 a sample in [0, 0.99), 2 a negative one (back-off)
//   bits  0..1  how it ended: 0 past the far plane or the sample bound, 1 negative first
//               sample, 2 refined hit
// A ray that returns before marching (no volume in range) has trace 0.
inline int64_t march_trace(int taken_sw, int mode, int taken_end, int end) {
    return (int64_t(taken_sw) << 40) | (int64_t(taken_end) << 8) | (int64_t(mode) << 4) | int64_t(end);
}

template <class T>
long long raycast(const T* f, int n, float width_f, float mu_f, const Pose<T>& pose, const M3<T>& inv_k,
                  V4<T>* vmap, V4<T>* nmap, int w, int cw, int ch, const RaycastParams& rp,
                  int64_t* trace = nullptr) {
    const T width = T(width_f), mu = T(mu_f);
    const M3<T> ray_m = mul(pose.R, inv_k);
    const V3<T> o = pose.t;
    const T half = width * T(0.5);
    const T large = mu * T(rp.step_l), small = mu * T(rp.step_s);
    long long samples = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : samples)
    for (int j = 0; j < ch; ++j)
        for (int i = 0; i < cw; ++i) {
            V4<T>& ov = vmap[size_t(j) * w + i];
            V4<T>& on = nmap[size_t(j) * w + i];
            const V3<T> dir = mul(ray_m, V3<T>{T(float(i) + 0.5f), T(float(j) + 0.5f), T(1)});
            const V3<T> inv_dir{T(1) / dir.x, T(1) / dir.y, T(1) / dir.z};
            T tn, tf;
            intersect_bbox(o, inv_dir, -half, half, tn, tf);
            bool early = false;
            T near_d = 0, far_d = 0;
            if (tf < T(0)) {
                early = true;
            } else {
                near_d = std::max(T(rp.min_d), tn);
                far_d = std::min(T(rp.max_d), tf);
                if (near_d >= far_d) early = true;
            }
            if (early) {
                if (!rp.keep_on_miss) {
                    ov = {T(0), T(0), T(0), T(kInvalid)};
                    on = {T(0), T(0), T(0), T(kInvalid)};
                }
                if (trace) trace[size_t(j) * w + i] = 0;
                continue;
            }
            T inc = large, prev = 0, precise = 0;
            int guard = 0;   // the CUDA library's bound on samples per ray
            int taken = 0, taken_sw = 0, mode = 0, end = 0;
            T base = near_d;   // exact_positions: t = base + idx * inc
            int idx = 0;
            // the reference's for loop: t = near; while t < far; t += inc (or the exact position)
            T t = near_d;
            while (t < far_d && guard < (1 << 16)) {
                const V3<T> p = add(o, scale(dir, t));
                const V3<T> u = to_uvw(p, width);
                const T tsdf = sample(f, n, u.x, u.y, u.z, rp.tex9bit);
                ++samples;
                ++taken;
                if (tsdf < T(0)) {
                    if (t != near_d) {
                        if (inc == large) {
                            t -= mu;
                            inc = small;
                            taken_sw = taken;
                            mode = 2;
                            base = t;
                            idx = 0;
                            t = rp.exact_positions ? T(std::fma(T(idx + 1), inc, base)) : T(t + inc);
                            ++idx;
                            ++guard;
                            continue;
                        }
                        precise = t - inc * prev / (tsdf - prev);
                        end = 2;
                    } else {
                        end = 1;
                    }
                    break;
                } else if (tsdf < T(0.99f)) {
                    if (inc == large) {
                        taken_sw = taken;
                        mode = 1;
                        base = t;
                        idx = 0;
                    }
                    inc = small;
                }
                prev = tsdf;
                ++guard;
                ++idx;
                t = rp.exact_positions ? T(std::fma(T(idx), inc, base)) : T(t + inc);
            }
            if (trace) trace[size_t(j) * w + i] = march_trace(taken_sw, mode, taken, end);
            if (precise != T(0)) {
                const V3<T> vtx = add(o, scale(dir, precise));
                V3<T> g = gradient(vtx, f, n, width, mu, rp.tex9bit);
                samples += 6;
                const T gn = length(g);
                if (depth_valid(gn)) {
                    g = {g.x / gn, g.y / gn, g.z / gn};
                    ov = {vtx.x, vtx.y, vtx.z, T(kValid)};
                    on = {g.x, g.y, g.z, T(kValid)};
                    continue;
                }
            }
            ov = {T(0), T(0), T(0), T(kInvalid)};
            on = {T(0), T(0), T(0), T(kInvalid)};
        }
    return samples;
}

// voxel-centre coordinates exactly as the reference forms them in float
// (project/src/tsdf.cu:27 and the per-slice "point.z += resolution" at :31)
inline void voxel_axes(int n, float width, std::vector<float>& xs, std::vector<float>& zs) {
    const float res = width / float(n - 1);   // project/src/voxel_grid.h:44
    const float base = -width * 0.5f;
    xs.resize(n);
    zs.resize(n);
    for (int i = 0; i < n; ++i) xs[i] = base + float(i) * res;
    float z = base + (-res);
    for (int k = 0; k < n; ++k) {
        z = z + res;
        zs[k] = z;
    }
}

// kernel::fuse, project/src/tsdf.cu:20-75 (frustum bounds w x h instead of the literal
// 640 x 480).  Returns the number of voxels updated.
template <class T>
long long fuse(const T* depth, int w, int h, const M3<T>& k0, T* F, T* Wt, int n, int cover_n, float width,
               float mu_f, float max_w, const Pose<T>& pose, float min_d, float max_d) {
    std::vector<float> xs, zs;
    voxel_axes(n, width, xs, zs);
    const Pose<T> inv = pose_inverse(pose);
    const T mu = T(mu_f);
    long long updated = 0;
#pragma omp parallel for schedule(static) reduction(+ : updated)
    for (int j = 0; j < cover_n; ++j)
        for (int i = 0; i < cover_n; ++i)
            for (int k = 0; k < n; ++k) {
                const V3<T> p{T(xs[i]), T(xs[j]), T(zs[k])};
                const V3<T> pe = pose_apply(inv, p);
                V3<T> px = mul(k0, pe);
                px = {px.x / px.z, px.y / px.z, px.z / px.z};
                if (!(pe.z >= T(min_d) && pe.z < T(max_d) && px.x >= T(0) && px.x < T(w) && px.y >= T(0) &&
                      px.y < T(h)))
                    continue;
                const T d = depth[size_t(to_int_device(px.y)) * w + to_int_device(px.x)];
                if (!depth_valid(d)) continue;
                const T diff = d - pe.z;
                if (diff >= -mu) {
                    const T fn = std::min(T(1), diff / mu);
                    const T wn = T(1) / d;
                    const size_t idx = (size_t(k) * n + j) * n + i;
                    const T f0 = F[idx], w0 = Wt[idx];
                    F[idx] = (f0 * w0 + fn * wn) / (w0 + wn);
                    T w1 = w0 + wn;
                    if (max_w > 0.0f && w1 > T(max_w)) w1 = T(max_w);
                    Wt[idx] = w1;
                    ++updated;
                }
            }
    return updated;
}

// ---- ICP ----

struct IcpParams { float dist, angle; };

// constructIcpResidualsKernel, project/src/icp.cu:7-82, with computeCorrespondence,
// areVerticesTooFarAway, areNormalsTooDifferent, computeAndFillA/B (project/src/icp.cuh:40-95).
// Returns whether the pixel produced a residual; row a / scalar b are zero otherwise.
template <class T>
bool icp_row(const V4<T>* vmap, const V4<T>* tv, const V4<T>* tn, int w, int h, int u, int v,
             const M3<T>& Rp, V3<T> tp, const M3<T>& Rc, V3<T> tc, const M3<T>& K, const IcpParams& ip,
             T a[6], T& b) {
    for (int q = 0; q < 6; ++q) a[q] = 0;
    b = 0;
    if (!map_valid(vmap, w, h, u, v)) return false;
    const V4<T>& vc4 = vmap[size_t(v) * w + u];
    const V3<T> s = add(mul(Rc, V3<T>{vc4.x, vc4.y, vc4.z}), tc);
    // computeCorrespondence: (K * transpose(R_prev)) * (s - t_prev), floor(x / z)
    const V3<T> pt = mul(mul(K, transpose(Rp)), sub(s, tp));
    const int uc = to_int_device(std::floor(pt.x / pt.z));
    const int vc = to_int_device(std::floor(pt.y / pt.z));
    if (uc < 0 || vc < 0 || uc >= w || vc >= h || !map_valid(tv, w, h, uc, vc) || !map_valid(tn, w, h, uc, vc))
        return false;
    const V4<T>& d4 = tv[size_t(vc) * w + uc];
    const V3<T> d{d4.x, d4.y, d4.z};
    if (length(sub(s, d)) > T(ip.dist)) return false;
    const V4<T>& n4 = tn[size_t(vc) * w + uc];
    const V3<T> n{n4.x, n4.y, n4.z};
    const V4<T> ns = compute_normal(vmap, w, h, u, v);
    if (ns.w == T(kInvalid)) return false;
    const V3<T> nr = normalize(mul(Rc, V3<T>{ns.x, ns.y, ns.z}));
    const T ang = std::acos(dot(nr, n));
    if (ang > T(ip.angle)) return false;
    a[0] = n.y * s.z - n.z * s.y;
    a[1] = n.z * s.x - n.x * s.z;
    a[2] = n.x * s.y - n.y * s.x;
    a[3] = n.x; a[4] = n.y; a[5] = n.z;
    b = n.x * d.x + n.y * d.y + n.z * d.z - n.x * s.x - n.y * s.y - n.z * s.z;
    return true;
}

// Normal equations A^T A and A^T b.  The reference forms them with cublasSgemm/Sgemv
// (project/src/linear_least_squares.cpp:29-34); here rows are summed in double, row by
// row into per-image-row partials that are then added in order (deterministic for any
// thread count).
struct NormalEq { double ata[36]; double atb[6]; };

template <class T>
NormalEq icp_normal_equations(const V4<T>* vmap, const V4<T>* tv, const V4<T>* tn, int w, int h, int cw,
                              int ch, const M3<T>& Rp, V3<T> tp, const M3<T>& Rc, V3<T> tc, const M3<T>& K,
                              const IcpParams& ip, uint8_t* mask) {
    std::vector<double> rows(size_t(ch) * 42, 0.0);
#pragma omp parallel for schedule(static)
    for (int v = 0; v < ch; ++v) {
        double* acc = &rows[size_t(v) * 42];
        for (int u = 0; u < cw; ++u) {
            T a[6], b;
            const bool ok = icp_row(vmap, tv, tn, w, h, u, v, Rp, tp, Rc, tc, K, ip, a, b);
            if (mask) mask[size_t(v) * w + u] = ok ? 1 : 0;
            if (!ok) continue;
            for (int r = 0; r < 6; ++r) {
                for (int c = 0; c < 6; ++c) acc[r * 6 + c] += double(a[r]) * double(a[c]);
                acc[36 + r] += double(a[r]) * double(b);
            }
        }
    }
    NormalEq e{};
    for (int v = 0; v < ch; ++v)
        for (int q = 0; q < 42; ++q) {
            if (q < 36) e.ata[q] += rows[size_t(v) * 42 + q];
            else e.atb[q - 36] += rows[size_t(v) * 42 + q];
        }
    return e;
}

// Cholesky (LLT, lower) solve of the 6x6 normal equations: the reference calls Eigen's
// LLT<Matrix<float,6,6>>::solve (project/src/linear_least_squares.cpp:41).  A pivot that
// is not positive gives a NaN solution (the reference's updatePose then throws).
template <class T> void cholesky_solve(const double ata_d[36], const double atb_d[6], T x[6]) {
    T A[6][6], b[6], L[6][6] = {};
    for (int r = 0; r < 6; ++r) {
        b[r] = T(atb_d[r]);
        for (int c = 0; c < 6; ++c) A[r][c] = T(ata_d[r * 6 + c]);
    }
    for (int j = 0; j < 6; ++j) {
        T d = A[j][j];
        for (int k = 0; k < j; ++k) d -= L[j][k] * L[j][k];
        if (!(d > T(0))) {
            for (int q = 0; q < 6; ++q) x[q] = std::numeric_limits<T>::quiet_NaN();
            return;
        }
        const T ljj = std::sqrt(d);
        L[j][j] = ljj;
        for (int i = j + 1; i < 6; ++i) {
            T s = A[i][j];
            for (int k = 0; k < j; ++k) s -= L[i][k] * L[j][k];
            L[i][j] = s / ljj;
        }
    }
    T y[6];
    for (int i = 0; i < 6; ++i) {
        T s = b[i];
        for (int k = 0; k < i; ++k) s -= L[i][k] * y[k];
        y[i] = s / L[i][i];
    }
    for (int i = 5; i >= 0; --i) {
        T s = y[i];
        for (int k = i + 1; k < 6; ++k) s -= L[k][i] * x[k];
        x[i] = s / L[i][i];
    }
}

// Rotation from the ICP angles: the reference calls glm::orientate3(vec3(beta, alpha, gamma))
// (project/src/icp.cpp:82), documented as the Euler composition Y * X * Z, which with that
// argument order is  R_y(gamma) * R_x(beta) * R_z(alpha)  -- beta about x, gamma about y,
// alpha about z.
template <class T> M3<T> euler_yxz(T beta, T gamma, T alpha) {
    const T cx = std::cos(beta), sx = std::sin(beta);
    const T cy = std::cos(gamma), sy = std::sin(gamma);
    const T cz = std::cos(alpha), sz = std::sin(alpha);
    // rows of R = Ry * Rx * Rz
    const T r00 = cy * cz + sy * sx * sz, r01 = -cy * sz + sy * sx * cz, r02 = sy * cx;
    const T r10 = cx * sz, r11 = cx * cz, r12 = -sx;
    const T r20 = -sy * cz + cy * sx * sz, r21 = sy * sz + cy * sx * cz, r22 = cy * cx;
    M3<T> m;
    m.c[0][0] = r00; m.c[0][1] = r10; m.c[0][2] = r20;
    m.c[1][0] = r01; m.c[1][1] = r11; m.c[1][2] = r21;
    m.c[2][0] = r02; m.c[2][1] = r12; m.c[2][2] = r22;
    return m;
}

// ICP::updatePose, project/src/icp.cpp:65-87.  Returns false for a non-finite solution.
template <class T> bool update_pose(Pose<T>& P, const T x[6]) {
    for (int q = 0; q < 6; ++q)
        if (!std::isfinite(x[q])) return false;
    const M3<T> dR = euler_yxz(x[0], x[1], x[2]);
    const M3<T> dRt = transpose(dR);
    P.R = mul(dRt, P.R);
    P.t = add(mul(dRt, P.t), V3<T>{x[3], x[4], x[5]});
    return true;
}

// poseError, project/src/general_helper.cpp:11-21
template <class T> void pose_error(const Pose<T>& a, const Pose<T>& b, T& ang, T& dist) {
    const V3<T> v = normalize(V3<T>{T(1), T(1), T(1)});
    ang = length(sub(mul(a.R, v), mul(b.R, v)));
    dist = length(sub(a.t, b.t));
}

// ---- pipeline state (the reference's KinectFusion, project/src/kinect_fusion.cpp) ----

template <class T> struct Pipeline {
    kf_config cfg{};
    int L = 1;
    int w[KF_MAX_LEVELS]{}, h[KF_MAX_LEVELS]{};
    int cw[KF_MAX_LEVELS]{}, ch[KF_MAX_LEVELS]{}, icw[KF_MAX_LEVELS]{}, ich[KF_MAX_LEVELS]{};
    M3<T> K[KF_MAX_LEVELS], iK[KF_MAX_LEVELS];
    std::vector<T> depth_m, depth[KF_MAX_LEVELS];
    std::vector<V4<T>> vmap[KF_MAX_LEVELS], pv[KF_MAX_LEVELS], pn[KF_MAX_LEVELS];
    std::vector<uint8_t> mask[KF_MAX_LEVELS];
    std::vector<T> F, Wt;
    int n = 0, cover_n = 0;
    Pose<T> pose{};
    int frame = 0, status = 0;
    int iters_done[KF_MAX_LEVELS]{};
    long long last_samples[KF_MAX_LEVELS]{};
    std::vector<int64_t> trace[KF_MAX_LEVELS];   // march decision traces of the last raycast
    long long last_fused = 0;
    int tex9bit = 0;

    explicit Pipeline(const kf_config& c) : cfg(c) {
        L = std::max(1, std::min(c.levels, KF_MAX_LEVELS));
        for (int l = 0; l < L; ++l) {
            w[l] = c.width >> l;
            h[l] = c.height >> l;
            cw[l] = cover8(w[l], c.compat_trunc8);
            ch[l] = cover8(h[l], c.compat_trunc8);
            icw[l] = cover_icp(w[l], c.compat_trunc8);
            ich[l] = cover_icp(h[l], c.compat_trunc8);
            K[l] = intrinsics<T>(c, l);
            iK[l] = inverse(K[l]);
            depth[l].assign(size_t(w[l]) * h[l], T(0));
            vmap[l].assign(size_t(w[l]) * h[l], V4<T>{0, 0, 0, 0});
            pv[l].assign(size_t(w[l]) * h[l], V4<T>{0, 0, 0, 0});
            pn[l].assign(size_t(w[l]) * h[l], V4<T>{0, 0, 0, 0});
            mask[l].assign(size_t(w[l]) * h[l], 0);
            trace[l].assign(size_t(w[l]) * h[l], 0);
        }
        depth_m.assign(size_t(c.width) * c.height, T(0));
        n = c.volume_n;
        cover_n = cover8(n, c.compat_trunc8);
        reset();
    }
    void reset() {
        const size_t nv = size_t(n) * n * n;
        F.assign(nv, T(2));   // Voxel{f = 2, w = 0}, project/src/voxel_grid.h:8-15
        Wt.assign(nv, T(0));
        pose = pose_from16<T>(cfg.initial_pose);
        frame = 0;
        status = 0;
    }
    void fuse_now() {
        last_fused = fuse(depth_m.data(), cfg.width, cfg.height, K[0], F.data(), Wt.data(), n, cover_n,
                          cfg.volume_width, cfg.mu, cfg.max_weight, pose, cfg.min_depth, cfg.max_depth);
    }
    // KinectFusion::startTracking loop body / initializeTracking
    // (project/src/kinect_fusion.cpp:44-94, :116-183)
    int process(const uint16_t* raw) {
        for (int l = 0; l < KF_MAX_LEVELS; ++l) iters_done[l] = 0;
        convert(raw, depth_m.data(), cfg.width, cfg.height, cw[0], ch[0], cfg.depth_scale, cfg.unmirror);
        if (frame == 0) {
            fuse_now();
            ++frame;
            status = KF_OK;
            return status;
        }
        // depthFrameToVertexPyramid (:116-135)
        bilateral(depth_m.data(), depth[0].data(), w[0], h[0], cw[0], ch[0], cfg.bilateral_sigma_s,
                  cfg.bilateral_sigma_r, cfg.bilateral_radius);
        vertex_map(depth[0].data(), vmap[0].data(), w[0], cw[0], ch[0], iK[0]);
        for (int l = 1; l < L; ++l) {
            down_sample(depth[l - 1].data(), depth[l].data(), w[l], h[l], cw[l], ch[l], cfg.bilateral_sigma_r);
            vertex_map(depth[l].data(), vmap[l].data(), w[l], cw[l], ch[l], iK[l]);
        }
        // raycastTsdf (:137-144), at the previous frame's pose
        RaycastParams rp{cfg.min_depth, cfg.max_depth, cfg.step_large, cfg.step_small, cfg.keep_on_miss, tex9bit};
        for (int l = 0; l < L; ++l)
            last_samples[l] = raycast(F.data(), n, cfg.volume_width, cfg.mu, pose, iK[l], pv[l].data(),
                                      pn[l].data(), w[l], cw[l], ch[l], rp, trace[l].data());
        // computePose (:146-161) -> ICP::computePose (project/src/icp.cpp:25-58)
        Pose<T> est = pose;
        const bool ok = compute_pose(est);
        if (!ok) {
            status = KF_ERR_NONFINITE;
            ++frame;
            return status;
        }
        pose = est;
        // fuseCurrentDepthToTSDF (:179-183), unfiltered metres map
        fuse_now();
        ++frame;
        status = KF_OK;
        return status;
    }
    bool compute_pose(Pose<T>& est) {
        const Pose<T> prev = pose;
        const IcpParams ip{cfg.dist_thresh, cfg.angle_thresh};
        for (int l = L - 1; l >= 0; --l) {
            for (int it = 0; it < cfg.iters[l]; ++it) {
                NormalEq e = icp_normal_equations(vmap[l].data(), pv[l].data(), pn[l].data(), w[l], h[l], icw[l],
                                                  ich[l], prev.R, prev.t, est.R, est.t, K[l], ip,
                                                  cfg.export_icp_mask ? mask[l].data() : nullptr);
                T x[6];
                cholesky_solve<T>(e.ata, e.atb, x);
                const Pose<T> before = est;
                ++iters_done[l];
                if (!update_pose(est, x)) return false;
                T ang, dist;
                pose_error(before, est, ang, dist);
                if (ang < T(cfg.stop_angle) && dist < T(cfg.stop_dist)) break;
            }
        }
        return true;
    }
};

template <class T> void to_float4(const std::vector<V4<T>>& src, float* dst) {
    for (size_t i = 0; i < src.size(); ++i) {
        dst[4 * i + 0] = float(src[i].x);
        dst[4 * i + 1] = float(src[i].y);
        dst[4 * i + 2] = float(src[i].z);
        dst[4 * i + 3] = float(src[i].w);
    }
}
template <class T> std::vector<V4<T>> from_float4(const float* src, size_t count) {
    std::vector<V4<T>> v(count);
    for (size_t i = 0; i < count; ++i) v[i] = {T(src[4 * i]), T(src[4 * i + 1]), T(src[4 * i + 2]), T(src[4 * i + 3])};
    return v;
}
template <class T> std::vector<T> from_float(const float* src, size_t count) {
    return std::vector<T>(src, src + count);
}

struct PipelineHandle {
    int prec;
    void* p;
};

}  // namespace

// ------------------------------------------------------------------------------------------
// C entry points (loaded with ctypes by tests/ and bench.py).  prec: 0 = float, 1 = double.
// Map arguments are float32 arrays laid out as in include/kf_api.h.
// ------------------------------------------------------------------------------------------
extern "C" {

int kfo_version(void) { return 1; }

float kfo_half_value(uint16_t u) { return u16_to_half_value(u); }

int kfo_convert(const uint16_t* raw, float* out, int w, int h, float scale, int unmirror, int trunc8) {
    convert<float>(raw, out, w, h, cover8(w, trunc8), cover8(h, trunc8), scale, unmirror);
    return 0;
}

int kfo_bilateral(const float* in, float* out, int w, int h, float ss, float sr, int radius, int trunc8,
                  int prec) {
    if (prec) {
        std::vector<double> a = from_float<double>(in, size_t(w) * h), b(size_t(w) * h);
        for (size_t i = 0; i < b.size(); ++i) b[i] = out[i];
        bilateral<double>(a.data(), b.data(), w, h, cover8(w, trunc8), cover8(h, trunc8), ss, sr, radius);
        for (size_t i = 0; i < b.size(); ++i) out[i] = float(b[i]);
    } else {
        bilateral<float>(in, out, w, h, cover8(w, trunc8), cover8(h, trunc8), ss, sr, radius);
    }
    return 0;
}

int kfo_down_sample(const float* in, float* out, int w_out, int h_out, float sr, int trunc8, int prec) {
    if (prec) {
        std::vector<double> a = from_float<double>(in, size_t(w_out) * h_out * 4), b(size_t(w_out) * h_out);
        for (size_t i = 0; i < b.size(); ++i) b[i] = out[i];
        down_sample<double>(a.data(), b.data(), w_out, h_out, cover8(w_out, trunc8), cover8(h_out, trunc8), sr);
        for (size_t i = 0; i < b.size(); ++i) out[i] = float(b[i]);
    } else {
        down_sample<float>(in, out, w_out, h_out, cover8(w_out, trunc8), cover8(h_out, trunc8), sr);
    }
    return 0;
}

int kfo_vertex_map(const float* depth, float* vmap, int w, int h, const float inv_k[9], int trunc8, int prec) {
    const size_t np = size_t(w) * h;
    if (prec) {
        std::vector<double> d = from_float<double>(depth, np);
        std::vector<V4<double>> v = from_float4<double>(vmap, np);
        vertex_map<double>(d.data(), v.data(), w, cover8(w, trunc8), cover8(h, trunc8), from_flat9<double>(inv_k));
        to_float4(v, vmap);
    } else {
        std::vector<V4<float>> v = from_float4<float>(vmap, np);
        vertex_map<float>(depth, v.data(), w, cover8(w, trunc8), cover8(h, trunc8), from_flat9<float>(inv_k));
        to_float4(v, vmap);
    }
    return 0;
}

int kfo_normal_map(const float* vmap, float* nmap, int w, int h, int trunc8, int prec) {
    const size_t np = size_t(w) * h;
    if (prec) {
        std::vector<V4<double>> v = from_float4<double>(vmap, np), nn = from_float4<double>(nmap, np);
        normal_map<double>(v.data(), nn.data(), w, h, cover8(w, trunc8), cover8(h, trunc8));
        to_float4(nn, nmap);
    } else {
        std::vector<V4<float>> v = from_float4<float>(vmap, np), nn = from_float4<float>(nmap, np);
        normal_map<float>(v.data(), nn.data(), w, h, cover8(w, trunc8), cover8(h, trunc8));
        to_float4(nn, nmap);
    }
    return 0;
}

// computeNormal at one pixel (test/transformation_tests.cpp:41-59 wraps the device helper)
int kfo_compute_normal(const float* vmap, int w, int h, int i, int j, float out[4]) {
    std::vector<V4<float>> v = from_float4<float>(vmap, size_t(w) * h);
    V4<float> n = compute_normal(v.data(), w, h, i, j);
    out[0] = n.x; out[1] = n.y; out[2] = n.z; out[3] = n.w;
    return 0;
}

// trace (may be NULL): w * h march decision traces (march_trace)
long long kfo_raycast(const float* tsdf_f, int n, float width, float mu, const float pose[16],
                      const float inv_k[9], float* vmap, float* nmap, int w, int h, float min_d, float max_d,
                      float step_l, float step_s, int keep_on_miss, int tex9bit, int trunc8, int prec,
                      int64_t* trace, int exact_positions) {
    const size_t np = size_t(w) * h;
    RaycastParams rp{min_d, max_d, step_l, step_s, keep_on_miss, tex9bit, exact_positions};
    long long samples;
    if (prec) {
        std::vector<double> f = from_float<double>(tsdf_f, size_t(n) * n * n);
        std::vector<V4<double>> v = from_float4<double>(vmap, np), nn = from_float4<double>(nmap, np);
        samples = raycast<double>(f.data(), n, width, mu, pose_from16<double>(pose), from_flat9<double>(inv_k),
                                  v.data(), nn.data(), w, cover8(w, trunc8), cover8(h, trunc8), rp, trace);
        to_float4(v, vmap);
        to_float4(nn, nmap);
    } else {
        std::vector<V4<float>> v = from_float4<float>(vmap, np), nn = from_float4<float>(nmap, np);
        samples = raycast<float>(tsdf_f, n, width, mu, pose_from16<float>(pose), from_flat9<float>(inv_k),
                                 v.data(), nn.data(), w, cover8(w, trunc8), cover8(h, trunc8), rp, trace);
        to_float4(v, vmap);
        to_float4(nn, nmap);
    }
    return samples;
}

long long kfo_fuse(const float* depth_m, int w, int h, const float k[9], float* tsdf_f, float* tsdf_w, int n,
                   float width, float mu, float max_w, const float pose[16], float min_d, float max_d, int trunc8,
                   int prec) {
    const size_t nv = size_t(n) * n * n;
    long long upd;
    if (prec) {
        std::vector<double> d = from_float<double>(depth_m, size_t(w) * h);
        std::vector<double> F = from_float<double>(tsdf_f, nv), W = from_float<double>(tsdf_w, nv);
        upd = fuse<double>(d.data(), w, h, from_flat9<double>(k), F.data(), W.data(), n, cover8(n, trunc8), width,
                           mu, max_w, pose_from16<double>(pose), min_d, max_d);
        for (size_t i = 0; i < nv; ++i) { tsdf_f[i] = float(F[i]); tsdf_w[i] = float(W[i]); }
    } else {
        upd = fuse<float>(depth_m, w, h, from_flat9<float>(k), tsdf_f, tsdf_w, n, cover8(n, trunc8), width, mu,
                          max_w, pose_from16<float>(pose), min_d, max_d);
    }
    return upd;
}

// voxel-centre coordinate tables (x/y axis and accumulated z axis), for the tests
int kfo_voxel_axes(int n, float width, float* xs, float* zs) {
    std::vector<float> a, b;
    voxel_axes(n, width, a, b);
    std::memcpy(xs, a.data(), sizeof(float) * n);
    std::memcpy(zs, b.data(), sizeof(float) * n);
    return 0;
}

// constructIcpResiduals for a whole map: A row-major (w*h x 6), b (w*h).  Rows outside the
// (trunc8) cover are left untouched.  Returns the number of residual rows.
int kfo_icp_residuals(const float* vmap, const float* tv, const float* tn, int w, int h, const float prev_R[9],
                      const float prev_t[3], const float cur_R[9], const float cur_t[3], const float k[9],
                      float dist, float angle, float* A, float* b, uint8_t* mask, int trunc8) {
    const size_t np = size_t(w) * h;
    std::vector<V4<float>> v = from_float4<float>(vmap, np), a2 = from_float4<float>(tv, np),
                           a3 = from_float4<float>(tn, np);
    const M3<float> Rp = from_flat9<float>(prev_R), Rc = from_flat9<float>(cur_R), K = from_flat9<float>(k);
    const V3<float> tp{prev_t[0], prev_t[1], prev_t[2]}, tc{cur_t[0], cur_t[1], cur_t[2]};
    const IcpParams ip{dist, angle};
    const int cw = cover_icp(w, trunc8), ch = cover_icp(h, trunc8);
    int count = 0;
    for (int vv = 0; vv < ch; ++vv)
        for (int u = 0; u < cw; ++u) {
            float a[6], bb;
            const bool ok = icp_row(v.data(), a2.data(), a3.data(), w, h, u, vv, Rp, tp, Rc, tc, K, ip, a, bb);
            const size_t idx = size_t(vv) * w + u;
            for (int q = 0; q < 6; ++q) A[idx * 6 + q] = a[q];
            b[idx] = bb;
            if (mask) mask[idx] = ok ? 1 : 0;
            count += ok ? 1 : 0;
        }
    return count;
}

// computeAndFillA / computeAndFillB (project/src/icp.cuh:72-95) for one correspondence:
// s = transformed source vertex, n = target normal, d = target vertex
int kfo_fill_a_b(const float s[3], const float n[3], const float d[3], float a[6], float* b) {
    a[0] = n[1] * s[2] - n[2] * s[1];
    a[1] = n[2] * s[0] - n[0] * s[2];
    a[2] = n[0] * s[1] - n[1] * s[0];
    a[3] = n[0]; a[4] = n[1]; a[5] = n[2];
    *b = n[0] * d[0] + n[1] * d[1] + n[2] * d[2] - n[0] * s[0] - n[1] * s[1] - n[2] * s[2];
    return 0;
}

// LinearLeastSquares::solve (project/src/linear_least_squares.cpp:23-44)
int kfo_solve_lls(const float* A, const float* b, int n, float x[6], int prec) {
    double ata[36] = {}, atb[6] = {};
    for (int i = 0; i < n; ++i)
        for (int r = 0; r < 6; ++r) {
            for (int c = 0; c < 6; ++c) ata[r * 6 + c] += double(A[size_t(i) * 6 + r]) * double(A[size_t(i) * 6 + c]);
            atb[r] += double(A[size_t(i) * 6 + r]) * double(b[i]);
        }
    if (prec) {
        double xd[6];
        cholesky_solve<double>(ata, atb, xd);
        for (int q = 0; q < 6; ++q) x[q] = float(xd[q]);
    } else {
        cholesky_solve<float>(ata, atb, x);
    }
    return 0;
}

// ICP::updatePose (project/src/icp.cpp:65-87) on a column-major 4x4
int kfo_update_pose(float pose[16], const float x[6], int prec) {
    if (prec) {
        Pose<double> P = pose_from16<double>(pose);
        double xd[6];
        for (int q = 0; q < 6; ++q) xd[q] = x[q];
        if (!update_pose(P, xd)) return KF_ERR_NONFINITE;
        pose_to16(P, pose);
    } else {
        Pose<float> P = pose_from16<float>(pose);
        if (!update_pose(P, x)) return KF_ERR_NONFINITE;
        pose_to16(P, pose);
    }
    return 0;
}

int kfo_euler_yxz(float beta, float gamma, float alpha, float out9[9]) {
    M3<double> m = euler_yxz<double>(beta, gamma, alpha);
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) out9[c * 3 + r] = float(m.c[c][r]);
    return 0;
}

int kfo_pose_error(const float p1[16], const float p2[16], float out[2]) {
    float a, d;
    pose_error(pose_from16<float>(p1), pose_from16<float>(p2), a, d);
    out[0] = a;
    out[1] = d;
    return 0;
}

// computeCorrespondence (project/src/icp.cuh:40-48) for one vertex
int kfo_compute_correspondence(const float vtx[3], const float R[9], const float t[3], const float k[9], int out[2]) {
    const M3<float> Rm = from_flat9<float>(R), K = from_flat9<float>(k);
    const V3<float> s{vtx[0], vtx[1], vtx[2]}, tt{t[0], t[1], t[2]};
    const V3<float> pt = mul(mul(K, transpose(Rm)), sub(s, tt));
    out[0] = to_int_device(std::floor(pt.x / pt.z));
    out[1] = to_int_device(std::floor(pt.y / pt.z));
    return 0;
}

// areNormalsTooDifferent (project/src/icp.cuh:56-64)
int kfo_normals_too_different(const float n[3], const float tn[3], const float R[9], float angle) {
    const M3<float> Rm = from_flat9<float>(R);
    const V3<float> nr = normalize(mul(Rm, V3<float>{n[0], n[1], n[2]}));
    const float ang = std::acos(dot(nr, V3<float>{tn[0], tn[1], tn[2]}));
    return ang > angle ? 1 : 0;
}

// ICP::computePose on given pyramids (each pointer array holds `levels` maps)
int kfo_compute_pose(const float* const* vmaps, const float* const* tvs, const float* const* tns, const kf_config* c,
                     const float pose[16], float pose_out[16], int iters_out[KF_MAX_LEVELS], int prec) {
    auto run = [&](auto tag) -> int {
        using T = decltype(tag);
        Pipeline<T> P(*c);
        for (int l = 0; l < P.L; ++l) {
            const size_t np = size_t(P.w[l]) * P.h[l];
            P.vmap[l] = from_float4<T>(vmaps[l], np);
            P.pv[l] = from_float4<T>(tvs[l], np);
            P.pn[l] = from_float4<T>(tns[l], np);
        }
        P.pose = pose_from16<T>(pose);
        Pose<T> est = P.pose;
        const bool ok = P.compute_pose(est);
        for (int l = 0; l < KF_MAX_LEVELS; ++l) iters_out[l] = P.iters_done[l];
        pose_to16(est, pose_out);
        return ok ? 0 : KF_ERR_NONFINITE;
    };
    return prec ? run(double(0)) : run(float(0));
}

// ---- pipeline ----

void* kfo_pipeline_create(const kf_config* c, int prec, int tex9bit) {
    PipelineHandle* h = new PipelineHandle;
    h->prec = prec;
    if (prec) {
        auto* p = new Pipeline<double>(*c);
        p->tex9bit = tex9bit;
        h->p = p;
    } else {
        auto* p = new Pipeline<float>(*c);
        p->tex9bit = tex9bit;
        h->p = p;
    }
    return h;
}

void kfo_pipeline_destroy(void* hp) {
    PipelineHandle* h = static_cast<PipelineHandle*>(hp);
    if (!h) return;
    if (h->prec) delete static_cast<Pipeline<double>*>(h->p);
    else delete static_cast<Pipeline<float>*>(h->p);
    delete h;
}

#define KFO_DISPATCH(h, expr)                                             \
    do {                                                                  \
        PipelineHandle* hh = static_cast<PipelineHandle*>(h);             \
        if (hh->prec) {                                                   \
            auto* P = static_cast<Pipeline<double>*>(hh->p);              \
            expr;                                                         \
        } else {                                                          \
            auto* P = static_cast<Pipeline<float>*>(hh->p);               \
            expr;                                                         \
        }                                                                 \
    } while (0)

int kfo_pipeline_frame(void* h, const uint16_t* raw, float pose_out[16]) {
    int st = 0;
    KFO_DISPATCH(h, { st = P->process(raw); if (pose_out) pose_to16(P->pose, pose_out); });
    return st;
}

int kfo_pipeline_reset(void* h) {
    KFO_DISPATCH(h, P->reset());
    return 0;
}

int kfo_pipeline_get_pose(void* h, float pose[16]) {
    KFO_DISPATCH(h, pose_to16(P->pose, pose));
    return 0;
}

int kfo_pipeline_set_pose(void* hp, const float pose[16]) {
    PipelineHandle* h = static_cast<PipelineHandle*>(hp);
    if (h->prec) static_cast<Pipeline<double>*>(h->p)->pose = pose_from16<double>(pose);
    else static_cast<Pipeline<float>*>(h->p)->pose = pose_from16<float>(pose);
    return 0;
}

int kfo_pipeline_get_iters(void* h, int iters[KF_MAX_LEVELS]) {
    KFO_DISPATCH(h, for (int l = 0; l < KF_MAX_LEVELS; ++l) iters[l] = P->iters_done[l]);
    return 0;
}

int kfo_pipeline_get_depth(void* h, int level, float* dst) {
    KFO_DISPATCH(h, {
        const auto& v = level < 0 ? P->depth_m : P->depth[level];
        for (size_t i = 0; i < v.size(); ++i) dst[i] = float(v[i]);
    });
    return 0;
}

int kfo_pipeline_get_vertex(void* h, int level, float* dst) {
    KFO_DISPATCH(h, to_float4(P->vmap[level], dst));
    return 0;
}

int kfo_pipeline_get_raycast(void* h, int level, float* vtx, float* nrm) {
    KFO_DISPATCH(h, { to_float4(P->pv[level], vtx); to_float4(P->pn[level], nrm); });
    return 0;
}

// march decision traces of the last frame's raycast at `level` (march_trace encoding)
int kfo_pipeline_get_trace(void* h, int level, int64_t* dst) {
    KFO_DISPATCH(h, std::memcpy(dst, P->trace[level].data(), P->trace[level].size() * sizeof(int64_t)));
    return 0;
}

int kfo_pipeline_get_mask(void* h, int level, uint8_t* dst) {
    KFO_DISPATCH(h, std::memcpy(dst, P->mask[level].data(), P->mask[level].size()));
    return 0;
}

// distance and weight arrays (n^3 each, x fastest), as float
int kfo_pipeline_get_tsdf(void* h, float* f, float* w) {
    KFO_DISPATCH(h, {
        for (size_t i = 0; i < P->F.size(); ++i) { f[i] = float(P->F[i]); w[i] = float(P->Wt[i]); }
    });
    return 0;
}

int kfo_pipeline_set_tsdf(void* h, const float* f, const float* w) {
    KFO_DISPATCH(h, {
        for (size_t i = 0; i < P->F.size(); ++i) { P->F[i] = f[i]; P->Wt[i] = w[i]; }
    });
    return 0;
}

long long kfo_pipeline_last_samples(void* h, int level) {
    long long s = 0;
    KFO_DISPATCH(h, s = P->last_samples[level]);
    return s;
}

long long kfo_pipeline_last_fused(void* h) {
    long long s = 0;
    KFO_DISPATCH(h, s = P->last_fused);
    return s;
}

// ---- display kernels (project/src/display.cu:63-105), RGBA8 out ----

// static_cast<unsigned char>(x) on the device: truncation, saturated to [0, 255], NaN -> 0
static unsigned to_u8(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 255.0f) return 255u;
    return unsigned(x);
}

// normalMapToWindowContentKernel (display.cu:63-81): normalize(Rinv * n) * 255 as r, g, b
void kfo_display_normals(const float* nm, int w, int h, const float rinv[9], unsigned char* rgba) {
    for (int j = 0; j < h; ++j)
        for (int i = 0; i < w; ++i) {
            const float* n = nm + (size_t(j) * w + i) * 4;
            float v[3];
            for (int r = 0; r < 3; ++r) v[r] = rinv[r] * n[0] + rinv[3 + r] * n[1] + rinv[6 + r] * n[2];
            const float s = 1.0f / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            unsigned char* o = rgba + (size_t(j) * w + i) * 4;
            for (int r = 0; r < 3; ++r) o[r] = (unsigned char)to_u8(v[r] * s * 255.0f);
            o[3] = 255;
        }
}

// shadingToWindowContentKernel (display.cu:83-105): min(|n . normalize(R K^-1 (i+.5, j+.5, 1))|, 1)
void kfo_display_shading(const float* nm, int w, int h, const float pose[16], const float ik[9], unsigned char* rgba) {
    for (int j = 0; j < h; ++j)
        for (int i = 0; i < w; ++i) {
            const float p[3] = {float(i) + 0.5f, float(j) + 0.5f, 1.0f};
            float q[3], d[3];
            for (int r = 0; r < 3; ++r) q[r] = ik[r] * p[0] + ik[3 + r] * p[1] + ik[6 + r] * p[2];
            for (int r = 0; r < 3; ++r) d[r] = pose[r] * q[0] + pose[4 + r] * q[1] + pose[8 + r] * q[2];
            const float s = 1.0f / std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            const float* n = nm + (size_t(j) * w + i) * 4;
            const float rad = std::min(std::fabs((n[0] * d[0] + n[1] * d[1] + n[2] * d[2]) * s), 1.0f);
            unsigned char* o = rgba + (size_t(j) * w + i) * 4;
            o[0] = o[1] = o[2] = (unsigned char)to_u8(rad * 255.0f);
            o[3] = 255;
        }
}

}  // extern "C"
