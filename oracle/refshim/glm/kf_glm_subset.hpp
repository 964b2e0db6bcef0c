// TEST INFRASTRUCTURE ONLY: the part of the glm math library that the reference's compute
// files call, so that those files compile as they are, where they lie.
//
// glm (OpenGL Mathematics, https://github.com/g-truc/glm) is a git submodule of the
// reference (.gitmodules: 3rd/glm) that the reference's checkout leaves empty, at no pinned
// commit.  This header restates, in new code, the published definitions of the types and
// functions the compiled reference files use (GLSL semantics: column-major matrices, m[c][r]
// is column c, row r; matrix * vector sums the columns scaled by the vector's components):
//   vec2, vec3, vec4, ivec2, mat3, mat4; + - * / on vectors and scalars; matrix * vector and
//   matrix * matrix; dot, cross, length, distance, normalize (v * 1 / sqrt(dot(v, v))),
//   transpose, inverse (adjugate / determinant), floor, min, max, abs, acos, radians,
//   degrees, orientate3 / yawPitchRoll (R = Ry(yaw) Rx(pitch) Rz(roll); orientate3(a)
//   = yawPitchRoll(a.z, a.x, a.y)), and tquat with mat3_cast / mat4_cast (the rotation
//   matrix of a unit quaternion).
// The order in which the sums are written follows those definitions; where the absent
// library wrote a sum in another order, results differ from a build with it in the last
// bit only.  Nothing in the CUDA library includes this header.
#pragma once

#include <cmath>
#include <cuda_runtime.h>

#if defined(__CUDACC__)
#define KFG_HD __host__ __device__ __forceinline__
#else
#define KFG_HD inline
#endif

namespace glm {

struct vec4;

struct vec2 {
    float x, y;
    KFG_HD vec2() : x(0.f), y(0.f) {}
    KFG_HD explicit vec2(float s) : x(s), y(s) {}
    KFG_HD vec2(float a, float b) : x(a), y(b) {}
    KFG_HD float& operator[](int i) { return (&x)[i]; }
    KFG_HD const float& operator[](int i) const { return (&x)[i]; }
};

struct ivec2 {
    int x, y;
    KFG_HD ivec2() : x(0), y(0) {}
    KFG_HD explicit ivec2(int s) : x(s), y(s) {}
    KFG_HD ivec2(int a, int b) : x(a), y(b) {}
    KFG_HD ivec2 operator-(const ivec2& o) const { return ivec2(x - o.x, y - o.y); }
};

struct vec3 {
    float x, y, z;
    KFG_HD vec3() : x(0.f), y(0.f), z(0.f) {}
    KFG_HD explicit vec3(float s) : x(s), y(s), z(s) {}
    template <class A, class B, class C>
    KFG_HD vec3(A a, B b, C c) : x(static_cast<float>(a)), y(static_cast<float>(b)), z(static_cast<float>(c)) {}
    KFG_HD vec3(const vec4& v);   // drops w (glm converts implicitly)
    KFG_HD float& operator[](int i) { return (&x)[i]; }
    KFG_HD const float& operator[](int i) const { return (&x)[i]; }
    KFG_HD vec3& operator+=(const vec3& o) { x += o.x; y += o.y; z += o.z; return *this; }
    KFG_HD vec3& operator-=(const vec3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    KFG_HD vec3& operator*=(float s) { x *= s; y *= s; z *= s; return *this; }
    KFG_HD vec3& operator/=(float s) { x /= s; y /= s; z /= s; return *this; }
};

struct vec4 {
    float x, y, z, w;
    KFG_HD vec4() : x(0.f), y(0.f), z(0.f), w(0.f) {}
    KFG_HD explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
    template <class A, class B, class C, class D>
    KFG_HD vec4(A a, B b, C c, D d)
        : x(static_cast<float>(a)), y(static_cast<float>(b)), z(static_cast<float>(c)), w(static_cast<float>(d)) {}
    KFG_HD vec4(const vec3& v, float s) : x(v.x), y(v.y), z(v.z), w(s) {}
    KFG_HD float& operator[](int i) { return (&x)[i]; }
    KFG_HD const float& operator[](int i) const { return (&x)[i]; }
};

KFG_HD vec3::vec3(const vec4& v) : x(v.x), y(v.y), z(v.z) {}

// ---- vector arithmetic (componentwise) ----
KFG_HD vec3 operator+(const vec3& a, const vec3& b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
KFG_HD vec3 operator-(const vec3& a, const vec3& b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
KFG_HD vec3 operator*(const vec3& a, const vec3& b) { return vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
KFG_HD vec3 operator/(const vec3& a, const vec3& b) { return vec3(a.x / b.x, a.y / b.y, a.z / b.z); }
KFG_HD vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }
KFG_HD vec3 operator+(const vec3& a, float s) { return vec3(a.x + s, a.y + s, a.z + s); }
KFG_HD vec3 operator-(const vec3& a, float s) { return vec3(a.x - s, a.y - s, a.z - s); }
KFG_HD vec3 operator*(const vec3& a, float s) { return vec3(a.x * s, a.y * s, a.z * s); }
KFG_HD vec3 operator*(float s, const vec3& a) { return vec3(s * a.x, s * a.y, s * a.z); }
KFG_HD vec3 operator/(const vec3& a, float s) { return vec3(a.x / s, a.y / s, a.z / s); }
KFG_HD vec3 operator/(float s, const vec3& a) { return vec3(s / a.x, s / a.y, s / a.z); }
KFG_HD bool operator==(const vec3& a, const vec3& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

KFG_HD vec4 operator+(const vec4& a, const vec4& b) { return vec4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
KFG_HD vec4 operator-(const vec4& a, const vec4& b) { return vec4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
KFG_HD vec4 operator*(const vec4& a, float s) { return vec4(a.x * s, a.y * s, a.z * s, a.w * s); }
KFG_HD vec4 operator*(float s, const vec4& a) { return vec4(s * a.x, s * a.y, s * a.z, s * a.w); }
KFG_HD vec4 operator/(const vec4& a, float s) { return vec4(a.x / s, a.y / s, a.z / s, a.w / s); }

KFG_HD vec2 operator-(const vec2& a, const vec2& b) { return vec2(a.x - b.x, a.y - b.y); }
KFG_HD vec2 operator*(const vec2& a, float s) { return vec2(a.x * s, a.y * s); }

// ---- matrices: columns ----
struct mat4;

struct mat3 {
    vec3 c[3];
    KFG_HD mat3() : mat3(1.0f) {}
    KFG_HD explicit mat3(float d) {
        c[0] = vec3(d, 0.f, 0.f);
        c[1] = vec3(0.f, d, 0.f);
        c[2] = vec3(0.f, 0.f, d);
    }
    KFG_HD mat3(const vec3& a, const vec3& b, const vec3& d) { c[0] = a; c[1] = b; c[2] = d; }
    KFG_HD explicit mat3(const mat4& m);   // upper-left 3 x 3
    KFG_HD vec3& operator[](int i) { return c[i]; }
    KFG_HD const vec3& operator[](int i) const { return c[i]; }
};

struct mat4 {
    vec4 c[4];
    KFG_HD mat4() : mat4(1.0f) {}
    KFG_HD explicit mat4(float d) {
        c[0] = vec4(d, 0.f, 0.f, 0.f);
        c[1] = vec4(0.f, d, 0.f, 0.f);
        c[2] = vec4(0.f, 0.f, d, 0.f);
        c[3] = vec4(0.f, 0.f, 0.f, d);
    }
    KFG_HD mat4(const vec4& a, const vec4& b, const vec4& d, const vec4& e) { c[0] = a; c[1] = b; c[2] = d; c[3] = e; }
    KFG_HD explicit mat4(const mat3& m) {   // m in the upper left, 1 at [3][3]
        c[0] = vec4(m[0], 0.f);
        c[1] = vec4(m[1], 0.f);
        c[2] = vec4(m[2], 0.f);
        c[3] = vec4(0.f, 0.f, 0.f, 1.f);
    }
    KFG_HD vec4& operator[](int i) { return c[i]; }
    KFG_HD const vec4& operator[](int i) const { return c[i]; }
};

KFG_HD mat3::mat3(const mat4& m) {
    c[0] = vec3(m[0]);
    c[1] = vec3(m[1]);
    c[2] = vec3(m[2]);
}

// matrix * vector: column 0 scaled by v.x, plus column 1 by v.y, plus column 2 by v.z
KFG_HD vec3 operator*(const mat3& m, const vec3& v) {
    return vec3(m[0][0] * v.x + m[1][0] * v.y + m[2][0] * v.z,
                m[0][1] * v.x + m[1][1] * v.y + m[2][1] * v.z,
                m[0][2] * v.x + m[1][2] * v.y + m[2][2] * v.z);
}
KFG_HD vec4 operator*(const mat4& m, const vec4& v) {
    return vec4(m[0][0] * v.x + m[1][0] * v.y + m[2][0] * v.z + m[3][0] * v.w,
                m[0][1] * v.x + m[1][1] * v.y + m[2][1] * v.z + m[3][1] * v.w,
                m[0][2] * v.x + m[1][2] * v.y + m[2][2] * v.z + m[3][2] * v.w,
                m[0][3] * v.x + m[1][3] * v.y + m[2][3] * v.z + m[3][3] * v.w);
}
// matrix * matrix: column j of the product is a * b[j]
KFG_HD mat3 operator*(const mat3& a, const mat3& b) { return mat3(a * b[0], a * b[1], a * b[2]); }
KFG_HD mat4 operator*(const mat4& a, const mat4& b) { return mat4(a * b[0], a * b[1], a * b[2], a * b[3]); }
KFG_HD mat3 operator*(const mat3& a, float s) { return mat3(a[0] * s, a[1] * s, a[2] * s); }

// ---- geometric functions ----
KFG_HD float dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
KFG_HD float dot(const vec4& a, const vec4& b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
KFG_HD vec3 cross(const vec3& a, const vec3& b) {
    return vec3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
KFG_HD float inversesqrt(float x) { return 1.0f / sqrtf(x); }
KFG_HD float length(const vec3& v) { return sqrtf(dot(v, v)); }
KFG_HD float distance(const vec3& a, const vec3& b) { return length(b - a); }
KFG_HD vec3 normalize(const vec3& v) { return v * inversesqrt(dot(v, v)); }

// ---- common functions (scalar forms) ----
KFG_HD float floor(float x) { return floorf(x); }
KFG_HD float abs(float x) { return fabsf(x); }
KFG_HD float acos(float x) { return acosf(x); }
KFG_HD float min(float a, float b) { return (b < a) ? b : a; }
KFG_HD float max(float a, float b) { return (a < b) ? b : a; }
KFG_HD float radians(float deg) { return deg * 0.01745329251994329576923690768489f; }
KFG_HD float degrees(float rad) { return rad * 57.295779513082320876798154814105f; }

// ---- matrix functions ----
KFG_HD mat3 transpose(const mat3& m) {
    return mat3(vec3(m[0][0], m[1][0], m[2][0]), vec3(m[0][1], m[1][1], m[2][1]), vec3(m[0][2], m[1][2], m[2][2]));
}

// inverse = adjugate / determinant (cofactor expansion along the first column)
KFG_HD mat3 inverse(const mat3& m) {
    const float c00 = m[1][1] * m[2][2] - m[2][1] * m[1][2];
    const float c01 = m[0][1] * m[2][2] - m[2][1] * m[0][2];
    const float c02 = m[0][1] * m[1][2] - m[1][1] * m[0][2];
    const float det = m[0][0] * c00 - m[1][0] * c01 + m[2][0] * c02;
    const float s = 1.0f / det;
    mat3 r;
    r[0][0] = +c00 * s;
    r[1][0] = -(m[1][0] * m[2][2] - m[2][0] * m[1][2]) * s;
    r[2][0] = +(m[1][0] * m[2][1] - m[2][0] * m[1][1]) * s;
    r[0][1] = -c01 * s;
    r[1][1] = +(m[0][0] * m[2][2] - m[2][0] * m[0][2]) * s;
    r[2][1] = -(m[0][0] * m[2][1] - m[2][0] * m[0][1]) * s;
    r[0][2] = +c02 * s;
    r[1][2] = -(m[0][0] * m[1][2] - m[1][0] * m[0][2]) * s;
    r[2][2] = +(m[0][0] * m[1][1] - m[1][0] * m[0][1]) * s;
    return r;
}

// inverse of a 4 x 4 by the 2 x 2 sub-determinants of its column pairs (Laplace expansion)
KFG_HD mat4 inverse(const mat4& m) {
    // a[i][j] = element of row i, column j
    float a[4][4];
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) a[r][c] = m[c][r];
    const float s0 = a[0][0] * a[1][1] - a[1][0] * a[0][1];
    const float s1 = a[0][0] * a[1][2] - a[1][0] * a[0][2];
    const float s2 = a[0][0] * a[1][3] - a[1][0] * a[0][3];
    const float s3 = a[0][1] * a[1][2] - a[1][1] * a[0][2];
    const float s4 = a[0][1] * a[1][3] - a[1][1] * a[0][3];
    const float s5 = a[0][2] * a[1][3] - a[1][2] * a[0][3];
    const float c5 = a[2][2] * a[3][3] - a[3][2] * a[2][3];
    const float c4 = a[2][1] * a[3][3] - a[3][1] * a[2][3];
    const float c3 = a[2][1] * a[3][2] - a[3][1] * a[2][2];
    const float c2 = a[2][0] * a[3][3] - a[3][0] * a[2][3];
    const float c1 = a[2][0] * a[3][2] - a[3][0] * a[2][2];
    const float c0 = a[2][0] * a[3][1] - a[3][0] * a[2][1];
    const float det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
    const float k = 1.0f / det;
    float b[4][4];
    b[0][0] = (a[1][1] * c5 - a[1][2] * c4 + a[1][3] * c3) * k;
    b[0][1] = (-a[0][1] * c5 + a[0][2] * c4 - a[0][3] * c3) * k;
    b[0][2] = (a[3][1] * s5 - a[3][2] * s4 + a[3][3] * s3) * k;
    b[0][3] = (-a[2][1] * s5 + a[2][2] * s4 - a[2][3] * s3) * k;
    b[1][0] = (-a[1][0] * c5 + a[1][2] * c2 - a[1][3] * c1) * k;
    b[1][1] = (a[0][0] * c5 - a[0][2] * c2 + a[0][3] * c1) * k;
    b[1][2] = (-a[3][0] * s5 + a[3][2] * s2 - a[3][3] * s1) * k;
    b[1][3] = (a[2][0] * s5 - a[2][2] * s2 + a[2][3] * s1) * k;
    b[2][0] = (a[1][0] * c4 - a[1][1] * c2 + a[1][3] * c0) * k;
    b[2][1] = (-a[0][0] * c4 + a[0][1] * c2 - a[0][3] * c0) * k;
    b[2][2] = (a[3][0] * s4 - a[3][1] * s2 + a[3][3] * s0) * k;
    b[2][3] = (-a[2][0] * s4 + a[2][1] * s2 - a[2][3] * s0) * k;
    b[3][0] = (-a[1][0] * c3 + a[1][1] * c1 - a[1][2] * c0) * k;
    b[3][1] = (a[0][0] * c3 - a[0][1] * c1 + a[0][2] * c0) * k;
    b[3][2] = (-a[3][0] * s3 + a[3][1] * s1 - a[3][2] * s0) * k;
    b[3][3] = (a[2][0] * s3 - a[2][1] * s1 + a[2][2] * s0) * k;
    mat4 r;
    for (int c = 0; c < 4; ++c)
        for (int rr = 0; rr < 4; ++rr) r[c][rr] = b[rr][c];
    return r;
}

// Euler-angle rotation: R = Ry(yaw) * Rx(pitch) * Rz(roll), as a 4 x 4
KFG_HD mat4 yawPitchRoll(float yaw, float pitch, float roll) {
    const float ch = cosf(yaw), sh = sinf(yaw);
    const float cp = cosf(pitch), sp = sinf(pitch);
    const float cb = cosf(roll), sb = sinf(roll);
    mat4 r;
    r[0][0] = ch * cb + sh * sp * sb;
    r[0][1] = sb * cp;
    r[0][2] = -sh * cb + ch * sp * sb;
    r[0][3] = 0.f;
    r[1][0] = -ch * sb + sh * sp * cb;
    r[1][1] = cb * cp;
    r[1][2] = sb * sh + ch * sp * cb;
    r[1][3] = 0.f;
    r[2][0] = sh * cp;
    r[2][1] = -sp;
    r[2][2] = ch * cp;
    r[2][3] = 0.f;
    r[3] = vec4(0.f, 0.f, 0.f, 1.f);
    return r;
}

// orientate3(angles): yawPitchRoll(angles.z, angles.x, angles.y) as a 3 x 3
KFG_HD mat3 orientate3(const vec3& angles) { return mat3(yawPitchRoll(angles.z, angles.x, angles.y)); }

// ---- quaternions (the reference's TUM reader, project/src/rgbd_dataset.cpp:28-70) ----
// tquat<T>: components x, y, z (vector part) and w (scalar part), default identity
template <class T>
struct tquat {
    T x, y, z, w;
    KFG_HD tquat() : x(T(0)), y(T(0)), z(T(0)), w(T(1)) {}
};
using quat = tquat<float>;

// mat3_cast: the rotation of a unit quaternion, 1 - 2(y^2 + z^2) ... by its nine products,
// column by column (m[c][r]); mat4_cast puts it in the upper left of the identity
KFG_HD mat3 mat3_cast(const tquat<float>& q) {
    const float xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z;
    const float xz = q.x * q.z, xy = q.x * q.y, yz = q.y * q.z;
    const float wx = q.w * q.x, wy = q.w * q.y, wz = q.w * q.z;
    mat3 m;
    m[0][0] = 1.f - 2.f * (yy + zz);
    m[0][1] = 2.f * (xy + wz);
    m[0][2] = 2.f * (xz - wy);
    m[1][0] = 2.f * (xy - wz);
    m[1][1] = 1.f - 2.f * (xx + zz);
    m[1][2] = 2.f * (yz + wx);
    m[2][0] = 2.f * (xz + wy);
    m[2][1] = 2.f * (yz - wx);
    m[2][2] = 1.f - 2.f * (xx + yy);
    return m;
}
KFG_HD mat4 mat4_cast(const tquat<float>& q) { return mat4(mat3_cast(q)); }

}  // namespace glm
