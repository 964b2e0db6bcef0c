// kf_march.h -- exact fast-forward of the raycaster's repeated float additions.
//
// The reference marches t <- fl(t + inc) sample after sample (project/src/raycast.cu:75-117).
// When a run of samples is known to be skippable, the march still has to land on exactly the
// float the reference's additions would produce.  Within one binade of t the additions add a
// constant number of ulps (unless inc falls exactly halfway between two ulp multiples, where
// round-to-even alternates), so whole runs can be advanced with integer arithmetic on the
// significand; a binade boundary or a tie is crossed with one ordinary float addition.
//
// Plain C++ (the tests also compile it for the host and compare it with the sequential
// additions).
#pragma once

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define KF_HD __host__ __device__ __forceinline__
#else
#define KF_HD inline
#endif

namespace kf {

KF_HD uint32_t f2u(float x) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(x);
#else
    uint32_t u;
    memcpy(&u, &x, 4);
    return u;
#endif
}

KF_HD float u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float x;
    memcpy(&x, &u, 4);
    return x;
#endif
}

// t after k >= 0 repeated additions t <- fl(t + inc), in closed form.  True (out set) when t
// and inc are positive normal floats, inc is not a rounding tie in t's binade and the k
// additions stay inside t's binade; false otherwise, and the caller adds one by one.
KF_HD bool add_k_times(float t, float inc, int k, float& out) {
    const uint32_t tb = f2u(t), ib = f2u(inc);
    const int e = int(tb >> 23), ei = int(ib >> 23);   // a set sign bit makes these >= 256
    if (e <= 0 || e >= 255 || ei <= 0 || ei > e) return false;
    const int sh = e - ei;
    if (sh > 24) return false;
    const int32_t m = int32_t((tb & 0x7fffffu) | 0x800000u);
    const int32_t mi = int32_t((ib & 0x7fffffu) | 0x800000u);
    int32_t D = mi >> sh;                                  // ulps of t's binade per addition
    if (sh > 0) {
        const int32_t r = mi & ((int32_t(1) << sh) - 1), half = int32_t(1) << (sh - 1);
        if (r == half) return false;                       // tie: round-to-even alternates
        if (r > half) ++D;
    }
    if (k < 0 || k > 127) return false;                    // k * D stays below 2^31
    const int32_t m1 = m + k * D;
    if (m1 > 0xffffff) return false;
    out = u2f((uint32_t(e) << 23) | (uint32_t(m1) & 0x7fffffu));
    return true;
}

// Repeats { prev = t; t = fl(t + inc); } at least once and until t >= limit or max_steps
// additions were made; returns the number of additions.  Equal, bit for bit, to the plain
// loop for any t, inc, limit (the closed form is used only for positive normal t, inc and
// limit; everything else takes the plain additions).
KF_HD int advance_steps(float& t, float& prev, float inc, float limit, int max_steps) {
    int k = 0;
    while (k < max_steps) {
        prev = t;
        t = t + inc;
        ++k;
        if (!(t < limit) || k >= max_steps) break;
        const uint32_t tb = f2u(t), ib = f2u(inc), lb = f2u(limit);
        const int e = int(tb >> 23), ei = int(ib >> 23), el = int(lb >> 23);   // sign bits must be 0
        if (e <= 0 || e >= 255 || ei <= 0 || ei > e || el >= 255 || el < e) continue;
        const int sh = e - ei;
        if (sh > 24) continue;
        const int32_t m = int32_t((tb & 0x7fffffu) | 0x800000u);   // t = m ulps of t's binade
        const int32_t mi = int32_t((ib & 0x7fffffu) | 0x800000u);
        int32_t q = mi >> sh, D = q;                                 // inc = q + r / 2^sh ulps
        if (sh > 0) {
            const int32_t r = mi & ((int32_t(1) << sh) - 1), half = int32_t(1) << (sh - 1);
            if (r == half) continue;                                 // tie: round-to-even alternates
            if (r > half) ++D;
        }
        if (D <= 0) continue;
        const int32_t room = (int32_t(0xffffff) - m) / D;           // additions staying in the binade
        int32_t j = room;
        if (el == e) {                                               // limit in the same binade
            const int32_t lm = int32_t((lb & 0x7fffffu) | 0x800000u);
            const int32_t need = (lm - m + D - 1) / D;               // first j with m + j D >= lm
            if (need < j) j = need;
        }
        if (j > max_steps - k) j = max_steps - k;
        if (j <= 0) continue;
        const int32_t m1 = m + j * D;
        prev = u2f((uint32_t(e) << 23) | (uint32_t(m1 - D) & 0x7fffffu));
        t = u2f((uint32_t(e) << 23) | (uint32_t(m1) & 0x7fffffu));
        k += j;
        if (!(t < limit)) break;
    }
    return k;
}

}  // namespace kf
