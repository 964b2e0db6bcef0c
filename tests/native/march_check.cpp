// Host check of kf::advance_steps and kf::add_k_times (kinectfusion-cuda_b200/csrc/kf_march.h)
// against the plain repeated float additions.  Built and run by tests/test_march_fastforward.py.
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "kf_march.h"

static uint64_t rng_state = 0x9e3779b97f4a7c15ull;
static uint64_t next_u64() {
    uint64_t z = (rng_state += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
static float uni(float a, float b) { return a + (b - a) * float(double(next_u64() >> 11) / 9007199254740992.0); }

static int plain(float& t, float& prev, float inc, float limit, int max_steps) {
    int k = 0;
    do {
        prev = t;
        t = t + inc;
        ++k;
    } while (t < limit && k < max_steps);
    return k;
}

int main(int argc, char** argv) {
    const int cases = argc > 1 ? atoi(argv[1]) : 200000;
    long long bad = 0, steps = 0;
    const float incs[] = {0.0398f, 0.002f, 0.02f * 1.99f, 0.03f * 0.1f, 0.003f, 0.06f};
    for (int c = 0; c < cases; ++c) {
        float t0, inc, limit;
        const int kind = int(next_u64() % 4);
        if (kind == 0) {           // the raycaster's range
            t0 = uni(0.4f, 6.0f);
            inc = incs[next_u64() % 6];
            limit = t0 + uni(0.0f, 2.0f);
        } else if (kind == 1) {    // across binade boundaries
            const float b = float(1 << int(next_u64() % 4));
            t0 = b - uni(0.0f, 0.3f);
            inc = incs[next_u64() % 6];
            limit = b + uni(0.0f, 1.0f);
        } else if (kind == 2) {    // random increments
            t0 = uni(0.1f, 8.0f);
            const uint32_t ib = (uint32_t(117 + next_u64() % 10) << 23) | uint32_t(next_u64() & 0x7fffffu);
            memcpy(&inc, &ib, 4);
            limit = t0 + uni(0.0f, 3.0f);
        } else {                   // increments exactly halfway between ulp multiples of t
            t0 = uni(1.0f, 2.0f);
            const uint32_t ib = (uint32_t(127 - 6) << 23) | (uint32_t(next_u64() & 0x7fffc0u) | 0x20u);
            memcpy(&inc, &ib, 4);
            limit = t0 + uni(0.0f, 1.5f);
        }
        const int max_steps = (next_u64() % 8 == 0) ? int(1 + next_u64() % 50) : 1 << 16;
        float ta = t0, pa = 0.f, tb = t0, pb = 0.f;
        const int ka = plain(ta, pa, inc, limit, max_steps);
        const int kb = kf::advance_steps(tb, pb, inc, limit, max_steps);
        steps += ka;
        if (ka != kb || memcmp(&ta, &tb, 4) || memcmp(&pa, &pb, 4)) {
            if (bad < 5)
                printf("mismatch t0=%.9g inc=%.9g limit=%.9g max=%d: plain k=%d t=%.9g prev=%.9g, fast k=%d t=%.9g prev=%.9g\n",
                       t0, inc, limit, max_steps, ka, ta, pa, kb, tb, pb);
            ++bad;
        }
    }
    // add_k_times: lane k of a cooperative march forms t + k increments in closed form
    long long kbad = 0, kused = 0;
    for (int c = 0; c < cases; ++c) {
        const float t0 = (c & 1) ? uni(0.4f, 6.0f) : float(1 << int(next_u64() % 3)) - uni(0.0f, 0.05f);
        float inc = incs[next_u64() % 6];
        if (c % 5 == 0) {   // random increments, ties included
            const uint32_t ib = (uint32_t(117 + next_u64() % 10) << 23) | uint32_t(next_u64() & 0x7fffffu);
            memcpy(&inc, &ib, 4);
        }
        const int k = int(next_u64() % 32);
        float seq = t0;
        for (int q = 0; q < k; ++q) seq = seq + inc;
        float fast = 0.f;
        if (kf::add_k_times(t0, inc, k, fast)) {
            ++kused;
            if (memcmp(&seq, &fast, 4)) {
                if (kbad < 5) printf("add_k_times mismatch t0=%.9g inc=%.9g k=%d: %.9g vs %.9g\n", t0, inc, k, seq, fast);
                ++kbad;
            }
        }
    }
    printf("cases %d steps %lld mismatches %lld; add_k_times closed form %lld of %d, mismatches %lld\n", cases,
           steps, bad, kused, cases, kbad);
    return (bad || kbad || kused < cases / 4) ? 1 : 0;
}
