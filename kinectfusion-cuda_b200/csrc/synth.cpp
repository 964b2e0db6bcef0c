// synth.cpp -- seeded synthetic depth sequences (libkfsynth.so, host only).
//
// Stand-in for the TUM RGB-D sequences the reference reads from disk
// (project/src/rgbd_dataset.cpp:6-77, project/src/main.cpp:18): those files are not available,
// so frames are ray-cast from an analytic scene.  World = the TSDF cube centred at the origin;
// the camera starts at (0, 0, -cube_width) looking along +z with y pointing down, so the scene
// lies inside the cube.  The scene is a ground plane, a 0.4 m sphere and a 0.5 m axis-aligned
// box, 1-3 m from the camera.  Depth is z-depth (project/src/measurement.cu:114-116 turns it
// back into vertices with K^-1 (u + 0.5, v + 0.5, 1)).  Noise: N(0, (0.0012 z^2)^2) metres,
// 3% of pixels dropped to 0, depths beyond 4 m dropped, rounded to uint16 millimetres.
// Randomness is a SplitMix64 counter hash of (seed, frame, pixel) so every pixel is
// reproducible on its own, whatever the thread count.

#include <cmath>
#include <cstdint>
#include <cstring>

namespace {

inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline double unit(uint64_t r) { return double(r >> 11) * (1.0 / 9007199254740992.0); }

struct Vec { double x, y, z; };
inline Vec operator+(Vec a, Vec b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec operator-(Vec a, Vec b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec operator*(Vec a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dotv(Vec a, Vec b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Vec crossv(Vec a, Vec b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline Vec normv(Vec a) { double l = std::sqrt(dotv(a, a)); return a * (1.0 / l); }

// column-major 4x4 camera->world from rotation columns and position
void make_pose(Vec cx, Vec cy, Vec cz, Vec pos, float* p) {
    std::memset(p, 0, 16 * sizeof(float));
    p[0] = float(cx.x); p[1] = float(cx.y); p[2] = float(cx.z);
    p[4] = float(cy.x); p[5] = float(cy.y); p[6] = float(cy.z);
    p[8] = float(cz.x); p[9] = float(cz.y); p[10] = float(cz.z);
    p[12] = float(pos.x); p[13] = float(pos.y); p[14] = float(pos.z); p[15] = 1.0f;
}

// rotation matrix (columns) of axis-angle vector r (Rodrigues)
void rodrigues(Vec r, Vec& c0, Vec& c1, Vec& c2) {
    const double th = std::sqrt(dotv(r, r));
    if (th < 1e-15) { c0 = {1, 0, 0}; c1 = {0, 1, 0}; c2 = {0, 0, 1}; return; }
    const Vec k = r * (1.0 / th);
    const double c = std::cos(th), s = std::sin(th), v = 1.0 - c;
    // R = c I + s [k]x + v k k^T ; columns
    c0 = {c + k.x * k.x * v, k.y * k.x * v + k.z * s, k.z * k.x * v - k.y * s};
    c1 = {k.x * k.y * v - k.z * s, c + k.y * k.y * v, k.z * k.y * v + k.x * s};
    c2 = {k.x * k.z * v + k.y * s, k.y * k.z * v - k.x * s, c + k.z * k.z * v};
}

}  // namespace

extern "C" {

typedef struct kfs_scene {
    float cube_width;
    float plane_y;        // ground plane y = plane_y (camera y axis points down)
    float sphere_c[3];
    float sphere_r;
    float box_lo[3], box_hi[3];
} kfs_scene;

// The analytic scene for a cube of the given width (camera start at (0, 0, -cube_width)).
int kfs_scene_make(float cube_width, kfs_scene* s) {
    if (!s || !(cube_width > 1.2f)) return 1;
    const float cz = -cube_width;
    s->cube_width = cube_width;
    s->plane_y = 0.45f;
    s->sphere_r = 0.2f;                       // 0.4 m diameter
    s->sphere_c[0] = -0.35f; s->sphere_c[1] = s->plane_y - s->sphere_r; s->sphere_c[2] = cz + 1.9f;
    const float bc[3] = {0.35f, s->plane_y - 0.25f, cz + 2.4f};   // 0.5 m box resting on the plane
    for (int a = 0; a < 3; ++a) { s->box_lo[a] = bc[a] - 0.25f; s->box_hi[a] = bc[a] + 0.25f; }
    return 0;
}

// Camera trajectories (poses column-major camera->world, frames x 16 floats).
//  kind 0: smooth seeded wobble around the start pose; per frame |dt| <= 2 cm and
//          rotation <= 1 degree about a seeded axis.
//  kind 1: seeded closed loop around the objects: the camera swings on an arc about a point
//          between the sphere and the box while looking at it (about 0.4 deg and 1.6 cm per
//          frame for 300 frames).
int kfs_trajectory(int kind, int frames, uint64_t seed, float cube_width, float* poses) {
    if (!poses || frames <= 0) return 1;
    const double pi = 3.14159265358979323846;
    const Vec start{0.0, 0.0, -double(cube_width)};
    uint64_t key = mix64(seed ^ 0x5eedull);
    auto rnd = [&key]() { key = mix64(key); return unit(key); };
    if (kind == 0) {
        double amp[3], per[3], ph[3];
        for (int a = 0; a < 3; ++a) {
            amp[a] = 0.06;                          // metres
            per[a] = 45.0 + 25.0 * rnd();           // frames
            ph[a] = 2.0 * pi * rnd();
        }
        Vec axis = normv(Vec{rnd() - 0.5, rnd() - 0.5, rnd() - 0.5});
        const double rot_amp = 4.0 * pi / 180.0, rot_per = 40.0 + 20.0 * rnd(), rot_ph = 2.0 * pi * rnd();
        for (int f = 0; f < frames; ++f) {
            Vec t{0, 0, 0};
            double* tc[3] = {&t.x, &t.y, &t.z};
            for (int a = 0; a < 3; ++a)
                *tc[a] = amp[a] * (std::sin(2.0 * pi * f / per[a] + ph[a]) - std::sin(ph[a]));
            const double th = rot_amp * (std::sin(2.0 * pi * f / rot_per + rot_ph) - std::sin(rot_ph));
            Vec c0, c1, c2;
            rodrigues(axis * th, c0, c1, c2);
            make_pose(c0, c1, c2, start + t, poses + 16 * size_t(f));
        }
        return 0;
    }
    if (kind == 1) {
        const Vec target{0.0, 0.0, -double(cube_width) + 2.15};
        const double radius = 2.15;
        const double arc = (18.0 + 6.0 * rnd()) * pi / 180.0;
        const double bob = 0.04 + 0.03 * rnd();
        const double period = double(frames);
        for (int f = 0; f < frames; ++f) {
            const double phi = arc * std::sin(2.0 * pi * f / period);
            const double dy = -bob * std::sin(4.0 * pi * f / period);
            const Vec pos{target.x - radius * std::sin(phi), target.y + dy, target.z - radius * std::cos(phi)};
            const Vec cz = normv(target - pos);
            const Vec down{0.0, 1.0, 0.0};
            const Vec cx = normv(crossv(down, cz));
            const Vec cy = crossv(cz, cx);
            make_pose(cx, cy, cz, pos, poses + 16 * size_t(f));
        }
        return 0;
    }
    return 2;
}

// Ray-cast one frame.  out: w*h uint16 millimetre depths (0 = no measurement).
// depth_true (may be NULL): noise-free z-depth in metres, 0 where the ray hits nothing.
// noise = 0 gives exact depths (still rounded to millimetres, no dropouts).
int kfs_render(const kfs_scene* s, const float pose[16], int w, int h, float fx, float fy, float cx, float cy,
               uint64_t seed, int frame, int noise, uint16_t* out, float* depth_true) {
    if (!s || !pose || !out || w <= 0 || h <= 0) return 1;
    const Vec c0{pose[0], pose[1], pose[2]}, c1{pose[4], pose[5], pose[6]}, c2{pose[8], pose[9], pose[10]};
    const Vec o{pose[12], pose[13], pose[14]};
    const uint64_t fkey = mix64(mix64(seed) ^ mix64(uint64_t(frame) + 0x9e37ull));
#pragma omp parallel for schedule(static)
    for (int j = 0; j < h; ++j) {
        for (int i = 0; i < w; ++i) {
            const Vec dc{(i + 0.5 - cx) / fx, (j + 0.5 - cy) / fy, 1.0};
            const Vec d = c0 * dc.x + c1 * dc.y + c2 * dc.z;   // world direction, camera z = 1
            double best = 1e30;
            // ground plane
            if (std::fabs(d.y) > 1e-12) {
                const double t = (s->plane_y - o.y) / d.y;
                if (t > 1e-6 && t < best) best = t;
            }
            // sphere
            {
                const Vec oc = o - Vec{s->sphere_c[0], s->sphere_c[1], s->sphere_c[2]};
                const double a = dotv(d, d), b = 2.0 * dotv(d, oc), c = dotv(oc, oc) - double(s->sphere_r) * s->sphere_r;
                const double disc = b * b - 4 * a * c;
                if (disc >= 0.0) {
                    const double sq = std::sqrt(disc);
                    double t = (-b - sq) / (2 * a);
                    if (t <= 1e-6) t = (-b + sq) / (2 * a);
                    if (t > 1e-6 && t < best) best = t;
                }
            }
            // box (slabs)
            {
                double tn = -1e30, tf = 1e30;
                const double oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
                bool hit = true;
                for (int a = 0; a < 3; ++a) {
                    if (std::fabs(dd[a]) < 1e-15) {
                        if (oo[a] < s->box_lo[a] || oo[a] > s->box_hi[a]) { hit = false; break; }
                        continue;
                    }
                    double t0 = (s->box_lo[a] - oo[a]) / dd[a], t1 = (s->box_hi[a] - oo[a]) / dd[a];
                    if (t0 > t1) { double tt = t0; t0 = t1; t1 = tt; }
                    if (t0 > tn) tn = t0;
                    if (t1 < tf) tf = t1;
                }
                if (hit && tn <= tf && tf > 1e-6) {
                    const double t = tn > 1e-6 ? tn : tf;
                    if (t < best) best = t;
                }
            }
            const size_t idx = size_t(j) * w + i;
            double z = best < 1e29 ? best : 0.0;   // z-depth because camera-frame d.z = 1
            if (depth_true) depth_true[idx] = float(z);
            if (z > 0.0 && noise) {
                const uint64_t base = fkey ^ (uint64_t(idx) * 0xD1B54A32D192ED03ull);
                const double u1 = unit(mix64(base + 1)), u2 = unit(mix64(base + 2)), u3 = unit(mix64(base + 3));
                const double g = std::sqrt(-2.0 * std::log(u1 > 1e-300 ? u1 : 1e-300)) * std::cos(2.0 * 3.14159265358979323846 * u2);
                z += g * 0.0012 * z * z;
                if (u3 < 0.03) z = 0.0;
            }
            if (z > 4.0) z = 0.0;
            long mm = z > 0.0 ? std::lround(z * 1000.0) : 0;
            if (mm < 0) mm = 0;
            if (mm > 65535) mm = 65535;
            out[idx] = uint16_t(mm);
        }
    }
    return 0;
}

}  // extern "C"
