// dataset.cpp -- TUM RGB-D sequence reader (the reference's RgbdDataset,
// project/src/rgbd_dataset.cpp:6-96, and DepthMap::update(path), project/src/depth_map.cpp:17-28)
// with its own 16-bit greyscale PNG decoder (the reference uses stb_image, which is absent).
//
// A sequence directory holds groundtruth.txt ("timestamp tx ty tz qx qy qz qw" after three
// comment lines), depth.txt ("timestamp relative/path.png" after three comment lines) and the
// 16-bit depth PNGs.  Each depth image is paired with the ground-truth pose whose timestamp
// is nearest, searched forward from the previous match as the reference does.
#include <zlib.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "kf_api.h"

struct kf_tum {
    std::vector<std::string> paths;
    std::vector<std::vector<float>> poses;   // column-major 4x4 camera -> world
};

namespace {

// glm::mat4_cast(quat) with the translation in column 3 (project/src/rgbd_dataset.cpp:68-70)
void pose_from(float tx, float ty, float tz, float qx, float qy, float qz, float qw, float* m) {
    const float xx = qx * qx, yy = qy * qy, zz = qz * qz;
    const float xy = qx * qy, xz = qx * qz, yz = qy * qz;
    const float wx = qw * qx, wy = qw * qy, wz = qw * qz;
    m[0] = 1.f - 2.f * (yy + zz); m[1] = 2.f * (xy + wz);       m[2] = 2.f * (xz - wy);       m[3] = 0.f;
    m[4] = 2.f * (xy - wz);       m[5] = 1.f - 2.f * (xx + zz); m[6] = 2.f * (yz + wx);       m[7] = 0.f;
    m[8] = 2.f * (xz + wy);       m[9] = 2.f * (yz - wx);       m[10] = 1.f - 2.f * (xx + yy); m[11] = 0.f;
    m[12] = tx; m[13] = ty; m[14] = tz; m[15] = 1.f;
}

uint32_t be32(const unsigned char* p) { return (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | p[3]; }

int paeth(int a, int b, int c) {
    const int p = a + b - c, pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
    if (pa <= pb && pa <= pc) return a;
    return pb <= pc ? b : c;
}

// 16-bit greyscale, non-interlaced PNG -> host-order uint16 (PNG stores big-endian samples)
kf_status read_png16(const std::string& path, std::vector<uint16_t>& out, int& w, int& h) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return KF_ERR_ARG;
    std::vector<unsigned char> buf((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    static const unsigned char sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (buf.size() < 8 || std::memcmp(buf.data(), sig, 8) != 0) return KF_ERR_ARG;
    size_t pos = 8;
    std::vector<unsigned char> idat;
    w = h = 0;
    while (pos + 12 <= buf.size()) {
        const uint32_t len = be32(&buf[pos]);
        if (pos + 12 + size_t(len) > buf.size()) return KF_ERR_ARG;
        const unsigned char* type = &buf[pos + 4];
        const unsigned char* data = &buf[pos + 8];
        if (!std::memcmp(type, "IHDR", 4)) {
            if (len < 13) return KF_ERR_ARG;
            w = int(be32(data));
            h = int(be32(data + 4));
            // bit depth 16, colour type 0 (greyscale), deflate, adaptive filters, no interlace
            if (data[8] != 16 || data[9] != 0 || data[10] != 0 || data[11] != 0 || data[12] != 0) return KF_ERR_SHAPE;
        } else if (!std::memcmp(type, "IDAT", 4)) {
            idat.insert(idat.end(), data, data + len);
        } else if (!std::memcmp(type, "IEND", 4)) {
            break;
        }
        pos += 12 + size_t(len);
    }
    if (w <= 0 || h <= 0 || w > 16384 || h > 16384) return KF_ERR_SHAPE;
    const size_t stride = size_t(w) * 2;
    std::vector<unsigned char> raw((stride + 1) * size_t(h));
    uLongf raw_len = uLongf(raw.size());
    if (uncompress(raw.data(), &raw_len, idat.data(), uLong(idat.size())) != Z_OK || raw_len != raw.size())
        return KF_ERR_ARG;
    // undo the per-row filters (bytes per pixel: 2)
    std::vector<unsigned char> prev(stride, 0), cur(stride);
    out.resize(size_t(w) * h);
    for (int y = 0; y < h; ++y) {
        const unsigned char* row = &raw[size_t(y) * (stride + 1)];
        const int filter = row[0];
        for (size_t x = 0; x < stride; ++x) {
            const int a = x >= 2 ? cur[x - 2] : 0, b = prev[x], c = x >= 2 ? prev[x - 2] : 0;
            int v = row[1 + x];
            switch (filter) {
                case 0: break;
                case 1: v += a; break;
                case 2: v += b; break;
                case 3: v += (a + b) / 2; break;
                case 4: v += paeth(a, b, c); break;
                default: return KF_ERR_ARG;
            }
            cur[x] = (unsigned char)(v & 0xff);
        }
        for (int x = 0; x < w; ++x) out[size_t(y) * w + x] = uint16_t((cur[2 * x] << 8) | cur[2 * x + 1]);
        std::swap(prev, cur);
    }
    return KF_OK;
}

void skip_lines(std::ifstream& f, int n) {
    std::string t;
    for (int i = 0; i < n; ++i) std::getline(f, t);
}

}  // namespace

extern "C" {

kf_status kf_tum_open(const char* dir, kf_tum** out) {
    if (!dir || !out) return KF_ERR_ARG;
    const std::string root(dir);
    std::ifstream gt(root + "/groundtruth.txt"), dl(root + "/depth.txt");
    if (!gt || !dl) return KF_ERR_ARG;
    skip_lines(gt, 3);
    std::vector<double> ts;
    std::vector<float> tr, qu;
    double t;
    while (gt >> t) {
        float v[7];
        for (float& x : v) gt >> x;
        if (!gt) return KF_ERR_ARG;
        ts.push_back(t);
        tr.insert(tr.end(), v, v + 3);
        qu.insert(qu.end(), v + 3, v + 7);
    }
    if (ts.empty()) return KF_ERR_ARG;
    kf_tum* d = new (std::nothrow) kf_tum;
    if (!d) return KF_ERR_ARG;
    skip_lines(dl, 3);
    int last = 0;
    const int n = int(ts.size());
    while (dl >> t) {
        // nearest ground-truth timestamp, searched forward from the last match
        double best = std::numeric_limits<double>::max();
        int best_i = -1;
        for (int i = last; i < n; ++i) {
            const double diff = std::fabs(t - ts[i]);
            if (diff < best) {
                best = diff;
                best_i = i;
            } else {
                last = best_i;
                break;
            }
        }
        std::string rel;
        dl >> rel;
        if (best_i < 0) best_i = n - 1;
        std::vector<float> m(16);
        pose_from(tr[3 * best_i], tr[3 * best_i + 1], tr[3 * best_i + 2], qu[4 * best_i], qu[4 * best_i + 1],
                  qu[4 * best_i + 2], qu[4 * best_i + 3], m.data());
        d->paths.push_back(root + "/" + rel);
        d->poses.push_back(m);
    }
    if (d->paths.empty()) { delete d; return KF_ERR_ARG; }
    *out = d;
    return KF_OK;
}

kf_status kf_tum_close(kf_tum* d) {
    if (!d) return KF_ERR_ARG;
    delete d;
    return KF_OK;
}

kf_status kf_tum_count(const kf_tum* d, int* count) {
    if (!d || !count) return KF_ERR_ARG;
    *count = int(d->paths.size());
    return KF_OK;
}

kf_status kf_tum_frame(const kf_tum* d, int index, uint16_t* depth, int w, int h, float pose[16]) {
    if (!d || index < 0 || index >= int(d->paths.size())) return KF_ERR_ARG;
    if (pose) std::memcpy(pose, d->poses[index].data(), sizeof(float) * 16);
    if (!depth) return KF_OK;
    std::vector<uint16_t> img;
    int iw = 0, ih = 0;
    const kf_status st = read_png16(d->paths[index], img, iw, ih);
    if (st != KF_OK) return st;
    if (iw != w || ih != h) return KF_ERR_SHAPE;
    std::memcpy(depth, img.data(), sizeof(uint16_t) * img.size());
    return KF_OK;
}

kf_status kf_tum_initial_pose_inverse(const kf_tum* d, float out[16]) {
    if (!d || !out || d->poses.empty()) return KF_ERR_ARG;
    // glm::inverse of the first pose (a general 4x4 inverse: the text file's quaternions are
    // not exactly of unit length), by cofactors in double
    const float* m = d->poses[0].data();
    double a[16], inv[16];
    for (int i = 0; i < 16; ++i) a[i] = m[i];
    inv[0] = a[5] * a[10] * a[15] - a[5] * a[11] * a[14] - a[9] * a[6] * a[15] + a[9] * a[7] * a[14] + a[13] * a[6] * a[11] - a[13] * a[7] * a[10];
    inv[4] = -a[4] * a[10] * a[15] + a[4] * a[11] * a[14] + a[8] * a[6] * a[15] - a[8] * a[7] * a[14] - a[12] * a[6] * a[11] + a[12] * a[7] * a[10];
    inv[8] = a[4] * a[9] * a[15] - a[4] * a[11] * a[13] - a[8] * a[5] * a[15] + a[8] * a[7] * a[13] + a[12] * a[5] * a[11] - a[12] * a[7] * a[9];
    inv[12] = -a[4] * a[9] * a[14] + a[4] * a[10] * a[13] + a[8] * a[5] * a[14] - a[8] * a[6] * a[13] - a[12] * a[5] * a[10] + a[12] * a[6] * a[9];
    inv[1] = -a[1] * a[10] * a[15] + a[1] * a[11] * a[14] + a[9] * a[2] * a[15] - a[9] * a[3] * a[14] - a[13] * a[2] * a[11] + a[13] * a[3] * a[10];
    inv[5] = a[0] * a[10] * a[15] - a[0] * a[11] * a[14] - a[8] * a[2] * a[15] + a[8] * a[3] * a[14] + a[12] * a[2] * a[11] - a[12] * a[3] * a[10];
    inv[9] = -a[0] * a[9] * a[15] + a[0] * a[11] * a[13] + a[8] * a[1] * a[15] - a[8] * a[3] * a[13] - a[12] * a[1] * a[11] + a[12] * a[3] * a[9];
    inv[13] = a[0] * a[9] * a[14] - a[0] * a[10] * a[13] - a[8] * a[1] * a[14] + a[8] * a[2] * a[13] + a[12] * a[1] * a[10] - a[12] * a[2] * a[9];
    inv[2] = a[1] * a[6] * a[15] - a[1] * a[7] * a[14] - a[5] * a[2] * a[15] + a[5] * a[3] * a[14] + a[13] * a[2] * a[7] - a[13] * a[3] * a[6];
    inv[6] = -a[0] * a[6] * a[15] + a[0] * a[7] * a[14] + a[4] * a[2] * a[15] - a[4] * a[3] * a[14] - a[12] * a[2] * a[7] + a[12] * a[3] * a[6];
    inv[10] = a[0] * a[5] * a[15] - a[0] * a[7] * a[13] - a[4] * a[1] * a[15] + a[4] * a[3] * a[13] + a[12] * a[1] * a[7] - a[12] * a[3] * a[5];
    inv[14] = -a[0] * a[5] * a[14] + a[0] * a[6] * a[13] + a[4] * a[1] * a[14] - a[4] * a[2] * a[13] - a[12] * a[1] * a[6] + a[12] * a[2] * a[5];
    inv[3] = -a[1] * a[6] * a[11] + a[1] * a[7] * a[10] + a[5] * a[2] * a[11] - a[5] * a[3] * a[10] - a[9] * a[2] * a[7] + a[9] * a[3] * a[6];
    inv[7] = a[0] * a[6] * a[11] - a[0] * a[7] * a[10] - a[4] * a[2] * a[11] + a[4] * a[3] * a[10] + a[8] * a[2] * a[7] - a[8] * a[3] * a[6];
    inv[11] = -a[0] * a[5] * a[11] + a[0] * a[7] * a[9] + a[4] * a[1] * a[11] - a[4] * a[3] * a[9] - a[8] * a[1] * a[7] + a[8] * a[3] * a[5];
    inv[15] = a[0] * a[5] * a[10] - a[0] * a[6] * a[9] - a[4] * a[1] * a[10] + a[4] * a[2] * a[9] + a[8] * a[1] * a[6] - a[8] * a[2] * a[5];
    const double det = a[0] * inv[0] + a[1] * inv[4] + a[2] * inv[8] + a[3] * inv[12];
    if (!(std::fabs(det) > 0.0)) return KF_ERR_NONFINITE;
    for (int i = 0; i < 16; ++i) out[i] = float(inv[i] / det);
    return KF_OK;
}

kf_status kf_png16_read(const char* path, uint16_t* dst, int w, int h) {
    if (!path || !dst) return KF_ERR_ARG;
    std::vector<uint16_t> img;
    int iw = 0, ih = 0;
    const kf_status st = read_png16(path, img, iw, ih);
    if (st != KF_OK) return st;
    if (iw != w || ih != h) return KF_ERR_SHAPE;
    std::memcpy(dst, img.data(), sizeof(uint16_t) * img.size());
    return KF_OK;
}

}  // extern "C"
