// k_display.cu -- headless versions of the reference's window-content kernels
// (project/src/display.cu:9-105).  The reference writes 32-bit pixels into the OpenGL
// window's CUDA surface; here they go to an RGBA8 image in device memory (row-major, 4 bytes
// per pixel: r, g, b, 255), which a caller can copy out or write to a file.
#include "kf_host.h"

namespace kf {

// static_cast<unsigned char>(x) of the reference's kernels: truncation toward zero, clamped to
// [0, 255] (the device's float-to-unsigned conversion saturates), NaN -> 0
__device__ __forceinline__ unsigned int to_u8(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 255.0f) return 255u;
    return unsigned(x);
}

// the reference packs (255 << 24) | (b << 16) | (g << 8) | r: bytes r, g, b, 255 in memory
__device__ __forceinline__ unsigned int pack_rgba(float r, float g, float b) {
    return (255u << 24) | (to_u8(b) << 16) | (to_u8(g) << 8) | to_u8(r);
}

// normalMapToWindowContentKernel (project/src/display.cu:63-81): the normal rotated by the
// inverse sensor rotation, normalised, components * 255 as r, g, b
__global__ void normals_rgba_kernel(const float4* __restrict__ nm, int w, int h, DispMats m, unsigned int* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= w || j >= h) return;
    const float4 n4 = nm[size_t(j) * w + i];
    F3 n = mv3(m.r, F3{n4.x, n4.y, n4.z});
    n = n * rsqrtf(dot3(n, n));
    out[size_t(j) * w + i] = pack_rgba(n.x * 255.0f, n.y * 255.0f, n.z * 255.0f);
}

// shadingToWindowContentKernel (project/src/display.cu:83-105): |normal . ray direction|,
// clamped to 1, as grey; the ray through the pixel centre is R K^-1 (i + .5, j + .5, 1)
__global__ void shading_rgba_kernel(const float4* __restrict__ nm, int w, int h, DispMats m, unsigned int* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= w || j >= h) return;
    const float4 n4 = nm[size_t(j) * w + i];
    F3 d = mv3(m.r, mv3(m.ik, F3{float(i) + 0.5f, float(j) + 0.5f, 1.0f}));
    d = d * rsqrtf(dot3(d, d));
    const float rad = fminf(fabsf(n4.x * d.x + n4.y * d.y + n4.z * d.z), 1.0f);
    out[size_t(j) * w + i] = pack_rgba(rad * 255.0f, rad * 255.0f, rad * 255.0f);
}

// oneFloatChannelToWindowContentKernel (project/src/display.cu:27-42): value * scale as grey
__global__ void float_rgba_kernel(const float* __restrict__ src, int w, int h, float scale, unsigned int* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= w || j >= h) return;
    const float v = src[size_t(j) * w + i] * scale;
    out[size_t(j) * w + i] = pack_rgba(v, v, v);
}

cudaError_t stage_display(int mode, const void* src, int w, int h, const DispMats& m, float scale, unsigned int* out,
                          cudaStream_t st) {
    const dim3 blk(32, 8), grd((w + 31) / 32, (h + 7) / 8);
    if (mode == kDisplayNormals)
        normals_rgba_kernel<<<grd, blk, 0, st>>>(static_cast<const float4*>(src), w, h, m, out);
    else if (mode == kDisplayShading)
        shading_rgba_kernel<<<grd, blk, 0, st>>>(static_cast<const float4*>(src), w, h, m, out);
    else
        float_rgba_kernel<<<grd, blk, 0, st>>>(static_cast<const float*>(src), w, h, scale, out);
    return cudaGetLastError();
}

}  // namespace kf
