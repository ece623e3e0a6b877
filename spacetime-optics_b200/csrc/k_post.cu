// Post-processing of the traced HDR frame, the reference's pyramid filters (render.cu:244-316,
// 732-753): a 2x2 box-filter pyramid of the frame, the visible-mode camera glare (bloom: an
// energy-conserving mix of the frame with its ever wider pyramid levels, weights 1/k) and the
// radio-mode interferometer beam (Gaussian blur of sigma pixels: down the pyramid while sigma / 2^k
// stays above 3 pixels, separable Gaussian of radius ceil(3 sigma) there, bilinear back up).
// Same filters and level sizes as the reference, so that a frame looks the same after them.  Each
// kernel is one pass over a level (HBM- / L2-bound, a few microseconds at 2048^2).
#include <cuda_runtime.h>

#include "so_launch.h"

namespace so {

namespace {

__global__ void k_down(const float4* __restrict__ src, int sw, int sh, float4* __restrict__ dst, int dw, int dh) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= dw || y >= dh) return;
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const float4 v = src[(long)min(2 * y + j, sh - 1) * sw + min(2 * x + i, sw - 1)];
            a.x += v.x;
            a.y += v.y;
            a.z += v.z;
            a.w += v.w;
        }
    dst[(long)y * dw + x] = make_float4(0.25f * a.x, 0.25f * a.y, 0.25f * a.z, 0.25f * a.w);
}

// Bilinear sample of a level at continuous pixel coordinates (pixel centres at +0.5), clamped.
__device__ __forceinline__ float4 bilinear(const float4* L, int w, int h, float x, float y) {
    x = fminf(fmaxf(x - 0.5f, 0.f), w - 1.001f);
    y = fminf(fmaxf(y - 0.5f, 0.f), h - 1.001f);
    const int ix = (int)x, iy = (int)y;
    const float fx = x - ix, fy = y - iy;
    const int ix1 = min(ix + 1, w - 1), iy1 = min(iy + 1, h - 1);
    const float4 a = L[(long)iy * w + ix], b = L[(long)iy * w + ix1], c = L[(long)iy1 * w + ix], d = L[(long)iy1 * w + ix1];
    float4 o;
    o.x = (1 - fy) * ((1 - fx) * a.x + fx * b.x) + fy * ((1 - fx) * c.x + fx * d.x);
    o.y = (1 - fy) * ((1 - fx) * a.y + fx * b.y) + fy * ((1 - fx) * c.y + fx * d.y);
    o.z = (1 - fy) * ((1 - fx) * a.z + fx * b.z) + fy * ((1 - fx) * c.z + fx * d.z);
    o.w = (1 - fy) * ((1 - fx) * a.w + fx * b.w) + fy * ((1 - fx) * c.w + fx * d.w);
    return o;
}

__global__ void k_bloom(float4* __restrict__ img, int W, int H, PostLevels L, float strength) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    float bx = 0.f, by = 0.f, bz = 0.f, ws = 0.f;
    for (int k = 1; k < L.n; ++k) {
        const float4 v = bilinear(L.p[k], L.w[k], L.h[k], (x + 0.5f) * L.w[k] / W, (y + 0.5f) * L.h[k] / H);
        const float w = 1.f / (float)k;
        bx += w * v.x;
        by += w * v.y;
        bz += w * v.z;
        ws += w;
    }
    const float4 o = img[(long)y * W + x];
    const float s = strength;
    img[(long)y * W + x] =
        make_float4((1 - s) * o.x + s * bx / ws, (1 - s) * o.y + s * by / ws, (1 - s) * o.z + s * bz / ws, o.w);
}

__global__ void k_gauss(const float4* __restrict__ src, float4* __restrict__ dst, int w, int h, float sigma, int horiz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int R = (int)ceilf(3.f * sigma);
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
    float ws = 0.f;
    for (int i = -R; i <= R; ++i) {
        const int xx = horiz ? min(max(x + i, 0), w - 1) : x, yy = horiz ? y : min(max(y + i, 0), h - 1);
        const float wgt = expf(-0.5f * i * i / (sigma * sigma));
        const float4 v = src[(long)yy * w + xx];
        a.x += wgt * v.x;
        a.y += wgt * v.y;
        a.z += wgt * v.z;
        a.w += wgt * v.w;
        ws += wgt;
    }
    dst[(long)y * w + x] = make_float4(a.x / ws, a.y / ws, a.z / ws, a.w / ws);
}

__global__ void k_upsample(const float4* __restrict__ L, int lw, int lh, float4* __restrict__ img, int W, int H) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    img[(long)y * W + x] = bilinear(L, lw, lh, (x + 0.5f) * lw / W, (y + 0.5f) * lh / H);
}

dim3 grid2(int w, int h) { return dim3((w + 15) / 16, (h + 15) / 16); }

}  // namespace

cudaError_t post_bloom(const PostLevels& L, float strength, cudaStream_t st) {
    for (int k = 1; k < L.n; ++k)
        k_down<<<grid2(L.w[k], L.h[k]), dim3(16, 16), 0, st>>>(L.p[k - 1], L.w[k - 1], L.h[k - 1], L.p[k], L.w[k], L.h[k]);
    k_bloom<<<grid2(L.w[0], L.h[0]), dim3(16, 16), 0, st>>>(L.p[0], L.w[0], L.h[0], L, strength);
    return cudaGetLastError();
}

cudaError_t post_radio_blur(const PostLevels& L, float4* tmp, double sigma, cudaStream_t st) {
    int k = 0;
    while (k + 1 < L.n && sigma / (1 << (k + 1)) > 3.0) ++k;
    for (int j = 1; j <= k; ++j)
        k_down<<<grid2(L.w[j], L.h[j]), dim3(16, 16), 0, st>>>(L.p[j - 1], L.w[j - 1], L.h[j - 1], L.p[j], L.w[j], L.h[j]);
    const float s = (float)(sigma / (1 << k));
    float4* lev = L.p[k];
    k_gauss<<<grid2(L.w[k], L.h[k]), dim3(16, 16), 0, st>>>(lev, tmp, L.w[k], L.h[k], s, 1);
    k_gauss<<<grid2(L.w[k], L.h[k]), dim3(16, 16), 0, st>>>(tmp, lev, L.w[k], L.h[k], s, 0);
    if (k > 0) k_upsample<<<grid2(L.w[0], L.h[0]), dim3(16, 16), 0, st>>>(lev, L.w[k], L.h[k], L.p[0], L.w[0], L.h[0]);
    return cudaGetLastError();
}

}  // namespace so
