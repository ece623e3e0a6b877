// ref_post_shim.cpp -- host build of the REFERENCE's own pyramid-filter kernels and of its k_adapt /
// k_dilate.  TEST INFRASTRUCTURE ONLY.
//
// render.cu as a whole needs nvcc and the font atlas, but its post filters (render.cu:244-316:
// k_down, bilinear, LevelPtrs, k_bloom, k_gauss, k_upsample) are plain per-pixel code.  oracle/Makefile
// cuts that line range out of the reference tree into _ref/post_kernels.inc (never committed) and
// this file compiles it as host C++ inside namespace refpost, where:
//   blockIdx / threadIdx / blockDim -> per-thread host variables set by launch2() below, which walks
//                                      the reference's grid2(w, h) x dim3(16, 16) launch shape;
//   __expf(x)                       -> expf(x) (k_gauss's weights; CUDA's __expf is approximate, so
//                                      the host figures differ from the GPU's in the last bits);
//   min / max on int                -> std::min / std::max.
// The launch sequences are Impl::bloom (render.cu:732-740) and Impl::radio_blur (:742-753) on the
// pyramid that Renderer::init sizes (:638-647), restated in bloom() / radio_blur() below.
//
// k_adapt / k_dilate (render.cu:130-150) come the same way from _ref/adapt_kernels.inc.  Host
// caveat: g++ (no -mfma, no contraction) evaluates k_adapt's s.y / n - mean * mean in two roundings
// where nvcc fuses it, so a pixel whose estimate sits on an integer may differ by one sample.
//
// Output: linked into oracle/_ref/libbhref.so; tests/golden/make_golden.py writes fixtures from it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#define __expf(x) expf(x)

namespace refpost {
using std::max;
using std::min;

struct Idx3 {
    unsigned x, y, z;
};
thread_local Idx3 blockIdx, threadIdx, blockDim;

constexpr int MAX_LEVELS = 9;  // render.cu:32
constexpr int CHUNK = 8;       // render.cu:30

#include "adapt_kernels.inc"
#include "post_kernels.inc"

// grid2(w, h) with 16 x 16 blocks (render.cu's launch shape for every filter kernel): every thread
// of every block, in order; the kernels return early outside the image.
template <class K>
void launch2(int w, int h, K kernel) {
    blockDim = {16u, 16u, 1u};
    const int gx = (w + 15) / 16, gy = (h + 15) / 16;
    for (int by = 0; by < gy; ++by)
        for (int bx = 0; bx < gx; ++bx)
            for (int ty = 0; ty < 16; ++ty)
                for (int tx = 0; tx < 16; ++tx) {
                    blockIdx = {(unsigned)bx, (unsigned)by, 0u};
                    threadIdx = {(unsigned)tx, (unsigned)ty, 0u};
                    kernel();
                }
}

struct Pyramid {
    std::vector<std::vector<float4>> lev;
    int lw[MAX_LEVELS], lh[MAX_LEVELS], n = 0;
    // level 0 is the frame itself; the others halve (rounding up) while both sides are >= 2
    Pyramid(const float* img, int W, int H) {
        int w = W, h = H;
        while (n < MAX_LEVELS && w >= 2 && h >= 2) {
            lw[n] = w;
            lh[n] = h;
            lev.emplace_back((size_t)w * h);
            ++n;
            w = (w + 1) / 2;
            h = (h + 1) / 2;
        }
        if (n > 0) std::memcpy(lev[0].data(), img, sizeof(float4) * (size_t)W * H);
    }
    void down(int k) {
        const float4* src = lev[k - 1].data();
        float4* dst = lev[k].data();
        const int sw = lw[k - 1], sh = lh[k - 1], dw = lw[k], dh = lh[k];
        launch2(dw, dh, [&] { k_down(src, sw, sh, dst, dw, dh); });
    }
};

void bloom(const float* img, float* out, int W, int H, float strength) {
    Pyramid P(img, W, H);
    for (int k = 1; k < P.n; ++k) P.down(k);
    LevelPtrs L;
    L.n = P.n;
    for (int k = 0; k < P.n; ++k) {
        L.p[k] = P.lev[k].data();
        L.w[k] = P.lw[k];
        L.h[k] = P.lh[k];
    }
    float4* d = P.lev[0].data();
    launch2(W, H, [&] { k_bloom(d, W, H, L, strength); });
    std::memcpy(out, d, sizeof(float4) * (size_t)W * H);
}

// A 1-D launch of 256-thread blocks over n items (render.cu:703).
template <class K>
void launch1(int n, K kernel) {
    blockDim = {256u, 1u, 1u};
    for (int b = 0; b < (n + 255) / 256; ++b)
        for (int t = 0; t < 256; ++t) {
            blockIdx = {(unsigned)b, 0u, 0u};
            threadIdx = {(unsigned)t, 0u, 0u};
            kernel();
        }
}

void radio_blur(const float* img, float* out, int W, int H, double sigma) {
    Pyramid P(img, W, H);
    int k = 0;
    while (k + 1 < P.n && sigma / (1 << (k + 1)) > 3.0) ++k;
    for (int j = 1; j <= k; ++j) P.down(j);
    const float s = (float)(sigma / (1 << k));
    float4* L = P.lev[k].data();
    const int w = P.lw[k], h = P.lh[k];
    std::vector<float4> tmp((size_t)w * h);
    float4* t = tmp.data();
    launch2(w, h, [&] { k_gauss(L, t, w, h, s, 1); });
    launch2(w, h, [&] { k_gauss(t, L, w, h, s, 0); });
    if (k > 0) {
        float4* d = P.lev[0].data();
        launch2(W, H, [&] { k_upsample(L, w, h, d, W, H); });
    }
    std::memcpy(out, P.lev[0].data(), sizeof(float4) * (size_t)W * H);
}
}  // namespace refpost

extern "C" {
// Impl::bloom on a W x H float4 frame (row-major, 4 floats per pixel); in and out may not overlap.
void ref_post_bloom(const float* img, float* out, int W, int H, float strength) {
    refpost::bloom(img, out, W, H, strength);
}
// k_adapt then k_dilate on a W x H frame (render.cu:702-704): ystat is W*H float2, nsamp W*H
// counts; extra and chunks receive W*H counts each.
void ref_adapt_dilate(const float* ystat, const uint32_t* nsamp, int W, int H, float yref, float target, int extra_max,
                      uint32_t* extra, uint32_t* chunks) {
    using namespace refpost;
    const float2* ys = reinterpret_cast<const float2*>(ystat);
    const int n = W * H;
    launch1(n, [&] { k_adapt(ys, nsamp, n, yref, target, extra_max, extra); });
    launch2(W, H, [&] { k_dilate(extra, chunks, W, H, extra_max); });
}
// Impl::radio_blur with a beam of sigma pixels.
void ref_post_radio_blur(const float* img, float* out, int W, int H, double sigma) {
    refpost::radio_blur(img, out, W, H, sigma);
}
}
