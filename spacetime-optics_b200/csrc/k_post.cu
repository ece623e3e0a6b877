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

// ---- luminance statistics (render.cu:771-790) -----------------------------------------------------
namespace {

// Y per pixel with the host expression's roundings (float in radio mode, double in visible mode;
// explicit _rn operations so that no multiply-add is fused), and the block maxima of Y > 0.
__global__ void __launch_bounds__(256) k_lum(const float4* __restrict__ img, long long n, int radio, float hide,
                                             float* __restrict__ lum, double* __restrict__ part) {
    __shared__ double sm[256];
    double m = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float4 c = img[i];
        double Y;
        if (radio) {
            const float d = fmaxf(__fsub_rn(__fsub_rn(__fsub_rn(c.x, c.y), c.z), c.w), 0.f);
            Y = (double)__fsub_rn(c.x, __fmul_rn(hide, d));
        } else {
            Y = __dadd_rn(__dadd_rn(__dmul_rn(0.2126, (double)c.x), __dmul_rn(0.7152, (double)c.y)),
                          __dmul_rn(0.0722, (double)c.z));
        }
        lum[i] = Y > 0.0 ? (float)Y : -1.f;
        if (Y > 0.0) m = fmax(m, Y);
    }
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sm[0];
}

__global__ void __launch_bounds__(256) k_lum_max(const double* __restrict__ part, int nb, LumStat* st) {
    __shared__ double sm[256];
    double m = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) m = fmax(m, part[i]);
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        st->mx = sm[0];
        st->pv = 0.f;
        st->nsig = 0;
        st->k = 0;
        st->prefix = 0;
    }
}

// Radix pass over the significant values (v > mx 1e-5, v as double): pass 0 bins bits 30..19 of the
// float pattern, pass 1 bits 18..8 of those whose bits 30..19 are the selected prefix, pass 2 bits
// 7..0 of those whose bits 30..8 are.  (Positive floats order as their bit patterns.)
__global__ void __launch_bounds__(256) k_lum_hist(const float* __restrict__ lum, long long n, const LumStat* st,
                                                  int pass, unsigned* __restrict__ hist) {
    __shared__ unsigned sh[LUM_HIST];
    for (int b = threadIdx.x; b < LUM_HIST; b += blockDim.x) sh[b] = 0;
    __syncthreads();
    const double thr = __dmul_rn(st->mx, 1e-5);
    const unsigned prefix = st->prefix;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float v = lum[i];
        if (!(v > 0.f) || !((double)v > thr)) continue;
        const unsigned u = __float_as_uint(v);
        if (pass == 0) atomicAdd(&sh[(u >> 19) & 4095u], 1u);
        else if (pass == 1 && (u >> 19) == prefix) atomicAdd(&sh[(u >> 8) & 2047u], 1u);
        else if (pass == 2 && (u >> 8) == prefix) atomicAdd(&sh[u & 255u], 1u);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < LUM_HIST; b += blockDim.x)
        if (sh[b]) atomicAdd(&hist[b], sh[b]);
}

// The bin holding rank k (one thread: at most 4096 bins), then the rank inside it.  After pass 0
// the rank is min(n - 1, (size_t)(percentile (n - 1))) of the n significant values, as the host's.
__global__ void k_lum_pick(const unsigned* __restrict__ hist, int pass, double percentile, LumStat* st) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int nb = pass == 0 ? 4096 : pass == 1 ? 2048 : 256;
    unsigned long long k = st->k;
    if (pass == 0) {
        unsigned long long n = 0;
        for (int b = 0; b < nb; ++b) n += hist[b];
        st->nsig = n;
        if (n == 0) return;
        k = (unsigned long long)(percentile * (double)(n - 1));
        if (k > n - 1) k = n - 1;
    }
    if (st->nsig == 0) return;
    unsigned long long cum = 0;
    int b = 0;
    for (; b < nb - 1; ++b) {
        if (cum + hist[b] > k) break;
        cum += hist[b];
    }
    st->k = k - cum;
    if (pass == 0) st->prefix = (unsigned)b;
    else if (pass == 1) st->prefix = (st->prefix << 11) | (unsigned)b;
    else st->pv = __uint_as_float((st->prefix << 8) | (unsigned)b);
}

}  // namespace

cudaError_t post_luminance(const float4* img, long long n, int radio, float hide, double percentile,
                           const LumScratch& s, cudaStream_t st) {
    k_lum<<<LUM_BLOCKS, 256, 0, st>>>(img, n, radio, hide, s.lum, s.part);
    k_lum_max<<<1, 256, 0, st>>>(s.part, LUM_BLOCKS, s.stat);
    for (int pass = 0; pass < 3; ++pass) {
        cudaError_t e = cudaMemsetAsync(s.hist, 0, LUM_HIST * sizeof(unsigned), st);
        if (e != cudaSuccess) return e;
        k_lum_hist<<<LUM_BLOCKS, 256, 0, st>>>(s.lum, n, s.stat, pass, s.hist);
        k_lum_pick<<<1, 32, 0, st>>>(s.hist, pass, percentile, s.stat);
    }
    return cudaGetLastError();
}

}  // namespace so
