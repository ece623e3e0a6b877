// k_frame.cu -- per-frame kernels around the tracer: resolve, deterministic reductions and the
// adaptive-resampling passes.
//
// Reference: k_resolve (blackholes/src/render.cu:227-242), the fsum of k_pass1 (render.cu:116-127),
// k_adapt (:130-140), k_dilate (:142-150), the exclusive scan k_scan_block/top/add (:152-194) and
// k_pass2's float atomics (:196-224).  Differences by design:
//   * sums are deterministic: the frame flux is a fixed-order FP64 tree over pixels, and pass-2
//     chunk sums are added to their pixel in chunk order by one thread per pixel (no float atomics);
//   * the scan is a single-pass decoupled-lookback scan (one launch instead of three).
#include <cuda_runtime.h>

#include <cstdint>

#include "so_launch.h"

namespace so {

namespace {
constexpr unsigned FULL = 0xffffffffu;
}

// img = accum / nsamp; visible mode converts XYZ to linear sRGB x 683 (render.cu:227-242).  img may be
// accum itself (the batch and the fixed-scratch flux resolve in place), so that pair is not
// __restrict__; each thread reads its pixel before it writes it.
__global__ void k_resolve(float4* img, const float4* accum, const uint32_t* __restrict__ nsamp, uint32_t nconst,
                          long long npix, int visible) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    float inv = 1.f / (float)(nsamp ? nsamp[p] : nconst);
    float4 a = accum[p];
    a.x *= inv;
    a.y *= inv;
    a.z *= inv;
    a.w *= inv;
    if (visible) {
        float X = a.x, Y = a.y, Z = a.z;
        float r = 3.2404542f * X - 1.5371385f * Y - 0.4985314f * Z;
        float g = -0.9692660f * X + 1.8760108f * Y + 0.0415560f * Z;
        float b = 0.0556434f * X - 0.2040259f * Y + 1.0572252f * Z;
        img[p] = make_float4(683.f * r, 683.f * g, 683.f * b, 683.f * a.w);
    } else {
        img[p] = a;
    }
}

// Fixed-order sum of one float channel (stride floats apart) into FP64: block partials in out[block].
__global__ void k_sum_channel(const float* __restrict__ v, int stride, long long n, double* __restrict__ out) {
    __shared__ double ws[32];
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s += (double)v[i * stride];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(FULL, s, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(FULL, s, o);
        if (threadIdx.x == 0) out[blockIdx.x] = s;
    }
}
// Final fixed-order sum of nb partials.
__global__ void k_sum_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
    __shared__ double ws[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) s += part[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(FULL, s, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(FULL, s, o);
        if (threadIdx.x == 0) *out = s;
    }
}

// k_adapt (render.cu:130-140): extra samples so that the standard error of the mean luminance falls
// below target * (mean + yref).
__global__ void k_adapt(const float2* __restrict__ ystat, uint32_t spp, long long npix, const double* __restrict__ fsum,
                        double yscale, float target, int extra_max, uint32_t* __restrict__ extra) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    float yref = (float)(0.03 * (*fsum) * yscale + 1e-37);
    float n = (float)spp;
    float2 s = ystat[p];
    float mean = s.x / n, var = fmaxf(s.y / n - mean * mean, 0.f);
    float se = sqrtf(var / n), den = target * (mean + yref);
    float want = n * (se / den) * (se / den);
    extra[p] = (uint32_t)fminf(fmaxf(ceilf(want) - n, 0.f), (float)extra_max);
}

// k_dilate (render.cu:142-150): 3x3 max of the extra-sample counts, in chunks of `chunk` samples.
__global__ void k_dilate(const uint32_t* __restrict__ extra, uint32_t* __restrict__ chunks, int W, int H, int extra_max,
                         int chunk) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    uint32_t m = 0;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx)
            m = max(m, extra[min(max(y + dy, 0), H - 1) * W + min(max(x + dx, 0), W - 1)]);
    chunks[y * W + x] = (min(m, (uint32_t)extra_max) + chunk - 1) / chunk;
}

// Single-pass exclusive scan with decoupled look-back (Merrill & Garland 2016).  Each block scans
// SCAN_TILE elements, publishes its aggregate (flag 1) and, once its predecessors are known, its
// inclusive prefix (flag 2).  A block only waits on blocks with smaller tile index, which were
// scheduled earlier because tiles are taken from a counter, so the look-back always finishes; the
// wait is still bounded by an iteration limit, after which the block records an error and writes a
// well-defined (but wrong) result instead of spinning.
constexpr int SCAN_TPB = 256, SCAN_PER = 8, SCAN_TILE = SCAN_TPB * SCAN_PER;
__global__ void k_scan_lookback(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, long long n,
                                unsigned long long* __restrict__ tile_state, unsigned int* __restrict__ tile_counter,
                                uint32_t* __restrict__ total, int* __restrict__ err) {
    __shared__ uint32_t s_tile;
    __shared__ uint32_t ws[SCAN_TPB / 32];
    __shared__ uint32_t s_prefix;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const long long base = (long long)tile * SCAN_TILE + (long long)threadIdx.x * SCAN_PER;
    uint32_t v[SCAN_PER], run = 0;
#pragma unroll
    for (int i = 0; i < SCAN_PER; ++i) {
        v[i] = base + i < n ? in[base + i] : 0u;
        run += v[i];
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) ws[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < SCAN_TPB / 32 ? ws[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(FULL, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < SCAN_TPB / 32) ws[lane] = wi - w;  // exclusive warp offsets
        if (lane == SCAN_TPB / 32 - 1) {
            const uint32_t agg = wi;
            uint32_t prefix = 0;
            if (tile == 0) {
                atomicExch(&tile_state[0], (2ull << 32) | agg);
            } else {
                atomicExch(&tile_state[tile], (1ull << 32) | agg);
                long long j = (long long)tile - 1;
                long long spins = 0;
                while (j >= 0) {
                    unsigned long long st = atomicAdd(&tile_state[j], 0ull);
                    uint32_t flag = (uint32_t)(st >> 32);
                    if (flag == 0) {
                        if (++spins > (1ll << 24)) {
                            atomicExch(err, 1);
                            break;
                        }
                        continue;
                    }
                    prefix += (uint32_t)st;
                    if (flag == 2) break;
                    --j;
                }
                atomicExch(&tile_state[tile], (2ull << 32) | (uint32_t)(prefix + agg));
            }
            s_prefix = prefix;
            if ((long long)(tile + 1) * SCAN_TILE >= n) *total = prefix + agg;
        }
    }
    __syncthreads();
    uint32_t off = s_prefix + ws[wid] + incl - run;
#pragma unroll
    for (int i = 0; i < SCAN_PER; ++i) {
        if (base + i < n) out[base + i] = off;
        off += v[i];
    }
}

// Pass-2 chunk sums -> pixels, in chunk order (replaces k_pass2's float atomics, render.cu:221-223).
__global__ void k_add_chunks(float4* __restrict__ accum, uint32_t* __restrict__ nsamp, const uint32_t* __restrict__ offsets,
                             const uint32_t* __restrict__ chunks, const float4* __restrict__ chunk_acc, long long npix,
                             int chunk) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    uint32_t c = chunks[p];
    if (c == 0) return;
    float4 a = accum[p];
    uint32_t o = offsets[p];
    for (uint32_t k = 0; k < c; ++k) {
        float4 v = chunk_acc[o + k];
        a.x += v.x;
        a.y += v.y;
        a.z += v.z;
        a.w += v.w;
    }
    accum[p] = a;
    nsamp[p] += c * (uint32_t)chunk;
}

// Per pixel: the sum of its spp samples in sample order and (sum Y, sum Y^2), as k_pass1 accumulates
// them (render.cu:103-113); the mixed path writes one result per sample first.  Compiled without
// flush-to-zero, so an all-FP64 mixed frame equals the plain FP64 frame bit for bit.
__global__ void k_gather_samples(const TraceLaunch L) {
    const long long npix = (long long)L.W * L.H;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f, ys = 0.f, yq = 0.f;
    const bool radio = L.scenes[0].mode == SO_MODE_RADIO;
    for (int s = 0; s < L.spp; ++s) {
        float4 v = L.sample_out[p * L.spp + s];
        a0 += v.x;
        a1 += v.y;
        a2 += v.z;
        a3 += v.w;
        float Y = radio ? v.x : v.y;
        ys += Y;
        yq += Y * Y;
    }
    reinterpret_cast<float4*>(L.accum)[p] = make_float4(a0, a1, a2, a3);
    if (L.ystat) reinterpret_cast<float2*>(L.ystat)[p] = make_float2(ys, yq);
}

cudaError_t launch_gather_samples(const TraceLaunch& L, cudaStream_t st) {
    long long npix = (long long)L.W * L.H;
    k_gather_samples<<<(int)((npix + 255) / 256), 256, 0, st>>>(L);
    return cudaGetLastError();
}

__global__ void k_fill_u32(uint32_t* __restrict__ p, uint32_t v, long long n) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// ---- host launchers --------------------------------------------------------------------------
static inline int blocks_for(long long n, int tpb) { return (int)((n + tpb - 1) / tpb); }

cudaError_t launch_resolve(float4* img, const float4* accum, const uint32_t* nsamp, uint32_t nconst, long long npix,
                           int visible, cudaStream_t st) {
    if (npix <= 0) return cudaSuccess;
    k_resolve<<<blocks_for(npix, 256), 256, 0, st>>>(img, accum, nsamp, nconst, npix, visible);
    return cudaGetLastError();
}

// part must hold SUM_MAX_PARTIALS doubles; result in *out.
cudaError_t launch_sum_channel(const float* v, int stride, long long n, double* part, double* out, int num_sms,
                               cudaStream_t st) {
    int nb = num_sms * 4;
    if (nb > SUM_MAX_PARTIALS) nb = SUM_MAX_PARTIALS;
    long long need = (n + 255) / 256;
    if (need < nb) nb = (int)(need > 0 ? need : 1);
    k_sum_channel<<<nb, 256, 0, st>>>(v, stride, n, part);
    k_sum_final<<<1, 256, 0, st>>>(part, nb, out);
    return cudaGetLastError();
}

cudaError_t launch_adapt(const float2* ystat, uint32_t spp, long long npix, const double* fsum, double yscale, float target,
                         int extra_max, uint32_t* extra, uint32_t* chunks, int W, int H, int chunk, cudaStream_t st) {
    k_adapt<<<blocks_for(npix, 256), 256, 0, st>>>(ystat, spp, npix, fsum, yscale, target, extra_max, extra);
    dim3 g((W + 15) / 16, (H + 15) / 16);
    k_dilate<<<g, dim3(16, 16), 0, st>>>(extra, chunks, W, H, extra_max, chunk);
    return cudaGetLastError();
}

long long scan_tiles(long long n) { return (n + SCAN_TILE - 1) / SCAN_TILE; }

// tile_state: scan_tiles(n) u64 + 1 u32 counter, zeroed by the caller.
cudaError_t launch_scan(const uint32_t* in, uint32_t* out, long long n, unsigned long long* tile_state,
                        unsigned int* tile_counter, uint32_t* total, int* err, cudaStream_t st) {
    long long nt = scan_tiles(n);
    if (nt < 1) nt = 1;
    k_scan_lookback<<<(int)nt, SCAN_TPB, 0, st>>>(in, out, n, tile_state, tile_counter, total, err);
    return cudaGetLastError();
}

cudaError_t launch_add_chunks(float4* accum, uint32_t* nsamp, const uint32_t* offsets, const uint32_t* chunks,
                              const float4* chunk_acc, long long npix, int chunk, cudaStream_t st) {
    k_add_chunks<<<blocks_for(npix, 256), 256, 0, st>>>(accum, nsamp, offsets, chunks, chunk_acc, npix, chunk);
    return cudaGetLastError();
}

cudaError_t launch_fill_u32(uint32_t* p, uint32_t v, long long n, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_fill_u32<<<blocks_for(n, 256), 256, 0, st>>>(p, v, n);
    return cudaGetLastError();
}

}  // namespace so
