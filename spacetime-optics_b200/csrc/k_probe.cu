// k_probe.cu -- FMA-pipe peak probe: the measured denominator of the tracers' roofline.
// Every thread runs 8 independent FMA chains (enough instruction-level parallelism to hide the
// pipe latency), on 8 CTAs of 256 threads per SM, and the kernel is timed with CUDA events.
#include <cuda_runtime.h>

#include "../../include/so_tracer.h"
#include "so_kerr.cuh"

namespace {
template <typename T>
__global__ void __launch_bounds__(256) k_fma_chains(T* out, int iters, T a, T b) {
    T x0 = (T)threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == (T)-12345.678) out[threadIdx.x] = s;  // keeps the chains live
}

template <typename T>
int probe(int nsm, int iters, double* tflops) {
    T* out = nullptr;
    if (cudaMalloc(&out, 256 * sizeof(T)) != cudaSuccess) return SO_ERR_ALLOC;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = nsm * 8;
    k_fma_chains<T><<<blocks, 256>>>(out, iters / 4, (T)0.999999, (T)1e-7);  // warm-up
    cudaEventRecord(e0);
    k_fma_chains<T><<<blocks, 256>>>(out, iters, (T)0.999999, (T)1e-7);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess || ms <= 0.f) return SO_ERR_CUDA;
    double flops = 2.0 * 8.0 * 16.0 * (double)iters * blocks * 256.0;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return SO_OK;
}
}  // namespace

__global__ void __launch_bounds__(256) k_sfu_chains(float* out, int iters, float b) {
    float x0 = threadIdx.x * 1e-3f, x1 = x0 + 0.1f, x2 = x0 + 0.2f, x3 = x0 + 0.3f, x4 = x0 + 0.4f, x5 = x0 + 0.5f,
          x6 = x0 + 0.6f, x7 = x0 + 0.7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            x0 = __cosf(x0) + b; x1 = __cosf(x1) + b; x2 = __cosf(x2) + b; x3 = __cosf(x3) + b;
            x4 = __cosf(x4) + b; x5 = __cosf(x5) + b; x6 = __cosf(x6) + b; x7 = __cosf(x7) + b;
        }
    }
    float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == -12345.678f) out[threadIdx.x] = s;
}

extern "C" int so_probe_sfu_peak(int device, double* gops) {
    if (!gops) return SO_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return SO_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return SO_ERR_CUDA;
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    float* out = nullptr;
    if (cudaMalloc(&out, 256 * sizeof(float)) != cudaSuccess) return SO_ERR_ALLOC;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = nsm * 8, iters = 500;
    k_sfu_chains<<<blocks, 256>>>(out, iters / 4, 1e-3f);
    cudaEventRecord(e0);
    k_sfu_chains<<<blocks, 256>>>(out, iters, 1e-3f);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess || ms <= 0.f) return SO_ERR_CUDA;
    *gops = 8.0 * 16.0 * (double)iters * blocks * 256.0 / (ms * 1e-3) / 1e9;
    return SO_OK;
}

extern "C" int so_probe_fma_peak(int device, double* fp64_tflops, double* fp32_tflops) {
    if (!fp64_tflops || !fp32_tflops) return SO_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return SO_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return SO_ERR_CUDA;
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    int rc = probe<double>(nsm, 2000, fp64_tflops);
    if (!rc) rc = probe<float>(nsm, 4000, fp32_tflops);
    return rc;
}

namespace {
__global__ void k_cos_turns(const double* __restrict__ t, double* __restrict__ out, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = so::cos_turns(t[i]);
}
}  // namespace

extern "C" int so_probe_cos_turns(const double* d_t, double* d_out, long long n) {
    if (n < 0 || (n > 0 && (!d_t || !d_out))) return SO_ERR_ARG;
    if (n == 0) return SO_OK;
    k_cos_turns<<<592, 256>>>(d_t, d_out, n);
    return cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess ? SO_OK : SO_ERR_CUDA;
}
