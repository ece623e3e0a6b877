// so_noalloc.cu -- the radio-flux measurement for callers that cannot allocate device memory.
//
// so_radio_flux (a renderer call) needs the renderer's buffers, which so_init obtains with
// cudaMalloc.  Some callers cannot allocate at the point where they need the flux: code running
// under a memory pool or arena that owns every device allocation of the process, a real-time loop
// whose allocations are all made up front, or a plugin host that forbids allocation inside its
// callbacks.  so_radio_flux_noalloc serves them: the caller hands in the scene, the frame, the plasma
// modes and a device double for the result, all in memory it already owns, and the working memory
// (per-pixel sums, reduction partials, ray-queue counters) comes from the fixed array below, which
// exists from the moment the library is loaded on a GPU.
//
// A turbulent reference-model flow is traced with the sheared noise evaluated at every flow step (the
// reference's turb_nt = 0 path): the renderer's default, 24 baked slices of 453 MB, cannot live in a
// fixed array.  Its flux therefore equals so_radio_flux's once that renderer has been switched to
// SO_FLOW_NOISE_INLINE; with the baked slices the two are different draws of the turbulence.
//
// The device address of the array is looked up once per device ordinal and kept for the life of the
// process.  cudaDeviceReset (or anything else that unloads the library's module from a device)
// between calls is not supported: the module may come back at another address.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "so_launch.h"

namespace so {
cudaError_t launch_trace64(const TraceLaunch& L, int variant, int num_sms, cudaStream_t st);
cudaError_t launch_resolve(float4* img, const float4* accum, const uint32_t* nsamp, uint32_t nconst, long long npix,
                           int visible, cudaStream_t st);
cudaError_t launch_sum_channel(const float* v, int stride, long long n, double* part, double* out, int num_sms,
                               cudaStream_t st);
void set_global_error(const std::string& msg);
}  // namespace so

namespace {

// Layout of the scratch array: [0, 256) counters and the frame's scene index (cleared every call),
// [256, 256 + 5120) the reduction partials (SUM_MAX_PARTIALS doubles) and the flux sum after them,
// then one float4 per pixel.
constexpr size_t OFF_COUNTERS = 0;
constexpr size_t OFF_PARTIALS = 256;
constexpr size_t OFF_SUM = OFF_PARTIALS + (size_t)so::SUM_MAX_PARTIALS * sizeof(double);
constexpr size_t OFF_ACCUM = 256 + 5120;
static_assert(sizeof(so::Counters) + sizeof(int) <= 256, "counters and scene index must fit the cleared header");
static_assert(OFF_SUM + sizeof(double) <= OFF_ACCUM, "partials and the flux sum must fit before the pixels");
constexpr size_t SCRATCH_BYTES = OFF_ACCUM + (size_t)SO_NOALLOC_MAX_PIXELS * 16;

// Held by every GPU that loads the library, until the process exits.
static __device__ __align__(256) unsigned char g_scratch[SCRATCH_BYTES];

struct DeviceScratch {
    unsigned char* base = nullptr;  // device address of g_scratch on this device
    int num_sms = 0;
};
std::mutex g_mu;
DeviceScratch g_dev[64];

// Jy = sum of I_nu * pixel solid angle / 1e-23, in the order so_radio_flux evaluates it.
__global__ void k_flux_to_jy(double* __restrict__ jy, const double* __restrict__ sum, double pix_sr) {
    *jy = *sum * pix_sr / 1e-23;
}

}  // namespace

extern "C" int so_radio_flux_noalloc(const so_scene* d_scene, const so_frame* d_frame, int n, double pix_sr,
                                     const so_plasma* plasma, const so_mode* d_modes, double* d_jy, void* stream) {
    using namespace so;
    if (!d_scene || !d_frame || !d_jy || n <= 0) {
        set_global_error("so_radio_flux_noalloc: NULL pointer or n <= 0");
        return SO_ERR_ARG;
    }
    if ((long long)n * n > SO_NOALLOC_MAX_PIXELS) {
        set_global_error("so_radio_flux_noalloc: n*n = " + std::to_string((long long)n * n) +
                         " pixels exceeds the fixed scratch of SO_NOALLOC_MAX_PIXELS = " +
                         std::to_string(SO_NOALLOC_MAX_PIXELS));
        return SO_ERR_SIZE;
    }
    const bool torus = plasma && plasma->model == SO_PLASMA_TORUS && plasma->n_modes > 0;
    if (torus && (!d_modes || plasma->n_modes > SO_MAX_MODES)) {
        set_global_error("so_radio_flux_noalloc: torus plasma needs 1..SO_MAX_MODES device modes");
        return SO_ERR_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        set_global_error("so_radio_flux_noalloc: no current CUDA device");
        return SO_ERR_NO_DEVICE;
    }
    // Set-up, once per device with that device current: the device address of the array.  The
    // first call on a device does this, so make it before any stream capture.
    DeviceScratch ds;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_dev[dev].base) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
            if (e != cudaSuccess) {
                set_global_error(std::string("so_radio_flux_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                return SO_ERR_CUDA;
            }
            int nsm = 0;
            if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm <= 0) nsm = 1;
            g_dev[dev].base = static_cast<unsigned char*>(p);
            g_dev[dev].num_sms = nsm;
        }
        ds = g_dev[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Counters* cnt = reinterpret_cast<Counters*>(ds.base + OFF_COUNTERS);
    int* frame_scene = reinterpret_cast<int*>(ds.base + OFF_COUNTERS + sizeof(Counters));
    double* partials = reinterpret_cast<double*>(ds.base + OFF_PARTIALS);
    double* sum = reinterpret_cast<double*>(ds.base + OFF_SUM);
    float4* accum = reinterpret_cast<float4*>(ds.base + OFF_ACCUM);
    // The array keeps the previous call's contents: clear the queue head, counters and scene index.
    cudaError_t e = cudaMemsetAsync(ds.base + OFF_COUNTERS, 0, 256, st);
    if (e == cudaSuccess) {
        TraceLaunch L;
        std::memset(&L, 0, sizeof L);
        L.scenes = d_scene;
        L.frames = d_frame;
        L.frame_scene = frame_scene;
        L.nframes = 1;
        L.kind = RAYS_PIXELS;
        L.nrays = (long long)n * n;
        L.W = n;
        L.H = n;
        L.spp = 2;  // Renderer::radio_flux (render.cu:801)
        L.jitter = 1;
        L.accum = reinterpret_cast<float*>(accum);
        L.counters = cnt;
        if (torus) {
            L.torus = 1;
            L.n_modes = plasma->n_modes;
            L.ne_index = plasma->ne_index;
            L.te_index = plasma->te_index;
            L.h_sph = plasma->h_sph;
            L.theta_e0 = 1.380649e-16 * plasma->te0_kelvin / (9.1093837e-28 * 2.99792458e10 * 2.99792458e10);
            L.half_var = 0.5 * plasma->turb_rms * plasma->turb_rms;
            L.modes = d_modes;
        }
        e = launch_trace64(L, VAR_RADIO, ds.num_sms, st);
    }
    if (e == cudaSuccess) e = launch_resolve(accum, accum, nullptr, 2u, (long long)n * n, 0, st);  // in place
    if (e == cudaSuccess)
        e = launch_sum_channel(reinterpret_cast<const float*>(accum), 4, (long long)n * n, partials, sum, ds.num_sms, st);
    if (e == cudaSuccess) {
        k_flux_to_jy<<<1, 1, 0, st>>>(d_jy, sum, pix_sr);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        set_global_error(std::string("so_radio_flux_noalloc: ") + cudaGetErrorString(e));
        return SO_ERR_CUDA;
    }
    return SO_OK;
}
