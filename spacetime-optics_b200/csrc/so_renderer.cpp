// so_renderer.cpp -- the Renderer of the reference (blackholes/src/renderer.hpp:72-88,
// render.cu:477-809) behind the C ABI of include/so_tracer.h.
//
// Per frame (so_render, render.cu:677-730 + 755-795):
//   frame descriptor -> device;  pass 1 (spp samples per pixel, persistent tracer kernel);
//   adaptive pass 2 (k_adapt, k_dilate, single-pass scan, chunked samples, deterministic add);
//   resolve;  device -> host copy of the HDR frame;  luminance percentile on the host.
// Differences from the reference: every failure is a status code (no abort), reductions are
// deterministic, per-frame scene data live in device memory (not __constant__), and there is no
// sky texture (SO_ERR_UNSUPPORTED).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "so_kerr.cuh"
#include "so_launch.h"

namespace so {
cudaError_t launch_trace64(const TraceLaunch& L, int variant, int num_sms, cudaStream_t st);
cudaError_t launch_trace_mixed(const TraceLaunch& L, int variant, int num_sms, cudaStream_t st);
cudaError_t launch_resolve(float4* img, const float4* accum, const uint32_t* nsamp, uint32_t nconst, long long npix,
                           int visible, cudaStream_t st);
cudaError_t launch_sum_channel(const float* v, int stride, long long n, double* part, double* out, int num_sms,
                               cudaStream_t st);
cudaError_t launch_adapt(const float2* ystat, uint32_t spp, long long npix, const double* fsum, double yscale,
                         float target, int extra_max, uint32_t* extra, uint32_t* chunks, int W, int H, int chunk,
                         cudaStream_t st);
long long scan_tiles(long long n);
cudaError_t launch_scan(const uint32_t* in, uint32_t* out, long long n, unsigned long long* tile_state,
                        unsigned int* tile_counter, uint32_t* total, int* err, cudaStream_t st);
cudaError_t launch_add_chunks(float4* accum, uint32_t* nsamp, const uint32_t* offsets, const uint32_t* chunks,
                              const float4* chunk_acc, long long npix, int chunk, cudaStream_t st);
cudaError_t launch_fill_u32(uint32_t* p, uint32_t v, long long n, cudaStream_t st);
}  // namespace so

using namespace so;

namespace {
constexpr int CHUNK = 8;  // samples per pass-2 job (render.cu:30)
// Message of the last failed call that has no renderer to hold it (so_init, the shot builders,
// so_radio_flux_noalloc, so_sur_gemm).  One per host thread, like errno: renderers on different
// GPUs may be driven from different threads, and a shared string would be a data race.
thread_local std::string g_init_error;

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

struct so_renderer {
    int device = 0, num_sms = 148;
    cudaStream_t st = nullptr;
    so_scene S{};            // host copy, table pointers = device tables
    so_settings rs{};
    float *d_disk = nullptr, *d_k2 = nullptr, *d_bb = nullptr;
    so_scene* d_scene = nullptr;
    so_frame* d_frame = nullptr;
    int* d_frame_scene = nullptr;
    // frame buffers
    long long npix = 0;
    float4 *d_accum = nullptr, *d_img = nullptr, *d_chunk_acc = nullptr;
    float2* d_ystat = nullptr;
    uint32_t *d_nsamp = nullptr, *d_extra = nullptr, *d_chunks = nullptr, *d_offsets = nullptr, *d_total = nullptr;
    unsigned long long* d_tiles = nullptr;
    int* d_err = nullptr;
    long long chunk_cap = 0;
    double *d_part = nullptr, *d_fsum = nullptr;
    Counters* d_cnt = nullptr;
    // per-ray buffers of so_trace_rays (grown on demand)
    long long ray_cap = 0;
    double *d_x = nullptr, *d_y = nullptr;
    void* d_rays = nullptr;  // packed outputs
    // plasma / precision
    so_plasma plasma{};
    so_mode* d_modes = nullptr;
    TurbModes* turb_modes = nullptr;  // the modes folded to FP32 for the batched turbulence sums
    int precision = SO_PREC_FP64;
    so_mixed_opts mixed{0.05, 3e-6, 0.0, 1e-4, 0.0, 0.0, 0, 0, 0, 0.0, 0, 0.0, 0};
    // deferred turbulence: record pool (segments of REC_SEG slots), grown when a frame runs out
    float4* d_rec = nullptr;
    float* d_rec_delta = nullptr;
    uint32_t* d_seg_next = nullptr;
    int2* d_ray_meta = nullptr;
    uint32_t* d_acc_list = nullptr;
    long long seg_cap = 0, meta_cap = 0;
    double rec_per_ray = 320.0;             // pool size per FP32 ray (records), doubled after a shortage
    unsigned long long* h_seg = nullptr;    // pinned: [0] segments requested, [1] rays short of segments
    cudaEvent_t ev_seg = nullptr;           // after the copy into h_seg
    bool seg_pending = false;
    bool last_defer = false;                // the last mixed frame deferred its turbulence
    long long pool_target = -1;             // pool size (segments) last asked for
    int waves = 1;                          // FP32 ray waves per frame (the pool holds one wave)
    long long wave_rays = 0;                // parked-list entries per wave
    int last_waves = 0;
    std::vector<cudaEvent_t> ev_wave;       // per wave: tracer end, sums end, transfer end
    // attempts of the reference's Mino-time approach of the central ray, for the key below
    int approach_it = 0;
    uint32_t* d_esc_list = nullptr;  // star-map frames on the mixed path: escaped FP32 rays
    long long esc_cap = 0;
    // baked flow turbulence (reference flow model with turbulence, radio mode): the frame's slices
    float* d_turb = nullptr;                       // SO_FLOW_NOISE_BAKED_FP32: the slices in plain memory
    cudaArray_t turb_arr[TURB_NT] = {};            // SO_FLOW_NOISE_BAKED: the slices as 3-D arrays,
    cudaSurfaceObject_t turb_surf[TURB_NT] = {};   // written through surfaces by the bake
    cudaTextureObject_t turb_texo[TURB_NT] = {};   // and read through the texture unit
    int flow_noise = SO_FLOW_NOISE_BAKED;
    TurbBake tb{};
    double approach_key[6] = {-1.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    // mixed-path buffers (grown on demand) and the critical-curve table of the current frame
    long long mixed_cap = 0;
    float4 *d_state = nullptr, *d_sample_out = nullptr;
    int8_t* d_sample_fate = nullptr;
    uint32_t *d_list32 = nullptr, *d_list64 = nullptr, *d_redo = nullptr, *d_parked = nullptr;
    unsigned long long* d_nlists = nullptr;
    Counters* d_cnt3 = nullptr;  // band and re-trace launches run on their own queue heads
    float* d_band = nullptr;
    double band_a = -1.0, band_th = -1.0;
    cudaStream_t st2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev32[2] = {nullptr, nullptr};  // around the FP32 tracer launch
    long long last_mixed_ns = 0;               // samples of the last mixed-precision pass 1
    // post filters: pyramid levels 1.. of d_img and a scratch frame (allocated on first use)
    PostLevels lev{};
    float4* d_tmp = nullptr;
    // star map (visible mode): mipmapped half2 texture and the pixel-corner escape coordinates
    int sky_requested = 0;  // the scene asked for the sky (sky_on at so_init)
    cudaMipmappedArray_t sky_mip = nullptr;
    cudaTextureObject_t sky_tex = 0;
    double *d_cx = nullptr, *d_cy = nullptr, *d_cth = nullptr, *d_cph = nullptr;
    int8_t* d_cfate = nullptr;
    float2* d_uvgrid = nullptr;
    long long corner_cap = 0;
    Counters* d_cnt_corner = nullptr;
    // luminance statistics of so_render (device buffers and the pinned result)
    LumScratch lum{};
    LumStat* h_lum = nullptr;
    // deferred FP64 passes of the plain tracer: record pool (segments of REC_SEG slots of rec64_w
    // doubles, each segment's link and owner), per-sample chain heads and end states, the recording
    // pass's counters, and the pool's use
    double* d_rec64 = nullptr;
    long long rec64_doubles = 0;               // size of d_rec64; segment arrays hold rec64_doubles / (REC_SEG * 5)
    uint32_t* d_seg_next64 = nullptr;
    uint2* d_seg_meta64 = nullptr;
    Sample64* d_samp64 = nullptr;
    int* d_job_head64 = nullptr;
    unsigned long long* d_rec64_ctl = nullptr;  // [0] segments taken, [1] samples that ran short, [2] records
    Counters* d_cnt64 = nullptr;
    long long seg_cap64 = 0, job_cap64 = 0, pool64_target = -1;
    double rec_per_sample64 = 320.0;           // pool size per sample (records), doubled after a shortage
    unsigned long long* h_rec64 = nullptr;     // pinned copies of d_rec64_ctl after each wave of the last deferred trace
    cudaEvent_t ev_rec64 = nullptr;
    bool rec64_pending = false;
    std::vector<cudaEvent_t> ev64;             // per wave: recording, sums, emission, replay boundaries (5 each)
    int waves64 = 0;                           // waves of the last deferred trace
    long long samples64 = 0;                   // samples of the last deferred trace (for the estimate)
    bool last_defer64 = false, last_emit64 = false;
    long long list_rays = 0;                   // rays of the last so_trace_rays whose counters d_cnt holds
    std::vector<so_batch*> batches;            // live batches on this renderer (detached by so_destroy)
    std::string err;
};

// Clears the renderer pointer of every live batch of r (so_destroy).
void detach_batches(so_renderer* r);

namespace {

int fail(so_renderer* r, int code, const std::string& msg) {
    if (r) r->err = msg;
    else g_init_error = msg;
    return code;
}
int cuda_fail(so_renderer* r, cudaError_t e, const char* what) {
    return fail(r, SO_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define SO_CK(r, x)                                      \
    do {                                                 \
        cudaError_t e_ = (x);                            \
        if (e_ != cudaSuccess) return cuda_fail(r, e_, #x); \
    } while (0)

template <typename T>
cudaError_t dalloc(T** p, size_t n) {
    return cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
}

int variant_of(const so_scene& S) {
    if (S.mode == SO_MODE_RADIO) return VAR_RADIO;
    if (S.disk_on) return VAR_DISK;
    return VAR_VACUUM;
}

void free_turb_arrays(so_renderer* r) {
    for (int k = 0; k < TURB_NT; ++k) {
        if (r->turb_texo[k]) cudaDestroyTextureObject(r->turb_texo[k]);
        if (r->turb_surf[k]) cudaDestroySurfaceObject(r->turb_surf[k]);
        if (r->turb_arr[k]) cudaFreeArray(r->turb_arr[k]);
        r->turb_texo[k] = 0;
        r->turb_surf[k] = 0;
        r->turb_arr[k] = nullptr;
    }
}

void free_all(so_renderer* r) {
    void* ps[] = {r->d_disk, r->d_k2, r->d_bb, r->d_scene, r->d_frame, r->d_frame_scene, r->d_accum, r->d_img,
                  r->d_chunk_acc, r->d_ystat, r->d_nsamp, r->d_extra, r->d_chunks, r->d_offsets, r->d_total,
                  r->d_tiles, r->d_err, r->d_part, r->d_fsum, r->d_cnt, r->d_x, r->d_y, r->d_rays, r->d_modes};
    for (void* p : ps)
        if (p) cudaFree(p);
    void* pm[] = {r->d_state, r->d_sample_out, r->d_sample_fate, r->d_list32, r->d_list64, r->d_redo, r->d_parked,
                  r->d_nlists, r->d_cnt3, r->d_band, r->d_rec, r->d_rec_delta, r->d_seg_next, r->d_ray_meta,
                  r->d_acc_list, r->d_turb, r->d_esc_list};
    for (void* p : pm)
        if (p) cudaFree(p);
    for (int k = 1; k < r->lev.n; ++k)
        if (r->lev.p[k]) cudaFree(r->lev.p[k]);
    if (r->d_tmp) cudaFree(r->d_tmp);
    for (cudaEvent_t e : r->ev32)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : r->ev_wave)
        if (e) cudaEventDestroy(e);
    if (r->ev_seg) cudaEventDestroy(r->ev_seg);
    if (r->h_seg) cudaFreeHost(r->h_seg);
    void* pl[] = {r->lum.lum, r->lum.part, r->lum.hist, r->lum.stat};
    for (void* p : pl)
        if (p) cudaFree(p);
    if (r->h_lum) cudaFreeHost(r->h_lum);
    void* pc[] = {r->d_cx, r->d_cy, r->d_cth, r->d_cph, r->d_cfate, r->d_uvgrid, r->d_cnt_corner};
    for (void* p : pc)
        if (p) cudaFree(p);
    if (r->sky_tex) cudaDestroyTextureObject(r->sky_tex);
    if (r->sky_mip) cudaFreeMipmappedArray(r->sky_mip);
    delete r->turb_modes;
    if (r->ev_fork) cudaEventDestroy(r->ev_fork);
    if (r->ev_join) cudaEventDestroy(r->ev_join);
    free_turb_arrays(r);
    void* p64[] = {r->d_rec64, r->d_seg_next64, r->d_seg_meta64, r->d_samp64, r->d_job_head64, r->d_rec64_ctl,
                   r->d_cnt64};
    for (void* p : p64)
        if (p) cudaFree(p);
    if (r->h_rec64) cudaFreeHost(r->h_rec64);
    if (r->ev_rec64) cudaEventDestroy(r->ev_rec64);
    for (cudaEvent_t e : r->ev64)
        if (e) cudaEventDestroy(e);
    if (r->st2) cudaStreamDestroy(r->st2);
    if (r->st) cudaStreamDestroy(r->st);
}

constexpr int BAND_N = 2048;

// Critical curve rho_c(psi) of a distant observer at inclination th (critical_curve_point,
// kerr.hpp:210-220, both signs of beta), tabulated on BAND_N image angles psi in [-pi, pi).
std::vector<float> band_table(double a, double th) {
    std::vector<float> out(BAND_N);
    if (a < 1e-4) {  // the 1/a parametrisation degenerates: Schwarzschild circle sqrt(27)
        for (auto& v : out) v = (float)std::sqrt(27.0);
        return out;
    }
    double rp0 = 2.0 * (1.0 + std::cos(2.0 / 3.0 * std::acos(-a))), rp1 = 2.0 * (1.0 + std::cos(2.0 / 3.0 * std::acos(a)));
    std::vector<std::pair<double, double>> pts;
    const int N = 40000;
    for (int i = 0; i <= N; ++i) {
        double rp = rp0 + (rp1 - rp0) * i / N, al, be;
        if (!critical_curve_point(a, th, rp, &al, &be)) continue;
        pts.push_back({std::atan2(be, al), std::hypot(al, be)});
        pts.push_back({std::atan2(-be, al), std::hypot(al, be)});
    }
    if (pts.size() < 4) {
        for (auto& v : out) v = (float)std::sqrt(27.0);
        return out;
    }
    std::sort(pts.begin(), pts.end());
    for (int j = 0; j < BAND_N; ++j) {
        double psi = -PI + 2.0 * PI * j / BAND_N;
        auto it = std::lower_bound(pts.begin(), pts.end(), std::make_pair(psi, -1.0));
        const auto& hi = it == pts.end() ? pts.front() : *it;
        const auto& lo = it == pts.begin() ? pts.back() : *(it - 1);
        double p0 = lo.first, p1 = hi.first;
        if (p1 < p0) p1 += 2.0 * PI;
        double pj = psi < p0 ? psi + 2.0 * PI : psi;
        double f = p1 > p0 ? (pj - p0) / (p1 - p0) : 0.0;
        out[j] = (float)(lo.second + (hi.second - lo.second) * f);
    }
    return out;
}

int upload_scene(so_renderer* r) {
    r->S.disk_lnT = r->d_disk;
    r->S.k2_lntab = r->d_k2;
    r->S.bb_xyz = r->d_bb;
    SO_CK(r, cudaMemcpyAsync(r->d_scene, &r->S, sizeof(so_scene), cudaMemcpyHostToDevice, r->st));
    return SO_OK;
}

// Baked flow turbulence as Renderer::init sets it up (render.cu:594-620): for a radio scene with
// the hot flow and its turbulence, TURB_NT slices over ln R in [ln(0.8 r+), ln(1.05 r_flow_max)],
// z / R within +-min(2, 5 h_r), retarded-time offsets -250 + 260 k / (TURB_NT - 1).  Otherwise (or
// with SO_FLOW_NOISE_INLINE) turb_nt = 0 and the kernels evaluate the sheared noise in place.
// SO_FLOW_NOISE_BAKED keeps the slices as the reference does: 3-D float arrays written through
// surfaces and read through texture objects with its sampler (normalised coordinates, linear
// filtering, phi wrapped, ln R and z / R clamped), whose handles go into so_scene.turb_tex.
// SO_FLOW_NOISE_BAKED_FP32 keeps them in plain device memory for the FP32 trilinear fetch that the
// CPU oracle repeats; turb_tex stays zero then.
int turb_setup(so_renderer* r) {
    so_scene& S = r->S;
    for (int k = 0; k < 24; ++k) S.turb_tex[k] = 0;
    const bool bake = S.flow_on && S.mode == SO_MODE_RADIO && S.flow_turb_amp > 0.f &&
                      (r->flow_noise == SO_FLOW_NOISE_BAKED || r->flow_noise == SO_FLOW_NOISE_BAKED_FP32);
    const bool tex = bake && r->flow_noise == SO_FLOW_NOISE_BAKED;
    if (!bake || tex) {
        if (r->d_turb) cudaFree(r->d_turb);
        r->d_turb = nullptr;
    }
    if (!tex) free_turb_arrays(r);
    if (!bake) {
        S.turb_nt = 0;
        return SO_OK;
    }
    if (tex) {
        cudaChannelFormatDesc fd = cudaCreateChannelDesc<float>();
        for (int k = 0; k < TURB_NT; ++k) {
            if (r->turb_arr[k]) continue;
            if (cudaMalloc3DArray(&r->turb_arr[k], &fd, make_cudaExtent(TURB_NPHI, TURB_NLR, TURB_NZ),
                                  cudaArraySurfaceLoadStore) != cudaSuccess) {
                free_turb_arrays(r);
                return fail(r, SO_ERR_ALLOC, "baked turbulence: 3-D array allocation");
            }
            cudaResourceDesc rd;
            std::memset(&rd, 0, sizeof rd);
            rd.resType = cudaResourceTypeArray;
            rd.res.array.array = r->turb_arr[k];
            cudaTextureDesc td;
            std::memset(&td, 0, sizeof td);
            td.addressMode[0] = cudaAddressModeWrap;
            td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
            td.filterMode = cudaFilterModeLinear;
            td.readMode = cudaReadModeElementType;
            td.normalizedCoords = 1;
            SO_CK(r, cudaCreateSurfaceObject(&r->turb_surf[k], &rd));
            SO_CK(r, cudaCreateTextureObject(&r->turb_texo[k], &rd, &td, nullptr));
        }
        for (int k = 0; k < TURB_NT; ++k) S.turb_tex[k] = (unsigned long long)r->turb_texo[k];
    } else if (!r->d_turb && dalloc(&r->d_turb, (size_t)TURB_NT * TURB_NPHI * TURB_NLR * TURB_NZ) != cudaSuccess) {
        return fail(r, SO_ERR_ALLOC, "baked turbulence: device allocation");
    }
    S.turb_nt = TURB_NT;
    S.turb_lr0 = (float)std::log(0.8 * S.rh);
    S.turb_lr1 = (float)std::log(S.r_flow_max * 1.05);
    S.turb_zmax = (float)std::min(2.0, 5.0 * S.h_r);
    S.turb_d0 = -250.f;
    S.turb_dd = 260.f / (TURB_NT - 1);
    for (int k = 0; k < TURB_NT; ++k) r->tb.delta[k] = S.turb_d0 + k * S.turb_dd;
    return SO_OK;
}

// The frame's bake (k_bake_turb): into the 3-D arrays (texture fetch) or the plain slices (FP32
// fetch, passed to the tracers as L.turb_field).
int bake_turbulence(so_renderer* r, TraceLaunch& L) {
    if (r->S.turb_nt <= 0) return SO_OK;
    if (r->turb_arr[0]) {
        SurfaceSet ss;
        for (int k = 0; k < TURB_NT; ++k) ss.s[k] = r->turb_surf[k];
        SO_CK(r, launch_bake_turb_surf(r->d_scene, r->d_frame, r->tb, ss, r->st));
        L.turb_field = nullptr;
        return SO_OK;
    }
    if (!r->d_turb) return SO_OK;
    SO_CK(r, launch_bake_turb(r->d_scene, r->d_frame, r->tb, r->d_turb, r->st));
    L.turb_field = r->d_turb;
    return SO_OK;
}

// Fills the plasma / precision part of a launch descriptor.
void launch_common(so_renderer* r, TraceLaunch& L) {
    std::memset(&L, 0, sizeof L);
    L.scenes = r->d_scene;
    L.frames = r->d_frame;
    L.frame_scene = r->d_frame_scene;
    L.nframes = 1;
    L.counters = r->d_cnt;
    const so_plasma& p = r->plasma;
    L.torus = p.model == SO_PLASMA_TORUS;
    L.n_modes = L.torus ? p.n_modes : 0;
    L.ne_index = p.ne_index;
    L.te_index = p.te_index;
    L.h_sph = p.h_sph;
    L.theta_e0 = 1.380649e-16 * p.te0_kelvin / (9.1093837e-28 * 2.99792458e10 * 2.99792458e10);
    L.half_var = 0.5 * p.turb_rms * p.turb_rms;
    L.modes = r->d_modes;
    L.band_m = r->mixed.band_m;
    L.tol32 = r->mixed.tol32;
    L.turn_r = r->mixed.turn_r;
    L.drift_tol = r->mixed.drift_tol;
}

// Buffers of the device luminance statistics (allocated on the first so_render).
int ensure_lum(so_renderer* r) {
    if (r->lum.lum) return SO_OK;
    if (dalloc(&r->lum.lum, (size_t)r->npix) != cudaSuccess || dalloc(&r->lum.part, LUM_BLOCKS) != cudaSuccess ||
        dalloc(&r->lum.hist, LUM_HIST) != cudaSuccess || dalloc(&r->lum.stat, 1) != cudaSuccess)
        return fail(r, SO_ERR_ALLOC, "luminance statistics: device allocation");
    SO_CK(r, cudaMallocHost((void**)&r->h_lum, sizeof(LumStat)));
    return SO_OK;
}

// Pyramid of the frame for the post filters, level sizes as the reference's (render.cu:638-647).
int ensure_post(so_renderer* r) {
    if (r->lev.n) return SO_OK;
    int w = r->rs.W, h = r->rs.H, n = 0;
    PostLevels L{};
    while (n < POST_MAX_LEVELS && w >= 2 && h >= 2) {
        L.w[n] = w;
        L.h[n] = h;
        if (n == 0) L.p[0] = r->d_img;
        else if (dalloc(&L.p[n], (size_t)w * h) != cudaSuccess) {
            for (int k = 1; k < n; ++k) cudaFree(L.p[k]);
            return fail(r, SO_ERR_ALLOC, "post filters: pyramid allocation");
        }
        ++n;
        w = (w + 1) / 2;
        h = (h + 1) / 2;
    }
    if (dalloc(&r->d_tmp, (size_t)r->npix) != cudaSuccess) {
        for (int k = 1; k < n; ++k) cudaFree(L.p[k]);
        return fail(r, SO_ERR_ALLOC, "post filters: scratch allocation");
    }
    L.n = n;
    r->lev = L;
    return SO_OK;
}

// The second queue: a stream, its fork / join events and the queue heads of launches made on it.
int ensure_side_queue(so_renderer* r) {
    if (!r->d_cnt3 && dalloc(&r->d_cnt3, 2) != cudaSuccess) return fail(r, SO_ERR_ALLOC, "second queue: allocation");
    if (!r->st2) SO_CK(r, cudaStreamCreateWithFlags(&r->st2, cudaStreamNonBlocking));
    if (!r->ev_fork) SO_CK(r, cudaEventCreateWithFlags(&r->ev_fork, cudaEventDisableTiming));
    if (!r->ev_join) SO_CK(r, cudaEventCreateWithFlags(&r->ev_join, cudaEventDisableTiming));
    return SO_OK;
}

// Record pool of the deferred FP64 passes for `jobs` tracer jobs of `per_job` samples, records of
// `w` doubles: rec_per_sample64 records per sample plus one partly filled segment per sample, within
// half of the free device memory and so_mixed_opts.pool_mb.  A launch the pool cannot hold at once
// runs in waves of *wave_jobs jobs (at most kMaxWaves64); where even that would leave waves too
// small to fill the GPU, it runs as one wave and the samples that do not fit are left to the replay
// pass (the same result, slower).  A shortage doubles the estimate for the next traces.
constexpr int kMaxWaves64 = 64;
constexpr long long kDeferMinJobs = 4096;
int ensure_records64(so_renderer* r, long long jobs, int per_job, int w, long long* wave_jobs) {
    if (!r->h_rec64) {
        SO_CK(r, cudaMallocHost((void**)&r->h_rec64, 3 * kMaxWaves64 * sizeof(unsigned long long)));
        std::memset(r->h_rec64, 0, 3 * kMaxWaves64 * sizeof(unsigned long long));
        SO_CK(r, cudaEventCreateWithFlags(&r->ev_rec64, cudaEventDisableTiming));
    }
    if (!r->d_rec64_ctl && dalloc(&r->d_rec64_ctl, 3) != cudaSuccess)
        return fail(r, SO_ERR_ALLOC, "FP64 record pool: allocation");
    if (!r->d_cnt64 && dalloc(&r->d_cnt64, 1) != cudaSuccess) return fail(r, SO_ERR_ALLOC, "FP64 record pool: allocation");
    if (r->rec64_pending && cudaEventQuery(r->ev_rec64) == cudaSuccess) {
        // the last deferred trace's records per sample, with a margin; doubled after a shortage
        r->rec64_pending = false;
        unsigned long long short_samples = 0, records = 0;
        for (int k = 0; k < r->waves64; ++k) {
            short_samples += r->h_rec64[3 * k + 1];
            records += r->h_rec64[3 * k + 2];
        }
        const double seen = r->samples64 > 0 ? 1.5 * (double)records / (double)r->samples64 : 0.0;
        r->rec_per_sample64 = std::max(short_samples > 0 ? 2.0 * r->rec_per_sample64 : r->rec_per_sample64, seen);
    }
    cudaGetLastError();  // a pending event reports cudaErrorNotReady
    const double seg_doubles = (double)REC_SEG * w;
    const double per_seg = seg_doubles * sizeof(double) + sizeof(uint32_t) + sizeof(uint2);
    const double seg_per_job = (r->rec_per_sample64 / REC_SEG + 1.0) * per_job;  // a partly filled segment per sample
    long long want = std::min<long long>((long long)std::ceil((double)jobs * seg_per_job), 0x7fffffffll);
    if (r->mixed.pool_mb > 0.0)
        want = std::min<long long>(want, std::max<long long>(1, (long long)(r->mixed.pool_mb * 1048576.0 / per_seg)));
    const long long want_d = (long long)(want * seg_doubles);
    if (r->rec64_doubles <= 0 || want_d > r->pool64_target ||
        (r->mixed.pool_mb > 0.0 && want_d < r->rec64_doubles)) {
        SO_CK(r, cudaStreamSynchronize(r->st));
        if (r->d_rec64) cudaFree(r->d_rec64);
        if (r->d_seg_next64) cudaFree(r->d_seg_next64);
        if (r->d_seg_meta64) cudaFree(r->d_seg_meta64);
        r->d_rec64 = nullptr;
        r->d_seg_next64 = nullptr;
        r->d_seg_meta64 = nullptr;
        r->rec64_doubles = 0;
        r->pool64_target = -1;
        size_t fr = 0, tot = 0;
        SO_CK(r, cudaMemGetInfo(&fr, &tot));
        // segment arrays sized for the narrowest record (REC64_W_TORUS doubles)
        const double per_double = sizeof(double) + (sizeof(uint32_t) + sizeof(uint2)) / (double)(REC_SEG * REC64_W_TORUS);
        const long long cap_d = std::min<long long>(want_d, (long long)(0.5 * (double)fr / per_double));
        const long long nseg = cap_d / (REC_SEG * REC64_W_TORUS);
        if (nseg < 1) return fail(r, SO_ERR_ALLOC, "FP64 record pool: no device memory");
        if (dalloc(&r->d_rec64, (size_t)cap_d) != cudaSuccess || dalloc(&r->d_seg_next64, (size_t)nseg) != cudaSuccess ||
            dalloc(&r->d_seg_meta64, (size_t)nseg) != cudaSuccess)
            return fail(r, SO_ERR_ALLOC, "FP64 record pool: device allocation");
        r->rec64_doubles = cap_d;
        r->pool64_target = want_d;
    }
    r->seg_cap64 = std::min<long long>(r->rec64_doubles / (REC_SEG * w), 0x7fffffffll);
    if (r->seg_cap64 < 1) return fail(r, SO_ERR_ALLOC, "FP64 record pool: no segment");
    long long wave = jobs;
    if ((double)r->seg_cap64 < (double)jobs * seg_per_job) {
        wave = (long long)((double)r->seg_cap64 / seg_per_job);
        const long long min_wave = std::max<long long>(kDeferMinJobs, (jobs + kMaxWaves64 - 1) / kMaxWaves64);
        if (wave < min_wave) wave = jobs;  // one wave; what does not fit goes to the replay pass
    }
    *wave_jobs = wave;
    const long long heads = wave * per_job;  // one chain per sample
    if (heads > r->job_cap64) {
        if (r->d_job_head64) cudaFree(r->d_job_head64);
        if (r->d_samp64) cudaFree(r->d_samp64);
        r->d_job_head64 = nullptr;
        r->d_samp64 = nullptr;
        r->job_cap64 = 0;
        if (dalloc(&r->d_job_head64, (size_t)heads) != cudaSuccess || dalloc(&r->d_samp64, (size_t)heads) != cudaSuccess)
            return fail(r, SO_ERR_ALLOC, "FP64 record pool: chain heads");
        r->job_cap64 = heads;
    }
    return SO_OK;
}

// Launches of the FP64 tracer.  A launch of at least kDeferMinJobs host-counted jobs on the
// renderer's stream defers work out of the tracer when it is a torus-plasma launch with FP64 sums,
// or a launch on the reference flow model: a recording pass (geometry only, one record per flow
// step that can emit) -> k_turb64_records (torus: the FP64 sums at every record) -> without a disk,
// k_emit64_records (flow_step at every record) -> k_transfer64 (ordered transfer; a ray list's ray
// cut on its opacity gets the fate, counts and crossings of the cut step from its record), with a
// replay pass behind them that runs only if the pool ran short; for torus disk scenes the replay
// pass instead of the emission kernels.  Each is bit for bit the in-tracer result, with the sums and
// the emission at full occupancy.  Everything else, and any launch whose pool cannot be had, runs
// in the tracer.
// The deferred passes of one launch on stream s, in waves of `wave` jobs through the pool that
// ensure_records64 set up: per wave a recording pass, the sums (sums: 0 none, 1 FP64, 2 FP32), the
// emission and ordered transfer (emit), and a replay pass that runs when the pool ran short (always,
// without emit).  With `timed` the phases are bracketed by events (not inside a graph capture).
// Each wave's pool counters go to h_rec64 for the shortage feedback and the statistics.
int enqueue_deferred64(so_renderer* r, const TraceLaunch& L, int var, cudaStream_t s, long long wave, int w, int sums,
                       bool emit, bool timed) {
    const int nw = (int)((L.nrays + wave - 1) / wave);
    if (nw > kMaxWaves64) return fail(r, SO_ERR_SIZE, "FP64 record pool: too many waves");
    if (timed) {
        while ((int)r->ev64.size() < 5 * nw) {
            cudaEvent_t e = nullptr;
            SO_CK(r, cudaEventCreate(&e));
            r->ev64.push_back(e);
        }
    }
    for (int k = 0; k < nw; ++k) {
        const long long j0 = (long long)k * wave;
        SO_CK(r, cudaMemsetAsync(r->d_rec64_ctl, 0, 3 * sizeof(unsigned long long), s));
        SO_CK(r, cudaMemsetAsync(r->d_cnt64, 0, sizeof(Counters), s));
        TraceLaunch L1 = L;
        L1.defer64 = 1;
        L1.emit32 = 0;
        L1.counters = r->d_cnt64;
        L1.rec64 = r->d_rec64;
        L1.rec64_w = w;
        L1.job0 = j0;
        L1.nrays = std::min<long long>(wave, L.nrays - j0);
        L1.seg_next64 = r->d_seg_next64;
        L1.seg_meta64 = r->d_seg_meta64;
        L1.samp64 = r->d_samp64;
        L1.job_head64 = r->d_job_head64;
        L1.seg_cap64 = r->seg_cap64;
        L1.rec64_ctl = r->d_rec64_ctl;
        TraceLaunch L2 = L1;
        L2.defer64 = 2;
        L2.counters = L.counters;
        L2.replay_if_short = emit ? 1 : 0;
        L2.emit32 = 0;
        cudaEvent_t* ev = timed ? &r->ev64[5 * k] : nullptr;
        if (ev) cudaEventRecord(ev[0], s);
        cudaError_t e = launch_trace64(L1, var, r->num_sms, s);
        if (e != cudaSuccess) return cuda_fail(r, e, "tracer launch (recording pass)");
        if (ev) cudaEventRecord(ev[1], s);
        if (sums == 1) e = launch_turb64_records(L1, r->num_sms, s);
        else if (sums == 2) e = launch_turb32_rec64(L1, *r->turb_modes, r->num_sms, s);
        if (e != cudaSuccess) return cuda_fail(r, e, "deferred turbulence sums");
        if (ev) cudaEventRecord(ev[2], s);
        if (emit) {
            TraceLaunch Le = L1;
            Le.counters = L.counters;
            e = launch_emit64_records(Le, r->num_sms, s);
            if (e != cudaSuccess) return cuda_fail(r, e, "FP64 deferred emission");
            e = launch_transfer64(Le, r->num_sms, s);
            if (e != cudaSuccess) return cuda_fail(r, e, "FP64 ordered transfer");
        }
        if (ev) cudaEventRecord(ev[3], s);
        // the replay pass's queue starts at the wave's first job (it reads each recorded sum back,
        // whichever form summed it, and sums the samples the pool could not hold in FP64)
        SO_CK(r, cudaMemsetAsync(&L.counters->next, 0, sizeof(unsigned long long), s));
        e = launch_trace64(L2, var, r->num_sms, s);
        if (e != cudaSuccess) return cuda_fail(r, e, "tracer launch (replay pass)");
        if (ev) cudaEventRecord(ev[4], s);
        SO_CK(r, cudaMemcpyAsync(r->h_rec64 + 3 * k, r->d_rec64_ctl, 3 * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, s));
    }
    r->waves64 = nw;
    return SO_OK;
}

int run_tracer(so_renderer* r, const TraceLaunch& L, cudaStream_t st = nullptr) {
    const int var = variant_of(r->S);
    const cudaStream_t s = st ? st : r->st;
    const bool torus = var == VAR_RADIO && L.torus && L.n_modes > 0;
    const bool emit_ok = !r->S.disk_on && r->S.max_steps < (1 << REC64_COUNT_BITS);
    const bool flow = var == VAR_RADIO && !torus && r->S.flow_on && emit_ok;
    const bool defer = ((torus && !L.emit32) || flow) && !L.nrays_dev && L.nrays >= kDeferMinJobs && s == r->st;
    r->last_defer64 = false;
    if (defer) {
        const int per_job = L.kind == RAYS_PIXELS ? L.spp : L.kind == RAYS_CHUNKS ? L.chunk : 1;
        const int w = (torus ? REC64_W_TORUS : REC64_W_FLOW) + (L.kind == RAYS_LIST ? 1 : 0);
        long long wave = 0;
        if (ensure_records64(r, L.nrays, per_job, w, &wave) == SO_OK) {
            r->samples64 = L.nrays * per_job;
            if (int rc = enqueue_deferred64(r, L, var, s, wave, w, torus ? 1 : 0, emit_ok, true)) return rc;
            SO_CK(r, cudaEventRecord(r->ev_rec64, s));
            r->rec64_pending = true;
            r->last_defer64 = true;
            r->last_emit64 = emit_ok;
            return SO_OK;
        }
        r->err.clear();  // no pool: run in the tracer
    }
    cudaError_t e = launch_trace64(L, var, r->num_sms, s);
    if (e != cudaSuccess) return cuda_fail(r, e, "tracer launch");
    return SO_OK;
}

// Escape (u, v) of the (W + 1) x (H + 1) pixel corners of the frame in d_frame (k_corners,
// render.cu:40-52, 686-691): the corner rays through the tracer's ray list (own counters), then
// sky_uv of those that escape.  Gives the pixel footprints for the star-map filtering.
int trace_corners(so_renderer* r, int W, int H) {
    const long long n = (long long)(W + 1) * (H + 1);
    if (n > r->corner_cap) {
        void* pc[] = {r->d_cx, r->d_cy, r->d_cth, r->d_cph, r->d_cfate, r->d_uvgrid};
        for (void* p : pc)
            if (p) cudaFree(p);
        r->d_cx = r->d_cy = r->d_cth = r->d_cph = nullptr;
        r->d_cfate = nullptr;
        r->d_uvgrid = nullptr;
        r->corner_cap = 0;
        if (dalloc(&r->d_cx, (size_t)n) != cudaSuccess || dalloc(&r->d_cy, (size_t)n) != cudaSuccess ||
            dalloc(&r->d_cth, (size_t)n) != cudaSuccess || dalloc(&r->d_cph, (size_t)n) != cudaSuccess ||
            dalloc(&r->d_cfate, (size_t)n) != cudaSuccess || dalloc(&r->d_uvgrid, (size_t)n) != cudaSuccess)
            return fail(r, SO_ERR_ALLOC, "sky corners: device allocation");
        r->corner_cap = n;
    }
    if (!r->d_cnt_corner && dalloc(&r->d_cnt_corner, 1) != cudaSuccess)
        return fail(r, SO_ERR_ALLOC, "sky corners: device allocation");
    SO_CK(r, cudaMemsetAsync(r->d_cnt_corner, 0, sizeof(Counters), r->st));
    SO_CK(r, launch_corner_points(r->d_frame, W, H, r->d_cx, r->d_cy, r->st));
    TraceLaunch L;
    launch_common(r, L);
    L.counters = r->d_cnt_corner;
    L.kind = RAYS_LIST;
    L.nrays = n;
    L.x = r->d_cx;
    L.y = r->d_cy;
    L.out.fate = r->d_cfate;
    L.out.theta = r->d_cth;
    L.out.phi = r->d_cph;
    int rc = run_tracer(r, L);
    if (rc) return rc;
    SO_CK(r, launch_corner_uv(r->d_scene, n, r->d_cfate, r->d_cth, r->d_cph, r->d_uvgrid, r->st));
    return SO_OK;
}

// Attempts the reference's Mino-time integrator (trace.cuh:80-96, with its disk step cap) takes for
// the frame's central ray from the camera down to r_sw.  Rays that far_approach brings to r_sw are
// credited with this count, so that the max_steps limit of the FP32 tracer counts about the
// reference's steps for the whole ray.
int mino_approach_attempts(const so_scene& S, const so_frame& F, double r_sw) {
    RayC c;
    double y[6], k1[6], yn[6], k7[6];
    camera_photon(S.a, F.kp, F.ph, F.t, view_dir(F, 0.0, 0.0), F.beta, c, y);
    rhs(c, y, k1);
    double h = initial_step(y);
    int it = 0;
    while (it < S.max_steps && y[0] >= r_sw) {
        ++it;
        double hc = h;
        if (S.disk_on) hc = std::fmin(hc, 0.3 / (std::fabs(y[3]) + 1e-30));
        double err = dp54(c, y, k1, hc, S.tol, yn, k7);
        if (!(err <= 1.0)) {
            h = reject_step(hc, err);
            continue;
        }
        for (int i = 0; i < 6; ++i) {
            y[i] = yn[i];
            k1[i] = k7[i];
        }
        project_radial(c, y, k1);
        h = accept_step(hc, err);
        if (y[0] > S.r_escape && y[1] > 0.0) break;
    }
    return it;
}

// Record pool of the deferred turbulence for ns FP32 rays: rec_per_ray records per ray on average
// plus one partly filled segment per ray, within half of the free device memory.  A frame that ran
// short (its rays re-traced in FP64, so still correct) doubles rec_per_ray for the next frames; the
// shortage is read from the previous frame's counters once they have arrived (no wait here).
int ensure_records(so_renderer* r, long long ns) {
    if (!r->h_seg) {
        SO_CK(r, cudaMallocHost((void**)&r->h_seg, 2 * sizeof(unsigned long long)));
        r->h_seg[0] = r->h_seg[1] = 0;
        SO_CK(r, cudaEventCreateWithFlags(&r->ev_seg, cudaEventDisableTiming));
    }
    if (r->seg_pending && cudaEventQuery(r->ev_seg) == cudaSuccess) {
        r->seg_pending = false;
        if (r->h_seg[1] > 0) r->rec_per_ray *= 2.0;
    }
    cudaGetLastError();  // a pending event reports cudaErrorNotReady
    const double per_seg = REC_SEG * (sizeof(float4) + sizeof(float)) + sizeof(uint32_t);
    const double seg_per_ray = r->rec_per_ray / REC_SEG + 1.0;  // with the partly filled last segment
    long long want = std::min<long long>((long long)std::ceil((double)ns * seg_per_ray), 0x7fffffffll);
    if (r->mixed.pool_mb > 0.0)
        want = std::min<long long>(want, std::max<long long>(1, (long long)(r->mixed.pool_mb * 1048576.0 / per_seg)));
    // grow to a larger estimate; shrink only to a lowered cap; retry after a failed allocation
    if (r->seg_cap <= 0 || want > r->pool_target || (r->mixed.pool_mb > 0.0 && want < r->seg_cap)) {
        SO_CK(r, cudaStreamSynchronize(r->st));
        if (r->d_rec) cudaFree(r->d_rec);
        if (r->d_rec_delta) cudaFree(r->d_rec_delta);
        if (r->d_seg_next) cudaFree(r->d_seg_next);
        r->d_rec = nullptr;
        r->d_rec_delta = nullptr;
        r->d_seg_next = nullptr;
        r->seg_cap = 0;
        r->pool_target = -1;
        size_t fr = 0, tot = 0;
        SO_CK(r, cudaMemGetInfo(&fr, &tot));
        const long long cap = std::min<long long>(want, (long long)(0.5 * (double)fr / per_seg));
        if (cap < 1) return fail(r, SO_ERR_ALLOC, "record pool: no device memory");
        if (dalloc(&r->d_rec, (size_t)cap * REC_SEG) != cudaSuccess ||
            dalloc(&r->d_rec_delta, (size_t)cap * REC_SEG) != cudaSuccess ||
            dalloc(&r->d_seg_next, (size_t)cap) != cudaSuccess)
            return fail(r, SO_ERR_ALLOC, "record pool: device allocation");
        r->seg_cap = cap;
        r->pool_target = want;
    }
    // waves of FP32 rays whose expected records fit the pool (at most 64)
    const long long per_wave = std::max<long long>(1, (long long)((double)r->seg_cap / seg_per_ray));
    r->waves = (int)std::min<long long>(64, (ns + per_wave - 1) / per_wave);
    r->wave_rays = (ns + r->waves - 1) / r->waves;
    while ((int)r->ev_wave.size() < 3 * r->waves) {
        cudaEvent_t e;
        SO_CK(r, cudaEventCreate(&e));
        r->ev_wave.push_back(e);
    }
    if (ns > r->meta_cap) {
        if (r->d_ray_meta) cudaFree(r->d_ray_meta);
        if (r->d_acc_list) cudaFree(r->d_acc_list);
        r->d_ray_meta = nullptr;
        r->d_acc_list = nullptr;
        r->meta_cap = 0;
        if (dalloc(&r->d_ray_meta, (size_t)ns) != cudaSuccess || dalloc(&r->d_acc_list, (size_t)ns) != cudaSuccess)
            return fail(r, SO_ERR_ALLOC, "record lists: device allocation");
        r->meta_cap = ns;
    }
    return SO_OK;
}

// Pass 1 of the mixed path into d_accum / d_ystat (see k_trace_mixed.cu):
//   route (band / FP32 lists) -> FP64 approach to r_switch -> FP32 tracer [-> turbulence sums ->
//   ordered transfer], with the band list traced by the FP64 tracer on a second stream meanwhile and
//   the FP64 re-trace list after it on that stream once the FP32 tracer has made the list, then the
//   per-pixel gather of the samples.  Counts stay on the device: nothing waits on the host.
int trace_pass1_mixed(so_renderer* r, const so_frame& f, TraceLaunch& L) {
    const long long ns = (long long)f.W * f.H * f.spp;
    r->last_mixed_ns = 0;
    if (ns > 0xffffffffll) return fail(r, SO_ERR_SIZE, "mixed path: more than 2^32 samples per frame");
    if (ns > r->mixed_cap) {
        void* pm[] = {r->d_state, r->d_sample_out, r->d_sample_fate, r->d_list32, r->d_list64, r->d_redo, r->d_parked};
        for (void* p : pm)
            if (p) cudaFree(p);
        r->d_state = r->d_sample_out = nullptr;
        r->d_sample_fate = nullptr;
        r->d_list32 = r->d_list64 = r->d_redo = r->d_parked = nullptr;
        r->mixed_cap = 0;
        if (dalloc(&r->d_state, (size_t)ns * 5) != cudaSuccess || dalloc(&r->d_sample_out, (size_t)ns) != cudaSuccess ||
            dalloc(&r->d_sample_fate, (size_t)ns) != cudaSuccess || dalloc(&r->d_list32, (size_t)ns) != cudaSuccess ||
            dalloc(&r->d_list64, (size_t)ns) != cudaSuccess || dalloc(&r->d_redo, (size_t)ns) != cudaSuccess ||
            dalloc(&r->d_parked, (size_t)ns) != cudaSuccess)
            return fail(r, SO_ERR_ALLOC, "mixed path: device allocation");
        r->mixed_cap = ns;
    }
    if (!r->d_nlists) {
        if (dalloc(&r->d_nlists, NLISTS) != cudaSuccess || (!r->d_band && dalloc(&r->d_band, BAND_N) != cudaSuccess))
            return fail(r, SO_ERR_ALLOC, "mixed path: device allocation");
        if (int rc = ensure_side_queue(r)) return rc;
        SO_CK(r, cudaEventCreate(&r->ev32[0]));
        SO_CK(r, cudaEventCreate(&r->ev32[1]));
    }
    if (r->band_a != r->S.a || r->band_th != f.th) {
        std::vector<float> tab = band_table(r->S.a, f.th);
        SO_CK(r, cudaMemcpyAsync(r->d_band, tab.data(), BAND_N * sizeof(float), cudaMemcpyHostToDevice, r->st));
        SO_CK(r, cudaStreamSynchronize(r->st));
        r->band_a = r->S.a;
        r->band_th = f.th;
    }
    double rsw = r->mixed.r_switch;
    if (!(rsw > 0.0)) {
        rsw = 100.0;
        if (r->S.flow_on) rsw = std::max(rsw, 1.5 * r->S.r_flow_max);
        if (r->S.disk_on) rsw = std::max(rsw, 1.2 * r->S.disk_rout);
    }
    L.r_switch = rsw;
    L.tol_approach = r->mixed.tol_approach > 0.0 ? r->mixed.tol_approach : 10.0 * r->S.tol;
    L.far_field = r->mixed.approach == 0 ? 1 : 0;
    const double key[6] = {r->S.a, r->S.tol, (double)r->S.disk_on, rsw, f.r, f.th};
    if (std::memcmp(key, r->approach_key, sizeof key) != 0) {
        r->approach_it = mino_approach_attempts(r->S, f, rsw);
        std::memcpy(r->approach_key, key, sizeof key);
    }
    L.approach_it = r->approach_it;
    L.t32_min_blocks = r->mixed.t32_blocks > 0 ? r->mixed.t32_blocks : 4;
    L.t32_max_att = r->mixed.fp32_max_attempts > 0 ? r->mixed.fp32_max_attempts : 2000;
    // outgoing rays beyond every emitter cannot come back: the FP32 tracer ends them as escaped
    double r_emit = 0.0;
    if (r->S.mode == SO_MODE_RADIO && r->S.flow_on) r_emit = std::max(r_emit, r->S.r_flow_max);
    if (r->S.disk_on) r_emit = std::max(r_emit, r->S.disk_rout);
    // star-map frames: escaping FP32 rays stop there and k_sky_escape carries them on in FP64
    const bool sky = L.sky_uv != nullptr && r->mixed.sky_fp32 != 0;
    if (sky) r_emit = std::max(r_emit, 10.0);
    L.r_emit = r_emit > 0.0 ? std::max(r_emit, 10.0) : 0.0;
    if (sky) {
        if (!r->d_esc_list || r->esc_cap < ns) {
            if (r->d_esc_list) cudaFree(r->d_esc_list);
            r->d_esc_list = nullptr;
            r->esc_cap = 0;
            if (dalloc(&r->d_esc_list, (size_t)ns) != cudaSuccess) return fail(r, SO_ERR_ALLOC, "sky escape list");
            r->esc_cap = ns;
        }
        L.esc_list = r->d_esc_list;
    }
    L.band_rho = r->d_band;
    L.band_n = BAND_N;
    L.nsamples = ns;
    L.state = r->d_state;
    L.sample_out = r->d_sample_out;
    L.sample_fate = r->d_sample_fate;
    L.list32 = r->d_list32;
    L.list64 = r->d_list64;
    L.redo = r->d_redo;
    L.parked = r->d_parked;
    L.nlists = r->d_nlists;
    SO_CK(r, cudaMemsetAsync(r->d_nlists, 0, NLISTS * sizeof(unsigned long long), r->st));
    SO_CK(r, cudaMemsetAsync(r->d_cnt3, 0, 2 * sizeof(Counters), r->st));
    // The reference's sheared fBm turbulence (flow or disk) evaluated in place uses a noise generation
    // k = floor(t / P) of the raw coordinate time t ~ -r_cam: a relative change eps of the radius moves
    // its phase by ~ (t / P) eps, so any integrator that is not the FP64 one decorrelates it.  Such
    // scenes, and radio scenes with a disk (not in the FP32 tracer), go to FP64 entirely.  A baked
    // flow field (turb_nt > 0) is sampled at the position and at t - t_ref(r), both well conditioned,
    // so the FP32 tracer takes those scenes.
    const bool all64 = (r->S.mode == SO_MODE_RADIO && r->S.flow_on && L.torus == 0 && r->S.flow_turb_amp > 0.f &&
                        r->S.turb_nt <= 0) ||
                       (L.sky_uv != nullptr && r->mixed.sky_fp32 == 0) ||  // star map: FP64 unless asked
                       (r->S.disk_on && r->S.disk_turb_amp > 0.f) || (r->S.mode == SO_MODE_RADIO && r->S.disk_on);
    SO_CK(r, launch_route(L, all64 ? 1 : 0, r->st));
    // band rays: plain FP64 tracer on the second stream, concurrently with the FP32 work
    SO_CK(r, cudaEventRecord(r->ev_fork, r->st));
    SO_CK(r, cudaStreamWaitEvent(r->st2, r->ev_fork, 0));
    TraceLaunch Lb = L;
    Lb.kind = RAYS_SAMPLES;
    Lb.list = r->d_list64;
    Lb.nrays = ns;
    Lb.nrays_dev = &r->d_nlists[1];
    Lb.counters = &r->d_cnt3[0];
    Lb.emit32 = 1;  // FP64 geometry in the band; the emission needs no more than FP32
    // The band and the re-trace take one CTA per SM, two when their rays carry the torus's
    // warp-cooperative turbulence sums (throughput work that more warps serve); otherwise their
    // rays are long latency-bound chains, and the full persistent grid (three 168-register CTAs,
    // every SM's register file) held the FP32 tracer off those SMs.  Measured, three / two / one
    // CTAs per SM: the reference flow frame at 1024^2 72.0 / 71.3 / 67.5 ms, the synchrotron frame
    // at 2048^2 210.3 / 207.4 / 210.3 ms, the vacuum shadow frame at 2048^2 one CTA 122.5 Mrays/s
    // against 119.8 with two; the images identical.
    Lb.ctas_per_sm = (L.torus && L.n_modes > 0) ? 2 : 1;
    int rc = run_tracer(r, Lb, r->st2);
    if (rc) return rc;
    const bool torus_defer = variant_of(r->S) == VAR_RADIO && L.torus && L.n_modes > 0;
    const bool flow_defer = variant_of(r->S) == VAR_RADIO && !L.torus && r->S.flow_on && !all64;
    const bool defer = (torus_defer || flow_defer) && r->mixed.turbulence == 0;
    L.defer = defer ? 1 : 0;
    if (defer) {
        rc = ensure_records(r, ns);
        if (rc) return rc;
        L.rec = r->d_rec;
        L.rec_delta = r->d_rec_delta;
        L.seg_next = r->d_seg_next;
        L.ray_meta = r->d_ray_meta;
        L.acc_list = r->d_acc_list;
        L.seg_cap = r->seg_cap;
    }
    SO_CK(r, launch_approach64(L, ns, r->num_sms, r->st));
    SO_CK(r, cudaEventRecord(r->ev32[0], r->st));
    // Deferred turbulence with a pool that holds only part of the frame's records: the parked FP32
    // rays are traced in waves (slices of the parked list), each wave's records summed and
    // transferred before the next wave reuses the pool.  Every ray's result depends on the ray alone,
    // so the image does not depend on the split.
    const int waves = defer ? r->waves : 1;
    for (int w = 0; w < waves; ++w) {
        TraceLaunch Lw = L;
        if (waves > 1) {
            Lw.wave_begin = (long long)w * r->wave_rays;
            Lw.wave_end = (long long)(w + 1) * r->wave_rays;
        }
        if (w > 0) {
            // tracer work counter; pool segments, accepted-ray list and the sums' work counters
            SO_CK(r, cudaMemsetAsync(&r->d_cnt->next, 0, sizeof(unsigned long long), r->st));
            SO_CK(r, cudaMemsetAsync(&r->d_nlists[4], 0, 2 * sizeof(unsigned long long), r->st));
            SO_CK(r, cudaMemsetAsync(&r->d_nlists[7], 0, 2 * sizeof(unsigned long long), r->st));
        }
        if (defer) SO_CK(r, cudaEventRecord(r->ev_wave[3 * w], r->st));
        SO_CK(r, launch_trace32(Lw, ns, variant_of(r->S), r->num_sms, r->st));
        if (w == waves - 1) {
            // FP64 re-trace of the rays the FP32 tracer handed back, on the second stream (after the band)
            SO_CK(r, cudaEventRecord(r->ev_fork, r->st));
            SO_CK(r, cudaStreamWaitEvent(r->st2, r->ev_fork, 0));
            TraceLaunch Lr = Lb;
            Lr.list = r->d_redo;
            Lr.nrays_dev = &r->d_nlists[2];
            Lr.counters = &r->d_cnt3[1];
            rc = run_tracer(r, Lr, r->st2);
            if (rc) return rc;
            SO_CK(r, cudaEventRecord(r->ev_join, r->st2));
        }
        if (defer) {
            SO_CK(r, cudaEventRecord(r->ev_wave[3 * w + 1], r->st));
            if (torus_defer) SO_CK(r, launch_turb_records(Lw, *r->turb_modes, r->num_sms, r->st));
            SO_CK(r, cudaEventRecord(r->ev_wave[3 * w + 2], r->st));
            SO_CK(r, launch_flow_records(Lw, r->num_sms, r->st));
        }
    }
    if (defer) {
        SO_CK(r, cudaMemcpyAsync(r->h_seg, &r->d_nlists[5], 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                 r->st));
        SO_CK(r, cudaEventRecord(r->ev_seg, r->st));
        r->seg_pending = true;
    }
    r->last_defer = defer;
    r->last_waves = waves;
    if (sky) SO_CK(r, launch_sky_escape(L, r->num_sms, r->st));
    SO_CK(r, cudaEventRecord(r->ev32[1], r->st));
    SO_CK(r, cudaStreamWaitEvent(r->st, r->ev_join, 0));
    SO_CK(r, launch_gather_samples(L, r->st));
    r->last_mixed_ns = ns;
    return SO_OK;
}

// The deferred FP64 passes' fields of so_stats for the last tracer launch (its stream synchronised).
void rec64_stats(so_renderer* r, so_stats* stats) {
    stats->ms_rec64 = stats->ms_sum64 = stats->ms_replay64 = stats->ms_emit64 = 0.0;
    stats->rec64_slots = stats->rec64_short = stats->rec64_records = 0;
    stats->emit64 = 0;
    stats->rec64_waves = 0;
    if (!r->last_defer64) return;
    unsigned long long slots = 0, short_samples = 0, records = 0;
    for (int k = 0; k < r->waves64; ++k) {
        float t[4] = {0.f, 0.f, 0.f, 0.f};
        for (int i = 0; i < 4; ++i) cudaEventElapsedTime(&t[i], r->ev64[5 * k + i], r->ev64[5 * k + i + 1]);
        stats->ms_rec64 += t[0];
        stats->ms_sum64 += t[1];
        stats->ms_emit64 += t[2];
        stats->ms_replay64 += t[3];
        slots += std::min<unsigned long long>(r->h_rec64[3 * k], (unsigned long long)r->seg_cap64) * REC_SEG;
        short_samples += r->h_rec64[3 * k + 1];
        records += r->h_rec64[3 * k + 2];
    }
    stats->emit64 = r->last_emit64 && short_samples == 0 ? 1 : 0;
    stats->rec64_slots = (long long)slots;
    stats->rec64_short = (long long)short_samples;
    stats->rec64_records = (long long)records;
    stats->rec64_waves = r->waves64;
}

int read_counters(so_renderer* r, Counters* c) {
    SO_CK(r, cudaMemcpyAsync(c, r->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, r->st));
    SO_CK(r, cudaStreamSynchronize(r->st));
    return SO_OK;
}

// Impl::trace (render.cu:677-730): pass 1, optional adaptive pass 2, resolve into img (d_img by
// default).  With stats == NULL nothing waits on the device except the adaptive pass's chunk count.
int trace_frame(so_renderer* r, const so_frame& f, bool adaptive, so_stats* stats, float4* img = nullptr) {
    if (!img) img = r->d_img;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    if (stats)
        for (auto& e : ev) cudaEventCreate(&e);
    struct EvGuard {
        cudaEvent_t* e;
        ~EvGuard() {
            for (int i = 0; i < 4; ++i)
                if (e[i]) cudaEventDestroy(e[i]);
        }
    } guard{ev};
    SO_CK(r, cudaMemcpyAsync(r->d_frame, &f, sizeof f, cudaMemcpyHostToDevice, r->st));
    SO_CK(r, cudaMemsetAsync(r->d_cnt, 0, sizeof(Counters), r->st));
    r->list_rays = 0;
    const long long n = (long long)f.W * f.H;
    TraceLaunch L;
    launch_common(r, L);
    L.kind = RAYS_PIXELS;
    L.nrays = n;
    L.W = f.W;
    L.H = f.H;
    L.spp = f.spp;
    L.jitter = 1;
    L.sample0 = 0;
    L.accum = (float*)r->d_accum;
    L.ystat = (float*)r->d_ystat;
    if (int brc = bake_turbulence(r, L)) return brc;
    if (stats) cudaEventRecord(ev[0], r->st);
    const bool mixed = r->precision == SO_PREC_MIXED;
    if (r->S.sky_on && r->S.mode == SO_MODE_VISIBLE) {
        int crc = trace_corners(r, f.W, f.H);
        if (crc) return crc;
        L.sky_uv = r->d_uvgrid;
        L.sky_grad_scale = 0.7f;
    }
    int rc = mixed ? trace_pass1_mixed(r, f, L) : run_tracer(r, L);
    if (rc) return rc;
    if (stats) cudaEventRecord(ev[1], r->st);
    long long samples = n * f.spp;
    const int extra_max = std::max(r->rs.spp_max - f.spp, 0);
    bool have_nsamp = false;
    if (adaptive && extra_max > 0) {
        // yref = 0.03 * fsum / (n spp) (render.cu:702), fsum = sum over pixels of sum_s Y.
        SO_CK(r, launch_sum_channel((const float*)r->d_ystat, 2, n, r->d_part, r->d_fsum, r->num_sms, r->st));
        SO_CK(r, launch_fill_u32(r->d_nsamp, (uint32_t)f.spp, n, r->st));
        have_nsamp = true;
        SO_CK(r, launch_adapt(r->d_ystat, (uint32_t)f.spp, n, r->d_fsum, 1.0 / ((double)n * f.spp), r->rs.target_err,
                              extra_max, r->d_extra, r->d_chunks, f.W, f.H, CHUNK, r->st));
        long long nt = scan_tiles(n);
        SO_CK(r, cudaMemsetAsync(r->d_tiles, 0, (size_t)(nt + 1) * sizeof(unsigned long long), r->st));
        SO_CK(r, cudaMemsetAsync(r->d_err, 0, sizeof(int), r->st));
        SO_CK(r, launch_scan(r->d_chunks, r->d_offsets, n, r->d_tiles, (unsigned int*)(r->d_tiles + nt), r->d_total,
                             r->d_err, r->st));
        uint32_t total = 0;
        int serr = 0;
        SO_CK(r, cudaMemcpyAsync(&total, r->d_total, 4, cudaMemcpyDeviceToHost, r->st));
        SO_CK(r, cudaMemcpyAsync(&serr, r->d_err, 4, cudaMemcpyDeviceToHost, r->st));
        SO_CK(r, cudaStreamSynchronize(r->st));
        if (serr) return fail(r, SO_ERR_WATCHDOG, "scan look-back gave up");
        if (total > 0) {
            if ((long long)total > r->chunk_cap) {
                if (r->d_chunk_acc) cudaFree(r->d_chunk_acc);
                r->d_chunk_acc = nullptr;
                r->chunk_cap = 0;
                SO_CK(r, dalloc(&r->d_chunk_acc, (size_t)total));
                r->chunk_cap = total;
            }
            TraceLaunch L2 = L;
            L2.kind = RAYS_CHUNKS;
            L2.nrays = total;
            L2.sample0 = f.spp;
            L2.offsets = r->d_offsets;
            L2.chunk_acc = (float*)r->d_chunk_acc;
            L2.chunk = CHUNK;
            L2.ystat = nullptr;
            L2.sky_grad_scale = 0.5f;
            // the queue head restarts for pass 2; the sample counters keep accumulating
            SO_CK(r, cudaMemsetAsync(&r->d_cnt->next, 0, sizeof(unsigned long long), r->st));
            if (stats) cudaEventRecord(ev[2], r->st);
            rc = run_tracer(r, L2);
            if (rc) return rc;
            if (stats) cudaEventRecord(ev[3], r->st);
            SO_CK(r, launch_add_chunks(r->d_accum, r->d_nsamp, r->d_offsets, r->d_chunks, r->d_chunk_acc, n, CHUNK,
                                       r->st));
            samples += (long long)total * CHUNK;
        }
    }
    SO_CK(r, launch_resolve(img, r->d_accum, have_nsamp ? r->d_nsamp : nullptr, (uint32_t)f.spp, n,
                            r->S.mode == SO_MODE_VISIBLE, r->st));
    if (stats) {
        Counters c;
        rc = read_counters(r, &c);
        if (rc) return rc;
        if (mixed) {
            Counters c3[2];
            SO_CK(r, cudaMemcpy(c3, r->d_cnt3, sizeof c3, cudaMemcpyDeviceToHost));
            stats->flow_steps_fp32 = (long long)c.flow_steps;
            stats->redo_turn = (long long)c.redo_turn;
            stats->redo_drift = (long long)c.redo_drift;
            stats->redo_limit = (long long)c.redo_limit;
            float ms32 = 0.f;
            cudaEventElapsedTime(&ms32, r->ev32[0], r->ev32[1]);
            stats->ms_fp32 = ms32;
            for (const Counters& x : c3) {
                c.attempts += x.attempts;
                c.accepted += x.accepted;
                c.step_limited += x.step_limited;
                c.flow_steps += x.flow_steps;
            }
            unsigned long long nl[NLISTS];
            SO_CK(r, cudaMemcpy(nl, r->d_nlists, sizeof nl, cudaMemcpyDeviceToHost));
            stats->ms_fp32_trace = ms32;
            stats->ms_turb = 0.0;
            stats->turb_records = 0;
            stats->redo_records = (long long)nl[6];
            stats->record_waves = 0;
            if (r->last_defer) {
                double ta = 0.0, tb = 0.0;
                for (int w = 0; w < r->last_waves; ++w) {
                    float a = 0.f, b = 0.f;
                    cudaEventElapsedTime(&a, r->ev_wave[3 * w], r->ev_wave[3 * w + 1]);
                    cudaEventElapsedTime(&b, r->ev_wave[3 * w + 1], r->ev_wave[3 * w + 2]);
                    ta += a;
                    tb += b;
                }
                stats->ms_fp32_trace = ta;
                stats->ms_turb = tb;
                stats->turb_records = (long long)nl[10] * REC_SEG;  // segments summed, all waves
                stats->record_waves = r->last_waves;
            }
            // c.attempts now holds FP32 attempts (k_trace32) + band + re-trace FP64 attempts;
            // the FP64 approach's attempts are in pad[0]
            stats->attempts_fp32 = (long long)(c.attempts - c3[0].attempts - c3[1].attempts);
            c.attempts += c.pad[0];
            c.fp64_rays = nl[1] + nl[2];  // band + re-traced rays
            stats->band_rays = (long long)nl[1];
        } else {
            stats->attempts_fp32 = 0;
            stats->band_rays = 0;
            stats->flow_steps_fp32 = 0;
            stats->ms_fp32 = 0.0;
            stats->redo_turn = stats->redo_drift = stats->redo_limit = 0;
            stats->ms_fp32_trace = stats->ms_turb = 0.0;
            stats->turb_records = stats->redo_records = 0;
            stats->record_waves = 0;
            c.fp64_rays = 0;
        }
        rec64_stats(r, stats);
        float ms1 = 0.f, ms2 = 0.f;
        cudaEventElapsedTime(&ms1, ev[0], ev[1]);
        if (cudaEventQuery(ev[3]) == cudaSuccess && cudaEventElapsedTime(&ms2, ev[2], ev[3]) != cudaSuccess) ms2 = 0.f;
        cudaGetLastError();
        stats->ms_kernel = (double)ms1 + (double)ms2;
        stats->flow_steps = (long long)c.flow_steps;
        stats->samples = samples;
        stats->step_limited = (long long)c.step_limited;
        stats->attempts = (long long)c.attempts;
        stats->accepted = (long long)c.accepted;
        stats->fp64_rays = (long long)c.fp64_rays;
    }
    return SO_OK;
}

int alloc_frame_buffers(so_renderer* r, int W, int H) {
    r->npix = (long long)W * H;
    const long long n = r->npix;
    SO_CK(r, dalloc(&r->d_accum, n));
    SO_CK(r, dalloc(&r->d_img, n));
    SO_CK(r, dalloc(&r->d_ystat, n));
    SO_CK(r, dalloc(&r->d_nsamp, n));
    SO_CK(r, dalloc(&r->d_extra, n));
    SO_CK(r, dalloc(&r->d_chunks, n));
    SO_CK(r, dalloc(&r->d_offsets, n));
    SO_CK(r, dalloc(&r->d_total, 1));
    SO_CK(r, dalloc(&r->d_tiles, scan_tiles(n) + 2));
    SO_CK(r, dalloc(&r->d_err, 1));
    return SO_OK;
}

// Packed device storage for so_trace_rays outputs.
struct RayBufs {
    int8_t *fate, *ncross;
    double *theta, *phi, *cross_r, *cross_g;
    float* I;
    int32_t *nacc, *natt;
};
size_t ray_bytes(long long n) { return (size_t)n * (2 + 8 * 2 + 16 + 4 * 2 + 48); }
RayBufs carve(void* base, long long n) {
    char* p = (char*)base;
    RayBufs b;
    b.theta = (double*)p;
    p += 8 * n;
    b.phi = (double*)p;
    p += 8 * n;
    b.cross_r = (double*)p;
    p += 24 * n;
    b.cross_g = (double*)p;
    p += 24 * n;
    b.I = (float*)p;
    p += 16 * n;
    b.nacc = (int32_t*)p;
    p += 4 * n;
    b.natt = (int32_t*)p;
    p += 4 * n;
    b.fate = (int8_t*)p;
    p += n;
    b.ncross = (int8_t*)p;
    return b;
}

}  // namespace

namespace so {
// Message returned by so_last_error(NULL), for entry points that have no renderer handle.
void set_global_error(const std::string& msg) { g_init_error = msg; }

// ---- services for the surrogate (so_surrogate.cpp) ----------------------------------------------
int rend_device(so_renderer* r) { return r->device; }
int rend_num_sms(so_renderer* r) { return r->num_sms; }
cudaStream_t rend_stream(so_renderer* r) { return r->st; }
const so_scene& rend_scene(so_renderer* r) { return r->S; }
const so_settings& rend_settings(so_renderer* r) { return r->rs; }
const so_scene* rend_scene_dev(so_renderer* r) { return r->d_scene; }
int rend_fail(so_renderer* r, int code, const char* msg) { return fail(r, code, msg); }

int rend_band_table(so_renderer* r, double th, const float** d_band, int* n) {
    if (!r->d_band && dalloc(&r->d_band, BAND_N) != cudaSuccess) return fail(r, SO_ERR_ALLOC, "band table allocation");
    if (r->band_a != r->S.a || r->band_th != th) {
        std::vector<float> tab = band_table(r->S.a, th);
        SO_CK(r, cudaMemcpyAsync(r->d_band, tab.data(), BAND_N * sizeof(float), cudaMemcpyHostToDevice, r->st));
        SO_CK(r, cudaStreamSynchronize(r->st));
        r->band_a = r->S.a;
        r->band_th = th;
    }
    *d_band = r->d_band;
    *n = BAND_N;
    return SO_OK;
}

int rend_upload_frame(so_renderer* r, const so_frame& f, const so_frame** d_frame) {
    SO_CK(r, cudaMemcpyAsync(r->d_frame, &f, sizeof(so_frame), cudaMemcpyHostToDevice, r->st));
    *d_frame = r->d_frame;
    return SO_OK;
}

int rend_trace_list(so_renderer* r, int n, const double* d_x, const double* d_y, const so_rays_out& d_out, int vacuum,
                    int side) {
    if (n <= 0) return SO_OK;
    cudaStream_t st = r->st;
    Counters* cnt = r->d_cnt;
    if (side) {
        if (int rc = ensure_side_queue(r)) return rc;
        SO_CK(r, cudaEventRecord(r->ev_fork, r->st));
        SO_CK(r, cudaStreamWaitEvent(r->st2, r->ev_fork, 0));
        st = r->st2;
        cnt = &r->d_cnt3[0];
    }
    SO_CK(r, cudaMemsetAsync(cnt, 0, sizeof(Counters), st));
    TraceLaunch L;
    launch_common(r, L);
    L.counters = cnt;
    L.kind = RAYS_LIST;
    L.nrays = n;
    L.x = d_x;
    L.y = d_y;
    L.out = d_out;
    L.record_cross = d_out.cross_r != nullptr && d_out.cross_g != nullptr;
    if (!L.record_cross) {
        L.out.cross_r = nullptr;
        L.out.cross_g = nullptr;
    }
    cudaError_t e = launch_trace64(L, vacuum ? VAR_VACUUM : variant_of(r->S), r->num_sms, st);
    if (e != cudaSuccess) return cuda_fail(r, e, "tracer launch");
    return SO_OK;
}

int rend_trace_list_frames(so_renderer* r, int n, const double* d_x, const double* d_y, const so_rays_out& d_out,
                           int vacuum, const so_scene* d_scenes, const so_frame* d_frames, const int* d_frame_scene,
                           int nframes) {
    if (n <= 0) return SO_OK;
    if (nframes <= 0 || !d_scenes || !d_frames || !d_frame_scene) return fail(r, SO_ERR_ARG, "trace list: frames");
    SO_CK(r, cudaMemsetAsync(r->d_cnt, 0, sizeof(Counters), r->st));
    r->list_rays = 0;
    TraceLaunch L;
    launch_common(r, L);
    L.scenes = d_scenes;
    L.frames = d_frames;
    L.frame_scene = d_frame_scene;
    L.nframes = nframes;
    L.list_frames = nframes;
    L.kind = RAYS_LIST;
    L.nrays = n;
    L.x = d_x;
    L.y = d_y;
    L.out = d_out;
    L.record_cross = d_out.cross_r != nullptr && d_out.cross_g != nullptr;
    if (!L.record_cross) {
        L.out.cross_r = nullptr;
        L.out.cross_g = nullptr;
    }
    cudaError_t e = launch_trace64(L, vacuum ? VAR_VACUUM : variant_of(r->S), r->num_sms, r->st);
    if (e != cudaSuccess) return cuda_fail(r, e, "tracer launch");
    return SO_OK;
}

int rend_join_side(so_renderer* r) {
    if (!r->st2) return SO_OK;
    SO_CK(r, cudaEventRecord(r->ev_join, r->st2));
    SO_CK(r, cudaStreamWaitEvent(r->st, r->ev_join, 0));
    return SO_OK;
}
}  // namespace so

extern "C" {

int so_init(so_renderer** out, int device, const so_scene* scene, const so_tables* tables, const so_settings* rs) {
    if (!out) return fail(nullptr, SO_ERR_ARG, "so_init: out is NULL");
    *out = nullptr;
    if (!scene || !tables || !rs) return fail(nullptr, SO_ERR_ARG, "so_init: NULL argument");
    if (rs->W <= 0 || rs->H <= 0 || rs->spp <= 0) return fail(nullptr, SO_ERR_ARG, "so_init: bad render settings");
    if (!tables->k2_ln || tables->k2_n < 2 || !tables->bb_xyz || tables->bb_n < 2 || !tables->disk_lnT ||
        tables->disk_n < 2)
        return fail(nullptr, SO_ERR_ARG, "so_init: missing tables");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return fail(nullptr, SO_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(nullptr, SO_ERR_ARG, "so_init: bad device index");
    so_renderer* r = new so_renderer;
    r->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&r->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&r->st, cudaStreamNonBlocking);
    int rc = SO_OK;
    if (e != cudaSuccess) rc = cuda_fail(nullptr, e, "so_init device");
    auto up = [&](float** d, const float* h, size_t n) -> int {
        if (dalloc(d, n) != cudaSuccess) return SO_ERR_ALLOC;
        if (cudaMemcpy(*d, h, n * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) return SO_ERR_CUDA;
        return SO_OK;
    };
    if (!rc) rc = up(&r->d_disk, tables->disk_lnT, (size_t)tables->disk_n);
    if (!rc) rc = up(&r->d_k2, tables->k2_ln, (size_t)tables->k2_n);
    if (!rc) rc = up(&r->d_bb, tables->bb_xyz, (size_t)tables->bb_n * 3);
    if (!rc && (dalloc(&r->d_scene, 1) != cudaSuccess || dalloc(&r->d_frame, 1) != cudaSuccess ||
                dalloc(&r->d_frame_scene, 1) != cudaSuccess || dalloc(&r->d_cnt, 1) != cudaSuccess ||
                dalloc(&r->d_part, 600) != cudaSuccess || dalloc(&r->d_fsum, 1) != cudaSuccess))
        rc = SO_ERR_ALLOC;
    if (!rc && cudaMemset(r->d_frame_scene, 0, sizeof(int)) != cudaSuccess) rc = SO_ERR_CUDA;
    if (!rc) {
        r->S = *scene;
        r->S.disk_n = tables->disk_n;
        r->S.k2_n = tables->k2_n;
        r->S.bb_n = tables->bb_n;
        r->rs = *rs;
        // the star map comes with so_set_sky; until then no sky (render.cu:550, 590-592)
        r->sky_requested = scene->sky_on ? 1 : 0;
        r->S.sky_on = 0;
        r->S.sky_tex = 0;
        rc = turb_setup(r);
        if (!rc) rc = upload_scene(r);
    }
    if (!rc) rc = alloc_frame_buffers(r, rs->W, rs->H);
    if (!rc && cudaStreamSynchronize(r->st) != cudaSuccess) rc = SO_ERR_CUDA;
    if (rc) {
        if (g_init_error.empty()) g_init_error = r->err.empty() ? "so_init failed" : r->err;
        free_all(r);
        delete r;
        return rc;
    }
    *out = r;
    return SO_OK;
}

int so_update_scene(so_renderer* r, const so_scene* scene) {
    if (!r || !scene) return fail(r, SO_ERR_ARG, "so_update_scene: NULL argument");
    // tables and the baked-turbulence set-up stay as so_init made them (render.cu:658-675)
    const so_scene keep = r->S;
    r->S = *scene;
    r->S.disk_n = keep.disk_n;
    r->S.k2_n = keep.k2_n;
    r->S.bb_n = keep.bb_n;
    r->S.sky_tex = keep.sky_tex;
    r->S.sky_on = keep.sky_on;
    for (int k = 0; k < 24; ++k) r->S.turb_tex[k] = keep.turb_tex[k];
    r->S.turb_nt = keep.turb_nt;
    r->S.turb_lr0 = keep.turb_lr0;
    r->S.turb_lr1 = keep.turb_lr1;
    r->S.turb_zmax = keep.turb_zmax;
    r->S.turb_d0 = keep.turb_d0;
    r->S.turb_dd = keep.turb_dd;
    return upload_scene(r);
}

int so_render(so_renderer* r, const so_frame* f_in, const so_post* post, double percentile, so_hdr_frame* out,
              so_stats* stats) {
    if (!r || !f_in || !out || !out->px) return fail(r, SO_ERR_ARG, "so_render: NULL argument");
    if (post && (!(post->bloom >= 0.f && post->bloom <= 1.f) || !(post->blur_sigma_px >= 0.0)))
        return fail(r, SO_ERR_ARG, "so_render: bloom must be in [0, 1] and blur_sigma_px >= 0");
    if (!(percentile >= 0.0 && percentile <= 1.0)) return fail(r, SO_ERR_ARG, "so_render: percentile must be in [0, 1]");
    if (cudaSetDevice(r->device) != cudaSuccess) return fail(r, SO_ERR_CUDA, "cudaSetDevice");
    so_frame f = *f_in;
    f.W = r->rs.W;
    f.H = r->rs.H;
    f.spp = r->rs.spp;
    double t0 = now_ms();
    int rc = trace_frame(r, f, true, stats);
    if (rc) return rc;
    double t1 = now_ms();
    // post filters (render.cu:766-767): glare in visible mode, interferometer beam in radio mode
    const bool bloom = post && r->S.mode == SO_MODE_VISIBLE && post->bloom > 0.f;
    const bool blur = post && r->S.mode == SO_MODE_RADIO && post->blur_sigma_px > 0.5;
    if (bloom || blur) {
        if (int prc = ensure_post(r)) return prc;
        cudaError_t e = bloom ? post_bloom(r->lev, post->bloom, r->st) : post_radio_blur(r->lev, r->d_tmp, post->blur_sigma_px, r->st);
        if (e != cudaSuccess) return cuda_fail(r, e, "post filters");
    }
    out->W = f.W;
    out->H = f.H;
    // Luminance percentile over significant pixels (render.cu:771-790), on the device: Y per pixel
    // (radio: I minus hide_direct times the direct light, visible: Rec. 709 luma), its maximum, and
    // the percentile of the values above 1e-5 of the maximum (the same order statistic as the
    // reference's nth_element), read back with the frame
    const float hide = post ? post->hide_direct : 0.f;
    if (int lrc = ensure_lum(r)) return lrc;
    SO_CK(r, post_luminance(r->d_img, r->npix, r->S.mode == SO_MODE_RADIO, hide, percentile, r->lum, r->st));
    SO_CK(r, cudaMemcpyAsync(out->px, r->d_img, (size_t)r->npix * sizeof(float4), cudaMemcpyDeviceToHost, r->st));
    SO_CK(r, cudaMemcpyAsync(r->h_lum, r->lum.stat, sizeof(LumStat), cudaMemcpyDeviceToHost, r->st));
    SO_CK(r, cudaStreamSynchronize(r->st));
    out->lum_percentile = r->h_lum->nsig ? (double)r->h_lum->pv : 0.0;
    out->lum_max = r->h_lum->mx;
    if (stats) {
        stats->ms_trace = t1 - t0;
        stats->ms_post = now_ms() - t1;
    }
    return SO_OK;
}

int so_render_device(so_renderer* r, const so_frame* f_in, float* d_px, so_stats* stats) {
    if (!r || !f_in || !d_px) return fail(r, SO_ERR_ARG, "so_render_device: NULL argument");
    if (cudaSetDevice(r->device) != cudaSuccess) return fail(r, SO_ERR_CUDA, "cudaSetDevice");
    so_frame f = *f_in;
    f.W = r->rs.W;
    f.H = r->rs.H;
    f.spp = r->rs.spp;
    double t0 = now_ms();
    int rc = trace_frame(r, f, true, stats, reinterpret_cast<float4*>(d_px));
    if (rc) return rc;
    if (stats) {
        stats->ms_trace = now_ms() - t0;
        stats->ms_post = 0.0;
    }
    return SO_OK;
}

int so_radio_flux(so_renderer* r, const so_frame* f_in, int n, double pix_sr, double* jy) {
    if (!r || !f_in || !jy || n <= 0) return fail(r, SO_ERR_ARG, "so_radio_flux: bad argument");
    if ((long long)n * n > r->npix) return fail(r, SO_ERR_SIZE, "so_radio_flux: n*n exceeds the frame buffers");
    if (cudaSetDevice(r->device) != cudaSuccess) return fail(r, SO_ERR_CUDA, "cudaSetDevice");
    so_frame f = *f_in;
    f.W = n;
    f.H = n;
    f.spp = 2;
    int rc = trace_frame(r, f, false, nullptr);
    if (rc) return rc;
    // sum of I_nu over the n x n image (render.cu:803-808), fixed-order FP64 sum on the device
    SO_CK(r, launch_sum_channel((const float*)r->d_img, 4, (long long)n * n, r->d_part, r->d_fsum, r->num_sms, r->st));
    double s = 0;
    SO_CK(r, cudaMemcpyAsync(&s, r->d_fsum, sizeof s, cudaMemcpyDeviceToHost, r->st));
    SO_CK(r, cudaStreamSynchronize(r->st));
    *jy = s * pix_sr / 1e-23;
    return SO_OK;
}

static int trace_rays_impl(so_renderer* r, const so_frame* f, int n, const double* d_x, const double* d_y,
                           const so_rays_out& d_out) {
    SO_CK(r, cudaMemcpyAsync(r->d_frame, f, sizeof(so_frame), cudaMemcpyHostToDevice, r->st));
    SO_CK(r, cudaMemsetAsync(r->d_cnt, 0, sizeof(Counters), r->st));
    r->list_rays = 0;
    TraceLaunch L;
    launch_common(r, L);
    if (int brc = bake_turbulence(r, L)) return brc;
    L.kind = RAYS_LIST;
    L.nrays = n;
    L.x = d_x;
    L.y = d_y;
    L.out = d_out;
    L.record_cross = d_out.cross_r != nullptr && d_out.cross_g != nullptr;
    if (!L.record_cross) {
        L.out.cross_r = nullptr;
        L.out.cross_g = nullptr;
    }
    const int rc = run_tracer(r, L);
    if (rc == SO_OK) r->list_rays = n;
    return rc;
}

int so_trace_stats(so_renderer* r, so_stats* stats) {
    if (!r || !stats) return fail(r, SO_ERR_ARG, "so_trace_stats: NULL argument");
    if (r->list_rays <= 0) return fail(r, SO_ERR_STATE, "so_trace_stats: no ray list traced since the last frame");
    if (cudaSetDevice(r->device) != cudaSuccess) return fail(r, SO_ERR_CUDA, "cudaSetDevice");
    Counters c;
    if (int rc = read_counters(r, &c)) return rc;
    std::memset(stats, 0, sizeof *stats);
    stats->samples = r->list_rays;
    stats->attempts = (long long)c.attempts;
    stats->accepted = (long long)c.accepted;
    stats->flow_steps = (long long)c.flow_steps;
    stats->step_limited = (long long)c.step_limited;
    rec64_stats(r, stats);
    return SO_OK;
}

int so_trace_rays_device(so_renderer* r, const so_frame* f, int n, const double* d_x, const double* d_y,
                         const so_rays_out* d_out) {
    if (!r || !f || !d_out || n < 0 || (n > 0 && (!d_x || !d_y))) return fail(r, SO_ERR_ARG, "so_trace_rays_device");
    if (n == 0) return SO_OK;
    if (cudaSetDevice(r->device) != cudaSuccess) return fail(r, SO_ERR_CUDA, "cudaSetDevice");
    return trace_rays_impl(r, f, n, d_x, d_y, *d_out);
}

int so_trace_rays(so_renderer* r, const so_frame* f, int n, const double* x, const double* y, const so_rays_out* out) {
    if (!r || !f || !out || n < 0 || (n > 0 && (!x || !y))) return fail(r, SO_ERR_ARG, "so_trace_rays");
    if (n == 0) return SO_OK;
    if (cudaSetDevice(r->device) != cudaSuccess) return fail(r, SO_ERR_CUDA, "cudaSetDevice");
    if (n > r->ray_cap) {
        if (r->d_x) cudaFree(r->d_x);
        if (r->d_y) cudaFree(r->d_y);
        if (r->d_rays) cudaFree(r->d_rays);
        r->d_x = r->d_y = nullptr;
        r->d_rays = nullptr;
        r->ray_cap = 0;
        if (dalloc(&r->d_x, n) != cudaSuccess || dalloc(&r->d_y, n) != cudaSuccess ||
            cudaMalloc(&r->d_rays, ray_bytes(n)) != cudaSuccess)
            return fail(r, SO_ERR_ALLOC, "so_trace_rays: device allocation");
        r->ray_cap = n;
    }
    SO_CK(r, cudaMemcpyAsync(r->d_x, x, (size_t)n * 8, cudaMemcpyHostToDevice, r->st));
    SO_CK(r, cudaMemcpyAsync(r->d_y, y, (size_t)n * 8, cudaMemcpyHostToDevice, r->st));
    RayBufs b = carve(r->d_rays, n);
    so_rays_out d;
    d.fate = out->fate ? b.fate : nullptr;
    d.ncross = out->ncross ? b.ncross : nullptr;
    d.theta = out->theta ? b.theta : nullptr;
    d.phi = out->phi ? b.phi : nullptr;
    d.I = out->I ? b.I : nullptr;
    d.n_accepted = out->n_accepted ? b.nacc : nullptr;
    d.n_attempts = out->n_attempts ? b.natt : nullptr;
    const bool cross = out->cross_r && out->cross_g;
    d.cross_r = cross ? b.cross_r : nullptr;
    d.cross_g = cross ? b.cross_g : nullptr;
    int rc = trace_rays_impl(r, f, n, r->d_x, r->d_y, d);
    if (rc) return rc;
    auto back = [&](void* h, const void* dv, size_t bytes) -> cudaError_t {
        return h ? cudaMemcpyAsync(h, dv, bytes, cudaMemcpyDeviceToHost, r->st) : cudaSuccess;
    };
    SO_CK(r, back(out->fate, b.fate, (size_t)n));
    SO_CK(r, back(out->ncross, b.ncross, (size_t)n));
    SO_CK(r, back(out->theta, b.theta, (size_t)n * 8));
    SO_CK(r, back(out->phi, b.phi, (size_t)n * 8));
    SO_CK(r, back(out->I, b.I, (size_t)n * 16));
    SO_CK(r, back(out->n_accepted, b.nacc, (size_t)n * 4));
    SO_CK(r, back(out->n_attempts, b.natt, (size_t)n * 4));
    if (cross) {
        SO_CK(r, back(out->cross_r, b.cross_r, (size_t)n * 24));
        SO_CK(r, back(out->cross_g, b.cross_g, (size_t)n * 24));
    }
    SO_CK(r, cudaStreamSynchronize(r->st));
    return SO_OK;
}

int so_last_fates(so_renderer* r, int8_t* fate, uint8_t* in_band, long long n) {
    if (!r || (!fate && !in_band) || n <= 0) return SO_ERR_ARG;
    if (r->last_mixed_ns == 0) return fail(r, SO_ERR_STATE, "so_last_fates: no mixed-precision frame rendered");
    if (n != r->last_mixed_ns) return fail(r, SO_ERR_ARG, "so_last_fates: n is not the frame's sample count");
    if (cudaSetDevice(r->device) != cudaSuccess) return fail(r, SO_ERR_CUDA, "cudaSetDevice");
    SO_CK(r, cudaStreamSynchronize(r->st));
    if (fate) SO_CK(r, cudaMemcpy(fate, r->d_sample_fate, (size_t)n, cudaMemcpyDeviceToHost));
    if (in_band) {
        unsigned long long nb = 0;
        SO_CK(r, cudaMemcpy(&nb, &r->d_nlists[1], sizeof nb, cudaMemcpyDeviceToHost));
        std::vector<uint32_t> ids((size_t)nb);
        if (nb) SO_CK(r, cudaMemcpy(ids.data(), r->d_list64, (size_t)nb * 4, cudaMemcpyDeviceToHost));
        std::memset(in_band, 0, (size_t)n);
        for (uint32_t id : ids)
            if ((long long)id < n) in_band[id] = 1;
    }
    return SO_OK;
}

int so_set_precision(so_renderer* r, int precision, const so_mixed_opts* opts) {
    if (!r) return SO_ERR_ARG;
    if (precision != SO_PREC_FP64 && precision != SO_PREC_MIXED) return fail(r, SO_ERR_ARG, "bad precision");
    if (opts && opts->approach != 0 && opts->approach != 1) return fail(r, SO_ERR_ARG, "so_mixed_opts.approach: 0 or 1");
    if (opts && opts->sky_fp32 != 0 && opts->sky_fp32 != 1) return fail(r, SO_ERR_ARG, "so_mixed_opts.sky_fp32: 0 or 1");
    if (opts && opts->turbulence != 0 && opts->turbulence != 1)
        return fail(r, SO_ERR_ARG, "so_mixed_opts.turbulence: 0 or 1");
    if (opts && !(opts->records_per_ray >= 0.0 && opts->records_per_ray <= 1e6))
        return fail(r, SO_ERR_ARG, "so_mixed_opts.records_per_ray: 0 .. 1e6");
    if (opts && !(opts->pool_mb >= 0.0 && opts->pool_mb <= 1e7))
        return fail(r, SO_ERR_ARG, "so_mixed_opts.pool_mb: 0 .. 1e7");
    if (opts && opts->records_per_ray > 0.0) r->rec_per_ray = opts->records_per_ray;
    r->precision = precision;
    if (opts) r->mixed = *opts;
    return SO_OK;
}

int so_set_plasma(so_renderer* r, const so_plasma* p, const so_mode* modes) {
    if (!r || !p) return SO_ERR_ARG;
    if (p->model != SO_PLASMA_REFERENCE && p->model != SO_PLASMA_TORUS) return fail(r, SO_ERR_ARG, "bad plasma model");
    if (p->model == SO_PLASMA_TORUS) {
        if (p->n_modes < 0 || p->n_modes > SO_MAX_MODES) return fail(r, SO_ERR_SIZE, "n_modes out of range");
        if (p->n_modes > 0 && !modes) return fail(r, SO_ERR_ARG, "modes missing");
        if (!(p->h_sph > 0)) return fail(r, SO_ERR_ARG, "h_sph must be > 0");
    }
    if (cudaSetDevice(r->device) != cudaSuccess) return fail(r, SO_ERR_CUDA, "cudaSetDevice");
    if (r->d_modes) {
        cudaFree(r->d_modes);
        r->d_modes = nullptr;
    }
    r->plasma = *p;
    if (p->model == SO_PLASMA_TORUS && p->n_modes > 0) {
        if (dalloc(&r->d_modes, (size_t)p->n_modes) != cudaSuccess) return fail(r, SO_ERR_ALLOC, "modes alloc");
        SO_CK(r, cudaMemcpy(r->d_modes, modes, (size_t)p->n_modes * sizeof(so_mode), cudaMemcpyHostToDevice));
        if (!r->turb_modes) r->turb_modes = new TurbModes;
        turb_modes_fold(modes, p->n_modes, r->turb_modes);
    }
    return SO_OK;
}

int so_set_sky(so_renderer* r, int w, int h, const uint16_t* data) {
    if (!r) return SO_ERR_ARG;
    if (w <= 0 || h <= 0 || !data || (long long)w * h > (1ll << 28))
        return fail(r, SO_ERR_ARG, "so_set_sky: w, h > 0 and a w x h half2 texel array");
    if (cudaSetDevice(r->device) != cudaSuccess) return fail(r, SO_ERR_CUDA, "cudaSetDevice");
    SO_CK(r, cudaStreamSynchronize(r->st));
    if (r->sky_tex) cudaDestroyTextureObject(r->sky_tex);
    if (r->sky_mip) cudaFreeMipmappedArray(r->sky_mip);
    r->sky_tex = 0;
    r->sky_mip = nullptr;
    r->S.sky_tex = 0;
    r->S.sky_on = 0;
    // mip chain down to 1 x 1, level l box-filtered from level l - 1 (render.cu:551-575)
    int levels = 1;
    while ((w >> levels) > 0 || (h >> levels) > 0) ++levels;
    cudaChannelFormatDesc fd = cudaCreateChannelDescHalf2();
    SO_CK(r, cudaMallocMipmappedArray(&r->sky_mip, &fd, make_cudaExtent(w, h, 0), levels, cudaArraySurfaceLoadStore));
    cudaArray_t l0;
    SO_CK(r, cudaGetMipmappedArrayLevel(&l0, r->sky_mip, 0));
    SO_CK(r, cudaMemcpy2DToArray(l0, 0, 0, data, (size_t)w * 4, (size_t)w * 4, h, cudaMemcpyHostToDevice));
    for (int l = 1; l < levels; ++l) {
        cudaArray_t a, b;
        SO_CK(r, cudaGetMipmappedArrayLevel(&a, r->sky_mip, l - 1));
        SO_CK(r, cudaGetMipmappedArrayLevel(&b, r->sky_mip, l));
        cudaResourceDesc ra = {}, rb = {};
        ra.resType = rb.resType = cudaResourceTypeArray;
        ra.res.array.array = a;
        rb.res.array.array = b;
        cudaSurfaceObject_t sa = 0, sb = 0;
        SO_CK(r, cudaCreateSurfaceObject(&sa, &ra));
        cudaError_t e = cudaCreateSurfaceObject(&sb, &rb);
        if (e == cudaSuccess) {
            const int sw = std::max(w >> (l - 1), 1), sh = std::max(h >> (l - 1), 1);
            const int dw = std::max(w >> l, 1), dh = std::max(h >> l, 1);
            e = launch_mip_half2(sa, sw, sh, sb, dw, dh, r->st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(r->st);
            cudaDestroySurfaceObject(sb);
        }
        cudaDestroySurfaceObject(sa);
        if (e != cudaSuccess) return cuda_fail(r, e, "so_set_sky: mip level");
    }
    // the reference's sampler: bilinear + linear between mips, anisotropy up to 16, u wrapped
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeMipmappedArray;
    rd.res.mipmap.mipmap = r->sky_mip;
    cudaTextureDesc td = {};
    td.addressMode[0] = cudaAddressModeWrap;
    td.addressMode[1] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 1;
    td.mipmapFilterMode = cudaFilterModeLinear;
    td.maxMipmapLevelClamp = (float)(levels - 1);
    td.maxAnisotropy = 16;
    SO_CK(r, cudaCreateTextureObject(&r->sky_tex, &rd, &td, nullptr));
    r->S.sky_tex = (unsigned long long)r->sky_tex;
    r->S.sky_on = r->sky_requested;
    return upload_scene(r);
}

int so_set_flow_noise(so_renderer* r, int mode) {
    if (!r) return SO_ERR_ARG;
    if (mode != SO_FLOW_NOISE_BAKED && mode != SO_FLOW_NOISE_INLINE && mode != SO_FLOW_NOISE_BAKED_FP32)
        return fail(r, SO_ERR_ARG,
                    "so_set_flow_noise: SO_FLOW_NOISE_BAKED, SO_FLOW_NOISE_INLINE or SO_FLOW_NOISE_BAKED_FP32");
    if (cudaSetDevice(r->device) != cudaSuccess) return fail(r, SO_ERR_CUDA, "cudaSetDevice");
    SO_CK(r, cudaStreamSynchronize(r->st));
    r->flow_noise = mode;
    if (int rc = turb_setup(r)) return rc;
    return upload_scene(r);
}

void* so_stream(so_renderer* r) { return r ? (void*)r->st : nullptr; }

const char* so_last_error(const so_renderer* r) { return r ? r->err.c_str() : g_init_error.c_str(); }

void so_destroy(so_renderer* r) {
    if (!r) return;
    detach_batches(r);  // so_batch_free still frees them
    cudaSetDevice(r->device);
    if (r->st) cudaStreamSynchronize(r->st);
    free_all(r);
    delete r;
}

// main.cpp:475-508: secant iteration on ln n0 so that radio_flux matches target_jy.
int so_normalize_flux(so_renderer* r, so_scene* scene, const so_frame* f_wide, int n, double pix_sr, double target_jy,
                      double* n0_out, double* jy_out) {
    if (!r || !scene || !f_wide || n <= 0 || !(target_jy > 0)) return fail(r, SO_ERR_ARG, "so_normalize_flux");
    double jy = 0;
    int rc = so_update_scene(r, scene);
    if (!rc) rc = so_radio_flux(r, f_wide, n, pix_sr, &jy);
    if (rc) return rc;
    double x0 = std::log(scene->n0), f0v = std::log(std::max(jy, 1e-30));
    double target = std::log(target_jy);
    double x1 = x0 + (target - f0v) / 1.5, f1v = 0;
    for (int it = 0; it < 8; ++it) {
        scene->n0 = std::exp(x1);
        rc = so_update_scene(r, scene);
        if (!rc) rc = so_radio_flux(r, f_wide, n, pix_sr, &jy);
        if (rc) return rc;
        f1v = std::log(std::max(jy, 1e-30));
        if (std::fabs(f1v - target) < 0.01) break;
        double slope = (f1v - f0v) / (x1 - x0);
        if (!(slope > 0.2)) slope = 1.5;
        x0 = x1;
        f0v = f1v;
        x1 = x1 + (target - f1v) / slope;
    }
    scene->n0 = std::exp(x1);
    rc = so_update_scene(r, scene);
    if (rc) return rc;
    if (n0_out) *n0_out = scene->n0;
    if (jy_out) *jy_out = std::exp(f1v);
    return SO_OK;
}

}  // extern "C"

// ---- batched frames (the persistent wavefront) -----------------------------------------------------
struct so_batch {
    so_renderer* r = nullptr;
    int nframes = 0, nscenes = 0, W = 0, H = 0, spp = 1, variant = VAR_VACUUM;
    so_scene* d_scenes = nullptr;
    so_frame* d_frames = nullptr;
    int* d_frame_scene = nullptr;
    Counters* d_cnt = nullptr;
    so_tune tune{0, 1, 0.0, 1, 1};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    float* graph_px = nullptr;  // output buffer baked into the graph
    so_tune graph_tune{-1, -1, 0.0, -1, -1};
    // deferred passes (radio frames without disks): decided and sized before each graph capture;
    // wave64 = 0 traces in one persistent launch
    bool defer_ok = false;
    long long wave64 = 0;
    int sums64 = 0;              // 0 none (reference flow, torus without modes), 1 FP64, 2 FP32 (mixed)
    int w64 = REC64_W_TORUS;     // doubles per record
};

void detach_batches(so_renderer* r) {
    for (so_batch* b : r->batches) b->r = nullptr;
    r->batches.clear();
}

namespace {

void batch_drop_graph(so_batch* b) {
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
    b->graph_px = nullptr;
}

// Pixels per interleaved tile: the requested tile, lowered to the largest power of two that divides
// W * H when it does not divide it itself (so no tile runs past a frame's end).
int batch_tile(const so_batch* b) {
    const long long npix = (long long)b->W * b->H;
    long long t = std::max(1, b->tune.tile);
    if (npix % t != 0) {
        t = 1;
        while (t * 2 <= std::max(1, b->tune.tile) && npix % (t * 2) == 0) t *= 2;
    }
    return (int)t;
}

bool same_tune(const so_tune& a, const so_tune& b) {
    return a.ctas_per_sm == b.ctas_per_sm && a.interleave == b.interleave && a.tile == b.tile &&
           a.queue_chunk == b.queue_chunk;
}

// The batch's launch descriptor: all frames, the tuned launch shape.
void batch_launch_desc(so_batch* b, float* d_px, TraceLaunch& L) {
    so_renderer* r = b->r;
    launch_common(r, L);
    L.scenes = b->d_scenes;
    L.frames = b->d_frames;
    L.frame_scene = b->d_frame_scene;
    L.nframes = b->nframes;
    L.counters = b->d_cnt;
    L.kind = RAYS_PIXELS;
    L.W = b->W;
    L.H = b->H;
    L.spp = b->spp;
    L.jitter = 1;
    L.nrays = (long long)b->W * b->H * b->nframes;
    L.accum = d_px;
    L.interleave = b->tune.interleave;
    L.tile = batch_tile(b);
    L.queue_chunk = std::max(1, b->tune.queue_chunk);
    L.ctas_per_sm = b->tune.ctas_per_sm;
    // mixed precision on a batch: FP64 geometry everywhere (photon-ring windows lie in the critical
    // band), FP32 turbulence sums
    L.emit32 = r->precision == SO_PREC_MIXED;
}

// Whether and how the batch's next capture defers its turbulence sums and emission: radio frame
// work of at least kDeferMinJobs jobs, through the renderer's record pool (sized here, outside the
// capture), in waves.  The torus plasma's sums in FP32 for mixed precision, FP64 otherwise; the
// reference flow model (its noise in place: a batch bakes no slices) and the torus without modes
// defer the emission alone.
void batch_plan(so_batch* b, float* d_px) {
    so_renderer* r = b->r;
    b->wave64 = 0;
    b->sums64 = 0;
    TraceLaunch L;
    batch_launch_desc(b, d_px, L);
    if (!b->defer_ok || b->variant != VAR_RADIO || L.nrays < kDeferMinJobs) return;
    const bool sums = L.torus && L.n_modes > 0;
    const int w = sums ? REC64_W_TORUS : REC64_W_FLOW;
    long long wave = 0;
    if (ensure_records64(r, L.nrays, b->spp, w, &wave) != SO_OK) {
        r->err.clear();  // no pool: one persistent launch
        return;
    }
    b->wave64 = wave;
    b->w64 = w;
    b->sums64 = !sums ? 0 : (r->precision == SO_PREC_MIXED && r->turb_modes) ? 2 : 1;
    r->samples64 = L.nrays * b->spp;
}

// The launch sequence of one batch: counter reset, the tracer over all frames (one persistent launch,
// or the deferred passes in waves), resolve.
int batch_enqueue(so_batch* b, float* d_px) {
    so_renderer* r = b->r;
    SO_CK(r, cudaMemsetAsync(b->d_cnt, 0, sizeof(Counters), r->st));
    TraceLaunch L;
    batch_launch_desc(b, d_px, L);
    if (b->wave64 > 0) {
        if (int rc = enqueue_deferred64(r, L, b->variant, r->st, b->wave64, b->w64, b->sums64, true, false))
            return rc;
    } else {
        cudaError_t e = launch_trace64(L, b->variant, r->num_sms, r->st);
        if (e != cudaSuccess) return cuda_fail(r, e, "batch tracer launch");
    }
    SO_CK(r, launch_resolve(reinterpret_cast<float4*>(d_px), reinterpret_cast<const float4*>(d_px), nullptr,
                            (uint32_t)b->spp, L.nrays, r->S.mode == SO_MODE_VISIBLE, r->st));
    return SO_OK;
}

int batch_capture(so_batch* b, float* d_px) {
    so_renderer* r = b->r;
    batch_drop_graph(b);
    batch_plan(b, d_px);
    SO_CK(r, cudaStreamBeginCapture(r->st, cudaStreamCaptureModeRelaxed));
    int rc = batch_enqueue(b, d_px);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(r->st, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(r, e, "batch graph capture");
    b->graph = g;
    SO_CK(r, cudaGraphInstantiate(&b->gexec, g, 0));
    b->graph_px = d_px;
    b->graph_tune = b->tune;
    return SO_OK;
}

}  // namespace

extern "C" {

int so_batch_create(so_renderer* r, const so_scene* scenes, int nscenes, const so_frame* frames, const int* frame_scene,
                    int nframes, int W, int H, int spp, so_batch** out) {
    if (!out) return fail(r, SO_ERR_ARG, "so_batch_create: out is NULL");
    *out = nullptr;
    if (!r || !scenes || !frames || !frame_scene || nscenes <= 0 || nframes <= 0 || W <= 0 || H <= 0 || spp <= 0)
        return fail(r, SO_ERR_ARG, "so_batch_create: bad argument");
    if ((long long)W * H * nframes > 0x7fffffffll) return fail(r, SO_ERR_SIZE, "so_batch_create: too many rays");
    for (int i = 0; i < nframes; ++i)
        if (frame_scene[i] < 0 || frame_scene[i] >= nscenes) return fail(r, SO_ERR_ARG, "so_batch_create: frame_scene");
    const int var = variant_of(scenes[0]);
    for (int s = 0; s < nscenes; ++s) {
        if (scenes[s].sky_on) return fail(r, SO_ERR_UNSUPPORTED, "so_batch_create: sky texture lookups");
        if (variant_of(scenes[s]) != var) return fail(r, SO_ERR_ARG, "so_batch_create: scenes of different modes");
        if (scenes[s].disk_on && scenes[s].a != r->S.a)
            return fail(r, SO_ERR_UNSUPPORTED, "so_batch_create: disk scenes need the renderer's spin (disk table)");
    }
    if (cudaSetDevice(r->device) != cudaSuccess) return fail(r, SO_ERR_CUDA, "cudaSetDevice");
    so_batch* b = new so_batch;
    b->r = r;
    b->defer_ok = true;
    for (int s = 0; s < nscenes; ++s)
        b->defer_ok = b->defer_ok && scenes[s].mode == SO_MODE_RADIO && scenes[s].flow_on && !scenes[s].disk_on &&
                      scenes[s].max_steps < (1 << REC64_COUNT_BITS);
    b->nframes = nframes;
    b->nscenes = nscenes;
    b->W = W;
    b->H = H;
    b->spp = spp;
    b->variant = var;
    std::vector<so_scene> sc(scenes, scenes + nscenes);
    for (so_scene& s : sc) {  // the renderer's device tables
        // the reference flow's turbulence in place: a batch bakes no per-frame slices, so no scene
        // may point at textures of another frame's bake
        s.turb_nt = 0;
        for (int k = 0; k < 24; ++k) s.turb_tex[k] = 0;
        s.disk_lnT = r->d_disk;
        s.k2_lntab = r->d_k2;
        s.bb_xyz = r->d_bb;
        s.disk_n = r->S.disk_n;
        s.k2_n = r->S.k2_n;
        s.bb_n = r->S.bb_n;
    }
    std::vector<so_frame> fr(frames, frames + nframes);
    for (so_frame& f : fr) {
        f.W = W;
        f.H = H;
        f.spp = spp;
    }
    int rc = SO_OK;
    if (dalloc(&b->d_scenes, (size_t)nscenes) != cudaSuccess || dalloc(&b->d_frames, (size_t)nframes) != cudaSuccess ||
        dalloc(&b->d_frame_scene, (size_t)nframes) != cudaSuccess || dalloc(&b->d_cnt, 1) != cudaSuccess)
        rc = fail(r, SO_ERR_ALLOC, "so_batch_create: device allocation");
    if (!rc && (cudaMemcpy(b->d_scenes, sc.data(), sc.size() * sizeof(so_scene), cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(b->d_frames, fr.data(), fr.size() * sizeof(so_frame), cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(b->d_frame_scene, frame_scene, (size_t)nframes * sizeof(int), cudaMemcpyHostToDevice) !=
                    cudaSuccess))
        rc = fail(r, SO_ERR_CUDA, "so_batch_create: upload");
    if (rc) {
        so_batch_free(b);
        return rc;
    }
    r->batches.push_back(b);
    *out = b;
    return SO_OK;
}

int so_batch_render(so_batch* b, float* d_px, so_stats* stats) {
    if (!b || !d_px) return SO_ERR_ARG;
    if (!b->r) return SO_ERR_STATE;  // its renderer was destroyed
    so_renderer* r = b->r;
    if (cudaSetDevice(r->device) != cudaSuccess) return fail(r, SO_ERR_CUDA, "cudaSetDevice");
    r->list_rays = 0;
    if (b->gexec && b->wave64 > 0 && r->rec64_pending) {
        // the previous launch of the deferred graph ran short of records: capture again with a larger
        // pool (ensure_records64 doubles the estimate)
        if (cudaEventQuery(r->ev_rec64) == cudaSuccess) {
            unsigned long long short_samples = 0;
            for (int k = 0; k < r->waves64; ++k) short_samples += r->h_rec64[3 * k + 1];
            if (short_samples > 0) batch_drop_graph(b);
        }
        cudaGetLastError();  // a pending event reports cudaErrorNotReady
    }
    if (!b->gexec || b->graph_px != d_px || !same_tune(b->graph_tune, b->tune)) {
        int rc = batch_capture(b, d_px);
        if (rc) return rc;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (stats) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, r->st);
    }
    cudaError_t e = cudaGraphLaunch(b->gexec, r->st);
    if (e != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        return cuda_fail(r, e, "so_batch_render graph launch");
    }
    if (b->wave64 > 0) {  // the graph copied each wave's pool counters out: note when they are there
        cudaEventRecord(r->ev_rec64, r->st);
        r->rec64_pending = true;
    }
    if (stats) {
        cudaEventRecord(e1, r->st);
        Counters c;
        e = cudaMemcpyAsync(&c, b->d_cnt, sizeof c, cudaMemcpyDeviceToHost, r->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(r->st);
        float ms = 0.f;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (e != cudaSuccess) return cuda_fail(r, e, "so_batch_render");
        std::memset(stats, 0, sizeof *stats);
        stats->samples = (long long)b->W * b->H * b->nframes * b->spp;
        stats->step_limited = (long long)c.step_limited;
        stats->attempts = (long long)c.attempts;
        stats->accepted = (long long)c.accepted;
        stats->flow_steps = (long long)c.flow_steps;
        stats->ms_kernel = ms;
        stats->ms_trace = ms;
        if (b->wave64 > 0) {  // the deferred passes' pool counters, copied out by the graph
            unsigned long long slots = 0, short_samples = 0, records = 0;
            for (int k = 0; k < r->waves64; ++k) {
                slots += std::min<unsigned long long>(r->h_rec64[3 * k], (unsigned long long)r->seg_cap64) * REC_SEG;
                short_samples += r->h_rec64[3 * k + 1];
                records += r->h_rec64[3 * k + 2];
            }
            stats->rec64_slots = (long long)slots;
            stats->rec64_short = (long long)short_samples;
            stats->rec64_records = (long long)records;
            stats->rec64_waves = r->waves64;
            stats->emit64 = short_samples == 0 ? 1 : 0;
        }
    }
    return SO_OK;
}

int so_batch_set_tune(so_batch* b, const so_tune* t) {
    if (!b || !t || t->ctas_per_sm < 0 || (t->interleave != 0 && t->interleave != 1) || t->tile < 0 ||
        t->queue_chunk < 0 || t->queue_chunk > 64)
        return SO_ERR_ARG;
    b->tune.ctas_per_sm = t->ctas_per_sm;
    b->tune.interleave = t->interleave;
    b->tune.tile = std::max(1, t->tile);
    b->tune.queue_chunk = std::max(1, t->queue_chunk);
    return SO_OK;
}

int so_batch_autotune(so_batch* b, float* d_px, so_tune* best) {
    if (!b || !d_px) return SO_ERR_ARG;
    if (!b->r) return SO_ERR_STATE;
    // warm-up with the full grid; then CTAs per SM from 1 up (the launcher caps the value at the
    // kernel's occupancy limit, so the sweep stops once a larger cap no longer helps)
    const int per_sm = 8;
    {
        so_tune keep = b->tune;
        b->tune.ctas_per_sm = 0;
        so_stats st;
        int rc = so_batch_render(b, d_px, &st);
        if (rc) return rc;
        b->tune = keep;
    }
    double ms = 0.0;
    auto trial = [&](so_tune t, so_tune* win) -> int {
        b->tune = t;
        so_stats st;
        int rc = so_batch_render(b, d_px, &st);
        if (rc) return rc;
        ms = t.ms = st.ms_kernel;
        if (t.ms < win->ms) *win = t;
        return SO_OK;
    };
    // 1. CTAs per SM x job order (ray by ray, one job per grab)
    so_tune winner{0, 1, 1e300, 1, 1};
    for (int inter = 0; inter <= 1; ++inter) {
        for (int c = 1; c <= per_sm; ++c) {
            if (int rc = trial(so_tune{c, inter, 0.0, 1, 1}, &winner)) return rc;
            // a larger cap than the occupancy limit launches the same grid: stop early
            if (c >= 2 && ms > 1.5 * winner.ms) break;
        }
    }
    // 2. tile of the interleaved order, 3. queue chunk, each around the winner so far
    if (winner.interleave) {
        for (int tile : {32, 1024}) {
            so_tune t = winner;
            t.tile = tile;
            if (int rc = trial(t, &winner)) return rc;
        }
    }
    for (int chunk : {2, 4}) {
        so_tune t = winner;
        t.queue_chunk = chunk;
        if (int rc = trial(t, &winner)) return rc;
    }
    b->tune = winner;
    if (best) *best = winner;
    return SO_OK;
}

void so_batch_free(so_batch* b) {
    if (!b) return;
    if (b->r) {
        cudaSetDevice(b->r->device);
        auto& v = b->r->batches;
        v.erase(std::remove(v.begin(), v.end(), b), v.end());
    }
    batch_drop_graph(b);
    void* ps[] = {b->d_scenes, b->d_frames, b->d_frame_scene, b->d_cnt};
    for (void* p : ps)
        if (p) cudaFree(p);
    delete b;
}

}  // extern "C"
