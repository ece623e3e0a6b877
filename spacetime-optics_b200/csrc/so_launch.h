// so_launch.h -- launch descriptors shared by the host renderer and the CUDA kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/so_tracer.h"

namespace so {

// What a tracer launch computes.
enum RayKind : int {
    RAYS_LIST = 0,   // explicit tangent-plane points x[i], y[i] of frame 0, one sample each
    RAYS_PIXELS = 1, // every pixel of every frame, spp samples per pixel (frames share W, H, spp)
    RAYS_CHUNKS = 2, // adaptive pass 2: job j = `chunk` more samples of the pixel owning chunk j
    RAYS_SAMPLES = 3 // job j = sample list[j] (pixel * spp + s) of the pixel grid; result per sample
};

// Scene features a kernel instantiation supports (uniform over the frames of one launch).
enum Variant : int {
    VAR_VACUUM = 0,  // no emission: geometry, fate, winding order, escape direction
    VAR_RADIO = 1,   // hot-flow synchrotron transfer (reference or torus plasma)
    VAR_DISK = 2     // thin disk at equatorial crossings
};

// Device counters of one launch (zeroed before the launch).
constexpr int REC_SEG = 16;  // flow-step record slots per segment

// Flow-step record of the deferred FP64 path, rec64_w doubles per slot: [0] r, [1] u = cos theta,
// [2] torus plasma: the advected azimuth of the turbulence position (k_turb64_records overwrites
// it with the sum delta); reference flow: phi, [3] the Mino step h, [4] tag, [5] reference flow
// only: t.  k_emit64_records then overwrites [0] with the step's emission dI and [1] with its
// transmission exp(-dtau).  The tag holds the image-order bucket (bits 0-1: psi / pi clamped to 3)
// and the ray's attempt, accepted-step and flow-step counts after this step (20 bits each from bit
// 2, 22 and 42; the path needs max_steps < 2^20).  A ray list's records carry one more double, last:
// the ray's equatorial crossings after this step (its ncross output when the opacity cut ends it
// there).
constexpr int REC64_W_TORUS = 5, REC64_W_FLOW = 6;
constexpr int REC64_COUNT_BITS = 20;
// End state of one sample after the recording pass.
struct Sample64 {
    double lam, E;            // the ray's constants of motion used by the emission
    int nrec;                 // records in its chain
    int natt, nacc, nflow;    // attempts, accepted steps, flow steps to its end
    int fate;                 // 0 step limit, -1 capture, 1 escape
    int fidx;                 // frame
};

// Baked flow turbulence (render.cu:447-460, 594-620): per frame, TURB_NT retarded-time slices of
// TURB_NPHI x TURB_NLR x TURB_NZ density factors on (phi, ln R, z/R), phi fastest, in HBM.
constexpr int TURB_NPHI = 512, TURB_NLR = 192, TURB_NZ = 48, TURB_NT = 24;
struct TurbBake {
    float delta[TURB_NT];  // retarded-time offset of each slice, d0 + k dd (host float, as render.cu:681)
};
constexpr int NLISTS = 12;
// Block partials of launch_sum_channel: at most this many doubles in its `part` buffer.
constexpr int SUM_MAX_PARTIALS = 592;

struct Counters {
    unsigned long long next;          // ray-queue head
    unsigned long long step_limited;  // samples that hit max_steps
    unsigned long long attempts;      // DP5(4) attempts
    unsigned long long accepted;      // accepted steps
    unsigned long long fp64_rays;     // mixed precision: rays (or restarts) integrated in FP64
    unsigned long long flow_steps;    // accepted steps that evaluated the hot-flow transfer
    unsigned long long pad[2];        // [0] FP64 approach attempts, [1] FP32 accepted steps
    unsigned long long redo_turn;     // mixed: FP32 rays re-traced for a radial turning point inside turn_r
    unsigned long long redo_drift;    // mixed: FP32 rays re-traced for constraint drift
    unsigned long long redo_limit;    // mixed: FP32 rays re-traced because they reached max_steps
};

// The frame's 2x2 box-filter pyramid for the post filters (level 0 is the frame itself).
constexpr int POST_MAX_LEVELS = 9;
struct PostLevels {
    float4* p[POST_MAX_LEVELS];
    int w[POST_MAX_LEVELS], h[POST_MAX_LEVELS];
    int n;
};
cudaError_t post_bloom(const PostLevels& L, float strength, cudaStream_t st);
cudaError_t post_radio_blur(const PostLevels& L, float4* tmp, double sigma, cudaStream_t st);

// Luminance statistics of the HDR frame (render.cu:771-790) on the device: the maximum of Y over
// the pixels with Y > 0 and the given percentile of the values above 1e-5 of that maximum (an exact
// order statistic, by radix selection on the float bit patterns).
struct LumStat {
    double mx;                // maximum luminance (0 if none positive)
    float pv;                 // percentile value (0 if no significant pixel)
    float pad_;
    unsigned long long nsig;  // significant pixels
    unsigned long long k;     // rank still to find inside the selected prefix
    unsigned prefix;          // selected high bits so far
    unsigned pad2_;
};
constexpr int LUM_BLOCKS = 1184;   // grid of the luminance pass (8 x 148)
constexpr int LUM_HIST = 4096;     // radix bins of the first pass
struct LumScratch {
    float* lum;               // per pixel: Y as float, or -1 if Y <= 0
    double* part;             // LUM_BLOCKS partial maxima
    unsigned* hist;           // LUM_HIST bins
    LumStat* stat;
};
cudaError_t post_luminance(const float4* img, long long n, int radio, float hide, double percentile,
                           const LumScratch& s, cudaStream_t st);

struct TraceLaunch {
    const so_scene* scenes;   // device array, indexed by frame_scene[f]
    const so_frame* frames;   // device array
    const int* frame_scene;   // device array
    int nframes;
    int kind;                 // RayKind
    int record_cross;         // RAYS_LIST: record the first 3 equatorial crossings
    long long nrays;          // RAYS_LIST: number of points; RAYS_PIXELS: W*H*nframes
    int W, H, spp;            // RAYS_PIXELS geometry (shared by the frames)
    int jitter;               // RAYS_PIXELS: 1 = R2 jitter per sample (reference), 0 = pixel centres
    int sample0;              // first sample index (pass 2 continues the sequence)
    // plasma
    int torus, n_modes;
    double ne_index, te_index, h_sph, theta_e0, half_var;
    const so_mode* modes;     // device array (n_modes)
    // inputs / outputs (device pointers)
    const double* x;
    const double* y;
    so_rays_out out;          // RAYS_LIST outputs (device pointers, NULL = skip)
    float* accum;             // RAYS_PIXELS: W*H*nframes*4 sums
    float* ystat;             // RAYS_PIXELS: W*H*nframes*2 (sum Y, sum Y^2), or NULL
    Counters* counters;
    const unsigned long long* nrays_dev;  // if set, the job count is read from device memory
    // RAYS_CHUNKS
    const uint32_t* offsets;  // exclusive scan of chunks per pixel (W*H)
    float* chunk_acc;         // per chunk: 4 float sums
    int chunk;                // samples per chunk
    // RAYS_SAMPLES
    const uint32_t* list;     // sample ids
    float4* sample_out;       // per sample id: the sample's accumulated value
    int8_t* sample_fate;      // per sample id, or NULL
    // mixed precision
    double band_m, tol32, turn_r, drift_tol;
    double r_switch;          // FP64 approach down to this radius, FP32 inside
    double tol_approach;      // tolerance of the FP64 approach
    int far_field;            // FP64 approach: transport in 1/r (far_approach) where it applies
    int approach_it;          // attempts credited to a ray brought to r_switch by far_approach
                              // (the reference's Mino-time count there, for the max_steps limit)
    double r_emit;            // FP32 tracer: outgoing beyond this radius = escaped (0 = off)
    int t32_min_blocks;       // FP32 tracer register budget: resident CTAs per SM (4, 5 or 6)
    int t32_max_att;          // FP32 attempts after which a ray goes to the FP64 re-trace
    const float* turb_field;  // baked flow turbulence of this frame (NULL: inline sheared noise)
    const float2* sky_uv;     // visible mode with the star map: escape (u, v) of the pixel corners,
                              // (W + 1) x (H + 1), for the footprint of each pixel (NULL: no sky)
    float sky_grad_scale;     // footprint scale: 0.7 in pass 1, 0.5 in pass 2 (render.cu:102, 214)
    // batched frames (RAYS_PIXELS over nframes)
    int interleave;           // 0: job -> (frame = job / npix), 1: tiles of `tile` pixels cycle through the frames
    int tile;                 // interleave: consecutive pixels of one frame per tile (a divisor of W * H; <= 1: 1)
    int queue_chunk;          // consecutive jobs a lane takes per queue grab (<= 1: 1)
    int list_frames;          // RAYS_LIST: > 0 = ray i belongs to frame i % list_frames (else frame 0)
    int ctas_per_sm;          // persistent grid: CTAs per SM (0 = as many as fit)
    int emit32;               // FP64 tracer: torus turbulence sums in FP32 (geometry stays FP64)
    // deferred FP64 torus turbulence: pass 1 (defer64 = 1) integrates the geodesic only and records
    // every flow step that can change the transfer in its sample's chain of REC_SEG-slot segments;
    // k_turb64_records sums the modes at every record.  Then either k_emit64_records evaluates the
    // emission at every record and k_transfer64 applies them in order per sample, or pass 2
    // (defer64 = 2) integrates again and reads each sum back in order.  0 = sums in the tracer.
    int defer64;
    double* rec64;            // record pool: slot s at doubles rec64_w s .. (layout at REC64_W_TORUS)
    int rec64_w;              // doubles per record: REC64_W_TORUS or REC64_W_FLOW (+1 for a ray list)
    long long job0;           // deferred passes in waves: this launch's jobs are job0 .. job0 + nrays - 1
                              // of the frame's job numbering (chain heads and sample ends are indexed
                              // from job0)
    uint32_t* seg_next64;     // per segment: the sample's next segment
    uint2* seg_meta64;        // per segment: (sample id owning it, records in it)
    Sample64* samp64;         // per sample id: the recording pass's end state
    int* job_head64;          // per sample of a job (job * samples per job + s): its chain's first segment,
                              // -1 no records, -2 the pool ran out (the replay pass sums in place)
    long long seg_cap64;      // segments in the pool
    unsigned long long* rec64_ctl;  // [0] segments taken, [1] samples that ran out of segments, [2] records
    int replay_if_short;      // pass 2: runs only when a sample of pass 1 ran out of segments (the
                              // emission / transfer kernels then leave the frame to it)
    const float* band_rho;    // critical-curve radius (M) per image angle bin, band_n bins over 2 pi
    int band_n;
    float4* state;            // parked ray state, 5 float4 per sample id (SoA planes of nsamples)
    long long nsamples;       // W * H * spp
    uint32_t* list32;         // FP32 work list (sample ids), filled by the router / approach
    uint32_t* list64;         // FP64 work list (band rays), filled by the router
    uint32_t* redo;           // FP64 re-trace list (drift check / radial turning point near the hole)
    uint32_t* parked;         // rays parked at r_switch by the FP64 approach (the FP32 work list)
    // deferred torus turbulence (FP32 tracer, radio torus with Fourier modes): the tracer records
    // every emitting flow step, one batched kernel sums the modes at all records, one kernel runs
    // the ordered transfer per ray
    int defer;                // 1 = record flow steps instead of evaluating them in the tracer
    float4* rec;              // flow-step records (|r| sign bit = order bit 0, |h| sign = bit 1, u, phi_c)
    float* rec_delta;         // turbulence sum per record slot
    uint32_t* seg_next;       // per segment of REC_SEG record slots: the ray's next segment
    int2* ray_meta;           // per sample id: (first segment, record count)
    uint32_t* acc_list;       // rays with records, for the transfer kernel
    uint32_t* esc_list;       // star-map frames: FP32 rays that escaped, their end state parked in
                              // state (P4.x = transmittance), for k_sky_escape (count nlists[9])
    long long seg_cap;        // record segments available
    long long wave_begin, wave_end;  // deferred turbulence in waves: the FP32 tracer takes the parked
                                     // rays [wave_begin, wave_end) (wave_end <= 0: all of them)
    unsigned long long* nlists; // [0] list32, [1] list64, [2] redo, [3] parked, [4] acc_list counts,
                                // [5] record segments used, [6] rays re-traced for want of segments,
                                // [7] / [8] work heads of k_turb_records / k_flow_records,
                                // [9] sky escape list, [10] record segments summed over the waves
};

// Mixed-path kernels (k_trace_mixed.cu).
cudaError_t launch_route(const TraceLaunch& L, int all64, cudaStream_t st);
cudaError_t launch_approach64(const TraceLaunch& L, long long n, int num_sms, cudaStream_t st);
cudaError_t launch_trace32(const TraceLaunch& L, long long n, int variant, int num_sms, cudaStream_t st);
cudaError_t launch_bake_turb(const so_scene* d_scene, const so_frame* d_frame, const TurbBake& b, float* field,
                             cudaStream_t st);
// The same bake into TURB_NT 3-D float arrays through their surface objects (texture-fetch mode).
struct SurfaceSet {
    cudaSurfaceObject_t s[TURB_NT];
};
cudaError_t launch_bake_turb_surf(const so_scene* d_scene, const so_frame* d_frame, const TurbBake& b,
                                  const SurfaceSet& surf, cudaStream_t st);
// Sky: tangent-plane points of the (W + 1) x (H + 1) pixel corners of the frame in d_frame, the
// corners' escape (u, v) from the tracer's outputs, and one box-filtered half2 mip level.
cudaError_t launch_corner_points(const so_frame* d_frame, int W, int H, double* x, double* y, cudaStream_t st);
cudaError_t launch_corner_uv(const so_scene* d_scene, long long n, const int8_t* fate, const double* th,
                             const double* ph, float2* uv, cudaStream_t st);
cudaError_t launch_mip_half2(cudaSurfaceObject_t src, int sw, int sh, cudaSurfaceObject_t dst, int dw, int dh,
                             cudaStream_t st);
// Fourier modes of the torus turbulence in FP32 (phase folded into (-pi, pi]), passed to the batched
// sums as a kernel parameter (constant memory; up to SO_MAX_MODES = 1024, 20 KB).
struct TurbModes {
    float4 k[SO_MAX_MODES];  // kx, ky, kz, phase
    float a[SO_MAX_MODES];   // amplitude
    int n;
};
void turb_modes_fold(const so_mode* modes, int n, TurbModes* out);
cudaError_t launch_turb_records(const TraceLaunch& L, const TurbModes& M, int num_sms, cudaStream_t st);
// FP32 sums (SFU) at every record of a defer64 = 1 pass: the mixed form of launch_turb64_records.
cudaError_t launch_turb32_rec64(const TraceLaunch& L, const TurbModes& M, int num_sms, cudaStream_t st);
// FP64 sums at every record of a defer64 = 1 pass (modes from L.modes, L.n_modes of them), the
// emission at every record, and the ordered transfer of every job's samples into the outputs.
cudaError_t launch_turb64_records(const TraceLaunch& L, int num_sms, cudaStream_t st);
cudaError_t launch_emit64_records(const TraceLaunch& L, int num_sms, cudaStream_t st);
cudaError_t launch_transfer64(const TraceLaunch& L, int num_sms, cudaStream_t st);
cudaError_t launch_sky_escape(const TraceLaunch& L, int num_sms, cudaStream_t st);
cudaError_t launch_flow_records(const TraceLaunch& L, int num_sms, cudaStream_t st);
cudaError_t launch_gather_samples(const TraceLaunch& L, cudaStream_t st);

}  // namespace so
