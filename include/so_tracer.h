/* so_tracer.h -- C ABI of the B200-native Kerr ray tracer (bhrt's per-pixel tracer path).
 *
 * Drop-in boundary.  The reference exposes the path as the C++ class `Renderer`
 * (blackholes/src/renderer.hpp:72-88, implementation blackholes/src/render.cu:477-809) fed by the
 * POD structs `SceneGPU` / `FrameGPU` (blackholes/src/scene.hpp:12-80).  This header replaces that
 * class with an opaque handle and plain C entry points:
 *
 *   Renderer::init          (render.cu:531)  -> so_init
 *   Renderer::update_scene  (render.cu:658)  -> so_update_scene
 *   Renderer::render        (render.cu:755)  -> so_render
 *   Renderer::radio_flux    (render.cu:797)  -> so_radio_flux
 *   trace_ray per sample    (trace.cuh:62)   -> so_trace_rays (per-ray SoA, for parity work)
 *   CK() abort              (render.cu:20)   -> integer status + so_last_error
 *   ~Renderer               (render.cu:526)  -> so_destroy
 *
 * and the host builders that turn a shot .ini into those structs:
 *
 *   Config::load + --set    (common/config.cpp:52, blackholes/src/main.cpp:389-399) -> so_shot_load
 *   build_scene             (blackholes/src/scene_build.cpp:83)                     -> so_shot_scene
 *   build_shot              (blackholes/src/shot.cpp:73)                            -> so_shot_nframes
 *   make_frame              (blackholes/src/shot.cpp:116)                           -> so_shot_frame
 *   find_critical_point     (blackholes/src/shot.cpp:148)                           -> so_find_critical_point
 *   flux normalisation loop (blackholes/src/main.cpp:475-508)                       -> so_normalize_flux
 *
 * so_scene and so_frame have exactly the field order, types and meaning of SceneGPU and FrameGPU, so
 * the reference's structs can be passed by pointer unchanged.  Table pointers inside so_scene are
 * ignored on input: the renderer owns device copies of the tables given to so_init.
 *
 * Every entry point returns SO_OK (0) or a positive SO_ERR_* code and never aborts the process.
 * A renderer is used from one host thread at a time (as the reference's Renderer is).
 */
#ifndef SO_TRACER_H
#define SO_TRACER_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------------------------- */
enum {
    SO_OK = 0,
    SO_ERR_ARG = 1,        /* bad argument (null pointer, size <= 0, inconsistent sizes) */
    SO_ERR_CUDA = 2,       /* a CUDA runtime call failed; so_last_error has the CUDA message */
    SO_ERR_ALLOC = 3,      /* device or host allocation failed */
    SO_ERR_CONFIG = 4,     /* .ini parse error / missing file */
    SO_ERR_NO_DEVICE = 5,  /* no CUDA device, or the kernels were not built for it */
    SO_ERR_STATE = 6,      /* call not valid in the renderer's current state */
    SO_ERR_WATCHDOG = 7,   /* a device-side bounded wait gave up (persistent queue) */
    SO_ERR_SIZE = 8,       /* request larger than a fixed capacity */
    SO_ERR_UNSUPPORTED = 9 /* option outside the implemented path (e.g. the star map in batched frames) */
};

/* ---- enums shared with the reference (scene.hpp:16) ------------------------------------------ */
enum { SO_MODE_VISIBLE = 0, SO_MODE_RADIO = 1 };
/* Ray fates: trace.cuh:59 (+1 escaped, -1 captured, 0 step limit). */
enum { SO_FATE_LIMIT = 0, SO_FATE_ESCAPED = 1, SO_FATE_CAPTURED = -1 };
/* Integrator precision of so_render / so_trace_rays. */
enum { SO_PREC_FP64 = 0, SO_PREC_MIXED = 1 };
/* Hot-flow density / temperature model. */
enum { SO_PLASMA_REFERENCE = 0, SO_PLASMA_TORUS = 1 };

/* ---- geometry PODs (common.hpp:31-42, kerr.hpp:20-25) ---------------------------------------- */
typedef struct so_vec3 { double x, y, z; } so_vec3;
typedef struct so_mat3 { so_vec3 r0, r1, r2; } so_mat3; /* row-major */

typedef struct so_kerr_point {
    double r, s, c;                 /* r, sin(theta), cos(theta) */
    double Sigma, Delta, A, omega;  /* metric functions; omega = frame dragging */
    double e_nu, e_psi;             /* ZAMO lapse, sqrt(g_phiphi) */
    double sqrtSigma, sqrtSigmaDelta;
} so_kerr_point;

/* ---- scene: field-for-field SceneGPU (scene.hpp:18-69) ---------------------------------------- */
typedef struct so_scene {
    double a, rh, r_isco;
    double tol;
    int max_steps;
    double r_escape;
    double r_stop;
    double step_frac;
    int mode;

    int disk_on;
    double disk_rin, disk_rout;
    const float* disk_lnT;
    int disk_n;
    double disk_lr0, disk_dlr;
    float disk_turb_amp;
    float disk_turb_scale;
    float disk_tcorr;
    float disk_ld;
    float disk_fcol;
    float disk_plunge;

    int flow_on;
    double n0;
    double n_index, theta_index;
    double theta0;
    double h_r;
    double beta_p;
    double r_flow_max;
    double nu_obs;
    double rg_cm;
    double flow_kep;
    float flow_turb_amp, flow_turb_scale, flow_tcorr;
    unsigned long long turb_tex[24];
    int turb_nt;
    float turb_lr0, turb_lr1, turb_zmax, turb_d0, turb_dd;
    const float* k2_lntab;
    int k2_n;
    float k2_l0, k2_dl;

    int sky_on;
    unsigned long long sky_tex;
    float sky_scale;
    so_mat3 sky_rot;

    const float* bb_xyz;
    int bb_n;
    float bb_l0, bb_dl;

    uint32_t seed;
} so_scene;

/* ---- frame: field-for-field FrameGPU (scene.hpp:71-80) ---------------------------------------- */
typedef struct so_frame {
    double r, th, ph, t;     /* camera position (Boyer-Lindquist) and coordinate time */
    so_kerr_point kp;        /* metric functions at the camera */
    so_vec3 F, R, U;         /* forward / right / up in the ZAMO frame (e_r, e_theta, e_phi) */
    so_vec3 beta;            /* camera velocity relative to the ZAMO */
    double cx, cy;           /* view-centre offset (tangent-plane units) */
    double pix;              /* tangent-plane units per pixel */
    int W, H, spp;
    uint32_t seed;
} so_frame;

/* Host tables (SceneTables, renderer.hpp:19-23).  Copied to the device by so_init. */
typedef struct so_tables {
    const float* disk_lnT; int disk_n;   /* ln T(r) on the scene's ln r grid */
    const float* k2_ln;    int k2_n;     /* ln K2(1/Theta) */
    const float* bb_xyz;   int bb_n;     /* blackbody XYZ, 3 floats per entry */
} so_tables;

/* RenderSettings (renderer.hpp:25-29). */
typedef struct so_settings { int W, H, spp, spp_max; float target_err; } so_settings;

/* PostParams (renderer.hpp:31-35), applied by so_render as the reference does (render.cu:766-767):
 * bloom in [0, 1] (visible mode), blur_sigma_px (radio mode, applied above 0.5 pixel), hide_direct
 * (radio luminance statistics).  Tone mapping, HUD and image files are outside this library. */
typedef struct so_post { float bloom; double blur_sigma_px; float hide_direct; } so_post;

/* HdrFrame (renderer.hpp:41-46) with caller-owned pixels: px holds W*H*4 floats. */
typedef struct so_hdr_frame { int W, H; float* px; double lum_percentile, lum_max; } so_hdr_frame;

/* RenderStats (renderer.hpp:64-69) plus integrator counters. */
typedef struct so_stats {
    double ms_trace, ms_post;
    long long samples, step_limited;
    long long attempts;   /* DP5(4) step attempts over all samples */
    long long accepted;   /* accepted steps over all samples */
    long long fp64_rays;  /* mixed precision: rays integrated in FP64 end to end (band + re-traced) */
    long long flow_steps; /* accepted steps that evaluated the hot-flow transfer */
    double ms_kernel;     /* device time of the tracer launches (CUDA events), when measured */
    long long attempts_fp32; /* mixed precision: attempts made by the FP32 tracer (the rest are FP64) */
    long long band_rays;  /* mixed precision: rays routed to FP64 by the critical band */
    long long flow_steps_fp32; /* mixed precision: flow steps evaluated by the FP32 tracer */
    double ms_fp32;       /* mixed precision: device time of the FP32 tracer launch (CUDA events) */
    long long redo_turn;  /* mixed precision: FP32 rays re-traced for a radial turning point inside turn_r */
    long long redo_drift; /* mixed precision: FP32 rays re-traced for constraint drift above drift_tol */
    long long redo_limit; /* mixed precision: FP32 rays re-traced after reaching max_steps in FP32 */
    double ms_fp32_trace; /* mixed precision, deferred turbulence: device time of the FP32 geodesic tracer */
    double ms_turb;       /* ... of the batched turbulence sums (ms_fp32 covers tracer + sums + transfer) */
    long long turb_records; /* ... record slots summed (segments in use x 16) */
    long long redo_records; /* ... FP32 rays re-traced in FP64 because the record pool ran out */
    long long record_waves; /* ... waves the FP32 rays were traced in (the pool holds one wave's records) */
    double ms_rec64;      /* plain FP64, deferred passes (torus plasma; reference flow frames): device
                             time of the recording pass */
    double ms_sum64;      /* ... of the FP64 turbulence sums over all records (k_turb64_records) */
    double ms_replay64;   /* ... of the replay pass (geodesic again, sums read back, emission); with
                             deferred emission it runs only when the record pool ran out */
    long long rec64_slots; /* ... record slots summed (segments taken x 16) */
    long long rec64_short; /* ... samples summed in the tracer because the record pool ran out */
    long long rec64_records; /* ... records written (flow steps that needed a sum, up to each ray's end) */
    double ms_emit64;     /* ... deferred emission: device time of the emission at every record and the
                             ordered transfer (0 when the replay pass does the emission) */
    int emit64;           /* ... 1 = the last trace deferred its emission too, 0 = replay pass */
    int rec64_waves;      /* ... waves the last deferred trace ran in (the pool holds one wave) */
} so_stats;

/* Per-ray outputs of so_trace_rays.  Each pointer is a caller-owned host array, or NULL to skip. */
typedef struct so_rays_out {
    int8_t* fate;          /* SO_FATE_* */
    int8_t* ncross;        /* equatorial crossings (winding order), saturates at 127 */
    double* theta;         /* escape direction at infinity (escaped rays), else 0 */
    double* phi;
    float* I;              /* 4 floats per ray: trace_ray's accumulated value (trace.cuh:57-61) */
    int32_t* n_accepted;   /* accepted DP5(4) steps */
    int32_t* n_attempts;   /* DP5(4) step attempts */
    double* cross_r;       /* 3 per ray: Boyer-Lindquist r of the first 3 equatorial crossings, 0 if none */
    double* cross_g;       /* 3 per ray: redshift g = nu_obs/nu_emit of a circular prograde emitter there */
} so_rays_out;

/* Analytic torus plasma with Fourier-mode turbulence (the 1024^2 synchrotron frame):
 *   n_e  = n0 (r/r_+)^-ne_index exp(-z^2 / (2 (h_sph r)^2)) exp(delta - rms^2/2) (1 - e^{-(r-r_+)^2/0.25})
 *   T_e  = te0_kelvin (r/r_+)^-te_index
 *   delta = sum_m amp_m cos(k_m . X + phase_m),  X = (R cos phi_c, R sin phi_c, z),
 *   phi_c = phi - Omega_f(R) t  (the pattern is carried by the flow's angular velocity)
 * Field meaning of B, the flow velocity (flow_kep * Keplerian) and the transfer are the reference's
 * flow_step (emission.cuh:99-175).  Modes are drawn on the host from turb_seed by so_plasma_modes. */
typedef struct so_plasma {
    int model;               /* SO_PLASMA_REFERENCE (scene.hpp flow fields) or SO_PLASMA_TORUS */
    double ne_index;         /* 1.5 */
    double te0_kelvin;       /* 1e11 */
    double te_index;         /* 0.84 */
    double h_sph;            /* 0.3: Gaussian width of z in units of r */
    int n_modes;             /* number of Fourier modes, <= SO_MAX_MODES; 0 = no turbulence */
    double turb_rms;         /* rms of delta */
    double k_min, k_max;     /* |k| range, radians per M */
    double spectral_index;   /* 3-D power spectrum slope, -11/3 */
    uint32_t turb_seed;
} so_plasma;
#define SO_MAX_MODES 1024
/* One Fourier mode: wave vector (rad/M), phase (rad), amplitude. */
typedef struct so_mode { double kx, ky, kz, phase, amp; } so_mode;

/* Mixed-precision routing options (SO_PREC_MIXED).  A ray is integrated in FP64 from the camera
 * down to r_switch, then in FP32 with two-sum compensated state; rays inside the critical band are
 * FP64 throughout; an FP32 ray whose radial turning point falls inside turn_r, or whose
 * Carter-constant drift (checked in FP64 at the end) exceeds drift_tol, is re-integrated in FP64. */
typedef struct so_mixed_opts {
    double band_m;           /* FP64 for rays within this distance (M) of the analytic critical curve */
    double tol32;            /* FP32 integrator tolerance (reference error norm) */
    double turn_r;           /* radial turning point inside this radius (M): re-trace in FP64 (0 = off) */
    double drift_tol;        /* relative drift of p_u^2 - U(u) and p_r^2 - R(r) that triggers FP64 */
    double r_switch;         /* FP64 approach from the camera down to this radius (0 = automatic) */
    double tol_approach;     /* tolerance of the FP64 approach (0 = 10 x the scene's render.tolerance: the
                              * far field carries no emission, and the synchrotron frame's image moves
                              * by 2e-5 L1 and keeps every class for it, at 7 % less frame time) */
    int t32_blocks;          /* FP32 tracer: resident 128-thread CTAs per SM, 4, 5 or 6 (0 = 4) */
    int turbulence;          /* torus turbulence of the FP32 rays: 0 = deferred (the tracer records its
                              * emitting flow steps, one batched kernel sums the Fourier modes at all of
                              * them, one kernel runs the ordered transfer per ray; the record pool takes
                              * up to half of the free device memory), 1 = summed in the tracer
                              * (warp-cooperative, interleaved with the geodesic work) */
    int approach;            /* FP64 approach integrator: 0 = DP5(4) in the inverse radius 1/r on ingoing
                              * legs without a radial turning point above r_switch (a few steps where
                              * Mino time takes hundreds from a distant camera; other rays as 1),
                              * 1 = the reference's Mino-time DP5(4) for every ray */
    double records_per_ray;  /* deferred turbulence: record pool per FP32 ray at the renderer's first
                              * mixed frame (0 = 320; doubled after a frame that ran short, whose rays
                              * without a record slot are re-traced in FP64) */
    int sky_fp32;            /* visible frames with the star map: 0 = traced in FP64 (default, the plain
                              * image), 1 = FP32 rays off the band, their escape carried to r_escape in
                              * FP64 (~1.9x faster; escape directions within ~1e-6 rad, which shows
                              * where a magnified map is steep: L1 5e-3 on a point-star test map) */
    double pool_mb;          /* deferred turbulence: record pool size limit in MiB (0 = half of the free
                              * device memory); a frame whose records exceed it is traced in waves of
                              * FP32 rays that each fit (the image does not depend on the split).  Also
                              * caps the plain FP64 tracer's record pool (torus plasma, in either
                              * precision), beyond which samples are summed in the tracer: the same
                              * sums, bit for bit, at lower occupancy */
    int fp32_max_attempts;   /* FP32 attempts after which a ray is handed to the FP64 re-trace (0 = 2000:
                              * the FP32 controller stalls on a few rays far from the critical curve,
                              * which the FP64 tracer finishes normally; at 2048^2 the synchrotron
                              * frame's longest normal FP32 ray takes fewer) */
} so_mixed_opts;

/* ---- renderer lifecycle ---------------------------------------------------------------------- */
typedef struct so_renderer so_renderer;

/* Renderer::init (render.cu:531-656).  Creates the CUDA stream, uploads the tables and allocates
 * the frame buffers for rs->W x rs->H.  The star map (Renderer::init's SkyTexture) is given
 * afterwards by so_set_sky.
 * On failure *out is NULL and the status says why (no process abort). */
int so_init(so_renderer** out, int device, const so_scene* scene, const so_tables* tables,
            const so_settings* rs);
/* Renderer::update_scene (render.cu:658-675): scalar parameters only, tables stay. */
int so_update_scene(so_renderer* r, const so_scene* scene);
/* Renderer::render (render.cu:755-795): pass 1, adaptive pass 2, resolve; out->px is W*H*4 floats
 * owned by the caller.  f->W, f->H, f->spp are taken from the settings, as the reference does. */
int so_render(so_renderer* r, const so_frame* f, const so_post* post, double percentile,
              so_hdr_frame* out, so_stats* stats);
/* Renderer::radio_flux (render.cu:797-809): n x n frame, spp = 2, total flux density in Jy. */
int so_radio_flux(so_renderer* r, const so_frame* f, int n, double pix_sr, double* jy);
/* trace_ray (trace.cuh:62-165) for n explicit tangent-plane coordinates (x[i], y[i]) of frame f.
 * Host arrays in, host arrays out. */
int so_trace_rays(so_renderer* r, const so_frame* f, int n, const double* x, const double* y,
                  const so_rays_out* out);
/* so_render's tracing part with the HDR frame left in caller-owned DEVICE memory d_px (W*H*4
 * floats): pass 1, adaptive pass 2 and resolve, queued on so_stream(r).  With stats == NULL the
 * call does not synchronise; with stats it waits and fills the counters and ms_trace (device time
 * of the tracer launches, CUDA events). */
int so_render_device(so_renderer* r, const so_frame* f, float* d_px, so_stats* stats);
/* Renderer::radio_flux for callers that cannot allocate device memory (a process whose device
 * memory belongs to a pool or arena, a real-time loop that allocates only up front, a plugin host
 * that forbids allocation in its callbacks).  No reference counterpart: it needs no renderer and
 * calls no cudaMalloc / cudaFree.  The caller passes, in memory it owns: d_scene (device so_scene of
 * a radio scene whose table pointers are device pointers), d_frame (device so_frame built for width
 * n), plasma (host; NULL = the reference flow model) with its device modes d_modes, and d_jy (device
 * double that receives the flux density in Jy).  The n x n frame is traced at 2 samples per pixel,
 * with so_radio_flux's kernels in its order, asynchronously on `stream` (a cudaStream_t; NULL =
 * default stream).  A turbulent reference-model flow (plasma NULL, flow turbulence on) evaluates the
 * sheared noise at every flow step: the result equals so_radio_flux's on a renderer switched to
 * SO_FLOW_NOISE_INLINE, and differs from its default baked slices (another draw of the turbulence).
 * Working memory is a fixed device array of the library, SO_NOALLOC_MAX_PIXELS float4 plus 5.4 KB,
 * held by every GPU that loads the library until the process exits: n*n above SO_NOALLOC_MAX_PIXELS
 * returns SO_ERR_SIZE (message in so_last_error(NULL)).  The first call on a device looks the array
 * up (cudaGetSymbolAddress) with that device current; make it before any stream capture, and do not
 * reset the device (cudaDeviceReset) between calls.  All calls share the array, so calls that overlap
 * on the GPU race: order them on one stream. */
#define SO_NOALLOC_MAX_PIXELS 65536
int so_radio_flux_noalloc(const so_scene* d_scene, const so_frame* d_frame, int n, double pix_sr,
                          const so_plasma* plasma, const so_mode* d_modes, double* d_jy, void* stream);
/* Same as so_trace_rays with x, y and the outputs already in device memory (device pointers). */
int so_trace_rays_device(so_renderer* r, const so_frame* f, int n, const double* d_x, const double* d_y,
                         const so_rays_out* d_out);
/* Counters of the last so_trace_rays / so_trace_rays_device call (waits for it): samples (its rays),
 * attempts, accepted, flow_steps, step_limited, and whether and how its emission was deferred
 * (emit64, rec64_*, ms_rec64 .. ms_replay64); every other field 0.  No reference counterpart.
 * SO_ERR_STATE when a frame or batch was rendered after it, or no list was traced. */
int so_trace_stats(so_renderer* r, so_stats* stats);
/* The star map of Renderer::init's SkyTexture (renderer.hpp:14-17, render.cu:550-593): w x h texels
 * of half2 (brightness s, s T / 1e4) as 16-bit halves, row-major.  Made a mipmapped texture (box-
 * filtered levels down to 1 x 1) sampled as the reference samples it (bilinear and between levels,
 * anisotropy up to 16, u wrapped, v clamped).  Used when the scene given to so_init asked for the sky
 * (sky_on) and the mode is visible: every frame then traces the (W + 1) x (H + 1) pixel corners first
 * (k_corners) for the pixel footprints, and each escaping sample adds the star map's blackbody
 * radiance through its footprint (trace.cuh:149-161).  Without so_set_sky no sky is drawn, as the
 * reference without a texture.  Frames with the sky run in FP64 on the mixed path too. */
int so_set_sky(so_renderer* r, int w, int h, const uint16_t* data);
/* load_sky (scene_build.cpp:61-81): a .bhsk star map (uint32 magic "BHSK", width, height, float
 * brightness scale, then width x height half2 texels).  With data NULL only the header is read
 * (w, h, scale); else data receives w * h * 2 halves.  The reference multiplies sky.brightness
 * (so_scene.sky_scale) by the file's scale (main.cpp:461-467).  SO_ERR_CONFIG for a missing or bad
 * file. */
int so_sky_file(const char* path, int* w, int* h, float* scale, uint16_t* data);

/* Flow turbulence of the reference plasma model (radio mode, flow.turbulence > 0).
 * SO_FLOW_NOISE_BAKED (so_init's choice, as Renderer::init's, render.cu:594-620): before every
 * trace of a frame its turbulence is baked into 24 retarded-time slices of 512 x 192 x 48 density
 * factors on (phi, ln R, z/R) (453 MB of device memory, render.cu:449-460, 679-682) held as 3-D
 * arrays, and each flow step reads two of them through the texture unit with the reference's sampler
 * and interpolates in time (emission.cuh:112-124): the reference's own fetch, trilinear weights with 8
 * fractional bits.  SO_FLOW_NOISE_BAKED_FP32 keeps the slices in plain device memory and
 * interpolates them in FP32 with a fixed operation order, which the CPU oracle repeats exactly.
 * SO_FLOW_NOISE_INLINE evaluates the sheared fBm noise at every flow step (the reference's
 * turb_nt = 0 path) and frees the slices.  No effect on other plasma models.  The batched frames
 * (so_batch_*) and so_radio_flux_noalloc always evaluate the noise in place. */
enum { SO_FLOW_NOISE_BAKED = 0, SO_FLOW_NOISE_INLINE = 1, SO_FLOW_NOISE_BAKED_FP32 = 2 };
int so_set_flow_noise(so_renderer* r, int mode);

/* Precision and plasma extensions (no reference counterpart: the reference has one FP64 path and
 * the scene.hpp flow model). */
int so_set_precision(so_renderer* r, int precision, const so_mixed_opts* opts);
int so_set_plasma(so_renderer* r, const so_plasma* plasma, const so_mode* modes);
/* Termination class (SO_FATE_*) of every sample of the last mixed-precision frame (samples in
 * pixel-major order, spp per pixel) and whether the sample was routed to FP64 by the critical band
 * (1) or not (0); host arrays of n = W * H * spp entries, either may be NULL.  For checking that the
 * mixed path's classes outside the band are the FP64 ones.  No reference counterpart. */
int so_last_fates(so_renderer* r, int8_t* fate, uint8_t* in_band, long long n);
/* CUDA stream used by the renderer (cudaStream_t, as void*), for callers that order work on it. */
void* so_stream(so_renderer* r);
/* Message of the last failed call on r.  With r NULL: of the last failed call without a renderer
 * (so_init, so_shot_load, so_radio_flux_noalloc, so_sur_gemm) made by the calling thread. */
const char* so_last_error(const so_renderer* r);
/* Frees the renderer.  Batches made on it and not yet freed are detached: so_batch_render and
 * so_batch_autotune on them return SO_ERR_STATE, and so_batch_free still frees them. */
void so_destroy(so_renderer* r);

/* ---- batched frames: the persistent wavefront (no reference counterpart) --------------------- */
/* A batch of nframes frames of W x H pixels x spp samples, traced by ONE persistent FP64 launch:
 * the rays of all frames share one work queue, so frames of very different cost (spins, photon-ring
 * zooms, turbulence times) keep every lane busy until the last ray.  Frame i uses
 * scenes[frame_scene[i]]; every scene must have the same mode and use the renderer's tables (those
 * of so_init: the K2 and blackbody tables do not depend on the scene, the disk table depends on the
 * spin, so disk scenes must share a spin).  The plasma is the renderer's (so_set_plasma).  The launch
 * sequence (counter reset, tracer, resolve) is captured once into a CUDA graph and replayed.  A radio
 * batch of 4096 jobs or more (no disk) traces in deferred passes instead: a persistent recording
 * pass over all frames, the torus plasma's turbulence sums at its records (FP32 under
 * SO_PREC_MIXED, FP64 otherwise; none for the reference flow model, whose noise a batch evaluates
 * in place), the emission and the ordered transfer, in waves through the renderer's record pool
 * (sized before the capture, within so_mixed_opts.pool_mb); a batch that ran short of records is
 * captured again with a larger pool at its next so_batch_render. */
typedef struct so_batch so_batch;
/* Launch shape of the batch: resident CTAs per SM of the persistent grid (0 = as many as fit); the
 * job order (0 = frame after frame, 1 = frames interleaved in tiles of `tile` consecutive pixels,
 * tile <= 1 meaning ray by ray; a tile that does not divide W * H is lowered to the largest power of
 * two that does); and the queue chunk, the consecutive jobs a lane takes per grab from the shared
 * queue (<= 1: one).  None of them changes any ray's result.  ms: the batch time the tuner measured. */
typedef struct so_tune { int ctas_per_sm; int interleave; double ms; int tile; int queue_chunk; } so_tune;
int so_batch_create(so_renderer* r, const so_scene* scenes, int nscenes, const so_frame* frames,
                    const int* frame_scene, int nframes, int W, int H, int spp, so_batch** out);
/* Traces the batch into d_px (device memory, nframes * W * H * 4 floats, frame after frame) by
 * replaying the batch's CUDA graph on so_stream(r).  With stats: waits, fills the counters and
 * ms_kernel (graph time, CUDA events), and for deferred passes the rec64_* fields; without:
 * asynchronous. */
int so_batch_render(so_batch* b, float* d_px, so_stats* stats);
/* Autotuner: times every launch shape (CTAs per SM from 1 to the occupancy limit, both job orders)
 * on the batch, keeps the fastest for later so_batch_render calls and returns it in *best. */
int so_batch_autotune(so_batch* b, float* d_px, so_tune* best);
int so_batch_set_tune(so_batch* b, const so_tune* t);
void so_batch_free(so_batch* b);

/* ---- ray surrogate (no reference counterpart) ------------------------------------------------- */
/* A small MLP that maps an image-plane ray of a static camera -- Bardeen coordinates alpha, beta
 * (M), spin a, inclination (degrees) -- to what the FP64 integrator reports for it: termination
 * class, escape direction, and the radius and redshift of its first three equatorial crossings.
 * 64 Gaussian random frequencies of the inputs scaled to [-1, 1] give 128 features (sin, cos);
 * 4 hidden layers of 256 with tanh-form GELU; 12 outputs.  BF16 weights and activations with FP32
 * accumulation in tensor memory (tcgen05 kernels of this library), FP32 master weights, AdamW.
 * All pointers named d_* are device memory. */
#define SO_SUR_NFREQ 64
#define SO_SUR_HIDDEN 256
#define SO_SUR_LAYERS 4
#define SO_SUR_NOUT 12
#define SO_SUR_LDOUT 16 /* floats per output row (12 used) */
#define SO_SUR_NPARAMS 234512
typedef struct so_surrogate so_surrogate;
typedef struct so_sur_ray { float alpha, beta, spin, incl_deg; } so_sur_ray;
/* What the integrator reported for a ray.  Output row of the network: [0..2] class logits,
 * [3..5] direction, [6..8] u, [9..11] g. */
typedef struct so_sur_target {
    float cls;    /* 0 escaped, 1 captured, 2 step limit */
    float dir[3]; /* escape direction (sin th cos ph, sin th sin ph, cos th); 0 unless escaped */
    float u[3];   /* 1/r of the first three equatorial crossings; where there is none: 0 for a ray
                   * that escapes, 1/r_stop (where the integrator stopped) for one that is captured */
    float g[3];   /* redshift of a circular prograde emitter at those radii (0 inside the ISCO);
                   * -1 where there is no crossing (not trained on) */
    float pad[2];
} so_sur_target;
typedef struct so_sur_opts {
    float fourier_sigma;   /* std of the frequencies per unit of the scaled inputs */
    uint32_t seed;         /* frequencies and initial weights */
    int batch;             /* rays per optimiser step, a multiple of 128 */
    float lr, lr_final;    /* cosine schedule over the steps of one so_sur_train call */
    int warmup;            /* linear warm-up steps of that schedule */
    float beta1, beta2, eps, weight_decay;
    float w_dir, w_u, w_g; /* loss weights of direction, 1/r and redshift (class cross-entropy: 1) */
} so_sur_opts;
/* Mean loss terms per ray; accuracy = fraction of rays whose largest class logit is the target's. */
typedef struct so_sur_loss { double total, ce, dir, u, g, accuracy; long long rays; } so_sur_loss;
void so_sur_default_opts(so_sur_opts* o);
int so_sur_create(int device, const so_sur_opts* o, so_surrogate** out);
void so_sur_destroy(so_surrogate* s);
/* Master parameters (host, SO_SUR_NPARAMS floats: per layer weight [N x K] row-major then bias;
 * layer 0 256 x 128, layers 1-3 256 x 256, head 16 x 256 with rows 12-15 zero) and frequencies
 * (host, SO_SUR_NFREQ x 4).  Either pointer may be NULL. */
int so_sur_get_params(so_surrogate* s, float* params, float* freqs);
int so_sur_set_params(so_surrogate* s, const float* params, const float* freqs);
/* `steps` AdamW steps over n device rays / targets, batches taken cyclically (ray i of step k is
 * (k * batch + i) mod n); *last gets the loss of the last step. */
int so_sur_train(so_surrogate* s, const so_sur_ray* d_rays, const so_sur_target* d_tgt, long long n, int steps,
                 so_sur_loss* last);
/* Loss over the first n - n % 128 rays, no update. */
int so_sur_evaluate(so_surrogate* s, const so_sur_ray* d_rays, const so_sur_target* d_tgt, long long n,
                    so_sur_loss* loss);
/* One forward and backward pass over n rays (n % 128 == 0) at the current parameters, no update:
 * gradient of the mean loss in the master-parameter layout (host, SO_SUR_NPARAMS floats). */
int so_sur_gradients(so_surrogate* s, const so_sur_ray* d_rays, const so_sur_target* d_tgt, int n, float* grads,
                     so_sur_loss* loss);
/* Network outputs for n rays: d_out, n x SO_SUR_LDOUT floats.  Queued on `stream` (NULL = the
 * surrogate's own stream); the call returns once the work is queued. */
int so_sur_infer(so_surrogate* s, const so_sur_ray* d_rays, long long n, float* d_out, void* stream);
/* Form of the fused inference kernel: 1 CTA per SM (default; a 256-ray tile as two M=128 MMA
 * halves) or 2 (cluster pairs issuing cta_group::2 MMAs of M=256, each SM streaming half of every
 * weight chunk; measured slower on B200).  Both compute the same outputs to FP32 rounding; a
 * refused cluster launch falls back to 1. */
int so_sur_set_infer_ctas(so_surrogate* s, int ctas);
/* Training set from the FP64 integrator of renderer r: `groups` (spin, inclination) pairs drawn
 * uniformly from the ranges, n / groups rays each with alpha, beta uniform in [-xy_max, xy_max],
 * traced in vacuum from a static camera at f->r.  Stored interleaved (ray j of group g at
 * j * groups + g) so that consecutive rays come from different groups; all groups are traced by
 * one persistent launch.  The renderer's own scene and frame are left as they are. */
typedef struct so_sur_ranges { double a_min, a_max, incl_min, incl_max, xy_max; } so_sur_ranges;
int so_sur_dataset(so_renderer* r, const so_frame* f, long long n, int groups, uint32_t seed,
                   const so_sur_ranges* ranges, so_sur_ray* d_rays, so_sur_target* d_tgt, so_stats* stats);
/* Thin-disk frame through the surrogate: every pixel centre inside band_m of the analytic critical
 * curve goes to the FP64 integrator; of the others a random audit_frac sample (seeded) goes to the
 * integrator as well, and the surrogate shades the rest from its predicted crossing radii (the
 * redshift is the exact one of that radius and the ray's constants of motion).  The integrator
 * checks the surrogate on the audit rays.  Renderer r holds a visible-mode disk scene (no disk
 * turbulence); d_px is W x H x 4 floats of device memory, the same quantity so_trace_rays reports
 * as I at the pixel centres. */
typedef struct so_sur_frame_opts { double band_m, audit_frac; uint32_t audit_seed; } so_sur_frame_opts;
typedef struct so_sur_report {
    long long rays, surrogate_rays, band_rays, audit_rays;
    double ms_total, ms_route, ms_mlp, ms_shade, ms_integrator;
    /* surrogate against the integrator on the audit rays */
    long long audit_class_mismatch;
    double audit_dir_err;   /* mean angle between escape directions (rad), rays both call escaped */
    double audit_u_err;     /* mean |u - u_true| over the crossings the integrator found */
    double audit_r_err;     /* mean |r - r_true| / r_true over the crossings inside r = 50 */
    double audit_g_err;     /* mean |g - g_true| of the network's redshift head over those crossings */
    double audit_l1;        /* sum |I - I_true| / sum |I_true| of the Y channel */
    double audit_flux;      /* sum I / sum I_true - 1 of the Y channel */
} so_sur_report;
int so_sur_render(so_surrogate* s, so_renderer* r, const so_frame* f, const so_sur_frame_opts* o, float* d_px,
                  so_sur_report* rep);
/* The surrogate's tensor-core GEMM on its own, for numerics checks.  A [M x K] and B [N x K] are
 * BF16 row-major device arrays; M % 128 == 0, N <= 256 with N % 16 == 0 or N % 256 == 0,
 * (K / splits) % 16 == 0.  layout 0: d_c[m * N + n] = (A B^T)[m, n] + bias[n] (splits must be 1,
 * bias may be NULL); layout 1: d_c[s * M * N + m * N + n] = slice s of the reduction; layout 2:
 * d_c[s * M * N + n * M + m] = the same, transposed.  Synchronous; status as elsewhere. */
int so_sur_gemm(const void* d_a, const void* d_b, const float* d_bias, float* d_c, int M, int N, int K, int splits,
                int layout);

/* ---- shot / scene builders (host only) --------------------------------------------------------- */
typedef struct so_shot so_shot;
/* Scene information that does not go to the device (SceneInfo, scene_build.hpp:7-17). */
typedef struct so_scene_info {
    double mass_msun, distance_cm, rg_cm, tg_s, uas_per_m, disk_tmax, disk_mdot_edd;
    double radio_flux_target_jy;
} so_scene_info;
/* Loads a shot .ini (with include = ...) and applies "section.key=value" overrides. */
int so_shot_load(const char* ini_path, const char* const* overrides, int n_overrides, so_shot** out);
/* build_scene: scene scalars plus host tables owned by the shot (valid until so_shot_free). */
int so_shot_scene(const so_shot* s, so_scene* scene, so_tables* tables, so_scene_info* info);
/* RenderSettings from camera.width/height, render.spp/spp_max/target_error (main.cpp:410-415). */
int so_shot_settings(const so_shot* s, so_settings* rs);
int so_shot_nframes(const so_shot* s);
/* make_frame for frame index i; W is the image width used for the pixel scale. */
int so_shot_frame(const so_shot* s, int i, int W, uint32_t seed, so_frame* f);
/* find_critical_point on frame i's camera along image direction psi (rad); rho in M. */
int so_find_critical_point(const so_shot* s, int i, double a, double psi, double* rho);
/* State (r, r', u, u', phi, t) of the backward ray through image-plane point (x, y) of frame f
 * where it reaches radius r1 (< f->r), on the host (no device): method 0 = the mixed path's
 * far-field transport (DP5(4) in the inverse radius 1/r, landing exactly on r1), 1 = the reference's
 * Mino-time DP5(4) at tolerance tol, its last step shortened to stop within 1e-12 r1 above r1 (the
 * state then has that radius).  *attempts (may be NULL) gets the DP5 attempts.  SO_ERR_ARG where the
 * method does not apply (an outgoing ray, a radial turning point above r1; for method 0 also a
 * turning point near r1).  No reference counterpart: a check of the approach integrators. */
int so_approach_state(const so_scene* s, const so_frame* f, double x, double y, double r1, double tol, int method,
                      double* state, int* attempts);
/* Configuration value lookup (string form), for callers mirroring main.cpp's cfg.* reads. */
int so_shot_get(const so_shot* s, const char* key, char* buf, int buflen);
void so_shot_free(so_shot* s);
/* Flux normalisation of the hot flow (main.cpp:475-508): secant on ln n0 over radio_flux on an
 * n x n frame of width fov_m; updates the renderer's scene and returns the new n0. */
int so_normalize_flux(so_renderer* r, so_scene* scene, const so_frame* f_wide, int n, double pix_sr,
                      double target_jy, double* n0_out, double* jy_out);
/* Fourier modes of a torus plasma, drawn deterministically from p->turb_seed (p->n_modes entries). */
int so_plasma_modes(const so_plasma* p, so_mode* modes);

/* ---- measurement helper (no reference counterpart) --------------------------------------------- */
/* Peak FP64 / FP32 FMA throughput of `device` in TFLOP/s (FMA = 2 flops), measured by independent
 * FMA chains on every SM and timed with CUDA events: the roofline denominator for the tracers. */
int so_probe_fma_peak(int device, double* fp64_tflops, double* fp32_tflops);
/* Peak special-function-unit throughput (FP32 cosines, G ops/s) of `device`: the roofline of the
 * FP32 tracer, whose turbulence sum issues one SFU cosine per Fourier mode. */
int so_probe_sfu_peak(int device, double* gops);
/* The device's cos_turns (cos(2 pi t) of a phase in turns, used by the FP64 torus turbulence sums)
 * at n phases d_t[i] into d_out[i] (device arrays, current device; synchronous): for checking it
 * against the CPU oracle's restatement. */
int so_probe_cos_turns(const double* d_t, double* d_out, long long n);

/* ---- analytic helpers (kerr.hpp) --------------------------------------------------------------- */
/* kerr_point (kerr.hpp:27-42). */
void so_kerr_point_at(double a, double r, double th, so_kerr_point* kp);
/* critical_curve_point (kerr.hpp:210-220): Bardeen curve point for photon-orbit radius rp. */
int so_critical_curve_point(double a, double theta_o, double rp, double* alpha, double* beta_plus);

#ifdef __cplusplus
}
#endif

#endif /* SO_TRACER_H */
