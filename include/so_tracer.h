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
    SO_ERR_UNSUPPORTED = 9 /* option outside the implemented path (e.g. sky texture lookups) */
};

/* ---- enums shared with the reference (scene.hpp:16) ------------------------------------------ */
enum { SO_MODE_VISIBLE = 0, SO_MODE_RADIO = 1 };
/* Ray fates: trace.cuh:59 (+1 escaped, -1 captured, 0 step limit). */
enum { SO_FATE_LIMIT = 0, SO_FATE_ESCAPED = 1, SO_FATE_CAPTURED = -1 };
/* Integrator precision of so_render / so_trace_rays. */
enum { SO_PREC_FP64 = 0, SO_PREC_MIXED = 1 };
/* Hot-flow density / temperature model. */
enum { SO_PLASMA_REFERENCE = 0, SO_PLASMA_TORUS = 1 };

/* ---- geometry PODs (common.hpp:31-42, kerr.hpp:70-75) ---------------------------------------- */
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

/* PostParams (renderer.hpp:31-35).  blur_sigma_px > 0.5 and bloom > 0 return SO_ERR_UNSUPPORTED
 * (display post-processing is outside this library). */
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
    double tol_approach;     /* tolerance of the FP64 approach (0 = the scene's render.tolerance) */
    int t32_blocks;          /* FP32 tracer: resident 128-thread CTAs per SM, 4, 5 or 6 (0 = 4) */
} so_mixed_opts;

/* ---- renderer lifecycle ---------------------------------------------------------------------- */
typedef struct so_renderer so_renderer;

/* Renderer::init (render.cu:531-656).  Creates the CUDA stream, uploads the tables and allocates
 * the frame buffers for rs->W x rs->H.  The sky texture is not supported (scene->sky_on must be 0).
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
 * as so_radio_flux does, asynchronously on `stream` (a cudaStream_t; NULL = default stream).
 * Working memory is a fixed device array of the library, SO_NOALLOC_MAX_PIXELS float4 plus 5.4 KB,
 * held by every GPU that loads the library until the process exits: n*n above SO_NOALLOC_MAX_PIXELS
 * returns SO_ERR_SIZE (message in so_last_error(NULL)).  The first call on a device looks the array
 * up (cudaGetSymbolAddress) with that device current; make it before any stream capture.  All calls
 * share the array, so calls that overlap on the GPU race: order them on one stream. */
#define SO_NOALLOC_MAX_PIXELS 65536
int so_radio_flux_noalloc(const so_scene* d_scene, const so_frame* d_frame, int n, double pix_sr,
                          const so_plasma* plasma, const so_mode* d_modes, double* d_jy, void* stream);
/* Same as so_trace_rays with x, y and the outputs already in device memory (device pointers). */
int so_trace_rays_device(so_renderer* r, const so_frame* f, int n, const double* d_x, const double* d_y,
                         const so_rays_out* d_out);
/* Precision and plasma extensions (no reference counterpart: the reference has one FP64 path and
 * the scene.hpp flow model). */
int so_set_precision(so_renderer* r, int precision, const so_mixed_opts* opts);
int so_set_plasma(so_renderer* r, const so_plasma* plasma, const so_mode* modes);
/* CUDA stream used by the renderer (cudaStream_t, as void*), for callers that order work on it. */
void* so_stream(so_renderer* r);
/* Message of the last failed call on r (or of the last failed so_init when r is NULL). */
const char* so_last_error(const so_renderer* r);
void so_destroy(so_renderer* r);

/* ---- batched frames: the persistent wavefront (no reference counterpart) --------------------- */
/* A batch of nframes frames of W x H pixels x spp samples, traced by ONE persistent FP64 launch:
 * the rays of all frames share one work queue, so frames of very different cost (spins, photon-ring
 * zooms, turbulence times) keep every lane busy until the last ray.  Frame i uses
 * scenes[frame_scene[i]]; every scene must have the same mode and use the renderer's tables (those
 * of so_init: the K2 and blackbody tables do not depend on the scene, the disk table depends on the
 * spin, so disk scenes must share a spin).  The plasma is the renderer's (so_set_plasma).  The launch
 * sequence (counter reset, tracer, resolve) is captured once into a CUDA graph and replayed. */
typedef struct so_batch so_batch;
/* Launch shape of the batch: resident CTAs per SM of the persistent grid (0 = as many as fit), and
 * the job order (0 = frame after frame, 1 = frames interleaved ray by ray). */
typedef struct so_tune { int ctas_per_sm; int interleave; double ms; } so_tune;
int so_batch_create(so_renderer* r, const so_scene* scenes, int nscenes, const so_frame* frames,
                    const int* frame_scene, int nframes, int W, int H, int spp, so_batch** out);
/* Traces the batch into d_px (device memory, nframes * W * H * 4 floats, frame after frame) by
 * replaying the batch's CUDA graph on so_stream(r).  With stats: waits, fills the counters and
 * ms_kernel (graph time, CUDA events); without: asynchronous. */
int so_batch_render(so_batch* b, float* d_px, so_stats* stats);
/* Autotuner: times every launch shape (CTAs per SM from 1 to the occupancy limit, both job orders)
 * on the batch, keeps the fastest for later so_batch_render calls and returns it in *best. */
int so_batch_autotune(so_batch* b, float* d_px, so_tune* best);
int so_batch_set_tune(so_batch* b, const so_tune* t);
void so_batch_free(so_batch* b);

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

/* ---- analytic helpers (kerr.hpp) --------------------------------------------------------------- */
/* kerr_point (kerr.hpp:77-92). */
void so_kerr_point_at(double a, double r, double th, so_kerr_point* kp);
/* critical_curve_point (kerr.hpp:260-270): Bardeen curve point for photon-orbit radius rp. */
int so_critical_curve_point(double a, double theta_o, double rp, double* alpha, double* beta_plus);

#ifdef __cplusplus
}
#endif

#endif /* SO_TRACER_H */
