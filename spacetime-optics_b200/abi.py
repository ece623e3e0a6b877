"""ctypes mirror of include/so_tracer.h (the C ABI of the tracer library).

The struct layouts follow the header field for field; so_scene / so_frame in turn follow the
reference's SceneGPU / FrameGPU (blackholes/src/scene.hpp:12-80), which tests check against the
reference's own offsets.
"""
import ctypes as C

SO_OK = 0
SO_ERR_ARG, SO_ERR_CUDA, SO_ERR_ALLOC, SO_ERR_CONFIG, SO_ERR_NO_DEVICE = 1, 2, 3, 4, 5
SO_ERR_STATE, SO_ERR_WATCHDOG, SO_ERR_SIZE, SO_ERR_UNSUPPORTED = 6, 7, 8, 9
SO_MODE_VISIBLE, SO_MODE_RADIO = 0, 1
SO_FATE_LIMIT, SO_FATE_ESCAPED, SO_FATE_CAPTURED = 0, 1, -1
SO_PREC_FP64, SO_PREC_MIXED = 0, 1
SO_PLASMA_REFERENCE, SO_PLASMA_TORUS = 0, 1
SO_FLOW_NOISE_BAKED, SO_FLOW_NOISE_INLINE, SO_FLOW_NOISE_BAKED_FP32 = 0, 1, 2
SO_MAX_MODES = 1024


class Vec3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class Mat3(C.Structure):
    _fields_ = [("r0", Vec3), ("r1", Vec3), ("r2", Vec3)]


class KerrPoint(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("r", "s", "c", "Sigma", "Delta", "A", "omega", "e_nu", "e_psi", "sqrtSigma", "sqrtSigmaDelta")]


class Scene(C.Structure):
    _fields_ = [
        ("a", C.c_double), ("rh", C.c_double), ("r_isco", C.c_double), ("tol", C.c_double),
        ("max_steps", C.c_int), ("r_escape", C.c_double), ("r_stop", C.c_double), ("step_frac", C.c_double),
        ("mode", C.c_int),
        ("disk_on", C.c_int), ("disk_rin", C.c_double), ("disk_rout", C.c_double),
        ("disk_lnT", C.POINTER(C.c_float)), ("disk_n", C.c_int), ("disk_lr0", C.c_double), ("disk_dlr", C.c_double),
        ("disk_turb_amp", C.c_float), ("disk_turb_scale", C.c_float), ("disk_tcorr", C.c_float),
        ("disk_ld", C.c_float), ("disk_fcol", C.c_float), ("disk_plunge", C.c_float),
        ("flow_on", C.c_int), ("n0", C.c_double), ("n_index", C.c_double), ("theta_index", C.c_double),
        ("theta0", C.c_double), ("h_r", C.c_double), ("beta_p", C.c_double), ("r_flow_max", C.c_double),
        ("nu_obs", C.c_double), ("rg_cm", C.c_double), ("flow_kep", C.c_double),
        ("flow_turb_amp", C.c_float), ("flow_turb_scale", C.c_float), ("flow_tcorr", C.c_float),
        ("turb_tex", C.c_ulonglong * 24), ("turb_nt", C.c_int),
        ("turb_lr0", C.c_float), ("turb_lr1", C.c_float), ("turb_zmax", C.c_float), ("turb_d0", C.c_float),
        ("turb_dd", C.c_float),
        ("k2_lntab", C.POINTER(C.c_float)), ("k2_n", C.c_int), ("k2_l0", C.c_float), ("k2_dl", C.c_float),
        ("sky_on", C.c_int), ("sky_tex", C.c_ulonglong), ("sky_scale", C.c_float), ("sky_rot", Mat3),
        ("bb_xyz", C.POINTER(C.c_float)), ("bb_n", C.c_int), ("bb_l0", C.c_float), ("bb_dl", C.c_float),
        ("seed", C.c_uint32),
    ]


class Frame(C.Structure):
    _fields_ = [
        ("r", C.c_double), ("th", C.c_double), ("ph", C.c_double), ("t", C.c_double), ("kp", KerrPoint),
        ("F", Vec3), ("R", Vec3), ("U", Vec3), ("beta", Vec3), ("cx", C.c_double), ("cy", C.c_double),
        ("pix", C.c_double), ("W", C.c_int), ("H", C.c_int), ("spp", C.c_int), ("seed", C.c_uint32),
    ]


class Tables(C.Structure):
    _fields_ = [("disk_lnT", C.POINTER(C.c_float)), ("disk_n", C.c_int),
                ("k2_ln", C.POINTER(C.c_float)), ("k2_n", C.c_int),
                ("bb_xyz", C.POINTER(C.c_float)), ("bb_n", C.c_int)]


class Settings(C.Structure):
    _fields_ = [("W", C.c_int), ("H", C.c_int), ("spp", C.c_int), ("spp_max", C.c_int), ("target_err", C.c_float)]


class Post(C.Structure):
    _fields_ = [("bloom", C.c_float), ("blur_sigma_px", C.c_double), ("hide_direct", C.c_float)]


class HdrFrame(C.Structure):
    _fields_ = [("W", C.c_int), ("H", C.c_int), ("px", C.POINTER(C.c_float)),
                ("lum_percentile", C.c_double), ("lum_max", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("ms_trace", C.c_double), ("ms_post", C.c_double), ("samples", C.c_longlong),
                ("step_limited", C.c_longlong), ("attempts", C.c_longlong), ("accepted", C.c_longlong),
                ("fp64_rays", C.c_longlong), ("flow_steps", C.c_longlong), ("ms_kernel", C.c_double),
                ("attempts_fp32", C.c_longlong), ("band_rays", C.c_longlong), ("flow_steps_fp32", C.c_longlong),
                ("ms_fp32", C.c_double), ("redo_turn", C.c_longlong), ("redo_drift", C.c_longlong),
                ("redo_limit", C.c_longlong), ("ms_fp32_trace", C.c_double), ("ms_turb", C.c_double),
                ("turb_records", C.c_longlong), ("redo_records", C.c_longlong), ("record_waves", C.c_longlong),
                ("ms_rec64", C.c_double), ("ms_sum64", C.c_double), ("ms_replay64", C.c_double),
                ("rec64_slots", C.c_longlong), ("rec64_short", C.c_longlong), ("rec64_records", C.c_longlong),
                ("ms_emit64", C.c_double), ("emit64", C.c_int), ("rec64_waves", C.c_int)]


class RaysOut(C.Structure):
    _fields_ = [("fate", C.c_void_p), ("ncross", C.c_void_p), ("theta", C.c_void_p), ("phi", C.c_void_p),
                ("I", C.c_void_p), ("n_accepted", C.c_void_p), ("n_attempts", C.c_void_p),
                ("cross_r", C.c_void_p), ("cross_g", C.c_void_p)]


class Plasma(C.Structure):
    _fields_ = [("model", C.c_int), ("ne_index", C.c_double), ("te0_kelvin", C.c_double), ("te_index", C.c_double),
                ("h_sph", C.c_double), ("n_modes", C.c_int), ("turb_rms", C.c_double), ("k_min", C.c_double),
                ("k_max", C.c_double), ("spectral_index", C.c_double), ("turb_seed", C.c_uint32)]


class Mode(C.Structure):
    _fields_ = [("kx", C.c_double), ("ky", C.c_double), ("kz", C.c_double), ("phase", C.c_double),
                ("amp", C.c_double)]


class MixedOpts(C.Structure):
    _fields_ = [("band_m", C.c_double), ("tol32", C.c_double), ("turn_r", C.c_double), ("drift_tol", C.c_double),
                ("r_switch", C.c_double), ("tol_approach", C.c_double), ("t32_blocks", C.c_int),
                ("turbulence", C.c_int), ("approach", C.c_int), ("records_per_ray", C.c_double),
                ("sky_fp32", C.c_int), ("pool_mb", C.c_double), ("fp32_max_attempts", C.c_int)]


class Tune(C.Structure):
    _fields_ = [("ctas_per_sm", C.c_int), ("interleave", C.c_int), ("ms", C.c_double), ("tile", C.c_int),
                ("queue_chunk", C.c_int)]


class SurRay(C.Structure):
    _fields_ = [("alpha", C.c_float), ("beta", C.c_float), ("spin", C.c_float), ("incl_deg", C.c_float)]


class SurTarget(C.Structure):
    _fields_ = [("cls", C.c_float), ("dir", C.c_float * 3), ("u", C.c_float * 3), ("g", C.c_float * 3),
                ("pad", C.c_float * 2)]


class SurOpts(C.Structure):
    _fields_ = [("fourier_sigma", C.c_float), ("seed", C.c_uint32), ("batch", C.c_int), ("lr", C.c_float),
                ("lr_final", C.c_float), ("warmup", C.c_int), ("beta1", C.c_float), ("beta2", C.c_float),
                ("eps", C.c_float), ("weight_decay", C.c_float), ("w_dir", C.c_float), ("w_u", C.c_float),
                ("w_g", C.c_float)]


class SurLoss(C.Structure):
    _fields_ = [("total", C.c_double), ("ce", C.c_double), ("dir", C.c_double), ("u", C.c_double),
                ("g", C.c_double), ("accuracy", C.c_double), ("rays", C.c_longlong)]


class SurRanges(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("a_min", "a_max", "incl_min", "incl_max", "xy_max")]


class SurFrameOpts(C.Structure):
    _fields_ = [("band_m", C.c_double), ("audit_frac", C.c_double), ("audit_seed", C.c_uint32)]


class SurReport(C.Structure):
    _fields_ = ([(n, C.c_longlong) for n in ("rays", "surrogate_rays", "band_rays", "audit_rays")] +
                [(n, C.c_double) for n in ("ms_total", "ms_route", "ms_mlp", "ms_shade", "ms_integrator")] +
                [("audit_class_mismatch", C.c_longlong)] +
                [(n, C.c_double) for n in ("audit_dir_err", "audit_u_err", "audit_r_err", "audit_g_err",
                                           "audit_l1", "audit_flux")])


SUR_NFREQ = 64
SUR_HIDDEN = 256
SUR_LAYERS = 4
SUR_NOUT = 12
SUR_LDOUT = 16
SUR_NPARAMS = 234512


class SceneInfo(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("mass_msun", "distance_cm", "rg_cm", "tg_s", "uas_per_m", "disk_tmax",
                                          "disk_mdot_edd", "radio_flux_target_jy")]


# Field names of so_scene / so_frame whose offsets the reference layout check compares, in the order
# oracle/ref_shim.cpp's ref_layout() reports them (after the two sizeofs).
LAYOUT_FIELDS = [
    (Scene, "tol"), (Scene, "max_steps"), (Scene, "r_escape"), (Scene, "mode"), (Scene, "disk_on"),
    (Scene, "disk_lnT"), (Scene, "disk_turb_amp"), (Scene, "disk_plunge"), (Scene, "flow_on"), (Scene, "n0"),
    (Scene, "flow_kep"), (Scene, "flow_turb_amp"), (Scene, "turb_tex"), (Scene, "turb_nt"), (Scene, "turb_dd"),
    (Scene, "k2_lntab"), (Scene, "k2_n"), (Scene, "k2_dl"), (Scene, "sky_on"), (Scene, "sky_tex"),
    (Scene, "sky_rot"), (Scene, "bb_xyz"), (Scene, "bb_dl"), (Scene, "seed"), (Frame, "kp"), (Frame, "F"),
    (Frame, "beta"), (Frame, "cx"), (Frame, "pix"), (Frame, "W"), (Frame, "spp"), (Frame, "seed"),
]

# Every entry point include/so_tracer.h declares (checked against the built library's exports).
EXPORTS = [
    "so_init", "so_update_scene", "so_render", "so_render_device", "so_radio_flux", "so_trace_rays",
    "so_trace_rays_device", "so_trace_stats", "so_probe_fma_peak", "so_probe_sfu_peak", "so_probe_cos_turns", "so_radio_flux_noalloc",
    "so_batch_create", "so_batch_render", "so_batch_autotune", "so_batch_set_tune", "so_batch_free",
    "so_set_precision", "so_set_plasma", "so_set_flow_noise", "so_set_sky", "so_sky_file", "so_stream", "so_last_error", "so_destroy",
    "so_shot_load", "so_shot_scene", "so_shot_settings", "so_shot_nframes", "so_shot_frame",
    "so_find_critical_point", "so_approach_state", "so_shot_get", "so_shot_free", "so_normalize_flux", "so_plasma_modes",
    "so_kerr_point_at", "so_critical_curve_point",
    "so_sur_default_opts", "so_sur_create", "so_sur_destroy", "so_sur_get_params", "so_sur_set_params",
    "so_sur_train", "so_sur_evaluate", "so_sur_gradients", "so_sur_infer", "so_sur_set_infer_ctas", "so_sur_dataset", "so_sur_render",
    "so_sur_gemm", "so_last_fates",
]
