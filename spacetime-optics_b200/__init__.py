"""spacetime-optics_b200: B200-native Kerr ray tracer (the per-pixel tracer path of bhrt).

The product is the shared library ``libso_tracer.so`` (CUDA kernels for sm_100a plus the C ABI of
include/so_tracer.h).  This module is a thin ctypes binding over that ABI, mirroring the
reference's Renderer (blackholes/src/renderer.hpp:72-88) and shot builders so that callers and
tests read like the reference's own code.  There is no CPU fallback: if the library or a CUDA
device is missing, every call raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi
from .abi import (Frame, HdrFrame, MixedOpts, Mode, Plasma, Post, RaysOut, Scene, SceneInfo, Settings, Stats,
                  Tables)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libso_tracer.so")
SHOTS = os.path.join(HERE, "shots")

_lib = None


class TracerError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"status {code}: {msg}")
        self.code = code


def lib():
    """The loaded tracer library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise TracerError(abi.SO_ERR_NO_DEVICE, f"{LIB_PATH} missing: build it first (__graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        vp = C.c_void_p
        L.so_init.argtypes = [P(vp), C.c_int, P(Scene), P(Tables), P(Settings)]
        L.so_update_scene.argtypes = [vp, P(Scene)]
        L.so_render.argtypes = [vp, P(Frame), P(Post), C.c_double, P(HdrFrame), P(Stats)]
        L.so_render_device.argtypes = [vp, P(Frame), vp, P(Stats)]
        L.so_probe_fma_peak.argtypes = [C.c_int, P(C.c_double), P(C.c_double)]
        L.so_probe_sfu_peak.argtypes = [C.c_int, P(C.c_double)]
        L.so_probe_cos_turns.argtypes = [vp, vp, C.c_longlong]
        L.so_radio_flux_noalloc.argtypes = [vp, vp, C.c_int, C.c_double, P(Plasma), vp, vp, vp]
        L.so_batch_create.argtypes = [vp, P(Scene), C.c_int, P(Frame), P(C.c_int), C.c_int, C.c_int, C.c_int,
                                      C.c_int, P(vp)]
        L.so_batch_render.argtypes = [vp, vp, P(Stats)]
        L.so_batch_autotune.argtypes = [vp, vp, P(abi.Tune)]
        L.so_batch_set_tune.argtypes = [vp, P(abi.Tune)]
        L.so_batch_free.argtypes = [vp]
        L.so_batch_free.restype = None
        L.so_radio_flux.argtypes = [vp, P(Frame), C.c_int, C.c_double, P(C.c_double)]
        L.so_trace_rays.argtypes = [vp, P(Frame), C.c_int, vp, vp, P(RaysOut)]
        L.so_trace_rays_device.argtypes = [vp, P(Frame), C.c_int, vp, vp, P(RaysOut)]
        L.so_trace_stats.argtypes = [vp, P(Stats)]
        L.so_set_precision.argtypes = [vp, C.c_int, P(MixedOpts)]
        L.so_set_plasma.argtypes = [vp, P(Plasma), P(Mode)]
        L.so_set_flow_noise.argtypes = [vp, C.c_int]
        L.so_set_sky.argtypes = [vp, C.c_int, C.c_int, vp]
        L.so_sky_file.argtypes = [C.c_char_p, P(C.c_int), P(C.c_int), P(C.c_float), vp]
        L.so_stream.argtypes = [vp]
        L.so_stream.restype = vp
        L.so_last_error.argtypes = [vp]
        L.so_last_error.restype = C.c_char_p
        L.so_destroy.argtypes = [vp]
        L.so_destroy.restype = None
        L.so_shot_load.argtypes = [C.c_char_p, P(C.c_char_p), C.c_int, P(vp)]
        L.so_shot_scene.argtypes = [vp, P(Scene), P(Tables), P(SceneInfo)]
        L.so_shot_settings.argtypes = [vp, P(Settings)]
        L.so_shot_nframes.argtypes = [vp]
        L.so_shot_frame.argtypes = [vp, C.c_int, C.c_int, C.c_uint32, P(Frame)]
        L.so_find_critical_point.argtypes = [vp, C.c_int, C.c_double, C.c_double, P(C.c_double)]
        L.so_approach_state.argtypes = [P(Scene), P(Frame), C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                        P(C.c_double), P(C.c_int)]
        L.so_shot_get.argtypes = [vp, C.c_char_p, C.c_char_p, C.c_int]
        L.so_shot_free.argtypes = [vp]
        L.so_shot_free.restype = None
        L.so_normalize_flux.argtypes = [vp, P(Scene), P(Frame), C.c_int, C.c_double, C.c_double, P(C.c_double),
                                        P(C.c_double)]
        L.so_plasma_modes.argtypes = [P(Plasma), P(Mode)]
        L.so_kerr_point_at.argtypes = [C.c_double, C.c_double, C.c_double, P(abi.KerrPoint)]
        L.so_kerr_point_at.restype = None
        L.so_critical_curve_point.argtypes = [C.c_double, C.c_double, C.c_double, P(C.c_double), P(C.c_double)]
        L.so_sur_default_opts.argtypes = [P(abi.SurOpts)]
        L.so_sur_default_opts.restype = None
        L.so_sur_create.argtypes = [C.c_int, P(abi.SurOpts), P(vp)]
        L.so_sur_destroy.argtypes = [vp]
        L.so_sur_destroy.restype = None
        L.so_sur_get_params.argtypes = [vp, vp, vp]
        L.so_sur_set_params.argtypes = [vp, vp, vp]
        L.so_sur_train.argtypes = [vp, vp, vp, C.c_longlong, C.c_int, P(abi.SurLoss)]
        L.so_sur_evaluate.argtypes = [vp, vp, vp, C.c_longlong, P(abi.SurLoss)]
        L.so_sur_gradients.argtypes = [vp, vp, vp, C.c_int, vp, P(abi.SurLoss)]
        L.so_sur_infer.argtypes = [vp, vp, C.c_longlong, vp, vp]
        L.so_sur_set_infer_ctas.argtypes = [vp, C.c_int]
        L.so_sur_dataset.argtypes = [vp, P(Frame), C.c_longlong, C.c_int, C.c_uint32, P(abi.SurRanges), vp, vp,
                                     P(Stats)]
        L.so_sur_render.argtypes = [vp, vp, P(Frame), P(abi.SurFrameOpts), vp, P(abi.SurReport)]
        L.so_sur_gemm.argtypes = [vp, vp, vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.so_last_fates.argtypes = [vp, vp, vp, C.c_longlong]
        _lib = L
    return _lib


def _check(rc, handle=None):
    if rc != abi.SO_OK:
        msg = lib().so_last_error(handle).decode(errors="replace")
        raise TracerError(rc, msg)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Shot:
    """A shot .ini (reference schema plus the [so] section), with --set style overrides."""

    def __init__(self, path, overrides=()):
        if not os.path.isabs(path) and not os.path.exists(path):
            path = os.path.join(SHOTS, path)
        self.path = path
        arr = (C.c_char_p * max(1, len(overrides)))(*[s.encode() for s in overrides])
        h = C.c_void_p()
        rc = lib().so_shot_load(path.encode(), arr, len(overrides), C.byref(h))
        if rc != abi.SO_OK:
            raise TracerError(rc, f"cannot load shot {path}")
        self.h = h
        self.scene = Scene()
        self.tables = Tables()
        self.info = SceneInfo()
        _check(lib().so_shot_scene(self.h, C.byref(self.scene), C.byref(self.tables), C.byref(self.info)))
        self.settings = Settings()
        _check(lib().so_shot_settings(self.h, C.byref(self.settings)))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.so_shot_free(self.h)
            self.h = None

    def nframes(self):
        return lib().so_shot_nframes(self.h)

    def frame(self, i=0, W=None, seed=None):
        f = Frame()
        W = self.settings.W if W is None else W
        seed = (0x9E3779B9 * (i + 1)) & 0xFFFFFFFF if seed is None else seed  # main.cpp:529
        _check(lib().so_shot_frame(self.h, i, W, seed, C.byref(f)))
        f.W, f.H, f.spp = self.settings.W, self.settings.H, self.settings.spp
        return f

    def get(self, key, default=None):
        buf = C.create_string_buffer(4096)
        if lib().so_shot_get(self.h, key.encode(), buf, 4096) != abi.SO_OK:
            return default
        return buf.value.decode()

    def num(self, key, default):
        v = self.get(key)
        try:
            return float(v) if v is not None else default
        except ValueError:
            return default

    def find_critical_point(self, psi, i=0):
        rho = C.c_double()
        _check(lib().so_find_critical_point(self.h, i, self.scene.a, psi, C.byref(rho)))
        return rho.value

    def plasma(self):
        """The [so] torus plasma of this shot, or None (reference flow model)."""
        if self.get("so.plasma", "reference") != "torus":
            return None
        p = Plasma()
        p.model = abi.SO_PLASMA_TORUS
        p.ne_index = self.num("so.ne_index", 1.5)
        p.te0_kelvin = self.num("so.te0_kelvin", 1e11)
        p.te_index = self.num("so.te_index", 0.84)
        p.h_sph = self.num("so.h_sph", 0.3)
        p.n_modes = int(self.num("so.modes", 512))
        p.turb_rms = self.num("so.turb_rms", 0.3)
        p.k_min = self.num("so.k_min", 2 * np.pi / 20)
        p.k_max = self.num("so.k_max", 2 * np.pi / 0.5)
        p.spectral_index = self.num("so.spectral_index", -11.0 / 3.0)
        p.turb_seed = int(self.num("so.turb_seed", 1))
        return p


def sky_file(path):
    """so_sky_file: (texels uint16 [h, w, 2], scale) of a .bhsk star map."""
    w, h, sc = C.c_int(), C.c_int(), C.c_float()
    _check(lib().so_sky_file(path.encode(), C.byref(w), C.byref(h), C.byref(sc), None))
    t = np.empty((h.value, w.value, 2), np.uint16)
    _check(lib().so_sky_file(path.encode(), C.byref(w), C.byref(h), C.byref(sc), t.ctypes.data_as(C.c_void_p)))
    return t, sc.value


def approach_state(scene, frame, x, y, r1, tol, method):
    """so_approach_state: (state [r, r', u, u', phi, t], attempts) of the backward ray through image
    point (x, y) at radius r1; method 0 = far-field transport in 1/r, 1 = Mino-time DP5(4)."""
    st = (C.c_double * 6)()
    att = C.c_int(0)
    _check(lib().so_approach_state(C.byref(scene), C.byref(frame), x, y, r1, tol, method, st, C.byref(att)))
    return np.array(st[:]), att.value


def plasma_modes(p):
    """Fourier modes of a torus plasma (so_plasma_modes), as a ctypes array of Mode."""
    arr = (Mode * max(1, p.n_modes))()
    _check(lib().so_plasma_modes(C.byref(p), arr))
    return arr


def modes_to_numpy(arr, n):
    return np.ctypeslib.as_array(C.cast(arr, C.POINTER(C.c_double)), shape=(n, 5)).copy()


class Renderer:
    """Renderer (render.cu:477-809) through the C ABI."""

    def __init__(self, scene, tables, settings, device=0):
        h = C.c_void_p()
        rc = lib().so_init(C.byref(h), device, C.byref(scene), C.byref(tables), C.byref(settings))
        if rc != abi.SO_OK:
            raise TracerError(rc, lib().so_last_error(None).decode(errors="replace"))
        self.h = h
        self.settings = settings
        self.scene = scene

    def close(self):
        if getattr(self, "h", None):
            lib().so_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def update_scene(self, scene):
        self.scene = scene
        _check(lib().so_update_scene(self.h, C.byref(scene)), self.h)

    def set_sky(self, texels):
        """Star map (so_set_sky): uint16 array [h, w, 2] of half2 texels (s, s T / 1e4)."""
        t = np.ascontiguousarray(texels, np.uint16)
        if t.ndim != 3 or t.shape[2] != 2:
            raise ValueError("texels must be [h, w, 2] uint16")
        _check(lib().so_set_sky(self.h, t.shape[1], t.shape[0], t.ctypes.data_as(C.c_void_p)), self.h)

    def set_flow_noise(self, mode):
        """Reference flow turbulence: abi.SO_FLOW_NOISE_BAKED (default: baked slices through the texture
        unit), abi.SO_FLOW_NOISE_BAKED_FP32 (baked, FP32 trilinear as the oracle) or abi.SO_FLOW_NOISE_INLINE."""
        _check(lib().so_set_flow_noise(self.h, mode), self.h)

    def set_plasma(self, plasma, modes=None):
        if plasma is None:
            plasma = Plasma()
            plasma.model = abi.SO_PLASMA_REFERENCE
        if modes is None and plasma.model == abi.SO_PLASMA_TORUS and plasma.n_modes > 0:
            modes = plasma_modes(plasma)
        _check(lib().so_set_plasma(self.h, C.byref(plasma), modes), self.h)
        return modes

    def set_precision(self, precision, band_m=0.05, tol32=3e-6, turn_r=0.0, drift_tol=1e-4, r_switch=0.0,
                      tol_approach=0.0, t32_blocks=0, turbulence=0, approach=0, records_per_ray=0.0,
                      fp32_max_attempts=0, sky_fp32=0, pool_mb=0.0):
        o = MixedOpts(band_m, tol32, turn_r, drift_tol, r_switch, tol_approach, t32_blocks, turbulence, approach,
                      records_per_ray, sky_fp32, pool_mb, fp32_max_attempts)
        _check(lib().so_set_precision(self.h, precision, C.byref(o)), self.h)

    def render(self, frame, percentile=0.995, hide_direct=0.0, out=None, bloom=0.0, blur_sigma_px=0.0):
        W, H = self.settings.W, self.settings.H
        if out is None:
            out = np.empty((H, W, 4), np.float32)
        hdr = HdrFrame(W, H, out.ctypes.data_as(C.POINTER(C.c_float)), 0.0, 0.0)
        st = Stats()
        post = Post(bloom, blur_sigma_px, hide_direct)
        _check(lib().so_render(self.h, C.byref(frame), C.byref(post), percentile, C.byref(hdr), C.byref(st)), self.h)
        return out, hdr, st

    def render_device(self, frame, d_px, stats=False):
        """Trace into caller-owned device memory (an address, e.g. torch tensor.data_ptr()).  Without
        stats the call is asynchronous on self.stream()."""
        st = Stats() if stats else None
        _check(lib().so_render_device(self.h, C.byref(frame), C.c_void_p(d_px), C.byref(st) if st else None),
               self.h)
        return st

    def last_fates(self, n):
        """(fate int8[n], in_band bool[n]) of the last mixed-precision frame's samples."""
        fate = np.zeros(n, np.int8)
        band = np.zeros(n, np.uint8)
        _check(lib().so_last_fates(self.h, _ptr(fate), _ptr(band), n), self.h)
        return fate, band.astype(bool)

    def stream(self):
        """The renderer's CUDA stream handle (cudaStream_t as an int)."""
        return lib().so_stream(self.h)

    def radio_flux(self, frame, n, pix_sr):
        jy = C.c_double()
        _check(lib().so_radio_flux(self.h, C.byref(frame), n, pix_sr, C.byref(jy)), self.h)
        return jy.value

    def trace_rays(self, frame, x, y, cross=False):
        x = np.ascontiguousarray(x, np.float64)
        y = np.ascontiguousarray(y, np.float64)
        n = x.size
        # so_trace_rays writes every element of every output it is given
        o = dict(fate=np.empty(n, np.int8), ncross=np.empty(n, np.int8), theta=np.empty(n), phi=np.empty(n),
                 I=np.empty((n, 4), np.float32), n_accepted=np.empty(n, np.int32), n_attempts=np.empty(n, np.int32))
        if cross:
            o["cross_r"] = np.empty((n, 3))
            o["cross_g"] = np.empty((n, 3))
        ro = RaysOut(*[_ptr(o.get(k)) for k in ("fate", "ncross", "theta", "phi", "I", "n_accepted", "n_attempts",
                                                 "cross_r", "cross_g")])
        _check(lib().so_trace_rays(self.h, C.byref(frame), n, _ptr(x), _ptr(y), C.byref(ro)), self.h)
        return o

    def trace_stats(self):
        """Counters of the last trace_rays call (so_trace_stats)."""
        st = Stats()
        _check(lib().so_trace_stats(self.h, C.byref(st)), self.h)
        return st

    def normalize_flux(self, scene, frame_wide, n, pix_sr, target_jy):
        n0 = C.c_double()
        jy = C.c_double()
        _check(lib().so_normalize_flux(self.h, C.byref(scene), C.byref(frame_wide), n, pix_sr, target_jy,
                                       C.byref(n0), C.byref(jy)), self.h)
        self.scene = scene
        return n0.value, jy.value


class Batch:
    """Many frames traced by one persistent launch (so_batch_*), replayed as a CUDA graph."""

    def __init__(self, renderer, scenes, frames, frame_scene, W, H, spp=1):
        self.r = renderer
        sc = (Scene * len(scenes))(*scenes)
        fr = (Frame * len(frames))(*frames)
        fs = (C.c_int * len(frame_scene))(*frame_scene)
        h = C.c_void_p()
        _check(lib().so_batch_create(renderer.h, sc, len(scenes), fr, fs, len(frames), W, H, spp, C.byref(h)),
               renderer.h)
        self.h = h
        self.n = len(frames)
        self.W, self.H = W, H

    def render(self, d_px, stats=False):
        st = Stats() if stats else None
        _check(lib().so_batch_render(self.h, C.c_void_p(d_px), C.byref(st) if st else None), self.r.h)
        return st

    def autotune(self, d_px):
        t = abi.Tune()
        _check(lib().so_batch_autotune(self.h, C.c_void_p(d_px), C.byref(t)), self.r.h)
        return t

    def set_tune(self, ctas_per_sm, interleave, tile=1, queue_chunk=1):
        t = abi.Tune(ctas_per_sm, interleave, 0.0, tile, queue_chunk)
        _check(lib().so_batch_set_tune(self.h, C.byref(t)), self.r.h)

    def close(self):
        if getattr(self, "h", None):
            lib().so_batch_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def probe_fma_peak(device=0):
    """Measured FP64 and FP32 FMA-pipe peaks of the device, TFLOP/s (so_probe_fma_peak)."""
    a, b = C.c_double(), C.c_double()
    _check(lib().so_probe_fma_peak(device, C.byref(a), C.byref(b)))
    return a.value, b.value


def probe_sfu_peak(device=0):
    """Measured SFU cosine throughput of the device, G ops/s (so_probe_sfu_peak)."""
    g = C.c_double()
    _check(lib().so_probe_sfu_peak(device, C.byref(g)))
    return g.value


class Surrogate:
    """The ray surrogate (so_sur_*): an MLP from (alpha, beta, spin, inclination) to the integrator's
    termination class, escape direction and first three equatorial crossings, trained and run by the
    library's tensor-core kernels.  Device arrays are torch CUDA tensors (float32): rays [n, 4],
    targets [n, 12], outputs [n, 16]."""

    def __init__(self, device=0, **opts):
        o = abi.SurOpts()
        lib().so_sur_default_opts(C.byref(o))
        for k, v in opts.items():
            setattr(o, k, v)
        h = C.c_void_p()
        _check(lib().so_sur_create(device, C.byref(o), C.byref(h)))
        self.h = h
        self.opts = o
        self.device = device

    def params(self):
        p = np.empty(abi.SUR_NPARAMS, np.float32)
        f = np.empty((abi.SUR_NFREQ, 4), np.float32)
        _check(lib().so_sur_get_params(self.h, _ptr(p), _ptr(f)))
        return p, f

    def set_params(self, p=None, f=None):
        p = None if p is None else np.ascontiguousarray(p, np.float32)
        f = None if f is None else np.ascontiguousarray(f, np.float32)
        _check(lib().so_sur_set_params(self.h, _ptr(p), _ptr(f)))

    def dataset(self, renderer, frame, n, groups, seed=1, a=(0.0, 0.99), incl=(5.0, 175.0), xy_max=12.0):
        """(rays, targets, stats): n rays from the FP64 integrator of `renderer` (camera at frame.r)."""
        import torch
        rays = torch.empty((n, 4), dtype=torch.float32, device=f"cuda:{self.device}")
        tgt = torch.empty((n, 12), dtype=torch.float32, device=f"cuda:{self.device}")
        rg = abi.SurRanges(a[0], a[1], incl[0], incl[1], xy_max)
        st = Stats()
        _check(lib().so_sur_dataset(renderer.h, C.byref(frame), n, groups, seed, C.byref(rg), rays.data_ptr(),
                                    tgt.data_ptr(), C.byref(st)), renderer.h)
        return rays, tgt, st

    def train(self, rays, tgt, steps):
        loss = abi.SurLoss()
        _check(lib().so_sur_train(self.h, rays.data_ptr(), tgt.data_ptr(), rays.shape[0], steps, C.byref(loss)))
        return loss

    def evaluate(self, rays, tgt):
        loss = abi.SurLoss()
        _check(lib().so_sur_evaluate(self.h, rays.data_ptr(), tgt.data_ptr(), rays.shape[0], C.byref(loss)))
        return loss

    def gradients(self, rays, tgt):
        g = np.empty(abi.SUR_NPARAMS, np.float32)
        loss = abi.SurLoss()
        _check(lib().so_sur_gradients(self.h, rays.data_ptr(), tgt.data_ptr(), rays.shape[0], _ptr(g),
                                      C.byref(loss)))
        return g, loss

    def infer(self, rays):
        """Outputs [n, 16], queued on torch's current stream."""
        import torch
        out = torch.empty((rays.shape[0], abi.SUR_LDOUT), dtype=torch.float32, device=rays.device)
        st = torch.cuda.current_stream(rays.device).cuda_stream
        _check(lib().so_sur_infer(self.h, rays.data_ptr(), rays.shape[0], out.data_ptr(), C.c_void_p(st)))
        return out

    def set_infer_ctas(self, ctas):
        """Fused inference kernel form: 1 CTA per tile (default) or 2 (cta_group::2 cluster pairs)."""
        _check(lib().so_sur_set_infer_ctas(self.h, ctas))

    def render(self, renderer, frame, band_m=0.5, audit_frac=0.01, audit_seed=2, out=None):
        """Surrogate thin-disk frame into out (torch [H, W, 4] float32 on the device) and its report."""
        import torch
        W, H = renderer.settings.W, renderer.settings.H
        if out is None:
            out = torch.zeros((H, W, 4), dtype=torch.float32, device=f"cuda:{self.device}")
        o = abi.SurFrameOpts(band_m, audit_frac, audit_seed)
        rep = abi.SurReport()
        _check(lib().so_sur_render(self.h, renderer.h, C.byref(frame), C.byref(o), out.data_ptr(), C.byref(rep)))
        return out, rep

    def close(self):
        if self.h:
            lib().so_sur_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sur_gemm(a, b, bias=None, splits=1, layout=0):
    """so_sur_gemm on torch bf16 CUDA tensors a [M, K], b [N, K]: the float32 product [M, N]
    (layout 0), or its per-slice planes [splits, M, N] (layout 1) or transposed [splits, N, M] (2)."""
    import torch
    M, K = a.shape
    N = b.shape[0]
    shape = {0: (M, N), 1: (splits, M, N), 2: (splits, N, M)}[layout]
    c = torch.zeros(shape, dtype=torch.float32, device=a.device)
    _check(lib().so_sur_gemm(a.data_ptr(), b.data_ptr(), None if bias is None else bias.data_ptr(), c.data_ptr(),
                             M, N, K, splits, layout))
    return c


def pixel_centres(frame, W, H):
    """Tangent-plane coordinates of the pixel centres of a W x H frame (render.cu:79-80, jitter 1/2)."""
    px = np.arange(W, dtype=np.float64)
    py = np.arange(H, dtype=np.float64)
    X = (px[None, :] + 0.5 - 0.5 * W) * frame.pix
    Y = (0.5 * H - (py[:, None] + 0.5)) * frame.pix
    return np.broadcast_to(X, (H, W)).ravel().copy(), np.broadcast_to(Y, (H, W)).ravel().copy()
