"""ctypes access to the CPU checkers under oracle/ (test infrastructure).

libso_oracle.so is the C restatement of the reference tracer (oracle/so_oracle.c); _ref/libbhref.so
is the reference's own host code compiled from its sources (oracle/ref_shim.cpp + oracle/Makefile).
Only tests, the smoke check and bench.py's CPU baseline use these.
"""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "libso_oracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libbhref.so")

_pkg = sys.modules.get("spacetime_optics_b200")
if _pkg is None:
    import conftest  # noqa: F401  (registers the package)
    _pkg = conftest.load_package()
abi = _pkg.abi
Scene, Frame, Plasma, Mode, RaysOut, Vec3, KerrPoint = abi.Scene, abi.Frame, abi.Plasma, abi.Mode, abi.RaysOut, abi.Vec3, abi.KerrPoint

_orc = None
_ref = None


def oracle():
    global _orc
    if _orc is None:
        L = C.CDLL(ORACLE_SO)
        P, vp = C.POINTER, C.c_void_p
        L.orc_trace_rays.argtypes = [P(Scene), vp, vp, P(Frame), C.c_int, vp, vp, P(RaysOut), C.c_int]
        L.orc_render_pass1.argtypes = [P(Scene), vp, vp, P(Frame), C.c_int, vp, vp, P(C.c_longlong), P(C.c_longlong),
                                       C.c_int]
        L.orc_vacuum_fate.argtypes = [C.c_double, P(Frame), Vec3, C.c_double, C.c_double, C.c_int]
        L.orc_find_critical_point.argtypes = [P(Frame), C.c_double, C.c_double, C.c_double]
        L.orc_find_critical_point.restype = C.c_double
        L.orc_critical_curve_point.argtypes = [C.c_double, C.c_double, C.c_double, P(C.c_double), P(C.c_double)]
        L.orc_kerr_point.argtypes = [C.c_double, C.c_double, C.c_double, P(KerrPoint)]
        L.orc_kerr_point.restype = None
        L.orc_radial_drift.argtypes = [C.c_double, C.c_double, C.c_double, Vec3, C.c_double, C.c_int, P(C.c_int)]
        L.orc_radial_drift.restype = C.c_double
        L.orc_set_sky.argtypes = [C.c_double] * 4
        L.orc_set_sky.restype = None
        L.orc_turb_setup.argtypes = [P(Scene)]
        L.orc_turb_setup.restype = None
        L.orc_fbm3.argtypes = [C.c_int, vp, vp, vp, C.c_int, C.c_uint32, vp]
        L.orc_fbm3.restype = None
        L.orc_sheared_noise.argtypes = [P(Scene), C.c_int, vp, vp, vp, vp, C.c_float, C.c_float, C.c_uint32, vp]
        L.orc_sheared_noise.restype = None
        L.orc_render_chunks.argtypes = [P(Scene), vp, vp, P(Frame), C.c_longlong, vp, vp, C.c_int, vp,
                                        P(C.c_longlong), C.c_int]
        L.orc_turb_layer.argtypes = [P(Scene), P(Frame), C.c_int, C.c_int, vp]
        L.orc_turb_layer.restype = None
        L.so_rpow5.argtypes = [C.c_double]
        L.so_rpow5.restype = C.c_double
        _orc = L
    return _orc


def have_ref():
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        L = C.CDLL(REF_SO)
        P, vp = C.POINTER, C.c_void_p
        L.ref_layout.argtypes = [P(C.c_longlong), C.c_int]
        L.ref_shot_load.argtypes = [C.c_char_p, P(C.c_char_p), C.c_int]
        L.ref_shot_load.restype = vp
        L.ref_shot_free.argtypes = [vp]
        L.ref_shot_nframes.argtypes = [vp]
        L.ref_shot_scene.argtypes = [vp, vp]
        L.ref_shot_tables.argtypes = [vp] + [P(P(C.c_float)), P(C.c_int)] * 3
        L.ref_shot_info.argtypes = [vp, P(C.c_double)]
        L.ref_shot_settings.argtypes = [vp, P(C.c_int), P(C.c_float)]
        L.ref_shot_frame.argtypes = [vp, C.c_int, C.c_int, C.c_uint32, vp]
        L.ref_find_critical_point.argtypes = [vp, C.c_int, C.c_double, C.c_double]
        L.ref_find_critical_point.restype = C.c_double
        L.ref_find_critical_point_cam.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double]
        L.ref_find_critical_point_cam.restype = C.c_double
        L.ref_critical_curve_point.argtypes = [C.c_double, C.c_double, C.c_double, P(C.c_double), P(C.c_double)]
        L.ref_kerr_point.argtypes = [C.c_double, C.c_double, C.c_double, vp]
        L.ref_radial_drift.argtypes = [P(C.c_int)]
        L.ref_radial_drift.restype = C.c_double
        L.ref_trace_rays.argtypes = [vp, vp, C.c_int, vp, vp, vp, vp, C.c_int]
        L.ref_trace_vacuum.argtypes = [vp, vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, C.c_int]
        L.ref_render_pass1.argtypes = [vp, vp, vp, P(C.c_longlong), C.c_int]
        L.ref_render_chunks.argtypes = [vp, vp, C.c_longlong, vp, vp, C.c_int, vp, C.c_int]
        L.ref_fbm3.argtypes = [C.c_int, vp, vp, vp, C.c_int, C.c_uint32, vp]
        L.ref_fbm3.restype = None
        L.ref_sheared_noise.argtypes = [vp, C.c_int, vp, vp, vp, vp, C.c_float, C.c_float, C.c_uint32, vp]
        L.ref_sheared_noise.restype = None
        L.ref_bake_turb_layer.argtypes = [vp, vp, C.c_float, C.c_int, vp]
        L.ref_bake_turb_layer.restype = None
        L.ref_adapt_dilate.argtypes = [vp, vp, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, vp, vp]
        L.ref_adapt_dilate.restype = None
        L.ref_post_bloom.argtypes = [vp, vp, C.c_int, C.c_int, C.c_float]
        L.ref_post_bloom.restype = None
        L.ref_post_radio_blur.argtypes = [vp, vp, C.c_int, C.c_int, C.c_double]
        L.ref_post_radio_blur.restype = None
        _ref = L
    return _ref


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def baked(scene):
    """Copy of scene with the baked flow turbulence set up as the renderer does (orc_turb_setup)."""
    sc = Scene.from_buffer_copy(scene)
    oracle().orc_turb_setup(C.byref(sc))
    return sc


def orc_trace(scene, frame, x, y, plasma=None, modes=None, threads=8, cross=False):
    """trace_ray of the C oracle for tangent-plane points (x, y)."""
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    n = x.size
    o = dict(fate=np.zeros(n, np.int8), ncross=np.zeros(n, np.int8), theta=np.zeros(n), phi=np.zeros(n),
             I=np.zeros((n, 4), np.float32), n_accepted=np.zeros(n, np.int32), n_attempts=np.zeros(n, np.int32),
             cross_r=np.zeros((n, 3)), cross_g=np.zeros((n, 3)))
    ro = RaysOut(*[_p(o[k]) for k in ("fate", "ncross", "theta", "phi", "I", "n_accepted", "n_attempts", "cross_r",
                                      "cross_g")])
    pl = C.byref(plasma) if plasma is not None else None
    rc = oracle().orc_trace_rays(C.byref(scene), pl, modes, C.byref(frame), n, _p(x), _p(y), C.byref(ro), threads)
    assert rc == 0
    if not cross:
        o.pop("cross_r")
        o.pop("cross_g")
    return o


def orc_pass1(scene, frame, plasma=None, modes=None, jitter=1, threads=8):
    W, H = frame.W, frame.H
    acc = np.zeros((H, W, 4), np.float32)
    ys = np.zeros((H, W, 2), np.float32)
    lim = C.c_longlong()
    att = C.c_longlong()
    pl = C.byref(plasma) if plasma is not None else None
    rc = oracle().orc_render_pass1(C.byref(scene), pl, modes, C.byref(frame), jitter, _p(acc), _p(ys), C.byref(lim),
                                   C.byref(att), threads)
    assert rc == 0
    return acc, ys, lim.value, att.value


def orc_chunks(scene, frame, pix, s0, count, plasma=None, modes=None, threads=8):
    """Sums of samples s0 .. s0 + count - 1 of pixels pix (pass-2 chunks), the C oracle's tracer."""
    pix = np.ascontiguousarray(pix, np.int64)
    s0 = np.ascontiguousarray(s0, np.int32)
    out = np.zeros((pix.size, 4), np.float32)
    lim = C.c_longlong()
    pl = C.byref(plasma) if plasma is not None else None
    rc = oracle().orc_render_chunks(C.byref(scene), pl, modes, C.byref(frame), pix.size, _p(pix), _p(s0), count,
                                    _p(out), C.byref(lim), threads)
    assert rc == 0
    return out


def orc_render_adaptive(scene, frame, spp_max, target, plasma=None, modes=None, threads=8):
    """The whole adaptive frame (pass 1, k_adapt, k_dilate, scan, pass 2, resolve) on the oracle:
    (image [H, W, 4], nsamp [H, W], chunks [H, W])."""
    acc, ys, _, _ = orc_pass1(scene, frame, plasma, modes, 1, threads)
    fr = frame_driver()
    return fr.render_adaptive(acc, ys, frame.spp, spp_max, target,
                              lambda p, s, c: orc_chunks(scene, frame, p, s, c, plasma, modes, threads),
                              visible=scene.mode == abi.SO_MODE_VISIBLE)


def ref_chunks(scene, frame, pix, s0, count, threads=8):
    """The same chunk sums through the reference's own sample_pixel / trace_ray (ref_shim.cpp)."""
    pix = np.ascontiguousarray(pix, np.int64)
    s0 = np.ascontiguousarray(s0, np.int32)
    out = np.zeros((pix.size, 4), np.float32)
    ref().ref_render_chunks(C.byref(scene), C.byref(frame), pix.size, _p(pix), _p(s0), count, _p(out), threads)
    return out


def orc_turb_layer(scene, frame, k, l):
    """Layer l (0 .. 47) of the oracle's baked turbulence slice k (0 .. 23): [192, 512] float32,
    rows ln R, columns phi.  scene must carry the bake's set-up (baked())."""
    out = np.zeros((192, 512), np.float32)
    oracle().orc_turb_layer(C.byref(scene), C.byref(frame), k, l, _p(out))
    return out


def ref_bake_layer(scene, frame, k, l):
    """The same layer from the reference's own k_bake_turb (render.cu:448-461, run on the host by
    oracle/ref_shim.cpp) with the slice's time offset turb_d0 + k * turb_dd (render.cu:680)."""
    delta = np.float32(np.float32(scene.turb_d0) + np.float32(k) * np.float32(scene.turb_dd))
    out = np.zeros((192, 512), np.float32)
    ref().ref_bake_turb_layer(C.byref(scene), C.byref(frame), float(delta), l, _p(out))
    return out


def ref_adapt_dilate(ystat, nsamp, yref, target, extra_max):
    """The reference's own k_adapt and k_dilate (render.cu:130-150, run on the host by
    oracle/ref_post_shim.cpp) on ystat [H, W, 2] float32 and nsamp [H, W]: (extra, chunks)."""
    ystat = np.ascontiguousarray(ystat, np.float32)
    nsamp = np.ascontiguousarray(nsamp, np.uint32)
    H, W = ystat.shape[:2]
    extra = np.zeros((H, W), np.uint32)
    chunks = np.zeros((H, W), np.uint32)
    ref().ref_adapt_dilate(_p(ystat), _p(nsamp), W, H, yref, target, extra_max, _p(extra), _p(chunks))
    return extra, chunks


def ref_post(img, bloom=None, sigma=None):
    """The reference's own pyramid filters (render.cu:244-316, run host-side by
    oracle/ref_post_shim.cpp) on a float32 frame [H, W, 4]: Impl::bloom with strength `bloom`, or
    Impl::radio_blur with a beam of `sigma` pixels."""
    img = np.ascontiguousarray(img, np.float32)
    H, W = img.shape[:2]
    out = np.zeros_like(img)
    if bloom is not None:
        ref().ref_post_bloom(_p(img), _p(out), W, H, bloom)
    else:
        ref().ref_post_radio_blur(_p(img), _p(out), W, H, sigma)
    return out


class RefShot:
    """The reference's own Config/build_scene/build_shot/make_frame on a shot file."""

    def __init__(self, path, overrides=()):
        arr = (C.c_char_p * max(1, len(overrides)))(*[s.encode() for s in overrides])
        self.h = ref().ref_shot_load(path.encode(), arr, len(overrides))
        assert self.h, f"reference could not load {path}"
        self.scene = Scene()
        ref().ref_shot_scene(self.h, C.byref(self.scene))
        d, k, b = P3 = (C.POINTER(C.c_float)(), C.POINTER(C.c_float)(), C.POINTER(C.c_float)())
        nd, nk, nb = C.c_int(), C.c_int(), C.c_int()
        ref().ref_shot_tables(self.h, C.byref(d), C.byref(nd), C.byref(k), C.byref(nk), C.byref(b), C.byref(nb))
        self.disk = np.ctypeslib.as_array(d, shape=(nd.value,)).copy()
        self.k2 = np.ctypeslib.as_array(k, shape=(nk.value,)).copy()
        self.bb = np.ctypeslib.as_array(b, shape=(nb.value * 3,)).copy()
        info = (C.c_double * 8)()
        ref().ref_shot_info(self.h, info)
        self.info = list(info)
        s4 = (C.c_int * 4)()
        te = C.c_float()
        ref().ref_shot_settings(self.h, s4, C.byref(te))
        self.settings = (s4[0], s4[1], s4[2], s4[3], te.value)

    def frame(self, i=0, W=None, seed=None):
        f = Frame()
        W = self.settings[0] if W is None else W
        seed = (0x9E3779B9 * (i + 1)) & 0xFFFFFFFF if seed is None else seed
        ref().ref_shot_frame(self.h, i, W, seed, C.byref(f))
        f.W, f.H, f.spp = self.settings[0], self.settings[1], self.settings[2]
        return f

    def __del__(self):
        if getattr(self, "h", None) and _ref is not None:
            _ref.ref_shot_free(self.h)
            self.h = None


def ref_vacuum(scene, frame, x, y, threads=8):
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    n = x.size
    o = dict(fate=np.zeros(n, np.int8), ncross=np.zeros(n, np.int8), theta=np.zeros(n), phi=np.zeros(n),
             n_accepted=np.zeros(n, np.int32), n_attempts=np.zeros(n, np.int32))
    ref().ref_trace_vacuum(C.byref(scene), C.byref(frame), n, _p(x), _p(y), _p(o["fate"]), _p(o["ncross"]),
                           _p(o["theta"]), _p(o["phi"]), _p(o["n_accepted"]), _p(o["n_attempts"]), threads)
    return o


def ref_trace(scene, frame, x, y, threads=8):
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    n = x.size
    fate = np.zeros(n, np.int8)
    I = np.zeros((n, 4), np.float32)
    ref().ref_trace_rays(C.byref(scene), C.byref(frame), n, _p(x), _p(y), _p(fate), _p(I), threads)
    return dict(fate=fate, I=I)


def ref_pass1(scene, frame, threads=8):
    acc = np.zeros((frame.H, frame.W, 4), np.float32)
    lim = C.c_longlong()
    ref().ref_render_pass1(C.byref(scene), C.byref(frame), _p(acc), C.byref(lim), threads)
    return acc, lim.value


def noise(lib, kind, x, y, z, seed, scene=None, scale=None, tcorr=None, t=None, oct=4):
    """fbm3 (kind "fbm3": float x, y, z) or sheared_noise (kind "sheared": double R, phi, z, t with the
    scene's spin / ISCO) at n points, from the oracle (lib "orc") or the reference (lib "ref")."""
    n = len(x)
    out = np.zeros(n, np.float32)
    if kind == "fbm3":
        a = [np.ascontiguousarray(v, np.float32) for v in (x, y, z)]
        f = oracle().orc_fbm3 if lib == "orc" else ref().ref_fbm3
        f(n, _p(a[0]), _p(a[1]), _p(a[2]), oct, seed, _p(out))
    else:
        a = [np.ascontiguousarray(v, np.float64) for v in (x, y, z, t)]
        if lib == "orc":
            oracle().orc_sheared_noise(C.byref(scene), n, *(_p(v) for v in a), scale, tcorr, seed, _p(out))
        else:
            ref().ref_sheared_noise(C.byref(scene), n, *(_p(v) for v in a), scale, tcorr, seed, _p(out))
    return out


def _module(name, fname):
    import importlib.util
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "oracle", fname))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def mlp():
    """oracle/so_mlp.py: the float64 restatement of the ray surrogate network."""
    return _module("so_mlp_oracle", "so_mlp.py")


def frame_driver():
    """oracle/so_frame.py: adaptive resampling and resolve around the tracer."""
    return _module("so_frame_oracle", "so_frame.py")


def post():
    """oracle/so_post.py: the pyramid post filters (bloom, radio beam)."""
    return _module("so_post_oracle", "so_post.py")
