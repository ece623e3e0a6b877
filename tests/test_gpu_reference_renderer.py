"""The reference's own CUDA renderer beside this library, on the same GPU and the same frames.

oracle/_ref/libbhref_gpu.so is the reference's render.cu compiled unmodified for sm_100a (with the
reference Makefile's nvcc flags) together with its host builders; oracle/ref_gpu_harness.cpp drives
its Renderer::render the way its main program does (same shot, same per-frame seed).  Both render
the reference hot flow (m87_reference_flow.ini) at 2 R2-jittered samples per pixel, no adaptive pass:

* without turbulence both are the reference's integrator and emission in FP64 on the same GPU, so the
  images differ only by rounding (the reference lets nvcc contract multiply-adds and calls libdevice
  pow; this library spells its fma and uses its own err^-1/5): per pixel and in total flux;
* with the turbulence baked into 24 retarded-time slices (the reference's default), this library's
  default fetches them through the texture unit with the reference's sampler as the reference does,
  so the images again differ only through rounding.  Rounding-level differences in a ray's state
  can change one accept / reject decision of the step controller, after which the ray samples the
  flow at other points: over a rough turbulence field that changes the image far more than over a
  smooth one.  The test measures that sensitivity on this library alone, as the difference made by
  moving the pixel scale one ulp, and bounds the difference to the reference by it;
  SO_FLOW_NOISE_BAKED_FP32, which interpolates the same slices in FP32 as the CPU oracle does,
  differs by the texture unit's 8-bit interpolation weights: its image L1 and total-flux difference
  are reported and bounded (emission.cuh:112-124, render.cu:594-620);
* the reference's own trace time (its ms_trace) and so_render's for the same frame.
"""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libbhref_gpu.so")
SHOT = os.path.join(ROOT, "spacetime-optics_b200", "shots", "m87_reference_flow.ini")


@pytest.fixture(scope="module")
def refgpu():
    if not os.path.exists(LIB):
        pytest.skip("oracle/_ref/libbhref_gpu.so not built (the reference tree was absent at build time)")
    L = C.CDLL(LIB)
    L.refgpu_open.argtypes = [C.c_char_p, C.POINTER(C.c_char_p), C.c_int, C.c_int, C.c_char_p, C.c_int]
    L.refgpu_open.restype = C.c_void_p
    L.refgpu_size.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.refgpu_render.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                                C.POINTER(C.c_longlong)]
    L.refgpu_close.argtypes = [C.c_void_p]
    L.refgpu_close.restype = None
    return L


def _reference_frame(L, overrides, frame=0):
    arr = (C.c_char_p * len(overrides))(*[o.encode() for o in overrides])
    err = C.create_string_buffer(512)
    h = L.refgpu_open(SHOT.encode(), arr, len(overrides), 0, err, 512)
    assert h, err.value
    W, H, n = C.c_int(), C.c_int(), C.c_int()
    L.refgpu_size(h, C.byref(W), C.byref(H), C.byref(n))
    img = np.zeros((H.value, W.value, 4), np.float32)
    ms, samples, lim = C.c_double(), C.c_longlong(), C.c_longlong()
    L.refgpu_render(h, frame, img.ctypes.data_as(C.c_void_p), C.byref(ms), C.byref(samples), C.byref(lim))  # warm-up
    times = []
    for _ in range(3):
        assert L.refgpu_render(h, frame, img.ctypes.data_as(C.c_void_p), C.byref(ms), C.byref(samples),
                               C.byref(lim)) == 0
        times.append(ms.value)
    L.refgpu_close(h)
    return img, min(times), samples.value


def _our_frame(so, overrides, frame=0, noise=None, ulp=False):
    sh = so.Shot(SHOT, overrides)
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    if noise is not None:
        r.set_flow_noise(noise)
    f = sh.frame(frame)
    if ulp:  # every ray's direction moved by rounding-level amounts
        f.pix = float(np.nextafter(f.pix, np.inf))
    r.render(f)  # warm-up
    times = []
    for _ in range(3):
        img, _, st = r.render(f)
        times.append(st.ms_trace)
    r.close()
    return img, min(times), st.samples


def _diff(ours, ref):
    a, b = ours[..., 0].astype(np.float64), ref[..., 0].astype(np.float64)
    return {"l1": float(np.abs(a - b).sum() / np.abs(b).sum()), "flux": float(a.sum() / b.sum() - 1.0),
            "max_pixel": float(np.abs(a - b).max() / np.abs(b).max())}


def test_reference_renderer_same_frames(so, refgpu):
    size = ["camera.width=256", "camera.height=256", "render.spp=2", "render.spp_max=2"]
    report = {}
    cases = (("no turbulence", ["flow.turbulence=0"], None), ("baked turbulence", [], None),
             ("baked turbulence, FP32 fetch", [], so.abi.SO_FLOW_NOISE_BAKED_FP32))
    refs = {}
    for tag, extra, noise in cases:
        ov = size + extra
        key = tuple(ov)
        if key not in refs:
            refs[key] = _reference_frame(refgpu, ov)
        ref, ms_ref, n_ref = refs[key]
        ours, ms_ours, n_ours = _our_frame(so, ov, noise=noise)
        assert n_ref == n_ours == 256 * 256 * 2
        assert ref[..., 0].max() > 0
        report[tag] = {**_diff(ours, ref), "ms_reference": round(ms_ref, 2), "ms_ours": round(ms_ours, 2)}
        if noise is None:
            moved, _, _ = _our_frame(so, ov, ulp=True)
            report[tag]["rounding_scale"] = _diff(moved, ours)
    print("reference renderer vs this library, 256^2 x 2 samples:", report)
    # same integrator, emission and fetch: agreement at the level a one-ulp change makes on this
    # library alone (and within 1e-5 whatever that level)
    for tag in ("no turbulence", "baked turbulence"):
        rep, scale = report[tag], report[tag]["rounding_scale"]
        assert rep["l1"] < max(1e-6, 10 * scale["l1"]) and rep["l1"] < 1e-5, tag
        assert abs(rep["flux"]) < max(1e-7, 10 * abs(scale["flux"]), 10 * scale["l1"]) and abs(rep["flux"]) < 1e-5, tag
    # FP32 trilinear against the texture unit's interpolation of the same baked slices
    fp32 = report["baked turbulence, FP32 fetch"]
    assert fp32["l1"] < 2e-3 and abs(fp32["flux"]) < 1e-3


def test_reference_renderer_timing_flow_1024(so, refgpu):
    """The flow workload of the bench (1024^2, 1 sample per pixel, step fraction 0.01, baked
    turbulence): the reference's trace time and this library's, FP64 and mixed precision."""
    ov = ["camera.width=1024", "camera.height=1024", "render.spp=1", "render.spp_max=1", "render.step_fraction=0.01"]
    ref, ms_ref, _ = _reference_frame(refgpu, ov)
    sh = so.Shot(SHOT, ov)
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    f = sh.frame(0)
    out = {}
    for name, prec in (("fp64", so.abi.SO_PREC_FP64), ("mixed", so.abi.SO_PREC_MIXED)):
        r.set_precision(prec)
        r.render(f)
        ts, img = [], None
        for _ in range(3):
            img, _, st = r.render(f)
            ts.append(st.ms_trace)
        out[name] = {"ms": round(min(ts), 2), **_diff(img, ref)}
    r.close()
    print(f"flow 1024^2: reference renderer {ms_ref:.1f} ms; this library {out}")
    assert out["fp64"]["l1"] < 1e-5
