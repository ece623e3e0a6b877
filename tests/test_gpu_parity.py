"""Parity of the CUDA FP64 tracer with the CPU oracle and the reference's golden vectors.

All calls go through the C ABI (libso_tracer.so).  Bars:
  * kernel vs oracle (same operations, bit-reproducible trajectories): fate, winding order and step
    counts exact for every ray; escape direction within 1e-13 relative (only libm vs libdevice acos
    / atan2 differ); specific intensity within float-accumulation precision (1e-6 of the maximum).
  * kernel vs the reference's own code (golden fixtures): fate / winding order exact, escape
    direction within 1e-9 relative.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def shadow(so):
    sh = so.Shot("shadow_selftest_256.ini")
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    yield sh, r
    r.close()


def _cmp_geometry(o, k, rtol_dir=1e-13):
    assert np.array_equal(o["fate"], k["fate"])
    assert np.array_equal(o["ncross"], k["ncross"])
    assert np.array_equal(o["n_accepted"], k["n_accepted"])
    assert np.array_equal(o["n_attempts"], k["n_attempts"])
    esc = o["fate"] == 1
    for key in ("theta", "phi"):
        rel = np.abs(o[key][esc] - k[key][esc]) / np.maximum(np.abs(o[key][esc]), 1e-300)
        assert rel.max(initial=0.0) <= rtol_dir, (key, rel.max())


def _threads():
    return max(8, os.cpu_count() or 8)


def test_shadow_grid_bitexact_vs_oracle(so, orc, shadow):
    """The whole 256^2 shadow self-test grid (65,536 pixel centres): kernel == oracle on every ray
    (fate, winding order, accepted and attempted step counts; escape direction 1e-13 relative)."""
    sh, r = shadow
    f = sh.frame(0)
    X, Y = so.pixel_centres(f, 256, 256)
    k = r.trace_rays(f, X, Y)
    o = orc.orc_trace(sh.scene, f, X, Y, threads=_threads())
    _cmp_geometry(o, k)
    assert (k["fate"] == -1).sum() > 15000 and (k["fate"] == 1).sum() > 40000


def test_shadow_full_grid_vs_reference(so, shadow):
    """The whole 256^2 grid against the reference's own trace_ray (golden/shadow_grid_256.npz):
    class and winding order identical on all 65,536 rays; escape direction within 1e-9 relative,
    or within 1e-9 + 1e-11 x S on the ill-conditioned rays next to the critical curve (S = the
    direction's sensitivity to the ray's starting point, up to ~1e5 there; at most 0.1 % of the
    escaping rays may need it, each with S >= 100)."""
    import _parity
    sh, r = shadow
    f = sh.frame(0)
    X, Y = so.pixel_centres(f, 256, 256)
    rep = _parity.shadow_grid_vs_reference(r.trace_rays(f, X, Y))
    print("shadow grid vs reference:", rep)
    assert rep["n_accepted_equal"] > 0.999


def test_shadow_vs_reference_golden(so, shadow):
    g = np.load(os.path.join(GOLD, "shadow_rays.npz"))
    sh, r = shadow
    k = r.trace_rays(sh.frame(0), g["x"], g["y"])
    assert np.array_equal(k["fate"], g["fate"])
    assert np.array_equal(k["ncross"], g["ncross"])
    esc = g["fate"] == 1
    for key in ("theta", "phi"):
        rel = np.abs(k[key][esc] - g[key][esc]) / np.maximum(np.abs(g[key][esc]), 1e-300)
        assert rel.max() < 1e-9, (key, rel.max())


def test_spin_inclination_sweep(so, orc):
    """golden/sweep_rays.npz: the shadow shot at eight other spins and inclinations (spin clamp at
    both ends, a = 0.998 and 0.9999, edge-on, 0.5 deg off the pole, below the plane, on the pole).
    The package's shot builder gives the reference's scene and frame for each; the kernel equals
    the oracle on every ray (fate, winding order, step counts; escape direction 1e-13 relative) and
    the reference's trace_ray in fate, winding order and escape direction (1e-9 relative)."""
    g = np.load(os.path.join(GOLD, "sweep_rays.npz"))
    for c, (spin, incl) in enumerate(g["cases"]):
        sh = so.Shot("shadow_selftest_256.ini", [f"bh.spin={spin}", f"camera.incl={incl}"])
        assert sh.scene.a == float(g[f"c{c}_a"])
        f = sh.frame(0)
        assert bytes(memoryview(f)) == g[f"c{c}_frame"].tobytes(), (spin, incl)
        x, y = g[f"c{c}_x"], g[f"c{c}_y"]
        r = so.Renderer(sh.scene, sh.tables, sh.settings)
        try:
            k = r.trace_rays(f, x, y)
        finally:
            r.close()
        _cmp_geometry(orc.orc_trace(sh.scene, f, x, y), k)
        assert np.array_equal(k["fate"], g[f"c{c}_fate"]), (spin, incl)
        assert np.array_equal(k["ncross"], g[f"c{c}_ncross"]), (spin, incl)
        esc = k["fate"] == 1
        for key in ("theta", "phi"):
            ref = g[f"c{c}_{key}"][esc]
            rel = np.abs(k[key][esc] - ref) / np.maximum(np.abs(ref), 1e-300)
            assert rel.max(initial=0.0) < 1e-9, (spin, incl, key, rel.max())


def test_crossing_records_vs_oracle(so, orc, shadow):
    """First three equatorial crossings (radius, circular-emitter redshift) recorded per ray."""
    sh, r = shadow
    f = sh.frame(0)
    X, Y = so.pixel_centres(f, 256, 256)
    X, Y = X[7::97], Y[7::97]
    k = r.trace_rays(f, X, Y, cross=True)
    o = orc.orc_trace(sh.scene, f, X, Y, cross=True)
    assert np.array_equal(k["ncross"], o["ncross"])
    assert np.array_equal(k["cross_r"], o["cross_r"])
    np.testing.assert_allclose(k["cross_g"], o["cross_g"], rtol=1e-14, atol=0)
    assert (k["cross_r"][:, 0] > 0).mean() > 0.5


def test_analytic_shadow_edge(so, shadow):
    """bhrt --selftest on the GPU: the fate transition along the horizontal image axis of a distant
    camera (r = 1e7) sits on the analytic Bardeen critical curve (kerr.hpp:210-220)."""
    import ctypes as C
    for a, incl in ((0.94, 17.0), (0.5, 90.0), (0.99, 90.0)):
        import tempfile
        with tempfile.NamedTemporaryFile("w", suffix=".ini", delete=False) as fh:
            fh.write(f"[bh]\nspin = {a}\n[render]\nmode = visible\ntolerance = 1e-12\nmax_steps = 2000000\n"
                     f"r_escape = 200\nhorizon_margin = 0.001\n[disk]\nenabled = 0\n[sky]\nenabled = 0\n"
                     f"[camera]\nr = 1e7\nincl = {incl}\nfov_m = 30\nwidth = 8\nheight = 8\n")
            path = fh.name
        try:
            sh = so.Shot(path)
            r = so.Renderer(sh.scene, sh.tables, sh.settings)
            f = sh.frame(0)
            th = incl * np.pi / 180
            rp0 = 2.0 * (1.0 + np.cos(2.0 / 3.0 * np.arccos(-a)))
            rp1 = 2.0 * (1.0 + np.cos(2.0 / 3.0 * np.arccos(a)))
            al, be = C.c_double(), C.c_double()
            alphas = []
            # the extreme alphas sit where beta = 0, at the ends of the visible photon-orbit range:
            # sample as densely as the reference's self-test does (main.cpp:338)
            for i in range(200001):
                rp = rp0 + (rp1 - rp0) * i / 200000.0
                if so.lib().so_critical_curve_point(a, th, rp, C.byref(al), C.byref(be)):
                    alphas.append(al.value)
            amin, amax = min(alphas), max(alphas)
            for edge, lo, hi in ((amax, amax - 0.05, amax + 0.05), (amin, amin - 0.05, amin + 0.05)):
                xs = np.linspace(lo, hi, 4001)
                k = r.trace_rays(f, xs / 1e7, np.zeros_like(xs))
                fate = k["fate"]
                cap = fate == -1
                # one transition captured <-> escaped inside the window
                trans = np.nonzero(cap[1:] != cap[:-1])[0]
                assert len(trans) >= 1
                x_edge = xs[trans[0]] if edge == amax else xs[trans[-1]]
                assert abs(x_edge - edge) < 5e-4, (a, incl, x_edge, edge)
            r.close()
        finally:
            os.unlink(path)


def test_reference_flow_turbulent_vs_oracle(so, orc):
    """The reference's hot flow with its fBm turbulence evaluated in place (SO_FLOW_NOISE_INLINE,
    the reference's turb_nt = 0 path), radio mode, 48 x 48 pixel centres."""
    sh = so.Shot("m87_reference_flow.ini", ["camera.width=48", "camera.height=48"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_flow_noise(so.abi.SO_FLOW_NOISE_INLINE)
    f = sh.frame(0)
    X, Y = so.pixel_centres(f, 48, 48)
    k = r.trace_rays(f, X, Y)
    o = orc.orc_trace(sh.scene, f, X, Y)
    _cmp_geometry(o, k, rtol_dir=1e-12)
    I0, I1 = o["I"].astype(np.float64), k["I"].astype(np.float64)
    assert I0[:, 0].max() > 0
    assert np.abs(I0 - I1).max() <= 1e-6 * I0[:, 0].max()
    assert abs(I0[:, 0].sum() - I1[:, 0].sum()) <= 1e-6 * I0[:, 0].sum()
    r.close()


def test_reference_flow_baked_turbulence_vs_oracle(so, orc):
    """The turbulent reference flow baked per frame into 24 retarded-time slices (render.cu:449-460,
    emission.cuh:112-124).  With SO_FLOW_NOISE_BAKED_FP32 (slices in plain memory, FP32 trilinear in
    a fixed order) against the oracle, whose texels are the bake formula at each texel centre and
    whose interpolation repeats the kernel's: geometry exact, intensity within 1e-6 of the maximum.
    The default SO_FLOW_NOISE_BAKED reads the same slices through the texture unit (the reference's
    own fetch, weights with 8 fractional bits): same geometry, intensity within 2 % of the maximum
    per ray and 1e-3 in total (the reference's own renderer is matched at rounding level instead:
    tests/test_gpu_reference_renderer.py).  Switching modes reproduces each image exactly.  Baked and
    in-place images are different draws of the same turbulence, not one an approximation of the
    other: at the camera's coordinate time (t ~ -1e7 M) the sheared noise decorrelates over relative
    radius changes of ~1e-5, far below the bake's 2 per cent cells, so only their sizes are compared."""
    sh = so.Shot("m87_reference_flow.ini", ["camera.width=40", "camera.height=40"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    f = sh.frame(0)
    X, Y = so.pixel_centres(f, 40, 40)
    kt = r.trace_rays(f, X, Y)  # default: texture fetch
    r.set_flow_noise(so.abi.SO_FLOW_NOISE_BAKED_FP32)
    k = r.trace_rays(f, X, Y)
    o = orc.orc_trace(orc.baked(sh.scene), f, X, Y)
    _cmp_geometry(o, k, rtol_dir=1e-12)
    I0, I1 = o["I"].astype(np.float64), k["I"].astype(np.float64)
    assert I0[:, 0].max() > 0
    assert np.abs(I0 - I1).max() <= 1e-6 * I0[:, 0].max()
    _cmp_geometry(o, kt, rtol_dir=1e-12)
    It = kt["I"].astype(np.float64)
    assert np.abs(It - I1).max() <= 2e-2 * I1[:, 0].max()
    assert abs(It[:, 0].sum() / I1[:, 0].sum() - 1.0) < 1e-3
    r.set_flow_noise(so.abi.SO_FLOW_NOISE_INLINE)
    ki = r.trace_rays(f, X, Y)
    r.set_flow_noise(so.abi.SO_FLOW_NOISE_BAKED_FP32)
    assert np.array_equal(r.trace_rays(f, X, Y)["I"], k["I"])
    r.set_flow_noise(so.abi.SO_FLOW_NOISE_BAKED)
    assert np.array_equal(r.trace_rays(f, X, Y)["I"], kt["I"])
    Ii = ki["I"].astype(np.float64)
    assert not np.array_equal(Ii, I1)
    assert 0.5 < Ii[:, 0].sum() / I1[:, 0].sum() < 2.0
    with pytest.raises(so.TracerError):
        r.set_flow_noise(3)
    r.close()


def test_reference_flow_vs_reference_golden(so):
    g = np.load(os.path.join(GOLD, "flow_rays.npz"))
    sh = so.Shot("m87_reference_flow.ini", ["flow.turbulence=0", "camera.width=32", "camera.height=32"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    k = r.trace_rays(sh.frame(0), g["x"], g["y"])
    assert np.array_equal(k["fate"], g["fate"])
    I0, I1 = g["I"].astype(np.float64), k["I"].astype(np.float64)
    assert np.abs(I0 - I1).max() <= 1e-5 * I0[:, 0].max()
    assert abs(I0[:, 0].sum() - I1[:, 0].sum()) <= 1e-7 * I0[:, 0].sum()
    # Per ray: the reference accumulates I in float, one rounding of (float)(trans * dI) per flow
    # step, so FP64 emission that differs in its last bits moves a ray's float sum by a few float
    # ulps (2^-24 = 6e-8) where the rounding of one step flips; every other ray is bit-identical.
    rep = _intensity_report(g["I"], k["I"])
    print("reference flow vs reference:", rep)
    assert rep["rel_max"] <= 16 * 2.0 ** -24 and rep["bit_identical"] > 0.85
    r.close()


def _intensity_report(I0, I1, frac=1e-3):
    """Per-ray relative difference of channel 0 over the rays above frac of the maximum, and the
    fraction of rays whose four float channels are bit-identical."""
    a, b = I0[:, 0].astype(np.float64), I1[:, 0].astype(np.float64)
    big = a > frac * a.max()
    rel = np.abs(a - b)[big] / a[big]
    return {"rays": len(a), "above": int(big.sum()), "rel_max": float(rel.max()),
            "rel_p99": float(np.percentile(rel, 99)), "bit_identical": float((I0 == I1).all(axis=1).mean())}


def test_cos_turns_device_equals_oracle(so, orc):
    """The device's cos_turns (FP64 torus turbulence) equals the oracle's restatement bit for bit."""
    import ctypes as C
    import torch
    rng = np.random.default_rng(9)
    t = np.concatenate([rng.uniform(-300, 300, 200000), rng.uniform(-1, 1, 50000), np.arange(-8, 8.001, 1 / 256)])
    d_t = torch.tensor(t, dtype=torch.float64, device="cuda")
    d_o = torch.empty_like(d_t)
    assert so.lib().so_probe_cos_turns(C.c_void_p(d_t.data_ptr()), C.c_void_p(d_o.data_ptr()), t.size) == 0
    f = orc.oracle().orc_cos_turns
    f.argtypes, f.restype = [C.c_double], C.c_double
    want = np.array([f(float(x)) for x in t])
    assert np.array_equal(d_o.cpu().numpy().view(np.uint64), want.view(np.uint64))


def test_torus_1024_strided_vs_oracle(so, orc):
    """Config synchrotron_1024 (a = 0.94, i = 163 deg, +-12 M, 230 GHz, 512-mode torus turbulence):
    every 61st pixel centre of the 1024^2 frame (17,190 rays) through the FP64 kernel against the
    oracle.  Geometry exact (fate, winding order, step counts), escape direction 1e-12 relative,
    intensity within 1e-6 of the frame maximum and, per ray above 1e-3 of the maximum, within 1e-5
    relative (float accumulation of FP64 emission whose cosines round differently in libdevice and
    libm)."""
    sh = so.Shot("synchrotron_1024.ini")
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    p = sh.plasma()
    modes = r.set_plasma(p)
    f = sh.frame(0)
    X, Y = so.pixel_centres(f, 1024, 1024)
    X, Y = X[::61], Y[::61]
    assert X.size >= 16000
    k = r.trace_rays(f, X, Y)
    o = orc.orc_trace(sh.scene, f, X, Y, plasma=p, modes=modes, threads=_threads())
    _cmp_geometry(o, k, rtol_dir=1e-12)
    I0, I1 = o["I"].astype(np.float64), k["I"].astype(np.float64)
    assert I0[:, 0].max() > 0
    assert np.abs(I0 - I1).max() <= 1e-6 * I0[:, 0].max()
    rep = _intensity_report(o["I"], k["I"])
    print("torus 1024 strided vs oracle:", rep)
    assert rep["rel_max"] <= 1e-5 and rep["above"] > 1500
    r.close()


def test_deferred_fp64_sums_multi_sample_frame(so, orc):
    """The plain FP64 tracer on a torus frame of >= 4096 pixels defers its turbulence sums and its
    emission (recording pass, k_turb64_records, k_emit64_records, k_transfer64), one record chain
    per sample.  A 64 x 64 frame at 2 samples per pixel equals, bit for bit, the same frame with the
    record pool capped so that nearly every sample is summed in the tracer by the replay pass
    instead, and matches the oracle's pass 1 within 1e-6 of the frame maximum."""
    n = 64
    sh = so.Shot("synchrotron_1024.ini", [f"camera.width={n}", f"camera.height={n}", "render.spp=2",
                                          "render.spp_max=2", "flow.n0=1594262.8"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    p = sh.plasma()
    modes = r.set_plasma(p)
    f = sh.frame(0)
    r.set_precision(so.abi.SO_PREC_FP64)
    a, _, sa = r.render(f)
    assert sa.rec64_slots > 0 and sa.rec64_short == 0 and sa.rec64_records > 0 and sa.emit64 == 1
    r.set_precision(so.abi.SO_PREC_FP64, pool_mb=0.001)  # two segments: the rest is summed in place
    b, _, sb = r.render(f)
    assert sb.rec64_short > 0.9 * n * n * 2
    assert np.array_equal(a, b)
    assert sa.attempts == sb.attempts and sa.flow_steps == sb.flow_steps
    acc, ys, lim, att = orc.orc_pass1(sh.scene, f, plasma=p, modes=modes, threads=_threads())
    ref = acc / 2.0
    assert ref[..., 0].max() > 0
    assert np.abs(a - ref).max() <= 1e-6 * ref[..., 0].max()
    assert sa.attempts == att
    r.close()


def _deferred_pair(so, overrides):
    """One torus frame rendered twice through the plain FP64 path: with deferred emission
    (k_emit64_records + k_transfer64) and with the record pool capped to two segments, so that the
    recording pass runs short and the replay pass (in-tracer emission) renders the frame."""
    sh = so.Shot("synchrotron_1024.ini", overrides)
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_plasma(sh.plasma())
    f = sh.frame(0)
    r.set_precision(so.abi.SO_PREC_FP64)
    a, _, sa = r.render(f)
    r.set_precision(so.abi.SO_PREC_FP64, pool_mb=0.001)
    b, _, sb = r.render(f)
    r.close()
    return a, sa, b, sb


def _counts(st):
    return st.attempts, st.accepted, st.flow_steps, st.step_limited, st.samples


def test_deferred_fp64_emission_opacity_cut(so):
    """Deferred emission ends a sample at the transfer's 1e-5 opacity cut with the counts recorded at
    that step.  At the normalised density and at 1000 times it (where many rays are cut), the frame
    and every counter equal the replay pass's bit for bit, and the dense frame makes fewer attempts
    than the same geometry without cuts."""
    n = 64
    base = [f"camera.width={n}", f"camera.height={n}", "render.spp=2", "render.spp_max=2"]
    thin = _deferred_pair(so, base + ["flow.n0=1594262.8"])
    thick = _deferred_pair(so, base + ["flow.n0=1594262800.0"])
    for a, sa, b, sb in (thin, thick):
        assert sa.emit64 == 1 and sa.rec64_short == 0 and sa.ms_emit64 > 0
        assert sb.emit64 == 0 and sb.rec64_short > 0
        assert np.array_equal(a, b)
        assert _counts(sa) == _counts(sb)
    assert thick[1].attempts < thin[1].attempts
    print("opacity cut: attempts", thin[1].attempts, "->", thick[1].attempts)


def test_deferred_fp64_emission_adaptive_chunks(so):
    """Adaptive pass 2 on a torus frame (chunks of 8 samples, well over the deferral threshold of
    4096 jobs): the frame with deferred emission in both passes equals the replay pass's bit for
    bit, counters included."""
    n = 128
    a, sa, b, sb = _deferred_pair(so, [f"camera.width={n}", f"camera.height={n}", "render.spp=2",
                                       "render.spp_max=34", "render.target_error=0.005", "flow.n0=1594262.8"])
    assert sa.samples - n * n * 2 >= 4096 * 8, sa.samples  # pass 2 ran at least 4096 chunks
    assert sa.emit64 == 1 and sb.emit64 == 0
    assert np.array_equal(a, b)
    assert _counts(sa) == _counts(sb)


def test_deferred_fp64_waves(so):
    """A record pool that holds about a third of the frame: the deferred passes run in waves of
    consecutive jobs, and the frame and every counter equal the single-wave frame's bit for bit."""
    n = 128
    ov = [f"camera.width={n}", f"camera.height={n}", "render.spp=2", "render.spp_max=2", "flow.n0=1594262.8"]

    def render(pool_mb):
        sh = so.Shot("synchrotron_1024.ini", ov)
        r = so.Renderer(sh.scene, sh.tables, sh.settings)
        r.set_plasma(sh.plasma())
        r.set_precision(so.abi.SO_PREC_FP64, pool_mb=pool_mb)
        img, _, st = r.render(sh.frame(0))
        r.close()
        return img, st

    a, sa = render(0.0)
    b, sb = render(140.0)
    print("waves:", sa.rec64_waves, "->", sb.rec64_waves, "records", sa.rec64_records, sb.rec64_records)
    assert sa.rec64_waves == 1 and sb.rec64_waves >= 3
    assert sa.emit64 == 1 and sb.emit64 == 1 and sb.rec64_short == 0
    assert sa.rec64_records == sb.rec64_records
    assert np.array_equal(a, b)
    assert _counts(sa) == _counts(sb)


@pytest.mark.parametrize("noise", ["BAKED", "BAKED_FP32", "INLINE"])
def test_deferred_fp64_emission_reference_flow(so, noise):
    """Frames of the reference flow model defer their emission too (recording pass,
    k_emit64_records, k_transfer64).  For each turbulence fetch (texture unit, FP32 trilinear,
    in-place noise) the frame and its counters equal the in-tracer frame's (record pool capped to
    one segment, so the replay pass renders it) bit for bit."""
    n = 96
    sh = so.Shot("m87_reference_flow.ini", [f"camera.width={n}", f"camera.height={n}", "render.spp=2",
                                            "render.spp_max=2"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_flow_noise(getattr(so.abi, "SO_FLOW_NOISE_" + noise))
    f = sh.frame(0)
    r.set_precision(so.abi.SO_PREC_FP64)
    a, _, sa = r.render(f)
    r.set_precision(so.abi.SO_PREC_FP64, pool_mb=0.001)
    b, _, sb = r.render(f)
    r.close()
    assert sa.emit64 == 1 and sa.rec64_records > 0 and sa.rec64_short == 0 and sa.ms_sum64 < 0.05
    assert sb.emit64 == 0 and sb.rec64_short > 0
    assert a[..., 0].max() > 0
    assert np.array_equal(a, b)
    assert _counts(sa) == _counts(sb)


_LIST_CASES = {
    # shot, density override (normal, 1000x), set-up
    "flow_inline": ("m87_reference_flow.ini", "flow.n0", 3e5,
                    lambda so, r, sh: r.set_flow_noise(so.abi.SO_FLOW_NOISE_INLINE)),
    "flow_texture": ("m87_reference_flow.ini", "flow.n0", 3e5, lambda so, r, sh: None),
    "torus": ("synchrotron_1024.ini", "flow.n0", 1594262.8, lambda so, r, sh: r.set_plasma(sh.plasma())),
}


def _list_pair(so, case, scale, n=72):
    """n x n pixel centres (over the deferral threshold of 4096 rays) through so_trace_rays twice:
    with the deferred passes, and with the record pool capped to one segment, so that the replay
    pass (emission in the tracer) traces the list."""
    shot, key, n0, setup = _LIST_CASES[case]
    sh = so.Shot(shot, [f"camera.width={n}", f"camera.height={n}", f"{key}={n0 * scale!r}"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    setup(so, r, sh)
    f = sh.frame(0)
    X, Y = so.pixel_centres(f, n, n)
    r.set_precision(so.abi.SO_PREC_FP64)
    a = r.trace_rays(f, X, Y, cross=True)
    sa = r.trace_stats()
    r.set_precision(so.abi.SO_PREC_FP64, pool_mb=0.001)
    b = r.trace_rays(f, X, Y, cross=True)
    sb = r.trace_stats()
    r.close()
    return a, sa, b, sb


@pytest.mark.parametrize("case", sorted(_LIST_CASES))
def test_deferred_fp64_ray_list(so, case):
    """Ray lists defer their emission like frames: the recording pass writes each ray's outputs
    without emission, and the ordered transfer writes its intensity and, for a ray the 1e-5 opacity
    cut ends, the tracer's outputs at the cut (captured, no escape direction, that step's counts,
    winding order and crossings).  At the normal density and at 1000 times it, every per-ray output
    (fate, winding order, escape direction, intensity, step counts, the first three crossings'
    radius and redshift) and the counters equal the in-tracer list's bit for bit."""
    out = {}
    for scale in (1.0, 1000.0):
        a, sa, b, sb = _list_pair(so, case, scale)
        assert sa.emit64 == 1 and sa.rec64_short == 0 and sa.rec64_records > 0 and sa.samples == a["fate"].size
        assert sb.emit64 == 0 and sb.rec64_short > 0
        for k in a:
            assert np.array_equal(a[k], b[k]), (scale, k)
        assert _counts(sa) == _counts(sb)
        assert a["I"][:, 0].max() > 0
        out[scale] = (a, sa)
    (thin, st), (thick, sk) = out[1.0], out[1000.0]
    cut = (thick["fate"] == -1) & (thin["fate"] != -1)
    fewer = thick["ncross"] < thin["ncross"]
    print(f"{case}: rays cut on their opacity {int(cut.sum())}, crossings dropped {int(fewer.sum())}, "
          f"attempts {st.attempts} -> {sk.attempts}")
    assert cut.any() and sk.attempts < st.attempts
    assert np.all(thick["theta"][cut] == 0) and np.all(thick["n_attempts"] <= thin["n_attempts"])


def test_deferred_fp64_torus_without_modes(so, orc):
    """The torus plasma without turbulence (n_modes = 0) defers its emission through records of the
    flow form (no sums), with the torus's own vertical profile deciding which steps record and the
    torus density in the emission: a 96 x 96 frame (2 samples) equals the in-tracer frame bit for
    bit, counters included, and a 64 x 64 ray list (4096 rays, deferred) equals the oracle (geometry
    exact, intensity within 1e-6 of the maximum)."""
    ov = ["so.modes=0", "flow.n0=1594262.8"]
    a, sa, b, sb = _deferred_pair(so, ["camera.width=96", "camera.height=96", "render.spp=2", "render.spp_max=2", *ov])
    assert sa.emit64 == 1 and sa.rec64_records > 0 and sa.rec64_short == 0 and sa.ms_sum64 < 0.05
    assert sb.emit64 == 0 and sb.rec64_short > 0
    assert a[..., 0].max() > 0
    assert np.array_equal(a, b)
    assert _counts(sa) == _counts(sb)
    n = 64
    sh = so.Shot("synchrotron_1024.ini", [f"camera.width={n}", f"camera.height={n}", *ov])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    p = sh.plasma()
    assert p.n_modes == 0
    r.set_plasma(p)
    f = sh.frame(0)
    X, Y = so.pixel_centres(f, n, n)
    k = r.trace_rays(f, X, Y)
    st = r.trace_stats()
    r.close()
    assert st.emit64 == 1 and st.rec64_short == 0
    o = orc.orc_trace(sh.scene, f, X, Y, plasma=p, threads=_threads())
    _cmp_geometry(o, k, rtol_dir=1e-12)
    I0, I1 = o["I"].astype(np.float64), k["I"].astype(np.float64)
    assert I0[:, 0].max() > 0
    assert np.abs(I0 - I1).max() <= 1e-6 * I0[:, 0].max()


def test_deferred_fp64_ray_list_waves(so):
    """A ray list whose records the pool holds only in part runs the deferred passes in waves of
    consecutive rays (each writing its rays' outputs at their own indices): 256 x 256 pixel centres
    on the reference flow model with a pool planned for about 40 % of the rays, every output and
    counter bit-identical to the single-wave list."""
    n = 256
    sh = so.Shot("m87_reference_flow.ini", [f"camera.width={n}", f"camera.height={n}", "flow.n0=3e7"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_flow_noise(so.abi.SO_FLOW_NOISE_INLINE)
    f = sh.frame(0)
    X, Y = so.pixel_centres(f, n, n)
    r.set_precision(so.abi.SO_PREC_FP64)
    a = r.trace_rays(f, X, Y, cross=True)
    sa = r.trace_stats()
    # the pool is planned from the records per ray seen so far (1.5 x, at least 320) plus a partly
    # filled segment per ray: size it for about 40 % of the rays, segments of 16 records of 7 doubles
    # with their 12 bytes of links
    est = max(320.0, 1.5 * sa.rec64_records / (n * n))
    r.set_precision(so.abi.SO_PREC_FP64, pool_mb=n * n / 2.5 * (est / 16 + 1) * (16 * 7 * 8 + 12) / 2 ** 20)
    b = r.trace_rays(f, X, Y, cross=True)
    sb = r.trace_stats()
    r.close()
    print("ray list waves:", sa.rec64_waves, "->", sb.rec64_waves, "records", sa.rec64_records, sb.rec64_records,
          "cut", int((a["fate"] == -1).sum()))
    assert sa.rec64_waves == 1 and sb.rec64_waves >= 2
    assert sa.emit64 == 1 and sb.emit64 == 1 and sb.rec64_short == 0
    assert sa.rec64_records == sb.rec64_records
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert _counts(sa) == _counts(sb)


def test_trace_stats_state(so):
    """so_trace_stats reports the last ray list only: after a frame it is a state error."""
    sh = so.Shot("shadow_selftest_256.ini", ["camera.width=16", "camera.height=16"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    f = sh.frame(0)
    X, Y = so.pixel_centres(f, 16, 16)
    k = r.trace_rays(f, X, Y)
    st = r.trace_stats()
    assert st.samples == 256 and st.accepted == int(k["n_accepted"].sum()) and st.attempts == int(k["n_attempts"].sum())
    assert st.emit64 == 0 and st.rec64_waves == 0
    r.render(f)
    with pytest.raises(so.TracerError) as e:
        r.trace_stats()
    assert e.value.code == so.abi.SO_ERR_STATE
    r.close()


def test_torus_plasma_vs_oracle(so, orc):
    """Synchrotron torus with 512 Fourier modes (FP64 everywhere), 40 x 40 over the +-12 M field."""
    sh = so.Shot("synchrotron_1024.ini", ["camera.width=40", "camera.height=40"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    p = sh.plasma()
    modes = r.set_plasma(p)
    f = sh.frame(0)
    X, Y = so.pixel_centres(f, 40, 40)
    k = r.trace_rays(f, X, Y)
    o = orc.orc_trace(sh.scene, f, X, Y, plasma=p, modes=modes)
    _cmp_geometry(o, k, rtol_dir=1e-12)
    I0, I1 = o["I"].astype(np.float64), k["I"].astype(np.float64)
    assert I0[:, 0].max() > 0
    assert np.abs(I0 - I1).max() <= 1e-6 * I0[:, 0].max()
    r.close()


def test_thin_disk_vs_oracle_and_golden(so, orc):
    g = np.load(os.path.join(GOLD, "disk_rays.npz"))
    sh = so.Shot("thin_disk_4096.ini", ["camera.width=40", "camera.height=40"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    f = sh.frame(0)
    k = r.trace_rays(f, g["x"], g["y"])
    o = orc.orc_trace(sh.scene, f, g["x"], g["y"])
    _cmp_geometry(o, k, rtol_dir=1e-12)
    scale = np.abs(g["I"]).max()
    # the disk colour is a float stage (expf of the NT table, logf into the blackbody table): device
    # and host float exp/log round differently in the last bits, amplified by the Planck slope
    assert np.abs(k["I"].astype(np.float64) - o["I"]).max() <= 1e-5 * scale
    assert np.array_equal(k["fate"], g["fate"])
    assert np.abs(k["I"].astype(np.float64) - g["I"]).max() <= 1e-5 * scale
    # per ray (the oracle is bit-identical to the reference on every one of these rays): the device's
    # float expf / logf in the temperature and blackbody stages move a pixel by at most ~2e-5 relative
    rep = _intensity_report(g["I"][:, 1:2], k["I"][:, 1:2])
    print("thin disk vs reference (Y):", rep)
    assert rep["rel_max"] <= 1e-4
    r.close()


def test_render_pass1_jitter_vs_oracle(so, orc):
    """so_render with spp = 2 R2-jittered samples, no adaptive pass and the flow turbulence baked for
    the frame (FP32 fetch, which the oracle repeats) == oracle pass 1 / spp."""
    sh = so.Shot("m87_reference_flow.ini", ["camera.width=32", "camera.height=24", "render.spp=2",
                                            "render.spp_max=2"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_flow_noise(so.abi.SO_FLOW_NOISE_BAKED_FP32)
    f = sh.frame(0)
    img, hdr, st = r.render(f)
    acc, ys, lim, att = orc.orc_pass1(orc.baked(sh.scene), f)
    ref = acc / 2.0
    assert np.abs(img - ref).max() <= 1e-6 * ref[..., 0].max()
    assert st.samples == 32 * 24 * 2 and st.step_limited == lim and st.attempts == att
    assert hdr.lum_max > 0 and 0 < hdr.lum_percentile <= hdr.lum_max
    r.close()


def test_adaptive_render_deterministic(so):
    """Adaptive pass 2 (k_adapt, k_dilate, scan, chunked samples) is deterministic and adds samples."""
    sh = so.Shot("m87_reference_flow.ini", ["camera.width=48", "camera.height=32", "render.spp=2",
                                            "render.spp_max=34", "render.target_error=0.02"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    f = sh.frame(0)
    a, _, s1 = r.render(f)
    b, _, s2 = r.render(f)
    assert np.array_equal(a, b)
    assert s1.samples > 48 * 32 * 2 and s1.samples == s2.samples
    assert (s1.samples - 48 * 32 * 2) % 8 == 0
    r.close()


def test_radio_flux_matches_image_sum(so, orc):
    sh = so.Shot("m87_reference_flow.ini", ["camera.width=64", "camera.height=64", "flow.turbulence=0"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    f = sh.frame(0, W=24)
    jy = r.radio_flux(f, 24, 1.0)
    f.W, f.H, f.spp = 24, 24, 2
    acc, _, _, _ = orc.orc_pass1(sh.scene, f)
    ref = (acc[..., 0] / np.float32(2)).astype(np.float64).sum() / 1e-23
    assert abs(jy - ref) <= 1e-6 * ref
    r.close()


def test_status_codes_on_gpu(so):
    sh = so.Shot("shadow_selftest_256.ini")
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    f = sh.frame(0)
    import ctypes as C
    L = so.lib()
    out = np.zeros((256, 256, 4), np.float32)
    hdr = so.abi.HdrFrame(256, 256, out.ctypes.data_as(C.POINTER(C.c_float)), 0, 0)
    post = so.abi.Post(1.5, 0.0, 0.0)  # bloom strength outside [0, 1]
    assert L.so_render(r.h, C.byref(f), C.byref(post), 0.5, C.byref(hdr), None) == so.abi.SO_ERR_ARG
    jy = C.c_double()
    assert L.so_radio_flux(r.h, C.byref(f), 300, 1.0, C.byref(jy)) == so.abi.SO_ERR_SIZE
    assert b"frame buffers" in L.so_last_error(r.h)
    p = so.abi.Plasma()
    p.model = so.abi.SO_PLASMA_TORUS
    p.n_modes = 5000
    p.h_sph = 0.3
    assert L.so_set_plasma(r.h, C.byref(p), None) == so.abi.SO_ERR_SIZE
    # the renderer stays usable after the rejected calls
    k = r.trace_rays(f, np.array([0.0, 0.01]), np.array([0.0, 0.0]))
    assert k["fate"][0] == -1 and k["fate"][1] == 1
    r.close()


def test_step_limit_counts(so, orc):
    """max_steps bounds every ray; step-limited samples are reported (render.cu:83, 126)."""
    sh = so.Shot("shadow_selftest_256.ini", ["render.max_steps=50", "camera.width=16", "camera.height=16"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    f = sh.frame(0)
    X, Y = so.pixel_centres(f, 16, 16)
    k = r.trace_rays(f, X, Y)
    o = orc.orc_trace(sh.scene, f, X, Y)
    assert np.array_equal(k["fate"], o["fate"]) and (k["fate"] == 0).all()
    assert (k["n_attempts"] == 50).all()
    r.close()
