"""Mixed-precision path (FP32 far from the critical curve, FP64 in the band, at the far-field
approach and for re-traced rays) against the plain FP64 kernel on the same frames.

Bar (the synchrotron scene's target): relative L1 image error <= 1e-3 and total-flux error <= 0.1%
against the FP64 render; the band and re-trace lists are exercised.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _render_pair(so, shot, overrides, plasma=True, **mixed):
    sh = so.Shot(shot, overrides)
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    if plasma:
        r.set_plasma(sh.plasma())
    f = sh.frame(0)
    r.set_precision(so.abi.SO_PREC_FP64)
    img64, _, st64 = r.render(f)
    r.set_precision(so.abi.SO_PREC_MIXED, **mixed)
    img32, _, st32 = r.render(f)
    r.close()
    return img64, img32, st64, st32


def _errors(img64, img32):
    a, b = img64[..., 0].astype(np.float64), img32[..., 0].astype(np.float64)
    l1 = np.abs(a - b).sum() / np.abs(a).sum()
    flux = abs(b.sum() / a.sum() - 1.0)
    return l1, flux


# density of the 0.6 Jy normalisation of the synchrotron frame (the bench normalises it itself)
N0 = "flow.n0=1594262.8"


def test_mixed_synchrotron_image_error(so):
    """Torus plasma with 512 modes at 192^2 over the +-12 M field: L1 <= 1e-3, flux <= 0.1%."""
    img64, img32, st64, st32 = _render_pair(so, "synchrotron_1024.ini",
                                            ["camera.width=192", "camera.height=192", N0])
    l1, flux = _errors(img64, img32)
    assert img64[..., 0].max() > 0
    assert l1 <= 1e-3, l1
    assert flux <= 1e-3, flux
    assert st32.band_rays > 0 and st32.attempts_fp32 > 0
    assert st32.samples == st64.samples == 192 * 192


def test_mixed_turning_point_retrace(so):
    """turn_r > 0 re-traces the FP32 rays whose radial turning point falls inside it, in FP64."""
    img64, img32, _, st32 = _render_pair(so, "synchrotron_1024.ini", ["camera.width=96", "camera.height=96", N0],
                                         turn_r=3.5)
    assert st32.redo_turn > 0
    assert st32.fp64_rays == st32.band_rays + st32.redo_turn + st32.redo_drift + st32.redo_limit
    l1, flux = _errors(img64, img32)
    assert l1 <= 1e-3 and flux <= 1e-3


def test_mixed_reference_fbm_is_all_fp64(so):
    """The reference's fBm turbulence evaluated in place is ill-conditioned in the coordinate time, so
    the mixed path traces such scenes entirely in FP64: the image equals the FP64 one bit for bit."""
    sh = so.Shot("m87_reference_flow.ini", ["camera.width=48", "camera.height=48", "render.spp=1",
                                            "render.spp_max=1"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_flow_noise(so.abi.SO_FLOW_NOISE_INLINE)
    f = sh.frame(0)
    r.set_precision(so.abi.SO_PREC_FP64)
    img64, _, _ = r.render(f)
    r.set_precision(so.abi.SO_PREC_MIXED)
    img32, _, st32 = r.render(f)
    assert st32.band_rays == 48 * 48 and st32.attempts_fp32 == 0
    assert np.array_equal(img64, img32)
    r.close()


def test_mixed_reference_flow_baked_turbulence(so):
    """The same flow with its turbulence baked per frame (the renderer's default): sampled at the
    position and the retarded time, it is well conditioned, and the FP32 tracer takes the rays off
    the band.  Emission quadrature converged (step fraction 0.01) as for the flow without
    turbulence: L1 <= 2e-3, flux <= 1e-3 against the FP64 frame with the same baked field."""
    img64, img32, _, st32 = _render_pair(so, "m87_reference_flow.ini", ["camera.width=96", "camera.height=96",
                                                                         "render.spp=1", "render.spp_max=1",
                                                                         "render.step_fraction=0.01"], plasma=False)
    assert st32.attempts_fp32 > 0 and st32.band_rays < 96 * 96 // 4
    l1, flux = _errors(img64, img32)
    assert img64[..., 0].max() > 0
    assert l1 <= 2e-3 and flux <= 1e-3, (l1, flux)


def test_mixed_reference_flow_without_turbulence(so):
    """The reference's thin (h/r = 0.15) flow: at its step fraction 0.04 the emission quadrature moves
    by ~5e-3 with the step sequence, so compare with the quadrature converged (0.01)."""
    img64, img32, _, st32 = _render_pair(so, "m87_reference_flow.ini", ["camera.width=96", "camera.height=96",
                                                                         "render.spp=1", "render.spp_max=1",
                                                                         "flow.turbulence=0",
                                                                         "render.step_fraction=0.01"], plasma=False)
    assert st32.attempts_fp32 > 0
    l1, flux = _errors(img64, img32)
    assert l1 <= 2e-3 and flux <= 1e-3, (l1, flux)


def test_mixed_band_width_zero_and_all_fp64(so):
    """band 0: every ray starts FP32; a band covering the field: every ray has FP64 geometry (its
    turbulence sums are FP32, so the image is the FP64 one to FP32 emission precision)."""
    sh = so.Shot("synchrotron_1024.ini", ["camera.width=64", "camera.height=64", N0])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_plasma(sh.plasma())
    f = sh.frame(0)
    r.set_precision(so.abi.SO_PREC_FP64)
    img64, _, _ = r.render(f)
    r.set_precision(so.abi.SO_PREC_MIXED, band_m=1e6)
    imgb, _, stb = r.render(f)
    assert stb.band_rays == 64 * 64 and stb.attempts_fp32 == 0
    l1, flux = _errors(img64, imgb)
    assert l1 < 1e-4 and flux < 1e-5, (l1, flux)
    r.set_precision(so.abi.SO_PREC_MIXED, band_m=0.0)
    img0, _, st0 = r.render(f)
    assert st0.band_rays == 0
    l1, flux = _errors(img64, img0)
    assert l1 < 1e-2 and flux < 1e-2
    r.close()


def test_mixed_retrace_list(so):
    """A zero drift tolerance sends every FP32 ray back to FP64 geometry: the image then is the FP64
    one to FP32 emission precision."""
    sh = so.Shot("synchrotron_1024.ini", ["camera.width=48", "camera.height=48", N0])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_plasma(sh.plasma())
    f = sh.frame(0)
    r.set_precision(so.abi.SO_PREC_FP64)
    img64, _, _ = r.render(f)
    r.set_precision(so.abi.SO_PREC_MIXED, drift_tol=0.0)
    imgm, _, st = r.render(f)
    assert st.fp64_rays == 48 * 48
    l1, flux = _errors(img64, imgm)
    assert l1 < 1e-4 and flux < 1e-5, (l1, flux)
    r.close()


def test_mixed_deterministic(so):
    sh = so.Shot("synchrotron_1024.ini", ["camera.width=64", "camera.height=64", N0])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_plasma(sh.plasma())
    r.set_precision(so.abi.SO_PREC_MIXED)
    f = sh.frame(0)
    a, _, _ = r.render(f)
    b, _, _ = r.render(f)
    assert np.array_equal(a, b)
    r.close()


def test_mixed_classes_exact_outside_band(so):
    """Outside the critical band every sample of the mixed path ends with the FP64 termination class
    (the same samples traced with the band covering the field: FP64 geometry throughout)."""
    W = 192
    sh = so.Shot("synchrotron_1024.ini", [f"camera.width={W}", f"camera.height={W}", N0])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_plasma(sh.plasma())
    f = sh.frame(0)
    n = W * W * sh.settings.spp
    r.set_precision(so.abi.SO_PREC_MIXED)
    r.render(f)
    fm, band = r.last_fates(n)
    r.set_precision(so.abi.SO_PREC_MIXED, band_m=1e6)
    r.render(f)
    f64, allband = r.last_fates(n)
    assert allband.all()
    out = ~band
    assert 0.9 * n < out.sum() < n
    assert set(np.unique(f64)) >= {-1, 1}
    assert np.array_equal(fm[out], f64[out]), int((fm[out] != f64[out]).sum())
    r.close()


def _mixed_fates(so, r, f, n, **mixed):
    r.set_precision(so.abi.SO_PREC_MIXED, **mixed)
    img, _, st = r.render(f)
    fm, band = r.last_fates(n)
    return img, st, fm


def test_deferred_turbulence_matches_in_tracer_sums(so):
    """The deferred form (flow-step records, batched mode sums, warp-per-ray transfer) gives the
    image of the in-tracer sums within 1e-5 relative L1 (FP32 summation order and the scanned
    transmittance) and the same termination class for every sample, also at a density 1000 times
    the normalised one, where the transfer ends many rays on their opacity."""
    W = 128
    thin = None
    for n0, opaque in ((N0, False), ("flow.n0=1594262800.0", True)):
        sh = so.Shot("synchrotron_1024.ini", [f"camera.width={W}", f"camera.height={W}", n0])
        r = so.Renderer(sh.scene, sh.tables, sh.settings)
        r.set_plasma(sh.plasma())
        f = sh.frame(0)
        n = W * W * sh.settings.spp
        a, sa, fa = _mixed_fates(so, r, f, n, turbulence=1)
        b, sb, fb = _mixed_fates(so, r, f, n, turbulence=0)
        assert sa.turb_records == 0 and sb.turb_records >= sb.flow_steps_fp32 > 0
        assert sb.redo_records == 0
        l1, flux = _errors(a, b)
        assert l1 <= 1e-5 and flux <= 1e-5, (l1, flux)
        assert np.array_equal(fa, fb), int((fa != fb).sum())
        if opaque:
            # ended on opacity: captured where the normal-density frame escapes
            assert ((fb == -1) & (thin == 1)).sum() > 100
        thin = fb
        r.close()


@pytest.mark.parametrize("noise,turb", [("BAKED", []), ("BAKED_FP32", []), ("BAKED", ["flow.turbulence=0"])],
                         ids=["texture", "fp32_fetch", "no_turbulence"])
def test_deferred_emission_reference_flow(so, noise, turb):
    """The reference flow model's FP32 rays defer their emission too: the tracer records each flow
    step with the baked turbulence factor it fetched (as the in-line form fetches it) and the
    warp-per-ray transfer runs flow_step32 on the records.  The image equals the in-line form's
    within 1e-5 relative L1 (the scanned transmittance) with the same termination class for every
    sample, and stays within the mixed path's bar of the FP64 frame."""
    W = 96
    sh = so.Shot("m87_reference_flow.ini", [f"camera.width={W}", f"camera.height={W}", "render.spp=1",
                                            "render.spp_max=1", "render.step_fraction=0.01", *turb])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_flow_noise(getattr(so.abi, "SO_FLOW_NOISE_" + noise))
    f = sh.frame(0)
    n = W * W
    r.set_precision(so.abi.SO_PREC_FP64)
    img64, _, _ = r.render(f)
    a, sa, fa = _mixed_fates(so, r, f, n, turbulence=1)
    b, sb, fb = _mixed_fates(so, r, f, n, turbulence=0)
    r.close()
    assert sa.record_waves == 0 and sb.record_waves >= 1 and sb.turb_records == 0 and sb.redo_records == 0
    assert sb.attempts_fp32 > 0 and b[..., 0].max() > 0
    l1, flux = _errors(a, b)
    assert l1 <= 1e-5 and flux <= 1e-5, (l1, flux)
    assert np.array_equal(fa, fb), int((fa != fb).sum())
    l1, flux = _errors(img64, b)
    assert l1 <= 2e-3 and flux <= 1e-3, (l1, flux)


def test_deferred_turbulence_record_pool_shortage(so):
    """A record pool far too small for the frame: the rays that find no record slot are re-traced
    in FP64, so the image stays within the mixed path's bar of the FP64 frame, and the next frame's
    pool is larger."""
    W = 96
    sh = so.Shot("synchrotron_1024.ini", [f"camera.width={W}", f"camera.height={W}", N0])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_plasma(sh.plasma())
    f = sh.frame(0)
    r.set_precision(so.abi.SO_PREC_FP64)
    img64, _, _ = r.render(f)
    r.set_precision(so.abi.SO_PREC_MIXED, records_per_ray=1.0)
    img1, _, st1 = r.render(f)
    assert st1.redo_records > 0
    l1, flux = _errors(img64, img1)
    assert l1 <= 1e-3 and flux <= 1e-3, (l1, flux)
    redo = [st1.redo_records]
    for _ in range(8):
        _, _, st = r.render(f)
        redo.append(st.redo_records)
    assert redo[-1] < redo[0], redo
    with pytest.raises(so.TracerError):
        r.set_precision(so.abi.SO_PREC_MIXED, turbulence=2)
    r.close()


def test_deferred_turbulence_record_waves(so):
    """A record pool capped below the frame's records: the FP32 rays are traced in waves that each
    fit the pool, and once no ray runs short of records the image is bit-identical to the frame
    traced in one wave (every ray's result depends on the ray alone)."""
    W = 128
    sh = so.Shot("synchrotron_1024.ini", [f"camera.width={W}", f"camera.height={W}", N0])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_plasma(sh.plasma())
    f = sh.frame(0)
    r.set_precision(so.abi.SO_PREC_MIXED)
    one, _, st1 = r.render(f)
    assert st1.record_waves == 1 and st1.redo_records == 0
    r.set_precision(so.abi.SO_PREC_MIXED, pool_mb=2.0)
    for _ in range(6):  # a wave short of records doubles the estimate for the next frame
        img, _, st = r.render(f)
        if st.redo_records == 0:
            break
    assert st.redo_records == 0 and st.record_waves > 1, (st.redo_records, st.record_waves)
    assert st.turb_records == st1.turb_records
    assert np.array_equal(img, one)
    with pytest.raises(so.TracerError):
        r.set_precision(so.abi.SO_PREC_MIXED, pool_mb=-1.0)
    r.close()


def test_mixed_shadow_scene_classes(so):
    """The vacuum shadow self-test scene (a = 0.94, i = 17 deg, observer at 1000 M, pixel centres over
    +-8 M, tolerance 1e-10) through the mixed path: FP32 geometry outside the critical band, the
    scene's FP64 tolerance inside it.  Every sample outside the band ends with the termination class
    of the plain FP64 tracer, and the band holds the shadow edge."""
    W = 256
    sh = so.Shot("shadow_selftest_256.ini", [])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    f = sh.frame(0)
    n = W * W
    r.set_precision(so.abi.SO_PREC_MIXED)
    _, _, st = r.render(f)
    fm, band = r.last_fates(n)
    assert 0 < st.band_rays == int(band.sum()) < n // 4
    assert st.attempts_fp32 > 0
    r.set_precision(so.abi.SO_PREC_MIXED, band_m=1e6)
    r.render(f)
    f64, allband = r.last_fates(n)
    assert allband.all()
    out = ~band
    assert set(np.unique(f64[out])) == {-1, 1}
    assert np.array_equal(fm[out], f64[out]), int((fm[out] != f64[out]).sum())
    # the band straddles the shadow edge: both classes inside it
    assert (f64[band] == -1).any() and (f64[band] == 1).any()
    r.close()


@pytest.mark.parametrize("W,H", [(37, 23), (5, 3), (1, 1)])
def test_mixed_ragged_and_tiny_frames(so, W, H):
    """Frames of odd, non-square and sub-warp sizes through the mixed path (deferred turbulence on):
    every sample outside the band ends with the FP64 termination class, the image is finite and, at
    37 x 23, within the mixed path's bar of the FP64 frame."""
    sh = so.Shot("synchrotron_1024.ini", [f"camera.width={W}", f"camera.height={H}", N0])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_plasma(sh.plasma())
    f = sh.frame(0)
    n = W * H * sh.settings.spp
    r.set_precision(so.abi.SO_PREC_FP64)
    img64, _, _ = r.render(f)
    r.set_precision(so.abi.SO_PREC_MIXED)
    img, _, st = r.render(f)
    assert img.shape == (H, W, 4) and np.isfinite(img).all()
    fm, band = r.last_fates(n)
    r.set_precision(so.abi.SO_PREC_MIXED, band_m=1e6)
    r.render(f)
    f64, _ = r.last_fates(n)
    assert np.array_equal(fm[~band], f64[~band])
    if W * H > 100:
        assert st.turb_records > 0
        l1, flux = _errors(img64, img)
        assert l1 <= 1e-3 and flux <= 1e-3, (l1, flux)
    r.close()


def test_trace_rays_empty_list(so):
    """An empty ray list is a no-op through both the host and the device entry points."""
    sh = so.Shot("shadow_selftest_256.ini", ["camera.width=8", "camera.height=8"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    f = sh.frame(0)
    k = r.trace_rays(f, np.zeros(0), np.zeros(0))
    assert all(v.size == 0 for v in k.values() if isinstance(v, np.ndarray))
    import ctypes as C
    out = so.abi.RaysOut()
    assert so.lib().so_trace_rays_device(r.h, C.byref(f), 0, None, None, C.byref(out)) == so.abi.SO_OK
    assert so.lib().so_trace_rays(r.h, C.byref(f), -1, None, None, C.byref(out)) == so.abi.SO_ERR_ARG
    # still usable afterwards
    k = r.trace_rays(f, np.array([0.0, 0.01]), np.array([0.0, 0.0]))
    assert k["fate"][0] == -1 and k["fate"][1] == 1
    r.close()
