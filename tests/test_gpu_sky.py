"""Star map of the visible mode (so_set_sky, trace.cuh:24-43, 149-161, render.cu:40-72, 550-593).

The texture unit's anisotropic mip filtering of a sampled map has no CPU form, so:
  * a constant map, which every filter returns unchanged, checks the rest of the path exactly
    against the oracle: escape direction, galactic (u, v), blackbody at the camera-shifted
    temperature, brightness scale and the disk's transmittance in front (1e-5 of the maximum);
  * a map that varies linearly in latitude checks the (u, v) mapping, the rotation and the pixel
    footprints against the oracle's analytic map, within the texels' half precision (1 per cent);
  * the mixed path traces star-map frames in FP64 by default (bit for bit the plain image); with
    sky_fp32 (FP32 rays whose escape is carried to r_escape in FP64) both smooth maps stay within
    the mixed path's image bar of the FP64 frame (L1 <= 1e-3).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _texels(w, h, s_of_uv, T):
    u = (np.arange(w) + 0.5) / w
    v = (np.arange(h) + 0.5) / h
    s = s_of_uv(u[None, :], v[:, None]) * np.ones((h, w))
    t = np.empty((h, w, 2), np.uint16)
    t[..., 0] = s.astype(np.float16).view(np.uint16)
    t[..., 1] = (s * T / 1e4).astype(np.float16).view(np.uint16)
    return t


def _oracle_frame(orc, scene, f, sky):
    """Oracle pass 1 with the analytic map, resolved as so_render resolves a visible frame: the
    sample mean, XYZ to linear sRGB times 683 (render.cu:227-242)."""
    orc.oracle().orc_set_sky(*sky)
    try:
        acc, _, _, _ = orc.orc_pass1(scene, f)
    finally:
        orc.oracle().orc_set_sky(0.0, 0.0, 0.0, 0.0)
    a = acc.astype(np.float64) / f.spp
    X, Y, Z = a[..., 0], a[..., 1], a[..., 2]
    out = np.empty_like(a)
    out[..., 0] = 683.0 * (3.2404542 * X - 1.5371385 * Y - 0.4985314 * Z)
    out[..., 1] = 683.0 * (-0.9692660 * X + 1.8760108 * Y + 0.0415560 * Z)
    out[..., 2] = 683.0 * (0.0556434 * X - 0.2040259 * Y + 1.0572252 * Z)
    out[..., 3] = 683.0 * a[..., 3]
    return out


def _close(img, ref, tol):
    scale = np.abs(ref).max()
    return np.abs(img.astype(np.float64) - ref).max() / scale


def test_constant_sky_vs_oracle(so, orc):
    """Thin disk (r_out 7 M, so that the sky shows around it) in front of a constant star map
    (s = 2, T = 5000 K), 2 samples per pixel: within
    1e-5 of the frame's maximum, the bar of the disk's float colour stages."""
    W, H = 64, 48
    sh = so.Shot("thin_disk_4096.ini", [f"camera.width={W}", f"camera.height={H}", "render.spp=2",
                                        "render.spp_max=2", "sky.enabled=1", "sky.brightness=0.5",
                                        "disk.r_out=7"])
    assert sh.scene.sky_on == 1
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    f = sh.frame(0)
    dark, _, _ = r.render(f)  # no map given yet: no sky, as the reference without a texture
    ref_dark = _oracle_frame(orc, sh.scene, f, (0.0, 0.0, 0.0, 0.0))
    assert _close(dark, ref_dark, 1e-5) <= 1e-5
    r.set_sky(_texels(128, 64, lambda u, v: 2.0 + 0.0 * u, 5000.0))
    img, _, st = r.render(f)
    ref = _oracle_frame(orc, sh.scene, f, (2.0, 0.0, 0.0, 5000.0))
    assert _close(img, ref, 1e-5) <= 1e-5, _close(img, ref, 1e-5)
    sky_px = ((dark[..., 1] == 0) & (img[..., 1] > 0)).sum()  # no disk in front, sky behind
    assert sky_px > W * H // 4, sky_px
    # mixed path: star-map frames in FP64 by default (the plain image bit for bit) ...
    r.set_precision(so.abi.SO_PREC_MIXED)
    img64m, _, st64m = r.render(f)
    assert np.array_equal(img64m, img) and st64m.attempts_fp32 == 0
    # ... or, with sky_fp32, FP32 rays off the band whose escape is carried to r_escape in FP64
    r.set_precision(so.abi.SO_PREC_MIXED, sky_fp32=1)
    img32, _, st32 = r.render(f)
    assert st32.attempts_fp32 > 0
    a, b = img[..., 1].astype(np.float64), img32[..., 1].astype(np.float64)
    assert np.abs(a - b).sum() / np.abs(a).sum() <= 1e-3
    sky_only = (dark[..., 1] == 0) & (img[..., 1] > 0)
    assert np.abs(a[sky_only] - b[sky_only]).max() <= 1e-4 * a[sky_only].max()
    r.close()


def test_latitude_gradient_sky_vs_oracle(so, orc):
    """Vacuum, 40 x 40 degrees of sky: brightness 1 + v (v the galactic latitude coordinate),
    6000 K; per-pixel relative difference from the oracle's analytic map below 1 per cent away
    from the shadow's edge, total within 0.5 per cent."""
    W = 48
    sh = so.Shot("shadow_selftest_256.ini", [f"camera.width={W}", f"camera.height={W}", "render.spp=1",
                                             "render.spp_max=1", "sky.enabled=1", "camera.fov_m=700",
                                             "sky.b_deg=20"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    f = sh.frame(0)
    r.set_sky(_texels(512, 256, lambda u, v: 1.0 + v, 6000.0))
    img, _, _ = r.render(f)
    ref = _oracle_frame(orc, sh.scene, f, (1.0, 0.0, 1.0, 6000.0))
    y0, y1 = ref[..., 1], img[..., 1].astype(np.float64)
    lit = y0 > 0
    assert lit.sum() > W * W // 2
    rel = np.abs(y1[lit] - y0[lit]) / y0[lit]
    assert np.median(rel) < 1e-2 and np.percentile(rel, 90) < 1e-2, (np.median(rel), np.percentile(rel, 90))
    assert abs(y1.sum() / y0.sum() - 1.0) < 5e-3
    # the map's latitude gradient is visible across the frame
    assert y0[lit].max() / y0[lit].min() > 1.05
    # mixed path with sky_fp32 (FP32 rays, FP64 transport to r_escape) against the FP64 frame
    r.set_precision(so.abi.SO_PREC_MIXED, sky_fp32=1)
    img32, _, st32 = r.render(f)
    assert st32.attempts_fp32 > 0
    y2 = img32[..., 1].astype(np.float64)
    assert np.abs(y2 - y1).sum() / np.abs(y1).sum() <= 1e-3, np.abs(y2 - y1).sum() / np.abs(y1).sum()
    r.close()
