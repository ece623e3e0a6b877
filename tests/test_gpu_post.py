"""Post filters on the GPU (so_render with so_post): the radio interferometer beam and the visible
glare against the CPU oracle oracle/so_post.py applied to the same unfiltered frame (largest
difference <= 1e-5 of the frame's maximum: both sum the same float taps, in different orders)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_radio_beam_matches_oracle(so, orc):
    sh = so.Shot("synchrotron_1024.ini", ["camera.width=96", "camera.height=80", "flow.n0=1594262.8"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_plasma(sh.plasma())
    f = sh.frame(0)
    img, _, _ = r.render(f)
    assert img[..., 0].max() > 0
    for sigma in (2.0, 7.0, 13.0):  # levels 0, 1 and 2 of the pyramid
        out, _, _ = r.render(f, blur_sigma_px=sigma)
        ref = orc.post().radio_blur(img.astype(np.float64), sigma)
        err = np.abs(out - ref).max() / np.abs(ref).max()
        assert err <= 1e-5, (sigma, err)
    # below half a pixel the beam is not applied
    out, _, _ = r.render(f, blur_sigma_px=0.4)
    assert np.array_equal(out, img)
    r.close()


def test_visible_glare_matches_oracle(so, orc):
    sh = so.Shot("thin_disk_4096.ini", ["camera.width=96", "camera.height=80"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    f = sh.frame(0)
    img, _, _ = r.render(f)
    out, hdr, _ = r.render(f, bloom=0.3)
    ref = orc.post().bloom(img.astype(np.float64), 0.3)
    err = np.abs(out - ref).max() / np.abs(ref).max()
    assert err <= 1e-5, err
    assert np.array_equal(out[..., 3], img[..., 3])  # the order channel is untouched
    r.close()


def _lum_stats(img, radio, hide, p):
    """The reference's host luminance statistics (render.cu:771-790) in numpy, same roundings."""
    c = img.reshape(-1, 4).astype(np.float32)
    if radio:
        d = np.maximum(((c[:, 0] - c[:, 1]) - c[:, 2]) - c[:, 3], np.float32(0))
        Y = (c[:, 0] - np.float32(hide) * d).astype(np.float64)
    else:
        Y = (0.2126 * c[:, 0].astype(np.float64) + 0.7152 * c[:, 1].astype(np.float64)) + \
            0.0722 * c[:, 2].astype(np.float64)
    pos = Y > 0
    mx = float(Y[pos].max()) if pos.any() else 0.0
    lum = Y[pos].astype(np.float32)
    sig = lum[lum.astype(np.float64) > mx * 1e-5]
    if sig.size == 0:
        return 0.0, mx
    idx = min(sig.size - 1, int(p * (sig.size - 1)))
    return float(np.partition(sig, idx)[idx]), mx


@pytest.mark.parametrize("shot, radio, hide, pct", [
    ("m87_reference_flow.ini", True, 0.0, 0.995),
    ("m87_reference_flow.ini", True, 0.6, 0.5),
    ("thin_disk_4096.ini", False, 0.0, 0.9),
    ("thin_disk_4096.ini", False, 0.0, 1.0),
])
def test_luminance_statistics_exact(so, shot, radio, hide, pct):
    """so_render's luminance maximum and percentile (computed on the device by radix selection) are
    exactly the reference's host statistics of the returned frame."""
    sh = so.Shot(shot, ["camera.width=80", "camera.height=60", "render.spp=1", "render.spp_max=1"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    img, hdr, _ = r.render(sh.frame(0), percentile=pct, hide_direct=hide)
    pv, mx = _lum_stats(img, radio, hide, pct)
    assert mx > 0
    assert hdr.lum_max == mx, (hdr.lum_max, mx)
    assert hdr.lum_percentile == pv, (hdr.lum_percentile, pv)
    with pytest.raises(so.TracerError):
        r.render(sh.frame(0), percentile=1.5)
    r.close()
