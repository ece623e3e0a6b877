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
