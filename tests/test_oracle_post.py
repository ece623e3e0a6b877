"""CPU checks of the post-filter oracle (oracle/so_post.py): level sizes as the reference's pyramid,
constant frames unchanged by bloom and blur, a point spread by the beam into a Gaussian of the
requested width, and the golden fixture of the reference's own filter kernels (the reference ships
no test vectors for them; tests/golden/make_golden.py runs its k_down / k_bloom / k_gauss /
k_upsample on the host)."""
import os

import numpy as np

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_level_sizes(orc):
    p = orc.post()
    assert p.level_sizes(7, 5) == [(7, 5), (4, 3), (2, 2)]
    assert len(p.level_sizes(2048, 2048)) == 9


def test_constant_frames(orc):
    p = orc.post()
    img = np.ones((37, 53, 4)) * np.array([1.0, 2.0, 3.0, 4.0])
    assert np.allclose(p.bloom(img, 0.4), img)
    for s in (1.2, 7.5, 40.0):
        assert np.allclose(p.radio_blur(img, s), img)


def test_beam_width(orc):
    p = orc.post()
    img = np.zeros((129, 129, 4))
    img[64, 64, 0] = 1.0
    out = p.radio_blur(img, 2.5)[..., 0]
    assert abs(out.sum() - 1.0) < 1e-9
    yy, xx = np.mgrid[0:129, 0:129]
    var = (out * (xx - 64) ** 2).sum() / out.sum()
    assert abs(np.sqrt(var) - 2.5) < 0.05


def test_filters_vs_reference_kernels(orc):
    """The oracle (FP64) against the reference's float32 kernels, through all four pyramid levels
    that the beams reach (0 .. 3, with k_upsample) and both bloom strengths: within 2e-6 of the
    frame maximum, the rounding of the reference's float32 sums."""
    p = orc.post()
    g = np.load(os.path.join(GOLD, "post_filters.npz"))
    cases = [k for k in g.files if k not in ("a", "b")]
    assert len(cases) == 7
    for k in cases:
        src = g[k[0]]
        kind, val = k.split("_")[1:]
        o = p.bloom(src, float(val)) if kind == "bloom" else p.radio_blur(src, float(val))
        ref = g[k]
        assert np.abs(o - ref).max() <= 2e-6 * np.abs(ref).max(), k
    # the fixture exercises the deeper levels: a 30-pixel beam runs on level 3 of 64 x 48
    assert p.level_sizes(64, 48)[3] == (8, 6)
