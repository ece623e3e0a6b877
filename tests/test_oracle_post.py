"""CPU checks of the post-filter oracle (oracle/so_post.py): level sizes as the reference's pyramid,
constant frames unchanged by bloom and blur, and a point spread by the beam into a Gaussian of the
requested width (the reference has no test vectors for these filters)."""
import numpy as np


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
