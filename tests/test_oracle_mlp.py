"""CPU checks of the surrogate oracle (oracle/so_mlp.py): its parameter layout against the library's
header, its BF16 rounding against known values, and its analytic gradient against central finite
differences in float64 (the oracle has no reference counterpart to be pinned to, so the
finite-difference check is its pin)."""
import numpy as np


def _random_case(m, n=96, seed=3):
    rng = np.random.default_rng(seed)
    lay, total = m.layout()
    p = np.zeros(total)
    for l, (w, b, nn, k) in enumerate(lay):
        rows = nn if l < m.NHID else m.NOUT
        W = rng.uniform(-1, 1, (nn, k)) / np.sqrt(k)
        W[rows:] = 0.0
        p[w:w + nn * k] = W.ravel()
        p[b:b + rows] = rng.uniform(-1, 1, rows) / np.sqrt(k)
    freq = rng.normal(0, 2.0, (m.NFREQ, 4))
    rays = np.stack([rng.uniform(-12, 12, n), rng.uniform(-12, 12, n), rng.uniform(0, 0.99, n),
                     rng.uniform(5, 175, n)], axis=1)
    tgt = np.zeros((n, 12))
    tgt[:, 0] = rng.integers(0, 3, n)
    d = rng.normal(size=(n, 3))
    tgt[:, 1:4] = d / np.linalg.norm(d, axis=1, keepdims=True) * (tgt[:, :1] == 0)
    u = rng.uniform(0, 0.5, (n, 3)) * (rng.uniform(size=(n, 3)) < 0.7)
    tgt[:, 4:7] = u
    tgt[:, 7:10] = np.where(u > 0, rng.uniform(0.3, 1.4, (n, 3)), -1.0)
    return p, freq, rays, tgt


def test_layout_matches_header(orc, so):
    m = orc.mlp()
    lay, total = m.layout()
    assert total == so.abi.SUR_NPARAMS
    assert all(w % 8 == 0 for (w, _, _, _) in lay)


def test_bf16_rounding(orc):
    m = orc.mlp()
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -3.140625, 1e-3, 65504.0])
    got = m.bf16(x)
    want = np.array([1.0, 1.0, 1.0 + 2 ** -7, -3.140625, 0.00099945068359375, 65536.0])
    assert np.array_equal(got, want), got
    import torch
    r = np.random.default_rng(1).normal(size=10000) * 10.0 ** np.random.default_rng(2).integers(-6, 6, 10000)
    ref = torch.tensor(r, dtype=torch.float32).to(torch.bfloat16).double().numpy()
    assert np.array_equal(m.bf16(r), ref)


def test_gradient_against_finite_differences(orc):
    m = orc.mlp()
    p, freq, rays, tgt = _random_case(m)
    g, _ = m.gradients(p, freq, rays, tgt)
    lay, total = m.layout()
    rng = np.random.default_rng(7)
    idx = []
    for l, (w, b, n, k) in enumerate(lay):
        rows = n if l < m.NHID else m.NOUT
        idx += list(w + rng.integers(0, rows * k, 6)) + list(b + rng.integers(0, rows, 3))
    h = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += h
        lp = m.mean_loss(q, freq, rays, tgt)
        q[i] -= 2 * h
        lm = m.mean_loss(q, freq, rays, tgt)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_mode_stays_close_to_exact(orc):
    """The GPU's rounding points move the gradient by about the BF16 unit roundoff, not more."""
    m = orc.mlp()
    p, freq, rays, tgt = _random_case(m, n=256, seed=5)
    g0, _ = m.gradients(p, freq, rays, tgt)
    g1, _ = m.gradients(p, freq, rays, tgt, rounding=True)
    assert np.linalg.norm(g1 - g0) / np.linalg.norm(g0) < 3e-2
