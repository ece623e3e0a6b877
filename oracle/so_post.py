"""so_post.py -- CPU oracle of the post filters.  TEST INFRASTRUCTURE ONLY.

numpy restatement of the reference's pyramid filters on the HDR frame (blackholes/src/render.cu):
k_down (:245-254), bilinear (:256-270), k_bloom (:279-294), k_gauss (:296-310), k_upsample
(:312-316), the pyramid sizes (:638-647), Impl::bloom (:732-740) and Impl::radio_blur (:742-753).
Frames are float arrays [H, W, 4].  The reference ships no test vectors for these filters: this
oracle is checked by properties (constant frames stay constant, the blur spreads a point like a
Gaussian of the requested width) and against the reference's own kernels run on the host
(tests/golden/post_filters.npz, within 2e-6 of the frame maximum); the GPU filters are checked
against it.
"""
import numpy as np

MAX_LEVELS = 9


def level_sizes(W, H):
    out, w, h = [], W, H
    while len(out) < MAX_LEVELS and w >= 2 and h >= 2:
        out.append((w, h))
        w, h = (w + 1) // 2, (h + 1) // 2
    return out


def down(src, dw, dh):
    sh, sw = src.shape[:2]
    y = np.arange(dh)[:, None]
    x = np.arange(dw)[None, :]
    a = np.zeros((dh, dw, 4))
    for j in (0, 1):
        for i in (0, 1):
            a += src[np.minimum(2 * y + j, sh - 1), np.minimum(2 * x + i, sw - 1)]
    return 0.25 * a


def bilinear(L, x, y):
    h, w = L.shape[:2]
    x = np.clip(x - 0.5, 0.0, w - 1.001)
    y = np.clip(y - 0.5, 0.0, h - 1.001)
    ix, iy = x.astype(np.int64), y.astype(np.int64)
    fx, fy = (x - ix)[..., None], (y - iy)[..., None]
    ix1, iy1 = np.minimum(ix + 1, w - 1), np.minimum(iy + 1, h - 1)
    a, b, c, d = L[iy, ix], L[iy, ix1], L[iy1, ix], L[iy1, ix1]
    return (1 - fy) * ((1 - fx) * a + fx * b) + fy * ((1 - fx) * c + fx * d)


def pyramid(img, n=None):
    H, W = img.shape[:2]
    sizes = level_sizes(W, H)
    levs = [np.asarray(img, np.float64)]
    for k in range(1, len(sizes) if n is None else n):
        levs.append(down(levs[-1], *sizes[k]))
    return levs, sizes


def bloom(img, strength):
    levs, sizes = pyramid(img)
    H, W = img.shape[:2]
    y, x = np.meshgrid(np.arange(H) + 0.5, np.arange(W) + 0.5, indexing="ij")
    b = np.zeros((H, W, 3))
    ws = 0.0
    for k in range(1, len(levs)):
        w_k, h_k = sizes[k]
        v = bilinear(levs[k], x * w_k / W, y * h_k / H)
        b += v[..., :3] / k
        ws += 1.0 / k
    o = np.asarray(img, np.float64).copy()
    o[..., :3] = (1 - strength) * o[..., :3] + strength * b / ws
    return o


def gauss(src, sigma, horiz):
    h, w = src.shape[:2]
    R = int(np.ceil(3.0 * sigma))
    a = np.zeros_like(src, dtype=np.float64)
    ws = 0.0
    for i in range(-R, R + 1):
        wgt = np.exp(-0.5 * i * i / (sigma * sigma))
        if horiz:
            idx = np.clip(np.arange(w) + i, 0, w - 1)
            a += wgt * src[:, idx]
        else:
            idx = np.clip(np.arange(h) + i, 0, h - 1)
            a += wgt * src[idx, :]
        ws += wgt
    return a / ws


def radio_blur(img, sigma):
    H, W = img.shape[:2]
    sizes = level_sizes(W, H)
    k = 0
    while k + 1 < len(sizes) and sigma / (1 << (k + 1)) > 3.0:
        k += 1
    levs, _ = pyramid(img, k + 1)
    s = sigma / (1 << k)
    L = gauss(gauss(levs[k], s, True), s, False)
    if k == 0:
        return L
    y, x = np.meshgrid(np.arange(H) + 0.5, np.arange(W) + 0.5, indexing="ij")
    lw, lh = sizes[k]
    return bilinear(L, x * lw / W, y * lh / H)
