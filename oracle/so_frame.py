"""so_frame.py -- CPU oracle of the frame driver around the tracer.  TEST INFRASTRUCTURE ONLY.

numpy restatement of the reference's adaptive resampling (blackholes/src/render.cu) in the order the
CUDA path runs it: pass 1 (k_pass1, :89-128: accum and (sum Y, sum Y^2) per pixel), the frame
luminance sum and yref (Impl::trace, :700-703), k_adapt (:130-140), k_dilate (:142-150), the
exclusive scan (:152-194), pass 2 in chunks of CHUNK samples (k_pass2, :196-224) and k_resolve
(:227-242).  The reference adds the chunk sums to their pixels with float atomics (an order that
changes from run to run); this oracle adds them in chunk order, as the CUDA path does.

The samples themselves come from a callable that returns chunk sums (the C oracle's
orc_render_chunks, or the reference's own sample_pixel through ref_render_chunks), so this file
holds only the per-pixel arithmetic.  All per-pixel quantities are float32 as in the kernels; the
frame sum is FP64.
"""
import numpy as np

CHUNK = 8  # samples per pass-2 job (render.cu:30)
F32 = np.float32


def _fused_var(q, mean):
    """q - mean * mean with one rounding (the kernel's contracted multiply-subtract): mean^2 of a
    float is exact in FP64, so the FP64 difference rounds once more only in rare ties."""
    return (q.astype(np.float64) - mean.astype(np.float64) * mean.astype(np.float64)).astype(F32)


def adapt(ystat, spp, fsum, npix, target, extra_max):
    """k_adapt: extra samples per pixel so that the standard error of the mean luminance falls below
    target * (mean + yref); yref = 0.03 * (frame luminance sum) / (npix * spp)."""
    yref = F32(0.03 * fsum * (1.0 / (float(npix) * spp)) + 1e-37)
    n = F32(spp)
    sx, sy = ystat[..., 0].astype(F32), ystat[..., 1].astype(F32)
    mean = sx / n
    var = np.maximum(_fused_var(sy / n, mean), F32(0))
    se = np.sqrt(var / n).astype(F32)
    den = F32(target) * (mean + yref)
    q = se / den
    want = (n * q) * q
    return np.minimum(np.maximum(np.ceil(want) - n, F32(0)), F32(extra_max)).astype(np.uint32)


def dilate(extra, extra_max, chunk=CHUNK):
    """k_dilate: 3x3 maximum (edges clamped), capped at extra_max, in whole chunks."""
    H, W = extra.shape
    p = np.pad(extra, 1, mode="edge")
    m = np.zeros_like(extra)
    for dy in range(3):
        for dx in range(3):
            m = np.maximum(m, p[dy:dy + H, dx:dx + W])
    return (np.minimum(m, np.uint32(extra_max)) + np.uint32(chunk - 1)) // np.uint32(chunk)


def render_adaptive(acc1, ystat, spp, spp_max, target, chunk_sums, visible=False):
    """The adaptive frame from its pass-1 arrays (acc1 [H, W, 4], ystat [H, W, 2]).

    chunk_sums(pix, s0, count) -> float32 [len(pix), 4]: the sum of samples s0 .. s0 + count - 1 of
    each listed pixel.  Returns (image [H, W, 4], nsamp [H, W], chunks [H, W])."""
    H, W = acc1.shape[:2]
    npix = W * H
    extra_max = max(spp_max - spp, 0)
    acc = acc1.astype(F32).copy()
    nsamp = np.full((H, W), spp, np.uint32)
    chunks = np.zeros((H, W), np.uint32)
    if extra_max > 0:
        fsum = float(np.sum(ystat[..., 0].astype(np.float64)))
        extra = adapt(ystat, spp, fsum, npix, target, extra_max)
        chunks = dilate(extra, extra_max)
        c = chunks.reshape(-1).astype(np.int64)
        offsets = np.concatenate([[0], np.cumsum(c)[:-1]])
        total = int(c.sum())
        if total:
            pix = np.repeat(np.arange(npix, dtype=np.int64), c)
            k = np.arange(total, dtype=np.int64) - offsets[pix]
            s0 = (spp + k * CHUNK).astype(np.int32)
            sums = chunk_sums(pix, s0, CHUNK)
            flat = acc.reshape(-1, 4)
            for kk in range(int(c.max())):       # chunk order, one float add per chunk
                sel = k == kk
                flat[pix[sel]] += sums[sel]
            nsamp += chunks * np.uint32(CHUNK)
    img = resolve(acc, nsamp, visible)
    return img, nsamp, chunks


def resolve(acc, nsamp, visible=False):
    """k_resolve: the per-pixel mean; visible frames go from XYZ to linear sRGB x 683."""
    inv = (F32(1) / nsamp.astype(F32))[..., None]
    a = (acc.astype(F32) * inv).astype(F32)
    if not visible:
        return a
    X, Y, Z = a[..., 0], a[..., 1], a[..., 2]
    r = F32(3.2404542) * X - F32(1.5371385) * Y - F32(0.4985314) * Z
    g = F32(-0.9692660) * X + F32(1.8760108) * Y + F32(0.0415560) * Z
    b = F32(0.0556434) * X - F32(0.2040259) * Y + F32(1.0572252) * Z
    return np.stack([F32(683) * r, F32(683) * g, F32(683) * b, F32(683) * a[..., 3]], axis=-1).astype(F32)
