"""so_mlp.py -- CPU oracle of the ray surrogate.  TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only tests load it.  It restates, in numpy float64,
the surrogate network that the library trains and runs on the tensor cores (include/so_tracer.h,
"ray surrogate"): the Fourier features, the four tanh-form GELU layers, the 12-output head, the
loss (class cross-entropy plus weighted squared errors of direction, 1/r and redshift) and its
gradient in the library's flat parameter layout.  The surrogate has no reference counterpart (the
reference renders with the integrator only), so its parity is pinned two ways: the analytic gradient
here is checked against central finite differences in float64 (tests/test_oracle_mlp.py), and
the GPU gradient is checked against this oracle.

Two arithmetic modes:
  exact    float64 everywhere, weights taken from the FP32 master parameters;
  bf16     the GPU's rounding points: BF16 weights, features, activations, GELU derivatives and
           back-propagated gradients (round to nearest even), FP32-valued pre-activations,
           head-bias gradient from the unrounded dL/dO.  Products and sums are still float64 (the GPU sums BF16 products in
           FP32), so the two agree to the accumulation error plus rare one-ulp BF16 flips.
"""
import numpy as np

NFREQ, NFEAT, HID, NHID, NOUT, LDO = 64, 128, 256, 4, 12, 16
XY_SCALE, A_MID, I_MID, I_HALF = 12.0, 0.495, 90.0, 85.0
GELU_C, GELU_K = 0.7978845608028654, 0.044715


def layout():
    """[(w_offset, b_offset, n, k)] per layer and the total: weights [n x k] row-major, then bias."""
    out, off = [], 0
    for l in range(NHID + 1):
        n = HID if l < NHID else LDO
        k = NFEAT if l == 0 else HID
        w = off
        off += n * k
        out.append((w, off, n, k))
        off += n
    return out, off


def bf16(x):
    """Round to bfloat16 (nearest, ties to even) and return as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params, rounding):
    lay, _ = layout()
    p = np.asarray(params, dtype=np.float64)
    W, b = [], []
    for (w, bo, n, k) in lay:
        Wl = p[w:w + n * k].reshape(n, k)
        W.append(bf16(Wl) if rounding else Wl)
        b.append(p[bo:bo + n])
    return W, b


def scaled_inputs(rays):
    r = np.asarray(rays, dtype=np.float64)
    return np.stack([r[:, 0] / XY_SCALE, r[:, 1] / XY_SCALE, (r[:, 2] - A_MID) / A_MID, (r[:, 3] - I_MID) / I_HALF],
                    axis=1)


def features(rays, freq, rounding=False):
    z = 2.0 * np.pi * scaled_inputs(rays) @ np.asarray(freq, dtype=np.float64).T
    X = np.concatenate([np.sin(z), np.cos(z)], axis=1)
    return bf16(X) if rounding else X


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(GELU_C * (z + GELU_K * z ** 3)))


def gelu_grad(z):
    t = np.tanh(GELU_C * (z + GELU_K * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_C * (1.0 + 3.0 * GELU_K * z * z)


def forward(params, freq, rays, rounding=False):
    """Head outputs [n x 16] and the cache of the backward pass."""
    W, b = unpack(params, rounding)
    X = features(rays, freq, rounding)
    acts, zs = [X], []
    a = X
    for l in range(NHID):
        z = a @ W[l].T + b[l]
        if rounding:
            z = z.astype(np.float32).astype(np.float64)
        zs.append(z)
        a = gelu(z)
        if rounding:
            a = bf16(a)
        acts.append(a)
    O = a @ W[NHID].T + b[NHID]
    return O, (W, acts, zs)


def loss_grad_outputs(O, tgt, w_dir, w_u, w_g):
    """Per-ray loss terms (sums over the batch) and dL/dO of the mean loss."""
    t = np.asarray(tgt, dtype=np.float64)
    n = O.shape[0]
    cls = t[:, 0].astype(np.int64)
    lo = O[:, :3]
    m = lo.max(axis=1, keepdims=True)
    e = np.exp(lo - m)
    s = e.sum(axis=1, keepdims=True)
    p = e / s
    ce = (np.log(s[:, 0]) + m[:, 0] - lo[np.arange(n), cls])
    d = np.zeros((n, LDO))
    d[:, :3] = p
    d[np.arange(n), cls] -= 1.0
    esc = (cls == 0)[:, None]
    dd = O[:, 3:6] - t[:, 1:4]
    d[:, 3:6] = np.where(esc, 2.0 * w_dir * dd, 0.0)
    du = O[:, 6:9] - t[:, 4:7]
    d[:, 6:9] = 2.0 * w_u * du
    has = t[:, 7:10] >= 0.0
    dg = O[:, 9:12] - t[:, 7:10]
    d[:, 9:12] = np.where(has, 2.0 * w_g * dg, 0.0)
    ld = np.where(esc, dd * dd, 0.0).sum(axis=1)
    lu = (du * du).sum(axis=1)
    lg = np.where(has, dg * dg, 0.0).sum(axis=1)
    am = lo.argmax(axis=1)
    terms = {
        "ce": ce.sum(), "dir": ld.sum(), "u": lu.sum(), "g": lg.sum(), "correct": float((am == cls).sum()),
        "total": (ce + w_dir * ld + w_u * lu + w_g * lg).sum(),
    }
    return terms, d / n


def gradients(params, freq, rays, tgt, w_dir=1.0, w_u=10.0, w_g=1.0, rounding=False):
    """(gradient of the mean loss in the flat layout, loss terms summed over the rays)."""
    lay, total = layout()
    O, (W, acts, zs) = forward(params, freq, rays, rounding)
    terms, dO = loss_grad_outputs(O, tgt, w_dir, w_u, w_g)
    g = np.zeros(total)
    wh, bh, n, k = lay[NHID]
    g[bh:bh + n] = dO.sum(axis=0)
    dOr = bf16(dO) if rounding else dO
    g[wh:wh + n * k] = (dOr.T @ acts[NHID]).ravel()
    gd = [bf16(gelu_grad(z)) if rounding else gelu_grad(z) for z in zs]
    dz = (dOr @ W[NHID]) * gd[NHID - 1]
    if rounding:
        dz = bf16(dz)
    for l in range(NHID - 1, -1, -1):
        w, bo, n, k = lay[l]
        g[w:w + n * k] = (dz.T @ acts[l]).ravel()
        g[bo:bo + n] = dz.sum(axis=0)
        if l > 0:
            dz = (dz @ W[l]) * gd[l - 1]
            if rounding:
                dz = bf16(dz)
    return g, terms


def mean_loss(params, freq, rays, tgt, w_dir=1.0, w_u=10.0, w_g=1.0):
    O, _ = forward(params, freq, rays, False)
    terms, _ = loss_grad_outputs(O, tgt, w_dir, w_u, w_g)
    return terms["total"] / O.shape[0]
