"""Config photon_ring_batch: the 64 photon-ring zoom frames (4 spins x 2 inclinations x 8 turbulence
time offsets of the synchrotron torus, windows centred on the critical curve at magnifications
1e3 .. 4e4, tolerance 1e-11, up to 60000 steps; the reference's photon-ring shot,
blackholes/shots/02_photon_ring_zoom.ini:9-11) traced by ONE persistent batch launch, checked frame by
frame against the C oracle on a strided sample of pixels (the oracle runs the same R2-jittered sample
through its own trace_ray restatement).

* FP64 batch: every sampled pixel within 1e-6 of its frame's sampled maximum (float accumulation of
  FP64 emission; the geometry is the oracle's bit for bit).
* Mixed batch (EMIT32: FP64 geometry, FP32 turbulence sums): the sample's relative L1 and total flux
  within the mixed path's bars, 1e-3, on every frame.

The windows are 256^2 here (the bench's 512^2 windows at half the pixel density, same frames)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W = 256
STRIDE = 509  # 129 pixels of each 256^2 frame


@pytest.fixture(scope="module")
def ring(so):
    import importlib
    wf = importlib.import_module("spacetime_optics_b200.wavefront")
    shots = wf.photon_ring_shots(so, W)
    assert len(shots) == 8 and all(sh.nframes() == 8 for sh in shots)
    r = so.Renderer(shots[0].scene, shots[0].tables, shots[0].settings)
    p = shots[0].plasma()
    modes = r.set_plasma(p)
    scenes, frames, fs = [], [], []
    for si, sh in enumerate(shots):
        scenes.append(sh.scene)
        for i in range(sh.nframes()):
            frames.append(sh.frame(i))
            fs.append(si)
    yield r, p, modes, shots, scenes, frames, fs
    r.close()


def _oracle_samples(orc, shots, scenes, frames, fs, p, modes):
    pix = np.arange(0, W * W, STRIDE, dtype=np.int64)
    out = []
    for fi, f in enumerate(frames):
        f.W, f.H, f.spp = W, W, 1
        out.append(orc.orc_chunks(scenes[fs[fi]], f, pix, np.zeros(pix.size, np.int32), 1, plasma=p, modes=modes,
                                  threads=max(8, os.cpu_count() or 8)))
    return pix, np.stack(out)


def _batch(so, r, scenes, frames, fs):
    import torch
    b = so.Batch(r, scenes, frames, fs, W, W, 1)
    out = torch.zeros((len(frames), W, W, 4), dtype=torch.float32, device="cuda")
    st = b.render(out.data_ptr(), stats=True)
    torch.cuda.synchronize()
    img = out.cpu().numpy().reshape(len(frames), W * W, 4)
    b.close()
    return img, st


def test_photon_ring_batch_vs_oracle(so, orc, ring):
    r, p, modes, shots, scenes, frames, fs = ring
    pix, want = _oracle_samples(orc, shots, scenes, frames, fs, p, modes)
    assert len(frames) == 64

    r.set_precision(so.abi.SO_PREC_FP64)
    img, st = _batch(so, r, scenes, frames, fs)
    assert st.samples == 64 * W * W
    got = img[:, pix, :].astype(np.float64)
    w = want.astype(np.float64)
    worst = 0.0
    for fi in range(64):
        mx = w[fi, :, 0].max()
        assert mx > 0, fi
        d = np.abs(got[fi] - w[fi]).max() / mx
        worst = max(worst, d)
        assert d <= 1e-6, (fi, d)
    print(f"photon-ring FP64 batch vs oracle: 64 frames x {pix.size} px, max |diff| / frame max = {worst:.2e}, "
          f"{st.attempts / st.samples:.0f} attempts and {st.flow_steps / st.samples:.0f} flow steps per ray")

    r.set_precision(so.abi.SO_PREC_MIXED)
    img, st = _batch(so, r, scenes, frames, fs)
    got = img[:, pix, 0].astype(np.float64)
    l1 = np.abs(got - w[..., 0]).sum(axis=1) / w[..., 0].sum(axis=1)
    flux = np.abs(got.sum(axis=1) - w[..., 0].sum(axis=1)) / w[..., 0].sum(axis=1)
    print(f"photon-ring mixed batch vs oracle: L1 max {l1.max():.2e} mean {l1.mean():.2e}, flux max {flux.max():.2e}")
    assert l1.max() <= 1e-3 and flux.max() <= 1e-3
    r.set_precision(so.abi.SO_PREC_FP64)
