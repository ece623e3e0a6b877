"""Batched frames in one persistent launch (so_batch_*): every frame of the batch equals its
single-frame render bit for bit, for both job orders and any grid size, replayed as a CUDA graph;
the autotuner picks a launch shape that reproduces the same images."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _wavefront(so):
    import importlib
    return importlib.import_module("spacetime_optics_b200.wavefront")


def test_batch_matches_single_frames(so):
    import torch
    wf = _wavefront(so)
    W = 24
    shots = wf.photon_ring_shots(so, W, spins=(0.5, 0.94), inclinations=(60.0,), times=(0.0, 150.0, 300.0),
                                 zooms=(30.0, 100.0, 300.0), tolerance=1e-10, max_steps=20000)
    sh0 = shots[0]
    r = so.Renderer(sh0.scene, sh0.tables, sh0.settings)
    r.set_plasma(sh0.plasma())
    scenes, frames, fs = [], [], []
    for si, sh in enumerate(shots):
        scenes.append(sh.scene)
        for i in range(sh.nframes()):
            frames.append(sh.frame(i))
            fs.append(si)
    assert len(frames) == 6
    # single-frame references, one renderer per scene (the scene scalars differ by spin)
    ref = []
    for si, sh in enumerate(shots):
        rr = so.Renderer(sh.scene, sh.tables, sh.settings)
        rr.set_plasma(sh.plasma())
        for i in range(sh.nframes()):
            img, _, _ = rr.render(sh.frame(i))
            ref.append(img)
        rr.close()
    ref = np.stack(ref)
    assert ref[..., 0].max() > 0
    b = so.Batch(r, scenes, frames, fs, W, W, 1)
    out = torch.zeros((len(frames), W, W, 4), dtype=torch.float32, device="cuda")
    # launch shapes, job orders, interleave tiles (1024 does not divide 24 x 24: lowered to 64) and
    # queue chunks change which lane traces which ray, never a ray's result
    for inter, ctas, tile, chunk in ((0, 0, 1, 1), (0, 1, 1, 1), (1, 0, 1, 1), (1, 1, 1, 1), (1, 0, 32, 1),
                                     (1, 0, 1024, 3), (0, 2, 1, 4)):
        b.set_tune(ctas, inter, tile, chunk)
        out.zero_()
        st = b.render(out.data_ptr(), stats=True)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), ref), (inter, ctas, tile, chunk)
        assert st.samples == len(frames) * W * W and st.attempts > 0
    # graph replay without stats (asynchronous) gives the same again
    out.zero_()
    b.render(out.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref)
    t = b.autotune(out.data_ptr())
    assert t.ctas_per_sm >= 1 and t.interleave in (0, 1) and t.ms > 0 and t.tile >= 1 and t.queue_chunk >= 1
    out.zero_()
    b.render(out.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref)
    # mixed precision on a batch: FP64 geometry, FP32 turbulence sums
    r.set_precision(so.abi.SO_PREC_MIXED)
    b2 = so.Batch(r, scenes, frames, fs, W, W, 1)
    out.zero_()
    b2.render(out.data_ptr())
    torch.cuda.synchronize()
    got = out.cpu().numpy()[..., 0].astype(np.float64)
    want = ref[..., 0].astype(np.float64)
    assert np.abs(got - want).sum() / want.sum() < 1e-4
    b2.close()
    b.close()
    r.close()


def test_batch_deferred_matches_single_frames(so):
    """A batch of >= 4096 jobs on the torus plasma defers its sums and emission (recording pass over
    all frames, sums, emission, ordered transfer, in waves through the renderer's record pool,
    captured in the batch's graph).  FP64: every frame equals the single-frame render (each below
    the deferral threshold, so traced with the sums in the tracer) bit for bit, with the pool
    uncapped, capped to a few waves, and too small for a wave (the replay pass renders the batch),
    for two launch shapes.  Mixed precision (FP32 sums at the
    records): within 1e-4 relative L1 of the FP64 frames."""
    import torch
    wf = _wavefront(so)
    W = 48
    shots = wf.photon_ring_shots(so, W, spins=(0.5, 0.94), inclinations=(60.0,), times=(0.0, 150.0, 300.0),
                                 zooms=(30.0, 100.0, 300.0), tolerance=1e-10, max_steps=20000)
    sh0 = shots[0]
    scenes, frames, fs, ref = [], [], [], []
    for si, sh in enumerate(shots):
        scenes.append(sh.scene)
        rr = so.Renderer(sh.scene, sh.tables, sh.settings)
        rr.set_plasma(sh.plasma())
        for i in range(sh.nframes()):
            frames.append(sh.frame(i))
            fs.append(si)
            img, _, _ = rr.render(sh.frame(i))
            ref.append(img)
        rr.close()
    ref = np.stack(ref)
    assert len(frames) * W * W >= 4096 and ref[..., 0].max() > 0
    r = so.Renderer(sh0.scene, sh0.tables, sh0.settings)
    r.set_plasma(sh0.plasma())
    out = torch.zeros((len(frames), W, W, 4), dtype=torch.float32, device="cuda")
    for pool_mb in (0.0, 64.0, 4.0):  # one wave; a few waves; a pool too small for a wave (replay)
        r.set_precision(so.abi.SO_PREC_FP64, pool_mb=pool_mb)
        b = so.Batch(r, scenes, frames, fs, W, W, 1)
        for inter, ctas, tile, chunk in ((0, 0, 1, 1), (1, 0, 32, 3)):
            b.set_tune(ctas, inter, tile, chunk)
            for _ in range(3):  # a run short of records is recaptured with a larger pool
                out.zero_()
                st = b.render(out.data_ptr(), stats=True)
                torch.cuda.synchronize()
            assert np.array_equal(out.cpu().numpy(), ref), (pool_mb, inter, ctas, tile, chunk)
            assert st.samples == len(frames) * W * W and st.attempts > 0
        b.close()
    r.set_precision(so.abi.SO_PREC_MIXED)
    b = so.Batch(r, scenes, frames, fs, W, W, 1)
    out.zero_()
    b.render(out.data_ptr())
    torch.cuda.synchronize()
    got = out.cpu().numpy()[..., 0].astype(np.float64)
    want = ref[..., 0].astype(np.float64)
    assert np.abs(got - want).sum() / want.sum() < 1e-4
    b.close()
    r.close()


@pytest.mark.parametrize("plasma", ["reference_flow", "torus_without_modes"])
def test_batch_deferred_emission_without_sums(so, plasma):
    """Batches with no mode sums defer their emission alone: the reference flow model (its sheared
    noise in place, as every batch evaluates it) over three spins, and the torus plasma without
    turbulence.  Every frame equals its single-frame render (below the deferral threshold, emission in
    the tracer; the reference model with SO_FLOW_NOISE_INLINE) bit for bit, with the pool uncapped and
    too small for a wave (the replay pass renders the batch); mixed precision changes nothing here
    (no FP32 sums to take)."""
    import torch
    W = 48
    if plasma == "reference_flow":
        shots = [so.Shot("m87_reference_flow.ini", [f"camera.width={W}", f"camera.height={W}", f"bh.spin={a}",
                                                    "render.spp=1", "render.spp_max=1"]) for a in (0.5, 0.94, 0.99)]
    else:
        shots = [so.Shot("synchrotron_1024.ini", [f"camera.width={W}", f"camera.height={W}", f"bh.spin={a}",
                                                  "so.modes=0", "flow.n0=1594262.8"]) for a in (0.5, 0.94, 0.99)]
    scenes, frames, fs, ref = [], [], [], []
    for si, sh in enumerate(shots):
        scenes.append(sh.scene)
        rr = so.Renderer(sh.scene, sh.tables, sh.settings)
        rr.set_plasma(sh.plasma() if plasma != "reference_flow" else None)
        if plasma == "reference_flow":
            rr.set_flow_noise(so.abi.SO_FLOW_NOISE_INLINE)
        frames.append(sh.frame(0))
        fs.append(si)
        img, _, _ = rr.render(sh.frame(0))
        ref.append(img)
        rr.close()
    ref = np.stack(ref)
    assert len(frames) * W * W >= 4096 and ref[..., 0].max() > 0
    sh0 = shots[0]
    r = so.Renderer(sh0.scene, sh0.tables, sh0.settings)
    r.set_plasma(sh0.plasma() if plasma != "reference_flow" else None)
    out = torch.zeros((len(frames), W, W, 4), dtype=torch.float32, device="cuda")
    for prec, pool_mb in ((so.abi.SO_PREC_FP64, 0.0), (so.abi.SO_PREC_FP64, 0.001), (so.abi.SO_PREC_MIXED, 0.0)):
        r.set_precision(prec, pool_mb=pool_mb)
        b = so.Batch(r, scenes, frames, fs, W, W, 1)
        for _ in range(2):
            out.zero_()
            st = b.render(out.data_ptr(), stats=True)
            torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), ref), (prec, pool_mb)
        if pool_mb == 0.0:
            assert st.emit64 == 1 and st.rec64_records > 0 and st.rec64_short == 0 and st.ms_sum64 < 0.05
        else:
            assert st.emit64 == 0 and st.rec64_short > 0
        b.close()
    r.close()


def test_batch_rejects_bad_input(so):
    import ctypes as C
    sh = so.Shot("synchrotron_1024.ini", ["camera.width=8", "camera.height=8"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    f = sh.frame(0)
    with pytest.raises(so.TracerError):
        so.Batch(r, [sh.scene], [f], [1], 8, 8, 1)  # scene index out of range
    vis = so.Shot("shadow_selftest_256.ini").scene
    with pytest.raises(so.TracerError):
        so.Batch(r, [sh.scene, vis], [f, f], [0, 1], 8, 8, 1)  # different modes
    L = so.lib()
    h = C.c_void_p()
    assert L.so_batch_create(r.h, None, 0, None, None, 0, 8, 8, 1, C.byref(h)) == so.abi.SO_ERR_ARG
    r.close()


def test_batch_after_its_renderer_is_destroyed(so):
    """A batch whose renderer is destroyed first is detached: rendering it is a state error, freeing
    it is still safe, and no CUDA error is left behind for the next caller on the thread."""
    import torch
    sh = so.Shot("synchrotron_1024.ini", ["camera.width=8", "camera.height=8"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    b = so.Batch(r, [sh.scene], [sh.frame(0)], [0], 8, 8, 1)
    out = torch.zeros((1, 8, 8, 4), dtype=torch.float32, device="cuda")
    b.render(out.data_ptr())
    torch.cuda.synchronize()
    r.close()
    with pytest.raises(so.TracerError) as e:
        b.render(out.data_ptr())
    assert e.value.code == so.abi.SO_ERR_STATE
    b.close()
    torch.zeros(4, device="cuda").add_(1.0)
    torch.cuda.synchronize()
