"""so_radio_flux_noalloc: the flux measurement for callers that cannot allocate device memory.

Such a caller (a process whose device memory belongs to a pool or arena, a real-time loop that only
allocates up front, a plugin host that forbids allocation inside its callbacks) owns every buffer it
hands in; the entry point's working memory is the library's fixed device array.  The test prepares
those buffers with torch (the caller's memory), then checks that two calls in a row through the C ABI
give the flux that the renderer's so_radio_flux gives on the same frame, that the second call leaves
the device's free memory unchanged, and that a frame larger than the fixed array is refused.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_bytes(torch, obj):
    return torch.tensor(np.frombuffer(bytes(memoryview(obj)), np.uint8).copy(), device="cuda")


def test_radio_flux_noalloc_matches_renderer(so):
    import torch
    n = 64
    sh = so.Shot("synchrotron_1024.ini", [f"camera.width={n}", f"camera.height={n}", "flow.n0=1594262.8"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    p = sh.plasma()
    modes = r.set_plasma(p)
    f = sh.frame(0, W=n)
    pix_sr = (24.0 / n * sh.info.rg_cm / sh.info.distance_cm) ** 2
    ref = r.radio_flux(f, n, pix_sr)
    assert ref > 0

    # the caller's device memory: tables, scene with device table pointers, frame, modes, result
    t = sh.tables
    d_disk = torch.tensor(np.ctypeslib.as_array(t.disk_lnT, (t.disk_n,)).copy(), device="cuda")
    d_k2 = torch.tensor(np.ctypeslib.as_array(t.k2_ln, (t.k2_n,)).copy(), device="cuda")
    d_bb = torch.tensor(np.ctypeslib.as_array(t.bb_xyz, (3 * t.bb_n,)).copy(), device="cuda")
    scene = so.abi.Scene.from_buffer_copy(bytes(memoryview(sh.scene)))
    F = C.POINTER(C.c_float)
    scene.disk_lnT = C.cast(C.c_void_p(d_disk.data_ptr()), F)
    scene.k2_lntab = C.cast(C.c_void_p(d_k2.data_ptr()), F)
    scene.bb_xyz = C.cast(C.c_void_p(d_bb.data_ptr()), F)
    frame = so.abi.Frame.from_buffer_copy(bytes(memoryview(f)))
    frame.W, frame.H, frame.spp = n, n, 2
    d_scene = _device_bytes(torch, scene)
    d_frame = _device_bytes(torch, frame)
    d_modes = torch.tensor(so.modes_to_numpy(modes, p.n_modes), device="cuda")
    d_jy = torch.zeros(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()

    lib = so.lib()
    free = []
    for call in range(2):
        d_jy.fill_(-1.0)
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        rc = lib.so_radio_flux_noalloc(C.c_void_p(d_scene.data_ptr()), C.c_void_p(d_frame.data_ptr()), n, pix_sr,
                                       C.byref(p), C.c_void_p(d_modes.data_ptr()), C.c_void_p(d_jy.data_ptr()),
                                       None)
        assert rc == so.abi.SO_OK, lib.so_last_error(None)
        torch.cuda.synchronize()
        jy = d_jy.item()
        # same kernels in the same order as so_radio_flux: agreement to the last bits
        assert abs(jy - ref) <= 1e-12 * abs(ref), (call, jy, ref)
    # the second call allocated nothing on the device
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free[1]

    rc = lib.so_radio_flux_noalloc(C.c_void_p(d_scene.data_ptr()), C.c_void_p(d_frame.data_ptr()), 257, pix_sr,
                                   C.byref(p), C.c_void_p(d_modes.data_ptr()), C.c_void_p(d_jy.data_ptr()), None)
    assert rc == so.abi.SO_ERR_SIZE
    assert b"SO_NOALLOC_MAX_PIXELS" in lib.so_last_error(None)
    r.close()
