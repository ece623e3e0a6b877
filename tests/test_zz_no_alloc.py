"""so_radio_flux_noalloc: the flux measurement for callers that cannot allocate device memory.

Such a caller (a process whose device memory belongs to a pool or arena, a real-time loop that only
allocates up front, a plugin host that forbids allocation inside its callbacks) owns every buffer it
hands in; the entry point's working memory is the library's fixed device array.  The tests prepare
those buffers with torch (the caller's memory), then check through the C ABI that two calls in a row
give the flux that the renderer's so_radio_flux gives on the same frame, that the second call leaves
the device's free memory unchanged, and that a frame larger than the fixed array is refused.  On the
turbulent reference flow the entry point evaluates the noise in place: it must equal so_radio_flux
with SO_FLOW_NOISE_INLINE, and it is another draw than the renderer's default baked slices.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_bytes(torch, obj):
    return torch.tensor(np.frombuffer(bytes(memoryview(obj)), np.uint8).copy(), device="cuda")


class _CallerBuffers:
    """The scene (with device table pointers), the frame, the modes and the result in device memory
    that the caller owns."""

    def __init__(self, so, sh, f, n, modes, n_modes):
        import torch
        t = sh.tables
        self.keep = [torch.tensor(np.ctypeslib.as_array(t.disk_lnT, (t.disk_n,)).copy(), device="cuda"),
                     torch.tensor(np.ctypeslib.as_array(t.k2_ln, (t.k2_n,)).copy(), device="cuda"),
                     torch.tensor(np.ctypeslib.as_array(t.bb_xyz, (3 * t.bb_n,)).copy(), device="cuda")]
        scene = so.abi.Scene.from_buffer_copy(bytes(memoryview(sh.scene)))
        F = C.POINTER(C.c_float)
        scene.disk_lnT = C.cast(C.c_void_p(self.keep[0].data_ptr()), F)
        scene.k2_lntab = C.cast(C.c_void_p(self.keep[1].data_ptr()), F)
        scene.bb_xyz = C.cast(C.c_void_p(self.keep[2].data_ptr()), F)
        frame = so.abi.Frame.from_buffer_copy(bytes(memoryview(f)))
        frame.W, frame.H, frame.spp = n, n, 2
        self.scene = _device_bytes(torch, scene)
        self.frame = _device_bytes(torch, frame)
        self.modes = (torch.tensor(so.modes_to_numpy(modes, n_modes), device="cuda") if modes is not None
                      else torch.zeros(5, dtype=torch.float64, device="cuda"))
        self.jy = torch.zeros(1, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()

    def call(self, so, n, pix_sr, plasma):
        lib = so.lib()
        return lib.so_radio_flux_noalloc(C.c_void_p(self.scene.data_ptr()), C.c_void_p(self.frame.data_ptr()), n,
                                         pix_sr, C.byref(plasma) if plasma is not None else None,
                                         C.c_void_p(self.modes.data_ptr()), C.c_void_p(self.jy.data_ptr()), None)


def _two_calls(so, buf, n, pix_sr, plasma, ref):
    """Two calls in a row, each equal to ref; returns the free device memory before each call."""
    import torch
    lib = so.lib()
    free = []
    for call in range(2):
        buf.jy.fill_(-1.0)
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        rc = buf.call(so, n, pix_sr, plasma)
        assert rc == so.abi.SO_OK, lib.so_last_error(None)
        torch.cuda.synchronize()
        jy = buf.jy.item()
        # same kernels in the same order as so_radio_flux: agreement to the last bits
        assert abs(jy - ref) <= 1e-12 * abs(ref), (call, jy, ref)
    return free


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

    buf = _CallerBuffers(so, sh, f, n, modes, p.n_modes)
    free = _two_calls(so, buf, n, pix_sr, p, ref)
    # the second call allocated nothing on the device
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free[1]

    lib = so.lib()
    rc = buf.call(so, 257, pix_sr, p)
    assert rc == so.abi.SO_ERR_SIZE
    assert b"SO_NOALLOC_MAX_PIXELS" in lib.so_last_error(None)
    r.close()


def test_radio_flux_noalloc_reference_flow(so):
    """The reference flow model (plasma NULL): without turbulence the renderer's flux; with turbulence
    the renderer's flux under SO_FLOW_NOISE_INLINE, and not the default baked slices' flux."""
    import torch
    n = 48
    pix_sr = 1e-20
    for turb in ("0", "0.8"):
        sh = so.Shot("m87_reference_flow.ini", [f"camera.width={n}", f"camera.height={n}", f"flow.turbulence={turb}"])
        f = sh.frame(0, W=n)
        r = so.Renderer(sh.scene, sh.tables, sh.settings)
        baked = r.radio_flux(f, n, pix_sr)
        r.set_flow_noise(so.abi.SO_FLOW_NOISE_INLINE)
        inline = r.radio_flux(f, n, pix_sr)
        assert inline > 0
        buf = _CallerBuffers(so, sh, f, n, None, 0)
        free = _two_calls(so, buf, n, pix_sr, None, inline)
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free[1]
        if turb == "0":
            assert abs(baked - inline) <= 1e-12 * inline  # no turbulence: the same frame either way
        else:
            # the baked slices are a different draw of the turbulence (documented in the header)
            assert abs(baked - inline) > 1e-3 * inline, (baked, inline)
        r.close()
