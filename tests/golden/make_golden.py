"""Generates the golden fixtures of tests/golden from the REFERENCE's own code.

The reference (orrnithogalum/spacetime-optics, bhrt) has no test vectors of its own: its only check
is `bhrt --selftest` (blackholes/src/main.cpp:323-372), which prints shadow-edge extents and a
radial-constraint drift.  The fixtures here are therefore produced by running the reference's code
itself, compiled for the host from its sources by oracle/Makefile into oracle/_ref/libbhref.so:
trace.cuh's trace_ray (via oracle/ref_shim.cpp), kerr.hpp's integrator, scene_build.cpp,
shot.cpp and config.cpp.

Run from the repository root (needs the reference tree to build oracle/_ref):
    make -f oracle/Makefile && python tests/golden/make_golden.py
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import conftest  # noqa: E402

so = conftest.load_package()
import _oracle as O  # noqa: E402

SHOTS = os.path.join(ROOT, "spacetime-optics_b200", "shots")


def scene_bytes(s):
    return np.frombuffer(bytes(memoryview(s)), np.uint8).copy()


def main():
    lib = O.ref()
    out = {}
    # 1. Struct layout of SceneGPU / FrameGPU
    buf = (C.c_longlong * 64)()
    n = lib.ref_layout(buf, 64)
    np.save(os.path.join(HERE, "layout.npy"), np.array(buf[:n], np.int64))

    # 2. Shadow self-test scene: rays on a strided subset of the 256^2 pixel-centre grid
    R = O.RefShot(os.path.join(SHOTS, "shadow_selftest_256.ini"))
    f = R.frame(0)
    X, Y = so.pixel_centres(f, 256, 256)
    idx = np.arange(0, 256 * 256, 29)
    v = O.ref_vacuum(R.scene, f, X[idx], Y[idx])
    np.savez_compressed(os.path.join(HERE, "shadow_rays.npz"), idx=idx, x=X[idx], y=Y[idx], **v)

    # 3. Host builders: scene / frame structs and tables for every shipped shot
    for name in ("shadow_selftest_256", "synchrotron_1024", "m87_reference_flow", "thin_disk_4096"):
        Rs = O.RefShot(os.path.join(SHOTS, name + ".ini"))
        fr = Rs.frame(0)
        np.savez_compressed(os.path.join(HERE, f"build_{name}.npz"), scene=scene_bytes(Rs.scene),
                            frame=scene_bytes(fr), disk=Rs.disk, k2=Rs.k2, bb=Rs.bb,
                            info=np.array(Rs.info), settings=np.array(Rs.settings[:4], np.int64),
                            target_err=np.float32(Rs.settings[4]))

    # 4. Hot flow, the reference's model without turbulence (its fBm time phase is ill-conditioned:
    #    the noise generation and advection use the raw coordinate time t ~ -r_cam, so 1e-10 of
    #    position moves the noise by ~1e-4), 32 x 32 pixel centres, and pass 1 with R2 jitter at
    #    spp = 2
    Rf = O.RefShot(os.path.join(SHOTS, "m87_reference_flow.ini"), ["flow.turbulence=0", "camera.width=32",
                                                                    "camera.height=32"])
    ff = Rf.frame(0)
    Xf, Yf = so.pixel_centres(ff, 32, 32)
    t = O.ref_trace(Rf.scene, ff, Xf, Yf)
    acc, lim = O.ref_pass1(Rf.scene, ff)
    np.savez_compressed(os.path.join(HERE, "flow_rays.npz"), x=Xf, y=Yf, fate=t["fate"], I=t["I"], pass1=acc,
                        step_limited=np.int64(lim))

    # 5. Thin disk (visible mode, XYZ), 40 x 40 pixel centres
    Rd = O.RefShot(os.path.join(SHOTS, "thin_disk_4096.ini"), ["camera.width=40", "camera.height=40"])
    fd = Rd.frame(0)
    Xd, Yd = so.pixel_centres(fd, 40, 40)
    t = O.ref_trace(Rd.scene, fd, Xd, Yd)
    np.savez_compressed(os.path.join(HERE, "disk_rays.npz"), x=Xd, y=Yd, fate=t["fate"], I=t["I"])

    # 6. The reference self-test (main.cpp:323-371): shadow edges vs the analytic Bardeen curve
    rows = []
    for a in (0.5, 0.94, 0.99):
        for incl in (90.0, 17.0):
            th = incl * np.pi / 180
            rp0 = 2.0 * (1.0 + np.cos(2.0 / 3.0 * np.arccos(-a)))
            rp1 = 2.0 * (1.0 + np.cos(2.0 / 3.0 * np.arccos(a)))
            amin, amax = 1e9, -1e9
            al, be = C.c_double(), C.c_double()
            for i in range(0, 200001):
                rp = rp0 + (rp1 - rp0) * i / 200000.0
                if lib.ref_critical_curve_point(a, th, rp, C.byref(al), C.byref(be)):
                    amin = min(amin, al.value)
                    amax = max(amax, al.value)
            xp = lib.ref_find_critical_point_cam(a, 1e7, th, 0.0)
            xm = lib.ref_find_critical_point_cam(a, 1e7, th, np.pi)
            rows.append((a, incl, -xm, xp, amin, amax))
    steps = C.c_int()
    drift = lib.ref_radial_drift(C.byref(steps))
    # critical_curve_point samples
    ccp = []
    for a in (0.3, 0.94):
        for incl in (17.0, 60.0, 163.0):
            for rp in np.linspace(1.9, 3.9, 9):
                ok = lib.ref_critical_curve_point(a, incl * np.pi / 180, rp, C.byref(al), C.byref(be))
                ccp.append((a, incl, rp, ok, al.value if ok else 0.0, be.value if ok else 0.0))
    kp = []
    for a, r, th in ((0.94, 1000.0, 0.3), (0.5, 1e7, 2.8), (0.99, 6.0, 1.2)):
        k = O.KerrPoint()
        lib.ref_kerr_point(a, r, th, C.byref(k))
        kp.append([a, r, th] + [getattr(k, n) for n, _ in O.KerrPoint._fields_])
    np.savez_compressed(os.path.join(HERE, "selftest.npz"), edges=np.array(rows), drift=np.float64(drift),
                        drift_steps=np.int64(steps.value), ccp=np.array(ccp), kerr_point=np.array(kp))
    noise_fixture()
    print("golden fixtures written to", HERE)


def noise_fixture():
    """7. The reference's noise, function by function (whole rays through turbulence are
    ill-conditioned in the noise phase): fbm3 at random float points for three seeds, and
    sheared_noise with the reference flow's and the thin disk's turbulence parameters at random
    (R, phi, z) and times up to 1e5 M and up to 1e7 M (the camera's coordinate time)."""
    rng = np.random.default_rng(20261203)
    n = 2048
    x, y, z = (rng.uniform(-40, 40, n).astype(np.float32) for _ in range(3))
    seeds = np.array([1, 0x51f15eed ^ 7, 123456789], np.uint32)
    fbm = np.stack([O.noise("ref", "fbm3", x, y, z, int(sd)) for sd in seeds])
    out = dict(fx=x, fy=y, fz=z, fseeds=seeds, fbm3=fbm)
    for tag, shot, disk in (("flow", "m87_reference_flow", False), ("disk", "thin_disk_4096", True)):
        S = O.RefShot(os.path.join(SHOTS, shot + ".ini")).scene
        scale, tcorr = (S.disk_turb_scale, S.disk_tcorr) if disk else (S.flow_turb_scale, S.flow_tcorr)
        seed = S.seed if disk else S.seed ^ 0x51f15eed
        R = rng.uniform(1.5, 60, n)
        phi = rng.uniform(0, 2 * np.pi, n)
        zz = np.zeros(n) if disk else rng.uniform(-0.4, 0.4, n) * R
        t = np.concatenate([rng.uniform(-1e5, 1e5, n // 2), rng.uniform(-1e7, 1e7, n - n // 2)])
        out.update({f"{tag}_scene": scene_bytes(S), f"{tag}_R": R, f"{tag}_phi": phi, f"{tag}_z": zz, f"{tag}_t": t,
                    f"{tag}_param": np.array([scale, tcorr], np.float32), f"{tag}_seed": np.uint32(seed),
                    f"{tag}_noise": O.noise("ref", "sheared", R, phi, zz, seed, scene=S, scale=scale, tcorr=tcorr,
                                             t=t)})
    np.savez_compressed(os.path.join(HERE, "noise.npz"), **out)


# Vacuum scenes beyond the shadow self-test: spins and inclinations that reach the builder's spin
# clamp (build_scene keeps a in [1e-6, 0.9999]), the near-extremal horizon, an edge-on camera, a
# camera 0.5 deg off the pole, one below the plane, and a camera ON the pole (sin(theta) = 0: every
# ray's phi derivative is infinite, the error estimate NaN, so each ray only shrinks its step until
# max_steps and ends step-limited -- the reference's behaviour, reproduced, not fixed).
SWEEP = ((0.0, 60.0), (-0.7, 75.0), (0.5, 90.0), (0.998, 45.0), (0.94, 0.5), (0.3, 163.0), (1.0, 30.0),
         (0.94, 0.0))


def sweep_fixture():
    """8. Spin / inclination sweep on the shadow self-test shot: 256 rays (every 257th pixel centre
    of the 256^2 grid) per scene, 16 for the pole camera, traced by the reference's trace_ray."""
    out = dict(cases=np.array(SWEEP))
    for c, (spin, incl) in enumerate(SWEEP):
        ov = [f"bh.spin={spin}", f"camera.incl={incl}"]
        R = O.RefShot(os.path.join(SHOTS, "shadow_selftest_256.ini"), ov)
        f = R.frame(0)
        X, Y = so.pixel_centres(f, 256, 256)
        idx = np.arange(0, 256 * 256, 257 if incl > 0 else 4099)
        v = O.ref_vacuum(R.scene, f, X[idx], Y[idx])
        out.update({f"c{c}_x": X[idx], f"c{c}_y": Y[idx], f"c{c}_a": np.float64(R.scene.a),
                    f"c{c}_scene": scene_bytes(R.scene), f"c{c}_frame": scene_bytes(f)})
        out.update({f"c{c}_{k}": val for k, val in v.items()})
    np.savez_compressed(os.path.join(HERE, "sweep_rays.npz"), **out)


# Emission at other spins and inclinations: the thin disk (its Novikov-Thorne table follows the
# spin's ISCO) and the reference hot flow without turbulence (the noise phase is ill-conditioned).
EMISSION = (("thin_disk_4096", 0.5, 30.0), ("thin_disk_4096", 0.998, 85.0),
            ("m87_reference_flow", 0.3, 40.0), ("m87_reference_flow", 1.0, 100.0))


def emission_fixture():
    """9. 24 x 24 pixel centres per case, traced by the reference's trace_ray with its own scene
    and tables for that spin (stored with the rays)."""
    out = dict(cases=np.array([(0 if sh.startswith("thin") else 1, a, i) for sh, a, i in EMISSION]))
    k2 = bb = None
    for c, (shot, spin, incl) in enumerate(EMISSION):
        ov = [f"bh.spin={spin}", f"camera.incl={incl}", "camera.width=24", "camera.height=24"]
        if shot.startswith("m87"):
            ov.append("flow.turbulence=0")
        R = O.RefShot(os.path.join(SHOTS, shot + ".ini"), ov)
        f = R.frame(0)
        X, Y = so.pixel_centres(f, 24, 24)
        t = O.ref_trace(R.scene, f, X, Y)
        out.update({f"c{c}_x": X, f"c{c}_y": Y, f"c{c}_fate": t["fate"], f"c{c}_I": t["I"],
                    f"c{c}_scene": scene_bytes(R.scene), f"c{c}_frame": scene_bytes(f), f"c{c}_disk": R.disk})
        # the K2 and blackbody tables do not depend on the spin: stored once
        assert k2 is None or (np.array_equal(k2, R.k2) and np.array_equal(bb, R.bb))
        k2, bb = R.k2, R.bb
    np.savez_compressed(os.path.join(HERE, "emission_rays.npz"), k2=k2, bb=bb, **out)


def chunks_fixture():
    """10. Pass-2 chunk sums (k_pass2, render.cu:196-224) through the reference's own sample_pixel
    jitter and trace_ray: the reference hot flow (turbulence off) at 48 x 32, spp 2; the first
    chunk (samples 2 .. 9) of every pixel and the fourth chunk (samples 26 .. 33) of every 7th."""
    ov = ["camera.width=48", "camera.height=32", "render.spp=2", "render.spp_max=34", "flow.turbulence=0"]
    R = O.RefShot(os.path.join(SHOTS, "m87_reference_flow.ini"), ov)
    f = R.frame(0)
    n = 48 * 32
    pix = np.concatenate([np.arange(n), np.arange(0, n, 7)]).astype(np.int64)
    s0 = np.concatenate([np.full(n, 2), np.full(len(range(0, n, 7)), 2 + 3 * 8)]).astype(np.int32)
    sums = O.ref_chunks(R.scene, f, pix, s0, 8)
    np.savez_compressed(os.path.join(HERE, "chunk_rays.npz"), scene=scene_bytes(R.scene), frame=scene_bytes(f),
                        pix=pix, s0=s0, count=np.int32(8), sums=sums)


def turb_fixture():
    """12. Baked flow turbulence texels (k_bake_turb, render.cu:448-461) from the reference's own
    kernel run on the host: the reference hot flow's scene with the bake set-up of render.cu:614-619,
    three (time slice, height layer) pairs, every 4th texel in ln R and in phi."""
    R = O.RefShot(os.path.join(SHOTS, "m87_reference_flow.ini"), [])
    f = R.frame(0)
    sc = O.baked(R.scene)
    kl = np.array([[0, 24], [23, 3], [11, 47]], np.int32)
    tex = np.stack([O.ref_bake_layer(sc, f, int(k), int(l))[::4, ::4] for k, l in kl])
    np.savez_compressed(os.path.join(HERE, "turb_bake.npz"), scene=scene_bytes(sc), frame=scene_bytes(f), kl=kl,
                        texels=tex)


def shadow_grid_fixture():
    """14. The whole 256^2 pixel-centre grid of the shadow self-test shot (a = 0.94, i = 17 deg,
    r_obs = 1000 M, tolerance 1e-10): all 65,536 rays traced by the reference's trace_ray.  Escape
    directions are stored for the escaping rays only (in grid order), the integers for every ray.
    Near the critical curve a ray's escape direction amplifies any difference in its step sequence
    by orders of magnitude.  Each escaping ray therefore also carries its sensitivity S (float32): the
    relative change of the reference's escape direction per relative change of the ray's image-plane
    position, by a finite difference of 1e-12 in x and in y (the largest over x, y and theta, phi)."""
    R = O.RefShot(os.path.join(SHOTS, "shadow_selftest_256.ini"))
    f = R.frame(0)
    X, Y = so.pixel_centres(f, 256, 256)
    v = O.ref_vacuum(R.scene, f, X, Y)
    esc = v["fate"] == 1
    eps = 1e-12
    sens = np.zeros(int(esc.sum()))
    for sx, sy in ((1, 0), (0, 1)):
        p = O.ref_vacuum(R.scene, f, X[esc] * (1 + sx * eps), Y[esc] * (1 + sy * eps))
        for k in ("theta", "phi"):
            d = np.abs(p[k] - v[k][esc]) / np.abs(v[k][esc]) / eps
            d[p["fate"] != 1] = np.inf
            sens = np.maximum(sens, d)
    np.savez_compressed(os.path.join(HERE, "shadow_grid_256.npz"), fate=v["fate"], ncross=v["ncross"],
                        theta_esc=v["theta"][esc], phi_esc=v["phi"][esc], n_accepted=v["n_accepted"],
                        n_attempts=v["n_attempts"], dir_sensitivity=sens.astype(np.float32))


# An animated shot exercising every camera track the builders support: log-space tracks (r, zoom),
# linear tracks (inclination, roll, yaw, pitch, zoom target, time), an orbiting camera with a boost,
# offsets and the critical-curve zoom target at 40 deg, in visible mode at spin 0.7.
ANIM_INI = """[shot]
name = anim
duration = 2
fps = 3
[bh]
spin = 0.7
[render]
mode = visible
[camera]
r = 500
incl = 35
phi = 10
roll = 20
yaw = 1.5
pitch = -2
fov_m = 24
width = 64
height = 48
motion = orbit
target = 1
offset_x_m = 0.3
offset_y_m = -0.2
target_psi_deg = 40
[track]
camera.r = 0:500, 1:80, 2:40
camera.incl = 0:35, 0.7:60, 2:85
camera.zoom = 0:1, 1:3, 2:50
camera.roll = 0:20, 2:-40
camera.yaw = 0:1.5, 1:-1, 2:0.5
camera.pitch = 0:-2, 2:2
camera.target = 0:0, 1.5:1
time.t_m = 0:0, 2:100
"""


def anim_fixture():
    """15. The animated shot ANIM_INI through the reference's build_scene / build_shot / make_frame:
    the scene, its tables and info, and every frame (6) of the shot."""
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "anim.ini")
        with open(path, "w") as fh:
            fh.write(ANIM_INI)
        R = O.RefShot(path)
        frames = np.stack([scene_bytes(R.frame(i)) for i in range(6)])
        np.savez_compressed(os.path.join(HERE, "build_anim.npz"), ini=np.array(ANIM_INI), scene=scene_bytes(R.scene),
                            frames=frames, disk=R.disk, k2=R.k2, bb=R.bb, info=np.array(R.info),
                            settings=np.array(R.settings[:4], np.int64))


def adapt_fixture():
    """13. k_adapt and k_dilate (render.cu:130-150) from the reference's own kernels run on the host,
    on seeded luminance statistics of a 48 x 32 frame at spp 2 (log-normal samples whose spread grows
    from 0 to 0.15 across the frame, so the extra counts run from 0 to the cap; a block of empty
    pixels), yref as Impl::trace forms it (render.cu:702), target 0.02, extra_max 32."""
    rng = np.random.default_rng(13)
    H, W, spp = 32, 48, 2
    yy, xx = np.mgrid[0:H, 0:W]
    mu = np.sin(xx / 7.0) + 0.5 * np.cos(yy / 5.0)
    sig = (0.15 * xx / (W - 1))[..., None]
    Y = np.exp(mu[..., None] + sig * rng.normal(0.0, 1.0, (H, W, spp))).astype(np.float32)
    Y[4:9, 30:40] = 0
    ys = np.stack([Y.sum(-1, dtype=np.float32), (Y * Y).sum(-1, dtype=np.float32)], -1).astype(np.float32)
    fsum = float(ys[..., 0].astype(np.float64).sum())
    yref = np.float32(0.03 * fsum / (float(H * W) * spp) + 1e-37)
    extra, chunks = O.ref_adapt_dilate(ys, np.full((H, W), spp, np.uint32), float(yref), 0.02, 32)
    np.savez_compressed(os.path.join(HERE, "adapt.npz"), ystat=ys, spp=np.int32(spp), fsum=np.float64(fsum),
                        target=np.float32(0.02), extra_max=np.int32(32), extra=extra, chunks=chunks)


def post_fixture():
    """11. The post filters (render.cu:244-316 through Impl::bloom :732-740 and Impl::radio_blur
    :742-753) run by the reference's own kernels, compiled for the host by oracle/ref_post_shim.cpp:
    a 41 x 29 frame of peaky random values (bloom at strengths 0.35 and 1, beams of 0.8, 4 and 7.5
    pixels: pyramid levels 0 and 1) and a 64 x 48 frame of a few bright points on a faint floor
    (beams of 13 and 30 pixels: levels 2 and 3, then k_upsample)."""
    rng = np.random.default_rng(11)
    a = (rng.random((29, 41, 4)) ** 6).astype(np.float32)
    b = np.full((48, 64, 4), 1e-3, np.float32)
    for _ in range(6):
        b[rng.integers(48), rng.integers(64)] += rng.random(4).astype(np.float32) * 50
    out = {"a": a, "b": b}
    for st in (0.35, 1.0):
        out[f"a_bloom_{st}"] = O.ref_post(a, bloom=st)
    for sg in (0.8, 4.0, 7.5):
        out[f"a_blur_{sg}"] = O.ref_post(a, sigma=sg)
    for sg in (13.0, 30.0):
        out[f"b_blur_{sg}"] = O.ref_post(b, sigma=sg)
    np.savez_compressed(os.path.join(HERE, "post_filters.npz"), **out)


if __name__ == "__main__":
    # no argument: every fixture; otherwise only the named ones (noise, sweep, emission, chunks, post, turb, adapt,
    # shadow_grid, anim)
    if len(sys.argv) == 1:
        main()
        sweep_fixture()
        emission_fixture()
        chunks_fixture()
        post_fixture()
        turb_fixture()
        adapt_fixture()
        shadow_grid_fixture()
        anim_fixture()
    for name in sys.argv[1:]:
        {"noise": noise_fixture, "sweep": sweep_fixture, "emission": emission_fixture,
         "chunks": chunks_fixture, "post": post_fixture,
         "turb": turb_fixture, "adapt": adapt_fixture, "shadow_grid": shadow_grid_fixture,
         "anim": anim_fixture}[name]()
