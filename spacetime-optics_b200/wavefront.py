"""Photon-ring zoom batches for the persistent wavefront (so_batch_*).

The batch of the photon-ring benchmark: 4 spins x 2 inclinations x 8 turbulence time offsets of the
synchrotron torus plasma, each a W x W window centred on the critical curve (the zoom target of the
reference's photon-ring shot, blackholes/shots/02_photon_ring_zoom.ini: image angle -100 deg, found by
bisection on the vacuum fate, shot.cpp:148-164) at a magnification between 1e3 and 4e4, log-spaced over
the time offsets.  Integration as in that shot: tolerance 1e-11, up to 60000 steps.
"""
import numpy as np

SPINS = (0.0, 0.5, 0.9, 0.99)
INCLINATIONS = (17.0, 60.0)
TIMES = tuple(50.0 * k for k in range(8))
ZOOMS = tuple(1e3 * 40.0 ** (k / 7.0) for k in range(8))
N0 = 1594262.8  # the synchrotron frame's 0.6 Jy normalisation


def photon_ring_shots(so, W=512, spins=SPINS, inclinations=INCLINATIONS, times=TIMES, zooms=ZOOMS,
                      tolerance=1e-11, max_steps=60000):
    """One Shot per (spin, inclination); its frames are the time offsets / zooms."""
    n = len(times)
    zt = ", ".join(f"{i}:{z:.6f}" for i, z in enumerate(zooms[:n]))
    tt = ", ".join(f"{i}:{t:.6f}" for i, t in enumerate(times))
    shots = []
    for a in spins:
        for inc in inclinations:
            ov = [f"bh.spin={a}", f"camera.incl={inc}", f"camera.width={W}", f"camera.height={W}",
                  f"render.tolerance={tolerance}", f"render.max_steps={max_steps}", f"flow.n0={N0}",
                  "camera.target_psi_deg=-100", "camera.target=1", "shot.fps=1", f"shot.frames={n}",
                  f"track.camera.zoom={zt}", f"track.time.t_m={tt}"]
            shots.append(so.Shot("synchrotron_1024.ini", ov))
    return shots


def photon_ring_batch(so, renderer, W=512, **kw):
    """(Batch, shots, scenes, frames, frame_scene) for the renderer (which must carry the torus plasma)."""
    shots = photon_ring_shots(so, W, **kw)
    scenes, frames, frame_scene = [], [], []
    for si, sh in enumerate(shots):
        scenes.append(sh.scene)
        for i in range(sh.nframes()):
            f = sh.frame(i)
            frames.append(f)
            frame_scene.append(si)
    b = so.Batch(renderer, scenes, frames, frame_scene, W, W, 1)
    return b, shots, scenes, frames, frame_scene
