"""Shared checks of the parity tests (CPU oracle tests and GPU kernel tests)."""
import os

import numpy as np

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def shadow_grid_vs_reference(res, g=None, base=1e-9, per_sens=1e-11):
    """Per-pixel parity of a traced 256^2 shadow self-test grid `res` (fate, ncross, theta, phi,
    n_accepted, n_attempts over all 65,536 pixel centres, grid order) with the reference's own
    trace_ray (golden/shadow_grid_256.npz).

    Termination class and winding order must be identical on every ray.  The escape direction must
    agree within base + per_sens x S relative, S being the ray's sensitivity stored in the fixture
    (relative change of the direction per relative change of the ray's image-plane position).  Two
    FP64 integrators whose roundings differ in the last bit (err^-1/5, fma placement) differ like
    two rays started ~1e-12 apart: for the ~1e5 of the rays next to the critical curve that is above
    1e-9, for nearly every ray far below.  Returns a summary dict for the report."""
    if g is None:
        g = np.load(os.path.join(GOLD, "shadow_grid_256.npz"))
    assert res["fate"].shape == (65536,)
    assert np.array_equal(res["fate"], g["fate"]), np.nonzero(res["fate"] != g["fate"])[0][:10]
    assert np.array_equal(res["ncross"], g["ncross"]), np.nonzero(res["ncross"] != g["ncross"])[0][:10]
    esc = g["fate"] == 1
    sens = g["dir_sensitivity"].astype(np.float64)
    out = {"rays": 65536, "escaped": int(esc.sum()), "captured": int((g["fate"] == -1).sum())}
    beyond = np.zeros(int(esc.sum()), bool)
    for k in ("theta", "phi"):
        ref = g[f"{k}_esc"]
        rel = np.abs(res[k][esc] - ref) / np.abs(ref)
        bar = base + per_sens * sens
        assert (rel <= bar).all(), (k, np.nonzero(rel > bar)[0][:10], rel[rel > bar][:10], sens[rel > bar][:10])
        beyond |= rel > base
        out[f"{k}_rel_max"] = float(rel.max())
        out[f"{k}_rel_p999"] = float(np.percentile(rel, 99.9))
    # the rays beyond 1e-9 are few, and every one of them is ill-conditioned
    out["dir_beyond_base"] = int(beyond.sum())
    out["sens_min_beyond"] = float(sens[beyond].min()) if beyond.any() else None
    assert beyond.sum() <= 0.001 * esc.sum()
    assert (sens[beyond] >= 100).all()
    for k in ("n_accepted", "n_attempts"):
        out[f"{k}_equal"] = float((res[k] == g[k]).mean())
    return out
