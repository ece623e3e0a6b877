"""Benchmark of the Kerr ray tracer on the 2048^2 thermal-synchrotron scene (one B200 per rank).

Workload: the synchrotron frame of spacetime-optics_b200/shots/synchrotron_1024.ini rendered at
2048 x 2048 (a = 0.94, inclination 163 deg, field of view +-12 M, 230 GHz, analytic torus plasma with
512 Fourier modes of turbulence, flux normalised to 0.6 Jy), one sample per pixel centre.
One "step" = one frame traced end to end.

  value  Mrays/s of the fastest path (mixed precision when built and selected, else plain FP64),
         device buffers only (so_render_device), CUDA events on the renderer's stream.
  e2e    the same frame through so_render with host buffers: the frame descriptor goes host->device
         and the 2048 x 2048 x 4 float image comes back device->host every step.
Multi-GPU: frames are independent, so N ranks each render their own frame (weak scaling, no
collective on the data path); the max over ranks of the device time gives the job time.

--impl reference times the reference's own CPU tracer (oracle/_ref, built from the reference
sources) on the host cores over a bounded sample of the same pixels.  The torus plasma is not part
of the reference, so that arm runs the reference's own flow model with the torus's indices.
"""
import argparse
import ctypes as C
import importlib.util
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "spacetime-optics_b200")
METRIC = "Mrays/s at ≤1e-3 image error: surrogate/mixed vs plain FP64 kernel, 1 B200"

# Algorithmic FP64 flops (FMA = 2, divide = 1, sqrt = 1; comparisons, fabs and fmin/fmax not counted),
# counted from spacetime-optics_b200/csrc/so_kerr.cuh and so_emission.cuh:
FLOPS_ATTEMPT = 469        # one DP5(4) attempt: 6 RHS (31 each) + stage sums + 5th-order sum + error norm
FLOPS_ACCEPT = 49          # controller err^-1/5 (34) + projection (11) + psi bookkeeping excluded (radio)
FLOPS_FLOW = 160           # flow_step without the turbulence sum (transcendentals counted as 20 each)
FLOPS_MODE = 8 + 22        # one Fourier mode: 3 fma (k.X + phase) + fma accumulate + cos_turns (10 fma, 1 add,
                           # 1 multiply: 16 FP64 instructions per mode in all)
# SFU operations of the FP32 tracer (k_trace32): per attempt 7 RHS x 2 reciprocals + 5 error
# divides + err^-0.2 (2); per flow step ~20 (exp, log, sincos, rsqrt, divides) + one cosine per mode
SFU_ATTEMPT = 21
SFU_FLOW = 20


def load_package():
    if "spacetime_optics_b200" in sys.modules:
        return sys.modules["spacetime_optics_b200"]
    spec = importlib.util.spec_from_file_location("spacetime_optics_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["spacetime_optics_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while the timed region runs."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9 for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup(backend="nccl"):
    """One process per GPU from the torchrun environment; a process group only when WORLD_SIZE > 1
    (NCCL on GPUs; gloo for host-only runs of this logic)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def allreduce_max(x, world):
    """Max over ranks of a per-rank time: the job's time is its slowest rank's."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_frame(sh, rank):
    """Weak scaling: rank k renders frame 0 of the shot at turbulence time offset 50 k M."""
    f = sh.frame(0)
    f.t = f.t + 50.0 * rank
    return f


def job_rate(world, units_per_rank, ms_step):
    """Whole-job throughput (units per second over all ranks) from the max-over-ranks step time."""
    return world * units_per_rank / (ms_step * 1e-3)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# reference flow workload: the shot's baked fBm turbulence at a converged emission quadrature
FLOW_SHOT = "m87_reference_flow.ini"
FLOW_OVERRIDES = ["render.spp=1", "render.spp_max=1", "render.step_fraction=0.01"]


def build_scene(so, W, flux_norm=True, shot="synchrotron_1024.ini", extra=()):
    sh = so.Shot(shot, [f"camera.width={W}", f"camera.height={W}", *extra])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    p = sh.plasma()
    r.set_plasma(p)
    scene = sh.scene
    info = {}
    if flux_norm and sh.info.radio_flux_target_jy > 0:
        # flux normalisation (main.cpp:475-508) on a 160^2 frame of width flow.normalize_fov_m
        fov = sh.num("flow.normalize_fov_m", 40.0)
        tmp = so.Shot("synchrotron_1024.ini", ["camera.width=160", "camera.height=160", f"camera.fov_m={fov}"])
        fw = tmp.frame(0, W=160, seed=1)
        pix_sr = (fov / 160 * sh.info.rg_cm / sh.info.distance_cm) ** 2
        n0, jy = r.normalize_flux(scene, fw, 160, pix_sr, sh.info.radio_flux_target_jy)
        info = {"n0": n0, "flux_jy": jy}
    return sh, r, info


def run_ours(args, so, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    W = args.size
    flow = args.workload == "flow"
    if flow:
        sh, r, norm = build_scene(so, W, shot=FLOW_SHOT, extra=FLOW_OVERRIDES)
    else:
        sh, r, norm = build_scene(so, W)
    path = args.path
    if path == "auto":
        path = "mixed"
    f = rank_frame(sh, rank)
    npix = W * W
    d_img = torch.empty((W, W, 4), dtype=torch.float32, device="cuda")
    stream = torch.cuda.ExternalStream(r.stream())

    def set_prec(p):
        r.set_precision(so.abi.SO_PREC_MIXED if p == "mixed" else so.abi.SO_PREC_FP64)

    # larger-than-L2 buffer written between steps (the frame's inputs are tiny and stay cached;
    # flushing keeps each step cold like a fresh frame)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed_frames(n):
        """n frames, each after an L2 flush, timed by CUDA events on the renderer's stream, with the
        clocks sampled meanwhile: (ms per frame, clock summary)."""
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
        barrier(world)
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            for i in range(n):
                with torch.cuda.stream(stream):
                    flush.fill_(float(i))
                    ev[i][0].record(stream)
                r.render_device(f, d_img.data_ptr())
                with torch.cuda.stream(stream):
                    ev[i][1].record(stream)
            torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in ev], clk.summary()

    # The plain FP64 path under the same protocol as the measured path: warm-up, then >= 3 flushed,
    # event-timed frames with their own clock record; its image is the reference of the image error
    set_prec("fp64")
    for _ in range(min(max(args.warmup, 3), 5)):
        r.render_device(f, d_img.data_ptr())
    ms64, clk64 = timed_frames(max(3, min(args.steps, 5)))
    ms64_frame = allreduce_max(float(np.mean(ms64)), world)
    st64 = r.render_device(f, d_img.data_ptr(), stats=True)
    img64 = d_img.cpu().numpy().copy()
    plain = plain_fp64_record(so, sh, st64, ms64, ms64_frame, clk64, npix, world, local)
    set_prec(path)
    for _ in range(args.warmup):
        r.render_device(f, d_img.data_ptr())
    torch.cuda.synchronize()
    ms, clocks = timed_frames(args.steps)
    ms_step = float(np.mean(ms))
    barrier(world)
    ms_step = allreduce_max(ms_step, world)
    value = job_rate(world, npix, ms_step) / 1e6
    # instrumented step: counters and the tracer kernel's own device time (CUDA events in the library)
    st = r.render_device(f, d_img.data_ptr(), stats=True)
    img = d_img.cpu().numpy()
    classes = None
    if path == "mixed":
        # termination class of every sample outside the critical band against FP64 geometry (the
        # same samples with the band covering the field)
        ns = npix * sh.settings.spp
        fm, band = r.last_fates(ns)
        r.set_precision(so.abi.SO_PREC_MIXED, band_m=1e6)
        r.render_device(f, d_img.data_ptr(), stats=True)
        f64, _ = r.last_fates(ns)
        set_prec("mixed")
        out = ~band
        classes = {"samples_outside_band": int(out.sum()), "class_mismatch_outside_band": int((fm[out] != f64[out]).sum()),
                   "class_mismatch_in_band": int((fm[band] != f64[band]).sum())}
    err_l1 = float(np.abs(img[..., 0] - img64[..., 0]).sum() / max(np.abs(img64[..., 0]).sum(), 1e-300))
    flux_err = float(abs(img[..., 0].astype(np.float64).sum() / img64[..., 0].astype(np.float64).sum() - 1.0))
    fp64_mrays = plain["mrays_s"]
    # roofline of the dominant kernel: the FP64 tracer (plain path, FP64 pipe) or the FP32 tracer
    # (mixed path, SFU-bound: one cosine per Fourier mode per flow step)
    fp64_peak, fp32_peak = so.probe_fma_peak(local)
    pl = sh.plasma()
    n_modes = pl.n_modes if pl is not None else 0  # reference flow model: no Fourier modes
    if path == "fp64":
        flops = (st.attempts * FLOPS_ATTEMPT + st.accepted * FLOPS_ACCEPT +
                 st.flow_steps * (FLOPS_FLOW + n_modes * FLOPS_MODE))
        roof = {"bound": "fp64", "achieved": round(flops / (st.ms_kernel * 1e-3) / 1e12, 3),
                "peak": round(fp64_peak, 3), "unit": "TFLOP/s", "kernel": "k_trace64", "kernel_ms": st.ms_kernel,
                "per_launch": flops, "peak_source": "so_probe_fma_peak (measured FP64 FMA chains on this GPU)"}
    elif st.turb_records > 0:
        # deferred turbulence: the batched mode sums dominate, one SFU cosine per Fourier mode per
        # record slot (the FP32 tracer and the ordered transfer are listed beside it)
        sfu_peak = so.probe_sfu_peak(local)
        ops = st.turb_records * n_modes
        roof = {"bound": "sfu", "achieved": round(ops / (st.ms_turb * 1e-3) / 1e9, 3), "peak": round(sfu_peak, 3),
                "unit": "Gop/s", "kernel": "k_turb_records", "kernel_ms": st.ms_turb, "per_launch": ops,
                "peak_source": "so_probe_sfu_peak (measured SFU cosine chains on this GPU)",
                "fp32_tflops_peak": round(fp32_peak, 3), "tracer_k_trace32_ms": round(st.ms_fp32_trace, 3),
                "transfer_k_flow_records_ms": round(st.ms_fp32 - st.ms_fp32_trace - st.ms_turb, 3),
                "record_slots": st.turb_records}
        # DRAM bytes per record slot of k_turb_records from its ncu capture on the 512^2 frame
        # (profiles/k_turb_records_synchrotron512.md: 1.347 GB for 68.16 M slots), scaled by this
        # frame's slots; the algorithmic figure is 20 bytes per slot
        roof["traffic"] = round(19.77 * st.turb_records)
        roof["traffic_source"] = "ncu dram bytes per slot at 512^2 x this frame's record slots"
        roof["algorithmic_bytes"] = 20 * st.turb_records
    else:
        sfu_peak = so.probe_sfu_peak(local)
        ops = st.attempts_fp32 * SFU_ATTEMPT + st.flow_steps_fp32 * (SFU_FLOW + n_modes)
        roof = {"bound": "sfu", "achieved": round(ops / (st.ms_fp32 * 1e-3) / 1e9, 3), "peak": round(sfu_peak, 3),
                "unit": "Gop/s", "kernel": "k_trace32", "kernel_ms": st.ms_fp32, "per_launch": ops,
                "peak_source": "so_probe_sfu_peak (measured SFU cosine chains on this GPU)",
                "fp32_tflops_peak": round(fp32_peak, 3)}
        if st.record_waves > 0:  # deferred emission without mode sums (reference flow): tracer + transfer
            roof["kernels"] = "k_trace32 + k_flow_records"
            roof["tracer_k_trace32_ms"] = round(st.ms_fp32_trace, 3)
            roof["transfer_k_flow_records_ms"] = round(st.ms_fp32 - st.ms_fp32_trace - st.ms_turb, 3)
    roof["frac"] = round(roof["achieved"] / roof["peak"], 4)
    roof.setdefault("traffic", None)
    # e2e: host buffers through so_render (frame H2D, image D2H inside the timed region)
    host = np.empty((W, W, 4), np.float32)
    host_pinned = torch.empty((W, W, 4), dtype=torch.float32).pin_memory().numpy()
    for _ in range(2):
        r.render(f, out=host_pinned)
    torch.cuda.synchronize()
    e2e_ms = []
    for i in range(args.steps):
        t0 = time.perf_counter()
        r.render(f, out=host_pinned)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_step = allreduce_max(float(np.mean(e2e_ms)), world)
    e2e = world * npix / (e2e_step * 1e-3) / 1e6
    del host
    # per frame: tracer + resolve (plain); route, approach, band tracer, FP32 tracer, [turbulence sums,
    # transfer,] re-trace, gather, resolve (mixed); spp_max = spp, so no adaptive pass
    # (plain FP64 with deferred passes, per wave: recording pass, [torus sums,] emission, ordered
    # transfer, the replay launch that returns at once; then resolve)
    torus_sums = 0 if flow else 1
    plain_launches = (st.rec64_waves * (2 + torus_sums + (2 if st.emit64 else 0)) + 1) if st.rec64_slots else 2
    # mixed: route, approach, band tracer, FP32 tracer, re-trace, gather, resolve, and per wave of
    # the deferred form an FP32 tracer launch beyond the first, the mode sums (torus) and the transfer
    waves = max(st.record_waves, 1)
    mixed_launches = 7 + (waves - 1) + (waves * ((1 if st.turb_records > 0 else 0) + 1) if st.record_waves > 0 else 0)
    gpu_launches = args.steps * ((plain_launches if path == "fp64" else mixed_launches) + (1 if flow else 0))
    if flow:
        workload = (f"reference flow {W}x{W} (n ~ r^-1.1, fBm turbulence baked per frame into 24 slices of "
                    f"512x192x48), a=0.94, i=163 deg, fov 30 M, 230 GHz, step fraction 0.01, 1 R2-jittered "
                    f"sample/pixel (k_pass1 sampling)")
    else:
        workload = (f"synchrotron torus frame {W}x{W}, a=0.94, i=163 deg, fov +-12 M, 230 GHz, "
                    f"512 Fourier modes, 1 R2-jittered sample/pixel (k_pass1 sampling)")
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if path == "fp64" else "f32+f64", "data": "synthetic",
        "config": {"workload": workload, "path": path,
                   "band_rays": st.band_rays if path == "mixed" else None,
                   "fp64_rays": st.fp64_rays if path == "mixed" else None,
                   "plain_fp64_mrays_s": round(fp64_mrays, 4), "speedup_vs_plain_fp64": round(value / fp64_mrays, 3),
                   "plain_fp64": plain, "image_rel_l1_vs_fp64": err_l1,
                   "total_flux_err_vs_fp64": flux_err, "frames_per_s": round(1e3 / ms_step * world, 4),
                   "l2": "256 MiB buffer written between timed steps", **norm,
                   "attempts_per_ray": st.attempts / npix, "flow_steps_per_ray": st.flow_steps / npix,
                   "termination_class": classes},
        "roofline": roof,
        "e2e": {"value": round(e2e, 4), "unit": "Mrays/s", "h2d_bytes_per_step": C.sizeof(so.abi.Frame),
                "d2h_bytes_per_step": W * W * 16},
        "gpu_launches": gpu_launches,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not flow:
        line["cpu_baseline"] = cpu_baseline(so, sh, f, W, budget_s=args.cpu_seconds)
    r.close()
    if not flow and not args.no_same_scene:
        line["config"]["same_scene"] = same_scene_record(args, so, world, rank, local)
    return line


def plain_fp64_record(so, sh, st, ms, ms_frame, clocks, npix, world, local):
    """The plain FP64 path's frames: rate, phase times and rooflines against the measured FP64 FMA
    peak.  With the deferred torus turbulence the frame is recording pass + k_turb64_records +
    k_emit64_records + k_transfer64 (or a replay pass instead of the last two); the sums kernel is
    the dominant one, its algorithmic FLOPs are the recorded positions x modes x FLOPS_MODE.  The
    reference flow model's frames defer their emission only (recording pass + k_emit64_records +
    k_transfer64); their roofline is the whole frame's."""
    fp64_peak, _ = so.probe_fma_peak(local)
    pl = sh.plasma()
    n_modes = pl.n_modes if pl is not None else 0
    flops = (st.attempts * FLOPS_ATTEMPT + st.accepted * FLOPS_ACCEPT + st.flow_steps * (FLOPS_FLOW + n_modes * FLOPS_MODE))
    kernels = "k_trace64"
    if st.rec64_slots:
        sums = " + k_turb64_records" if n_modes else ""
        kernels = (f"k_trace64 (recording pass){sums} + k_emit64_records + k_transfer64" if st.emit64
                   else f"k_trace64 (recording + replay passes){sums}")
    whole = {"kernels": kernels,
             "ms": round(st.ms_kernel, 3), "achieved": round(flops / (st.ms_kernel * 1e-3) / 1e12, 3),
             "unit": "TFLOP/s", "per_launch": flops}
    rec = {"bound": "fp64", "kernel": "k_trace64", "achieved": whole["achieved"], "peak": round(fp64_peak, 3),
           "unit": "TFLOP/s", "kernel_ms": round(st.ms_kernel, 3), "per_launch": flops}
    if st.rec64_slots and n_modes:
        sflops = st.rec64_records * n_modes * FLOPS_MODE
        rec = {"bound": "fp64", "kernel": "k_turb64_records", "achieved": round(sflops / (st.ms_sum64 * 1e-3) / 1e12, 3),
               "peak": round(fp64_peak, 3), "unit": "TFLOP/s", "kernel_ms": round(st.ms_sum64, 3), "per_launch": sflops,
               "records": st.rec64_records, "slots_summed": st.rec64_slots, "samples_summed_in_tracer": st.rec64_short,
               "traffic": None, "algorithmic_bytes": 32 * st.rec64_records}
    rec["frac"] = round(rec["achieved"] / rec["peak"], 4)
    rec["peak_source"] = "so_probe_fma_peak (measured FP64 FMA chains on this GPU)"
    return {"mrays_s": round(world * npix / (ms_frame * 1e-3) / 1e6, 4), "ms_per_frame": round(ms_frame, 3),
            "frames": len(ms), "ms_frames": [round(x, 3) for x in ms], "clocks": clocks,
            "phases_ms": {"recording_pass": round(st.ms_rec64, 3), "turbulence_sums": round(st.ms_sum64, 3),
                          "emission_and_transfer": round(st.ms_emit64, 3), "replay_pass": round(st.ms_replay64, 3)},
            "deferred_emission": bool(st.emit64),
            "roofline": rec, "whole_frame": whole}


# The reference arm's scene (run_reference): the synchrotron geometry with the reference's own flow
# model at the torus's indices, fBm turbulence evaluated in place, fixed density.
REF_SCENE = ["flow.n_index=1.5", "flow.theta0=16.86", "flow.h_over_r=0.3", "flow.keplerian_fraction=0.8",
             "flow.turbulence=0.3", "flow.n0=1e6"]


def same_scene_record(args, so, world, rank, local):
    """This library on exactly the reference arm's scene and pixels (pixel centres, one sample, fBm in
    place), end to end through so_trace_rays with host arrays (the reference arm's per-ray call),
    beside the reference's own trace_ray on the host cores over a bounded sample of those pixels."""
    import torch
    W = args.size
    sh = so.Shot("synchrotron_1024.ini", [f"camera.width={W}", f"camera.height={W}", *REF_SCENE])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_flow_noise(so.abi.SO_FLOW_NOISE_INLINE)
    f = sh.frame(0)
    X, Y = so.pixel_centres(f, W, W)
    r.trace_rays(f, X, Y)  # warm-up: the record pool is sized for the full list here, not in a timed call
    torch.cuda.synchronize()
    t = []
    for _ in range(2):
        t0 = time.perf_counter()
        out = r.trace_rays(f, X, Y)
        t.append(time.perf_counter() - t0)
    st = r.trace_stats()
    r.close()
    ours = allreduce_max(float(np.mean(t)), world)
    rec = {"workload": f"reference arm's scene: synchrotron geometry {W}x{W}, reference flow model (n ~ r^-1.5, "
                       "Theta 16.86 r^-0.84, h/r 0.3, 0.8 Keplerian, fBm turbulence rms 0.3 in place, n0 1e6), "
                       "every pixel centre, FP64",
           "mrays_s_e2e": round(world * W * W / ours / 1e6, 4), "s_per_frame": round(ours, 3),
           "api": "so_trace_rays, host arrays in and out", "escaped": int((out["fate"] == 1).sum()),
           "s_calls": [round(x, 3) for x in t],
           "deferred_emission": bool(st.emit64), "records": st.rec64_records, "waves": st.rec64_waves,
           "phases_ms": {"recording_pass": round(st.ms_rec64, 3), "emission_and_transfer": round(st.ms_emit64, 3),
                         "replay_pass": round(st.ms_replay64, 3)}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import _oracle
        if _oracle.have_ref():
            R = _oracle.RefShot(os.path.join(PKG_DIR, "shots", "synchrotron_1024.ini"),
                                [f"camera.width={W}", f"camera.height={W}", *REF_SCENE])
            threads = os.cpu_count() or 1
            n = 65536
            idx = np.linspace(0, W * W - 1, n).astype(np.int64)
            fr = R.frame(0)
            t0 = time.perf_counter()
            _oracle.ref_trace(R.scene, fr, X[idx], Y[idx], threads=threads)
            dt = time.perf_counter() - t0
            v = n / dt / 1e6
            rec["reference_cpu"] = {"mrays_s": round(v, 6), "cores": threads,
                                    "sample": f"{n} evenly strided pixel centres, the reference's trace_ray "
                                              f"(oracle/_ref), {dt:.1f} s"}
            rec["speedup_vs_reference_cpu"] = round(rec["mrays_s_e2e"] / v, 1)
    return rec


def run_shadow(args, so, world, rank, local):
    """The vacuum shadow scene (a = 0.94, i = 17 deg, observer at 1000 M, pixel centres over +-8 M,
    DP5(4) tolerance 1e-10, no emission) at 2048^2 through the mixed path, against the plain FP64
    tracer on the same frame.  The per-image figure is the termination class of every sample (the
    image itself is empty without a sky or disk)."""
    import torch
    torch.cuda.set_device(local)
    W = args.size or 2048
    sh = so.Shot("shadow_selftest_256.ini", [f"camera.width={W}", f"camera.height={W}"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    f = rank_frame(sh, rank)
    npix = W * W
    d_img = torch.empty((W, W, 4), dtype=torch.float32, device="cuda")
    stream = torch.cuda.ExternalStream(r.stream())
    r.set_precision(so.abi.SO_PREC_FP64)
    st64 = r.render_device(f, d_img.data_ptr(), stats=True)
    path = "fp64" if args.path == "fp64" else "mixed"
    if path == "mixed":
        r.set_precision(so.abi.SO_PREC_MIXED)
    for _ in range(args.warmup):
        r.render_device(f, d_img.data_ptr())
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(i))
                ev[i][0].record(stream)
            r.render_device(f, d_img.data_ptr())
            with torch.cuda.stream(stream):
                ev[i][1].record(stream)
        torch.cuda.synchronize()
    ms_step = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    barrier(world)
    ms_step = allreduce_max(ms_step, world)
    value = job_rate(world, npix, ms_step) / 1e6
    st = r.render_device(f, d_img.data_ptr(), stats=True)
    classes = None
    if path == "mixed":
        fm, band = r.last_fates(npix)
        r.set_precision(so.abi.SO_PREC_MIXED, band_m=1e6)
        r.render_device(f, d_img.data_ptr())
        f64, _ = r.last_fates(npix)
        r.set_precision(so.abi.SO_PREC_MIXED)
        out = ~band
        classes = {"samples_outside_band": int(out.sum()),
                   "class_mismatch_outside_band": int((fm[out] != f64[out]).sum()),
                   "class_mismatch_in_band": int((fm[band] != f64[band]).sum())}
    fp64_peak, fp32_peak = so.probe_fma_peak(local)
    if path == "fp64":
        flops = st.attempts * FLOPS_ATTEMPT + st.accepted * FLOPS_ACCEPT
        roof = {"bound": "fp64", "achieved": round(flops / (st.ms_kernel * 1e-3) / 1e12, 3),
                "peak": round(fp64_peak, 3), "unit": "TFLOP/s", "kernel": "k_trace64", "kernel_ms": st.ms_kernel,
                "per_launch": flops, "peak_source": "so_probe_fma_peak (measured FP64 FMA chains on this GPU)"}
    else:
        # FP32 tracer: the DP5(4) attempt's algorithmic flops in FP32 (the two-sum compensation and
        # the FP32 reciprocals not counted) against the measured FP32 FMA rate
        flops = st.attempts_fp32 * FLOPS_ATTEMPT
        roof = {"bound": "fp32", "achieved": round(flops / (st.ms_fp32 * 1e-3) / 1e12, 3),
                "peak": round(fp32_peak, 3), "unit": "TFLOP/s", "kernel": "k_trace32", "kernel_ms": st.ms_fp32,
                "per_launch": flops, "peak_source": "so_probe_fma_peak (measured FP32 FMA chains on this GPU)"}
    roof["frac"] = round(roof["achieved"] / roof["peak"], 4)
    roof["traffic"] = None
    host_pinned = torch.empty((W, W, 4), dtype=torch.float32).pin_memory().numpy()
    for _ in range(2):
        r.render(f, out=host_pinned)
    torch.cuda.synchronize()
    e2e_ms = []
    for i in range(args.steps):
        t0 = time.perf_counter()
        r.render(f, out=host_pinned)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_step = allreduce_max(float(np.mean(e2e_ms)), world)
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if path == "fp64" else "f32+f64", "data": "synthetic",
        "config": {"workload": f"vacuum shadow scene {W}x{W}, a=0.94, i=17 deg, observer 1000 M, pixel centres "
                               f"over +-8 M, DP5(4) tolerance 1e-10", "path": path,
                   "band_rays": st.band_rays if path == "mixed" else None,
                   "fp64_rays": st.fp64_rays if path == "mixed" else None,
                   "plain_fp64_mrays_s": round(npix / (st64.ms_kernel * 1e-3) / 1e6, 4),
                   "attempts_per_ray": st.attempts / npix, "termination_class": classes,
                   "l2": "256 MiB buffer written between timed steps"},
        "roofline": roof,
        "e2e": {"value": round(world * npix / (e2e_step * 1e-3) / 1e6, 4), "unit": "Mrays/s",
                "h2d_bytes_per_step": C.sizeof(so.abi.Frame), "d2h_bytes_per_step": W * W * 16},
        "gpu_launches": args.steps * (2 if path == "fp64" else 7),
        "clocks": clk.summary(),
    }
    r.close()
    return line


def run_rays(args, so, world, rank, local):
    """The drop-in ray-list path on the reference arm's scene: the reference flow model with its fBm
    turbulence in place, every pixel centre of the W x W synchrotron geometry, one ray each.  `value`:
    so_trace_rays_device with the coordinates and every per-ray output (fate, winding order, escape
    direction, the four intensity bins, step counts) resident on the device; `e2e`: so_trace_rays
    with host arrays, the copies inside the timed region.  The CPU baseline is the reference's own
    trace_ray on the host cores over a bounded sample of the same pixels."""
    import torch
    torch.cuda.set_device(local)
    W = args.size or 2048
    sh = so.Shot("synchrotron_1024.ini", [f"camera.width={W}", f"camera.height={W}", *REF_SCENE])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    r.set_flow_noise(so.abi.SO_FLOW_NOISE_INLINE)
    f = rank_frame(sh, rank)
    X, Y = so.pixel_centres(f, W, W)
    n = X.size
    dev = torch.device("cuda", local)
    dx, dy = torch.from_numpy(X).to(dev), torch.from_numpy(Y).to(dev)
    outs = {"fate": torch.int8, "ncross": torch.int8, "theta": torch.float64, "phi": torch.float64,
            "I": torch.float32, "n_accepted": torch.int32, "n_attempts": torch.int32}
    d = {k: torch.empty((n, 4) if k == "I" else (n,), dtype=t, device=dev) for k, t in outs.items()}
    torch.cuda.synchronize()  # the coordinates are on the device before the library's stream reads them
    ro = so.abi.RaysOut(*[C.c_void_p(d[k].data_ptr()) if k in d else None
                          for k, _ in so.abi.RaysOut._fields_])
    lib = so.lib()

    def trace_device():
        rc = lib.so_trace_rays_device(r.h, C.byref(f), n, C.c_void_p(dx.data_ptr()), C.c_void_p(dy.data_ptr()),
                                      C.byref(ro))
        if rc != so.abi.SO_OK:
            raise so.TracerError(rc, lib.so_last_error(r.h).decode())

    stream = torch.cuda.ExternalStream(r.stream())
    for _ in range(args.warmup):
        trace_device()
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(i))
                ev[i][0].record(stream)
            trace_device()
            with torch.cuda.stream(stream):
                ev[i][1].record(stream)
        torch.cuda.synchronize()
    ms_step = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    st = r.trace_stats()
    barrier(world)
    ms_step = allreduce_max(ms_step, world)
    value = job_rate(world, n, ms_step) / 1e6
    fp64_peak, _ = so.probe_fma_peak(local)
    # the recording pass (the geodesics: DP5(4) attempts and accepted steps) is the longest kernel;
    # the emission at the records (fBm noise in place) and the ordered transfer follow it
    flops = st.attempts * FLOPS_ATTEMPT + st.accepted * FLOPS_ACCEPT
    roof = {"bound": "fp64", "achieved": round(flops / (st.ms_rec64 * 1e-3) / 1e12, 3), "peak": round(fp64_peak, 3),
            "unit": "TFLOP/s", "kernel": "k_trace64 (recording pass of the ray list)", "kernel_ms": st.ms_rec64,
            "per_launch": flops, "peak_source": "so_probe_fma_peak (measured FP64 FMA chains on this GPU)",
            "phases_ms": {"recording_pass": round(st.ms_rec64, 3), "emission_and_transfer": round(st.ms_emit64, 3),
                          "replay_pass": round(st.ms_replay64, 3)},
            "traffic": None}
    roof["frac"] = round(roof["achieved"] / roof["peak"], 4)
    k = r.trace_rays(f, X, Y)  # warm-up of the host-array form
    e2e_s = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        k = r.trace_rays(f, X, Y)
        e2e_s.append(time.perf_counter() - t0)
    e2e_step = allreduce_max(float(np.mean(e2e_s)), world)
    same = all(np.array_equal(k[key], d[key].cpu().numpy()) for key in outs)
    line = {
        "metric": "Mrays/s (so_trace_rays, every per-ray output)", "value": round(value, 4), "unit": "Mrays/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"reference arm's scene: synchrotron geometry {W}x{W}, reference flow model "
                               "(n ~ r^-1.5, Theta 16.86 r^-0.84, h/r 0.3, 0.8 Keplerian, fBm turbulence rms 0.3 "
                               "in place, n0 1e6), every pixel centre, one ray each", "path": "fp64",
                   "api": "so_trace_rays_device (value), so_trace_rays with host arrays (e2e)",
                   "deferred_emission": bool(st.emit64), "records": st.rec64_records, "waves": st.rec64_waves,
                   "attempts_per_ray": st.attempts / n, "flow_steps_per_ray": st.flow_steps / n,
                   "escaped": int((k["fate"] == 1).sum()), "host_and_device_outputs_identical": bool(same),
                   "l2": "256 MiB buffer written between timed steps"},
        "roofline": roof,
        "e2e": {"value": round(world * n / e2e_step / 1e6, 4), "unit": "Mrays/s", "h2d_bytes_per_step": 16 * n,
                "d2h_bytes_per_step": n * (1 + 1 + 8 + 8 + 16 + 4 + 4)},
        "gpu_launches": args.steps * 4 * max(st.rec64_waves, 1) if st.rec64_waves else args.steps,
        "clocks": clk.summary(),
    }
    r.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import _oracle
        if _oracle.have_ref():
            R = _oracle.RefShot(os.path.join(PKG_DIR, "shots", "synchrotron_1024.ini"),
                                [f"camera.width={W}", f"camera.height={W}", *REF_SCENE])
            threads = os.cpu_count() or 1
            m = 65536
            idx = np.linspace(0, n - 1, m).astype(np.int64)
            t0 = time.perf_counter()
            _oracle.ref_trace(R.scene, R.frame(0), X[idx], Y[idx], threads=threads)
            dt = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": round(m / dt / 1e6, 6), "unit": "Mrays/s", "cores": threads,
                                    "kind": "reference",
                                    "sample": f"{m} evenly strided pixel centres, the reference's trace_ray "
                                              f"(oracle/_ref), {dt:.1f} s"}
    return line


# surrogate network: forward FLOPs per ray (FMA = 2; the head is 16 wide on the tensor cores)
SUR_FLOPS_RAY = 2 * (128 * 256 + 3 * 256 * 256 + 256 * 16)
SUR_SIGMA = 0.35           # std of the random Fourier frequencies per unit of the scaled inputs


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return d, "MEASURED_PEAKS.json (measured on this pool's B200s)"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback figures"


def run_surrogate(args, so, world, rank, local):
    """Thin-disk frame through the ray surrogate: network trained on the GPU on rays of the FP64
    integrator, fused tensor-core inference, FP64 integrator in the critical band and on a 1% audit
    sample.  Compared with the same frame traced by the FP64 integrator for every pixel."""
    import torch
    torch.cuda.set_device(local)
    W = args.size or 4096
    sh = so.Shot("thin_disk_4096.ini", [f"camera.width={W}", f"camera.height={W}"])
    r = so.Renderer(sh.scene, sh.tables, sh.settings)
    f = sh.frame(0)
    sur = so.Surrogate(local, batch=65536, lr=2e-3, lr_final=5e-5, warmup=100, seed=1 + rank,
                       fourier_sigma=SUR_SIGMA)
    t0 = time.perf_counter()
    rays, tgt, st = sur.dataset(r, f, args.train_rays, 4096, seed=1 + rank)
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    last = sur.train(rays, tgt, args.train_steps)
    t_train = time.perf_counter() - t0
    del rays, tgt
    hr, ht, _ = sur.dataset(r, f, 1 << 18, 256, seed=1000 + rank)
    held = sur.evaluate(hr, ht)
    del hr, ht
    stream = torch.cuda.ExternalStream(r.stream())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed(band_m, audit, n):
        out = torch.zeros((W, W, 4), dtype=torch.float32, device="cuda")
        ms, rep = [], None
        for i in range(n):
            with torch.cuda.stream(stream):
                flush.fill_(float(i))
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
            out, rep = sur.render(r, f, band_m=band_m, audit_frac=audit, audit_seed=2, out=out)
            with torch.cuda.stream(stream):
                b.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        return out, rep, ms

    # the FP64 integrator on every pixel (same tracer, routing and scatter kernels)
    img64, rep64, ms64 = timed(1e9, 0.0, 2)
    ref = img64.cpu().numpy().astype(np.float64)
    for _ in range(args.warmup):
        timed(args.band, 0.01, 1)
    barrier(world)
    with ClockSampler(local) as clk:
        img, rep, ms = timed(args.band, 0.01, args.steps)
    ms_step = allreduce_max(float(np.mean(ms)), world)
    npix = W * W
    value = job_rate(world, npix, ms_step) / 1e6
    fp64_ms = float(np.mean(ms64))
    a = img.cpu().numpy().astype(np.float64)
    l1 = float(np.abs(a[..., 1] - ref[..., 1]).sum() / max(np.abs(ref[..., 1]).sum(), 1e-300))
    flux = float(a[..., 1].sum() / ref[..., 1].sum() - 1.0)
    peaks, src = measured_peaks()
    n_mlp = rep.surrogate_rays + rep.audit_rays
    flops = n_mlp * SUR_FLOPS_RAY
    achieved = flops / (rep.ms_mlp * 1e-3) / 1e12
    roof = {"bound": "tensor", "achieved": round(achieved, 2), "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
            "frac": round(achieved / peaks["bf16_tflops"], 4), "traffic": None, "kernel": "k_mlp_fused",
            "kernel_ms": rep.ms_mlp, "per_launch": flops, "peak_source": src + ", dense bf16 burst"}
    # Trade-off: the image error falls only as more pixels go to the integrator (the network's radius
    # error is spread evenly over the disk, so no per-pixel score singles out the bad pixels); the
    # seeded audit share is raised until the frame is at 1e-3 and the speed-up at each point recorded
    tradeoff = []
    for frac in (0.1, 0.3, 0.6, 0.8, 0.9, 0.95):
        im, rp, mss = timed(args.band, frac, 2)
        b = im.cpu().numpy().astype(np.float64)
        e = float(np.abs(b[..., 1] - ref[..., 1]).sum() / max(np.abs(ref[..., 1]).sum(), 1e-300))
        tradeoff.append({"integrator_share": round((rp.band_rays + rp.audit_rays) / rp.rays, 4), "image_rel_l1": e,
                         "ms": round(float(np.mean(mss)), 3), "speedup_vs_fp64": round(fp64_ms / float(np.mean(mss)), 3)})
    # e2e: the frame into host memory (descriptor in, 4 floats per pixel out)
    host = torch.empty((W, W, 4), dtype=torch.float32).pin_memory()
    e2e_ms = []
    for i in range(args.steps):
        t0 = time.perf_counter()
        out, _ = sur.render(r, f, band_m=args.band, audit_frac=0.01, audit_seed=2, out=img)
        host.copy_(out)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_step = allreduce_max(float(np.mean(e2e_ms)), world)
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16+f64", "data": "synthetic",
        "config": {"workload": f"thin Novikov-Thorne disk frame {W}x{W}, a=0.9, i=60 deg, r_cam=1000 M, fov +-12 M, "
                               "pixel centres; surrogate outside the critical band, FP64 integrator inside it and "
                               "on a 1% audit sample",
                   "band_m": args.band, "plain_fp64_mrays_s": round(npix / (fp64_ms * 1e-3) / 1e6, 4),
                   "plain_fp64_ms": round(fp64_ms, 3), "speedup_vs_fp64": round(fp64_ms / ms_step, 3),
                   "image_rel_l1_vs_fp64": l1, "total_flux_err_vs_fp64": flux,
                   "rays": rep.rays, "surrogate_rays": rep.surrogate_rays, "band_rays": rep.band_rays,
                   "audit_rays": rep.audit_rays, "ms_route": rep.ms_route, "ms_mlp": rep.ms_mlp,
                   "ms_shade": rep.ms_shade, "ms_integrator": rep.ms_integrator,
                   "audit": {"class_mismatch": rep.audit_class_mismatch, "dir_err_rad": rep.audit_dir_err,
                             "u_err": rep.audit_u_err, "r_rel_err": rep.audit_r_err, "g_err": rep.audit_g_err,
                             "l1": rep.audit_l1, "flux": rep.audit_flux},
                   "training": {"rays": args.train_rays, "steps": args.train_steps, "batch": 65536,
                                "dataset_s": round(t_data, 2), "train_s": round(t_train, 2),
                                "last_loss": last.total, "heldout_loss": held.total,
                                "heldout_class_accuracy": held.accuracy},
                   "l2": "256 MiB buffer written between timed steps", "frames_per_s": round(1e3 / ms_step * world, 3),
                   "tradeoff_integrator_share": tradeoff},
        "roofline": roof,
        "e2e": {"value": round(world * npix / (e2e_step * 1e-3) / 1e6, 4), "unit": "Mrays/s",
                "h2d_bytes_per_step": C.sizeof(so.abi.Frame), "d2h_bytes_per_step": W * W * 16},
        "gpu_launches": args.steps * 8,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_disk(so, sh, f, W, budget_s=args.cpu_seconds)
    sur.close()
    r.close()
    return line


def cpu_baseline_disk(so, sh, f, W, budget_s=15.0):
    """The oracle port on the thin-disk frame (FP64 integrator, disk emission), host cores."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle
    threads = os.cpu_count() or 1
    n = 4096
    t0 = time.perf_counter()
    x, y = _sample_pixels(so, f, W, n)
    _oracle.orc_trace(sh.scene, f, x, y, threads=threads)
    dt = time.perf_counter() - t0
    n2 = int(min(max(n * budget_s / max(dt, 1e-3), n), W * W))
    x, y = _sample_pixels(so, f, W, n2)
    t0 = time.perf_counter()
    _oracle.orc_trace(sh.scene, f, x, y, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": round(n2 / dt / 1e6, 6), "unit": "Mrays/s", "cores": threads, "kind": "port",
            "sample": f"{n2} evenly strided pixel centres of the {W}x{W} thin-disk frame, oracle/so_oracle.c, "
                      f"{threads} threads, {dt:.1f} s"}


def run_wavefront(args, so, world, rank, local):
    """The photon-ring batch: 4 spins x 2 inclinations x 8 turbulence times / zooms of the torus
    plasma, W x W windows on the critical curve, all frames in one job space: a persistent recording
    pass over every frame, the turbulence sums at its records (FP32 for mixed precision, FP64
    otherwise), the emission and the ordered transfer, in waves through the record pool, replayed
    from a CUDA graph; launch shape from the autotuner (run on a 128 x 128 copy of the batch)."""
    import importlib
    import torch
    torch.cuda.set_device(local)
    wf = importlib.import_module("spacetime_optics_b200.wavefront")
    W = args.size or 512
    prec = so.abi.SO_PREC_MIXED if args.path != "fp64" else so.abi.SO_PREC_FP64
    shots = wf.photon_ring_shots(so, 128)
    r = so.Renderer(shots[0].scene, shots[0].tables, shots[0].settings, device=local)
    r.set_plasma(shots[0].plasma())
    r.set_precision(prec)
    b, _, scenes, frames, fs = wf.photon_ring_batch(so, r, 128)
    small = torch.zeros((len(frames), 128, 128, 4), dtype=torch.float32, device="cuda")
    tune = b.autotune(small.data_ptr())
    b.close()
    b, _, scenes, frames, fs = wf.photon_ring_batch(so, r, W)
    b.set_tune(tune.ctas_per_sm, tune.interleave, tune.tile, tune.queue_chunk)
    out = torch.zeros((len(frames), W, W, 4), dtype=torch.float32, device="cuda")
    stream = torch.cuda.ExternalStream(r.stream())
    for _ in range(args.warmup):
        b.render(out.data_ptr())
    torch.cuda.synchronize()
    ms = []
    barrier(world)
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            b.render(out.data_ptr())
            with torch.cuda.stream(stream):
                e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
    ms_step = allreduce_max(float(np.mean(ms)), world)
    st = b.render(out.data_ptr(), stats=True)
    nrays = len(frames) * W * W
    value = job_rate(world, nrays, ms_step) / 1e6
    fp64_peak, _ = so.probe_fma_peak(local)
    n_modes = shots[0].plasma().n_modes
    if prec == so.abi.SO_PREC_FP64:
        # FP64 geometry and FP64 turbulence sums: FP64 pipe
        flops = (st.attempts * FLOPS_ATTEMPT + st.accepted * FLOPS_ACCEPT +
                 st.flow_steps * (FLOPS_FLOW + n_modes * FLOPS_MODE))
        achieved = flops / (ms_step * 1e-3) / 1e12
        roof = {"bound": "fp64", "achieved": round(achieved, 3), "peak": round(fp64_peak, 3), "unit": "TFLOP/s",
                "frac": round(achieved / fp64_peak, 4), "traffic": None,
                "kernel": ("whole batch: k_trace64 recording pass + k_turb64_records + k_emit64_records + k_transfer64"
                           if st.rec64_waves else "k_trace64"),
                "peak_source": "so_probe_fma_peak (measured FP64 FMA chains on this GPU)"}
    else:
        # FP64 geometry, FP32 turbulence sums: the SFU cosines (one per mode per flow step) dominate
        sfu_peak = so.probe_sfu_peak(local)
        ops = st.flow_steps * n_modes
        achieved = ops / (ms_step * 1e-3) / 1e9
        roof = {"bound": "sfu", "achieved": round(achieved, 3), "peak": round(sfu_peak, 3), "unit": "Gop/s",
                "frac": round(achieved / sfu_peak, 4), "traffic": None,
                "kernel": ("whole batch: k_trace64 recording pass + k_turb32_rec64 + k_emit64_records + k_transfer64"
                           if st.rec64_waves else "k_trace64 (FP32 sums)"),
                "peak_source": "so_probe_sfu_peak (measured SFU cosine chains on this GPU)",
                "fp64_geometry_flops": st.attempts * FLOPS_ATTEMPT + st.accepted * FLOPS_ACCEPT}
    # e2e: the batch through so_batch_render and every frame read back into pinned host memory (the
    # frames' descriptors were uploaded once at so_batch_create: no per-step input), at most 2 steps
    # (the copy runs on torch's stream, ordered after the library's: a pinned buffer used on the
    # library's stream would keep an event on it past r.close())
    host = torch.empty((len(frames), W, W, 4), dtype=torch.float32).pin_memory()
    e2e_s = []
    for _ in range(max(1, min(args.steps, 2))):
        t0 = time.perf_counter()
        b.render(out.data_ptr())
        torch.cuda.current_stream().wait_stream(stream)
        host.copy_(out, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        e2e_s.append(time.perf_counter() - t0)
    e2e_step = allreduce_max(float(np.mean(e2e_s)), world)
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == so.abi.SO_PREC_FP64 else "f64+f32", "data": "synthetic",
        "config": {"workload": f"photon-ring batch: {len(frames)} frames of {W}x{W} (spins 0/0.5/0.9/0.99, "
                               "incl 17/60 deg, 8 turbulence times, zoom 1e3-4e4 on the critical curve), torus "
                               "plasma with 512 modes, " + (f"deferred sums and emission in {st.rec64_waves} waves"
                                                            if st.rec64_waves else "one persistent launch") +
                               " replayed from a CUDA graph",
                   "tune": {"ctas_per_sm": tune.ctas_per_sm, "interleave": tune.interleave, "tile": tune.tile,
                            "queue_chunk": tune.queue_chunk, "tuned_on": "128x128"},
                   "frames_per_s": round(world * len(frames) / (ms_step * 1e-3), 4),
                   "attempts_per_ray": st.attempts / nrays, "flow_steps_per_ray": st.flow_steps / nrays,
                   "records": st.rec64_records, "record_waves": st.rec64_waves,
                   "samples_traced_in_place": st.rec64_short,
                   "l2": "inputs (mode table, frame descriptors) are small; no flush (one step is seconds long)"},
        "roofline": roof,
        "e2e": {"value": round(world * nrays / e2e_step / 1e6, 4), "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": nrays * 16},
        # per wave: recording pass, sums, emission, transfer, replay launch (returns at once); then
        # resolve; without waves: the persistent tracer and resolve
        "gpu_launches": args.steps * ((st.rec64_waves * 5 + 1) if st.rec64_waves else 2),
        "clocks": clk.summary(),
    }
    b.close()
    r.close()
    return line


def _sample_pixels(so, f, W, n):
    X, Y = so.pixel_centres(f, W, W)
    idx = np.linspace(0, W * W - 1, n).astype(np.int64)
    return X[idx], Y[idx]


def cpu_baseline(so, sh, f, W, budget_s=15.0):
    """The oracle port (the reference's algorithm restated in C, same torus workload) on the host cores,
    over a bounded, evenly strided sample of the frame's pixels."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle
    threads = os.cpu_count() or 1
    p = sh.plasma()
    modes = so.plasma_modes(p)
    n = 256
    t0 = time.perf_counter()
    x, y = _sample_pixels(so, f, W, n)
    _oracle.orc_trace(sh.scene, f, x, y, plasma=p, modes=modes, threads=threads)
    dt = time.perf_counter() - t0
    n2 = int(min(max(n * budget_s / max(dt, 1e-3), n), 2_000_000))
    x, y = _sample_pixels(so, f, W, n2)
    t0 = time.perf_counter()
    _oracle.orc_trace(sh.scene, f, x, y, plasma=p, modes=modes, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": round(n2 / dt / 1e6, 6), "unit": "Mrays/s", "cores": threads, "kind": "port",
            "sample": f"{n2} evenly strided pixel centres of the {W}x{W} frame, oracle/so_oracle.c, "
                      f"{threads} threads, {dt:.1f} s"}


def run_reference(args, so):
    """The reference's own trace_ray (oracle/_ref/libbhref.so, built from the reference sources) on
    this workload's geometry with the reference's own hot-flow model (the torus plasma and its
    Fourier turbulence are not part of the reference), all host threads, bounded samples."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle
    if not _oracle.have_ref():
        return {"impl": "reference", "unavailable": "oracle/_ref/libbhref.so was not built (reference tree absent)"}
    W = args.size
    path = os.path.join(PKG_DIR, "shots", "synchrotron_1024.ini")
    R = _oracle.RefShot(path, [f"camera.width={W}", f"camera.height={W}", "flow.n_index=1.5",
                               "flow.theta0=16.86", "flow.h_over_r=0.3", "flow.keplerian_fraction=0.8",
                               "flow.turbulence=0.3", "flow.n0=1e6"])
    f = R.frame(0)
    threads = os.cpu_count() or 1
    X, Y = so.pixel_centres(f, W, W)
    n = 256
    idx = np.linspace(0, W * W - 1, n).astype(np.int64)
    t0 = time.perf_counter()
    _oracle.ref_trace(R.scene, f, X[idx], Y[idx], threads=threads)
    dt = time.perf_counter() - t0
    per_step = max(10.0, min(30.0, 90.0 / max(args.steps + args.warmup, 1)))
    n2 = int(min(max(n * per_step / max(dt, 1e-3), n), W * W))
    idx = np.linspace(0, W * W - 1, n2).astype(np.int64)
    for _ in range(min(args.warmup, 1)):
        _oracle.ref_trace(R.scene, f, X[idx[:256]], Y[idx[:256]], threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _oracle.ref_trace(R.scene, f, X[idx], Y[idx], threads=threads)
        times.append(time.perf_counter() - t0)
    v = n2 / float(np.mean(times)) / 1e6
    return {"metric": METRIC, "value": round(v, 6), "unit": "Mrays/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(float(np.mean(times)) * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": f"synchrotron frame {W}x{W}, a=0.94, i=163 deg, fov +-12 M, 230 GHz, "
                                   "reference flow model (n ~ r^-1.5, Theta 16.86 (r)^-0.84, h/r 0.3, fBm turbulence "
                                   "rms 0.3)", "path": "reference host FP64"},
            "cpu_baseline": {"value": round(v, 6), "unit": "Mrays/s", "cores": threads, "kind": "reference",
                             "sample": f"{n2} evenly strided pixel centres per step, reference trace_ray "
                                       f"(oracle/_ref), {threads} threads"},
            "e2e": {"value": round(v, 6), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="synchrotron",
                    choices=["synchrotron", "surrogate", "wavefront", "shadow", "flow", "rays"])
    ap.add_argument("--size", type=int, default=0, help="frame width (default: synchrotron, shadow and rays 2048, surrogate 4096, wavefront 512, flow 1024)")
    ap.add_argument("--band", type=float, default=0.1, help="surrogate: critical band half-width (M)")
    ap.add_argument("--train-rays", type=int, default=1 << 24)
    ap.add_argument("--train-steps", type=int, default=40000)
    ap.add_argument("--path", default="auto", choices=["auto", "fp64", "mixed"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-same-scene", action="store_true", help="skip the reference arm's scene on this library")
    args = ap.parse_args()
    so = load_package()
    if args.impl == "reference":
        args.size = args.size or 2048
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return 0
        print(json.dumps(run_reference(args, so)), flush=True)
        return 0
    world, rank, local = dist_setup()
    if args.workload == "surrogate":
        line = run_surrogate(args, so, world, rank, local)
    elif args.workload == "wavefront":
        line = run_wavefront(args, so, world, rank, local)
    elif args.workload == "shadow":
        line = run_shadow(args, so, world, rank, local)
    elif args.workload == "rays":
        line = run_rays(args, so, world, rank, local)
    elif args.workload == "flow":
        args.size = args.size or 1024
        line = run_ours(args, so, world, rank, local)
    else:
        args.size = args.size or 2048
        line = run_ours(args, so, world, rank, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
