"""The multi-rank logic of bench.py on the host (gloo, world size 2): process-group set-up from the
torchrun environment, max-over-ranks timing, per-rank frames, whole-job throughput and the
reference arm printing on rank 0 only."""
import importlib.util
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as dist
    b = _bench()
    so = b.load_package()
    w, r, local = b.dist_setup("gloo")
    times = [12.5, 30.0]
    ms = b.allreduce_max(times[r], w)
    b.barrier(w)
    sh = so.Shot("synchrotron_1024.ini", ["camera.width=32", "camera.height=32"])
    f = b.rank_frame(sh, r)
    rate = b.job_rate(w, 1000, ms)
    q.put((r, w, ms, f.t, rate))
    dist.destroy_process_group()


def test_two_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, ms0, t0, rate0), (r1, w1, ms1, t1, rate1) = out
    assert (r0, r1, w0, w1) == (0, 1, 2, 2)
    assert ms0 == ms1 == 30.0            # the slower rank's time
    assert t1 - t0 == pytest.approx(50.0)  # each rank its own turbulence time
    assert rate0 == rate1 == pytest.approx(2 * 1000 / 0.030)


def test_reference_arm_prints_on_rank_zero_only(tmp_path):
    import subprocess
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0
    assert p.stdout.strip() == ""
