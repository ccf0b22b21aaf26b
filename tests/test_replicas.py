"""Multi-GPU is replicas only: N independent sessions, no collective on the
rendering path; bench.py's whole-job value is all ranks' pixels over the
slowest rank's device time.  Checked with world_size-2 gloo ranks on CPU,
and the reference arm's rank rule (rank 0 alone runs and prints)."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=2,
                            timeout=datetime.timedelta(seconds=60))
    local_ms = [100.0, 250.0][rank]  # rank 1 is the slow one
    value, ms_max = bench.replica_value(1000000, 10, local_ms, 2, dist, device="cpu")
    out.put((rank, value, ms_max))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_value_is_all_pixels_over_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, value, ms_max in res:
        assert ms_max == 250.0
        assert abs(value - 2 * 1e6 * 10 / 0.25 / 1e6) < 1e-9  # 80 Mpix-frames/s on every rank


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", "0",
                        "--steps", "1", "--warmup", "1", "--gpus", "2"], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", "0",
                        "--steps", "1", "--warmup", "1", "--reference-seconds", "2"], env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
