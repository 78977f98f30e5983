"""The multi-GPU host logic of bench.py on CPU: two gloo ranks (the GPU runs
use NCCL, one rank per GPU, replicas with no data-path collective).  The
step time is the slowest rank's, every rank ends with the same value, and
the throughput counts the work of all ranks; the reference arm prints only
on rank 0."""
import datetime
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


def _rank(rank, ws, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    import bench
    t = bench.max_over_ranks(0.25 * (rank + 1), ws, device="cpu")
    q.put((rank, t, bench.job_throughput(1000.0, ws, t)))
    dist.barrier()
    dist.destroy_process_group()


def test_step_time_is_the_slowest_rank_and_throughput_counts_all_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [0.5, 0.5]
    assert all(abs(g[2] - 2 * 1000.0 / 0.5) < 1e-9 for g in got)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(0.3, 1) == 0.3
    assert bench.job_throughput(10.0, 1, 2.0) == 5.0


def test_reference_arm_prints_only_on_rank_zero():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_gpus_two_starts_two_ranks_and_reports_two():
    """`bench.py --gpus 2` run directly (no torchrun around it) starts two ranks
    under torchrun itself; on the reference arm rank 0 alone prints, with
    n_gpus 2, and the other rank exits 0 without work.  A 64^3 volume keeps the
    CPU work to a second."""
    import json
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "LOCAL_RANK", "WORLD_SIZE", "MASTER_ADDR",
                                                            "MASTER_PORT")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--size", "64", "--steps", "1", "--warmup", "3"],
                       capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    assert lines[0]["n_gpus"] == 2 and lines[0]["impl"] == "reference"
