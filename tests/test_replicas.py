"""The multi-rank host logic of bench.py on CPU with the gloo backend,
world size 2: the max-over-ranks timing reduction, and the reference arm
launched as a multi-GPU bench run is (torch.distributed.run, rendezvous on
127.0.0.1), where rank 0 alone prints one JSON line and every rank exits 0."""
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


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    ms = 10.0 + 5.0 * rank                       # rank 1 is the slower one
    m = bench.allreduce_max(dist, ms, "cpu")
    bench.barrier(dist)
    out.put((rank, m, world * bench.sim_days_per_hour(100, m / 1e3)))
    dist.destroy_process_group()


def test_max_over_ranks_two_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]   # every rank sees the slowest rank's time
    assert res[0][2] == res[1][2] > 0


def test_reference_arm_under_torchrun_prints_once():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--lmin", "3", "--level", "4", "--nz", "2", "--cpu-seconds", "0.5"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
