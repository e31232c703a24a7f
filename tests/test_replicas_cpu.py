"""The multi-GPU form of bench.py is replicas only: every rank runs its own trajectory, the ranks
meet at barriers, and the job time is the max over ranks.  These host-side pieces run here as
two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, ws, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    import bench
    w, r, l = bench.dist_env()
    bench.barrier(ws)
    t = bench.reduce_max(0.5 + rank, ws)  # rank r "took" 0.5 + r seconds
    bench.barrier(ws)
    out.put((rank, w, r, l, t))
    dist.destroy_process_group()


def test_two_ranks_take_the_max_time():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[0] for x in res] == [0, 1]
    for rank, w, r, l, t in res:
        assert (w, r, l) == (2, rank, rank)
        assert t == pytest.approx(1.5)  # both ranks see the slowest rank's time


def test_bench_gpus_flag_launches_that_many_ranks():
    """`bench.py --gpus 2` started without a launcher starts itself again as two ranks with the
    environment torchrun would give them; the reference arm (CPU only) then prints one line, from
    rank 0, with n_gpus = 2."""
    import json
    import subprocess
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0", "--n", "32"],
                       capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    assert lines[0]["n_gpus"] == 2 and lines[0]["impl"] == "reference"
