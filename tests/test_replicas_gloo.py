"""Multi-process paths of bench.py on CPU (gloo, world size 2): the job time is the maximum
over ranks, and the reference arm runs on rank 0 only (rank 1 exits without output, rank 0
prints the job's one line)."""
import datetime
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, REPO)
    import bench
    v = bench.max_over_ranks_of(10.0 + 5.0 * rank, dist, "cpu")
    q.put((rank, v))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: 15.0, 1: 15.0}


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


def test_reference_arm_rank0_prints_one_line_for_the_job():
    """Rank 0 of a 2-rank job runs the reference's CPU path alone (small grid here) and prints
    the one JSON line, with the job's GPU count."""
    import json
    env = dict(os.environ, RANK="0", WORLD_SIZE="2", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--ne", "12", "--steps", "1", "--warmup", "3"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["n_gpus"] == 2 and out["higher_is_better"] is False
    assert out["value"] > 0 and out["config"]["ne"] == [12, 12, 12] and out["config"]["iterations"] > 0
    assert out["e2e"]["value"] == out["value"] and out["cpu_baseline"]["kind"] in ("reference", "port")
