"""The multi-GPU host logic on CPU (gloo, world size 2).  The search shards
by beam with no data exchange (replicas): each rank searches its own gulp,
the step time is the maximum over ranks and the job's value is world x
beam-seconds / that time.  Ranks here are CPU processes; no GPU is used."""
import os
import socket
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r's timings: the batched, plain and end-to-end steps
        mine = [10.0 + rank, 30.0 - 5.0 * rank, 12.5 + 0.25 * rank]
        got = bench.max_over_ranks(torch, dist, mine, "cpu")
        value = bench.whole_job_value(world, 773.0941, got[0])
        dist.barrier()
        q.put((rank, got, value))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_value_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, value in out:
        assert got == [11.0, 30.0, 12.75]          # slowest rank per timing
        assert value == pytest.approx(2 * 773.0941 / 0.011)


def test_single_rank_value_and_identity():
    assert bench.max_over_ranks(torch, None, [3.0, 4.0], "cpu") == [3.0, 4.0]
    assert bench.whole_job_value(1, 773.0941, 12.0) == pytest.approx(773.0941 / 0.012)


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun, ranks other than 0 of the reference arm exit 0 without
    work and print nothing."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, env=env, timeout=120, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
