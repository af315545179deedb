"""The multi-GPU bench logic on CPU: two gloo ranks.

With N GPUs the bench runs N z slabs of one channel (their exchanges are
covered by the slab schedule test) and reports the job time as the slowest
rank's, so every rank must agree on the max of the per-rank times; the reference arm prints one line
from rank 0 and the other ranks exit without work.  Both are checked with
torch.distributed over gloo, world size 2, no GPU."""
import os
import socket
import subprocess
import sys


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    w, r, _ = bench.dist_setup(world, backend="gloo")
    times = [12.5, 17.25]  # this rank's timed region, ms
    bench.barrier(w)
    q.put((r, w, bench.max_over_ranks(times[r], w, device="cpu")))
    import torch.distributed as dist
    dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(out) == [(0, 2, 17.25), (1, 2, 17.25)]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    bench.barrier(1)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
