"""The multi-GPU path of bench.py on CPU: replicas on world_size 2 with the
gloo backend.  Every rank reports its own time; the job time is the largest
(max over ranks), the whole-job throughput counts every replica's steps, and
the reference arm prints on rank 0 only."""
import io
import multiprocessing as mp
import os
import socket
import sys
from contextlib import redirect_stdout

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from datetime import timedelta

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(10.0 * (rank + 1), world)   # rank 0: 10 ms, rank 1: 20 ms
        q.put((rank, t, bench.job_throughput(world, 5, t * 1e-3)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, thr in out:
        assert t == 20.0                      # the slowest replica
        assert abs(thr - 2 * 5 / 0.020) < 1e-9  # 10 steps in 20 ms


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.job_throughput(1, 4, 2.0) == 2.0


def test_reference_arm_prints_on_rank_zero_only():
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        pass
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(Args(), rank=1)   # other ranks exit without work
    assert buf.getvalue() == ""
