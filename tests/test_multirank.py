"""The N > 1 path of bench.py on CPU: world_size-2 gloo ranks (replicas only --
each rank proves its own seeded frames; the only collective is the max of the
step time over ranks), and the reference arm runs on rank 0 alone."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        ms = [12.5, 20.0][rank]
        m = bench.max_over_ranks(ms, world, "cpu")
        out[rank] = (m, bench.job_throughput(64, m, world), bench.replica_seed(rank))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_max_step_time_and_distinct_frames():
    world = 2
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 20.0
    assert res[0][1] == res[1][1] == 2 * 64 / 0.020
    assert res[0][2] != res[1][2]


def test_reference_arm_runs_on_rank_zero_only():
    sys.path.insert(0, ROOT)
    import bench

    class A:
        steps, warmup = 1, 3
    buf = io.StringIO()
    with redirect_stdout(buf):
        assert bench.reference_arm(A(), rank=1, world=2) is None
    assert buf.getvalue() == ""
