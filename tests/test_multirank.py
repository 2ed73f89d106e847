"""The N > 1 path of bench.py on CPU: two gloo ranks agree on the slowest
rank's time, the whole-job rate counts every rank's units, and under the
reference arm only rank 0 does work (the others return at once)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    got = bench.max_over_ranks(10.0 + 5.0 * rank, ws, "cpu")
    assert bench.dist_env() == (ws, rank, rank)
    # reference arm: ranks other than 0 return without timing anything
    if rank != 0:
        class A:
            steps, warmup, gpus = 1, 1, ws
        bench.run_reference_arm(A)
    out.put((rank, got, bench.whole_job_rate(1000.0, ws, got)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, got, rate in res:
        assert got == 15.0                      # the slower rank's time
        assert rate == pytest.approx(2 * 1000.0 / 15e-3)
