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


def test_partition_scenes_balances_and_covers():
    """The batched configuration's scene split: every scene on exactly one
    rank, loads within one scene of each other, the same split everywhere."""
    sys.path.insert(0, ROOT)
    from voxarmps_b200 import config
    _, scenes = config.baseline(4)
    sizes = [len(s["x"]) for s in scenes]
    for ws in (1, 2, 3, 4, 8):
        parts = config.partition_scenes(sizes, ws)
        assert len(parts) == ws
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[k] for k in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)
        assert parts == config.partition_scenes(sizes, ws)
    with pytest.raises(ValueError):
        config.partition_scenes(sizes, 0)


def _split_worker(rank, ws, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    cfg, case, scenes = bench.build_case(0, 4, None, rank, ws)
    n = len(case["x"])
    total = bench.sum_over_ranks(float(n), ws, "cpu")
    out.put((rank, n, int(scenes[2].shape[0]), total))
    dist.barrier()
    dist.destroy_process_group()


def test_batched_scenes_split_over_two_gloo_ranks():
    """bench.py --config 4 under two ranks: each rank builds only its share
    of the 64 scenes, and the whole-job particle count (summed over ranks)
    equals the single-rank batch."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    sys.path.insert(0, ROOT)
    import bench
    _, full, fscenes = bench.build_case(0, 4)
    assert res[0][2] + res[1][2] == int(fscenes[2].shape[0]) == 64
    assert res[0][1] + res[1][1] == len(full["x"])
    for _, _, _, total in res:
        assert total == len(full["x"])
