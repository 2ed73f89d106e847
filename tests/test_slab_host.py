"""Host logic of the slab decomposition (voxarmps_b200/slab.py) on two gloo
ranks, no GPU: slab edges, migration of owned particles to the rank whose
slab holds them, the ghost sets within the halo, and the ghost-value
exchange plan (a stand-in context holding one value per local particle
takes the place of the GPU context; the product always drives a real one).
Also the in-process communicator's collectives."""
import os
import socket
import threading

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from voxarmps_b200 import slab


class ArrayContext:
    """Stand-in for a context: one double per local particle per field."""

    def __init__(self, values):
        self.v = {"cg_p": np.array(values, np.float64)}

    def get_rows(self, field, rows):
        return self.v[field][np.asarray(rows)]

    def set_rows(self, field, rows, vals):
        self.v[field][np.asarray(rows)] = vals


def scene(n=400, seed=3):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, 1.0, n)
    return {"x": x, "y": rng.uniform(0.0, 0.5, n), "gid": np.arange(n)}


def check_rank(rank, size, comm, sc, halo):
    cfg = {"dim": 2, "re_s": 0.021, "re_l": 0.04, "l0": 0.01, "delta": 0.002}
    # rank r starts with every size-th particle (any split works)
    mine = np.arange(rank, len(sc["x"]), size)
    fields = {k: np.zeros(len(mine)) for k in slab.CARRIED}
    fields["x"], fields["y"] = sc["x"][mine], sc["y"][mine]
    fields["p"] = sc["gid"][mine].astype(float)  # a tag to follow the particles
    r = slab.SlabRank(comm, cfg, sc["gid"][mine], np.ones(len(mine), np.int32), fields)
    r.halo = halo
    x_all = np.concatenate(comm.allgatherv(r.f["x"]))
    edges = slab.slab_edges(x_all, size)
    r._migrate(edges)
    # owned: exactly the particles of this slab, each carrying its own tag
    want = np.nonzero(slab.owners(sc["x"], edges) == rank)[0]
    assert np.array_equal(r.gid, want)
    assert np.array_equal(r.f["p"], want.astype(float))
    r._build_local(edges)
    lo, hi = edges[rank] - halo, edges[rank + 1] + halo
    want_local = np.nonzero((sc["x"] >= lo) & (sc["x"] < hi))[0]
    assert np.array_equal(r.lgid, want_local)  # owned + ghosts, by global id
    assert np.array_equal(r.lown == 1, np.isin(r.lgid, want))
    # ghost exchange: ghosts start wrong and must receive their owners' values
    r.s = ArrayContext(np.where(r.lown == 1, r.lgid * 10.0, -1.0))
    r.exchange_ghosts("cg_p")
    assert np.array_equal(r.s.v["cg_p"], r.lgid * 10.0)
    # the sums every rank gets are the same bits
    tot = comm.allreduce_sum(np.array([float(len(r.gid)), 0.1 * (rank + 1)]))
    assert tot[0] == len(sc["x"])
    return True


def _worker(rank, size, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        ok = check_rank(rank, size, slab.TorchComm("cpu"), scene(), halo=0.13)
        q.put((rank, ok, None))
    except Exception as e:  # report to the parent
        q.put((rank, False, repr(e)))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_migrate_ghost_and_exchange():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    for rank, ok, err in res:
        assert ok, (rank, err)


@pytest.mark.parametrize("size", [1, 3])
def test_local_comm_ranks(size):
    world = slab.LocalComm.World(size)
    out, errs = [None] * size, []

    def run(r):
        try:
            out[r] = check_rank(r, size, slab.LocalComm(world, r), scene(), halo=0.13)
        except Exception as e:
            errs.append(repr(e))
            world.barrier.abort()

    th = [threading.Thread(target=run, args=(r,)) for r in range(size)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=60)
    assert not errs, errs
    assert all(out)


def test_slab_edges_balance_counts():
    x = np.random.default_rng(0).uniform(0, 1, 1001)
    for size in (2, 3, 8):
        e = slab.slab_edges(x, size)
        counts = np.bincount(slab.owners(x, e), minlength=size)
        assert counts.sum() == len(x) and counts.max() - counts.min() <= 2
