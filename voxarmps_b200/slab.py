"""One scene split between several contexts: slab decomposition along x.

The reference advances one scene in one process (VoxarMPS/VoxarMPS/main.cu:
1027-1363).  Here each rank -- one process per GPU under torchrun, or one
thread per context in ``LocalComm`` -- owns the particles of one slab of the
scene, x in [edges[r], edges[r + 1]), and holds ghost copies of the other
ranks' particles within ``halo`` of its slab.  Per step:

1. the slab edges split the particles into equal counts (every rank computes
   the same edges from an all-reduced histogram-free rule: the quantiles of
   the gathered x, exchanged once per step);
2. every rank sends each other rank its owned particles that lie within the
   halo of that rank's slab (all fields carried between steps); local
   particles are ordered by global id, so cells order them as the single
   scene does and every owned row's neighbour sums run in the same order;
3. the stages run on owned and ghost particles alike (a ghost near the
   halo's outer edge gets wrong values, which reach no owned particle: the
   halo covers one step's chain of neighbour dependencies, 2 re_l + 2 re_s);
4. the PPE is one Jacobi-PCG over the scene: each rank assembles and
   iterates on its owned unknown rows (ghost rows are columns only), the
   ghost entries of the initial guess and of the search direction are
   exchanged before each product, and the dot products are summed over the
   ranks (``Comm.allreduce_sum``); after the solve the ghosts receive their
   owners' pressures (PHATCALC and the gradient read them);
5. the owned particles' states are read back; ownership follows x at the
   next step's edges, which migrates particles across slab faces.

Exchanges go through a ``Comm``: ``TorchComm`` over torch.distributed (NCCL
between GPUs, gloo on CPU; host buffers) or ``LocalComm`` for contexts in one
process.  Nothing here waits inside a kernel: every exchange is a host step
between two launches.  The PPE's dot products are summed per rank, then over
the ranks, so the solution differs from the single context's in rounding
(both meet the same relative residual); the explicit stages of owned rows
are the single context's, bit for bit, when their neighbourhoods are
complete.
"""
from __future__ import annotations

import threading

import numpy as np

# fields carried from one step to the next (besides ptype and the global id):
# the state, the previous step's pressure and its minimum (PREDICTION's
# explicit pressure part), p^(n-1) and the corrected velocities (SPS and the
# collision read them, walls keep theirs)
CARRIED = ("x", "y", "z", "u", "v", "w", "p", "pnew", "phat", "pold", "un", "vn", "wn")


# ---- communicators ----------------------------------------------------------

class Comm:
    """What the decomposition needs from a communicator."""

    rank = 0
    size = 1

    def allreduce_sum(self, v: np.ndarray) -> np.ndarray:
        raise NotImplementedError

    def allreduce_max(self, v: np.ndarray) -> np.ndarray:
        raise NotImplementedError

    def alltoallv(self, sends: list) -> list:
        """sends[r]: a 1-D float64 array for rank r; returns what every rank
        sent to this one (index = source rank)."""
        raise NotImplementedError

    def allgatherv(self, v: np.ndarray) -> list:
        return self.alltoallv([v] * self.size)


class LocalComm(Comm):
    """Ranks as threads of one process (contexts on one GPU or several):
    collectives meet at a barrier; the data moves through shared lists."""

    class World:
        def __init__(self, size: int):
            self.size = size
            self.barrier = threading.Barrier(size)
            self.box = [None] * size

    def __init__(self, world: "LocalComm.World", rank: int):
        self.w = world
        self.rank = rank
        self.size = world.size

    def _share(self, item):
        self.w.barrier.wait()
        self.w.box[self.rank] = item
        self.w.barrier.wait()
        out = list(self.w.box)
        self.w.barrier.wait()
        return out

    def allreduce_sum(self, v):
        # a fixed order over the ranks: every rank gets the same bits
        parts = self._share(np.array(v, np.float64))
        acc = np.zeros_like(parts[0])
        for p in parts:
            acc = acc + p
        return acc

    def allreduce_max(self, v):
        parts = self._share(np.array(v, np.float64))
        return np.max(np.stack(parts), axis=0)

    def alltoallv(self, sends):
        table = self._share([np.array(s, np.float64) for s in sends])
        return [table[src][self.rank] for src in range(self.size)]


class TorchComm(Comm):
    """torch.distributed (already initialised): gloo or NCCL.  Host arrays are
    moved through tensors on `device`; sums run in rank order (all-gather,
    then a fixed-order sum) so that every rank gets the same bits."""

    def __init__(self, device: str = "cpu"):
        import torch.distributed as dist
        self.dist = dist
        self.rank = dist.get_rank()
        self.size = dist.get_world_size()
        self.device = device

    def _t(self, a):
        import torch
        return torch.as_tensor(np.ascontiguousarray(a, np.float64), device=self.device)

    def allreduce_sum(self, v):
        import torch
        t = self._t(v)
        parts = [torch.empty_like(t) for _ in range(self.size)]
        self.dist.all_gather(parts, t)
        acc = parts[0].clone()
        for p in parts[1:]:
            acc += p
        return acc.cpu().numpy()

    def allreduce_max(self, v):
        t = self._t(v)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return t.cpu().numpy()

    def alltoallv(self, sends):
        import torch
        counts = self._t([len(s) for s in sends])
        allc = [torch.empty_like(counts) for _ in range(self.size)]
        self.dist.all_gather(allc, counts)
        recv_n = [int(allc[src][self.rank].item()) for src in range(self.size)]
        width = max(1, int(max(int(c.max().item()) for c in allc)))
        out_t = [torch.zeros(width, dtype=torch.float64, device=self.device)
                 for _ in range(self.size)]
        in_t = []
        for s in sends:
            t = torch.zeros(width, dtype=torch.float64, device=self.device)
            if len(s):
                t[:len(s)] = self._t(s)
            in_t.append(t)
        self.dist.all_to_all(out_t, in_t) if self.dist.get_backend() == "nccl" else \
            self._gloo_alltoall(out_t, in_t)
        return [out_t[src][:recv_n[src]].cpu().numpy() for src in range(self.size)]

    def _gloo_alltoall(self, out_t, in_t):
        # pairwise exchange: lower rank sends first (gloo has no all_to_all)
        out_t[self.rank].copy_(in_t[self.rank])
        for peer in range(self.size):
            if peer == self.rank:
                continue
            if self.rank < peer:
                self.dist.send(in_t[peer], peer)
                self.dist.recv(out_t[peer], peer)
            else:
                self.dist.recv(out_t[peer], peer)
                self.dist.send(in_t[peer], peer)


# ---- the decomposition (host logic only) -------------------------------------

def halo_width(cfg: dict) -> float:
    """Distance over which one step's neighbour dependencies reach: the
    Laplacian radius twice (prediction, then the PPE row) and the PND radius
    twice (n* and PHATCALC / the gradient), plus one spacing of slack."""
    slack = cfg["delta"] if cfg["dim"] == 3 else 0.0
    return 2 * (cfg["re_l"] + slack) + 2 * (cfg["re_s"] + slack) + cfg["l0"]


def slab_edges(x_all: np.ndarray, size: int) -> np.ndarray:
    """Edges of `size` slabs with equal particle counts (edges[0] = -inf,
    edges[size] = +inf): the midpoints between the sorted x at the count
    quantiles."""
    xs = np.sort(np.asarray(x_all, np.float64))
    edges = np.empty(size + 1)
    edges[0], edges[size] = -np.inf, np.inf
    n = len(xs)
    for r in range(1, size):
        k = (n * r) // size
        edges[r] = 0.5 * (xs[k - 1] + xs[k]) if 0 < k < n else xs[min(max(k, 0), n - 1)]
    return edges


def owners(x: np.ndarray, edges: np.ndarray) -> np.ndarray:
    """Rank owning each x (slab r: edges[r] <= x < edges[r + 1])."""
    return np.searchsorted(edges, np.asarray(x, np.float64), side="right") - 1


def ghost_targets(x: np.ndarray, edges: np.ndarray, halo: float, me: int) -> list:
    """For particles owned by `me`, the other ranks that need a ghost copy of
    each (x within halo of their slab): a list over ranks of index arrays."""
    size = len(edges) - 1
    out = []
    for r in range(size):
        if r == me:
            out.append(np.zeros(0, np.int64))
            continue
        lo, hi = edges[r] - halo, edges[r + 1] + halo
        out.append(np.nonzero((x >= lo) & (x < hi))[0])
    return out


# ---- a rank ------------------------------------------------------------------

class SlabRank:
    """This rank's share of one scene.  `cfg` is the whole scene's
    configuration (its box and PMAX: every rank uses the same cell grids);
    `gid`, `ptype` and the CARRIED fields are the particles this rank owns at
    the start (any split works: the first step redistributes them)."""

    def __init__(self, comm: Comm, cfg: dict, gid, ptype, fields: dict, device: int = 0,
                 solver_factory=None):
        from . import Solver
        self.comm = comm
        self.cfg = dict(cfg)
        self.dev = device
        self.make = solver_factory or (lambda c: Solver(c, device=device))
        self.halo = halo_width(self.cfg)
        self.gid = np.asarray(gid, np.int64)
        self.ptype = np.asarray(ptype, np.int32)
        self.f = {k: np.asarray(fields.get(k, np.zeros(len(self.gid))), np.float64).copy()
                  for k in CARRIED}
        self.n0 = None
        self.s = None
        self.last = {}

    # -- exchanges ------------------------------------------------------------
    def _pack(self, idx):
        cols = [self.gid[idx].astype(np.float64), self.ptype[idx].astype(np.float64)]
        cols += [self.f[k][idx] for k in CARRIED]
        return np.stack(cols, axis=1).reshape(-1) if len(idx) else np.zeros(0)

    @staticmethod
    def _unpack(buf):
        w = 2 + len(CARRIED)
        a = np.asarray(buf, np.float64).reshape(-1, w)
        return (a[:, 0].astype(np.int64), a[:, 1].astype(np.int32),
                {k: a[:, 2 + i].copy() for i, k in enumerate(CARRIED)})

    def _migrate(self, edges):
        """Owned particles to the rank whose slab holds their x."""
        own = owners(self.f["x"], edges)
        sends = [self._pack(np.nonzero(own == r)[0]) for r in range(self.comm.size)]
        got = self.comm.alltoallv(sends)
        parts = [self._unpack(g) for g in got if len(g)]
        if parts:
            self.gid = np.concatenate([p[0] for p in parts])
            self.ptype = np.concatenate([p[1] for p in parts])
            self.f = {k: np.concatenate([p[2][k] for p in parts]) for k in CARRIED}
        else:
            self.gid = np.zeros(0, np.int64)
            self.ptype = np.zeros(0, np.int32)
            self.f = {k: np.zeros(0) for k in CARRIED}
        order = np.argsort(self.gid, kind="stable")
        self.gid, self.ptype = self.gid[order], self.ptype[order]
        self.f = {k: v[order] for k, v in self.f.items()}

    def _build_local(self, edges):
        """Owned particles plus ghosts, ordered by global id; the exchange
        plan for ghost values (rows to send per rank, rows to receive)."""
        tgt = ghost_targets(self.f["x"], edges, self.halo, self.comm.rank)
        got = self.comm.alltoallv([self._pack(t) for t in tgt])
        g_gid, g_pt, g_f, g_src = [self.gid], [self.ptype], {k: [self.f[k]] for k in CARRIED}, \
            [np.full(len(self.gid), self.comm.rank)]
        for src, buf in enumerate(got):
            if not len(buf):
                continue
            a, b, c = self._unpack(buf)
            g_gid.append(a)
            g_pt.append(b)
            for k in CARRIED:
                g_f[k].append(c[k])
            g_src.append(np.full(len(a), src))
        gid = np.concatenate(g_gid)
        order = np.argsort(gid, kind="stable")
        self.lgid = gid[order]
        self.lpt = np.concatenate(g_pt)[order]
        self.lf = {k: np.concatenate(v)[order] for k, v in g_f.items()}
        self.lsrc = np.concatenate(g_src)[order]  # owner rank of each local particle
        self.lown = (self.lsrc == self.comm.rank).astype(np.int32)
        pos = {int(g): i for i, g in enumerate(self.lgid)}
        # rows this rank sends (its owned ones that are ghosts elsewhere), in
        # global-id order, and the rows its ghosts fill, per source rank
        self.send_rows = [np.array([pos[int(g)] for g in np.sort(self.gid[t])], np.int32)
                          for t in tgt]
        self.recv_rows = [np.nonzero(self.lsrc == r)[0].astype(np.int32) if r != self.comm.rank
                          else np.zeros(0, np.int32) for r in range(self.comm.size)]

    def exchange_ghosts(self, field: str):
        """Ghost entries of `field` receive their owners' values."""
        s = self.s
        sends = [s.get_rows(field, rows) if len(rows) else np.zeros(0) for rows in self.send_rows]
        got = self.comm.alltoallv(sends)
        for src, vals in enumerate(got):
            rows = self.recv_rows[src]
            if len(rows):
                s.set_rows(field, rows, vals)

    # -- one step ---------------------------------------------------------------
    def _setup(self):
        x_all = np.concatenate(self.comm.allgatherv(self.f["x"]))
        edges = slab_edges(x_all, self.comm.size)
        self._migrate(edges)
        self._build_local(edges)
        case = {"dim": self.cfg["dim"], "ptype": self.lpt,
                **{k: self.lf[k] for k in ("x", "y", "z", "u", "v", "w", "p")}}
        if self.s is not None:
            self.s.close()
        s = self.s = self.make(self.cfg)
        s.upload(case)
        s.init()  # lists and a local n0, replaced by the scene's below
        if self.n0 is None:
            # the scene's n0 (main.cu:964-1012, the largest PND of the first
            # state): a ghost lacks neighbours beyond the halo, so its PND is
            # never above its true value, and the largest over all contexts
            # is the scene's
            self.n0 = self.comm.allreduce_max(np.array([s.scalar("n0_s"), s.scalar("n0_l")]))
        s.set_n0(float(self.n0[0]), float(self.n0[1]))
        for k in ("pnew", "phat", "pold", "un", "vn") + (("wn",) if self.cfg["dim"] == 3 else ()):
            s.set(k, self.lf[k])
        s.set_owned(self.lown)
        return s

    def _ppe(self, s):
        cfg = self.cfg
        s.ppe_assemble()
        self.exchange_ghosts("pnew")  # the initial guess on the ghost rows
        bb, rz, rr = self.comm.allreduce_sum(s.dcg_start())
        tol2 = cfg["cg_tol"] ** 2
        it = 0
        done = bb == 0.0 or rr <= tol2 * bb
        while not done and it < cfg["cg_max"]:
            self.exchange_ghosts("cg_p")
            ps = float(self.comm.allreduce_sum(np.array([s.dcg_spmv()]))[0])
            alpha = rz / ps
            rz_new, rr = self.comm.allreduce_sum(s.dcg_update(alpha))
            it += 1
            if rr <= tol2 * bb or not np.isfinite(rr) or it >= cfg["cg_max"]:
                break
            s.dcg_direction(rz_new / rz)
            rz = rz_new
        relres = float(np.sqrt(rr / bb)) if bb > 0 else 0.0
        status = s.dcg_finish(it, relres, float(bb))
        self.exchange_ghosts("pnew")  # the owners' solved pressures
        self.last = {"cg_iters": it, "cg_relres": relres}
        return status

    def step(self) -> int:
        """One time step of the scene (main.cu:1036-1337); returns this rank's
        MPS_ERR_* bits."""
        cfg = self.cfg
        s = self._setup()
        st = 0
        if cfg["method"] != 3 and not cfg["ppe_at_predicted"]:
            st |= s.pnd()
        st |= s.neighbors()
        if cfg["turb"]:
            st |= s.sps()
        st |= s.vfraction()
        st |= s.viscosity()
        st |= s.predict()
        st |= s.pnd_star()
        if cfg["method"] != 3:
            st |= s.bcon()
            st |= self._ppe(s)
        else:
            s.pressure()
        st |= s.phat()
        st |= s.pressure_gradient()
        st |= s.integrate()
        st |= s.collision()
        st |= s.commit()
        # the owned particles' states for the next step
        own_rows = np.nonzero(self.lown == 1)[0]
        for k in CARRIED:
            if cfg["dim"] == 2 and k in ("z", "w", "wn"):
                self.f[k] = np.zeros(len(own_rows))
                continue
            self.f[k] = s.get(k)[own_rows]
        self.gid = self.lgid[own_rows]
        self.ptype = self.lpt[own_rows]
        return st

    def gather(self, field: str):
        """(global ids, values) of this rank's owned particles."""
        return self.gid.copy(), self.f[field].copy()

    def close(self):
        if self.s is not None:
            self.s.close()
            self.s = None
