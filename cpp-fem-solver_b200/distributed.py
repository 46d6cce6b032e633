"""Row-partitioned block matrices across ranks, one GPU per rank.

The reference distributes a BlockMatrix by contiguous block rows and runs
BlockMatrix::distributed_matvec over MPI (blockMatrix.hpp:317-437), with the
partitioner of its MPI test (test_BlockMatrix_mpi.cpp:283-354).  Here:

* ``row_range`` / ``owner`` -- the partition: rank p of P owns block rows
  [nbr p / P, nbr (p+1) / P), and block column c belongs to the rank whose
  rows contain c.  (The reference's test takes the owner as c P / nbr, which
  disagrees with its own row split when P does not divide nbr -- with 196
  rows on 3 ranks it assigns row 65 to rank 0 although rank 1 owns it, and
  the owner then indexes outside its rows.)
* ``halo_plan`` -- steps 2-5 of the reference's partitioner: the ghost
  columns (referenced, not owned; sorted, unique), the receive table grouped
  by owner, the request exchange (the reference's MPI_Alltoall(v); here any
  ``exchange`` callable, torch.distributed by default) and the send table.
* ``DistBlockMatrix`` -- one rank's rows on its GPU (a b2s BAIJ handle with
  global columns and its halo, b2s_baij_set_halo).  ``matvec`` packs the rows
  other ranks read, exchanges them with torch.distributed point-to-point
  operations (NCCL between GPUs) while the owned-column blocks are multiplied,
  then adds the ghost-column blocks: the reference's overlap, and its
  arithmetic bit for bit.
* ``DistBlockMatrix.cg`` -- CG with block-Jacobi (the mini-CG of the
  reference's MPI test, test_BlockMatrix_mpi.cpp:160-180) whose dot products
  are local fixed-order reductions summed across ranks in rank order, so every
  rank takes the same steps and the result does not depend on the
  communication library's reduction order.  The reference has no distributed
  Krylov solver (its dots are rank-local); this is the extension its MPI path
  needs.

Preconditioners other than block-Jacobi (IC/ILU triangular solves, the
greedy AMG aggregation, SSOR across colours) do not partition exactly; they
stay single-GPU (or replicas of independent systems).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def row_range(nbr: int, rank: int, nranks: int) -> tuple[int, int]:
    """Block rows [start, end) of `rank` (test_BlockMatrix_mpi.cpp:287-289)."""
    return nbr * rank // nranks, nbr * (rank + 1) // nranks


def owner(cols, nbr: int, nranks: int):
    """Rank whose rows (row_range) contain each block column."""
    starts = np.array([row_range(nbr, p, nranks)[0] for p in range(nranks)], np.int64)
    return np.searchsorted(starts, np.asarray(cols, np.int64), side="right") - 1


@dataclass
class HaloPlan:
    start: int
    end: int
    recv_procs: list = field(default_factory=list)
    recv_cnts: list = field(default_factory=list)
    recv_global: np.ndarray = None  # ghost block columns, grouped by owner, ascending
    send_procs: list = field(default_factory=list)
    send_cnts: list = field(default_factory=list)
    send_local: np.ndarray = None   # owned block rows other ranks read, grouped by destination

    @property
    def n_owned(self) -> int:
        return self.end - self.start

    @property
    def n_ghost(self) -> int:
        return int(len(self.recv_global))


def ghost_requests(local_ci, nbr: int, rank: int, nranks: int):
    """Ghost columns of a rank's rows and the list of them each rank owns."""
    cols = np.unique(np.asarray(local_ci, np.uint32))
    own = owner(cols, nbr, nranks)
    ghosts = cols[own != rank]
    gown = own[own != rank]
    return ghosts, [ghosts[gown == p] for p in range(nranks)]


def halo_plan(local_ci, nbr: int, rank: int, nranks: int, exchange) -> HaloPlan:
    """The halo tables of one rank.  exchange(requests) takes this rank's
    requests (requests[p]: the global rows it reads from rank p) and returns
    the requests every rank sends to it (received[p]: the global rows rank p
    reads from this one) -- the reference's MPI_Alltoall / MPI_Alltoallv."""
    start, end = row_range(nbr, rank, nranks)
    ghosts, requests = ghost_requests(local_ci, nbr, rank, nranks)
    plan = HaloPlan(start, end)
    plan.recv_global = ghosts.astype(np.uint32)
    for p in range(nranks):
        if len(requests[p]):
            plan.recv_procs.append(p)
            plan.recv_cnts.append(int(len(requests[p])))
    received = exchange(requests)
    sends = []
    for p in range(nranks):
        rows = np.asarray(received[p], np.int64)
        if len(rows):
            if rows.min() < start or rows.max() >= end:
                raise ValueError(f"rank {p} requests rows that rank {rank} does not own")
            plan.send_procs.append(p)
            plan.send_cnts.append(int(len(rows)))
            sends.append(rows - start)
    plan.send_local = (np.concatenate(sends) if sends else np.zeros(0, np.int64)).astype(np.uint32)
    return plan


def torch_exchange(group=None):
    """exchange() over torch.distributed (any backend): every rank's request
    lists gathered, each rank keeps the lists addressed to it."""
    import torch.distributed as dist

    def exchange(requests):
        gathered = [None] * dist.get_world_size(group)
        dist.all_gather_object(gathered, [np.asarray(r, np.uint32).tolist() for r in requests], group=group)
        me = dist.get_rank(group)
        return [np.asarray(g[me], np.uint32) for g in gathered]

    return exchange


def local_rows(rp, ci, v, bs: int, start: int, end: int):
    """Block rows [start, end) of a global BAIJ (column numbering kept global)."""
    rp = np.asarray(rp, np.int64)
    a, b = int(rp[start]), int(rp[end])
    lrp = (rp[start:end + 1] - a).astype(np.uint32)
    return lrp, np.asarray(ci[a:b], np.uint32), np.asarray(v[a * bs * bs:b * bs * bs], np.float64)


def diagonal_blocks(lrp, lci, lv, bs: int, start: int):
    """The diagonal block of every local row (block row i meets global column
    start + i), as a block-diagonal BAIJ in local numbering."""
    n = len(lrp) - 1
    bv = bs * bs
    out = np.zeros(n * bv)
    for i in range(n):
        seg = lci[lrp[i]:lrp[i + 1]]
        k = np.searchsorted(seg, start + i)
        if k == len(seg) or seg[k] != start + i:
            raise ValueError(f"block row {start + i} has no diagonal block")
        p = lrp[i] + k
        out[i * bv:(i + 1) * bv] = lv[p * bv:(p + 1) * bv]
    return np.arange(n + 1, dtype=np.uint32), np.arange(n, dtype=np.uint32), out


class GpuHaloOps:
    """The device steps of one rank (b2s C ABI on the context's stream)."""

    def __init__(self, b2s, ctx, bs, plan: HaloPlan, nbr_global, lrp, lci, lv):
        self.b2s, self.ctx, self.bs = b2s, ctx, bs
        self.A = b2s.BAIJ(ctx, bs, plan.n_owned, nbr_global, lrp, lci, lv)
        self.A.set_halo(plan.recv_procs, plan.recv_cnts, plan.recv_global, plan.send_procs, plan.send_cnts,
                        plan.send_local, plan.start)
        drp, dci, dv = diagonal_blocks(lrp, lci, lv, bs, plan.start)
        self.D = b2s.BAIJ(ctx, bs, plan.n_owned, plan.n_owned, drp, dci, dv)
        self.M = b2s.Precond(ctx, self.D, b2s.PC_BJACOBI)

    def pack(self, x, buf):
        self.A.halo_pack_device(x.data_ptr(), buf.data_ptr())

    def owned(self, xf, y):
        self.A.dist_matvec_owned_device(xf.data_ptr(), y.data_ptr())

    def ghost(self, xf, y):
        self.A.dist_matvec_ghost_device(xf.data_ptr(), y.data_ptr())

    def dot(self, a, b) -> float:
        return self.b2s.dot_device(self.ctx, a.numel(), a.data_ptr(), b.data_ptr())

    def precond(self, r, z):
        self.ctx.check(self.b2s.lib().b2s_pc_apply_device(self.ctx.h, self.M.h, self.b2s.C.c_void_p(r.data_ptr()),
                                                          self.b2s.C.c_void_p(z.data_ptr())), "block Jacobi")


class DistBlockMatrix:
    """One rank's block rows of a row-partitioned BAIJ with its halo.

    Built from the global arrays (every rank passes the same ones, as the
    reference's MPI test does) or, with ``local=(lrp, lci, lv)``, from this
    rank's rows alone.  Vectors are torch tensors of this rank's owned
    entries on its device.  The device steps are the GPU ones; the CPU tests
    pass ``make_ops(plan, lrp, lci, lv)`` returning a host stand-in, to check
    the partition and the exchange on gloo ranks."""

    def __init__(self, bs, nbr_global, rp=None, ci=None, v=None, *, rank, nranks, ctx=None, group=None,
                 exchange=None, make_ops=None, local=None, device=None):
        import torch
        self.bs, self.nbr, self.rank, self.nranks, self.group = bs, nbr_global, rank, nranks, group
        start, end = row_range(nbr_global, rank, nranks)
        lrp, lci, lv = local if local is not None else local_rows(rp, ci, v, bs, start, end)
        self.plan = halo_plan(lci, nbr_global, rank, nranks, exchange or torch_exchange(group))
        ops = make_ops(self.plan, lrp, lci, lv) if make_ops is not None else None
        if ops is None:
            import importlib
            b2s = importlib.import_module(__name__.rpartition(".")[0] or "b2s")
            ops = GpuHaloOps(b2s, ctx, bs, self.plan, nbr_global, lrp, lci, lv)
            device = device or torch.device("cuda", ctx.device)
            self.stream = torch.cuda.ExternalStream(b2s.lib().b2s_ctx_stream(ctx.h))
        else:
            self.stream = None
        self.ops = ops
        self.device = device or torch.device("cpu")
        no, ng = self.plan.n_owned * bs, self.plan.n_ghost * bs
        self.x_full = torch.zeros(no + ng, dtype=torch.float64, device=self.device)
        self.send_buf = torch.zeros(max(len(self.plan.send_local) * bs, 1), dtype=torch.float64, device=self.device)

    # -------------------------------------------------------------- streams
    def _on_stream(self):
        import contextlib

        import torch
        return torch.cuda.stream(self.stream) if self.stream is not None else contextlib.nullcontext()

    # -------------------------------------------------------------- exchange
    def _start_exchange(self):
        """Point-to-point sends of the packed rows and receives into the ghost
        region, all posted at once (the reference's MPI_Isend / MPI_Irecv)."""
        import torch.distributed as dist
        ops, bs = [], self.bs
        off = self.plan.n_owned * bs
        for p, c in zip(self.plan.recv_procs, self.plan.recv_cnts):
            ops.append(dist.P2POp(dist.irecv, self.x_full[off:off + c * bs], self._peer(p), self.group))
            off += c * bs
        off = 0
        for p, c in zip(self.plan.send_procs, self.plan.send_cnts):
            ops.append(dist.P2POp(dist.isend, self.send_buf[off:off + c * bs], self._peer(p), self.group))
            off += c * bs
        return dist.batch_isend_irecv(ops) if ops else []

    def _peer(self, p):
        import torch.distributed as dist
        return p if self.group is None else dist.get_global_rank(self.group, p)

    def matvec(self, x):
        """y = A x over the partition (BlockMatrix::distributed_matvec)."""
        import torch
        no = self.plan.n_owned * self.bs
        y = torch.empty(no, dtype=torch.float64, device=self.device)
        with self._on_stream():
            self.x_full[:no].copy_(x)
            self.ops.pack(x, self.send_buf)
            reqs = self._start_exchange()
            self.ops.owned(self.x_full, y)  # overlaps the exchange
            for r in reqs:
                r.wait()
            self.ops.ghost(self.x_full, y)
        return y

    # -------------------------------------------------------------- reductions
    def gsum(self, local: float) -> float:
        """Sum of one value per rank, in rank order (the same on every rank)."""
        import torch
        import torch.distributed as dist
        if self.nranks == 1 and not (dist.is_available() and dist.is_initialized()):
            return float(local)
        t = torch.tensor([local], dtype=torch.float64, device=self.device)
        parts = [torch.empty_like(t) for _ in range(self.nranks)]
        dist.all_gather(parts, t, group=self.group)
        total = 0.0
        for q in parts:
            total += float(q.item())
        return total

    def dot(self, a, b) -> float:
        with self._on_stream():
            return self.gsum(self.ops.dot(a, b))

    # -------------------------------------------------------------- CG
    def cg(self, b, tol=1e-8, maxit=3000):
        """CG with block-Jacobi across the partition (the reference MPI test's
        mini-CG, test_BlockMatrix_mpi.cpp:160-180, with global dots).
        Returns (x_owned, it), it the index of the last iteration run."""
        import torch
        with self._on_stream():
            x = torch.zeros_like(b)
            r = b.clone()
            z = torch.empty_like(b)
            self.ops.precond(r, z)
            p = z.clone()
        rz = self.dot(r, z)
        nb = float(np.sqrt(self.dot(b, b)))
        it = 0
        for it in range(maxit):
            Ap = self.matvec(p)
            alpha = rz / self.dot(p, Ap)
            with self._on_stream():
                x.add_(alpha * p)
                r.sub_(alpha * Ap)
            if np.sqrt(self.dot(r, r)) / nb < tol:
                break
            with self._on_stream():
                self.ops.precond(r, z)
            rz2 = self.dot(r, z)
            beta = rz2 / rz
            with self._on_stream():
                p.mul_(beta).add_(z)
            rz = rz2
        return x, it
