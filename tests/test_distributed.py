"""Row-partitioned BAIJ across ranks on CPU (gloo, world sizes 2 and 3):
the halo plan of the reference's MPI partitioner (test_BlockMatrix_mpi.cpp:
283-354), the exchange over torch.distributed point-to-point operations, and
distributed CG with dots summed across ranks.

The device steps (pack, owned-column and ghost-column matvec, block-Jacobi)
are replaced by a host stand-in built on the oracle's restatement of
BlockMatrix::distributed_matvec (blockMatrix.hpp:351-437); the GPU kernels
themselves are checked against the same restatement in
test_gpu_distributed.py.  Checks, as the reference's T5: every rank's
receive table equals the matching send table of its peer, the gathered
distributed product equals the restatement over each rank's rows bit for bit
and the serial matvec within 1e-12, and distributed CG reaches the serial
block-Jacobi CG's solution."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class OracleOps:
    """Host stand-in for the device steps of one rank (test only)."""

    def __init__(self, orc, bs, plan, lrp, lci, lv):
        self.orc, self.bs, self.no = orc, bs, plan.n_owned
        pos = {int(g): plan.n_owned + k for k, g in enumerate(plan.recv_global)}
        self.rp, self.v = lrp, lv
        self.lci = np.array([g - plan.start if plan.start <= g < plan.end else pos[int(g)] for g in lci], np.uint32)
        self.send = plan.send_local.astype(np.int64)
        from b2s.distributed import diagonal_blocks
        drp, dci, dv = diagonal_blocks(lrp, lci, lv, bs, plan.start)
        self.D = orc.blk(bs, plan.n_owned, plan.n_owned, drp, dci, dv)
        self.M = orc.blk_pc(self.D, "jacobi")

    def pack(self, x, buf):
        xv = x.numpy().reshape(-1, self.bs)
        if len(self.send):
            buf[:len(self.send) * self.bs] = torch.from_numpy(xv[self.send].reshape(-1).copy())

    def owned(self, xf, y):
        x = xf.numpy().copy()
        x[self.no * self.bs:] = 0.0  # the owned pass reads no ghost
        y[:] = torch.from_numpy(self.orc.blk_dist_matvec(self.bs, self.rp, self.lci, self.v, self.no, x))

    def ghost(self, xf, y):
        y[:] = torch.from_numpy(self.orc.blk_dist_matvec(self.bs, self.rp, self.lci, self.v, self.no, xf.numpy()))

    def dot(self, a, b):
        return float(self.orc.dot(a.numpy(), b.numpy()))

    def precond(self, r, z):
        z[:] = torch.from_numpy(self.M.apply(r.numpy()))


def worker(rank, world, port, N, out):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import conftest
    conftest.load_b2s()
    import oracle
    import problems as P
    from b2s.distributed import DistBlockMatrix, local_rows, row_range
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        orc = oracle.Orc()
        bs = 3
        n, rp, ci, v = P.make_test_scalar(N, bs)
        Bo = orc.blk_condense(bs, orc.csr(n, n, rp, ci, v), n // bs, n // bs)
        brp, bci, bv = Bo.export()
        nbr = n // bs
        D = DistBlockMatrix(bs, nbr, brp, bci, bv, rank=rank, nranks=world,
                            make_ops=lambda plan, a, b, c: OracleOps(orc, bs, plan, a, b, c))
        start, end = row_range(nbr, rank, world)
        plans = [None] * world
        dist.all_gather_object(plans, (D.plan.start, D.plan.recv_procs, D.plan.recv_cnts, D.plan.recv_global.tolist(),
                                       D.plan.send_procs, D.plan.send_cnts, D.plan.send_local.tolist()))
        # T5: the distributed product against the serial one and the restatement
        xg = P.drand(np.arange(n) + 5)
        y = D.matvec(torch.from_numpy(xg[start * bs:end * bs].copy()))
        ys = [None] * world
        dist.all_gather_object(ys, y.numpy())
        yd = np.concatenate(ys)
        # CG with block Jacobi across the partition
        bg = 1.0 + 0.5 * P.drand(np.arange(n) + 7)
        x, it = D.cg(torch.from_numpy(bg[start * bs:end * bs].copy()), tol=1e-8, maxit=3000)
        xs = [None] * world
        dist.all_gather_object(xs, x.numpy())
        if rank == 0:
            out.put(("ok", plans, yd, np.concatenate(xs), it))
    except Exception as e:  # reported to the parent
        import traceback
        out.put(("error", traceback.format_exc(), None, None, None))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_distributed_halo_and_cg(b2s, orc, world):
    import problems as P
    from b2s.distributed import local_rows, row_range
    N, bs = 14, 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, N, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        res = q.get(timeout=240)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert res[0] == "ok", res[1]
    _, plans, yd, xd, it = res
    assert all(p.exitcode == 0 for p in procs)
    n, rp, ci, v = P.make_test_scalar(N, bs)
    Bo = orc.blk_condense(bs, orc.csr(n, n, rp, ci, v), n // bs, n // bs)
    brp, bci, bv = Bo.export()
    nbr = n // bs
    # receive tables of every rank match the send tables of its peers
    for p in range(world):
        start_p, rprocs, rcnts, rglob = plans[p][0], plans[p][1], plans[p][2], plans[p][3]
        off = 0
        for q_, c in zip(rprocs, rcnts):
            sprocs, scnts, sloc, start_q = plans[q_][4], plans[q_][5], plans[q_][6], plans[q_][0]
            k = sprocs.index(p)
            so = sum(scnts[:k])
            assert [g - start_q for g in rglob[off:off + c]] == sloc[so:so + scnts[k]]
            off += c
        _, lci, _ = local_rows(brp, bci, bv, bs, *row_range(nbr, p, world))
        s, e = row_range(nbr, p, world)
        ghosts = sorted({int(g) for g in lci if not (s <= g < e)})
        assert rglob == ghosts
    # the product: the restatement over each rank's rows (bit for bit), the serial matvec (T5: 1e-12)
    xg = P.drand(np.arange(n) + 5)
    parts = []
    for p in range(world):
        s, e = row_range(nbr, p, world)
        lrp, lci, lv = local_rows(brp, bci, bv, bs, s, e)
        glob = np.asarray(plans[p][3], np.int64)
        pos = {int(g): (e - s) + k for k, g in enumerate(glob)}
        lloc = np.array([g - s if s <= g < e else pos[int(g)] for g in lci], np.uint32)
        xfull = np.concatenate([xg[s * bs:e * bs], xg.reshape(-1, bs)[glob].reshape(-1)])
        parts.append(orc.blk_dist_matvec(bs, lrp, lloc, lv, e - s, xfull))
    assert np.array_equal(yd, np.concatenate(parts))
    assert np.max(np.abs(yd - orc.blk_matvec(Bo, xg))) < 1e-12
    # CG: the serial block-Jacobi PCG's solution and iteration count
    bg = 1.0 + 0.5 * P.drand(np.arange(n) + 7)
    xo, io = orc.blk_solve_pc(Bo, 0, orc.blk_pc(Bo, "jacobi"), bg, 1e-8, 3000)
    r = bg - orc.blk_matvec(Bo, xd)
    assert np.linalg.norm(r) / np.linalg.norm(bg) < 1.5e-8
    assert abs(it - (io + 1)) <= 2, (it, io)
    assert np.linalg.norm(xd - xo) / np.linalg.norm(xo) < 1e-9


def replica_worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        seeds = bench.replica_seeds(rank, 25)
        # each replica's own time; the job's time is the largest
        got = bench.max_over_ranks(10.0 + rank, torch.device("cpu"))
        allseeds = [None] * world
        dist.all_gather_object(allseeds, seeds)
        out.put((rank, got, allseeds))
    finally:
        dist.destroy_process_group()


def test_replica_harness_two_ranks():
    """bench.py's replicas on two gloo ranks: disjoint seed ranges (rank 0 on
    the held-out seeds 2000+) and the time reduced to the maximum on every
    rank."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=replica_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    for rank, got, allseeds in res:
        assert got == 11.0
        assert allseeds[0][0] == 2000 and not set(allseeds[0]) & set(allseeds[1])


def test_owner_matches_row_split(b2s):
    """Every block column's owner is the rank whose row range holds it, for
    process counts that do and do not divide the row count."""
    from b2s.distributed import owner, row_range
    for nbr in (1, 7, 196, 1000):
        for P_ in (1, 2, 3, 5, 8):
            own = owner(np.arange(nbr), nbr, P_)
            for p in range(P_):
                s, e = row_range(nbr, p, P_)
                assert np.all(own[s:e] == p)
