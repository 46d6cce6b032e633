"""The device steps of the row-partitioned BAIJ (b2s_baij_set_halo, the pack,
owned-column and ghost-column kernels of distributed_matvec,
blockMatrix.hpp:317-437) on one GPU.

P ranks are emulated one after another in one process: each rank's rows get
their own handle, halo and buffers, and the exchange becomes device copies
from the senders' packed buffers into the receivers' ghost regions.  No kernel
waits on another rank's, so this is safe on one GPU and shows the data path
that NCCL drives between GPUs.  The products equal the oracle's restatement
of the reference's MPI branch bit for bit, and the serial matvec within 1e-12
(the reference's T5, test_BlockMatrix_mpi.cpp:397-405).  A one-rank NCCL
process group runs the distributed CG end to end on the device."""
import os

import numpy as np
import pytest
import torch

import problems as P

pytestmark = pytest.mark.gpu


def global_baij(orc, N, bs):
    n, rp, ci, v = P.make_test_scalar(N, bs)
    Bo = orc.blk_condense(bs, orc.csr(n, n, rp, ci, v), n // bs, n // bs)
    return (n // bs,) + Bo.export() + (Bo,)


def emulated_exchange(bci_all, nbr, nranks):
    """exchange() for rank r computed from every rank's requests (what the
    all-to-all would deliver)."""
    from b2s.distributed import ghost_requests
    reqs = [ghost_requests(c, nbr, r, nranks)[1] for r, c in enumerate(bci_all)]
    return lambda r: (lambda requests: [reqs[p][r] for p in range(nranks)])


@pytest.mark.parametrize("bs,nranks", [(3, 2), (3, 3), (1, 4), (2, 3)])
def test_emulated_ranks_matvec(b2s, ctx, orc, bs, nranks):
    from b2s.distributed import DistBlockMatrix, local_rows, row_range
    nbr, brp, bci, bv, Bo = global_baij(orc, 17, bs)
    locs = [local_rows(brp, bci, bv, bs, *row_range(nbr, r, nranks)) for r in range(nranks)]
    ex = emulated_exchange([l[1] for l in locs], nbr, nranks)
    D = [DistBlockMatrix(bs, nbr, brp, bci, bv, rank=r, nranks=nranks, ctx=ctx, exchange=ex(r))
         for r in range(nranks)]
    xg = P.drand(np.arange(nbr * bs) + 5)
    dev = torch.device("cuda", 0)
    ys = []
    with D[0]._on_stream():
        for r, d in enumerate(D):
            s, e = row_range(nbr, r, nranks)
            x = torch.from_numpy(xg[s * bs:e * bs].copy()).to(dev)
            d.x_full[:len(x)].copy_(x)
            d.ops.pack(x, d.send_buf)
        for r, d in enumerate(D):  # the exchange: senders' packed rows -> receivers' ghost regions
            off = d.plan.n_owned * bs
            for p, c in zip(d.plan.recv_procs, d.plan.recv_cnts):
                sp = D[p].plan
                k = sp.send_procs.index(r)
                so = sum(sp.send_cnts[:k]) * bs
                d.x_full[off:off + c * bs].copy_(D[p].send_buf[so:so + c * bs])
                off += c * bs
        for r, d in enumerate(D):
            y = torch.empty(d.plan.n_owned * bs, dtype=torch.float64, device=dev)
            d.ops.owned(d.x_full, y)
            d.ops.ghost(d.x_full, y)
            ys.append(y)
    torch.cuda.synchronize()
    for r, d in enumerate(D):
        s, e = row_range(nbr, r, nranks)
        lrp, lci, lv = locs[r]
        pos = {int(g): (e - s) + k for k, g in enumerate(d.plan.recv_global)}
        lloc = np.array([g - s if s <= g < e else pos[int(g)] for g in lci], np.uint32)
        xfull = np.concatenate([xg[s * bs:e * bs], xg.reshape(-1, bs)[d.plan.recv_global.astype(np.int64)].reshape(-1)])
        assert np.array_equal(d.x_full.cpu().numpy(), xfull)
        assert np.array_equal(ys[r].cpu().numpy(), orc.blk_dist_matvec(bs, lrp, lloc, lv, e - s, xfull)), r
    yd = np.concatenate([y.cpu().numpy() for y in ys])
    assert np.max(np.abs(yd - orc.blk_matvec(Bo, xg))) < 1e-12


def test_set_halo_rejects_bad_tables(b2s, ctx, orc):
    from b2s.distributed import local_rows, row_range
    nbr, brp, bci, bv, _ = global_baij(orc, 8, 3)
    s, e = row_range(nbr, 0, 2)
    lrp, lci, lv = local_rows(brp, bci, bv, 3, s, e)
    A = b2s.BAIJ(ctx, 3, e - s, nbr, lrp, lci, lv)
    ghosts = sorted({int(g) for g in lci if g >= e})
    with pytest.raises(ValueError):  # a referenced column missing from the ghost list
        A.set_halo([1], [len(ghosts) - 1], ghosts[:-1], [], [], [], s)
    with pytest.raises(ValueError):  # a ghost that this rank owns
        A.set_halo([1], [len(ghosts) + 1], ghosts + [0], [], [], [], s)
    with pytest.raises(ValueError):  # a send row outside the owned rows
        A.set_halo([1], [len(ghosts)], ghosts, [1], [1], [e - s], s)
    A.set_halo([1], [len(ghosts)], ghosts, [1], [2], [0, 1], s)
    assert A.halo_info() == (e - s, len(ghosts), 2)


def test_distributed_cg_one_rank_nccl(b2s, ctx, orc, tmp_path):
    """A one-rank NCCL process group through DistBlockMatrix.cg: the same
    block-Jacobi CG as the single-GPU solver, every step on the device."""
    import torch.distributed as dist
    from b2s.distributed import DistBlockMatrix
    nbr, brp, bci, bv, Bo = global_baij(orc, 24, 3)
    store = dist.FileStore(str(tmp_path / "store"), 1)
    dist.init_process_group("nccl", store=store, rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        D = DistBlockMatrix(3, nbr, brp, bci, bv, rank=0, nranks=1, ctx=ctx)
        b = 1.0 + 0.5 * P.drand(np.arange(nbr * 3) + 7)
        x, it = D.cg(torch.from_numpy(b).to("cuda"), tol=1e-8, maxit=3000)
        torch.cuda.synchronize()
        x = x.cpu().numpy()
    finally:
        dist.destroy_process_group()
    xo, io = orc.blk_solve_pc(Bo, 0, orc.blk_pc(Bo, "jacobi"), b, 1e-8, 3000)
    assert abs(it - (io + 1)) <= 2
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-9
    assert np.linalg.norm(b - orc.blk_matvec(Bo, x)) / np.linalg.norm(b) < 1.5e-8
