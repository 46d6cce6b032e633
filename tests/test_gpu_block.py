"""Block path on the GPU (blockMatrix.hpp): block ILU(0) factors and applies
bit-exact against the restatement for BS = 1 and 3, block GMRES with the
reference's string table, and the block PCG extension; the elasticity (Q1)
operator with FP32 block-ILU."""
import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def condensed(orc, bs, N):
    n, rp, ci, v = P.make_test_scalar(N, 3) if bs == 3 else P.poisson2d(N)
    Bo = orc.blk_condense(bs, orc.csr(n, n, rp, ci, v), n // bs, n // bs)
    return n, Bo, Bo.export()


@pytest.mark.parametrize("bs", [1, 3])
@pytest.mark.parametrize("trsv", [1, 2])
def test_bilu0_bit_exact(b2s, ctx, orc, bs, trsv):
    n, Bo, (brp, bci, bv) = condensed(orc, bs, 30)
    B = b2s.BAIJ(ctx, bs, n // bs, n // bs, brp, bci, bv)
    M = b2s.Precond(ctx, B, b2s.PC_BILU0, trsv=trsv)
    po = orc.blk_pc(Bo, "ilu0")
    e = orc.blk_ilu0_export(po, bs)
    for what, keys in (("bilu0.L", ("Lrp", "Lci", "Lv")), ("bilu0.U", ("Urp", "Uci", "Uv"))):
        got = M.export(what)
        assert all(np.array_equal(g, e[k]) for g, k in zip(got, keys)), what
    _, ud, inv = M.export("bilu0.inv")
    assert np.array_equal(ud, e["Udiag"]) and np.array_equal(inv, e["inv_diag"])
    r = P.drand(np.arange(n) + 3)
    assert np.array_equal(M.apply(r), po.apply(r))


def _bilu0_factor_equal(M, e):
    for what, keys in (("bilu0.L", ("Lrp", "Lci", "Lv")), ("bilu0.U", ("Urp", "Uci", "Uv"))):
        got = M.export(what)
        assert all(np.array_equal(g, e[k]) for g, k in zip(got, keys)), what
    _, ud, inv = M.export("bilu0.inv")
    assert np.array_equal(ud, e["Udiag"]) and np.array_equal(inv, e["inv_diag"])


def test_bilu0_factor_elasticity_bit_exact(b2s, ctx, orc):
    """27-point block rows (13 lower blocks): the warp-per-row factor with its
    U_JK lookups cached in shared memory gives the reference's factors."""
    nbr, rp, ci, v = b2s.gen_elasticity_q1(6)
    B = b2s.BAIJ(ctx, 3, nbr, nbr, rp, ci, v)
    Bo = orc.blk(3, nbr, nbr, rp, ci, v)
    _bilu0_factor_equal(b2s.Precond(ctx, B, b2s.PC_BILU0), orc.blk_ilu0_export(orc.blk_pc(Bo, "ilu0"), 3))


@pytest.mark.parametrize("bs", [2, 4])
def test_bilu0_factor_wide_rows_bit_exact(b2s, ctx, orc, bs):
    """Rows of up to 40 lower blocks (more than the 32 whose lookups are
    cached): the lookups run inline and the factors still match."""
    nb, w = 96, 40
    rng = np.random.default_rng(11 + bs)
    rp, ci, vals = [0], [], []
    for i in range(nb):
        cols = [j for j in range(max(0, i - w), min(nb, i + 6)) if j == i or rng.random() < 0.85]
        for j in cols:
            blk = rng.uniform(-1.0, 1.0, (bs, bs))
            if j == i:
                blk += np.eye(bs) * (4.0 * w)
            vals.append(blk.ravel())
        ci += cols
        rp.append(len(ci))
    rp, ci, v = np.array(rp, np.uint32), np.array(ci, np.uint32), np.concatenate(vals)
    assert max(int(np.sum(ci[rp[i]:rp[i + 1]] < i)) for i in range(nb)) > 32
    B = b2s.BAIJ(ctx, bs, nb, nb, rp, ci, v)
    Bo = orc.blk(bs, nb, nb, rp, ci, v)
    M = b2s.Precond(ctx, B, b2s.PC_BILU0)
    po = orc.blk_pc(Bo, "ilu0")
    _bilu0_factor_equal(M, orc.blk_ilu0_export(po, bs))
    r = b2s.uniform(3, nb * bs)
    assert np.array_equal(M.apply(r), po.apply(r))


def test_bilu0_elasticity(b2s, ctx, orc):
    nbr, rp, ci, v = b2s.gen_elasticity_q1(8)
    B = b2s.BAIJ(ctx, 3, nbr, nbr, rp, ci, v)
    Bo = orc.blk(3, nbr, nbr, rp, ci, v)
    po = orc.blk_pc(Bo, "ilu0")
    r = b2s.uniform(5, 3 * nbr)
    z64 = b2s.Precond(ctx, B, b2s.PC_BILU0).apply(r)
    assert np.array_equal(z64, po.apply(r))
    z32 = b2s.Precond(ctx, B, b2s.PC_BILU0, precision=b2s.FP32).apply(r)
    assert rel(z32, z64) < 1e-4


@pytest.mark.parametrize("pc", ["none", "blockjacobi", "blockilu"])
def test_block_gmres_strings(b2s, ctx, orc, pc):
    n, Bo, (brp, bci, bv) = condensed(orc, 3, 24)
    B = b2s.BAIJ(ctx, 3, n // 3, n // 3, brp, bci, bv)
    b = 1.0 + 0.5 * P.drand(np.arange(n) + 7)
    kind = b2s.pc_kind_from_name(b2s.BLOCK_GMRES, pc)
    M = b2s.Precond(ctx, B, kind) if kind != b2s.PC_NONE else None
    x, st = b2s.solve(ctx, B, b, b2s.GMRES, M, tol=1e-8, maxit=500, restart=30)
    xo, io = orc.blk_gmres(Bo, b, pc, 1e-8, 500, 30)
    assert abs(st["it"] - io) <= 2 and rel(x, xo) < 1e-9


def test_block_pcg_ilu_vs_jacobi(b2s, ctx, orc):
    """T7 of test_BlockMatrix_mpi.cpp:422-445: block ILU needs no more CG
    iterations than block Jacobi and the true residual is below 1e-6."""
    n, Bo, (brp, bci, bv) = condensed(orc, 3, 64)
    B = b2s.BAIJ(ctx, 3, n // 3, n // 3, brp, bci, bv)
    b = 1.0 + 0.5 * P.drand(np.arange(n) + 7)
    xj, sj = b2s.solve(ctx, B, b, b2s.PCG, b2s.Precond(ctx, B, b2s.PC_BJACOBI), tol=1e-8, maxit=3000)
    xi, si = b2s.solve(ctx, B, b, b2s.PCG, b2s.Precond(ctx, B, b2s.PC_BILU0), tol=1e-8, maxit=3000)
    assert si["iterations"] <= sj["iterations"]
    assert si["relres_true"] < 1e-6 and sj["relres_true"] < 1e-6
    xo, io = orc.blk_solve_pc(Bo, 0, orc.blk_pc(Bo, "ilu0"), b, 1e-8, 3000)
    assert abs(si["it"] - io) <= 2 and rel(xi, xo) < 1e-9


def test_bilu0_missing_diag(b2s, ctx):
    # 2 block rows, second has no diagonal block
    rp = np.array([0, 1, 2], np.uint32)
    ci = np.array([0, 0], np.uint32)
    v = np.tile(np.eye(3).ravel(), 2)
    B = b2s.BAIJ(ctx, 3, 2, 2, rp, ci, v)
    with pytest.raises(RuntimeError) as e:
        b2s.Precond(ctx, B, b2s.PC_BILU0)
    assert e.value.status == b2s.MISSING_DIAG
    v2 = np.concatenate([np.zeros(9), np.eye(3).ravel()])
    B2 = b2s.BAIJ(ctx, 3, 2, 2, np.array([0, 1, 2], np.uint32), np.array([0, 1], np.uint32), v2)
    with pytest.raises(RuntimeError) as e:
        b2s.Precond(ctx, B2, b2s.PC_BILU0)
    assert e.value.status == b2s.SINGULAR_BLOCK
