"""Smoothed-aggregation AMG on the GPU (blockMatrix.hpp:874-1179).

With amg_ref_coarse=1 the whole hierarchy (aggregates, A, P, D^-1 on every
level) and the V-cycle output equal the restatement bit for bit -- the
restatement itself equals the compiled reference (tests/test_oracle_pin.py).
The library default (parallel aggregation: distance-2 independent roots by a
fixed per-row key, then neighbour assignment; correct pivoted coarse LU;
"amg_mis" in the oracle) and the sequential three-phase rule ("amg_std") are
checked the same way; PCG with them converges where the reference's capped
greedy hierarchy stalls and blows up (32^3).  The reference-rule modes are
parity modes."""
import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def hier_cases(b2s):
    return {
        "bs1_poisson2d": (1,) + P.poisson2d(40),
        "bs3_mpi": (3,) + P.make_test_scalar(20, 3),
        "bs1_poisson3d": (1,) + b2s.gen_poisson3d(14),
    }


MODES = {  # (amg_aggregation, amg_ref_coarse) -> oracle kind
    "reference": (1, 1, "amg"),        # the reference's greedy rule and coarsest elimination
    "ref_exact": (1, 0, "amg_exact"),  # reference greedy rule, correct coarsest LU
    "parallel": (0, 0, "amg_mis"),     # the library default
    "three_phase": (2, 0, "amg_std"),  # sequential three-phase rule
}


@pytest.mark.parametrize("case", ["bs1_poisson2d", "bs3_mpi", "bs1_poisson3d"])
@pytest.mark.parametrize("mode", list(MODES))
def test_amg_hierarchy_and_vcycle(b2s, ctx, orc, case, mode):
    bs, n, rp, ci, v = hier_cases(b2s)[case]
    Ao = orc.csr(n, n, rp, ci, v)
    Bo = orc.blk_condense(bs, Ao, n // bs, n // bs)
    brp, bci, bv = Bo.export()
    B = b2s.BAIJ(ctx, bs, n // bs, n // bs, brp, bci, bv)
    aggm, ref_coarse, okind = MODES[mode]
    M = b2s.Precond(ctx, B, b2s.PC_BSA_AMG, amg_ref_coarse=ref_coarse, amg_aggregation=aggm)
    po = orc.blk_pc(Bo, okind)
    levels = orc.amg_export(po, bs)
    _, nrows, _ = M.export("amg.levels")
    assert list(nrows) == [lv["nrows"] for lv in levels]
    for k, lv in enumerate(levels):
        Arp, Aci, Av = M.export(f"amg.{k}.A")
        assert np.array_equal(Arp, lv["Arp"]) and np.array_equal(Aci, lv["Aci"]) and np.array_equal(Av, lv["Av"]), k
        assert np.array_equal(M.export(f"amg.{k}.dinv")[2], lv["diag_inv"]), k
        if "Prp" in lv:
            Prp, Pci, Pv = M.export(f"amg.{k}.P")
            assert np.array_equal(Prp, lv["Prp"]) and np.array_equal(Pci, lv["Pci"]) and np.array_equal(Pv, lv["Pv"])
            agg = M.export(f"amg.{k}.agg")[1]
            assert np.array_equal(agg.astype(np.int32), orc.amg_aggregates(po, k, lv["nrows"]))
    r = P.drand(np.arange(n) + 5)
    assert np.array_equal(M.apply(r), po.apply(r))


def test_scalar_amg_string_is_sa(b2s, ctx, orc):
    n, rp, ci, v = b2s.gen_poisson3d(16)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    M = b2s.Precond(ctx, A, b2s.pc_kind_from_name(b2s.PCG, "amg"))
    po = orc.pc(orc.csr(n, n, rp, ci, v), "sa_amg_mis")
    r = b2s.uniform(8, n)
    assert np.array_equal(M.apply(r), po.apply(r))


def test_amg_pcg_converges(b2s, ctx, orc):
    n, rp, ci, v = b2s.gen_poisson3d(32)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(0, n)
    M = b2s.Precond(ctx, A, b2s.PC_SA_AMG)
    x, st = b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-10, maxit=500)
    assert st["status"] == 0 and st["relres_true"] < 2e-10
    xo, io = orc.solve_pc(orc.csr(n, n, rp, ci, v), 0, orc.pc(orc.csr(n, n, rp, ci, v), "sa_amg_mis"), b,
                          1e-10, 500)
    assert abs(st["it"] - io) <= 2
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-8


def test_parallel_aggregation_properties(b2s, ctx, orc):
    # aggregate ids are dense (0..nagg-1), repeated builds give the same
    # aggregates, and they equal the oracle's serial restatement
    n, rp, ci, v = b2s.gen_grf_diffusion(96, seed=3)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    aggs = [b2s.Precond(ctx, A, b2s.PC_SA_AMG).export("amg.0.agg")[1] for _ in range(2)]
    assert np.array_equal(aggs[0], aggs[1])
    a = aggs[0].astype(np.int64)
    assert a.min() == 0 and len(np.unique(a)) == a.max() + 1
    po = orc.pc(orc.csr(n, n, rp, ci, v), "sa_amg_mis")
    assert np.array_equal(a.astype(np.int32), orc.amg_aggregates(po, 0, n))


def test_block_amg_elasticity_pcg(b2s, ctx):
    nbr, rp, ci, v = b2s.gen_elasticity_q1(12)
    B = b2s.BAIJ(ctx, 3, nbr, nbr, rp, ci, v)
    b = b2s.uniform(1, 3 * nbr)
    M = b2s.Precond(ctx, B, b2s.PC_BSA_AMG)
    x, st = b2s.solve(ctx, B, b, b2s.PCG, M, tol=1e-8, maxit=2000)
    assert st["status"] == 0 and st["relres_true"] < 2e-8


@pytest.mark.parametrize("case", ["poisson3d", "elasticity"])
def test_amg_fp32_values(b2s, ctx, case):
    """precision=FP32 keeps FP32 copies of A, P, R and D^-1 on every level
    (FP64 vectors and arithmetic): the V-cycle agrees with the FP64 one to
    single-precision accuracy, and PCG reaches the same FP64-verified
    tolerance within a couple of iterations of it."""
    if case == "poisson3d":
        n, rp, ci, v = b2s.gen_poisson3d(32)
        A, kind = b2s.CSR(ctx, n, n, rp, ci, v), b2s.PC_SA_AMG
    else:
        nbr, rp, ci, v = b2s.gen_elasticity_q1(12)
        A, kind, n = b2s.BAIJ(ctx, 3, nbr, nbr, rp, ci, v), b2s.PC_BSA_AMG, 3 * nbr
    M64 = b2s.Precond(ctx, A, kind)
    M32 = b2s.Precond(ctx, A, kind, precision=b2s.FP32)
    r = b2s.uniform(4, n)
    z64, z32 = M64.apply(r), M32.apply(r)
    assert not np.array_equal(z32, z64)
    assert rel(z32, z64) < 1e-5
    b = b2s.uniform(1, n)
    _, s64 = b2s.solve(ctx, A, b, b2s.PCG, M64, tol=1e-8, maxit=2000)
    _, s32 = b2s.solve(ctx, A, b, b2s.PCG, M32, tol=1e-8, maxit=2000)
    assert s32["status"] == 0 and s32["relres_true"] < 2e-8
    assert abs(s32["iterations"] - s64["iterations"]) <= 2


def test_amg_wide_galerkin_rows(b2s, ctx, orc):
    """A row and column that touch every node (weak couplings, so the
    aggregates stay those of the grid) give Galerkin rows with more distinct
    columns than the symbolic product's per-warp hash table holds: the
    product takes the candidate-sort path and the hierarchy still equals the
    restatement bit for bit."""
    n0, rp0, ci0, v0 = P.poisson2d(80)
    rows = [dict(zip(ci0[rp0[i]:rp0[i + 1]].tolist(), v0[rp0[i]:rp0[i + 1]].tolist())) for i in range(n0)]
    for i in range(1, n0):
        w = -1e-3 * (1.0 + (i % 7) / 7.0)
        rows[0][i] = rows[0].get(i, 0.0) + w
        rows[i][0] = rows[i].get(0, 0.0) + w
    rows[0][0] += 2.0 * n0 * 1e-3
    rp, ci, v = [0], [], []
    for r in rows:
        for j in sorted(r):
            ci.append(j)
            v.append(r[j])
        rp.append(len(ci))
    rp, ci, v = np.array(rp, np.uint32), np.array(ci, np.uint32), np.array(v)
    B = b2s.BAIJ(ctx, 1, n0, n0, rp, ci, v)
    Bo = orc.blk_condense(1, orc.csr(n0, n0, rp, ci, v), n0, n0)
    M = b2s.Precond(ctx, B, b2s.PC_BSA_AMG)
    levels = orc.amg_export(orc.blk_pc(Bo, "amg_mis"), 1)
    assert max(np.diff(levels[1]["Arp"])) > 512  # wider than the hash table
    _, nrows, _ = M.export("amg.levels")
    assert list(nrows) == [lv["nrows"] for lv in levels]
    for k, lv in enumerate(levels):
        Arp, Aci, Av = M.export(f"amg.{k}.A")
        assert np.array_equal(Arp, lv["Arp"]) and np.array_equal(Aci, lv["Aci"]) and np.array_equal(Av, lv["Av"]), k


@pytest.mark.parametrize("case", ["poisson2d_48", "poisson3d_16", "maxit"])
def test_stationary_amg(b2s, ctx, orc, case):
    """SMatrix::amg (array.cpp:4534-4563) as B2S_STATIONARY with the SA V-cycle:
    x += V-cycle(b - A x) from x = 0, the true residual checked before every
    correction.  The V-cycle equals the oracle's bit for bit and x is updated
    elementwise, so the iterates are the oracle's bit for bit; only the norm's
    association differs, which could move a stop by one check at most."""
    if case == "poisson3d_16":
        n, rp, ci, v = b2s.gen_poisson3d(16)
    else:
        n, rp, ci, v = P.poisson2d(48)
    tol, maxit = (1e-10, 200) if case != "maxit" else (1e-14, 5)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(11, n)
    M = b2s.Precond(ctx, A, b2s.PC_SA_AMG)
    x, st = b2s.solve(ctx, A, b, b2s.STATIONARY, M, tol=tol, maxit=maxit)
    Ao = orc.csr(n, n, rp, ci, v)
    xo, io = orc.solve_pc(Ao, 5, orc.pc(Ao, "sa_amg_mis"), b, tol, maxit)
    assert st["status"] == 0
    if case == "maxit":
        assert st["it"] == io == maxit - 1 and st["iterations"] == maxit
        assert np.array_equal(x, xo)
    else:
        assert abs(st["it"] - io) <= 1
        if st["it"] == io:
            assert np.array_equal(x, xo)
        assert st["relres_true"] < tol and 0 < st["it"] < maxit
    # the Python mirror of the drop-in call
    Ms = b2s.SMatrix(n, n, v, row_ptr=rp, col_idx=ci)
    xs, its = b2s.SMatrix.amg(Ms, b, tol, maxit)
    assert its == st["it"] and np.array_equal(xs, x)


def test_stationary_zero_rhs_and_maxit0(b2s, ctx):
    n, rp, ci, v = P.poisson2d(16)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    M = b2s.Precond(ctx, A, b2s.PC_SA_AMG)
    x, st = b2s.solve(ctx, A, np.zeros(n), b2s.STATIONARY, M, tol=1e-10, maxit=50)
    assert st["it"] == 0 and not x.any()
    x, st = b2s.solve(ctx, A, b2s.uniform(2, n), b2s.STATIONARY, M, tol=1e-10, maxit=0)
    assert st["it"] == 0 and not x.any()
