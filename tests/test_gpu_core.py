"""GPU parity of the core path through the C ABI: SpMV, dot, BAIJ matvec and
the Krylov solvers with identity / diagonal / block-Jacobi preconditioners,
against the C restatement (oracle/b2s_oracle.c).

Tolerances: SpMV and BAIJ matvec rows are summed in the reference's order,
so they must be bit-exact.  Solver results differ from the oracle only by the
association of the dot products (fixed-order tree on the GPU, ascending on
the CPU): iteration counts within +/-2, relative solution difference below
1e-10 unless the problem is ill-conditioned (stated per case)."""
import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def long_row_matrix(n=5000):
    """Row 0 is dense (n nonzeros, > the staging capacity), row 1 empty."""
    R, Cc, V = [], [], []
    for j in range(n):
        R.append(0); Cc.append(j); V.append(1.0 / (j + 1))
    for i in range(2, n):
        R += [i, i]; Cc += [i, i - 1]; V += [2.0, -0.5]
    rp, ci, v = P.coo_to_csr(n, n, R, Cc, V)
    return n, rp, ci, v


@pytest.mark.parametrize("case", ["poisson", "random", "longrow", "tiny", "rect", "big3d", "rows33"])
def test_spmv_bit_exact(b2s, ctx, orc, case):
    # one thread per row below 2^20 rows of <= 32 nonzeros ("poisson", "random",
    # "rect", "tiny"); the warp kernel above ("big3d": 102^3 rows; "longrow",
    # "rows33": a row longer than 32)
    if case == "rect":
        n, m = 300, 500
        rng = np.random.default_rng(0)
        dense = (rng.random((n, m)) < 0.02) * rng.uniform(-1, 1, (n, m))
        rp = np.concatenate([[0], np.cumsum((dense != 0).sum(1))]).astype(np.uint32)
        ci = np.nonzero(dense)[1].astype(np.uint32)
        v = dense[dense != 0]
    else:
        n, rp, ci, v = {"poisson": lambda: P.poisson2d(100), "random": lambda: P.random_spd(3000, 0.004, 1),
                        "big3d": lambda: b2s.gen_poisson3d(102), "rows33": lambda: long_row_matrix(33),
                        "longrow": long_row_matrix, "tiny": lambda: P.coo_to_csr(1, 1, [0], [0], [3.0]) and
                        (1, *P.coo_to_csr(1, 1, [0], [0], [3.0]))}[case]()
        m = n
    A = b2s.CSR(ctx, n, m, rp, ci, v)
    x = np.random.default_rng(5).uniform(-1, 1, m)
    y = A.spmv(x)
    yo = orc.spmv(orc.csr(n, m, rp, ci, v), x)
    assert np.array_equal(y, yo)


def test_dot_deterministic(b2s, ctx):
    rng = np.random.default_rng(1)
    for n in (0, 1, 255, 256, 100003, 3_000_000):
        a, b = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
        d1, d2 = b2s.dot(ctx, a, b), b2s.dot(ctx, a, b)
        assert d1 == d2
        ref = float(np.dot(a, b))
        assert abs(d1 - ref) <= 1e-13 * max(1.0, np.abs(a * b).sum())


@pytest.mark.parametrize("bs", [1, 2, 3, 4])
def test_baij_matvec_bit_exact(b2s, ctx, orc, bs):
    n, rp, ci, v = P.make_test_scalar(40, 3) if bs == 3 else P.poisson2d(60)
    Ao = orc.csr(n, n, rp, ci, v)
    nb = n // bs
    Bo = orc.blk_condense(bs, Ao, nb, nb)
    brp, bci, bv = Bo.export()
    B = b2s.BAIJ(ctx, bs, nb, nb, brp, bci, bv)
    x = P.drand(np.arange(n))
    assert np.array_equal(B.matvec(x), orc.blk_matvec(Bo, x))


@pytest.mark.parametrize("bs", [2, 3, 4])
def test_baij_matvec_irregular(b2s, ctx, orc, bs):
    # ragged block rows: empty rows, single blocks and rows of 100+ blocks,
    # which span several passes of the warp kernel
    rng = np.random.default_rng(bs)
    nb = 700
    lens = rng.integers(0, 12, nb)
    lens[::97] = 0
    lens[5] = 150
    lens[400] = 90
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint32)
    ci = np.concatenate([np.sort(rng.choice(nb, size=k, replace=False)) for k in lens]).astype(np.uint32)
    v = rng.uniform(-1, 1, len(ci) * bs * bs)
    B = b2s.BAIJ(ctx, bs, nb, nb, rp, ci, v)
    Bo = orc.blk(bs, nb, nb, rp, ci, v)
    x = rng.uniform(-1, 1, nb * bs)
    assert np.array_equal(B.matvec(x), orc.blk_matvec(Bo, x))


def test_baij_elasticity_matvec(b2s, ctx, orc):
    nbr, rp, ci, v = b2s.gen_elasticity_q1(10)
    B = b2s.BAIJ(ctx, 3, nbr, nbr, rp, ci, v)
    Bo = orc.blk(3, nbr, nbr, rp, ci, v)
    x = b2s.uniform(3, 3 * nbr)
    assert np.array_equal(B.matvec(x), orc.blk_matvec(Bo, x))


SOLVER_CASES = [
    (b"pcg", 0, "none"), (b"pcg", 0, "diag"), (b"pcg", 0, "cg"),
    (b"bicgstab", 1, "none"), (b"bicgstab", 1, "diag"),
    (b"gmres", 2, "none"), (b"gmres", 2, "diag"),
]


@pytest.mark.parametrize("name,method,pc", SOLVER_CASES)
def test_solver_parity(b2s, ctx, orc, name, method, pc):
    n, rp, ci, v = P.poisson2d(48) if method == 0 else P.convdiff2d(48)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(11, n)
    kind = b2s.pc_kind_from_name(method, pc)
    M = b2s.Precond(ctx, A, kind) if kind != b2s.PC_NONE else None
    x, st = b2s.solve(ctx, A, b, method, M, tol=1e-8, maxit=3000, restart=20)
    xo, io = orc.solve(orc.csr(n, n, rp, ci, v), method, pc, b, 1e-8, 3000, 20)
    assert st["status"] == 0
    assert abs(st["it"] - io) <= 2, (st["it"], io)
    assert st["relres_true"] < 1e-8 * 1.5
    assert rel(x, xo) < 1e-9, rel(x, xo)


def test_pcg_maxit_and_zero_rhs(b2s, ctx, orc):
    n, rp, ci, v = P.poisson2d(30)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    x, st = b2s.solve(ctx, A, np.zeros(n), b2s.PCG, None, tol=1e-8)
    assert st["it"] == 0 and not x.any()
    b = b2s.uniform(1, n)
    x, st = b2s.solve(ctx, A, b, b2s.PCG, None, tol=1e-12, maxit=5)
    xo, io = orc.solve(orc.csr(n, n, rp, ci, v), 0, "none", b, 1e-12, 5)
    assert st["it"] == io == 4
    assert rel(x, xo) < 1e-12


def test_pcg_not_spd_raises(b2s, ctx):
    n, rp, ci, v = P.poisson2d(10)
    v = v.copy()
    rows = np.repeat(np.arange(n), np.diff(rp))
    v[(rows == ci) & (rows == 3)] = -4.0
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    with pytest.raises(RuntimeError):
        b2s.Precond(ctx, A, b2s.PC_DIAG)
    S = b2s.SMatrix(n, n, v, row_ptr=rp, col_idx=ci)
    with pytest.raises(RuntimeError):
        b2s.SMatrix.pcg(S, np.ones(n), "diag", 1e-8, 100)
    with pytest.raises(ValueError):
        b2s.SMatrix.pcg(S, np.ones(n + 1), "none")
    with pytest.raises(ValueError):
        b2s.SMatrix.pcg(S, np.ones(n), "bogus")


def test_smatrix_mirror(b2s, orc):
    n, rp, ci, v = P.poisson2d(25)
    rows = np.repeat(np.arange(n), np.diff(rp))
    S = b2s.SMatrix(n, n, v, rows, ci)
    assert np.array_equal(S.row_ptr(), rp) and np.array_equal(S.col_idx(), ci)
    b = b2s.uniform(2, n)
    x, it = b2s.SMatrix.pcg(S, b, "jacobi", 1e-8, 2000)
    xo, io = orc.solve(orc.csr(n, n, rp, ci, v), 0, "jacobi", b, 1e-8, 2000)
    assert abs(it - io) <= 2 and rel(x, xo) < 1e-9
    assert np.array_equal(b2s.SMatrix.spmv(S, b), orc.spmv(orc.csr(n, n, rp, ci, v), b))


def test_block_gmres_bjacobi(b2s, ctx, orc):
    n, rp, ci, v = P.make_test_scalar(20, 3)
    Bo = orc.blk_condense(3, orc.csr(n, n, rp, ci, v), n // 3, n // 3)
    brp, bci, bv = Bo.export()
    B = b2s.BAIJ(ctx, 3, n // 3, n // 3, brp, bci, bv)
    b = 1.0 + 0.5 * P.drand(np.arange(n) + 7)
    M = b2s.Precond(ctx, B, b2s.PC_BJACOBI)
    x, st = b2s.solve(ctx, B, b, b2s.GMRES, M, tol=1e-8, maxit=500, restart=30)
    xo, io = orc.blk_gmres(Bo, b, "blockjacobi", 1e-8, 500, 30)
    assert abs(st["it"] - io) <= 2 and rel(x, xo) < 1e-9
    x2, st2 = b2s.solve(ctx, B, b, b2s.PCG, M, tol=1e-8, maxit=500)
    assert st2["relres_true"] < 1e-8 * 1.5


def test_host_preconditioner(b2s, ctx, orc):
    n, rp, ci, v = P.poisson2d(20)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    d = v[np.repeat(np.arange(n), np.diff(rp)) == ci]
    M = b2s.HostPrecond(ctx, n, lambda r: r / d)
    b = b2s.uniform(4, n)
    x, st = b2s.solve(ctx, A, b, b2s.GMRES, M, tol=1e-8, maxit=500, restart=10, use_graphs=0)
    xo, io = orc.solve(orc.csr(n, n, rp, ci, v), 2, "diag", b, 1e-8, 500, 10)
    assert abs(st["it"] - io) <= 2 and rel(x, xo) < 1e-9


def test_graphs_match_eager(b2s, ctx):
    n, rp, ci, v = P.poisson2d(40)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(9, n)
    M = b2s.Precond(ctx, A, b2s.PC_DIAG)
    x1, s1 = b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-8, use_graphs=1, check_every=8)
    x2, s2 = b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-8, use_graphs=0, check_every=3)
    assert np.array_equal(x1, x2) and s1["it"] == s2["it"]


@pytest.mark.parametrize("flexible", [False, True])
def test_gmres_cgs2(b2s, ctx, orc, flexible):
    """Classical Gram-Schmidt twice is a different algorithm from the
    reference's MGS (the same Krylov space, other rounding), so it is held to
    accuracy, not to the reference's iterates: the same iteration count within
    +/-2, and an error against the FP64 solution (rtol 1e-13) no larger than
    twice the reference MGS solve's own error at the same tolerance."""
    n, rp, ci, v = P.convdiff2d(60)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(13, n)
    M = b2s.Precond(ctx, A, b2s.PC_ILU0)
    method = b2s.FGMRES if flexible else b2s.GMRES
    x, st = b2s.solve(ctx, A, b, method, M, tol=1e-8, maxit=2000, restart=30, orth=b2s.ORTH_CGS2)
    Ao = orc.csr(n, n, rp, ci, v)
    xo, io = orc.solve(Ao, 2, "ilu", b, 1e-8, 2000, 30)
    xt, _ = orc.solve(Ao, 2, "ilu", b, 1e-13, 2000, 30)
    assert abs(st["it"] - io) <= 2
    assert rel(x, xt) <= 2 * rel(xo, xt) + 1e-13, (rel(x, xt), rel(xo, xt))
    assert st["relres_true"] < 2e-8


def test_fgmres_fp32_refinement(b2s, ctx):
    """FP32 ILU(0) inside FP64 FGMRES with iterative refinement reaches 1e-10."""
    n, rp, ci, v = b2s.gen_convdiff3d(24)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(14, n)
    M = b2s.Precond(ctx, A, b2s.PC_ILU0, precision=b2s.FP32)
    x, st = b2s.solve(ctx, A, b, b2s.FGMRES, M, tol=1e-10, maxit=500, restart=30, ir_steps=5, ir_inner_tol=1e-6)
    assert st["relres_true"] < 1e-10
    r = b - A.spmv(x)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-10


def rect_random(n, m, density, seed):
    rng = np.random.default_rng(seed)
    dense = (rng.random((n, m)) < density) * rng.uniform(-1, 1, (n, m))
    rp = np.concatenate([[0], np.cumsum((dense != 0).sum(1))]).astype(np.uint32)
    return rp, np.nonzero(dense)[1].astype(np.uint32), dense[dense != 0]


@pytest.mark.parametrize("case", ["poisson_sq", "rect", "wide", "diag"])
def test_csr_matmul_transpose(b2s, ctx, orc, ref, case):
    """C = A B and A^T on the device (b2s_csr_matmul / b2s_csr_transpose) equal
    the restatement bit for bit: sorted columns, each entry summed in the
    reference's order.  Where every product column is touched by two or more
    rows the compiled reference gives the same arrays; "diag" is a product
    whose columns are each touched by one row, where the reference's marker
    array (not reset between its passes) drops them (tested on the CPU in
    test_oracle_pin.py::test_reference_spgemm_single_touch_defect)."""
    if case == "poisson_sq":
        n, rp, ci, v = P.poisson2d(40)
        a, b = (n, n, rp, ci, v), (n, n, rp, ci, v)
    elif case == "rect":
        a = (300, 500) + rect_random(300, 500, 0.02, 1)
        b = (500, 200) + rect_random(500, 200, 0.03, 2)
    elif case == "wide":  # product rows wider than the symbolic hash table (512 columns)
        a = (64, 64) + rect_random(64, 64, 0.5, 3)
        b = (64, 2000) + rect_random(64, 2000, 0.5, 4)
    else:
        n = 1000
        rp = np.arange(n + 1, dtype=np.uint32)
        d = np.linspace(1.0, 2.0, n)
        a = b = (n, n, rp, rp[:-1].copy(), d)
    A, B = b2s.CSR(ctx, *a), b2s.CSR(ctx, *b)
    C = A.matmul(B)
    Ao, Bo = orc.csr(*a), orc.csr(*b)
    Co = orc.matmul(Ao, Bo).export()
    assert np.array_equal(C.rp, Co[0]) and np.array_equal(C.ci, Co[1]) and np.array_equal(C.v, Co[2])
    if case != "diag":
        Cr = ref.matmul(ref.csr(*a), ref.csr(*b)).export()
        assert all(np.array_equal(x, y) for x, y in zip(Co, Cr))
    T = A.transpose()
    To = orc.transpose(Ao).export()
    assert (T.n, T.m) == (a[1], a[0])
    assert np.array_equal(T.rp, To[0]) and np.array_equal(T.ci, To[1]) and np.array_equal(T.v, To[2])
    Tr = ref.transpose(ref.csr(*a)).export()
    assert all(np.array_equal(x, y) for x, y in zip(To, Tr))
    # the product is a usable operator: its SpMV equals A (B x)
    x = np.random.default_rng(6).uniform(-1, 1, b[1])
    assert rel(C.spmv(x), A.spmv(B.spmv(x))) < 1e-13


def test_csr_matmul_shape_error(b2s, ctx):
    n, rp, ci, v = P.poisson2d(8)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    B = b2s.CSR(ctx, 3, 3, np.zeros(4, np.uint32), np.zeros(0, np.uint32), np.zeros(0))
    with pytest.raises(b2s.B2SInvalidArgument):
        A.matmul(B)
    M = b2s.SMatrix(n, n, v, row_ptr=rp, col_idx=ci)
    with pytest.raises(ValueError):
        M * b2s.SMatrix(3, 3, np.zeros(0), row_ptr=np.zeros(4, np.uint32), col_idx=np.zeros(0, np.uint32))
    P2 = M * M
    assert P2.rows() == n and np.array_equal(M.transpose().col_idx(), ci)
