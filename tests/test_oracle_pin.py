"""Pins the C restatement (oracle/b2s_oracle.c) against the reference library
compiled from its own sources (oracle/_ref/libref.so), at one OpenMP thread,
bit for bit.  The reference ships no golden vectors, so the compiled reference
is the pin; every GPU parity test then compares against the restatement."""
import numpy as np
import pytest

import problems as P

METHODS = {0: ["none", "diag", "ic", "ilu", "ssor", "cg", "Jacobi", "incomplete_cholesky"],
           1: ["none", "diag", "ilu", "ic", "ssor"],
           2: ["none", "diag", "ilu", "ic", "ssor"]}


def both(orc, ref, n, rp, ci, v):
    return orc.csr(n, n, rp, ci, v), ref.csr(n, n, rp, ci, v)


@pytest.mark.parametrize("gen", ["poisson", "convdiff", "random"])
def test_csr_spmv_and_coo(orc, ref, gen):
    n, rp, ci, v = {"poisson": lambda: P.poisson2d(17), "convdiff": lambda: P.convdiff2d(15),
                    "random": lambda: P.random_spd(300, 0.02, 7)}[gen]()
    rows = np.repeat(np.arange(n), np.diff(rp))
    # COO with shuffled order, an explicit zero and a split duplicate
    perm = np.random.default_rng(1).permutation(len(v))
    R, Cc, V = rows[perm], ci[perm], v[perm].copy()
    R = np.concatenate([R, [0, 0]]); Cc = np.concatenate([Cc, [ci[0], n - 1]]); V = np.concatenate([V, [0.5, 0.0]])
    Ao, Ar = orc.csr_from_coo(n, n, V, R, Cc), ref.csr_from_coo(n, n, V, R, Cc)
    for a, b in zip(Ao.export(), Ar.export()):
        assert np.array_equal(a, b)
    x = np.random.default_rng(2).uniform(-1, 1, n)
    assert np.array_equal(orc.spmv(Ao, x), ref.spmv(Ar, x))
    assert orc.dot(x, x) == ref.dot(x, x)
    for a, b in zip(orc.transpose(Ao).export(), ref.transpose(Ar).export()):
        assert np.array_equal(a, b)
    for a, b in zip(orc.matmul(Ao, Ao).export(), ref.matmul(Ar, Ar).export()):
        assert np.array_equal(a, b)


def test_reference_spgemm_single_touch_defect(orc, ref):
    """The reference's SMatrix::operator* (array.cpp:2336-2447) shares its
    marker array between the symbolic and the numeric pass without resetting
    it, so in the numeric pass a column that only one row of the product
    touches still carries that row's mark from the symbolic pass and is
    skipped: its slot keeps (column 0, value 0).  At one thread a diagonal
    times a diagonal loses every entry.  The restatement (and the library)
    keep them; every other product is equal bit for bit."""
    n = 6
    rp = np.arange(n + 1, dtype=np.uint32)
    ci = rp[:-1].copy()
    d = np.arange(1.0, n + 1)
    Cr = ref.matmul(ref.csr(n, n, rp, ci, d), ref.csr(n, n, rp, ci, d)).export()
    Co = orc.matmul(orc.csr(n, n, rp, ci, d), orc.csr(n, n, rp, ci, d)).export()
    assert np.array_equal(Cr[0], rp) and not Cr[1].any() and not Cr[2].any()
    assert np.array_equal(Co[1], ci) and np.array_equal(Co[2], d * d)


def test_stationary_loop(orc):
    """The restatement of SMatrix::amg's loop (array.cpp:4534-4563) with an
    identity preconditioner is Richardson's iteration x += (b - A x): on a
    matrix scaled so that I - A is a contraction it stops at the first index
    whose true residual passes, and it = maxit - 1 when the loop runs out."""
    n, rp, ci, v = P.poisson2d(6)
    v = v / 8.0
    Ao = orc.csr(n, n, rp, ci, v)
    b = np.linspace(-1.0, 1.0, n)
    x, it = orc.solve_pc(Ao, 5, None, b, 1e-6, 10000)
    xs, rel = np.zeros(n), []
    for k in range(it + 1):
        r = b - orc.spmv(Ao, xs)
        rel.append(np.sqrt(np.sum(r * r)) / np.sqrt(np.sum(b * b)))
        if rel[-1] < 1e-6:
            break
        xs = xs + r
    assert len(rel) == it + 1 and rel[-1] < 1e-6 and min(rel[:-1]) >= 1e-6
    assert np.array_equal(x, xs)
    x5, it5 = orc.solve_pc(Ao, 5, None, b, 1e-30, 5)
    assert it5 == 4


def test_coo_out_of_range(orc, ref):
    import oracle
    for lib in (orc, ref):
        with pytest.raises(oracle.OracleError):
            lib.csr_from_coo(2, 2, [1.0], [2], [0])


@pytest.mark.parametrize("method", [0, 1, 2])
def test_solvers_bit_exact(orc, ref, method):
    n, rp, ci, v = P.poisson2d(20) if method == 0 else P.convdiff2d(18)
    Ao, Ar = both(orc, ref, n, rp, ci, v)
    b = np.random.default_rng(3).uniform(-1, 1, n)
    for p in METHODS[method]:
        if method != 0 and p in ("ic",):
            continue
        xo, io = orc.solve(Ao, method, p, b, 1e-8, 3000, 20)
        xr, ir = ref.solve(Ar, method, p, b, 1e-8, 3000, 20)
        assert io == ir, (method, p)
        assert np.array_equal(xo, xr), (method, p)


def test_pcg_edge_cases(orc, ref):
    import oracle
    n, rp, ci, v = P.poisson2d(6)
    Ao, Ar = both(orc, ref, n, rp, ci, v)
    z = np.zeros(n)
    for lib, A in ((orc, Ao), (ref, Ar)):
        x, it = lib.solve(A, 0, "bogus", z)          # b = 0 returns before the name is checked
        assert it == 0 and not x.any()
        with pytest.raises(oracle.OracleError) as e:
            lib.solve(A, 0, "bogus", np.ones(n))
        assert e.value.status == 1
        x, it = lib.solve(A, 0, "none", np.ones(n), tol=1e-8, maxit=3)  # max_iter reached
        assert it == 2
    # a negative diagonal: diag preconditioner throws runtime_error in both
    v2 = v.copy(); v2[0] = -4.0
    Ao2, Ar2 = both(orc, ref, n, rp, ci, v2)
    for lib, A in ((orc, Ao2), (ref, Ar2)):
        with pytest.raises(oracle.OracleError) as e:
            lib.solve(A, 0, "diag", np.ones(n))
        assert e.value.status == 2


@pytest.mark.parametrize("kind", ["diag", "ic0", "ilu0", "ssor"])
def test_preconditioner_apply_and_factors(orc, ref, kind):
    n, rp, ci, v = P.random_spd(400, 0.015, 11)
    Ao, Ar = both(orc, ref, n, rp, ci, v)
    po, pr = orc.pc(Ao, kind), ref.pc(Ar, kind)
    r = np.random.default_rng(4).uniform(-1, 1, n)
    assert np.array_equal(po.apply(r), pr.apply(r))
    if kind == "ic0":
        eo, er = orc.ic0_export(po), ref.ic0_export(pr)
        assert all(np.array_equal(eo[k], er[k]) for k in eo)
    if kind == "ilu0":
        eo, er = orc.ilu0_export(po), ref.ilu0_export(pr)
        assert all(np.array_equal(eo[k], er[k]) for k in eo)
    if kind == "ssor":
        co, cr = orc.colour_export(po), ref.redblack(Ar)
        assert co[0] == cr[0]
        assert all(np.array_equal(a, b) for a, b in zip(co[1:], cr[1:]))


def test_colouring_bipartite_and_greedy(orc, ref):
    for n, rp, ci, v in (P.poisson2d(12), P.random_spd(200, 0.03, 5)):
        Ao, Ar = both(orc, ref, n, rp, ci, v)
        co, cr = orc.colour_export(orc.pc(Ao, "ssor")), ref.redblack(Ar)
        assert co[0] == cr[0]
        assert all(np.array_equal(a, b) for a, b in zip(co[1:], cr[1:]))


@pytest.mark.parametrize("bs", [1, 3])
def test_block_path_bit_exact(orc, ref, bs):
    n, rp, ci, v = P.make_test_scalar(9, 3) if bs == 3 else P.poisson2d(20)
    Ao, Ar = both(orc, ref, n, rp, ci, v)
    nb = n // bs
    Bo, Br = orc.blk_condense(bs, Ao, nb, nb), ref.blk_condense(bs, Ar, nb, nb)
    for a, b in zip(Bo.export(), Br.export()):
        assert np.array_equal(a, b)
    x = P.drand(np.arange(n))
    assert np.array_equal(orc.blk_matvec(Bo, x), ref.blk_matvec(Br, x))
    for a, b in zip(orc.blk_transpose(Bo).export(), ref.blk_transpose(Br).export()):
        assert np.array_equal(a, b)
    po, pr = orc.blk_pc(Bo, "ilu0"), ref.blk_pc(Br, "ilu0")
    assert np.array_equal(po.apply(x), pr.apply(x))
    eo, er = orc.blk_ilu0_export(po, bs), ref.blk_ilu0_export(pr, bs)
    assert all(np.array_equal(eo[k], er[k]) for k in eo)
    for p in ("none", "blockjacobi", "blockilu"):
        xo, io = orc.blk_gmres(Bo, x, p, 1e-8, 500, 30)
        xr, ir = ref.blk_gmres(Br, x, p, 1e-8, 500, 30)
        assert io == ir and np.array_equal(xo, xr)


@pytest.mark.parametrize("bs,N", [(1, 24), (3, 12)])
def test_sa_amg_hierarchy_bit_exact(orc, ref, bs, N):
    n, rp, ci, v = P.make_test_scalar(N, 3) if bs == 3 else P.poisson2d(N)
    Ao, Ar = both(orc, ref, n, rp, ci, v)
    nb = n // bs
    Bo, Br = orc.blk_condense(bs, Ao, nb, nb), ref.blk_condense(bs, Ar, nb, nb)
    po, pr = orc.blk_pc(Bo, "amg"), ref.blk_pc(Br, "amg")
    lo, lr = orc.amg_export(po, bs), ref.amg_export(pr, bs)
    assert len(lo) == len(lr) >= 2
    for a, c in zip(lo, lr):
        assert set(a) == set(c)
        for k in a:
            assert np.array_equal(a[k], c[k]), k
    r = P.drand(np.arange(n) + 5)
    assert np.array_equal(po.apply(r), pr.apply(r))


def test_levels_restatement(orc):
    n, rp, ci, v = P.poisson2d(9)
    lev, nl = orc.levels(n, rp, ci, upper=False)
    assert nl == 2 * 9 - 1
    i, j = np.divmod(np.arange(n), 9)
    assert np.array_equal(lev, i + j)
    levu, nlu = orc.levels(n, rp, ci, upper=True)
    assert nlu == nl and np.array_equal(levu, (8 - i) + (8 - j))


def _sor_restated(n, rp, ci, v, b, omega, tol, maxit):
    """SMatrix::sor (array.cpp:3843-3945) restated row by row in Python floats."""
    diag = np.zeros(n)
    for i in range(n):
        for p in range(rp[i], rp[i + 1]):
            if ci[p] == i:
                diag[i] = v[p]
    x = [0.0] * n
    normb = float(np.sqrt(sum(bi * bi for bi in b)))
    it_end = 0
    for it in range(maxit):
        for i in range(n):
            sigma = float(b[i])
            for p in range(rp[i], rp[i + 1]):
                j = int(ci[p])
                if j != i:
                    sigma -= float(v[p]) * x[j]
            x[i] += omega * (sigma / float(diag[i]) - x[i])
        err = 0.0
        for i in range(n):
            ri = float(b[i])
            for p in range(rp[i], rp[i + 1]):
                ri -= float(v[p]) * x[int(ci[p])]
            err += ri * ri
        it_end = it
        if np.sqrt(err) / normb < tol:
            break
    return np.array(x), it_end


def test_sor_reference_pinned(ref):
    """The compiled reference's SOR against a row-by-row restatement (one
    OpenMP thread, so the residual sums in row order): same iterates, same
    count."""
    import problems as P
    n, rp, ci, v = P.convdiff2d(8)
    b = np.random.default_rng(4).uniform(-1, 1, n)
    x, it = ref.sor(ref.csr(n, n, rp, ci, v), b, 1.3, 1e-9, 500)
    xr, itr = _sor_restated(n, rp, ci, v, b, 1.3, 1e-9, 500)
    assert it == itr and np.array_equal(x, xr)


def schur_restated(orc, Ao_pc, So_pc, scale, B, Bt, nv, r):
    """make_schur_preconditioner's seven steps (blockMatrix.hpp:637-685)."""
    ru, rp = r[:nv], r[nv:]
    wu = Ao_pc.apply(ru)
    rpm = orc.spmv(B, wu) - rp
    zp = rpm.copy() if So_pc is None else scale * So_pc.apply(rpm)
    rum = ru - orc.spmv(Bt, zp)
    return np.concatenate([Ao_pc.apply(rum), zp])


def test_schur_composition_pinned(orc, ref):
    """The reference's Schur composition (compiled) equals its seven steps over
    the restatement's ILU(0), SpMVs and the identity, bit for bit."""
    K, A, B, Bt = P.stokes1d(60)
    nv, np_ = A[0], B[0]
    Ar, Br, Btr = (ref.csr(*m) for m in (A, B, Bt))
    Ao, Bo, Bto = (orc.csr(*m) for m in (A, B, Bt))
    pc = ref.schur(nv, np_, Br, Btr, ref.pc(Ar, "ilu0"))
    r = P.drand(np.arange(nv + np_) + 3)
    assert np.array_equal(pc.apply(r), schur_restated(orc, orc.pc(Ao, "ilu0"), None, 1.0, Bo, Bto, nv, r))
