"""Multicolour SSOR on the GPU (array.cpp:2947-3164): colouring and
renumbering identical to the restatement, apply bit-exact, PCG parity."""
import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mat", ["bipartite", "greedy", "convdiff"])
def test_ssor_colouring_and_apply(b2s, ctx, orc, mat):
    n, rp, ci, v = {"bipartite": lambda: P.poisson2d(45), "greedy": lambda: P.random_spd(1200, 0.005, 9),
                    "convdiff": lambda: P.convdiff2d(40)}[mat]()
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    for omega in (1.2, 0.7):
        M = b2s.Precond(ctx, A, b2s.PC_SSOR, omega=omega)
        po = orc.pc(orc.csr(n, n, rp, ci, v), "ssor", omega)
        nc, cptr, nid, perm, d2 = orc.colour_export(po)
        rp_, ci_, v_ = M.export("ssor.colour")
        assert len(rp_) == nc + 1 and np.array_equal(rp_, cptr)
        assert np.array_equal(ci_, nid) and np.array_equal(v_, d2)
        r = b2s.uniform(41, n)
        assert np.array_equal(M.apply(r), po.apply(r))


def test_ssor_bad_omega(b2s, ctx):
    n, rp, ci, v = P.poisson2d(5)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    for w in (0.0, 2.0, -1.0):
        with pytest.raises(ValueError):
            b2s.Precond(ctx, A, b2s.PC_SSOR, omega=w)


@pytest.mark.parametrize("method", [0, 1, 2])
def test_ssor_solver_parity(b2s, ctx, orc, method):
    n, rp, ci, v = P.poisson2d(40) if method == 0 else P.convdiff2d(40)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(42, n)
    M = b2s.Precond(ctx, A, b2s.PC_SSOR)
    x, st = b2s.solve(ctx, A, b, method, M, tol=1e-8, maxit=2000, restart=30)
    xo, io = orc.solve(orc.csr(n, n, rp, ci, v), method, "ssor", b, 1e-8, 2000, 30)
    assert abs(st["it"] - io) <= 2
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-9
