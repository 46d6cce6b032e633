"""Stand-alone SOR solvers (b2s_sor: SMatrix::sor and SMatrix::sor_rb,
array.cpp:3843-4189) against the compiled reference on the same inputs.
Every row is updated in the reference's order, so the iterates are the same
bits; the stopping test uses a residual norm summed in a different order
(the device's fixed tree vs the reference's loop), so when the two stop at
the same sweep the solutions must be identical, and otherwise they may be
one sweep apart."""
import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu

MATS = {
    "poisson2d": lambda: P.poisson2d(30),           # bipartite: two colours
    "random": lambda: P.random_spd(900, 0.006, 2),  # odd cycles: greedy colours
    "convdiff": lambda: P.convdiff2d(30),           # nonsymmetric values
}


@pytest.mark.parametrize("mat", list(MATS))
@pytest.mark.parametrize("red_black", [False, True])
@pytest.mark.parametrize("omega", [1.0, 1.6])
def test_sor_matches_reference(b2s, ctx, ref, mat, red_black, omega):
    n, rp, ci, v = MATS[mat]()
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(77, n)
    x, st = b2s.sor(ctx, A, b, omega, 1e-8, 3000, red_black)
    xr, itr = ref.sor(ref.csr(n, n, rp, ci, v), b, omega, 1e-8, 3000, red_black)
    assert abs(st["it"] - itr) <= 1, (st["it"], itr)
    if st["it"] == itr:
        assert np.array_equal(x, xr)
    else:
        assert np.linalg.norm(x - xr) <= 1e-6 * np.linalg.norm(xr)
    assert st["relres"] < 1e-8 or st["it"] == 2999


def test_sor_max_iter_and_zero_rhs(b2s, ctx, ref):
    n, rp, ci, v = P.poisson2d(20)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(3, n)
    for rb in (False, True):
        x, st = b2s.sor(ctx, A, b, 1.2, 1e-14, 7, rb)
        xr, itr = ref.sor(ref.csr(n, n, rp, ci, v), b, 1.2, 1e-14, 7, rb)
        assert st["it"] == itr == 6
        assert np.array_equal(x, xr)
        # zero right-hand side: x = 0, it = 0, before the omega check
        x0, s0 = b2s.sor(ctx, A, np.zeros(n), 3.0, 1e-8, 100, rb)
        assert not x0.any() and s0["it"] == 0


def test_sor_errors(b2s, ctx):
    n, rp, ci, v = P.poisson2d(8)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(4, n)
    for rb in (False, True):
        with pytest.raises(ValueError) as e:
            b2s.sor(ctx, A, b, 2.0, 1e-8, 100, rb)
        assert e.value.status == b2s.INVALID_ARG
    rows = np.repeat(np.arange(n), np.diff(rp))
    keep = ~((rows == ci) & (rows == 5))
    rp3 = np.concatenate([[0], np.cumsum(np.bincount(rows[keep], minlength=n))]).astype(np.uint32)
    A3 = b2s.CSR(ctx, n, n, rp3, ci[keep], v[keep])
    for rb in (False, True):
        with pytest.raises(RuntimeError) as e:
            b2s.sor(ctx, A3, b, 1.2, 1e-8, 100, rb)
        assert e.value.status == b2s.MISSING_DIAG
    R = b2s.CSR(ctx, 3, 4, np.array([0, 1, 2, 3], np.uint32), np.array([0, 1, 2], np.uint32), np.ones(3))
    with pytest.raises(ValueError) as e:
        b2s.sor(ctx, R, np.ones(3), 1.2, 1e-8, 10)
    assert e.value.status == b2s.SHAPE
