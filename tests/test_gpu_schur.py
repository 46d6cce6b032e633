"""The Schur-complement saddle-point preconditioner on the device
(b2s_pc_create_schur; make_schur_preconditioner, blockMatrix.hpp:637-685)
against the reference compiled from its sources, with the reference's own
known-answer solves:

* 1-D Stokes, N_vel = 100, 500, 1000, velocity ILU(0), pressure identity,
  GMRES(50): ||x - x_exact|| < 1e-6 (test_BlockMatrix_schur.cpp:88-114);
* 3-D periodic MAC Stokes, velocity ILU(0), pressure identity and
  6.1 x AMG(Lp), GMRES(100) (test_BlockMatrix_schur3d.cpp:137-192), at N = 10
  and 16 (the reference's own block AMG set-up grows faster than linearly and
  needs minutes at its N = 50); the known answer is checked modulo the
  constant-pressure null space of the periodic system.

The apply equals the reference's composition bit for bit: its ILU(0), its
SpMVs, its elementwise differences, and -- for the pressure AMG -- the
library's block AMG in the reference's own rule (capped greedy aggregation,
its coarsest elimination), which equals the reference's V-cycle bit for bit.
GMRES then matches the reference's iteration count within +/-2 and its
solution within 1e-10 (only the dots' association differs).  (For n <= 4000
rows the reference's dots are serial, so its iterates are one association.)"""
import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def parts(b2s, ctx, A, B, Bt):
    return (b2s.CSR(ctx, *A), b2s.CSR(ctx, *B), b2s.CSR(ctx, *Bt))


def ref_amg_pressure(b2s, ctx, ref, Lp):
    """Pressure AMG on Lp: the library's block AMG in the reference's rule, and the reference's own."""
    n = Lp[0]
    Lpb = b2s.BAIJ(ctx, 1, n, n, *Lp[2:])
    Sg = b2s.Precond(ctx, Lpb, b2s.PC_BSA_AMG, amg_aggregation=1, amg_ref_coarse=1)
    Lr = ref.blk_condense(1, ref.csr(*Lp), n, n)
    return Lpb, Sg, ref.blk_pc(Lr, "amg")


@pytest.mark.parametrize("N_vel", [100, 500, 1000])
def test_schur_1d_stokes(b2s, ctx, ref, N_vel):
    K, A, B, Bt = P.stokes1d(N_vel)
    nv, np_ = A[0], B[0]
    Ad, Bd, Btd = parts(b2s, ctx, A, B, Bt)
    Ag = b2s.Precond(ctx, Ad, b2s.PC_ILU0)
    M = b2s.SchurPrecond(ctx, nv, np_, Bd, Btd, Ag)
    Mr = ref.schur(nv, np_, ref.csr(*B), ref.csr(*Bt), ref.pc(ref.csr(*A), "ilu0"))
    r = P.drand(np.arange(nv + np_) + 9)
    assert np.array_equal(M.apply(r), Mr.apply(r))
    Kd = b2s.CSR(ctx, *K)
    xe = P.drand(np.arange(K[0]))
    b = Kd.spmv(xe)
    x, st = b2s.solve(ctx, Kd, b, b2s.GMRES, M, tol=1e-10, maxit=2000, restart=50)
    xr, ir = ref.gmres_pc(ref.csr(*K), Mr, b, 50, 1e-10, 2000)
    assert np.linalg.norm(x - xe) < 1e-6
    assert abs(st["it"] - ir) <= 2, (st["it"], ir)
    assert rel(x, xr) < 1e-10


def known_answer_modulo_pressure_constant(x, xe, nv):
    """The periodic 3-D system is singular (a constant pressure is in the null
    space of K), so x can differ from x_exact by a constant pressure: the
    velocity part and the pressure part up to its mean must match."""
    du = np.linalg.norm(x[:nv] - xe[:nv])
    dp = x[nv:] - xe[nv:]
    return du, np.linalg.norm(dp - dp.mean())


@pytest.mark.parametrize("N", [10, 16])
def test_schur_3d_stokes(b2s, ctx, ref, N):
    """Velocity ILU(0), pressure identity: the apply and GMRES(100) against the
    reference.  The reference's own check (||x - x_exact|| < 1e-6) cannot hold:
    the periodic system is singular and its solve lands a constant pressure
    away from x_exact (||x - x_exact|| = 16 at N = 10 for the reference
    itself), so the known answer is checked modulo that constant.  With the
    pressure AMG in the reference's rule the apply still equals the
    reference's bit for bit; that AMG's coarsest elimination is defective and
    the reference's GMRES with it diverges (1e23 at N = 16), so its solve is
    taken with the library's SA-AMG in test_schur_library_amg_and_graphs."""
    K, A, B, Bt, Lp = P.stokes3d(N)
    nv, np_ = A[0], B[0]
    Ad, Bd, Btd = parts(b2s, ctx, A, B, Bt)
    Ag = b2s.Precond(ctx, Ad, b2s.PC_ILU0)
    Ar = ref.pc(ref.csr(*A), "ilu0")
    Brf, Btrf = ref.csr(*B), ref.csr(*Bt)
    Kd, Kr = b2s.CSR(ctx, *K), ref.csr(*K)
    xe = P.drand(np.arange(K[0]))
    b = Kd.spmv(xe)
    r = P.drand(np.arange(nv + np_) + 9)
    M = b2s.SchurPrecond(ctx, nv, np_, Bd, Btd, Ag)
    Mr = ref.schur(nv, np_, Brf, Btrf, Ar)
    assert np.array_equal(M.apply(r), Mr.apply(r))
    x, st = b2s.solve(ctx, Kd, b, b2s.GMRES, M, tol=1e-10, maxit=2000, restart=100)
    xr, ir = ref.gmres_pc(Kr, Mr, b, 100, 1e-10, 2000)
    assert abs(st["it"] - ir) <= 2, (st["it"], ir)
    assert rel(x, xr) < 1e-10
    du, dp = known_answer_modulo_pressure_constant(x, xe, nv)
    assert du < 1e-6 and dp < 1e-6, (du, dp)
    # pressure AMG in the reference's rule, scaled by 6.1: the same apply as the reference's
    Lpb, Sg, Sr = ref_amg_pressure(b2s, ctx, ref, Lp)
    M2 = b2s.SchurPrecond(ctx, nv, np_, Bd, Btd, Ag, b2s.ScaledPrecond(ctx, Sg, 6.1))
    Mr2 = ref.schur(nv, np_, Brf, Btrf, Ar, Sr, 6.1)
    assert np.array_equal(M2.apply(r), Mr2.apply(r))


def test_schur_library_amg_and_graphs(b2s, ctx):
    """The library's own SA-AMG on the pressure Laplacian (no reference rule):
    the known answer holds, and the whole solve replays from CUDA graphs
    (every part of the composition is device work).  (The scaled pressure
    AMG is not always the better Schur approximation at these sizes: 42
    GMRES steps against the identity's 33 at N = 12; the reference prints
    both counts and asserts neither.)"""
    K, A, B, Bt, Lp = P.stokes3d(12)
    nv, np_ = A[0], B[0]
    Ad, Bd, Btd = parts(b2s, ctx, A, B, Bt)
    Ag = b2s.Precond(ctx, Ad, b2s.PC_ILU0)
    Lpd = b2s.CSR(ctx, *Lp)
    S = b2s.ScaledPrecond(ctx, b2s.Precond(ctx, Lpd, b2s.PC_SA_AMG), 6.1)
    M = b2s.SchurPrecond(ctx, nv, np_, Bd, Btd, Ag, S)
    Kd = b2s.CSR(ctx, *K)
    xe = P.drand(np.arange(K[0]))
    b = Kd.spmv(xe)
    x1, s1 = b2s.solve(ctx, Kd, b, b2s.GMRES, M, tol=1e-10, maxit=2000, restart=100, use_graphs=1)
    x2, s2 = b2s.solve(ctx, Kd, b, b2s.GMRES, M, tol=1e-10, maxit=2000, restart=100, use_graphs=0)
    du, dp = known_answer_modulo_pressure_constant(x1, xe, nv)
    assert du < 1e-6 and dp < 1e-6, (du, dp)
    assert np.array_equal(x1, x2) and s1["it"] == s2["it"]


def test_schur_shape_errors(b2s, ctx):
    K, A, B, Bt = P.stokes1d(20)
    Ad, Bd, Btd = parts(b2s, ctx, A, B, Bt)
    Ag = b2s.Precond(ctx, Ad, b2s.PC_ILU0)
    with pytest.raises(ValueError):
        b2s.SchurPrecond(ctx, A[0], B[0], Btd, Bd, Ag)  # B and B^T swapped
    _, A2, _, _ = P.stokes1d(10)
    with pytest.raises(ValueError):  # a velocity preconditioner of the wrong size
        b2s.SchurPrecond(ctx, A[0], B[0], Bd, Btd, b2s.Precond(ctx, b2s.CSR(ctx, *A2), b2s.PC_DIAG))
