"""Learned IC(0): the GPU forward / backward kernels against PyTorch CPU
autograd of the same network (tests/gnn_ref.py), the untrained network equal
to IC(0), SPD-ness of the corrected factor, and the weight file round trip."""
import os

import numpy as np
import pytest

import problems as P

pytestmark = pytest.mark.gpu


def system(b2s, N=24, seed=3):
    n, rp, ci, v = b2s.gen_grf_diffusion(N, seed=seed, corr=0.2)
    return n, rp, ci, v


def test_untrained_is_ic0(b2s, ctx):
    n, rp, ci, v = system(b2s)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    L = b2s.Learner(ctx, seed=1)
    r = b2s.uniform(5, n)
    assert np.array_equal(L.precond(A).apply(r), b2s.Precond(ctx, A, b2s.PC_IC0).apply(r))


@pytest.mark.parametrize("loss_kind", [0, 1, 2])
def test_gradient_matches_autograd(b2s, ctx, orc, loss_kind):
    """loss 2 (LOSS_SWEEPS, 4 sweeps here) runs the hand-written adjoint back
    through both sweep sequences."""
    import gnn_ref
    n, rp, ci, v = system(b2s, N=20)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    L = b2s.Learner(ctx, seed=7, loss=loss_kind)
    L.set_sweeps(4, 0)
    p = L.params()
    rng = np.random.default_rng(0)
    # a non-zero head so every path carries gradient
    off = gnn_ref.OFF_OUT
    p[off:] = rng.normal(0, 0.05, len(p) - off).astype(np.float32)
    L.set_params(p)
    probes = rng.normal(size=(3, n))
    loss, grad = L.step(A, nprobes=3, probes=probes, update=False, want_grad=True)
    e = orc.ic0_export(orc.pc(orc.csr(n, n, rp, ci, v), "ic0"))
    rloss, rgrad, _ = gnn_ref.loss_and_grad(p, n, rp, ci, v, e["Lrp"], e["Lci"], e["Lv"], probes, loss_kind,
                                            sweeps=4)
    assert abs(loss - rloss) <= 1e-4 * abs(rloss)
    scale = np.abs(rgrad).max()
    err = np.abs(grad - rgrad).max() / scale
    assert err < 2e-3, err
    # per block (input, layers, head) relative error
    for a, b in ((0, gnn_ref.LAYER0), (gnn_ref.LAYER0, gnn_ref.OFF_OUT), (gnn_ref.OFF_OUT, gnn_ref.NPARAM)):
        num = np.linalg.norm(grad[a:b] - rgrad[a:b])
        den = np.linalg.norm(rgrad[a:b]) + 1e-30
        assert num / den < 5e-3, (a, b, num / den)


@pytest.mark.parametrize("loss_kind", [1, 0, 2])
def test_training_reduces_loss_and_stays_spd(b2s, ctx, tmp_path, loss_kind):
    # Adam on a fixed probe set (seed 0): the objective itself must go down
    n, rp, ci, v = system(b2s, N=32, seed=11)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    L = b2s.Learner(ctx, seed=2, loss=loss_kind)
    l0 = L.step(A, nprobes=4, seed=0, lr=0.0, update=False)
    for k in range(40):
        L.step(A, nprobes=4, seed=0, lr=1e-3)
    l1 = L.step(A, nprobes=4, seed=0, lr=0.0, update=False)
    assert l1 < l0, (l0, l1)
    M = L.precond(A)
    b = b2s.uniform(1, n)
    x, st = b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-8, maxit=2000)
    assert st["status"] == 0 and st["relres_true"] < 2e-8
    path = str(tmp_path / "w.bin")
    L.save(path)
    L2 = b2s.Learner(ctx, seed=99, weights=path)
    assert np.array_equal(L.params(), L2.params())
    r = b2s.uniform(3, n)
    assert np.array_equal(M.apply(r), L2.precond(A).apply(r))
    # via the preconditioner kind and a weight file
    M3 = b2s.Precond(ctx, A, b2s.PC_LEARNED_IC0, learned_weights=path)
    assert np.array_equal(M.apply(r), M3.apply(r))
    with open(path, "r+b") as f:
        f.seek(40)
        f.write(b"\x00\x01")
    with pytest.raises(ValueError):
        L2.load(path)


def _grf512(b2s, seed):
    n, rp, ci, v = b2s.gen_grf_diffusion(512, seed=seed, corr=0.05)
    return n, rp, ci, v, b2s.uniform(seed, n)


def test_trained_network_gains_over_ic0(b2s, ctx):
    """The shipped weights against the method without them: PCG on a held-out
    512^2 random-coefficient system (seed outside the training range) with
    the learned preconditioner needs at most 70% of plain IC(0)'s iterations,
    both verified to rtol 1e-8 by the FP64 true residual, with no fallback."""
    n, rp, ci, v, b = _grf512(b2s, 2001)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    M0 = b2s.Precond(ctx, A, b2s.PC_IC0)
    _, s0 = b2s.solve(ctx, A, b, b2s.PCG, M0, tol=1e-8, maxit=20000)
    ML = b2s.Precond(ctx, A, b2s.PC_LEARNED_IC0, precision=b2s.FP32)
    _, sl = b2s.solve(ctx, A, b, b2s.PCG, ML, tol=1e-8, maxit=20000)
    assert s0["relres_true"] < 1e-8 and sl["relres_true"] < 1e-8
    assert sl["fallbacks"] == 0
    assert sl["iterations"] <= 0.7 * s0["iterations"], (sl["iterations"], s0["iterations"])


def test_trained_network_gains_with_sweep_solves(b2s, ctx):
    """The same comparison with 8 Jacobi sweeps per triangle (the benchmark's
    default schedule): the learned factor needs at most 75% of plain FP32
    IC(0)'s iterations, both verified to rtol 1e-8 in FP64."""
    n, rp, ci, v, b = _grf512(b2s, 2001)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    opts = dict(precision=b2s.FP32, trsv=b2s.TRSV_JACOBI, trsv_sweeps=8)
    _, s0 = b2s.solve(ctx, A, b, b2s.PCG, b2s.Precond(ctx, A, b2s.PC_IC0, **opts), tol=1e-8, maxit=20000)
    _, sl = b2s.solve(ctx, A, b, b2s.PCG, b2s.Precond(ctx, A, b2s.PC_LEARNED_IC0, **opts), tol=1e-8, maxit=20000)
    assert s0["relres_true"] < 1e-8 and sl["relres_true"] < 1e-8
    assert sl["fallbacks"] == 0
    assert sl["iterations"] <= 0.75 * s0["iterations"], (sl["iterations"], s0["iterations"])


def test_learned_falls_back_on_stall(b2s, ctx):
    """A stall window of one iteration makes the guard fire at the first poll
    where the residual has not halved (on the 512^2 system PCG needs about 17
    iterations per halving, polls come every 8); plain FP64 IC(0) continues
    from the learned iterate to the same tolerance."""
    n, rp, ci, v, b = _grf512(b2s, 2002)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    M = b2s.Precond(ctx, A, b2s.PC_LEARNED_IC0, precision=b2s.FP32)
    x, st = b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-8, maxit=20000, stall_window=1)
    assert st["fallbacks"] == 1 and 0 < st["stalled_at"] < st["iterations"]
    assert st["status"] == 0 and st["relres_true"] < 1e-8
    # the residual checked on the host, independently of the device's FP64 check
    import scipy.sparse as sp
    Ah = sp.csr_matrix((v, ci, rp), shape=(n, n))
    assert np.linalg.norm(b - Ah @ x) < 1e-8 * np.linalg.norm(b)
    # the guard off: the learned solve runs to the tolerance on its own
    x2, s2 = b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-8, maxit=20000, stall_window=-1)
    assert s2["fallbacks"] == 0 and s2["relres_true"] < 1e-8


def test_learned_falls_back_on_divergence(b2s, ctx):
    """A network whose output layer is NaN gives a NaN factor: PCG stops with
    B2S_DIVERGED, and plain IC(0) restarts from x = 0 and converges."""
    n, rp, ci, v = system(b2s, N=32, seed=6)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    L = b2s.Learner(ctx, seed=3)
    p = L.params()
    import gnn_ref
    p[gnn_ref.OFF_OUT:] = np.nan
    L.set_params(p)
    M = L.precond(A)
    b = b2s.uniform(10, n)
    x, st = b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-8, maxit=3000)
    assert st["fallbacks"] == 1
    assert st["status"] == 0 and st["relres_true"] < 1e-8
    assert np.all(np.isfinite(x))
