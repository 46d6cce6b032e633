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


def test_gradient_matches_autograd(b2s, ctx, orc):
    import gnn_ref
    n, rp, ci, v = system(b2s, N=20)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    L = b2s.Learner(ctx, seed=7)
    p = L.params()
    rng = np.random.default_rng(0)
    # a non-zero head so every path carries gradient
    off = gnn_ref.OFF_OUT
    p[off:] = rng.normal(0, 0.05, len(p) - off).astype(np.float32)
    L.set_params(p)
    probes = rng.normal(size=(3, n))
    loss, grad = L.step(A, nprobes=3, probes=probes, update=False, want_grad=True)
    e = orc.ic0_export(orc.pc(orc.csr(n, n, rp, ci, v), "ic0"))
    rloss, rgrad, _ = gnn_ref.loss_and_grad(p, n, rp, ci, v, e["Lrp"], e["Lci"], e["Lv"], probes)
    assert abs(loss - rloss) <= 1e-4 * abs(rloss)
    scale = np.abs(rgrad).max()
    err = np.abs(grad - rgrad).max() / scale
    assert err < 2e-3, err
    # per block (input, layers, head) relative error
    for a, b in ((0, gnn_ref.LAYER0), (gnn_ref.LAYER0, gnn_ref.OFF_OUT), (gnn_ref.OFF_OUT, gnn_ref.NPARAM)):
        num = np.linalg.norm(grad[a:b] - rgrad[a:b])
        den = np.linalg.norm(rgrad[a:b]) + 1e-30
        assert num / den < 5e-3, (a, b, num / den)


def test_training_reduces_loss_and_stays_spd(b2s, ctx, tmp_path):
    n, rp, ci, v = system(b2s, N=32, seed=11)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    L = b2s.Learner(ctx, seed=2)
    l0 = L.step(A, nprobes=4, seed=0, lr=0.0, update=False)
    for k in range(40):
        L.step(A, nprobes=4, seed=k, lr=3e-3)
    l1 = L.step(A, nprobes=4, seed=0, lr=0.0, update=False)
    assert l1 < l0
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
