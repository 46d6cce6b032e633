"""The learned network's hidden dense layer on the tensor cores
(b2s_dense_bf16_device: tcgen05.mma kind::f16, BF16 operands, FP32
accumulation in tensor memory) against a plain PyTorch reference of the same
op, Y = bf16(X) W^T + b, computed in float64 on the CPU.

Tolerance: the products of two BF16 values are exact in FP32, so the only
error is the FP32 accumulation of K = 64 terms; each entry must agree with the
float64 result to 1e-5 of sum_k |bf16(x_k) w_k| (about 2^-24 per addition,
with a wide margin).  Rows past n must stay untouched (ragged last tile)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _run(b2s, torch, ctx, X, W, bias, k, no, guard=3):
    n = X.shape[0]
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(X).to(dev)
    w = torch.from_numpy(W).to(torch.bfloat16).to(dev)
    b = torch.from_numpy(bias).to(dev) if bias is not None else None
    y = torch.full((n + guard, no), 12345.0, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    st = b2s.lib().b2s_dense_bf16_device(ctx.h, n, k, no, C.c_void_p(x.data_ptr()), C.c_void_p(w.data_ptr()),
                                         C.c_void_p(b.data_ptr()) if b is not None else None,
                                         C.c_void_p(y.data_ptr()))
    ctx.check(st, "dense_bf16_device")
    ctx.check(b2s.lib().b2s_ctx_synchronize(ctx.h), "synchronize")
    out = y.cpu().numpy()
    return out[:n], out[n:], w.float().cpu().numpy()


def _reference(torch, X, Wb, bias):
    xb = torch.from_numpy(X).to(torch.bfloat16).to(torch.float64)
    wb = torch.from_numpy(Wb).to(torch.float64)
    y = xb @ wb.T
    scale = xb.abs() @ wb.abs().T
    if bias is not None:
        y = y + torch.from_numpy(bias).to(torch.float64)
        scale = scale + torch.from_numpy(np.abs(bias)).to(torch.float64)
    return y.numpy(), scale.numpy()


@pytest.mark.parametrize("no", [128, 64])
@pytest.mark.parametrize("n", [1, 127, 128, 129, 1000, 40000])
def test_dense_matches_torch(b2s, ctx, n, no):
    torch = pytest.importorskip("torch")
    k = 64
    rng = np.random.default_rng(n * 7 + no)
    X = rng.normal(0, 1, (n, k)).astype(np.float32)
    W = (rng.normal(0, 0.2, (no, k))).astype(np.float32)
    bias = rng.normal(0, 0.1, no).astype(np.float32) if n % 2 else None
    Y, tail, Wb = _run(b2s, torch, ctx, X, W, bias, k, no)
    ref, scale = _reference(torch, X, Wb, bias)
    err = np.abs(Y.astype(np.float64) - ref)
    assert np.all(err <= TOL * scale + 1e-30), float((err / (scale + 1e-30)).max())
    assert np.all(tail == 12345.0)


def test_dense_large_values_and_zero_rows(b2s, ctx):
    # rows of zeros, huge and tiny magnitudes (BF16 keeps the FP32 exponent range)
    torch = pytest.importorskip("torch")
    k, no, n = 64, 128, 300
    rng = np.random.default_rng(5)
    X = rng.normal(0, 1, (n, k)).astype(np.float32)
    X[::3] = 0.0
    X[1::7] *= 1e30
    X[2::11] *= 1e-30
    W = rng.normal(0, 1, (no, k)).astype(np.float32)
    Y, _, Wb = _run(b2s, torch, ctx, X, W, None, k, no)
    ref, scale = _reference(torch, X, Wb, None)
    assert np.all(np.abs(Y.astype(np.float64) - ref) <= TOL * scale + 1e-300)
    assert np.all(Y[::3] == 0.0)


def test_dense_rejects_bad_shapes_and_alignment(b2s, ctx):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    x = torch.zeros(64 * 64 + 4, dtype=torch.float32, device=dev)
    w = torch.zeros(128 * 64, dtype=torch.bfloat16, device=dev)
    y = torch.zeros(64 * 128, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    L = b2s.lib()
    st = L.b2s_dense_bf16_device(ctx.h, 64, 32, 128, C.c_void_p(x.data_ptr()), C.c_void_p(w.data_ptr()), None,
                                 C.c_void_p(y.data_ptr()))
    assert st == b2s.UNSUPPORTED
    st = L.b2s_dense_bf16_device(ctx.h, 64, 64, 128, C.c_void_p(x.data_ptr() + 4), C.c_void_p(w.data_ptr()), None,
                                 C.c_void_p(y.data_ptr()))
    assert st == b2s.INVALID_ARG
    # n = 0 is a no-op
    st = L.b2s_dense_bf16_device(ctx.h, 0, 64, 128, C.c_void_p(x.data_ptr()), C.c_void_p(w.data_ptr()), None,
                                 C.c_void_p(y.data_ptr()))
    assert st == b2s.OK
    ctx.check(L.b2s_ctx_synchronize(ctx.h), "synchronize")
