"""b2s_dot_noalloc, the entry point for callers that cannot allocate device
memory after set-up (for example a host application whose device memory is
handed out up front by another framework's allocator).  It must agree with
the regular b2s_dot_device entry point on the same device vectors, on two
calls in a row (the shared scratch array keeps the previous call's contents),
and reject sizes above its limit.

Tolerance: the two entry points reduce in different fixed orders (different
grids), so they agree to 1e-12 relative to sum |a_i b_i| (the scale of a dot
product's rounding error), not bit for bit.

This file is named so that pytest collects it last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12


def _dot_noalloc(b2s, torch, a, b, out):
    st = b2s.lib().b2s_dot_noalloc(C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), a.numel(),
                                   C.c_void_p(out.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return st


def test_dot_noalloc_matches_dot_device(b2s):
    torch = pytest.importorskip("torch")
    ctx = b2s.Context(0)
    rng = np.random.default_rng(2024)
    for n in (1, 1000, 2048 * 37 + 5, 1 << 21, 8388608):
        a = torch.from_numpy(rng.uniform(-1, 1, n)).cuda()
        b = torch.from_numpy(rng.uniform(-1, 1, n)).cuda()
        out = torch.zeros(1, dtype=torch.float64, device="cuda")
        ref = C.c_double()
        ctx.check(b2s.lib().b2s_dot_device(ctx.h, n, C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()),
                                           C.byref(ref)), "dot_device")
        for _ in range(2):  # two calls in a row share the scratch array
            out.zero_()
            assert _dot_noalloc(b2s, torch, a, b, out) == b2s.OK
            got = float(out.item())
            scale = float((a * b).abs().sum().item())
            assert abs(got - ref.value) <= REL_TOL * scale, (n, got, ref.value)
    ctx.close()


def test_dot_noalloc_rejects_oversize(b2s):
    torch = pytest.importorskip("torch")
    a = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = b2s.lib().b2s_dot_noalloc(C.c_void_p(a.data_ptr()), C.c_void_p(a.data_ptr()), 8388608 + 1,
                                   C.c_void_p(out.data_ptr()), None)
    assert st == b2s.INVALID_ARG
