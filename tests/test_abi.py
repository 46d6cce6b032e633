"""CPU checks of the boundary: libb2s.so loads, exports exactly the entry
points include/b2s.h declares, and the host-only parts (name tables,
generators) behave; no compute call needs a GPU here."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "b2s.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(b2s_[a-z0-9_]+)\s*\(", text)) - {"b2s_host_pc_fn"})


def test_library_exports_every_declared_symbol(b2s):
    path = b2s.load_extension()
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    assert sorted(b2s.EXPORTS) == declared_symbols()


def test_no_device_fails_loudly(b2s):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(b2s.B2SError) as e:
        b2s.Context(0)
    assert e.value.status == b2s.NO_DEVICE


@pytest.mark.parametrize("method,name,kind", [
    (0, "none", 0), (0, "CG", 0), (0, "Identity", 0), (0, "noprecond", 0), (0, "Diagonal", 1), (0, "jacobi", 1),
    (0, "ic", 2), (0, "ICHOL", 2), (0, "incomplete_cholesky", 2), (0, "ilu", 3), (0, "ILU0", 3), (0, "sor", 4),
    (0, "SSOR", 4), (0, "amg", 5), (1, "incomplete_cholesky", 2), (1, "ic0", 2), (2, "ic", 2), (2, "ssor", 4),
    (4, "blockjacobi", 7), (4, "blockilu", 8), (4, "blockilu0", 8), (4, "none", 0), (4, "identity", 0),
])
def test_precond_name_tables(b2s, method, name, kind):
    assert b2s.pc_kind_from_name(method, name) == kind


@pytest.mark.parametrize("method,name", [(1, "cg"), (2, "cg"), (2, "incomplete_cholesky"), (4, "BlockJacobi"),
                                         (4, "ilu"), (0, "bogus"), (0, "")])
def test_precond_name_rejected(b2s, method, name):
    with pytest.raises(ValueError):
        b2s.pc_kind_from_name(method, name)


def test_generators_structure(b2s):
    import problems as P
    n, rp, ci, v = b2s.gen_poisson2d(13)
    n2, rp2, ci2, v2 = P.poisson2d(13)
    assert n == n2 and np.array_equal(rp, rp2) and np.array_equal(ci, ci2) and np.array_equal(v, v2)
    n, rp, ci, v = b2s.gen_poisson3d(6)
    assert n == 216 and rp[-1] == 7 * 216 - 6 * 36
    d = v[np.repeat(np.arange(n), np.diff(rp)) == ci]
    assert np.all(d == 6.0)
    n, rp, ci, v = b2s.gen_convdiff3d(5, 10.0, 5.0, 2.5)
    rows = np.repeat(np.arange(n), np.diff(rp))
    assert np.all(v[rows == ci] == 6.0 + 17.5)
    assert np.all(v[ci == rows - 1] == -11.0) and np.all(v[ci == rows + 1] == -1.0)


def test_benchmark_sizes(b2s):
    """nnz of the benchmark configurations (C1-C3) and the elasticity structure (C4)."""
    n, rp, _, _ = b2s.gen_poisson2d(256)
    assert (n, rp[-1]) == (65536, 326656)
    n, rp, _, _ = b2s.gen_convdiff3d(96)
    assert (n, rp[-1]) == (884736, 6137856)
    nbr, rp, ci, v = b2s.gen_elasticity_q1(8)
    assert nbr == 8 * 81
    # symmetric, rigid-body modes in the kernel of the unclamped operator rows
    import scipy.sparse as sp
    bsr = sp.bsr_matrix((v.reshape(-1, 3, 3), ci, rp), shape=(3 * nbr, 3 * nbr)).tocsr()
    assert abs(bsr - bsr.T).max() < 1e-12
    assert np.all(np.linalg.eigvalsh(bsr.toarray()) > 0)


def test_elasticity_c4_size(b2s):
    nbr, nnzb = np.zeros(1, np.uint32), np.zeros(1, np.uint32)
    import ctypes as C
    a, bb = C.c_uint32(), C.c_uint32()
    assert b2s.lib().b2s_gen_elasticity_q1(64, 1.0, 0.3, C.byref(a), C.byref(bb), None, None, None) == 0
    assert a.value == 270400 and bb.value == 7077310


def test_grf_field(b2s):
    n, rp, ci, v, k = b2s.gen_grf_diffusion(64, seed=3, corr=0.05, var=2.0, with_k=True)
    assert n == 4096 and rp[-1] == 5 * 4096 - 4 * 64
    logk = np.log(k)
    assert abs(logk.var() - 2.0) < 1.2 and np.all(np.isfinite(logk))
    import scipy.sparse as sp
    A = sp.csr_matrix((v, ci, rp), shape=(n, n))
    assert abs(A - A.T).max() < 1e-12
    rows = np.repeat(np.arange(n), np.diff(rp))
    assert np.all(v[rows == ci] > 0) and np.all(v[rows != ci] < 0)
    # deterministic per seed, different across seeds
    _, _, _, v2 = b2s.gen_grf_diffusion(64, seed=3, corr=0.05, var=2.0)
    _, _, _, v3 = b2s.gen_grf_diffusion(64, seed=4, corr=0.05, var=2.0)
    assert np.array_equal(v, v2) and not np.array_equal(v, v3)


def test_grf_covariance(b2s):
    """Pointwise variance of log k over seeds matches the requested variance."""
    samples = np.array([np.log(b2s.gen_grf_diffusion(32, seed=s, corr=0.1, var=1.5, with_k=True)[4])
                        for s in range(60)])
    assert abs(samples.var(axis=0).mean() - 1.5) < 0.3


def test_uniform(b2s):
    u = b2s.uniform(7, 100000)
    assert u.min() >= -1 and u.max() < 1 and abs(u.mean()) < 0.01
    assert np.array_equal(u, b2s.uniform(7, 100000)) and not np.array_equal(u, b2s.uniform(8, 100000))
