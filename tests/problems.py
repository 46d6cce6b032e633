"""Small deterministic test problems (CSR arrays) shared by CPU and GPU tests."""
import numpy as np


def coo_to_csr(n, m, r, c, v):
    """Sorted, duplicate-free CSR from COO (no duplicates expected)."""
    r, c, v = np.asarray(r, np.int64), np.asarray(c, np.int64), np.asarray(v, np.float64)
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, r + 1, 1)
    return np.cumsum(rp).astype(np.uint32), c.astype(np.uint32), v


def poisson2d(N):
    R, Cc, V = [], [], []
    for i in range(N):
        for j in range(N):
            k = i * N + j
            R.append(k); Cc.append(k); V.append(4.0)
            for a, b in ((i - 1, j), (i + 1, j), (i, j - 1), (i, j + 1)):
                if 0 <= a < N and 0 <= b < N:
                    R.append(k); Cc.append(a * N + b); V.append(-1.0)
    rp, ci, v = coo_to_csr(N * N, N * N, R, Cc, V)
    return N * N, rp, ci, v


def convdiff2d(N, vx=5.0, vy=5.0):
    """test_SMatrix_gmres.cpp:75-112 stencil."""
    R, Cc, V = [], [], []
    for i in range(N):
        for j in range(N):
            k = i * N + j
            R.append(k); Cc.append(k); V.append(4.0 + vx + vy)
            if j > 0: R.append(k); Cc.append(k - 1); V.append(-1.0 - vx)
            if j < N - 1: R.append(k); Cc.append(k + 1); V.append(-1.0)
            if i > 0: R.append(k); Cc.append(k - N); V.append(-1.0 - vy)
            if i < N - 1: R.append(k); Cc.append(k + N); V.append(-1.0)
    rp, ci, v = coo_to_csr(N * N, N * N, R, Cc, V)
    return N * N, rp, ci, v


def random_spd(n, density, seed):
    """Random sparse SPD (diagonally dominant) with ragged rows."""
    rng = np.random.default_rng(seed)
    R, Cc, V = [], [], []
    for i in range(n):
        k = rng.binomial(n, density)
        cols = rng.choice(n, size=min(k, n), replace=False)
        for j in cols:
            if j < i:
                val = -rng.uniform(0.1, 1.0)
                R += [i, j]; Cc += [j, i]; V += [val, val]
    A = {}
    for r, c, v in zip(R, Cc, V):
        A[(r, c)] = A.get((r, c), 0.0) + v
    rows = [[] for _ in range(n)]
    for (r, c), v in A.items():
        rows[r].append((c, v))
    RR, CC, VV = [], [], []
    for i in range(n):
        s = sum(abs(v) for _, v in rows[i])
        for c, v in rows[i]:
            RR.append(i); CC.append(c); VV.append(v)
        RR.append(i); CC.append(i); VV.append(s + 1.0 + rng.uniform(0, 1))
    rp, ci, v = coo_to_csr(n, n, RR, CC, VV)
    return n, rp, ci, v


def make_test_scalar(N, BS=3):
    """test_BlockMatrix_mpi.cpp:29-59: node-major 2-D grid, BS components per node."""
    R, Cc, V = [], [], []
    for i in range(N):
        for j in range(N):
            idx = i * N + j
            for r in range(BS):
                row = idx * BS + r
                for c in range(BS):
                    R.append(row); Cc.append(idx * BS + c); V.append(4.0 + BS if r == c else 0.1)
                if j > 0: R.append(row); Cc.append((idx - 1) * BS + r); V.append(-1.0)
                if j < N - 1: R.append(row); Cc.append((idx + 1) * BS + r); V.append(-1.0)
                if i > 0: R.append(row); Cc.append((idx - N) * BS + r); V.append(-1.0)
                if i < N - 1: R.append(row); Cc.append((idx + N) * BS + r); V.append(-1.0)
    n = N * N * BS
    rp, ci, v = coo_to_csr(n, n, R, Cc, V)
    return n, rp, ci, v


def drand(i):
    """test_BlockMatrix_mpi.cpp:22-23 deterministic hash."""
    s = np.sin(np.asarray(i, np.float64) * 0.371 + 1.7) * 43758.5453
    return s - np.floor(s)
