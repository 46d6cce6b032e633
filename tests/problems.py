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


def coo_merge(n, m, r, c, v):
    """CSR from COO with duplicates summed in input order (as the reference's
    COO constructor merges them), explicit zeros kept out."""
    acc = {}
    for i, j, x in zip(r, c, v):
        acc[(i, j)] = acc.get((i, j), 0.0) + x
    keys = [k for k in acc if acc[k] != 0.0]
    return coo_to_csr(n, m, [k[0] for k in keys], [k[1] for k in keys], [acc[k] for k in keys])


def stokes1d(N_vel):
    """1-D Stokes saddle point of test_BlockMatrix_schur.cpp:34-80: K, A, B, B^T
    as (rows, cols, rp, ci, v)."""
    N_pres = N_vel - 1
    N = N_vel + N_pres
    R, Cc, V = [], [], []
    for i in range(N_vel):
        R.append(i); Cc.append(i); V.append(2.0)
        if i > 0: R.append(i); Cc.append(i - 1); V.append(-1.0)
        if i < N_vel - 1: R.append(i); Cc.append(i + 1); V.append(-1.0)
    for i in range(N_pres):
        R += [i + N_vel, i + N_vel, i, i + 1]
        Cc += [i, i + 1, i + N_vel, i + N_vel]
        V += [-1.0, 1.0, -1.0, 1.0]
    return split_saddle(N_vel, N_pres, R, Cc, V)


def split_saddle(N_vel, N_pres, R, Cc, V):
    N = N_vel + N_pres
    parts = {"A": ([], [], []), "B": ([], [], []), "Bt": ([], [], [])}
    for r, c, v in zip(R, Cc, V):
        if r < N_vel and c < N_vel:
            key, rr, cc = "A", r, c
        elif r >= N_vel and c < N_vel:
            key, rr, cc = "B", r - N_vel, c
        elif r < N_vel and c >= N_vel:
            key, rr, cc = "Bt", r, c - N_vel
        else:
            continue
        parts[key][0].append(rr); parts[key][1].append(cc); parts[key][2].append(v)
    K = (N, N) + coo_merge(N, N, R, Cc, V)
    A = (N_vel, N_vel) + coo_merge(N_vel, N_vel, *parts["A"])
    B = (N_pres, N_vel) + coo_merge(N_pres, N_vel, *parts["B"])
    Bt = (N_vel, N_pres) + coo_merge(N_vel, N_pres, *parts["Bt"])
    return K, A, B, Bt


def stokes3d(N, alpha=0.1):
    """3-D periodic MAC Stokes of test_BlockMatrix_schur3d.cpp:39-133: K, A,
    B, B^T and the pressure Laplacian Lp, as (rows, cols, rp, ci, v)."""
    N3 = N * N * N
    N_vel, N_pres = 3 * N3, N3
    idx = lambda i, j, k: i + j * N + k * N * N
    R, Cc, V = [], [], []
    for comp in range(3):
        off = comp * N3
        for k in range(N):
            for j in range(N):
                for i in range(N):
                    r = off + idx(i, j, k)
                    R.append(r); Cc.append(r); V.append(6.0 + alpha)
                    for (a, b_, c_) in (((i + 1) % N, j, k), ((i - 1 + N) % N, j, k), (i, (j + 1) % N, k),
                                        (i, (j - 1 + N) % N, k), (i, j, (k + 1) % N), (i, j, (k - 1 + N) % N)):
                        R.append(r); Cc.append(off + idx(a, b_, c_)); V.append(-1.0)
    LR, LC, LV = [], [], []
    for k in range(N):
        for j in range(N):
            for i in range(N):
                p = idx(i, j, k)
                rp_ = N_vel + p
                LR.append(p); LC.append(p); LV.append(6.0 + 1e-8)
                for (a, b_, c_) in (((i + 1) % N, j, k), ((i - 1 + N) % N, j, k), (i, (j + 1) % N, k),
                                    (i, (j - 1 + N) % N, k), (i, j, (k + 1) % N), (i, j, (k - 1 + N) % N)):
                    LR.append(p); LC.append(idx(a, b_, c_)); LV.append(-1.0)
                for comp, prev in ((0, idx((i - 1 + N) % N, j, k)), (1, idx(i, (j - 1 + N) % N, k)),
                                   (2, idx(i, j, (k - 1 + N) % N))):
                    uc, up = comp * N3 + p, comp * N3 + prev
                    R += [rp_, rp_, uc, up]
                    Cc += [uc, up, rp_, rp_]
                    V += [1.0, -1.0, 1.0, -1.0]
    K, A, B, Bt = split_saddle(N_vel, N_pres, R, Cc, V)
    Lp = (N_pres, N_pres) + coo_merge(N_pres, N_pres, LR, LC, LV)
    return K, A, B, Bt, Lp


def diffusion2d(nx, ny, seed):
    """-div(k grad u) on an nx x ny grid (x fastest), 5-point, face
    coefficients k = exp(N(0,1)) per face, Dirichlet outside: SPD."""
    rng = np.random.default_rng(seed)
    kx = np.exp(rng.standard_normal((ny, nx + 1)))
    ky = np.exp(rng.standard_normal((ny + 1, nx)))
    R, Cc, V = [], [], []
    for y in range(ny):
        for x in range(nx):
            i = y * nx + x
            d = kx[y, x] + kx[y, x + 1] + ky[y, x] + ky[y + 1, x]
            R.append(i); Cc.append(i); V.append(d)
            if x > 0: R.append(i); Cc.append(i - 1); V.append(-kx[y, x])
            if x + 1 < nx: R.append(i); Cc.append(i + 1); V.append(-kx[y, x + 1])
            if y > 0: R.append(i); Cc.append(i - nx); V.append(-ky[y, x])
            if y + 1 < ny: R.append(i); Cc.append(i + nx); V.append(-ky[y + 1, x])
    rp, ci, v = coo_to_csr(nx * ny, nx * ny, R, Cc, V)
    return nx * ny, rp, ci, v


def diffusion3d(nx, ny, nz, seed):
    """-div(k grad u) on an nx x ny x nz grid (x fastest, then y), 7-point,
    face coefficients k = exp(N(0,1)) per face, Dirichlet outside: SPD."""
    rng = np.random.default_rng(seed)
    kx = np.exp(rng.standard_normal((nz, ny, nx + 1)))
    ky = np.exp(rng.standard_normal((nz, ny + 1, nx)))
    kz = np.exp(rng.standard_normal((nz + 1, ny, nx)))
    R, Cc, V = [], [], []
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                i = (z * ny + y) * nx + x
                d = kx[z, y, x] + kx[z, y, x + 1] + ky[z, y, x] + ky[z, y + 1, x] + kz[z, y, x] + kz[z + 1, y, x]
                R.append(i); Cc.append(i); V.append(d)
                if x > 0: R.append(i); Cc.append(i - 1); V.append(-kx[z, y, x])
                if x + 1 < nx: R.append(i); Cc.append(i + 1); V.append(-kx[z, y, x + 1])
                if y > 0: R.append(i); Cc.append(i - nx); V.append(-ky[z, y, x])
                if y + 1 < ny: R.append(i); Cc.append(i + nx); V.append(-ky[z, y + 1, x])
                if z > 0: R.append(i); Cc.append(i - nx * ny); V.append(-kz[z, y, x])
                if z + 1 < nz: R.append(i); Cc.append(i + nx * ny); V.append(-kz[z + 1, y, x])
    n = nx * ny * nz
    rp, ci, v = coo_to_csr(n, n, R, Cc, V)
    return n, rp, ci, v
