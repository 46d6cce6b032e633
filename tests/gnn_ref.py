"""PyTorch (CPU, float64, autograd) restatement of the learned-IC(0) network
and its training loss, used as the gradient oracle for the GPU forward and
backward kernels (cpp-fem-solver_b200/csrc/learned.cu).  Test infrastructure."""
import numpy as np
import torch

H, FIN, FE, NL = 64, 8, 4, 3
OFF_WIN, OFF_BIN = 0, H * FIN
LAYER0 = OFF_BIN + H
L_WS, L_WM, L_WG = 0, H * H, 2 * H * H
L_BG = L_WG + H * FE
L_B = L_BG + H
L_SIZE = L_B + H
OFF_OUT = LAYER0 + NL * L_SIZE
O_U, O_V, O_W = 0, H, 2 * H
O_BO = 2 * H + FE
O_D = O_BO + 1
O_BD = O_D + H
NPARAM = OFF_OUT + O_BD + 1


def bf16_round(p):
    return torch.from_numpy(np.asarray(p, np.float32)).to(torch.bfloat16).to(torch.float64)


def features(n, rp, ci, v):
    rows = np.repeat(np.arange(n), np.diff(rp))
    diag = np.zeros(n)
    dm = rows == ci
    diag[rows[dm]] = v[dm]
    la = np.log(np.abs(diag) + 1e-300)
    off = ~dm
    a = np.abs(v) + 1e-300
    t = np.log(a) - la[rows]
    F = np.zeros((n, FIN))
    deg = np.bincount(rows[off], minlength=n)
    s = np.bincount(rows[off], weights=t[off], minlength=n)
    mn = np.full(n, 1e300)
    mx = np.full(n, -1e300)
    np.minimum.at(mn, rows[off], t[off])
    np.maximum.at(mx, rows[off], t[off])
    offs = np.bincount(rows[off], weights=a[off], minlength=n)
    F[:, 0] = np.where(deg > 0, s / np.maximum(deg, 1), 0)
    F[:, 1] = np.where(deg > 0, mn, 0)
    F[:, 2] = np.where(deg > 0, mx, 0)
    F[:, 3] = np.log(offs / np.abs(diag) + 1e-30)
    F[:, 4] = deg / 4.0
    F[:, 5] = la - la.mean()
    EF = np.zeros((len(v), FE))
    EF[off, 0] = t[off]
    EF[off, 1] = np.log(a[off]) - la[ci[off]]
    EF[off, 2] = la[ci[off]] - la[rows[off]]
    EF[off, 3] = np.where(ci[off] < rows[off], 1.0, -1.0)
    invdeg = np.where(deg > 0, 1.0 / np.maximum(deg, 1), 0.0)
    # the GPU stores features in FP32
    return (F.astype(np.float32).astype(np.float64), EF.astype(np.float32).astype(np.float64),
            invdeg.astype(np.float32).astype(np.float64), diag)


LOSS_PRECOND, LOSS_FACTOR, LOSS_SWEEPS = 0, 1, 2


def loss_and_grad(params, n, rp, ci, v, Lrp, Lci, L0, probes, loss_kind=LOSS_PRECOND, sweeps=6):
    """params: FP32 master parameters (rounded to BF16 as the GPU forward does).
    loss_kind: LOSS_PRECOND, mean_w ||w - (L~L~^T)^{-1} A w||^2 / ||w||^2,
    LOSS_FACTOR, mean_w ||(L~L~^T - A) w||^2 / ||A w||^2, or LOSS_SWEEPS, the
    first with (L~L~^T)^{-1} replaced by F^T F, F = `sweeps` Jacobi sweeps of
    L~ (y_0 = D^-1 r, y_s = D^-1 (r - N y_{s-1})) and F^T those of L~^T."""
    P = bf16_round(params).requires_grad_(True)
    F, EF, invdeg, diag = features(n, rp, ci, v)
    F, EF, invdeg = map(torch.from_numpy, (F, EF, invdeg))
    rows = np.repeat(np.arange(n), np.diff(rp))
    off = rows != ci
    src, dst = torch.from_numpy(rows[off]), torch.from_numpy(ci[off].astype(np.int64))
    Ef = EF[torch.from_numpy(np.nonzero(off)[0])]
    relu = torch.relu
    Win = P[OFF_WIN:OFF_WIN + H * FIN].view(H, FIN)
    h = relu(F @ Win.T + P[OFF_BIN:OFF_BIN + H])
    for l in range(NL):
        b0 = LAYER0 + l * L_SIZE
        Ws = P[b0 + L_WS:b0 + L_WS + H * H].view(H, H)
        Wm = P[b0 + L_WM:b0 + L_WM + H * H].view(H, H)
        Wg = P[b0 + L_WG:b0 + L_WG + H * FE].view(H, FE)
        bg = P[b0 + L_BG:b0 + L_BG + H]
        bl = P[b0 + L_B:b0 + L_B + H]
        # the tensor-core layer multiplies BF16-rounded node states; the
        # rounding passes the gradient straight through (dH = dS Ws + dM Wm)
        hb = h + (h.detach().to(torch.float32).to(torch.bfloat16).to(torch.float64) - h.detach())
        S, M = hb @ Ws.T, hb @ Wm.T
        g = torch.sigmoid(Ef @ Wg.T + bg)
        agg = torch.zeros(n, H, dtype=torch.float64).index_add(0, src, g * M[dst])
        pre = S + bl + invdeg[:, None] * agg
        h = relu(pre) + h
    Lrows = np.repeat(np.arange(n), np.diff(Lrp))
    isd = Lrows == Lci
    pA = torch.from_numpy((rp[Lrows] + (np.arange(len(Lci)) - Lrp[Lrows])).astype(np.int64))
    Lr, Lc = torch.from_numpy(Lrows), torch.from_numpy(Lci.astype(np.int64))
    u, vv, w = P[OFF_OUT + O_U:OFF_OUT + O_U + H], P[OFF_OUT + O_V:OFF_OUT + O_V + H], P[OFF_OUT + O_W:OFF_OUT + O_W + FE]
    bo, d, bd = P[OFF_OUT + O_BO], P[OFF_OUT + O_D:OFF_OUT + O_D + H], P[OFF_OUT + O_BD]
    c_off = h[Lr] @ u + h[Lc] @ vv + EF[pA] @ w + bo
    c_diag = h[Lr] @ d + bd
    c = torch.where(torch.from_numpy(isd), c_diag, c_off)
    Lt = torch.from_numpy(L0) * torch.exp(0.5 * torch.tanh(c))
    lo = torch.from_numpy(1e-3 * np.sqrt(np.abs(diag[Lrows])))
    Lt = torch.where(torch.from_numpy(isd), torch.maximum(Lt, lo), Lt)
    Lmat = torch.sparse_coo_tensor(torch.stack([Lr, Lc]), Lt, (n, n)).to_dense()
    A = torch.sparse_coo_tensor(torch.from_numpy(np.stack([rows, ci.astype(np.int64)])), torch.from_numpy(v),
                                (n, n)).to_dense()
    W = torch.from_numpy(np.asarray(probes).reshape(-1, n).T)
    AW = A @ W
    if loss_kind == LOSS_PRECOND:
        Y = torch.linalg.solve_triangular(Lmat, AW, upper=False)
        Z = torch.linalg.solve_triangular(Lmat.T, Y, upper=True)
        E = W - Z
        loss = ((E ** 2).sum(0) / (W ** 2).sum(0)).mean()
    elif loss_kind == LOSS_SWEEPS:
        D = torch.diagonal(Lmat)[:, None]
        N = Lmat - torch.diag(torch.diagonal(Lmat))
        Y = AW / D
        for _ in range(sweeps):
            Y = (AW - N @ Y) / D
        Z = Y / D
        for _ in range(sweeps):
            Z = (Y - N.T @ Z) / D
        E = W - Z
        loss = ((E ** 2).sum(0) / (W ** 2).sum(0)).mean()
    else:
        E = Lmat @ (Lmat.T @ W) - AW
        loss = ((E ** 2).sum(0) / (AW ** 2).sum(0)).mean()
    loss.backward()
    return float(loss), P.grad.numpy(), Lt.detach().numpy()
