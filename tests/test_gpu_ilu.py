"""IC(0) / ILU(0) on the GPU against the restatement (array.cpp:2522-2934):
factors, level sets and FP64 applies are bit-exact (each row evaluated in the
reference's order); the FP32 variant is checked against the FP64 apply
(relative 1e-5); PCG / BiCGSTAB / GMRES with ic / ilu within +/-2 iterations
and 1e-9 relative of the oracle's solution."""
import numpy as np
import pytest

import problems as P
import oracle

pytestmark = pytest.mark.gpu

MATS = {
    "poisson2d": lambda b2s: P.poisson2d(40),
    "random": lambda b2s: P.random_spd(1500, 0.004, 3),
    "poisson3d": lambda b2s: b2s.gen_poisson3d(12),
    "grf": lambda b2s: b2s.gen_grf_diffusion(48, seed=5),
}


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("mat", list(MATS))
@pytest.mark.parametrize("trsv", [1, 2, 3])
def test_ic0_bit_exact(b2s, ctx, orc, mat, trsv):
    n, rp, ci, v = MATS[mat](b2s)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    M = b2s.Precond(ctx, A, b2s.PC_IC0, trsv=trsv)
    po = orc.pc(orc.csr(n, n, rp, ci, v), "ic0")
    e = orc.ic0_export(po)
    Lrp, Lci, Lv = M.export("ic0.L")
    assert np.array_equal(Lrp, e["Lrp"]) and np.array_equal(Lci, e["Lci"]) and np.array_equal(Lv, e["Lv"])
    Trp, Tci, Tv = M.export("ic0.LT")
    assert np.array_equal(Trp, e["LTrp"]) and np.array_equal(Tci, e["LTci"]) and np.array_equal(Tv, e["LTv"])
    lev = M.export("levels.L")[1]
    lo, _ = orc.levels(n, e["Lrp"], e["Lci"], upper=False)
    assert np.array_equal(lev, lo)
    levu = M.export("levels.U")[1]
    lu, _ = orc.levels(n, e["LTrp"], e["LTci"], upper=True)
    assert np.array_equal(levu, lu)
    r = b2s.uniform(21, n)
    assert np.array_equal(M.apply(r), po.apply(r))


@pytest.mark.parametrize("spread,rhs_lo", [(60, -40), (500, -700)])
def test_fp64_chunk_division_bit_exact(b2s, ctx, orc, spread, rhs_lo):
    """FP64 chunked solves across the binary64 range: every quotient and
    every partial sum must equal the restatement's.  D A D with D = 2^k, k
    uniform in [0, spread] (the factorisations' absolute pivot test rules out
    tiny pivots), and right-hand sides whose entries span 2^rhs_lo .. 2^40, put
    the row sums and pivots from subnormal-adjacent to 2^500.  The IC(0) and
    ILU(0) applies must equal the restatement bit for bit."""
    n, rp, ci, v = P.random_spd(3000, 0.003, 11)
    rng = np.random.default_rng(spread)
    d = np.exp2(rng.integers(0, spread + 1, n).astype(np.float64))
    rows = np.repeat(np.arange(n), np.diff(rp.astype(np.int64)))
    vs = v * d[rows] * d[ci]
    A = b2s.CSR(ctx, n, n, rp, ci, vs)
    r = b2s.uniform(31, n) * np.exp2(rng.integers(rhs_lo, 41, n).astype(np.float64))
    for kind in ("ic0", "ilu0"):
        M = b2s.Precond(ctx, A, b2s.PC_NAMES[kind])
        po = orc.pc(orc.csr(n, n, rp, ci, vs), kind)
        assert np.array_equal(M.apply(r), po.apply(r)), kind


def _f32_apply(L, U, r, lower_unit):
    """The FP32 factor's apply as the GPU schedules compute it: FP32 values,
    each row summed in column order in FP32, times the divisor's reciprocal
    rounded once from FP64 (numpy float32 scalars: IEEE, no contraction)."""
    f32 = np.float32
    (lrp, lci, lv), (urp, uci, uv) = L, U
    n = len(lrp) - 1
    y = np.zeros(n, np.float32)
    for i in range(n):
        acc, dd = f32(r[i]), None
        for e in range(lrp[i], lrp[i + 1]):
            if lci[e] == i:
                dd = f32(lv[e])
            else:
                acc = f32(acc - f32(f32(lv[e]) * y[lci[e]]))
        y[i] = acc if lower_unit else f32(acc * f32(1.0 / np.float64(dd)))
    z = np.zeros(n, np.float32)
    for i in range(n - 1, -1, -1):
        acc, dd = f32(y[i]), None
        for e in range(urp[i], urp[i + 1]):
            if uci[e] == i:
                dd = f32(uv[e])
            else:
                acc = f32(acc - f32(f32(uv[e]) * z[uci[e]]))
        z[i] = f32(acc * f32(1.0 / np.float64(dd)))
    return z.astype(np.float64)


@pytest.mark.parametrize("nx,ny", [(40, 40), (33, 70), (200, 31), (7, 512), (64, 33), (16, 1500)])
def test_grid5_exact_solves(b2s, ctx, orc, nx, ny):
    """5-point grid factors take the lane-per-grid-line schedule (exported as
    "trsv.grid5"): one single-warp CTA per 32 lines, the boundary lines handed
    between CTAs as epoch-tagged words.  Shapes with one and up to 47 CTAs, a
    partial last warp and lines shorter than a warp; the IC(0) and ILU(0)
    applies (FP64) equal the restatement bit for bit (applied twice, so the
    second launch runs on the advanced epoch), and the FP32 factors' applies
    equal an FP32 emulation of the schedules' arithmetic bit for bit."""
    n, rp, ci, v = P.diffusion2d(nx, ny, seed=nx * ny)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    r = b2s.uniform(nx + ny, n)
    for kind in ("ic0", "ilu0"):
        M = b2s.Precond(ctx, A, b2s.PC_NAMES[kind])
        assert M.sizes("trsv.grid5") == (nx, ny, 1), kind
        po = orc.pc(orc.csr(n, n, rp, ci, v), kind)
        want = po.apply(r)
        assert np.array_equal(M.apply(r), want), kind
        assert np.array_equal(M.apply(r), want), kind
    for kind in ("ic0", "ilu0"):
        M32 = b2s.Precond(ctx, A, b2s.PC_NAMES[kind], precision=b2s.FP32)
        assert M32.sizes("trsv.grid5") == (nx, ny, 1), kind
        assert np.array_equal(M32.apply(r), _f32_want(M32, kind, r)), kind


def _f32_want(M32, kind, r):
    """The FP32 emulation (_f32_apply) of an FP32 factor's exact apply, from
    the factor the preconditioner exports."""
    n = len(r)
    if kind == "ic0":
        L, U = M32.export("ic0.L"), M32.export("ic0.LT")
        # L^T is stored strict: put the diagonal back from L (rows of L end with it)
        lrp, lci, lv = L
        d = lv[lrp[1:] - 1]
        urp, uci, uv = U
        rows = [(list(uci[urp[i]:urp[i + 1]]), list(uv[urp[i]:urp[i + 1]])) for i in range(n)]
        urp2, uci2, uv2 = [0], [], []
        for i, (c, vv) in enumerate(rows):
            uci2 += [i] + c
            uv2 += [d[i]] + vv
            urp2.append(len(uci2))
        U = (np.array(urp2), np.array(uci2), np.array(uv2))
        return _f32_apply(L, U, r, False)
    return _f32_apply(M32.export("ilu0.L"), M32.export("ilu0.U"), r, True)


@pytest.mark.parametrize("spread,rhs_lo", [(60, -40), (500, -700)])
def test_grid5_division_bit_exact(b2s, ctx, orc, spread, rhs_lo):
    """The grid schedule in FP64 across the binary64 range: a scaled 5-point
    system D A D (D = 2^k, k in [0, spread]) with right-hand sides from
    2^rhs_lo to 2^40; the IC(0) and ILU(0) applies must equal the restatement
    bit for bit."""
    nx, ny = 48, 70
    n, rp, ci, v = P.diffusion2d(nx, ny, seed=spread)
    rng = np.random.default_rng(spread + 1)
    d = np.exp2(rng.integers(0, spread + 1, n).astype(np.float64))
    rows = np.repeat(np.arange(n), np.diff(rp.astype(np.int64)))
    vs = v * d[rows] * d[ci]
    A = b2s.CSR(ctx, n, n, rp, ci, vs)
    r = b2s.uniform(37, n) * np.exp2(rng.integers(rhs_lo, 41, n).astype(np.float64))
    for kind in ("ic0", "ilu0"):
        M = b2s.Precond(ctx, A, b2s.PC_NAMES[kind])
        assert M.sizes("trsv.grid5") == (nx, ny, 1), kind
        po = orc.pc(orc.csr(n, n, rp, ci, vs), kind)
        assert np.array_equal(M.apply(r), po.apply(r)), kind


@pytest.mark.parametrize("nx,ny,nz", [(9, 40, 5), (33, 33, 3), (4, 70, 6), (64, 16, 9), (17, 96, 4), (12, 12, 12)])
def test_grid7_exact_solves(b2s, ctx, orc, nx, ny, nz):
    """7-point grid factors take the plane-by-plane grid schedule (exported as
    "trsv.grid7"): one warp per 32 lines of a plane, the plane's last line
    handed to the next block and every value to the next plane as
    epoch-tagged words.  Shapes with partial warps, up to 3 blocks per plane,
    lines shorter than a warp and up to 12 planes; the IC(0) and ILU(0)
    applies (FP64) equal the restatement bit for bit (applied twice: the
    second launch runs on the advanced epoch), and the FP32 factors' applies
    equal the FP32 emulation bit for bit."""
    n, rp, ci, v = P.diffusion3d(nx, ny, nz, seed=nx * ny + nz)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    r = b2s.uniform(nx + ny + nz, n)
    for kind in ("ic0", "ilu0"):
        M = b2s.Precond(ctx, A, b2s.PC_NAMES[kind])
        assert M.sizes("trsv.grid7") == (nx, ny, nz), kind
        assert M.sizes("trsv.grid5")[0] == 0, kind
        po = orc.pc(orc.csr(n, n, rp, ci, v), kind)
        want = po.apply(r)
        assert np.array_equal(M.apply(r), want), kind
        assert np.array_equal(M.apply(r), want), kind
    for kind in ("ic0", "ilu0"):
        M32 = b2s.Precond(ctx, A, b2s.PC_NAMES[kind], precision=b2s.FP32)
        assert M32.sizes("trsv.grid7") == (nx, ny, nz), kind
        assert np.array_equal(M32.apply(r), _f32_want(M32, kind, r)), kind


def test_grid7_division_bit_exact(b2s, ctx, orc):
    """The 7-point grid schedule in FP64 across the binary64 range (scaled
    system D A D, D = 2^k with k in [0, 500], right-hand sides from 2^-700
    to 2^40: quotients reach the subnormal range, so groups are redone with
    the division); IC(0) and ILU(0) applies equal the restatement bit for bit."""
    nx, ny, nz = 20, 36, 5
    n, rp, ci, v = P.diffusion3d(nx, ny, nz, seed=5)
    rng = np.random.default_rng(6)
    d = np.exp2(rng.integers(0, 501, n).astype(np.float64))
    rows = np.repeat(np.arange(n), np.diff(rp.astype(np.int64)))
    vs = v * d[rows] * d[ci]
    A = b2s.CSR(ctx, n, n, rp, ci, vs)
    r = b2s.uniform(41, n) * np.exp2(rng.integers(-700, 41, n).astype(np.float64))
    for kind in ("ic0", "ilu0"):
        M = b2s.Precond(ctx, A, b2s.PC_NAMES[kind])
        assert M.sizes("trsv.grid7") == (nx, ny, nz), kind
        po = orc.pc(orc.csr(n, n, rp, ci, vs), kind)
        assert np.array_equal(M.apply(r), po.apply(r)), kind


def test_grid5_not_taken_elsewhere(b2s, ctx):
    """Patterns that are not a 5-point grid's (7-point 3-D, random) and grids
    with more than 4096 lines keep the chunked schedule."""
    for n, rp, ci, v in (b2s.gen_poisson3d(12), P.random_spd(1500, 0.004, 3), P.diffusion2d(3, 4200, seed=3)):
        A = b2s.CSR(ctx, n, n, rp, ci, v)
        assert b2s.Precond(ctx, A, b2s.PC_IC0).sizes("trsv.grid5")[0] == 0
    # nor the 7-point schedule: random, 2-D, and a 3-D grid with one point per line
    for n, rp, ci, v in (P.random_spd(1500, 0.004, 3), P.diffusion2d(40, 40, seed=4), P.diffusion3d(1, 30, 20, seed=4)):
        A = b2s.CSR(ctx, n, n, rp, ci, v)
        assert b2s.Precond(ctx, A, b2s.PC_IC0).sizes("trsv.grid7")[0] == 0


@pytest.mark.parametrize("mat", ["poisson2d", "random", "poisson3d"])
@pytest.mark.parametrize("trsv", [1, 2, 3])
def test_ilu0_bit_exact(b2s, ctx, orc, mat, trsv):
    n, rp, ci, v = MATS[mat](b2s) if mat != "poisson2d" else P.convdiff2d(40)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    M = b2s.Precond(ctx, A, b2s.PC_ILU0, trsv=trsv)
    po = orc.pc(orc.csr(n, n, rp, ci, v), "ilu0")
    e = orc.ilu0_export(po)
    for what, (krp, kci, kv) in (("ilu0.L", ("Lrp", "Lci", "Lv")), ("ilu0.U", ("Urp", "Uci", "Uv"))):
        rp_, ci_, v_ = M.export(what)
        assert np.array_equal(rp_, e[krp]) and np.array_equal(ci_, e[kci]) and np.array_equal(v_, e[kv]), what
    r = b2s.uniform(22, n)
    assert np.array_equal(M.apply(r), po.apply(r))


@pytest.mark.parametrize("kind", ["ic0", "ilu0"])
def test_fp32_factor_apply(b2s, ctx, kind):
    n, rp, ci, v = b2s.gen_grf_diffusion(64, seed=2)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    k = b2s.PC_NAMES[kind]
    r = b2s.uniform(23, n)
    z64 = b2s.Precond(ctx, A, k).apply(r)
    for trsv in (1, 2, 3):
        z32 = b2s.Precond(ctx, A, k, precision=b2s.FP32, trsv=trsv).apply(r)
        assert rel(z32, z64) < 1e-5


def test_ic0_not_spd_and_missing_diag(b2s, ctx):
    n, rp, ci, v = P.poisson2d(8)
    v2 = v.copy()
    rows = np.repeat(np.arange(n), np.diff(rp))
    v2[(rows == ci) & (rows == 10)] = 0.5
    with pytest.raises(RuntimeError) as e:
        b2s.Precond(ctx, b2s.CSR(ctx, n, n, rp, ci, v2), b2s.PC_IC0)
    assert e.value.status == b2s.NOT_SPD
    keep = ~((rows == ci) & (rows == 7))
    rp3 = np.concatenate([[0], np.cumsum(np.bincount(rows[keep], minlength=n))]).astype(np.uint32)
    for kind in (b2s.PC_IC0, b2s.PC_ILU0):
        with pytest.raises(RuntimeError) as e:
            b2s.Precond(ctx, b2s.CSR(ctx, n, n, rp3, ci[keep], v[keep]), kind)
        assert e.value.status == b2s.MISSING_DIAG


@pytest.mark.parametrize("method,pc", [(0, "ic"), (0, "ilu"), (1, "ilu"), (2, "ilu"), (2, "ic")])
def test_solver_parity_ilu(b2s, ctx, orc, method, pc):
    # IC(0) needs an SPD matrix: GMRES + "ic" runs on the Poisson matrix
    n, rp, ci, v = P.poisson2d(50) if (method == 0 or pc == "ic") else P.convdiff2d(50)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(31, n)
    M = b2s.Precond(ctx, A, b2s.pc_kind_from_name(method, pc))
    x, st = b2s.solve(ctx, A, b, method, M, tol=1e-8, maxit=2000, restart=30)
    xo, io = orc.solve(orc.csr(n, n, rp, ci, v), method, pc, b, 1e-8, 2000, 30)
    assert abs(st["it"] - io) <= 2, (st["it"], io)
    assert rel(x, xo) < 1e-9
    assert st["relres_true"] < 1.5e-8


def test_ic0_nonsymmetric_raises_like_reference(b2s, ctx, orc):
    # the reference's IC(0) throws std::runtime_error on a non-positive pivot
    # (array.cpp:2649); on the upwind convection-diffusion matrix both
    # sides stop at setup
    n, rp, ci, v = P.convdiff2d(50)
    b = b2s.uniform(31, n)
    with pytest.raises(oracle.OracleError):
        orc.solve(orc.csr(n, n, rp, ci, v), 2, "ic", b, 1e-8, 2000, 30)
    with pytest.raises(RuntimeError) as e:
        b2s.Precond(ctx, b2s.CSR(ctx, n, n, rp, ci, v), b2s.pc_kind_from_name(2, "ic"))
    assert e.value.status == b2s.NOT_SPD


def test_grf_ic0_pcg_parity(b2s, ctx, orc):
    """64^2 GRF diffusion (k spans several decades).  The compiled reference's
    own solutions at 1, 2, 3, 4, 8 and 16 OpenMP threads differ by at most
    2.2e-15 (relative) on this system, with the same 89 iterations; the GPU's
    reduction tree is one more association of the same dots."""
    n, rp, ci, v = b2s.gen_grf_diffusion(64, seed=11)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(11, n)
    M = b2s.Precond(ctx, A, b2s.PC_IC0)
    x, st = b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-8, maxit=5000)
    xo, io = orc.solve(orc.csr(n, n, rp, ci, v), 0, "ic", b, 1e-8, 5000)
    assert abs(st["it"] - io) <= 2
    assert rel(x, xo) < 100 * 2.2e-15, rel(x, xo)


@pytest.mark.parametrize("schedule", ["chunk", "grid7"])
def test_chunk_wait_timeout_reported(b2s, ctx, schedule):
    """The exact solves' waits are bounded per launch.  With the bounds cut to
    one poll and no sleeps, the ILU(0) apply on the 128^3 Poisson matrix
    gives up: on the 7-point grid schedule (512 warps, each waiting on the
    warps of the block and plane before it), and on the chunked schedule
    (hundreds of chunks, each needing rows the chunk before it is still
    computing; one symmetric pair of entries added at rows 0 and 2 keeps the
    pattern off the grid schedule).  The call reports B2S_TIMEOUT and
    returns at once, every later wait of the launch skipped.  The context
    stays usable: with the default bounds the same apply gives the exact
    result again."""
    import time
    n, rp, ci, v = b2s.gen_poisson3d(128)
    if schedule == "chunk":
        rp = rp.astype(np.int64)
        # row 0 gets (0, 2) after its entry (0, 1); row 2 gets (2, 0) first
        p0 = int(np.searchsorted(ci[rp[0]:rp[1]], 2)) + rp[0]
        ci = np.insert(ci, p0, 2)
        v = np.insert(v, p0, -0.01)
        rp[1:] += 1
        ci = np.insert(ci, rp[2], 0)
        v = np.insert(v, rp[2], -0.01)
        rp[3:] += 1
        rp = rp.astype(np.uint32)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    M = b2s.Precond(ctx, A, b2s.PC_ILU0)
    assert (M.sizes("trsv.grid7")[0] > 0) == (schedule == "grid7")
    r = b2s.uniform(21, n)
    z0 = M.apply(r)
    ctx.set_wait_limits(1, 0)
    try:
        t0 = time.perf_counter()
        with pytest.raises(RuntimeError) as e:
            M.apply(r)
        dt = time.perf_counter() - t0
    finally:
        ctx.set_wait_limits(0, 0)
    assert e.value.status == b2s.TIMEOUT
    assert dt < 0.5, dt
    assert np.array_equal(M.apply(r), z0)


@pytest.mark.parametrize("kind", ["ic0", "ilu0"])
def test_jacobi_sweeps_exact_beyond_depth(b2s, ctx, kind):
    """B2S_TRSV_JACOBI is a truncated Neumann series of a nilpotent iteration:
    after as many sweeps as the triangle's DAG depth (23 levels on 12x12) it
    reproduces the exact FP64 solve bit for bit (same per-row order)."""
    n, rp, ci, v = P.poisson2d(12) if kind == "ic0" else P.convdiff2d(12)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    k = b2s.PC_NAMES[kind]
    r = b2s.uniform(41, n)
    z = b2s.Precond(ctx, A, k).apply(r)
    zj = b2s.Precond(ctx, A, k, trsv=b2s.TRSV_JACOBI, trsv_sweeps=24).apply(r)
    assert np.array_equal(zj, z)
    # fewer sweeps: an approximation, not the solve
    z2 = b2s.Precond(ctx, A, k, trsv=b2s.TRSV_JACOBI, trsv_sweeps=2).apply(r)
    assert not np.array_equal(z2, z)


def _sweeps_f32(rp, ci, vals, d, r, k, lower, S=1):
    """Pass 0 (each segment of S rows solved on its own) and k sweeps in
    float32: rows of a segment in dependency order, each row's strict entries
    in column order (current-pass values inside the segment, previous-pass
    values outside), one rounding per product and difference, then a product
    with the float32 reciprocal 1/d -- the kernels' arithmetic."""
    n = len(rp) - 1
    rows = np.repeat(np.arange(n), np.diff(rp))
    strict = (ci < rows) if lower else (ci > rows)
    rr, cc, vv = rows[strict], ci[strict].astype(np.int64), vals[strict].astype(np.float32)
    slot = np.zeros(len(rr), np.int64)
    for t in range(1, len(rr)):
        slot[t] = slot[t - 1] + 1 if rr[t] == rr[t - 1] else 0
    W = int(slot.max()) + 1 if len(rr) else 0
    d32, r32 = d.astype(np.float32), r.astype(np.float32)
    dinv = np.float32(1.0) / d32
    inside = (cc // S) == (rr // S)
    pos = rr % S
    yprev = None
    for s in range(k + 1):
        y = np.zeros(n, np.float32)
        acc = r32.copy()
        for q in (range(S) if lower else range(S - 1, -1, -1)):
            rows_q = np.arange(q, n, S)
            for e in range(W):
                m = (slot == e) & (pos == q)
                use = m & (inside | (s > 0))
                src = np.where(inside[use], y[cc[use]], yprev[cc[use]] if s > 0 else np.float32(0))
                acc[rr[use]] = acc[rr[use]] - vv[use] * src.astype(np.float32)
            y[rows_q] = acc[rows_q] * dinv[rows_q]
        yprev = y
    return y


@pytest.mark.parametrize("seg", [1, 8])
def test_jacobi_band_kernel_bit_exact_f32(b2s, ctx, seg):
    """FP32 IC(0) with 5 sweeps on a 96x96 grid (bandwidth 96: the one-launch
    banded kernel) against a float32 emulation of the passes, bit for bit;
    plain Jacobi (segment 1) and 8-row Gauss-Seidel segments."""
    import scipy.sparse as sp
    n, rp, ci, v = b2s.gen_grf_diffusion(96, seed=12, corr=0.1)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    M = b2s.Precond(ctx, A, b2s.PC_IC0, precision=b2s.FP32, trsv=b2s.TRSV_JACOBI, trsv_sweeps=5,
                    trsv_segment=seg)
    Lrp, Lci, Lv = M.export("ic0.L")
    d = sp.csr_matrix((Lv, Lci, Lrp), shape=(n, n)).diagonal()
    LT = sp.csr_matrix((Lv, Lci, Lrp), shape=(n, n)).T.tocsr()
    LT.sort_indices()
    r = b2s.uniform(43, n)
    y = _sweeps_f32(Lrp, Lci, Lv, d, r, 5, True, seg)
    z = _sweeps_f32(LT.indptr, LT.indices, LT.data, d, y, 5, False, seg)
    assert np.array_equal(M.apply(r), z.astype(np.float64))


def test_segment_global_kernel_bit_exact_f32(b2s, ctx):
    """A 12-row segment is not a banded-kernel width, so the one-launch-per-pass
    kernel runs; it must match the float32 emulation bit for bit."""
    import scipy.sparse as sp
    n, rp, ci, v = b2s.gen_grf_diffusion(40, seed=13, corr=0.1)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    M = b2s.Precond(ctx, A, b2s.PC_IC0, precision=b2s.FP32, trsv=b2s.TRSV_JACOBI, trsv_sweeps=3,
                    trsv_segment=12)
    Lrp, Lci, Lv = M.export("ic0.L")
    L = sp.csr_matrix((Lv, Lci, Lrp), shape=(n, n))
    d = L.diagonal()
    LT = L.T.tocsr()
    LT.sort_indices()
    r = b2s.uniform(44, n)
    y = _sweeps_f32(Lrp, Lci, Lv, d, r, 3, True, 12)
    z = _sweeps_f32(LT.indptr, LT.indices, LT.data, d, y, 3, False, 12)
    assert np.array_equal(M.apply(r), z.astype(np.float64))


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_jacobi_sweeps_match_series(b2s, ctx, orc, prec):
    """k sweeps against the series computed with numpy from the exported
    IC(0) factor: y = D^-1 r, k times y = D^-1 (r - N y); then the same on
    L^T.  FP64 to 1e-13, FP32 to 1e-5 (relative)."""
    import scipy.sparse as sp
    n, rp, ci, v = b2s.gen_grf_diffusion(40, seed=8)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    fp = b2s.FP32 if prec == "fp32" else b2s.FP64
    M = b2s.Precond(ctx, A, b2s.PC_IC0, precision=fp, trsv=b2s.TRSV_JACOBI, trsv_sweeps=3, trsv_segment=1)
    Lrp, Lci, Lv = M.export("ic0.L")
    L = sp.csr_matrix((Lv, Lci, Lrp), shape=(n, n))
    d = L.diagonal()
    N = sp.tril(L, -1).tocsr()
    r = b2s.uniform(42, n)
    y = r / d
    for _ in range(3):
        y = (r - N @ y) / d
    z = y / d
    for _ in range(3):
        z = (y - N.T @ z) / d
    tol = 1e-5 if prec == "fp32" else 1e-13
    assert rel(M.apply(r), z) < tol


def test_jacobi_sweeps_pcg(b2s, ctx):
    """PCG with 8-sweep IC(0) applies (FP32) converges to the FP64-verified
    tolerance within 15 % of the exact solves' iteration count."""
    n, rp, ci, v = b2s.gen_grf_diffusion(128, seed=2003, corr=0.05)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(3, n)
    _, s0 = b2s.solve(ctx, A, b, b2s.PCG, b2s.Precond(ctx, A, b2s.PC_IC0, precision=b2s.FP32), tol=1e-8, maxit=5000)
    Mj = b2s.Precond(ctx, A, b2s.PC_IC0, precision=b2s.FP32, trsv=b2s.TRSV_JACOBI, trsv_sweeps=8)
    _, sj = b2s.solve(ctx, A, b, b2s.PCG, Mj, tol=1e-8, maxit=5000)
    assert sj["status"] == 0 and sj["relres_true"] < 1e-8
    assert sj["iterations"] <= 1.15 * s0["iterations"], (sj["iterations"], s0["iterations"])


def test_jacobi_mode_checks(b2s, ctx):
    n, rp, ci, v = P.poisson2d(8)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    with pytest.raises(ValueError) as e:
        b2s.Precond(ctx, A, b2s.PC_IC0, trsv=7)
    assert e.value.status == b2s.INVALID_ARG
    with pytest.raises(ValueError) as e:
        b2s.Precond(ctx, A, b2s.PC_IC0, trsv=b2s.TRSV_JACOBI, trsv_sweeps=-1)
    assert e.value.status == b2s.INVALID_ARG
    with pytest.raises(ValueError) as e:
        b2s.Precond(ctx, A, b2s.PC_IC0, trsv=b2s.TRSV_JACOBI, trsv_segment=33)
    assert e.value.status == b2s.INVALID_ARG
    nb, brp, bci, bv = b2s.gen_elasticity_q1(3)
    B = b2s.BAIJ(ctx, 3, nb, nb, brp, bci, bv)
    with pytest.raises(b2s.B2SError) as e:
        b2s.Precond(ctx, B, b2s.PC_BILU0, trsv=b2s.TRSV_JACOBI)
    assert e.value.status == b2s.UNSUPPORTED


def test_fused_pcg_iteration_graph_and_polling_invariant(b2s, ctx):
    """With 8-row segments the banded sweep preconditioner runs PCG as three
    fused launches per iteration with the residual and direction in
    alternating buffers.  The result must not depend on how the iterations
    are batched: CUDA graphs on or off, and any polling interval (an odd one
    is rounded up to keep the buffer roles), give the same iterate bit for
    bit."""
    n, rp, ci, v = b2s.gen_grf_diffusion(128, seed=2005, corr=0.05)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(5, n)
    M = b2s.Precond(ctx, A, b2s.PC_IC0, precision=b2s.FP32, trsv=b2s.TRSV_JACOBI, trsv_sweeps=4, trsv_segment=8)
    runs = [b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-8, maxit=5000, use_graphs=g, check_every=c)
            for g, c in ((1, 0), (0, 0), (1, 3), (0, 5))]
    x0, s0 = runs[0]
    assert s0["status"] == 0 and s0["relres_true"] < 1e-8
    for x, s in runs[1:]:
        assert np.array_equal(x, x0) and s["iterations"] == s0["iterations"]


def test_fused_pcg_matches_host_pcg(b2s, ctx):
    """Fused PCG with the 8-sweep FP32 IC(0) against a float64 host PCG with
    the same (float64) sweep preconditioner: iteration counts within 3, and
    both iterates meet the tolerance."""
    import scipy.sparse as sp
    n, rp, ci, v = b2s.gen_grf_diffusion(64, seed=2006, corr=0.1)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(6, n)
    M = b2s.Precond(ctx, A, b2s.PC_IC0, precision=b2s.FP32, trsv=b2s.TRSV_JACOBI, trsv_sweeps=8, trsv_segment=1)
    x, st = b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-8, maxit=5000)
    Lrp, Lci, Lv = M.export("ic0.L")
    L = sp.csr_matrix((Lv, Lci, Lrp), shape=(n, n))
    d = L.diagonal()
    N = sp.tril(L, -1).tocsr()
    Ah = sp.csr_matrix((v, ci, rp), shape=(n, n))

    def pc(r):
        y = r / d
        for _ in range(8):
            y = (r - N @ y) / d
        z = y / d
        for _ in range(8):
            z = (y - N.T @ z) / d
        return z

    xh = np.zeros(n)
    r = b.copy()
    z = pc(r)
    p = z.copy()
    rz = r @ z
    it = 0
    while np.linalg.norm(r) >= 1e-8 * np.linalg.norm(b) and it < 5000:
        Ap = Ah @ p
        a = rz / (p @ Ap)
        xh += a * p
        r -= a * Ap
        it += 1
        if np.linalg.norm(r) < 1e-8 * np.linalg.norm(b):
            break
        z = pc(r)
        rz2 = r @ z
        p = z + (rz2 / rz) * p
        rz = rz2
    assert st["relres_true"] < 1e-8
    assert abs(st["iterations"] - it) <= 3, (st["iterations"], it)


def test_fixed_point_factor_exact_beyond_depth(b2s, ctx):
    """Fixed-point IC(0) sweeps use the exact row arithmetic, so with enough
    sweeps the factor equals the exact factorisation bit for bit: on 12x12
    the DAG has 23 levels and each level takes two sweeps (the off-diagonal
    entries of a row, then its pivot from them), so 50 suffice.  With 3
    sweeps the factor is close but not equal."""
    n, rp, ci, v = P.poisson2d(12)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    exact = b2s.Precond(ctx, A, b2s.PC_IC0).export("ic0.L")[2]
    deep = b2s.Precond(ctx, A, b2s.PC_IC0, factor_sweeps=50).export("ic0.L")[2]
    assert np.array_equal(deep, exact)
    few = b2s.Precond(ctx, A, b2s.PC_IC0, factor_sweeps=3).export("ic0.L")[2]
    assert not np.array_equal(few, exact)
    assert np.abs(few - exact).max() < 1e-2 * np.abs(exact).max()


def test_fixed_point_factor_pcg(b2s, ctx):
    """3 fixed-point sweeps with 8 Jacobi sweeps per triangle (the benchmark's
    learned configuration without the network): PCG meets the FP64-verified
    tolerance within 5% of the exact factor's iterations."""
    n, rp, ci, v = b2s.gen_grf_diffusion(128, seed=2004, corr=0.05)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(4, n)
    opts = dict(precision=b2s.FP32, trsv=b2s.TRSV_JACOBI, trsv_sweeps=8)
    _, s0 = b2s.solve(ctx, A, b, b2s.PCG, b2s.Precond(ctx, A, b2s.PC_IC0, **opts), tol=1e-8, maxit=5000)
    M = b2s.Precond(ctx, A, b2s.PC_IC0, factor_sweeps=3, **opts)
    _, s1 = b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-8, maxit=5000)
    assert s1["status"] == 0 and s1["relres_true"] < 1e-8
    assert s1["iterations"] <= 1.05 * s0["iterations"], (s1["iterations"], s0["iterations"])


def test_fixed_point_factor_errors_like_exact(b2s, ctx):
    n, rp, ci, v = P.poisson2d(8)
    rows = np.repeat(np.arange(n), np.diff(rp))
    v2 = v.copy()
    v2[(rows == ci) & (rows == 10)] = 0.5
    with pytest.raises(RuntimeError) as e:
        b2s.Precond(ctx, b2s.CSR(ctx, n, n, rp, ci, v2), b2s.PC_IC0, factor_sweeps=3)
    assert e.value.status == b2s.NOT_SPD
    keep = ~((rows == ci) & (rows == 7))
    rp3 = np.concatenate([[0], np.cumsum(np.bincount(rows[keep], minlength=n))]).astype(np.uint32)
    with pytest.raises(RuntimeError) as e:
        b2s.Precond(ctx, b2s.CSR(ctx, n, n, rp3, ci[keep], v[keep]), b2s.PC_IC0, factor_sweeps=3)
    assert e.value.status == b2s.MISSING_DIAG


def test_persistent_pcg_matches_launch_per_phase(b2s, ctx):
    """Plain Jacobi sweeps on a banded FP32 factor run the whole PCG loop in
    one cooperative persistent launch.  Against the same sweeps in FP64
    (one launch per sweep, host-driven loop): both meet the tolerance, the
    iteration counts agree within 3 and the iterates to 1e-6."""
    n, rp, ci, v = b2s.gen_grf_diffusion(256, seed=2007, corr=0.05)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(7, n)
    M = b2s.Precond(ctx, A, b2s.PC_IC0, precision=b2s.FP32, trsv=b2s.TRSV_JACOBI, trsv_sweeps=8)
    l0 = ctx.kernel_launches
    x1, s1 = b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-8, maxit=5000)
    launches = ctx.kernel_launches - l0
    assert s1["status"] == 0 and s1["relres_true"] < 1e-8
    assert launches < 20, launches  # setup of the solve + one persistent launch
    ref = b2s.Precond(ctx, A, b2s.PC_IC0, precision=b2s.FP64, trsv=b2s.TRSV_JACOBI, trsv_sweeps=8)
    x2, s2 = b2s.solve(ctx, A, b, b2s.PCG, ref, tol=1e-8, maxit=5000)
    assert s2["status"] == 0 and s2["relres_true"] < 1e-8
    assert abs(s1["iterations"] - s2["iterations"]) <= 3
    assert np.linalg.norm(x1 - x2) <= 1e-6 * np.linalg.norm(x2)


def test_persistent_pcg_stall_guard(b2s, ctx):
    """The persistent loop carries the learned solve's stall guard: with a
    one-iteration window it stops at once and plain IC(0) finishes."""
    n, rp, ci, v = b2s.gen_grf_diffusion(256, seed=2008, corr=0.05)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(8, n)
    M = b2s.Precond(ctx, A, b2s.PC_LEARNED_IC0, precision=b2s.FP32, trsv=b2s.TRSV_JACOBI, trsv_sweeps=8,
                    factor_sweeps=5)
    x, st = b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-8, maxit=20000, stall_window=1)
    assert st["fallbacks"] == 1 and 0 < st["stalled_at"] < st["iterations"]
    assert st["status"] == 0 and st["relres_true"] < 1e-8


@pytest.mark.parametrize("kind,k", [("ic0", 6), ("learned_ic0", 6), ("ic0", 8)])
def test_tiled_persistent_pcg(b2s, ctx, kind, k):
    """The benchmark's configuration on 512^2 GRF systems: FP32 IC(0) (plain
    or learned values, 5 fixed-point sweeps) applied by k Jacobi sweeps per
    triangle.  The 2-D tiled persistent kernel is planned (one CTA per SM at
    most) and runs the whole PCG loop in one launch.  Its rows compute what
    the strip kernel's do, so against it (persistent = 1) and against the
    three-launch iteration (persistent = 2) the iteration counts agree within
    2 and the iterates within 1e-6 (only the dots' association differs), and
    all three meet the FP64-verified tolerance."""
    n, rp, ci, v = b2s.gen_grf_diffusion(512, 2011, corr=0.05)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(2011, n)
    M = b2s.Precond(ctx, A, b2s.PC_NAMES[kind], precision=b2s.FP32, trsv=b2s.TRSV_JACOBI, trsv_sweeps=k,
                    factor_sweeps=5)
    ntiles, q, smem = M.sizes("pcg.tiles")
    assert 0 < ntiles <= 148 and 1 <= q <= 4 and smem <= 227 * 1024, (ntiles, q, smem)
    runs = {}
    for mode in (b2s.PERSIST_AUTO, b2s.PERSIST_STRIPS, b2s.PERSIST_OFF):
        l0 = ctx.kernel_launches
        x, st = b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-8, maxit=20000, stall_window=-1, persistent=mode)
        runs[mode] = (x, st, ctx.kernel_launches - l0)
        assert st["status"] == 0 and st["relres_true"] < 1e-8, (mode, st)
    x0, s0, l0 = runs[b2s.PERSIST_AUTO]
    assert l0 < 20, l0  # the solve's setup launches and one persistent launch
    for mode in (b2s.PERSIST_STRIPS, b2s.PERSIST_OFF):
        x1, s1, _ = runs[mode]
        assert abs(s1["iterations"] - s0["iterations"]) <= 2, (mode, s0["iterations"], s1["iterations"])
        assert np.linalg.norm(x1 - x0) <= 1e-6 * np.linalg.norm(x1)


def test_tiled_pcg_small_grid_and_repeat(b2s, ctx):
    """A 64^2 grid (tiles of a few dozen rows, one row per thread) and a
    repeated solve with the same preconditioner: the same iterate bit for
    bit (the all-reduce sums in tile order) and the FP64 tolerance met."""
    n, rp, ci, v = b2s.gen_grf_diffusion(64, 2012, corr=0.1)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(2012, n)
    M = b2s.Precond(ctx, A, b2s.PC_IC0, precision=b2s.FP32, trsv=b2s.TRSV_JACOBI, trsv_sweeps=4)
    assert M.sizes("pcg.tiles")[0] > 0
    x1, s1 = b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-10, maxit=5000)
    x2, s2 = b2s.solve(ctx, A, b, b2s.PCG, M, tol=1e-10, maxit=5000)
    assert s1["status"] == 0 and s1["relres_true"] < 1e-10
    assert np.array_equal(x1, x2) and s1["iterations"] == s2["iterations"]


@pytest.mark.parametrize("nx,ny,k", [(160, 120, 6), (90, 300, 4), (200, 200, 8)])
def test_tiled_grid_blobs_match_general_planner(b2s, ctx, monkeypatch, nx, ny, k):
    """A 5-point grid's tiles are laid out from closed forms and their index
    blobs built on the device; the general breadth-first planner (host) must
    give the same plan and the same blobs byte for byte, and the two
    preconditioners the same PCG iterate bit for bit."""
    from problems import diffusion2d
    n, rp, ci, v = diffusion2d(nx, ny, seed=nx + ny + k)
    A = b2s.CSR(ctx, n, n, rp, ci, v)
    b = b2s.uniform(nx * ny, n)
    opts = dict(precision=b2s.FP32, trsv=b2s.TRSV_JACOBI, trsv_sweeps=k)
    monkeypatch.delenv("B2S_TILE_PLANNER", raising=False)
    M_grid = b2s.Precond(ctx, A, b2s.PC_IC0, **opts)
    monkeypatch.setenv("B2S_TILE_PLANNER", "bfs")
    M_bfs = b2s.Precond(ctx, A, b2s.PC_IC0, **opts)
    monkeypatch.delenv("B2S_TILE_PLANNER")
    assert M_grid.sizes("pcg.tiles")[0] > 0
    assert M_grid.sizes("pcg.tiles") == M_bfs.sizes("pcg.tiles")
    _, blob_grid, _ = M_grid.export("pcg.tiles.idx")
    _, blob_bfs, _ = M_bfs.export("pcg.tiles.idx")
    assert blob_grid.size > 0 and np.array_equal(blob_grid, blob_bfs)
    x1, s1 = b2s.solve(ctx, A, b, b2s.PCG, M_grid, tol=1e-8, maxit=5000)
    x2, s2 = b2s.solve(ctx, A, b, b2s.PCG, M_bfs, tol=1e-8, maxit=5000)
    assert s1["status"] == 0 and s1["relres_true"] < 1e-8
    assert s1["iterations"] == s2["iterations"] and np.array_equal(x1, x2)
