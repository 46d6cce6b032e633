// Exercises the C++ drop-in headers (include/b2s/math/*.hpp) the way the
// reference's own test programs use sparse::SMatrix and block::BlockMatrix:
// known-answer checks with manufactured solutions, exit code 0 on success.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <vector>

#include "math/array.hpp"
#include "math/blockMatrix.hpp"

using namespace sparse;
using namespace block;

static int failures = 0;
#define CHECK(cond, ...)                        \
    do                                          \
    {                                           \
        if (!(cond))                            \
        {                                       \
            std::printf("FAIL: " __VA_ARGS__);  \
            std::printf("\n");                  \
            ++failures;                         \
        }                                       \
    } while (0)

static double drand(uint32_t i)
{
    double s = std::sin((double)i * 0.371 + 1.7) * 43758.5453;
    return s - std::floor(s);
}

static SMatrix poisson2d(uint32_t N)
{
    std::vector<double> v;
    std::vector<uint32_t> r, c;
    for (uint32_t i = 0; i < N; ++i)
        for (uint32_t j = 0; j < N; ++j)
        {
            const uint32_t k = i * N + j;
            r.push_back(k); c.push_back(k); v.push_back(4.0);
            if (j > 0) { r.push_back(k); c.push_back(k - 1); v.push_back(-1.0); }
            if (j + 1 < N) { r.push_back(k); c.push_back(k + 1); v.push_back(-1.0); }
            if (i > 0) { r.push_back(k); c.push_back(k - N); v.push_back(-1.0); }
            if (i + 1 < N) { r.push_back(k); c.push_back(k + N); v.push_back(-1.0); }
        }
    return SMatrix(N * N, N * N, v, r, c);
}

static double relres(const SMatrix& A, const std::vector<double>& x, const std::vector<double>& b)
{
    auto Ax = SMatrix::spmv(A, x);
    double rr = 0, bb = 0;
    for (size_t i = 0; i < b.size(); ++i) { rr += (b[i] - Ax[i]) * (b[i] - Ax[i]); bb += b[i] * b[i]; }
    return std::sqrt(rr / bb);
}

// 1-D Stokes (test_BlockMatrix_schur.cpp:38-80) with GMRES(50) + Schur(ILU0, I)
static void test_schur_1d(uint32_t N_vel)
{
    const uint32_t N_pres = N_vel - 1, N = N_vel + N_pres;
    std::vector<double> v, vA, vB, vBt;
    std::vector<uint32_t> r, c, rA, cA, rB, cB, rBt, cBt;
    for (uint32_t i = 0; i < N_vel; ++i)
    {
        r.push_back(i); c.push_back(i); v.push_back(2.0);
        if (i > 0) { r.push_back(i); c.push_back(i - 1); v.push_back(-1.0); }
        if (i + 1 < N_vel) { r.push_back(i); c.push_back(i + 1); v.push_back(-1.0); }
    }
    for (uint32_t i = 0; i < N_pres; ++i)
    {
        r.push_back(i + N_vel); c.push_back(i); v.push_back(-1.0);
        r.push_back(i + N_vel); c.push_back(i + 1); v.push_back(1.0);
        r.push_back(i); c.push_back(i + N_vel); v.push_back(-1.0);
        r.push_back(i + 1); c.push_back(i + N_vel); v.push_back(1.0);
    }
    for (size_t k = 0; k < v.size(); ++k)
    {
        if (r[k] < N_vel && c[k] < N_vel) { rA.push_back(r[k]); cA.push_back(c[k]); vA.push_back(v[k]); }
        if (r[k] >= N_vel && c[k] < N_vel) { rB.push_back(r[k] - N_vel); cB.push_back(c[k]); vB.push_back(v[k]); }
        if (r[k] < N_vel && c[k] >= N_vel) { rBt.push_back(r[k]); cBt.push_back(c[k] - N_vel); vBt.push_back(v[k]); }
    }
    SMatrix K(N, N, v, r, c), A(N_vel, N_vel, vA, rA, cA), B(N_pres, N_vel, vB, rB, cB), Bt(N_vel, N_pres, vBt, rBt, cBt);
    SaddlePointSystem sys;
    sys.n_vel = N_vel;
    sys.n_pres = N_pres;
    sys.spmv_A = [A](const std::vector<double>& x, std::vector<double>& y) { y = SMatrix::spmv(A, x); };
    sys.spmv_B = [B](const std::vector<double>& x, std::vector<double>& y) { y = SMatrix::spmv(B, x); };
    sys.spmv_Bt = [Bt](const std::vector<double>& x, std::vector<double>& y) { y = SMatrix::spmv(Bt, x); };
    auto Ap = SMatrix::make_ilu0_preconditioner(A);
    auto Sp = [](const std::vector<double>& x, std::vector<double>& z) { z = x; };
    auto schur = make_schur_preconditioner(sys, Ap, Sp);
    std::vector<double> xe(N);
    for (uint32_t i = 0; i < N; ++i) xe[i] = drand(i);
    auto b = SMatrix::spmv(K, xe);
    auto [x, it] = SMatrix::gmres(K, b, schur, 50);
    double err = 0;
    for (uint32_t i = 0; i < N; ++i) err += (x[i] - xe[i]) * (x[i] - xe[i]);
    std::printf("[Schur] N_vel=%u GMRES it=%d err=%.3e\n", N_vel, it + 1, std::sqrt(err));
    CHECK(std::sqrt(err) < 1e-6, "Schur 1-D N_vel=%u err=%.3e", N_vel, std::sqrt(err));
    // the device-resident composition (extension): the same iterates
    auto schur_dev = make_schur_preconditioner(sys, B, Bt, Ap);
    auto [xd, itd] = SMatrix::gmres(K, b, schur_dev, 50);
    double dd = 0;
    for (uint32_t i = 0; i < N; ++i) dd = std::max(dd, std::fabs(xd[i] - x[i]));
    CHECK(itd == it && dd == 0.0, "device Schur N_vel=%u: it %d vs %d, max diff %.3e", N_vel, itd, it, dd);
    auto scaled = make_scaled_preconditioner(Ap, 2.0);
    std::vector<double> r1(N_vel), z1, z2;
    for (uint32_t i = 0; i < N_vel; ++i) r1[i] = drand(i + 3);
    Ap(r1, z1);
    scaled(r1, z2);
    bool same = z1.size() == z2.size();
    for (size_t i = 0; same && i < z1.size(); ++i) same = z2[i] == 2.0 * z1[i];
    CHECK(same, "scaled preconditioner");
}

int main()
{
    // PCG with every preconditioner string (array.cpp:3482-3515)
    SMatrix A = poisson2d(64);
    std::vector<double> b(A.rows());
    for (uint32_t i = 0; i < A.rows(); ++i) b[i] = 2.0 * drand(i) - 1.0;
    for (const char* p : {"none", "CG", "diag", "Jacobi", "ic", "incomplete_cholesky", "ilu", "ssor", "amg"})
    {
        auto [x, it] = SMatrix::pcg(A, b, p, 1e-8, 2000);
        const double rr = relres(A, x, b);
        std::printf("[pcg %-20s] it=%4d relres=%.2e\n", p, it, rr);
        CHECK(rr < 2e-8, "pcg %s relres %.3e", p, rr);
    }
    for (const char* p : {"none", "ilu", "ssor"})
    {
        auto [x, it] = SMatrix::bicgstab(A, b, p, 1e-8, 2000);
        CHECK(relres(A, x, b) < 2e-8, "bicgstab %s", p);
        auto [x2, it2] = SMatrix::gmres(A, b, p, 30, 1e-8, 2000);
        CHECK(relres(A, x2, b) < 2e-8, "gmres %s", p);
    }
    // SOR, natural order and red-black (array.hpp:351-365)
    {
        SMatrix S = poisson2d(24);
        std::vector<double> bs(S.rows());
        for (uint32_t i = 0; i < S.rows(); ++i) bs[i] = 2.0 * drand(i + 7) - 1.0;
        auto [xs, its] = SMatrix::sor(S, bs, 1.6, 1e-8, 5000);
        CHECK(relres(S, xs, bs) < 1e-8, "sor relres");
        auto [xr, itr] = SMatrix::sor_rb(S, bs, 1.6, 1e-8, 5000);
        CHECK(relres(S, xr, bs) < 1e-8, "sor_rb relres");
        std::printf("[sor] it=%d  [sor_rb] it=%d\n", its, itr);
        bool bad = false;
        try { SMatrix::sor(S, bs, 2.5); } catch (const std::invalid_argument&) { bad = true; }
        CHECK(bad, "sor with omega >= 2 must throw std::invalid_argument");
    }
    // stand-alone AMG (array.hpp:367-372): x += V-cycle(r) until the true residual passes
    {
        auto [xa, ita] = SMatrix::amg(A, b, 1e-8, 200);
        const double ra = relres(A, xa, b);
        std::printf("[amg] it=%d relres=%.2e\n", ita, ra);
        CHECK(ra < 1e-8 && ita > 0 && ita < 200, "amg relres %.3e it %d", ra, ita);
        auto [x0, it0] = SMatrix::amg(A, std::vector<double>(A.rows(), 0.0));
        CHECK(it0 == 0 && x0.size() == A.rows(), "amg zero rhs");
    }
    // transpose and product on the device (array.cpp:2201-2447)
    {
        const SMatrix T = A.transpose();
        CHECK(T.rows() == A.cols() && T.nnz() == A.nnz() && T.row_ptr() == A.row_ptr() && T.col_idx() == A.col_idx() &&
                  T.values() == A.values(),
              "transpose of a symmetric matrix is itself");
        const SMatrix A2 = A * A;
        const std::vector<double> y1 = SMatrix::spmv(A2, b), y2 = SMatrix::spmv(A, SMatrix::spmv(A, b));
        double e = 0.0, nrm = 0.0;
        for (size_t i = 0; i < y1.size(); ++i) { e = std::max(e, std::fabs(y1[i] - y2[i])); nrm = std::max(nrm, std::fabs(y2[i])); }
        CHECK(e <= 1e-12 * nrm, "(A A) b == A (A b): %.3e", e);
        bool bad = false;
        try { (void)(A * SMatrix(3, 3, std::vector<uint32_t>(4, 0), {}, {})); } catch (const std::invalid_argument&) { bad = true; }
        CHECK(bad, "product with mismatched shapes must throw std::invalid_argument");
    }
    // exceptions
    bool threw = false;
    try { SMatrix::pcg(A, b, "bogus"); } catch (const std::invalid_argument&) { threw = true; }
    CHECK(threw, "unknown preconditioner must throw std::invalid_argument");
    threw = false;
    try { SMatrix::gmres(A, b, "incomplete_cholesky", 30); } catch (const std::invalid_argument&) { threw = true; }
    CHECK(threw, "gmres does not accept incomplete_cholesky");
    threw = false;
    {
        std::vector<double> v = A.values();
        for (uint32_t k = A.row_ptr()[5]; k < A.row_ptr()[6]; ++k)
            if (A.col_idx()[k] == 5) v[k] = -4.0;
        SMatrix Bad(A.rows(), A.cols(), A.row_ptr(), A.col_idx(), v);
        try { SMatrix::pcg(Bad, b, "diag"); } catch (const std::runtime_error&) { threw = true; }
    }
    CHECK(threw, "non-positive diagonal must throw std::runtime_error");
    // zero right-hand side: x = 0, it = 0 before the name is looked at
    {
        auto [x, it] = SMatrix::pcg(A, std::vector<double>(A.rows(), 0.0), "bogus");
        CHECK(it == 0, "zero rhs");
    }
    test_schur_1d(100);
    test_schur_1d(500);
    // block path: T1/T4/T7 of test_BlockMatrix_mpi.cpp on a node-major 2-D grid, BS=3
    {
        const uint32_t N = 48, BS = 3, n = N * N * BS;
        std::vector<double> v;
        std::vector<uint32_t> r, c;
        for (uint32_t i = 0; i < N; ++i)
            for (uint32_t j = 0; j < N; ++j)
            {
                const uint32_t idx = i * N + j;
                for (uint32_t rr = 0; rr < BS; ++rr)
                {
                    const uint32_t row = idx * BS + rr;
                    for (uint32_t cc = 0; cc < BS; ++cc) { r.push_back(row); c.push_back(idx * BS + cc); v.push_back(rr == cc ? 4.0 + BS : 0.1); }
                    if (j > 0) { r.push_back(row); c.push_back((idx - 1) * BS + rr); v.push_back(-1.0); }
                    if (j + 1 < N) { r.push_back(row); c.push_back((idx + 1) * BS + rr); v.push_back(-1.0); }
                    if (i > 0) { r.push_back(row); c.push_back((idx - N) * BS + rr); v.push_back(-1.0); }
                    if (i + 1 < N) { r.push_back(row); c.push_back((idx + N) * BS + rr); v.push_back(-1.0); }
                }
            }
        SMatrix S(n, n, v, r, c);
        using Blk = BlockMatrix<double, 3>;
        Blk Bm = Blk::condense(S, N * N, N * N);
        std::vector<double> x(n), y1, y2;
        for (uint32_t i = 0; i < n; ++i) x[i] = drand(i);
        y1 = SMatrix::spmv(S, x);
        Bm.matvec(x, y2);
        double e = 0;
        for (uint32_t i = 0; i < n; ++i) e = std::max(e, std::fabs(y1[i] - y2[i]));
        CHECK(e < 1e-12, "T1 condense+matvec %.3e", e);
        Bm.distributed_matvec(x, y2);
        CHECK(y2.size() == n, "distributed_matvec");
        std::vector<double> rhs(n);
        for (uint32_t i = 0; i < n; ++i) rhs[i] = 1.0 + 0.5 * drand(i + 7);
        auto [xj, itj] = Blk::gmres(Bm, rhs, "blockjacobi", 1e-8, 3000, 30);
        auto [xi, iti] = Blk::gmres(Bm, rhs, "blockilu", 1e-8, 3000, 30);
        std::printf("[block gmres] jacobi it=%d ilu it=%d\n", itj + 1, iti + 1);
        CHECK(iti <= itj, "T7 block ILU should need no more iterations than block Jacobi");
        auto ilu = make_block_ilu0_preconditioner(Bm);
        auto [xc, itc] = Blk::pcg(Bm, rhs, ilu, 1e-8, 3000);
        std::vector<double> Ax;
        Bm.matvec(xc, Ax);
        double rr = 0, bb = 0;
        for (uint32_t i = 0; i < n; ++i) { rr += (rhs[i] - Ax[i]) * (rhs[i] - Ax[i]); bb += rhs[i] * rhs[i]; }
        CHECK(std::sqrt(rr / bb) < 1e-6, "T4/T7 true residual %.3e", std::sqrt(rr / bb));
        auto amg = make_block_amg_preconditioner(Bm);
        auto [xa, ita] = Blk::pcg(Bm, rhs, amg, 1e-8, 3000);
        std::printf("[block pcg] ilu it=%d amg it=%d\n", itc, ita);
        threw = false;
        try { Blk::gmres(Bm, rhs, "BlockJacobi", 1e-8, 10, 5); } catch (const std::invalid_argument&) { threw = true; }
        CHECK(threw, "block gmres names are case-sensitive");
    }
    std::printf(failures ? "FAILED (%d)\n" : "ALL PASSED\n", failures);
    return failures ? 1 : 0;
}
