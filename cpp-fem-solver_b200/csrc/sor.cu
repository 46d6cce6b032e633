// Stand-alone SOR solvers (SMatrix::sor, array.cpp:3843-3945, and
// SMatrix::sor_rb, array.cpp:3946-4189), from x0 = 0 until the true relative
// residual ||b - A x|| / ||b|| drops below tol.
//
// Red-black (multicolour) SOR: the reference's colouring and renumbering
// (build_redblack, shared with the SSOR preconditioner); one launch per
// colour updates that colour's rows, whose neighbours all have other
// colours; the residual of the renumbered system follows.
//
// Natural-order SOR: row i uses the new values of its columns j < i and the
// old values of j > i -- a dependency DAG like a lower triangular solve, run
// as one sync-free traversal per sweep (rows in level order, bounded waits),
// the new iterate in a second buffer so no old value is overwritten early.
//
// Every row is updated as the reference does (sigma = b_i minus the
// off-diagonal products in column order; x_i += omega (sigma / d_i - x_i)),
// so the iterates match it bit for bit; the residual norm is a fixed-order
// device reduction.  The residual kernel's last block applies the stopping
// rule on the device (NaN/Inf: B2S_DIVERGED, the reference's runtime_error;
// it_end = it; stop below tol or at max_iter), and the host polls it every
// kSorPoll sweeps.
#include "b2s_internal.cuh"
#include "syncfree.cuh"
#include "trisolve.cuh"
#include "trsv_plan.hpp"

namespace b2s {

namespace {

constexpr int kSorPoll = 16;

__global__ void k_sor_permute(uint32_t n, const double* __restrict__ b, const uint32_t* __restrict__ new_id,
                              double* __restrict__ b2)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b2[new_id[i]] = b[i];
}

__global__ void k_sor_unpermute(uint32_t n, const double* __restrict__ x2, const uint32_t* __restrict__ new_id,
                                double* __restrict__ x)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = x2[new_id[i]];
}

// one colour [lo, hi) of the renumbered system (array.cpp:4138-4152)
__global__ void k_sor_colour(uint32_t lo, uint32_t hi, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                             const double* __restrict__ v, const double* __restrict__ d, const double* __restrict__ b,
                             double* x, double omega, const int* done)
{
    if (*done) return;
    for (uint32_t ii = lo + blockIdx.x * blockDim.x + threadIdx.x; ii < hi; ii += gridDim.x * blockDim.x)
    {
        double sigma = b[ii];
        for (uint32_t p = rp[ii]; p < rp[ii + 1]; ++p)
        {
            const uint32_t j = ci[p];
            if (j == ii) continue;
            sigma -= v[p] * x[j];  // neighbours have other colours: read only in this launch
        }
        x[ii] += omega * (sigma / d[ii] - x[ii]);
    }
}

// ||b - A x||^2 in a fixed order, then the stopping rule (array.cpp:3917-3943)
__global__ void __launch_bounds__(kThreads) k_sor_residual(uint32_t n, const uint32_t* __restrict__ rp,
                                                           const uint32_t* __restrict__ ci,
                                                           const double* __restrict__ v,
                                                           const double* __restrict__ b,
                                                           const double* __restrict__ x, KState* st, double* partial,
                                                           unsigned int* counter)
{
    if (st->done) return;
    double acc[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        double ri = b[i];
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p) ri -= v[p] * x[ci[p]];
        acc[0] += ri * ri;
    }
    if (grid_reduce_last<1>(acc, partial, counter) && threadIdx.x == 0)
    {
        const double normr = sqrt(acc[0]);
        st->normr = normr;
        st->relres = normr / st->normb;
        if (!isfinite(normr))
        {
            st->status = B2S_DIVERGED;
            st->done = 1;
            return;
        }
        st->it_end = st->it;
        st->iters = st->it + 1;
        if (st->relres < st->tol)
        {
            st->done = 1;
            return;
        }
        st->it += 1;
        if (st->it >= st->maxit) st->done = 1;
    }
}

// natural-order Gauss-Seidel / SOR row (array.cpp:3904-3915): new values of
// j < i (published by the traversal), old values of j > i
struct SorRowOp
{
    const uint32_t *rp, *ci;
    const double *v, *d, *b, *xold;
    double* xnew;
    double omega;
    __device__ bool ready(uint32_t row, const uint32_t* flags, uint32_t epoch) const
    {
        return deps_ready<true>(row, rp, ci, flags, epoch);
    }
    __device__ void compute(uint32_t row) const
    {
        double sigma = b[row];
        for (uint32_t p = rp[row]; p < rp[row + 1]; ++p)
        {
            const uint32_t j = ci[p];
            if (j == row) continue;
            sigma -= v[p] * (j < row ? __ldcg(&xnew[j]) : xold[j]);
        }
        xnew[row] = xold[row] + omega * (sigma / d[row] - xold[row]);
    }
};

__global__ void k_sor_diag(uint32_t n, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                           const double* __restrict__ v, double* __restrict__ d, int* bad)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        double dv = 0.0;
        bool found = false;
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
            if (ci[p] == i)
            {
                dv = v[p];
                found = true;
                break;
            }
        d[i] = dv;
        if (!found || fabs(dv) < 1e-300) atomicMin(bad, (int)i);
    }
}

struct SorResult
{
    int it = 0, iters = 0, status = B2S_OK;
    double relres = 0.0;
    float ms = 0.f;
};

// polls the device stopping rule; returns the final state
template <typename Sweep>
KState sor_iterate(b2s_ctx* ctx, Sweep&& sweep)
{
    KState h;
    for (;;)
    {
        for (int k = 0; k < kSorPoll; ++k) sweep();
        d2h(ctx, &h, ctx->kstate.p, sizeof(KState));
        sync(ctx);
        if (h.done) return h;
    }
}

SorResult run_sor(b2s_ctx* ctx, const CsrDev& A, bool red_black, double omega, double tol, int maxit, const double* b,
                  double* x)
{
    need(A.n == A.m, B2S_SHAPE, red_black ? "red-black SOR needs a square matrix" : "SOR needs a square matrix");
    need(maxit >= 0, B2S_INVALID_ARG, "SOR: maxit must be >= 0");
    const uint32_t n = A.n;
    SorResult res;
    B2S_CUDA(cudaMemsetAsync(x, 0, (size_t)n * sizeof(double), ctx->stream));
    const double normb = std::sqrt(dot_host(ctx, n, b, b));
    if (normb < 1e-300) return res;  // x = 0, it 0 (before the omega check, as the reference)
    need(omega > 0.0 && omega < 2.0, B2S_INVALID_ARG, "SOR: relaxation factor must satisfy 0 < omega < 2");
    if (maxit == 0) return res;
    KState h0;
    std::memset(&h0, 0, sizeof(h0));
    h0.normb = normb;
    h0.tol = tol;
    h0.maxit = maxit;
    KState* st = ctx->kstate.p;
    h2d(ctx, st, &h0, sizeof(KState));
    const int* done = &st->done;
    const unsigned g = stream_grid(ctx, n);
    reserve_reduction(ctx, g);
    cudaEvent_t e0, e1;
    B2S_CUDA(cudaEventCreate(&e0));
    B2S_CUDA(cudaEventCreate(&e1));
    B2S_CUDA(cudaEventRecord(e0, ctx->stream));
    KState h;
    if (red_black)
    {
        RedBlack rb;
        build_redblack(ctx, A, rb, "red-black SOR");
        DBuf<double> b2(n), x2(n);
        B2S_LAUNCH(ctx, k_sor_permute, g, kThreads, 0, n, b, rb.new_id.p, b2.p);
        B2S_CUDA(cudaMemsetAsync(x2.p, 0, x2.bytes(), ctx->stream));
        h = sor_iterate(ctx, [&] {
            for (uint32_t c = 0; c < rb.ncolor; ++c)
            {
                const uint32_t lo = rb.h_cptr[c], hi = rb.h_cptr[c + 1];
                if (lo >= hi) continue;
                B2S_LAUNCH(ctx, k_sor_colour, stream_grid(ctx, hi - lo), kThreads, 0, lo, hi, rb.rp2.p, rb.ci2.p,
                           rb.v2.p, rb.d2.p, b2.p, x2.p, omega, done);
            }
            B2S_LAUNCH(ctx, k_sor_residual, g, kThreads, 0, n, rb.rp2.p, rb.ci2.p, rb.v2.p, b2.p, x2.p, st,
                       ctx->partial.p, ctx->counter.p);
        });
        B2S_LAUNCH(ctx, k_sor_unpermute, g, kThreads, 0, n, x2.p, rb.new_id.p, x);
    }
    else
    {
        DBuf<double> d(n ? n : 1), xb(n ? n : 1);
        DBuf<int> bad(1);
        const int big = 0x7fffffff;
        h2d(ctx, bad.p, &big, sizeof(int));
        B2S_LAUNCH(ctx, k_sor_diag, g, kThreads, 0, n, A.rp.p, A.ci.p, A.v.p, d.p, bad.p);
        int hb = big;
        d2h(ctx, &hb, bad.p, sizeof(int));
        sync(ctx);
        if (hb != big) fail(B2S_MISSING_DIAG, "SOR failed: row " + std::to_string(hb) + " has no nonzero diagonal");
        // level order of the strict lower DAG
        A.host_pattern(ctx);
        std::vector<uint32_t> lev;
        compute_levels(n, A.h_rp.data(), A.h_ci.data(), true, lev);
        LevelSchedule sched;
        sched.build_host(ctx, lev);
        SyncFree sf;
        sf.init(ctx, n);
        B2S_CUDA(cudaMemsetAsync(xb.p, 0, xb.bytes(), ctx->stream));
        double* buf[2] = {x, xb.p};
        int cur = 0;  // buf[cur] holds the iterate
        h = sor_iterate(ctx, [&] {
            sf.run(ctx, sched.rows.p, false,
                   SorRowOp{A.rp.p, A.ci.p, A.v.p, d.p, b, buf[cur], buf[cur ^ 1], omega}, done);
            cur ^= 1;
            B2S_LAUNCH(ctx, k_sor_residual, g, kThreads, 0, n, A.rp.p, A.ci.p, A.v.p, b, buf[cur], st, ctx->partial.p,
                       ctx->counter.p);
        });
        // the sweeps after the stop skipped their work; the iterate is the
        // buffer written by the last executed sweep (iters sweeps in all)
        const int last = (h.iters & 1) ? 1 : 0;
        if (last == 1) d2d(ctx, x, xb.p, (size_t)n * sizeof(double));
        if (sf.status(ctx) != 0) fail(B2S_TIMEOUT, "SOR: the sweep's dependency wait gave up");
    }
    B2S_CUDA(cudaEventRecord(e1, ctx->stream));
    B2S_CUDA(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&res.ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (h.status == B2S_DIVERGED) fail(B2S_DIVERGED, "SOR diverged: NaN/Inf in the residual (check omega and the matrix)");
    res.it = h.it_end;
    res.iters = h.iters;
    res.status = h.status;
    res.relres = h.relres;
    return res;
}

}  // namespace

}  // namespace b2s

using namespace b2s;

extern "C" {

b2s_status b2s_sor_device(b2s_ctx* ctx, const b2s_csr* A, int red_black, double omega, double tol, int maxit,
                          const double* d_b, double* d_x, b2s_stats* stats)
{
    if (!ctx || !A) return B2S_INVALID_ARG;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    return guarded(ctx, [&] {
        const SorResult r = run_sor(ctx, A->d, red_black != 0, omega, tol, maxit, d_b, d_x);
        if (stats)
        {
            stats->it = r.it;
            stats->iterations = r.iters;
            stats->spmvs = r.iters;
            stats->status = r.status;
            stats->relres = r.relres;
            stats->relres_true = r.relres;
            stats->solve_ms = r.ms;
        }
    });
}

b2s_status b2s_sor(b2s_ctx* ctx, const b2s_csr* A, int red_black, double omega, double tol, int maxit, const double* b,
                   double* x, b2s_stats* stats)
{
    if (!ctx || !A || (A->d.n && (!b || !x))) return B2S_INVALID_ARG;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    return guarded(ctx, [&] {
        need(A->d.n == A->d.m, B2S_SHAPE, red_black ? "red-black SOR needs a square matrix" : "SOR needs a square matrix");
        const uint64_t n = A->d.n;
        DBuf<double> db(n ? n : 1), dx(n ? n : 1);
        h2d(ctx, db.p, b, n * sizeof(double));
        const SorResult r = run_sor(ctx, A->d, red_black != 0, omega, tol, maxit, db.p, dx.p);
        d2h(ctx, x, dx.p, n * sizeof(double));
        sync(ctx);
        if (stats)
        {
            stats->it = r.it;
            stats->iterations = r.iters;
            stats->spmvs = r.iters;
            stats->status = r.status;
            stats->relres = r.relres;
            stats->relres_true = r.relres;
            stats->solve_ms = r.ms;
        }
    });
}

}  // extern "C"
