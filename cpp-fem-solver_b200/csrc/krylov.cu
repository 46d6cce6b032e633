// Krylov drivers: PCG (SMatrix::pcg, array.cpp:3445-3601), BiCGSTAB
// (SMatrix::bicgstab, array.cpp:3602-3842), restarted GMRES (SMatrix::gmres,
// array.cpp:4190-4533; BlockMatrix::gmres, blockMatrix.hpp:688-866), flexible
// GMRES and iterative refinement.
//
// Every scalar of an iteration (alpha, beta, rho, omega, the Hessenberg column
// and its Givens rotations) lives on the device in a KState / small array and
// is computed by the last CTA of the reduction that produces it, so an
// iteration is a fixed sequence of kernel launches with no host round trip.
// The host enqueues `check_every` iterations (optionally as one CUDA graph),
// then reads the 96-byte state once to see whether the solve has finished.
// Once a kernel epilogue sets `done`, every later kernel returns at entry, so
// the extra iterations enqueued past convergence cost only launch time.
//
// The returned iteration counts follow the reference exactly:
//   stationary (SMatrix::amg) it_end = index of the last residual check
//   pcg      it_end = index of the last fully completed iteration
//   bicgstab it_end = index of the last iteration (it_end = it before the check)
//   gmres    it_end = total Arnoldi steps - 1
#include <cmath>

#include "spmv_staged.cuh"

namespace b2s {

namespace {

constexpr double kBreak = 1e-30;

// ---------------------------------------------------------------- operator

struct Operator
{
    const CsrDev* csr = nullptr;
    const BaijDev* baij = nullptr;
    uint64_t n = 0;
    unsigned red_blocks(const b2s_ctx* ctx) const
    {
        return csr ? std::max(csr->nblk, spmv_grid(ctx, *csr)) : stream_grid(ctx, n);
    }
    void apply(b2s_ctx* ctx, const double* x, double* y, const int* done) const
    {
        if (csr)
            spmv(ctx, *csr, x, y, done);
        else
            baij_matvec(ctx, *baij, x, y, done);
    }
};

// per-row epilogue applied after a BAIJ matvec (the CSR path fuses it into the SpMV)
template <typename Epi>
__global__ void __launch_bounds__(kThreads) k_rows_epi(uint64_t n, const double* __restrict__ y, const int* done, Epi epi,
                                                       double* partial, unsigned int* counter)
{
    if (done && *done) return;
    constexpr int NV = Epi::NV > 0 ? Epi::NV : 1;
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        epi.row((uint32_t)i, y[i], acc);
    if constexpr (Epi::NV > 0)
    {
        if (grid_reduce_last<Epi::NV>(acc, partial, counter))
            if (threadIdx.x == 0) epi.last(acc);
    }
}

// y = A x with a fused epilogue.  For BAIJ the product lands in `tmp` first.
template <typename Epi>
void op_apply_epi(b2s_ctx* ctx, const Operator& A, const double* x, double* tmp, const int* done, const Epi& epi)
{
    if (A.csr)
    {
        launch_spmv(ctx, *A.csr, x, done, epi);
        return;
    }
    baij_matvec(ctx, *A.baij, x, tmp, done);
    const unsigned g = stream_grid(ctx, A.n);
    reserve_reduction(ctx, g);
    B2S_LAUNCH(ctx, k_rows_epi<Epi>, g, kThreads, 0, A.n, tmp, done, epi, ctx->partial.p, ctx->counter.p);
}

// generic grid-stride kernel with reduction
template <typename Body>
__global__ void __launch_bounds__(kThreads) k_vec(uint64_t n, const int* done, Body body, double* partial,
                                                  unsigned int* counter)
{
    if (done && *done) return;
    constexpr int NV = Body::NV > 0 ? Body::NV : 1;
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        body.elem(i, acc);
    if constexpr (Body::NV > 0)
    {
        if (grid_reduce_last<Body::NV>(acc, partial, counter))
            if (threadIdx.x == 0) body.last(acc);
    }
}

template <typename Body>
void launch_vec(b2s_ctx* ctx, uint64_t n, const int* done, const Body& body)
{
    // one wave: no more CTAs than fit at once (bodies with many sums hold more registers)
    static const int occ = [] {
        int o = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_vec<Body>, kThreads, 0) != cudaSuccess) o = 0;
        return o;
    }();
    unsigned g = stream_grid(ctx, n);
    if (occ > 0) g = std::min(g, (unsigned)(occ * ctx->sm_count));
    if (Body::NV > 0) reserve_reduction(ctx, g);
    B2S_LAUNCH(ctx, k_vec<Body>, g, kThreads, 0, n, done, body, ctx->partial.p, ctx->counter.p);
}


// ----------------------------------------------------------------- common

// ||v||^2 -> normb, relres = 1; zero RHS ends the solve (x = 0, it 0)
struct BodyNormB
{
    static constexpr int NV = 1;
    const double* b;
    KState* st;
    __device__ void elem(uint64_t i, double* acc) const { acc[0] += b[i] * b[i]; }
    __device__ void last(const double* t) const
    {
        const double nb = sqrt(t[0]);
        st->normb = nb;
        st->normr = nb;
        st->relres = 1.0;
        st->aux[6] = nb;  // GMRES: beta of the first cycle
        if (nb < 1e-300) finish(st, B2S_OK);
    }
};

// true residual: y = A x arrives per row; acc += (b - y)^2; relres_true in aux[0]
struct EpiTrueRes
{
    static constexpr int NV = 1;
    const double* b;
    KState* st;
    __device__ void row(uint32_t r, double s, double* acc) const
    {
        const double d = b[r] - s;
        acc[0] += d * d;
    }
    __device__ void last(const double* t) const { st->aux[0] = st->normb > 0 ? sqrt(t[0]) / st->normb : 0.0; }
};

// --------------------------------------------------------------------- PCG

struct BodyRZInit  // rz_old = r.z (array.cpp:3524-3531)
{
    static constexpr int NV = 1;
    const double *r, *z;
    double* p;
    KState* st;
    __device__ void elem(uint64_t i, double* acc) const
    {
        p[i] = z[i];
        acc[0] += r[i] * z[i];
    }
    __device__ void last(const double* t) const
    {
        st->rz_old = t[0];
        if (t[0] <= 0.0) finish(st, B2S_NOT_SPD);
    }
};

// p_j = z_j + beta p_old_j formed where the SpMV gathers it (array.cpp:3590-3593)
struct XPNew
{
    const double *z, *p;
    const KState* st;
    double beta;
    __device__ void init() { beta = st->beta; }
    __device__ double at(uint32_t j) const { return __ldg(&z[j]) + beta * __ldg(&p[j]); }
};

struct EpiPAp  // Ap = A p; pAp = p.Ap; checks; alpha (array.cpp:3540-3557)
{
    static constexpr int NV = 1;
    double* Ap;
    const double* p;
    KState* st;
    __device__ void row(uint32_t r, double s, double* acc) const
    {
        Ap[r] = s;
        acc[0] += p[r] * s;
    }
    __device__ void last(const double* t) const
    {
        const double pAp = t[0];
        st->pAp = pAp;
        if (fabs(pAp) < kBreak)
        {
            finish(st, B2S_BREAKDOWN);
            st->iters = st->it + 1;
            return;
        }
        if (pAp <= 0.0)
        {
            finish(st, B2S_NOT_SPD);
            st->iters = st->it + 1;
            return;
        }
        st->alpha = st->rz_old / pAp;
    }
};

// EpiPAp with the direction update folded in: p_new = z + beta p_old (the
// row's own value, stored), Ap = A p_new, pAp = p_new.Ap
struct EpiPApUpd
{
    static constexpr int NV = 1;
    double *Ap, *pnew;
    const double *z, *pold;
    KState* st;
    __device__ void row(uint32_t r, double s, double* acc) const
    {
        const double pr = z[r] + st->beta * pold[r];
        pnew[r] = pr;
        Ap[r] = s;
        acc[0] += pr * s;
    }
    __device__ void last(const double* t) const { EpiPAp{Ap, pnew, st}.last(t); }
};

// residual check at the end of a PCG iteration; returns true when the solve ended



// x += alpha p; r -= alpha Ap; rr = r.r; FUSE 1: z = r, 2: z = r / d (array.cpp:3559-3578)
template <int FUSE>
struct BodyPcgUpdate
{
    static constexpr int NV = FUSE ? 2 : 1;
    double *x, *r, *z;
    const double *p, *Ap, *d;
    KState* st;
    __device__ void elem(uint64_t i, double* acc) const
    {
        const double alpha = st->alpha;
        x[i] += alpha * p[i];
        const double ri = r[i] - alpha * Ap[i];
        r[i] = ri;
        acc[0] += ri * ri;
        if (FUSE)
        {
            const double zi = FUSE == 2 ? ri / d[i] : ri;
            z[i] = zi;
            acc[1] += ri * zi;
        }
    }
    __device__ void last(const double* t) const
    {
        if (pcg_check_converged(st, t[0])) return;
        if (FUSE) pcg_next(st, t[1]);
    }
};

struct BodyRZ  // rz_new = r.z for a separate preconditioner
{
    static constexpr int NV = 1;
    const double *r, *z;
    KState* st;
    __device__ void elem(uint64_t i, double* acc) const { acc[0] += r[i] * z[i]; }
    __device__ void last(const double* t) const { pcg_next(st, t[0]); }
};

struct BodyPUpdate  // p = z + beta p (array.cpp:3590-3593)
{
    static constexpr int NV = 0;
    double* p;
    const double* z;
    const KState* st;
    __device__ void elem(uint64_t i, double*) const { p[i] = z[i] + st->beta * p[i]; }
    __device__ void last(const double*) const {}
};

// ---------------------------------------------------------------- BiCGSTAB

// speculative rho for the next iteration + the checks of array.cpp:3694-3716
__device__ __forceinline__ void bicg_begin(KState* st, double rho_new)
{
    st->rho_new = rho_new;
    if (fabs(rho_new) < kBreak || fabs(st->rho_old) < kBreak || fabs(st->omega) < kBreak)
    {
        st->iters = st->it;
        finish(st, B2S_BREAKDOWN);
        return;
    }
    st->beta = (rho_new / st->rho_old) * (st->alpha / st->omega);
}

struct BodyBicgInit  // rt = r = b; rho_new = rt.r; rho_old = alpha = omega = 1
{
    static constexpr int NV = 1;
    const double* b;
    double *r, *rt, *p, *v;
    KState* st;
    __device__ void elem(uint64_t i, double* acc) const
    {
        const double bi = b[i];
        r[i] = bi;
        rt[i] = bi;
        p[i] = 0.0;
        v[i] = 0.0;
        acc[0] += bi * bi;
    }
    __device__ void last(const double* t) const
    {
        st->rho_old = 1.0;
        st->alpha = 1.0;
        st->omega = 1.0;
        bicg_begin(st, t[0]);
    }
};

struct BodyBicgP  // p = r + beta (p - omega v)
{
    static constexpr int NV = 0;
    double* p;
    const double *r, *v;
    const KState* st;
    __device__ void elem(uint64_t i, double*) const { p[i] = r[i] + st->beta * (p[i] - st->omega * v[i]); }
    __device__ void last(const double*) const {}
};

struct EpiBicgV  // v = A y; rhat_v = rt.v; alpha
{
    static constexpr int NV = 1;
    double* v;
    const double* rt;
    KState* st;
    __device__ void row(uint32_t r, double s, double* acc) const
    {
        v[r] = s;
        acc[0] += rt[r] * s;
    }
    __device__ void last(const double* t) const
    {
        if (fabs(t[0]) < kBreak)
        {
            st->iters = st->it + 1;
            finish(st, B2S_BREAKDOWN);
            return;
        }
        st->alpha = st->rho_new / t[0];
    }
};

struct BodyBicgS  // s = r - alpha v
{
    static constexpr int NV = 0;
    double* s;
    const double *r, *v;
    const KState* st;
    __device__ void elem(uint64_t i, double*) const { s[i] = r[i] - st->alpha * v[i]; }
    __device__ void last(const double*) const {}
};

struct EpiBicgT  // t = A z; tt, ts; omega
{
    static constexpr int NV = 2;
    double* t;
    const double* s;
    KState* st;
    __device__ void row(uint32_t r, double val, double* acc) const
    {
        t[r] = val;
        acc[0] += val * val;
        acc[1] += val * s[r];
    }
    __device__ void last(const double* tot) const
    {
        if (tot[0] < kBreak)
        {
            st->iters = st->it + 1;
            finish(st, B2S_BREAKDOWN);
            return;
        }
        st->omega = tot[1] / tot[0];
    }
};

// x += alpha y + omega z; r = s - omega t; rr; rt.r (array.cpp:3765-3777)
struct BodyBicgXR
{
    static constexpr int NV = 2;
    double *x, *r;
    const double *y, *z, *s, *t, *rt;
    KState* st;
    __device__ void elem(uint64_t i, double* acc) const
    {
        x[i] += st->alpha * y[i] + st->omega * z[i];
        const double ri = s[i] - st->omega * t[i];
        r[i] = ri;
        acc[0] += ri * ri;
        acc[1] += rt[i] * ri;
    }
    __device__ void last(const double* tot) const
    {
        const double normr = sqrt(tot[0]);
        st->normr = normr;
        st->relres = normr / st->normb;
        st->it_end = st->it;
        st->iters = st->it + 1;
        if (st->relres < st->tol)
        {
            st->aux[1] = 1.0;  // the true residual decides
            return;
        }
        if (!(normr == normr) || isinf(normr))
        {
            st->it_end = st->maxit - 1;
            finish(st, B2S_DIVERGED);
            return;
        }
        st->rho_old = st->rho_new;
        st->it += 1;
        if (st->it >= st->maxit)
        {
            finish(st, B2S_OK);
            return;
        }
        bicg_begin(st, tot[1]);
    }
};

// true-residual check with residual replacement (array.cpp:3784-3828):
// r = b - A x, ||r||, rt.r
struct EpiBicgTrue
{
    static constexpr int NV = 2;
    const double *b, *rt;
    double* r;
    KState* st;
    __device__ void row(uint32_t i, double s, double* acc) const
    {
        const double ri = b[i] - s;
        r[i] = ri;
        acc[0] += ri * ri;
        acc[1] += rt[i] * ri;
    }
    __device__ void last(const double* tot) const
    {
        st->aux[1] = 0.0;
        const double tr = sqrt(tot[0]);
        if (tr / st->normb < st->tol)
        {
            st->relres = tr / st->normb;
            finish(st, B2S_OK);
            return;
        }
        st->normr = tr;
        st->relres = tr / st->normb;
        if (fabs(tot[1]) < kBreak)
        {
            finish(st, B2S_OK);  // the reference forces an exit here
            return;
        }
        st->rho_old = tot[1];
        st->it += 1;
        if (st->it >= st->maxit)
        {
            finish(st, B2S_OK);
            return;
        }
        bicg_begin(st, tot[1]);
    }
};

// flag = 1 unless the true-residual check of this iteration was requested
__global__ void k_bicg_guard(const KState* st, int* flag) { *flag = (st->done || st->aux[1] == 0.0) ? 1 : 0; }

// ------------------------------------------------------------------ GMRES

// small device arrays (m = restart): H[(m+1) x m], cs[m], sn[m], g[m+1], y[m]
struct GmSmall
{
    double *H, *cs, *sn, *g, *y;
    int m;
};

// extra KState fields used by GMRES
//   aux[2] = j (current column), aux[3] = j_used, aux[4] = total Arnoldi steps,
//   aux[5] = cycle_end flag, aux[6] = beta of the cycle
__device__ __forceinline__ int gm_j(const KState* st) { return (int)st->aux[2]; }

// V0 = b / normb (first cycle) -- the reference divides
struct BodyGmV0First
{
    static constexpr int NV = 0;
    double* V0;
    const double* b;
    const KState* st;
    __device__ void elem(uint64_t i, double*) const { V0[i] = b[i] / st->normb; }
    __device__ void last(const double*) const {}
};

// restart: V0 = b - A x, rr (array.cpp:4265-4283)
struct EpiGmRestart
{
    static constexpr int NV = 1;
    const double* b;
    double* V0;
    KState* st;
    GmSmall sm;
    __device__ void row(uint32_t i, double s, double* acc) const
    {
        const double ri = b[i] - s;
        V0[i] = ri;
        acc[0] += ri * ri;
    }
    __device__ void last(const double* t) const
    {
        const double beta = sqrt(t[0]);
        st->aux[6] = beta;
        if (beta / st->normb < st->tol)
        {
            st->relres = beta / st->normb;
            finish(st, B2S_OK);
        }
    }
};

struct BodyGmScale  // V0 /= beta
{
    static constexpr int NV = 0;
    double* V0;
    const KState* st;
    __device__ void elem(uint64_t i, double*) const { V0[i] /= st->aux[6]; }
    __device__ void last(const double*) const {}
};

__global__ void k_gm_cycle_begin(KState* st, GmSmall sm)
{
    if (st->done) return;
    const int m = sm.m;
    for (int i = 0; i <= m; ++i) sm.g[i] = 0.0;
    sm.g[0] = st->aux[6];
    for (int i = 0; i < (m + 1) * m; ++i) sm.H[i] = 0.0;
    st->aux[2] = 0.0;  // j
    st->aux[3] = 0.0;  // j_used
    st->aux[5] = 0.0;  // cycle_end
}

// MGS step i for column j (array.cpp:4307-4316):
//   if i > 0: w -= H[i-1][j] V[i-1];   acc = w . V[i]  -> H[i][j]
// For i == j+1 the dot is w.w and the column's tail runs (norm, Givens, check).
struct BodyGmMgs
{
    static constexpr int NV = 1;
    double* w;
    const double* Vprev;  // V[i-1] or null
    const double* Vi;     // V[i] or null for the norm step
    KState* st;
    GmSmall sm;
    int i;
    __device__ void elem(uint64_t t, double* acc) const
    {
        double wt = w[t];
        if (Vprev)
        {
            wt -= sm.H[(size_t)(i - 1) * sm.m + gm_j(st)] * Vprev[t];
            w[t] = wt;
        }
        acc[0] += Vi ? wt * Vi[t] : wt * wt;
    }
    __device__ void last(const double* tot) const;
};

__device__ void gm_column_tail(KState* st, GmSmall sm, double wnorm2)
{
    const int m = sm.m, j = gm_j(st);
    double* H = sm.H;
#define HH(a, b) H[(size_t)(a) * m + (b)]
    HH(j + 1, j) = sqrt(wnorm2);
    for (int i = 0; i < j; ++i)
    {
        const double t1 = sm.cs[i] * HH(i, j) + sm.sn[i] * HH(i + 1, j);
        const double t2 = -sm.sn[i] * HH(i, j) + sm.cs[i] * HH(i + 1, j);
        HH(i, j) = t1;
        HH(i + 1, j) = t2;
    }
    // hypot as in std::hypot
    const double den = hypot(HH(j, j), HH(j + 1, j));
    st->aux[7] = HH(j + 1, j);  // unrotated subdiagonal, for V[j+1] scaling
    if (den < kBreak)
    {
        finish(st, B2S_BREAKDOWN);
        return;
    }
    sm.cs[j] = HH(j, j) / den;
    sm.sn[j] = HH(j + 1, j) / den;
    HH(j, j) = sm.cs[j] * HH(j, j) + sm.sn[j] * HH(j + 1, j);
    HH(j + 1, j) = 0.0;
    const double g1 = sm.cs[j] * sm.g[j] + sm.sn[j] * sm.g[j + 1];
    const double g2 = -sm.sn[j] * sm.g[j] + sm.cs[j] * sm.g[j + 1];
    sm.g[j] = g1;
    sm.g[j + 1] = g2;
    st->aux[3] = (double)(j + 1);
    st->it_end = (int)st->aux[4];
    st->aux[4] += 1.0;
    st->iters = (int)st->aux[4];
    st->relres = fabs(g2) / st->normb;
    if (fabs(g2) / st->normb < st->tol)
    {
        st->aux[5] = 1.0;
        st->aux[0] = 1.0;  // converged: the outer loop ends after this cycle's update
    }
    else if (j + 1 >= m || (int)st->aux[4] >= st->maxit)
        st->aux[5] = 1.0;
    if (!(g2 == g2)) finish(st, B2S_DIVERGED);
#undef HH
}

__device__ void BodyGmMgs::last(const double* tot) const
{
    if (Vi)
        sm.H[(size_t)i * sm.m + gm_j(st)] = tot[0];
    else
        gm_column_tail(st, sm, tot[0]);
}

// V[j+1] = w * (1 / H[j+1][j]) when H[j+1][j] > 1e-30 (array.cpp:4319-4328), then j++
struct BodyGmNext
{
    static constexpr int NV = 0;
    double* Vnext;
    const double* w;
    const KState* st;
    __device__ void elem(uint64_t t, double*) const
    {
        const double h = st->aux[7];
        if (h > kBreak) Vnext[t] = w[t] * (1.0 / h);
    }
    __device__ void last(const double*) const {}
};

__global__ void k_gm_advance(KState* st)
{
    if (st->done) return;
    st->aux[2] += 1.0;
}

// back substitution R y = g (array.cpp:4369-4379)
__global__ void k_gm_backsub(KState* st, GmSmall sm)
{
    if (st->done && st->status != B2S_OK) return;
    const int m = sm.m, ju = (int)st->aux[3];
    for (int i = ju - 1; i >= 0; --i)
    {
        double sum = sm.g[i];
        for (int k = i + 1; k < ju; ++k) sum -= sm.H[(size_t)i * m + k] * sm.y[k];
        if (fabs(sm.H[(size_t)i * m + i]) < kBreak)
        {
            finish(st, B2S_BREAKDOWN);
            return;
        }
        sm.y[i] = sum / sm.H[(size_t)i * m + i];
    }
}

// z = V y over the used columns (array.cpp:4385-4392): acc summed in i order
struct BodyGmCombine
{
    static constexpr int NV = 0;
    double* z;
    const double* V;
    uint64_t n;
    const KState* st;
    GmSmall sm;
    __device__ void elem(uint64_t t, double*) const
    {
        const int ju = (int)st->aux[3];
        double acc = 0.0;
        for (int i = 0; i < ju; ++i) acc += sm.y[i] * V[(size_t)i * n + t];
        z[t] = acc;
    }
    __device__ void last(const double*) const {}
};

struct BodyAxpyOne  // x += dz
{
    static constexpr int NV = 0;
    double* x;
    const double* dz;
    __device__ void elem(uint64_t t, double*) const { x[t] += dz[t]; }
    __device__ void last(const double*) const {}
};

// CGS2 pass: h_i = w . V_i for a group of up to 8 basis vectors (one pass over w)
struct BodyGmDots
{
    static constexpr int NV = 8;
    const double* w;
    const double* V;
    uint64_t pn;
    int i0, cnt;
    double* hbuf;  // this pass's h (64 entries)
    KState* st;
    GmSmall sm;
    int pass;
    __device__ void elem(uint64_t t, double* acc) const
    {
        const double wt = w[t];
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (k < cnt) acc[k] += wt * V[(size_t)(i0 + k) * pn + t];
    }
    __device__ void last(const double* tot) const
    {
        const int j = gm_j(st);
        for (int k = 0; k < cnt; ++k)
        {
            hbuf[i0 + k] = tot[k];
            double& h = sm.H[(size_t)(i0 + k) * sm.m + j];
            h = pass == 0 ? tot[k] : h + tot[k];
        }
    }
};

// w -= sum_i h_i V_i over i <= j (one pass)
struct BodyGmUpdate
{
    static constexpr int NV = 0;
    double* w;
    const double* V;
    uint64_t pn;
    const double* hbuf;
    const KState* st;
    __device__ void elem(uint64_t t, double*) const
    {
        const int j = (int)st->aux[2];
        double wt = w[t];
        for (int i = 0; i <= j; ++i) wt -= hbuf[i] * V[(size_t)i * pn + t];
        w[t] = wt;
    }
    __device__ void last(const double*) const {}
};

__global__ void k_gm_flag_to_int(const KState* st, int* flag)
{
    // flag = 1 when the current cycle's inner loop must not run
    *flag = (st->done || st->aux[5] != 0.0) ? 1 : 0;
}

// ------------------------------------------------------------- host driver

struct Work
{
    b2s_ctx* ctx;
    double* base;
    size_t used = 0;
    Work(b2s_ctx* c, size_t doubles) : ctx(c)
    {
        c->ws.reserve(doubles);
        base = c->ws.p;
    }
    double* take(size_t k)
    {
        double* p = base + used;
        used += (k + 31) & ~size_t(31);  // 256-byte alignment
        return p;
    }
};

inline size_t padded(size_t k) { return (k + 31) & ~size_t(31); }

struct Solve
{
    b2s_ctx* ctx;
    Operator A;
    PcImpl* pc;
    b2s_solve_opts o;
    KState* st;
    int* done;  // &st->done
    int poll_every;
    bool graphs;
    // stall guard (learned IC(0)): the recursive residual must halve within
    // stall_window iterations, checked at every host poll; 0 = off
    int stall_window = 0;
    bool stalled = false;
    int stalled_at = 0;

    Solve(b2s_ctx* c, const Operator& op, PcImpl* p, const b2s_solve_opts& opts) : ctx(c), A(op), pc(p), o(opts)
    {
        st = ctx->kstate.p;
        done = &st->done;
        poll_every = o.check_every > 0 ? o.check_every : 8;
        graphs = o.use_graphs && !(pc && pc->is_host());
        reserve_reduction(ctx, std::max<unsigned>(A.red_blocks(ctx), stream_grid(ctx, A.n)));
    }

    void init_state()
    {
        KState h;
        std::memset(&h, 0, sizeof(h));
        h.tol = o.tol;
        h.maxit = o.maxit;
        h2d(ctx, st, &h, sizeof(h));
    }

    KState read_state()
    {
        d2h(ctx, ctx->h_kstate, st, sizeof(KState));
        sync(ctx);
        return *ctx->h_kstate;
    }

    void pc_apply(const double* r, double* z)
    {
        if (pc)
            pc->apply(ctx, r, z, done);
        else
            copy(ctx, z, r, A.n, done);
    }

    // runs body() `poll_every` times per host poll until *done; with graphs
    // the batch is captured once and replayed.
    template <typename F>
    void loop(F&& body)
    {
        cudaGraphExec_t exec = nullptr;
        cudaGraph_t graph = nullptr;
        uint64_t per_replay = 0;  // kernels in the captured batch
        if (graphs)
        {
            const uint64_t l0 = ctx->launches;
            B2S_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            for (int k = 0; k < poll_every; ++k) body();
            B2S_CUDA(cudaStreamEndCapture(ctx->stream, &graph));
            B2S_CUDA(cudaGraphInstantiate(&exec, graph, 0));
            // captured launches did not run; every replay runs them once
            per_replay = ctx->launches - l0;
            ctx->launches = l0;
        }
        double best = HUGE_VAL;
        int best_at = 0;
        for (;;)
        {
            if (exec)
            {
                B2S_CUDA(cudaGraphLaunch(exec, ctx->stream));
                ctx->launches += per_replay;
            }
            else
                for (int k = 0; k < poll_every; ++k) body();
            KState h = read_state();
            if (h.done) break;
            if (stall_window > 0)
            {
                if (h.relres < 0.5 * best)
                {
                    best = h.relres;
                    best_at = h.iters;
                }
                else if (h.iters - best_at >= stall_window)
                {
                    // stop here: the remaining kernels see done and skip
                    stalled = true;
                    stalled_at = h.iters;
                    const int one = 1;
                    h2d(ctx, done, &one, sizeof(int));
                    break;
                }
            }
        }
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }

    void true_residual(const double* b, const double* x, double* tmp)
    {
        op_apply_epi(ctx, A, x, tmp, nullptr, EpiTrueRes{b, st});
    }

    void finish_stats(b2s_stats* s, const KState& h, float ms)
    {
        if (!s) return;
        s->it = h.it_end;
        s->iterations = h.iters;
        s->status = h.status;
        s->relres = h.relres;
        s->relres_true = h.aux[0];
        s->solve_ms = ms;
    }
};

}  // namespace

// -------------------------------------------------------------------- PCG

static void run_pcg(Solve& S, const double* b, double* x, b2s_stats* stats)
{
    b2s_ctx* ctx = S.ctx;
    const uint64_t n = S.A.n;
    Work W(ctx, 7 * padded(n));
    double *r = W.take(n), *z = W.take(n), *p = W.take(n), *Ap = W.take(n);
    double *r1 = W.take(n), *p1 = W.take(n);  // second residual / direction (fused iteration)
    KState* st = S.st;
    const int* done = S.done;
    S.init_state();
    B2S_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    fill(ctx, x, 0.0, n);
    copy(ctx, r, b, n);
    launch_vec(ctx, n, done, BodyNormB{b, st});
    KState h = S.read_state();
    if (!h.done && 1.0 < S.o.tol)  // normr / normb == 1 for x0 = 0
    {
        h.done = 1;
        h2d(ctx, &st->done, &h.done, sizeof(int));
    }
    if (!h.done)
    {
        S.pc_apply(r, z);
        launch_vec(ctx, n, done, BodyRZInit{r, z, p, st});
        const PcImpl* pc = S.pc;
        const double* dfuse = pc ? pc->fused_diag() : nullptr;
        const int fuse = (!pc || pc->is_identity()) ? 1 : (dfuse ? 2 : 0);
        if (fuse == 0 && S.A.csr && pc->can_fuse_pcg())
        {
            // Three launches per iteration: the SpMV forms p = z + beta p_old
            // as it gathers and reduces p.Ap; the preconditioner's first
            // launch forms r = r_old - alpha Ap as it stages, updates x and
            // tests convergence; its second reduces r.z and steps beta.  The
            // residual and direction alternate between two buffers, so a
            // captured batch has an even number of iterations.
            // all iterations in one persistent launch when the preconditioner can
            if (S.o.persistent != 2 &&
                S.pc->pcg_persistent(ctx, *S.A.csr, x, r, r1, p, p1, z, Ap, st, S.stall_window, S.o.persistent))
            {
                const KState hs = S.read_state();
                if (hs.stalled)
                {
                    S.stalled = true;
                    S.stalled_at = hs.iters;
                }
                goto done_iterating;
            }
            if (S.poll_every & 1) S.poll_every += 1;
            int parity = 0;
            auto body = [&] {
                double* pold = parity ? p1 : p;
                double* pnew = parity ? p : p1;
                const double* rold = parity ? r1 : r;
                double* rnew = parity ? r : r1;
                launch_spmv_op(ctx, *S.A.csr, XPNew{z, pold, st, 0.0}, done, EpiPApUpd{Ap, pnew, z, pold, st});
                S.pc->pcg_update_apply(ctx, x, pnew, Ap, rold, rnew, z, st, done);
                parity ^= 1;
            };
            S.loop(body);
        }
        else
        {
        auto body = [&] {
            op_apply_epi(ctx, S.A, p, Ap, done, EpiPAp{Ap, p, st});
            if (fuse == 1)
                launch_vec(ctx, n, done, BodyPcgUpdate<1>{x, r, z, p, Ap, nullptr, st});
            else if (fuse == 2)
                launch_vec(ctx, n, done, BodyPcgUpdate<2>{x, r, z, p, Ap, dfuse, st});
            else
            {
                launch_vec(ctx, n, done, BodyPcgUpdate<0>{x, r, z, p, Ap, nullptr, st});
                // a preconditioner may fuse r.z and the scalar step into its apply
                if (!(S.pc && S.pc->apply_rz(ctx, r, z, st, done)))
                {
                    S.pc_apply(r, z);
                    launch_vec(ctx, n, done, BodyRZ{r, z, st});
                }
            }
            launch_vec(ctx, n, done, BodyPUpdate{p, z, st});
        };
        S.loop(body);
        }
    }
done_iterating:
    B2S_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    S.true_residual(b, x, Ap);
    h = S.read_state();
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    S.finish_stats(stats, h, ms);
}

// ---------------------------------------------------------------- BiCGSTAB

static void run_bicgstab(Solve& S, const double* b, double* x, b2s_stats* stats)
{
    b2s_ctx* ctx = S.ctx;
    const uint64_t n = S.A.n;
    Work W(ctx, 10 * padded(n));
    double *r = W.take(n), *rt = W.take(n), *p = W.take(n), *v = W.take(n), *y = W.take(n), *z = W.take(n),
           *s = W.take(n), *t = W.take(n), *tmp = W.take(n);
    KState* st = S.st;
    const int* done = S.done;
    S.init_state();
    B2S_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    fill(ctx, x, 0.0, n);
    launch_vec(ctx, n, done, BodyNormB{b, st});
    KState h = S.read_state();
    if (!h.done && 1.0 < S.o.tol)
    {
        h.done = 1;
        h2d(ctx, &st->done, &h.done, sizeof(int));
    }
    if (!h.done)
    {
        launch_vec(ctx, n, done, BodyBicgInit{b, r, rt, p, v, st});
        // the true-residual check runs only when requested: a flag array
        DBuf<int> flag(1);
        auto body = [&] {
            launch_vec(ctx, n, done, BodyBicgP{p, r, v, st});
            S.pc_apply(p, y);
            op_apply_epi(ctx, S.A, y, tmp, done, EpiBicgV{v, rt, st});
            launch_vec(ctx, n, done, BodyBicgS{s, r, v, st});
            S.pc_apply(s, z);
            op_apply_epi(ctx, S.A, z, tmp, done, EpiBicgT{t, s, st});
            launch_vec(ctx, n, done, BodyBicgXR{x, r, y, z, s, t, rt, st});
            // true residual only when aux[1] is set: a done-like guard flag
            B2S_LAUNCH(ctx, k_bicg_guard, 1, 1, 0, st, flag.p);
            op_apply_epi(ctx, S.A, x, tmp, flag.p, EpiBicgTrue{b, rt, r, st});
        };
        S.loop(body);
    }
    B2S_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    S.true_residual(b, x, tmp);
    h = S.read_state();
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    S.finish_stats(stats, h, ms);
}


// ------------------------------------------------------------------ GMRES

// restarted GMRES(m), right preconditioned (flexible == false), or FGMRES
// (flexible == true: Z_j = M^-1 V_j kept, x += Z y, no final apply).
static void run_gmres(Solve& S, const double* b, double* x, b2s_stats* stats, bool flexible)
{
    b2s_ctx* ctx = S.ctx;
    const uint64_t n = S.A.n;
    const int m = S.o.restart > 0 ? S.o.restart : 30;
    const size_t pn = padded(n);
    Work W(ctx, pn * ((size_t)m + 1 + (flexible ? (size_t)m : 0) + 4));
    double* V = W.take(pn * ((size_t)m + 1));
    double* Z = flexible ? W.take(pn * (size_t)m) : nullptr;
    double *w = W.take(n), *wt = W.take(n), *z = W.take(n), *dz = W.take(n);
    ctx->small.reserve((size_t)(m + 1) * m + 4 * ((size_t)m + 1));
    GmSmall sm;
    sm.m = m;
    sm.H = ctx->small.p;
    sm.cs = sm.H + (size_t)(m + 1) * m;
    sm.sn = sm.cs + m;
    sm.g = sm.sn + m;
    sm.y = sm.g + (m + 1);
    KState* st = S.st;
    const int* done = S.done;
    DBuf<int> gflag(1);
    DBuf<double> hbuf((size_t)m + 8);
    auto Vj = [&](int j) { return V + pn * (size_t)j; };
    auto Zj = [&](int j) { return Z + pn * (size_t)j; };

    S.init_state();
    B2S_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    fill(ctx, x, 0.0, n);
    launch_vec(ctx, n, done, BodyNormB{b, st});
    KState h = S.read_state();
    int cycle = 0;
    while (!h.done && h.aux[0] == 0.0 && (int)h.aux[4] < S.o.maxit)
    {
        if (cycle == 0)
            launch_vec(ctx, n, done, BodyGmV0First{Vj(0), b, st});
        else
        {
            op_apply_epi(ctx, S.A, x, w, done, EpiGmRestart{b, Vj(0), st, sm});
            launch_vec(ctx, n, done, BodyGmScale{Vj(0), st});
        }
        B2S_LAUNCH(ctx, k_gm_cycle_begin, 1, 1, 0, st, sm);
        const int poll = S.poll_every;
        for (int j = 0; j < m; ++j)
        {
            B2S_LAUNCH(ctx, k_gm_flag_to_int, 1, 1, 0, st, gflag.p);
            const int* g = gflag.p;
            double* zin = flexible ? Zj(j) : wt;
            if (S.pc)
                S.pc->apply(ctx, Vj(j), zin, g);
            else
                copy(ctx, zin, Vj(j), n, g);
            S.A.apply(ctx, zin, w, g);
            if (S.o.orth == B2S_ORTH_CGS2)
            {
                // classical Gram-Schmidt twice: batched dots, one update pass, repeated
                for (int pass = 0; pass < 2; ++pass)
                {
                    for (int i0 = 0; i0 <= j; i0 += 8)
                        launch_vec(ctx, n, g, BodyGmDots{w, V, pn, i0, std::min(8, j + 1 - i0), hbuf.p, st, sm, pass});
                    launch_vec(ctx, n, g, BodyGmUpdate{w, V, pn, hbuf.p, st});
                }
                launch_vec(ctx, n, g, BodyGmMgs{w, nullptr, nullptr, st, sm, j + 1});
            }
            else
            {
                for (int i = 0; i <= j; ++i)
                    launch_vec(ctx, n, g, BodyGmMgs{w, i > 0 ? Vj(i - 1) : nullptr, Vj(i), st, sm, i});
                launch_vec(ctx, n, g, BodyGmMgs{w, Vj(j), nullptr, st, sm, j + 1});
            }
            launch_vec(ctx, n, g, BodyGmNext{Vj(j + 1), w, st});
            B2S_LAUNCH(ctx, k_gm_advance, 1, 1, 0, st);
            if ((j + 1) % poll == 0 || j + 1 == m)
            {
                h = S.read_state();
                if (h.done || h.aux[5] != 0.0) break;
            }
        }
        // x += M^-1 (V y)   or   x += Z y
        B2S_LAUNCH(ctx, k_gm_backsub, 1, 1, 0, st, sm);
        if (flexible)
            launch_vec(ctx, n, done, BodyGmCombine{dz, Z, pn, st, sm});
        else
        {
            launch_vec(ctx, n, done, BodyGmCombine{z, V, pn, st, sm});
            if (S.pc)
                S.pc->apply(ctx, z, dz, done);
            else
                copy(ctx, dz, z, n, done);
        }
        launch_vec(ctx, n, done, BodyAxpyOne{x, dz});
        h = S.read_state();
        ++cycle;
    }
    B2S_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    S.true_residual(b, x, w);
    h = S.read_state();
    if (stats) stats->restarts = cycle;
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    S.finish_stats(stats, h, ms);
}

// ------------------------------------------------------ iterative refinement

struct BodyResidual  // r = b - Ax (Ax given), rr
{
    static constexpr int NV = 1;
    double* r;
    const double *b, *Ax;
    KState* st;
    __device__ void elem(uint64_t i, double* acc) const
    {
        const double ri = b[i] - Ax[i];
        r[i] = ri;
        acc[0] += ri * ri;
    }
    __device__ void last(const double* t) const { st->aux[0] = sqrt(t[0]); }
};

// ------------------------------------------------- stationary iteration
// SMatrix::amg (array.cpp:4534-4563): from x = 0, at index it: r = b - A x;
// stop with it_end = it when ||r|| / ||b|| < tol, else x += M^-1 r (one
// V-cycle from zero).  Running out of max_iter leaves it_end = max_iter - 1
// with every correction applied.

// r = b - A x per row, rr; the stopping test at index st->it
struct EpiStatRes
{
    static constexpr int NV = 1;
    double* r;
    const double* b;
    KState* st;
    __device__ void row(uint32_t i, double s, double* acc) const
    {
        const double d = b[i] - s;
        r[i] = d;
        acc[0] += d * d;
    }
    __device__ void last(const double* t) const
    {
        const double normr = sqrt(t[0]);
        st->normr = normr;
        st->relres = normr / st->normb;
        st->it_end = st->it;
        st->iters = st->it;
        if (st->relres < st->tol)
            finish(st, B2S_OK);
        else if (!(normr == normr) || isinf(normr))
        {
            st->it_end = st->maxit - 1;  // the reference runs on with NaN to max_iter
            finish(st, B2S_DIVERGED);
        }
    }
};

// x += d; next index; max_iter stop
struct BodyStatStep
{
    static constexpr int NV = 1;
    double* x;
    const double* d;
    KState* st;
    __device__ void elem(uint64_t i, double* acc) const
    {
        (void)acc;
        x[i] += d[i];
    }
    __device__ void last(const double* t) const
    {
        (void)t;
        st->it += 1;
        st->iters = st->it;
        if (st->it >= st->maxit) finish(st, B2S_OK);
    }
};

static void run_stationary(Solve& S, const double* b, double* x, b2s_stats* stats)
{
    b2s_ctx* ctx = S.ctx;
    const uint64_t n = S.A.n;
    Work W(ctx, 3 * padded(n));
    double *r = W.take(n), *d = W.take(n), *tmp = W.take(n);
    KState* st = S.st;
    const int* done = S.done;
    S.init_state();
    B2S_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    fill(ctx, x, 0.0, n);
    launch_vec(ctx, n, done, BodyNormB{b, st});
    KState h = S.read_state();
    if (!h.done && S.o.maxit == 0)  // the reference's loop body never runs
    {
        h.done = 1;
        h2d(ctx, &st->done, &h.done, sizeof(int));
    }
    if (!h.done)
    {
        auto body = [&] {
            op_apply_epi(ctx, S.A, x, tmp, done, EpiStatRes{r, b, st});
            S.pc_apply(r, d);
            launch_vec(ctx, n, done, BodyStatStep{x, d, st});
        };
        S.loop(body);
    }
    B2S_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    S.true_residual(b, x, tmp);
    h = S.read_state();
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    S.finish_stats(stats, h, ms);
}

static void run_method(Solve& S, b2s_method method, const double* b, double* x, b2s_stats* stats)
{
    switch (method)
    {
        case B2S_PCG: run_pcg(S, b, x, stats); break;
        case B2S_BICGSTAB: run_bicgstab(S, b, x, stats); break;
        case B2S_GMRES:
        case B2S_BLOCK_GMRES: run_gmres(S, b, x, stats, false); break;
        case B2S_FGMRES: run_gmres(S, b, x, stats, true); break;
        case B2S_STATIONARY: run_stationary(S, b, x, stats); break;
        default: fail(B2S_INVALID_ARG, "unknown Krylov method");
    }
}

// x = 0; repeat: r = b - A x (FP64), solve A d = r to ir_inner_tol, x += d,
// until ||b - A x|| / ||b|| < tol or ir_steps sweeps.
static void run_refined(b2s_ctx* ctx, const Operator& A, PcImpl* pc, b2s_method method, const b2s_solve_opts& o,
                        const double* b, double* x, b2s_stats* stats)
{
    const uint64_t n = A.n;
    DBuf<double> r(n), d(n), Ax(n), small(4);
    b2s_solve_opts in = o;
    in.ir_steps = 0;
    in.tol = o.ir_inner_tol > 0 ? o.ir_inner_tol : 1e-4;
    const double normb = std::sqrt(dot_host(ctx, n, b, b));
    fill(ctx, x, 0.0, n);
    copy(ctx, r.p, b, n);
    int total_it = 0, total_iters = 0, sweeps = 0, status = B2S_OK;
    double relres = normb > 0 ? 1.0 : 0.0;
    float ms_total = 0;
    cudaEvent_t e0, e1;
    B2S_CUDA(cudaEventCreate(&e0));
    B2S_CUDA(cudaEventCreate(&e1));
    B2S_CUDA(cudaEventRecord(e0, ctx->stream));
    while (normb >= 1e-300 && relres >= o.tol && sweeps < o.ir_steps)
    {
        Solve S(ctx, A, pc, in);
        b2s_stats inner;
        std::memset(&inner, 0, sizeof(inner));
        run_method(S, method, r.p, d.p, &inner);
        ++sweeps;
        total_it += inner.it + 1;
        total_iters += inner.iterations;
        if (inner.status != B2S_OK && inner.status != B2S_DIVERGED)
        {
            status = inner.status;
            break;
        }
        // x += d ; r = b - A x
        launch_vec(ctx, n, nullptr, BodyAxpyOne{x, d.p});
        A.apply(ctx, x, Ax.p, nullptr);
        KState* st = ctx->kstate.p;
        launch_vec(ctx, n, nullptr, BodyResidual{r.p, b, Ax.p, st});
        d2h(ctx, ctx->h_kstate, st, sizeof(KState));
        sync(ctx);
        relres = ctx->h_kstate->aux[0] / normb;
    }
    B2S_CUDA(cudaEventRecord(e1, ctx->stream));
    B2S_CUDA(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&ms_total, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (stats)
    {
        stats->it = total_it > 0 ? total_it - 1 : 0;
        stats->iterations = total_iters;
        stats->restarts = sweeps;
        stats->status = status;
        stats->relres = relres;
        stats->relres_true = relres;
        stats->solve_ms = ms_total;
    }
}

// Learned IC(0) with its fallback: the solve runs under the stall guard; if it
// stalls, breaks down (NOT_SPD / BREAKDOWN / DIVERGED) or ends unconverged,
// plain FP64 IC(0) takes over from the learned solve's iterate (from x = 0 if
// that is not finite): r = b - A x, solve A d = r to tol ||b|| / ||r||, x += d.
constexpr int kStallWindow = 200;

static void run_learned(b2s_ctx* ctx, const Operator& A, PcImpl* pc, b2s_method method, const b2s_solve_opts& o,
                        const double* b, double* x, b2s_stats* stats)
{
    b2s_stats s1;
    std::memset(&s1, 0, sizeof(s1));
    bool stalled = false;
    int stalled_at = 0;
    {
        Solve S(ctx, A, pc, o);
        S.stall_window = o.stall_window > 0 ? o.stall_window : kStallWindow;
        run_method(S, method, b, x, &s1);
        stalled = S.stalled;
        stalled_at = S.stalled_at;
    }
    const bool failed = s1.status == B2S_NOT_SPD || s1.status == B2S_BREAKDOWN || s1.status == B2S_DIVERGED;
    const bool unconverged = s1.status == B2S_OK && !(s1.relres_true < o.tol);
    if (!(stalled || failed || unconverged))
    {
        if (stats) *stats = s1;
        return;
    }
    const uint64_t n = A.n;
    DBuf<double> r(n), d(n), Ax(n);
    const double normb = std::sqrt(dot_host(ctx, n, b, b));
    KState* st = ctx->kstate.p;
    double normr = normb;
    if (std::isfinite(s1.relres_true))
    {
        A.apply(ctx, x, Ax.p, nullptr);
        launch_vec(ctx, n, nullptr, BodyResidual{r.p, b, Ax.p, st});
        d2h(ctx, ctx->h_kstate, st, sizeof(KState));
        sync(ctx);
        normr = ctx->h_kstate->aux[0];
    }
    if (!std::isfinite(normr) || !std::isfinite(s1.relres_true))
    {
        fill(ctx, x, 0.0, n);
        copy(ctx, r.p, b, n);
        normr = normb;
    }
    b2s_pc_opts po;
    b2s_pc_opts_default(&po);
    auto ic0 = make_pc_ic0(ctx, *A.csr, po);
    b2s_solve_opts in = o;
    in.tol = normr > 0 ? o.tol * normb / normr : o.tol;
    b2s_stats s2;
    std::memset(&s2, 0, sizeof(s2));
    if (normr > 0 && normb > 0 && normr / normb >= o.tol)
    {
        Solve S(ctx, A, ic0.get(), in);
        run_method(S, method, r.p, d.p, &s2);
        launch_vec(ctx, n, nullptr, BodyAxpyOne{x, d.p});
    }
    // FP64 true residual of the combined iterate
    A.apply(ctx, x, Ax.p, nullptr);
    launch_vec(ctx, n, nullptr, BodyResidual{r.p, b, Ax.p, st});
    d2h(ctx, ctx->h_kstate, st, sizeof(KState));
    sync(ctx);
    const double rel = normb > 0 ? ctx->h_kstate->aux[0] / normb : 0.0;
    if (stats)
    {
        stats->it = s1.it + s2.it + 1;
        stats->iterations = s1.iterations + s2.iterations;
        stats->spmvs = s1.spmvs + s2.spmvs + 2;
        stats->pc_applies = s1.pc_applies + s2.pc_applies;
        stats->restarts = s1.restarts + s2.restarts;
        stats->status = s2.status;
        stats->relres = rel;
        stats->relres_true = rel;
        stats->solve_ms = s1.solve_ms + s2.solve_ms;
        stats->fallbacks = 1;
        stats->stalled_at = stalled ? stalled_at : s1.iterations;
    }
}

static b2s_status solve_common(b2s_ctx* ctx, const Operator& A, b2s_pc* pc, b2s_method method,
                               const b2s_solve_opts* opts, const double* d_b, double* d_x, b2s_stats* stats)
{
    b2s_solve_opts o;
    b2s_solve_opts_default(&o);
    if (opts) o = *opts;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    need(!pc || pc->n == A.n, B2S_SHAPE, "preconditioner size differs from the matrix");
    need(o.maxit >= 0, B2S_INVALID_ARG, "maxit must be >= 0");
    need(method != B2S_GMRES || o.restart > 0, B2S_INVALID_ARG, "GMRES restart must be > 0");
    PcImpl* impl = pc ? pc->impl.get() : nullptr;
    const bool learned = pc && pc->kind == B2S_PC_LEARNED_IC0 && A.csr && o.stall_window >= 0;
    if (o.ir_steps > 0)
        run_refined(ctx, A, impl, method, o, d_b, d_x, stats);
    else if (learned)
        run_learned(ctx, A, impl, method, o, d_b, d_x, stats);
    else
    {
        Solve S(ctx, A, impl, o);
        run_method(S, method, d_b, d_x, stats);
    }
    if (stats && pc) stats->setup_ms = 0.0;
    // a bounded wait of a triangular solve that gave up fails the solve
    check_device_error(ctx, "a triangular-solve wait gave up during the solve");
    const int st = stats ? stats->status : B2S_OK;
    if (!stats)
    {
        KState h;
        d2h(ctx, &h, ctx->kstate.p, sizeof(KState));
        sync(ctx);
        if (h.status != B2S_OK && h.status != B2S_DIVERGED)
            fail((b2s_status)h.status, std::string("solver stopped: ") + b2s_status_name((b2s_status)h.status));
        return B2S_OK;
    }
    if (st != B2S_OK && st != B2S_DIVERGED)
        fail((b2s_status)st, std::string("solver stopped: ") + b2s_status_name((b2s_status)st));
    return B2S_OK;
}

}  // namespace b2s

using namespace b2s;

extern "C" {

b2s_status b2s_solve_device(b2s_ctx* ctx, const b2s_csr* A, b2s_pc* pc, b2s_method method,
                            const b2s_solve_opts* opts, const double* d_b, double* d_x, b2s_stats* stats)
{
    if (!ctx || !A) return B2S_INVALID_ARG;
    return guarded(ctx, [&] {
        need(A->d.n == A->d.m, B2S_SHAPE, "solver needs a square matrix");
        Operator op;
        op.csr = &A->d;
        op.n = A->d.n;
        solve_common(ctx, op, pc, method, opts, d_b, d_x, stats);
    });
}

b2s_status b2s_solve(b2s_ctx* ctx, const b2s_csr* A, b2s_pc* pc, b2s_method method, const b2s_solve_opts* opts,
                     const double* b, double* x, b2s_stats* stats)
{
    if (!ctx || !A || (A->d.n && (!b || !x))) return B2S_INVALID_ARG;
    return guarded(ctx, [&] {
        need(A->d.n == A->d.m, B2S_SHAPE, "solver needs a square matrix");
        const uint64_t n = A->d.n;
        DBuf<double> db(n), dx(n);
        h2d(ctx, db.p, b, db.bytes());
        Operator op;
        op.csr = &A->d;
        op.n = n;
        try
        {
            solve_common(ctx, op, pc, method, opts, db.p, dx.p, stats);
        }
        catch (const Error&)
        {
            d2h(ctx, x, dx.p, dx.bytes());  // the last iterate goes back with the error status
            sync(ctx);
            throw;
        }
        d2h(ctx, x, dx.p, dx.bytes());
        sync(ctx);
    });
}

b2s_status b2s_solve_baij_device(b2s_ctx* ctx, const b2s_baij* A, b2s_pc* pc, b2s_method method,
                                 const b2s_solve_opts* opts, const double* d_b, double* d_x, b2s_stats* stats)
{
    if (!ctx || !A) return B2S_INVALID_ARG;
    return guarded(ctx, [&] {
        need(A->d.nbr == A->d.nbc, B2S_SHAPE, "solver needs a square block matrix");
        Operator op;
        op.baij = &A->d;
        op.n = (uint64_t)A->d.nbr * A->d.bs;
        solve_common(ctx, op, pc, method, opts, d_b, d_x, stats);
    });
}

b2s_status b2s_solve_baij(b2s_ctx* ctx, const b2s_baij* A, b2s_pc* pc, b2s_method method, const b2s_solve_opts* opts,
                          const double* b, double* x, b2s_stats* stats)
{
    if (!ctx || !A) return B2S_INVALID_ARG;
    return guarded(ctx, [&] {
        need(A->d.nbr == A->d.nbc, B2S_SHAPE, "solver needs a square block matrix");
        const uint64_t n = (uint64_t)A->d.nbr * A->d.bs;
        need(n == 0 || (b && x), B2S_INVALID_ARG, "null vector");
        DBuf<double> db(n), dx(n);
        h2d(ctx, db.p, b, db.bytes());
        Operator op;
        op.baij = &A->d;
        op.n = n;
        try
        {
            solve_common(ctx, op, pc, method, opts, db.p, dx.p, stats);
        }
        catch (const Error&)
        {
            d2h(ctx, x, dx.p, dx.bytes());
            sync(ctx);
            throw;
        }
        d2h(ctx, x, dx.p, dx.bytes());
        sync(ctx);
    });
}

}  // extern "C"
