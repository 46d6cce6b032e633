// Multicolour SSOR preconditioner.
//   make_redblack_data        array.cpp:2947-3067 (colouring, renumbering, A2 = P A P^T, diag2)
//   make_ssor_preconditioner  array.cpp:3068-3164 (apply)
//
// The colouring is setup work on the pattern and runs on the host: the graph
// of A + A^T is 2-coloured by breadth-first search from each uncoloured seed
// in index order; if that finds an odd cycle, every vertex instead takes the
// smallest colour unused by its already-coloured neighbours, in index order.
// Rows are renumbered colour-major (stable inside a colour) -- the same
// colours and numbering as the reference, so the sweeps are identical.
// A2 = P A P^T is formed on the device (rows gathered, columns renumbered and
// re-sorted).  The apply runs one kernel per colour per sweep; rows of one
// colour are independent.  The gather f = P r is fused into the first forward
// colour and the scatter z = P^T z2 into every backward colour.
#include <algorithm>
#include <cmath>

#include "b2s_internal.cuh"

namespace b2s {

namespace {

void colour_graph(uint32_t n, const std::vector<uint32_t>& rp, const std::vector<uint32_t>& ci,
                  std::vector<int>& colour)
{
    const uint32_t nnz = rp[n];
    std::vector<uint32_t> tp(n + 1, 0), tr(nnz);
    for (uint32_t p = 0; p < nnz; ++p) tp[ci[p] + 1]++;
    for (uint32_t i = 0; i < n; ++i) tp[i + 1] += tp[i];
    {
        std::vector<uint32_t> off(tp.begin(), tp.end() - 1);
        for (uint32_t i = 0; i < n; ++i)
            for (uint32_t p = rp[i]; p < rp[i + 1]; ++p) tr[off[ci[p]]++] = i;
    }
    colour.assign(n, -1);
    bool bip = true;
    std::vector<uint32_t> queue;
    queue.reserve(n);
    for (uint32_t s = 0; s < n && bip; ++s)
    {
        if (colour[s] != -1) continue;
        colour[s] = 0;
        queue.clear();
        queue.push_back(s);
        for (size_t h = 0; h < queue.size() && bip; ++h)
        {
            const uint32_t i = queue[h];
            for (int pass = 0; pass < 2 && bip; ++pass)
            {
                const auto& ptr = pass ? tp : rp;
                const auto& idx = pass ? tr : ci;
                for (uint32_t p = ptr[i]; p < ptr[i + 1]; ++p)
                {
                    const uint32_t j = idx[p];
                    if (j == i) continue;
                    if (colour[j] == -1)
                    {
                        colour[j] = 1 - colour[i];
                        queue.push_back(j);
                    }
                    else if (colour[j] == colour[i])
                        bip = false;
                }
            }
        }
    }
    if (bip) return;
    std::fill(colour.begin(), colour.end(), -1);
    std::vector<char> used(n + 1, 0);
    std::vector<int> touched;
    for (uint32_t i = 0; i < n; ++i)
    {
        touched.clear();
        for (int pass = 0; pass < 2; ++pass)
        {
            const auto& ptr = pass ? tp : rp;
            const auto& idx = pass ? tr : ci;
            for (uint32_t p = ptr[i]; p < ptr[i + 1]; ++p)
            {
                const uint32_t j = idx[p];
                if (j == i) continue;
                const int c = colour[j];
                if (c >= 0 && !used[c])
                {
                    used[c] = 1;
                    touched.push_back(c);
                }
            }
        }
        int c = 0;
        while (used[c]) ++c;
        colour[i] = c;
        for (int t : touched) used[t] = 0;
    }
}

// A2 row ni = A row perm[ni] with columns renumbered, then sorted
__global__ void k_perm_fill(uint32_t n, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                            const double* __restrict__ v, const uint32_t* __restrict__ perm,
                            const uint32_t* __restrict__ new_id, const uint32_t* __restrict__ rp2,
                            uint32_t* __restrict__ ci2, double* __restrict__ v2, double* __restrict__ d2, int* bad)
{
    for (uint32_t ni = blockIdx.x * blockDim.x + threadIdx.x; ni < n; ni += gridDim.x * blockDim.x)
    {
        const uint32_t i = perm[ni];
        uint32_t d = rp2[ni];
        const uint32_t a = d;
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p, ++d)
        {
            ci2[d] = new_id[ci[p]];
            v2[d] = v[p];
        }
        // insertion sort by new column
        for (uint32_t p = a + 1; p < d; ++p)
        {
            const uint32_t c = ci2[p];
            const double x = v2[p];
            uint32_t q = p;
            while (q > a && ci2[q - 1] > c)
            {
                ci2[q] = ci2[q - 1];
                v2[q] = v2[q - 1];
                --q;
            }
            ci2[q] = c;
            v2[q] = x;
        }
        bool found = false;
        double dv = 0.0;
        for (uint32_t p = a; p < d; ++p)
            if (ci2[p] == ni)
            {
                dv = v2[p];
                found = true;
                break;
            }
        d2[ni] = dv;
        if (!found || fabs(dv) < 1e-300) atomicMin(bad, (int)ni);
    }
}

// forward sweep of colour [lo, hi): w_ii = (fw f_ii - sum_{j<ii} omega a_ij w_j) / d_ii
__global__ void k_ssor_fwd(uint32_t lo, uint32_t hi, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                           const double* __restrict__ v, const double* __restrict__ d2, const uint32_t* __restrict__ perm,
                           const double* __restrict__ r, double* __restrict__ w, double omega, double fw, const int* done)
{
    if (done && *done) return;
    for (uint32_t ii = lo + blockIdx.x * blockDim.x + threadIdx.x; ii < hi; ii += gridDim.x * blockDim.x)
    {
        double sigma = fw * r[perm[ii]];
        for (uint32_t p = rp[ii]; p < rp[ii + 1]; ++p)
        {
            const uint32_t j = ci[p];
            if (j < ii) sigma -= omega * v[p] * w[j];
        }
        w[ii] = sigma / d2[ii];
    }
}

// backward sweep: z2_ii = w_ii - (omega / d_ii) sum_{j>ii} a_ij z2_j ; z[perm[ii]] = z2_ii
__global__ void k_ssor_bwd(uint32_t lo, uint32_t hi, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                           const double* __restrict__ v, const double* __restrict__ d2, const uint32_t* __restrict__ perm,
                           const double* __restrict__ w, double* __restrict__ z2, double* __restrict__ z, double omega,
                           const int* done)
{
    if (done && *done) return;
    for (uint32_t ii = lo + blockIdx.x * blockDim.x + threadIdx.x; ii < hi; ii += gridDim.x * blockDim.x)
    {
        double sigma = 0.0;
        for (uint32_t p = rp[ii]; p < rp[ii + 1]; ++p)
        {
            const uint32_t j = ci[p];
            if (j > ii) sigma += v[p] * z2[j];
        }
        const double zi = w[ii] - (omega / d2[ii]) * sigma;
        z2[ii] = zi;
        z[perm[ii]] = zi;
    }
}

struct PcSSOR final : PcImpl
{
    uint32_t n = 0, ncolor = 0;
    double omega = 1.2;
    std::vector<uint32_t> h_cptr, h_new_id;
    DBuf<uint32_t> perm, new_id, rp2, ci2;
    DBuf<double> v2, d2, w, z2;

    void apply(b2s_ctx* ctx, const double* r, double* z, const int* done) override
    {
        const double fw = omega * (2.0 - omega);
        for (uint32_t c = 0; c < ncolor; ++c)
        {
            const uint32_t lo = h_cptr[c], hi = h_cptr[c + 1];
            if (lo >= hi) continue;
            B2S_LAUNCH(ctx, k_ssor_fwd, stream_grid(ctx, hi - lo), kThreads, 0, lo, hi, rp2.p, ci2.p, v2.p, d2.p,
                       perm.p, r, w.p, omega, fw, done);
        }
        for (uint32_t cc = ncolor; cc-- > 0;)
        {
            const uint32_t lo = h_cptr[cc], hi = h_cptr[cc + 1];
            if (lo >= hi) continue;
            B2S_LAUNCH(ctx, k_ssor_bwd, stream_grid(ctx, hi - lo), kThreads, 0, lo, hi, rp2.p, ci2.p, v2.p, d2.p,
                       perm.p, w.p, z2.p, z, omega, done);
        }
    }

    void export_data(b2s_ctx* ctx, const std::string& what, uint64_t* sizes, uint32_t* rp, uint32_t* ci,
                     double* v) override
    {
        if (what != "ssor.colour") return PcImpl::export_data(ctx, what, sizes, rp, ci, v);
        sizes[0] = ncolor + 1;
        sizes[1] = n;
        sizes[2] = n;
        if (rp) std::memcpy(rp, h_cptr.data(), (ncolor + 1) * sizeof(uint32_t));
        if (ci) std::memcpy(ci, h_new_id.data(), n * sizeof(uint32_t));
        if (v)
        {
            d2h(ctx, v, d2.p, n * sizeof(double));
            sync(ctx);
        }
    }
};

}  // namespace

// The reference's colouring of the graph of A + A^T (two colours by BFS when
// it is bipartite, greedy colours otherwise), rows renumbered colour by
// colour, and A2 = P A P^T with each row's columns sorted in the new
// numbering (array.cpp:2947-3040 for SSOR, 3946-4110 for red-black SOR).
void build_redblack(b2s_ctx* ctx, const CsrDev& A, RedBlack& rb, const char* what)
{
    const uint32_t n = A.n;
    rb.n = n;
    std::vector<int> colour;
    A.host_pattern(ctx);
    colour_graph(n, A.h_rp, A.h_ci, colour);
    uint32_t nc = 0;
    for (uint32_t i = 0; i < n; ++i) nc = std::max<uint32_t>(nc, (uint32_t)colour[i] + 1);
    rb.ncolor = nc;
    rb.h_cptr.assign(nc + 1, 0);
    for (uint32_t i = 0; i < n; ++i) rb.h_cptr[colour[i] + 1]++;
    for (uint32_t c = 0; c < nc; ++c) rb.h_cptr[c + 1] += rb.h_cptr[c];
    rb.h_new_id.resize(n);
    std::vector<uint32_t> off(rb.h_cptr.begin(), rb.h_cptr.end() - 1), perm(n);
    for (uint32_t i = 0; i < n; ++i) rb.h_new_id[i] = off[colour[i]]++;
    for (uint32_t i = 0; i < n; ++i) perm[rb.h_new_id[i]] = i;
    rb.perm = upload(ctx, perm.data(), n);
    rb.new_id = upload(ctx, rb.h_new_id.data(), n);
    std::vector<uint32_t> rp2(n + 1, 0);
    for (uint32_t ni = 0; ni < n; ++ni) rp2[ni + 1] = rp2[ni] + (A.h_rp[perm[ni] + 1] - A.h_rp[perm[ni]]);
    rb.rp2 = upload(ctx, rp2.data(), n + 1);
    rb.ci2.alloc(A.nnz ? A.nnz : 1);
    rb.v2.alloc(A.nnz ? A.nnz : 1);
    rb.d2.alloc(n ? n : 1);
    DBuf<int> bad(1);
    const int big = 0x7fffffff;
    h2d(ctx, bad.p, &big, sizeof(int));
    if (n)
        B2S_LAUNCH(ctx, k_perm_fill, stream_grid(ctx, n), kThreads, 0, n, A.rp.p, A.ci.p, A.v.p, rb.perm.p,
                   rb.new_id.p, rb.rp2.p, rb.ci2.p, rb.v2.p, rb.d2.p, bad.p);
    int h = big;
    d2h(ctx, &h, bad.p, sizeof(int));
    sync(ctx);
    if (h != big)
        fail(B2S_MISSING_DIAG, std::string(what) + " failed: missing nonzero diagonal (renumbered row " +
                                   std::to_string(h) + ")");
}

std::unique_ptr<PcImpl> make_pc_ssor(b2s_ctx* ctx, const CsrDev& A, const b2s_pc_opts& o)
{
    need(A.n == A.m, B2S_SHAPE, "SSOR needs a square matrix");
    need(o.omega > 0.0 && o.omega < 2.0, B2S_INVALID_ARG, "SSOR: relaxation factor must satisfy 0 < omega < 2");
    auto pc = std::make_unique<PcSSOR>();
    const uint32_t n = A.n;
    pc->n = n;
    pc->omega = o.omega;
    RedBlack rb;
    build_redblack(ctx, A, rb, "SSOR/red-black");
    pc->ncolor = rb.ncolor;
    pc->h_cptr = std::move(rb.h_cptr);
    pc->h_new_id = std::move(rb.h_new_id);
    pc->perm = std::move(rb.perm);
    pc->new_id = std::move(rb.new_id);
    pc->rp2 = std::move(rb.rp2);
    pc->ci2 = std::move(rb.ci2);
    pc->v2 = std::move(rb.v2);
    pc->d2 = std::move(rb.d2);
    pc->w.alloc(n ? n : 1);
    pc->z2.alloc(n ? n : 1);
    return pc;
}

}  // namespace b2s
