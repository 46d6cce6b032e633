// Smoothed-aggregation AMG on BAIJ operators (make_block_amg_preconditioner,
// blockMatrix.hpp:1051-1179; V-cycle blk_amg_vcycle, 946-1046).  The scalar
// "amg" preconditioner runs the same code on the BS = 1 condensed matrix, as
// test_BlockMatrix_schur3d.cpp:143-146 does with the reference.
//
// Setup, per level, all on the device:
//   diag_inv   Gauss-Jordan inverse of each diagonal block (a failed inverse
//              leaves zeros; the reference ignores the failure too)
//   strength   off-diagonal blocks with Frobenius norm >= 0.25 * row maximum
//   aggregates the reference's greedy rule -- rows in natural order, a row not
//              yet aggregated opens an aggregate and pulls in up to 3 of its
//              unaggregated strong neighbours in list order.  The rule is
//              sequential by definition; one thread walks it with the strong
//              lists streamed from HBM, which makes the aggregates identical
//              to the reference's.
//   P          (I - 2/3 D^-1 A) P_tent, one thread per row, blocks accumulated
//              in the reference's order and emitted with ascending aggregate
//   R = P^T    block transpose (rows sorted afterwards)
//   A_c        R (A P): two-phase block SpGEMM -- candidate columns, segmented
//              sort + unique for the pattern, then each output block summed in
//              the reference's (pa, pb) order: bit-equal Galerkin operators
//   coarsest   at most 50 block rows: dense elimination on one CTA, either the
//              reference's own (amg_ref_coarse = 1: rows swapped in the matrix
//              only, the V-cycle solve then repeats blockMatrix.hpp:958-1000
//              exactly) or a correct partial-pivot LU (default).
// Apply: one V(1,1) cycle with 2/3-damped block Jacobi; the pre-smoothing
// step starts from zero so its residual is the right-hand side itself.
#include <cub/cub.cuh>

#include <algorithm>

#include "baij_mv.cuh"
#include "block_ops.cuh"
#include "trisolve.cuh"

namespace b2s {

namespace {

constexpr double kTheta = 0.25, kOmega = 2.0 / 3.0;

// ------------------------------------------------------------ BAIJ helpers

__global__ void k_find_diag(uint32_t nb, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                            uint32_t* __restrict__ dptr)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
    {
        uint32_t d = 0xFFFFFFFFu;
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
            if (ci[p] == i)
            {
                d = p;
                break;
            }
        dptr[i] = d;
    }
}

// finalise a device-built BAIJ: diagonal pointers and the block count
void finish_baij(b2s_ctx* ctx, BaijDev& M)
{
    M.diag_ptr.alloc(M.nbr ? M.nbr : 1);
    if (M.nbr)
        B2S_LAUNCH(ctx, k_find_diag, stream_grid(ctx, M.nbr), kThreads, 0, M.nbr, M.rp.p, M.ci.p, M.diag_ptr.p);
    d2h(ctx, &M.nnzb, M.rp.p + M.nbr, sizeof(uint32_t));
    sync(ctx);
    if (M.bs == 1 && M.nbr && M.nnzb >= (uint64_t)kBaijStagedMinRow * M.nbr)
    {
        std::vector<uint32_t> h_rp(M.nbr + 1);
        d2h(ctx, h_rp.data(), M.rp.p, (M.nbr + 1) * sizeof(uint32_t));
        sync(ctx);
        baij_partition(ctx, M, h_rp.data());
    }
}

template <int BS>
__global__ void k_diag_inv(uint32_t nb, const double* __restrict__ v, const uint32_t* __restrict__ dptr,
                           double* __restrict__ dinv)
{
    constexpr int BV = BS * BS;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
    {
        double M[BV], Mi[BV];
        for (int k = 0; k < BV; ++k) Mi[k] = 0.0;
        if (dptr[i] != 0xFFFFFFFFu)
        {
            for (int k = 0; k < BV; ++k) M[k] = v[(size_t)dptr[i] * BV + k];
            double T[BV];
            if (blk_inv<BS>(M, T))
                for (int k = 0; k < BV; ++k) Mi[k] = T[k];
        }
        for (int k = 0; k < BV; ++k) dinv[(size_t)i * BV + k] = Mi[k];
    }
}

// ------------------------------------------------------------ strength

template <int BS>
__device__ __forceinline__ double fro(const double* b)
{
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < BS * BS; ++k) s += b[k] * b[k];
    return sqrt(s);
}

template <int BS>
__global__ void k_strength(uint32_t nb, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                           const double* __restrict__ v, const uint32_t* __restrict__ sp, uint32_t* __restrict__ cnt,
                           uint32_t* __restrict__ sc)
{
    constexpr int BV = BS * BS;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
    {
        double mx = 0.0;
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
            if (ci[p] != i)
            {
                const double f = fro<BS>(&v[(size_t)p * BV]);
                mx = mx < f ? f : mx;
            }
        const double thr = kTheta * mx;
        uint32_t c = 0, w = sp ? sp[i] : 0;
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
            if (ci[p] != i && fro<BS>(&v[(size_t)p * BV]) >= thr)
            {
                if (sc) sc[w++] = ci[p];
                ++c;
            }
        if (cnt) cnt[i] = c;
    }
    if (cnt && blockIdx.x == 0 && threadIdx.x == 0) cnt[nb] = 0;
}

// ------------------------------------------------------------ aggregation

// The greedy rule of blockMatrix.hpp:1101-1111, walked by one thread.
__global__ void k_aggregate(uint32_t nb, const uint32_t* __restrict__ sp, const uint32_t* __restrict__ sc,
                            int32_t* __restrict__ agg, uint32_t* __restrict__ nagg_out)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int32_t nagg = 0;
    for (uint32_t i = 0; i < nb; ++i)
    {
        if (agg[i] != -1) continue;
        agg[i] = nagg;
        int sz = 1;
        const uint32_t a = __ldg(&sp[i]), b = __ldg(&sp[i + 1]);
        for (uint32_t p = a; p < b && sz < 4; ++p)
        {
            const uint32_t j = __ldg(&sc[p]);
            if (agg[j] == -1)
            {
                agg[j] = nagg;
                ++sz;
            }
        }
        ++nagg;
    }
    *nagg_out = (uint32_t)nagg;
}

// Standard three-phase smoothed-aggregation rule (no reference counterpart):
// 1. a row whose strong neighbours are all free becomes a root and takes them
// all; 2. a free row joins the phase-1 aggregate of its first aggregated
// strong neighbour; 3. the remaining rows group with their free strong
// neighbours.  One thread walks the rows in natural order (the phases are
// order-dependent); snap holds the phase-1 aggregates.
__global__ void k_aggregate_std(uint32_t nb, const uint32_t* __restrict__ sp, const uint32_t* __restrict__ sc,
                                int32_t* __restrict__ agg, int32_t* __restrict__ snap, uint32_t* __restrict__ nagg_out)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int32_t nagg = 0;
    for (uint32_t i = 0; i < nb; ++i)
    {
        if (agg[i] != -1) continue;
        const uint32_t a = __ldg(&sp[i]), b = __ldg(&sp[i + 1]);
        bool free_all = true;
        for (uint32_t p = a; p < b; ++p)
            if (agg[__ldg(&sc[p])] != -1)
            {
                free_all = false;
                break;
            }
        if (!free_all) continue;
        agg[i] = nagg;
        for (uint32_t p = a; p < b; ++p) agg[__ldg(&sc[p])] = nagg;
        ++nagg;
    }
    for (uint32_t i = 0; i < nb; ++i) snap[i] = agg[i];
    for (uint32_t i = 0; i < nb; ++i)
    {
        if (snap[i] != -1) continue;
        for (uint32_t p = __ldg(&sp[i]); p < __ldg(&sp[i + 1]); ++p)
        {
            const int32_t g = snap[__ldg(&sc[p])];
            if (g != -1)
            {
                agg[i] = g;
                break;
            }
        }
    }
    for (uint32_t i = 0; i < nb; ++i)
    {
        if (agg[i] != -1) continue;
        agg[i] = nagg;
        for (uint32_t p = __ldg(&sp[i]); p < __ldg(&sp[i + 1]); ++p)
            if (agg[__ldg(&sc[p])] == -1) agg[__ldg(&sc[p])] = nagg;
        ++nagg;
    }
    *nagg_out = (uint32_t)nagg;
}

// Parallel aggregation (the library default; no reference counterpart).
// Deterministic, with every pass reading only state from the previous pass:
//   roots: a distance-2 independent set of the strength graph, chosen in
//     rounds.  Each row has a fixed key (an integer hash of the row in the
//     high word, the row + 1 in the low word).  In a round, m1(i) is the
//     largest key among the undecided rows of {i} U S(i), and an undecided
//     row whose key equals the largest m1 over {i} U S(i) becomes a root.
//     Undecided rows within two strength edges of a root then leave the set.
//     The undecided row with the largest key always becomes a root, so the
//     rounds end.
//   aggregates: roots are numbered in row order; a row with a root among its
//     strong neighbours joins the one with the largest key; a row still
//     without an aggregate then joins the aggregate of its assigned strong
//     neighbour with the largest key (as assigned after the first phase);
//     the rows left over become singletons, numbered after the roots in row
//     order.
// S(i) are the strong columns of row i (the same strength test as above).

__device__ __host__ __forceinline__ uint64_t agg_key(uint32_t i)
{
    // integer hash (xorshift-multiply mix) of the row, then the row itself
    uint32_t x = i;
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return ((uint64_t)x << 32) | (uint64_t)(i + 1u);
}

enum : uint8_t { kAggUndecided = 0, kAggRoot = 1, kAggOut = 2 };

__global__ void k_mis_m1(uint32_t n, const uint32_t* __restrict__ sp, const uint32_t* __restrict__ sc,
                         const uint8_t* __restrict__ st, uint64_t* __restrict__ m1)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        uint64_t m = st[i] == kAggUndecided ? agg_key(i) : 0ull;
        for (uint32_t p = sp[i]; p < sp[i + 1]; ++p)
        {
            const uint32_t j = sc[p];
            if (st[j] == kAggUndecided)
            {
                const uint64_t k = agg_key(j);
                m = k > m ? k : m;
            }
        }
        m1[i] = m;
    }
}

__global__ void k_mis_select(uint32_t n, const uint32_t* __restrict__ sp, const uint32_t* __restrict__ sc,
                             const uint64_t* __restrict__ m1, uint8_t* __restrict__ st)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        if (st[i] != kAggUndecided) continue;
        uint64_t m = m1[i];
        for (uint32_t p = sp[i]; p < sp[i + 1]; ++p)
        {
            const uint64_t k = m1[sc[p]];
            m = k > m ? k : m;
        }
        if (m == agg_key(i)) st[i] = kAggRoot;
    }
}

// c1(i): i is a root or has a strong neighbour that is one
__global__ void k_mis_cover1(uint32_t n, const uint32_t* __restrict__ sp, const uint32_t* __restrict__ sc,
                             const uint8_t* __restrict__ st, uint8_t* __restrict__ c1)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        uint8_t c = st[i] == kAggRoot;
        for (uint32_t p = sp[i]; p < sp[i + 1] && !c; ++p) c = st[sc[p]] == kAggRoot;
        c1[i] = c;
    }
}

// undecided rows with c1 on {i} U S(i) leave; counts the rows still undecided
__global__ void k_mis_cover2(uint32_t n, const uint32_t* __restrict__ sp, const uint32_t* __restrict__ sc,
                             const uint8_t* __restrict__ c1, uint8_t* __restrict__ st, uint32_t* __restrict__ left)
{
    uint32_t cnt = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        if (st[i] != kAggUndecided) continue;
        bool c = c1[i] != 0;
        for (uint32_t p = sp[i]; p < sp[i + 1] && !c; ++p) c = c1[sc[p]] != 0;
        if (c)
            st[i] = kAggOut;
        else
            ++cnt;
    }
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    if ((threadIdx.x & 31u) == 0 && cnt) atomicAdd(left, cnt);
}

__global__ void k_agg_flag(uint32_t n, const uint8_t* __restrict__ st, const int32_t* __restrict__ agg, int mode,
                           uint32_t* __restrict__ flag)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        flag[i] = mode == 0 ? (st[i] == kAggRoot) : (agg[i] < 0);
}

// roots take their number; other rows join the root neighbour with the largest key
__global__ void k_agg_roots(uint32_t n, const uint32_t* __restrict__ sp, const uint32_t* __restrict__ sc,
                            const uint8_t* __restrict__ st, const uint32_t* __restrict__ rank, int32_t* __restrict__ agg)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        if (st[i] == kAggRoot)
        {
            agg[i] = (int32_t)rank[i];
            continue;
        }
        uint64_t best = 0;
        int32_t g = -1;
        for (uint32_t p = sp[i]; p < sp[i + 1]; ++p)
        {
            const uint32_t j = sc[p];
            if (st[j] != kAggRoot) continue;
            const uint64_t k = agg_key(j);
            if (k > best)
            {
                best = k;
                g = (int32_t)rank[j];
            }
        }
        agg[i] = g;
    }
}

// rows still without an aggregate join the assigned strong neighbour with the largest key (snapshot)
__global__ void k_agg_extend(uint32_t n, const uint32_t* __restrict__ sp, const uint32_t* __restrict__ sc,
                             const int32_t* __restrict__ snap, int32_t* __restrict__ agg)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        if (snap[i] >= 0) continue;
        uint64_t best = 0;
        int32_t g = -1;
        for (uint32_t p = sp[i]; p < sp[i + 1]; ++p)
        {
            const uint32_t j = sc[p];
            if (snap[j] < 0) continue;
            const uint64_t k = agg_key(j);
            if (k > best)
            {
                best = k;
                g = snap[j];
            }
        }
        agg[i] = g;
    }
}

__global__ void k_agg_single(uint32_t n, uint32_t base, const uint32_t* __restrict__ rank, int32_t* __restrict__ agg)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (agg[i] < 0) agg[i] = (int32_t)(base + rank[i]);
}

// returns the aggregate count
static uint32_t aggregate_parallel(b2s_ctx* ctx, uint32_t n, const uint32_t* sp, const uint32_t* sc, int32_t* agg)
{
    if (!n) return 0;
    const unsigned g = stream_grid(ctx, n);
    DBuf<uint8_t> st(n), c1(n);
    DBuf<uint64_t> m1(n);
    DBuf<uint32_t> left(1), flag(n + 1), rank(n + 1);
    B2S_CUDA(cudaMemsetAsync(st.p, 0, n, ctx->stream));
    for (uint32_t round = 0;; ++round)
    {
        if (round > n) fail(B2S_CUDA_ERROR, "aggregation rounds did not terminate");
        B2S_CUDA(cudaMemsetAsync(left.p, 0, sizeof(uint32_t), ctx->stream));
        B2S_LAUNCH(ctx, k_mis_m1, g, kThreads, 0, n, sp, sc, st.p, m1.p);
        B2S_LAUNCH(ctx, k_mis_select, g, kThreads, 0, n, sp, sc, m1.p, st.p);
        B2S_LAUNCH(ctx, k_mis_cover1, g, kThreads, 0, n, sp, sc, st.p, c1.p);
        B2S_LAUNCH(ctx, k_mis_cover2, g, kThreads, 0, n, sp, sc, c1.p, st.p, left.p);
        uint32_t h = 0;
        d2h(ctx, &h, left.p, sizeof(uint32_t));
        sync(ctx);
        if (!h) break;
    }
    B2S_LAUNCH(ctx, k_agg_flag, g, kThreads, 0, n, st.p, (const int32_t*)nullptr, 0, flag.p);
    const uint32_t nroots = exclusive_scan(ctx, flag.p, rank.p, n);
    B2S_LAUNCH(ctx, k_agg_roots, g, kThreads, 0, n, sp, sc, st.p, rank.p, agg);
    DBuf<int32_t> snap(n);
    d2d(ctx, snap.p, agg, (size_t)n * sizeof(int32_t));
    B2S_LAUNCH(ctx, k_agg_extend, g, kThreads, 0, n, sp, sc, snap.p, agg);
    B2S_LAUNCH(ctx, k_agg_flag, g, kThreads, 0, n, st.p, agg, 1, flag.p);
    const uint32_t nsingle = exclusive_scan(ctx, flag.p, rank.p, n);
    if (nsingle) B2S_LAUNCH(ctx, k_agg_single, g, kThreads, 0, n, nroots, rank.p, agg);
    return nroots + nsingle;
}

// ------------------------------------------------------------ prolongation

// distinct aggregates among {agg[i]} U {agg[k] : k in row i}, ascending
__device__ __forceinline__ uint32_t p_row_cols(uint32_t i, const uint32_t* rp, const uint32_t* ci, const int32_t* agg,
                                               uint32_t* out)
{
    // count distinct; write ascending when out != null
    uint32_t cnt = 0;
    int32_t last = -1;
    for (;;)
    {
        // smallest candidate greater than `last`
        int32_t best = 0x7fffffff;
        const int32_t gi = agg[i];
        if (gi > last && gi < best) best = gi;
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
        {
            const int32_t g = agg[ci[p]];
            if (g > last && g < best) best = g;
        }
        if (best == 0x7fffffff) break;
        if (out) out[cnt] = (uint32_t)best;
        ++cnt;
        last = best;
    }
    return cnt;
}

__global__ void k_p_count(uint32_t nb, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                          const int32_t* __restrict__ agg, uint32_t* __restrict__ cnt)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
        cnt[i] = p_row_cols(i, rp, ci, agg, nullptr);
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt[nb] = 0;
}

template <int BS>
__global__ void k_p_fill(uint32_t nb, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                         const double* __restrict__ v, const double* __restrict__ dinv, const int32_t* __restrict__ agg,
                         const uint32_t* __restrict__ prp, uint32_t* __restrict__ pci, double* __restrict__ pv)
{
    constexpr int BV = BS * BS;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
    {
        const uint32_t base = prp[i];
        const uint32_t cnt = p_row_cols(i, rp, ci, agg, pci + base);
        for (uint32_t s = 0; s < cnt; ++s)
            for (int k = 0; k < BV; ++k) pv[(size_t)(base + s) * BV + k] = 0.0;
        auto slot = [&](uint32_t g) {
            uint32_t lo = 0, hi = cnt;
            while (lo < hi)
            {
                const uint32_t mid = (lo + hi) / 2;
                if (pci[base + mid] < g)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            return base + lo;
        };
        {
            double* I = &pv[(size_t)slot((uint32_t)agg[i]) * BV];
            for (int r = 0; r < BS; ++r) I[r * BS + r] = 1.0;
        }
        const double* Di = &dinv[(size_t)i * BV];
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
        {
            const double* ab = &v[(size_t)p * BV];
            double* dst = &pv[(size_t)slot((uint32_t)agg[ci[p]]) * BV];
            for (int r = 0; r < BS; ++r)
                for (int c = 0; c < BS; ++c)
                {
                    double s = 0.0;
                    for (int m = 0; m < BS; ++m) s += Di[r * BS + m] * ab[m * BS + c];
                    dst[r * BS + c] -= kOmega * s;
                }
        }
    }
}

// ------------------------------------------------------------ block transpose

__global__ void k_bt_count(uint32_t nb, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                           uint32_t* __restrict__ cnt)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p) atomicAdd(&cnt[ci[p]], 1u);
}

// T's entry d = A's entry perm[d], its block transposed; rows ascending by construction
template <int BS>
__global__ void k_bt_gather(uint32_t nnz, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ row_of,
                            const double* __restrict__ v, uint32_t* __restrict__ tci, double* __restrict__ tv)
{
    constexpr int BV = BS * BS;
    for (uint32_t d = blockIdx.x * blockDim.x + threadIdx.x; d < nnz; d += gridDim.x * blockDim.x)
    {
        const uint32_t p = perm[d];
        tci[d] = row_of[p];
#pragma unroll
        for (int r = 0; r < BS; ++r)
#pragma unroll
            for (int c = 0; c < BS; ++c) tv[(size_t)d * BV + r * BS + c] = v[(size_t)p * BV + c * BS + r];
    }
}

template <int BS>
void block_transpose(b2s_ctx* ctx, const BaijDev& A, BaijDev& T)
{
    constexpr int BV = BS * BS;
    T.bs = BS;
    T.nbr = A.nbc;
    T.nbc = A.nbr;
    DBuf<uint32_t> cnt(T.nbr + 1);
    B2S_CUDA(cudaMemsetAsync(cnt.p, 0, cnt.bytes(), ctx->stream));
    if (A.nbr) B2S_LAUNCH(ctx, k_bt_count, stream_grid(ctx, A.nbr), kThreads, 0, A.nbr, A.rp.p, A.ci.p, cnt.p);
    T.rp.alloc(T.nbr + 1);
    const uint32_t nnz = exclusive_scan(ctx, cnt.p, T.rp.p, T.nbr);
    T.ci.alloc(nnz ? nnz : 1);
    T.v.alloc(nnz ? (size_t)nnz * BV : 1);
    DBuf<uint32_t> perm, row_of;
    transpose_order(ctx, A.nbr, A.nbc, A.rp.p, A.ci.p, nnz, perm, row_of);
    if (nnz)
        B2S_LAUNCH(ctx, k_bt_gather<BS>, stream_grid(ctx, nnz), kThreads, 0, nnz, perm.p, row_of.p, A.v.p, T.ci.p,
                   T.v.p);
    finish_baij(ctx, T);
}

// ------------------------------------------------------------ block SpGEMM

__global__ void k_mm_ub(uint32_t nr, const uint32_t* __restrict__ arp, const uint32_t* __restrict__ aci,
                        const uint32_t* __restrict__ brp, uint32_t* __restrict__ cnt)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += gridDim.x * blockDim.x)
    {
        uint32_t c = 0;
        for (uint32_t p = arp[i]; p < arp[i + 1]; ++p) c += brp[aci[p] + 1] - brp[aci[p]];
        cnt[i] = c;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt[nr] = 0;
}

__global__ void k_mm_cand(uint32_t nr, const uint32_t* __restrict__ arp, const uint32_t* __restrict__ aci,
                          const uint32_t* __restrict__ brp, const uint32_t* __restrict__ bci,
                          const uint32_t* __restrict__ off, uint32_t* __restrict__ cand)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += gridDim.x * blockDim.x)
    {
        uint32_t w = off[i];
        for (uint32_t p = arp[i]; p < arp[i + 1]; ++p)
            for (uint32_t q = brp[aci[p]]; q < brp[aci[p] + 1]; ++q) cand[w++] = bci[q];
    }
}

__global__ void k_mm_unique_count(uint32_t nr, const uint32_t* __restrict__ off, const uint32_t* __restrict__ cand,
                                  uint32_t* __restrict__ cnt)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += gridDim.x * blockDim.x)
    {
        uint32_t c = 0;
        for (uint32_t k = off[i]; k < off[i + 1]; ++k) c += (k == off[i] || cand[k] != cand[k - 1]);
        cnt[i] = c;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt[nr] = 0;
}

__global__ void k_mm_unique_fill(uint32_t nr, const uint32_t* __restrict__ off, const uint32_t* __restrict__ cand,
                                 const uint32_t* __restrict__ crp, uint32_t* __restrict__ cci)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += gridDim.x * blockDim.x)
    {
        uint32_t w = crp[i];
        for (uint32_t k = off[i]; k < off[i + 1]; ++k)
            if (k == off[i] || cand[k] != cand[k - 1]) cci[w++] = cand[k];
    }
}

// Symbolic product, one warp per row i of C = A B: the distinct columns of
// the row are collected in a per-warp open-addressing hash table in shared
// memory (inserted with atomicCAS; the lanes take B's row entries in
// parallel).  COUNT: cnt[i] = their number.  Otherwise they are written in
// ascending order (rank sort, the columns being distinct) to cci[crp[i]...].
// A row whose columns do not fit the table raises *overflow and writes
// nothing; the caller then uses the sort-based symbolic product.
constexpr uint32_t kMmHashBits = 9;
constexpr uint32_t kMmHashSlots = 1u << kMmHashBits;  // per warp
constexpr uint32_t kMmEmpty = 0xFFFFFFFFu;

template <bool COUNT>
__global__ void __launch_bounds__(kThreads) k_mm_hash(uint32_t nr, const uint32_t* __restrict__ arp,
                                                      const uint32_t* __restrict__ aci,
                                                      const uint32_t* __restrict__ brp,
                                                      const uint32_t* __restrict__ bci, uint32_t* __restrict__ cnt,
                                                      const uint32_t* __restrict__ crp, uint32_t* __restrict__ cci,
                                                      int* overflow)
{
    __shared__ uint32_t table[kThreads / 32][kMmHashSlots];
    __shared__ uint32_t list[COUNT ? 1 : kThreads / 32][COUNT ? 1 : kMmHashSlots];
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    uint32_t* T = table[wid];
    if (COUNT && blockIdx.x == 0 && threadIdx.x == 0) cnt[nr] = 0;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t i = blockIdx.x * (blockDim.x >> 5) + wid; i < nr; i += warps)
    {
        for (uint32_t s = lane; s < kMmHashSlots; s += 32) T[s] = kMmEmpty;
        __syncwarp();
        uint32_t added = 0;
        bool full = false;
        const uint32_t a1 = arp[i + 1];
        for (uint32_t pa = arp[i]; pa < a1 && !full; ++pa)
        {
            const uint32_t k = aci[pa];
            const uint32_t b1 = brp[k + 1];
            for (uint32_t pb = brp[k] + lane; pb < b1; pb += 32)
            {
                const uint32_t j = bci[pb];
                uint32_t h = (j * 2654435761u) >> (32 - kMmHashBits);
                for (uint32_t probes = 0;; ++probes)
                {
                    if (probes == kMmHashSlots)
                    {
                        full = true;
                        break;
                    }
                    const uint32_t old = atomicCAS(&T[h], kMmEmpty, j);
                    if (old == kMmEmpty) ++added;
                    if (old == kMmEmpty || old == j) break;
                    h = (h + 1) & (kMmHashSlots - 1);
                }
            }
        }
        __syncwarp();
        if (__any_sync(0xffffffffu, full))
        {
            if (lane == 0)
            {
                atomicExch(overflow, 1);
                if (COUNT) cnt[i] = 0;
            }
            __syncwarp();
            continue;
        }
        uint32_t tot = added;
#pragma unroll
        for (int o = 16; o; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
        if (COUNT)
        {
            if (lane == 0) cnt[i] = tot;
        }
        else
        {
            uint32_t* Lst = list[wid];
            uint32_t base = 0;
            for (uint32_t s0 = 0; s0 < kMmHashSlots; s0 += 32)
            {
                const uint32_t v = T[s0 + lane];
                const bool has = v != kMmEmpty;
                const uint32_t m = __ballot_sync(0xffffffffu, has);
                if (has) Lst[base + __popc(m & ((1u << lane) - 1u))] = v;
                base += __popc(m);
            }
            __syncwarp();
            const uint32_t out = crp[i];
            for (uint32_t a = lane; a < base; a += 32)
            {
                const uint32_t v = Lst[a];
                uint32_t r = 0;
                for (uint32_t b = 0; b < base; ++b) r += Lst[b] < v;
                cci[out + r] = v;
            }
        }
        __syncwarp();  // the table and list are reused by the next row
    }
}

// C row i: every (pa, pb) product added into its column's block in the
// reference's order (blk_matmul, blockMatrix.hpp:883-932)
template <int BS>
__global__ void k_mm_numeric(uint32_t nr, const uint32_t* __restrict__ arp, const uint32_t* __restrict__ aci,
                             const double* __restrict__ av, const uint32_t* __restrict__ brp,
                             const uint32_t* __restrict__ bci, const double* __restrict__ bv,
                             const uint32_t* __restrict__ crp, const uint32_t* __restrict__ cci, double* __restrict__ cv)
{
    constexpr int BV = BS * BS;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += gridDim.x * blockDim.x)
    {
        const uint32_t c0 = crp[i], c1 = crp[i + 1];
        for (uint32_t s = c0; s < c1; ++s)
            for (int k = 0; k < BV; ++k) cv[(size_t)s * BV + k] = 0.0;
        for (uint32_t pa = arp[i]; pa < arp[i + 1]; ++pa)
        {
            const uint32_t k = aci[pa];
            const double* ab = &av[(size_t)pa * BV];
            for (uint32_t pb = brp[k]; pb < brp[k + 1]; ++pb)
            {
                const uint32_t j = bci[pb];
                uint32_t lo = c0, hi = c1;
                while (lo < hi)
                {
                    const uint32_t mid = (lo + hi) / 2;
                    if (cci[mid] < j)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                const double* bb = &bv[(size_t)pb * BV];
                double* cb = &cv[(size_t)lo * BV];
                for (int r = 0; r < BS; ++r)
                    for (int c = 0; c < BS; ++c)
                    {
                        double s = 0.0;
                        for (int m = 0; m < BS; ++m) s += ab[r * BS + m] * bb[m * BS + c];
                        cb[r * BS + c] += s;
                    }
            }
        }
    }
}

// The same product, one warp per C row: the warp walks A's row entries pa in
// order and its lanes take the entries pb of B's row k in parallel.  The
// entries of one B row have distinct columns, so within a pa no two lanes add
// into the same C block, and a __syncwarp between pa keeps every C block's
// additions in pa order -- the order of k_mm_numeric.  Used when B's rows are
// long (R (A P)); for short rows (A P) the thread-per-row kernel is faster.
template <int BS>
__global__ void k_mm_numeric_warp(uint32_t nr, const uint32_t* __restrict__ arp, const uint32_t* __restrict__ aci,
                                  const double* __restrict__ av, const uint32_t* __restrict__ brp,
                                  const uint32_t* __restrict__ bci, const double* __restrict__ bv,
                                  const uint32_t* __restrict__ crp, const uint32_t* __restrict__ cci,
                                  double* __restrict__ cv)
{
    constexpr int BV = BS * BS;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < nr; i += warps)
    {
        const uint32_t c0 = crp[i], c1 = crp[i + 1];
        for (uint32_t s = c0 * BV + lane; s < c1 * BV; s += 32) cv[s] = 0.0;
        __syncwarp();
        for (uint32_t pa = arp[i]; pa < arp[i + 1]; ++pa)
        {
            const uint32_t k = aci[pa];
            double ab[BV];
#pragma unroll
            for (int q = 0; q < BV; ++q) ab[q] = av[(size_t)pa * BV + q];
            for (uint32_t pb = brp[k] + lane; pb < brp[k + 1]; pb += 32)
            {
                const uint32_t j = bci[pb];
                uint32_t lo = c0, hi = c1;
                while (lo < hi)
                {
                    const uint32_t mid = (lo + hi) / 2;
                    if (cci[mid] < j)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                const double* bb = &bv[(size_t)pb * BV];
                double* cb = &cv[(size_t)lo * BV];
#pragma unroll
                for (int r = 0; r < BS; ++r)
#pragma unroll
                    for (int c = 0; c < BS; ++c)
                    {
                        double sum = 0.0;
#pragma unroll
                        for (int m = 0; m < BS; ++m) sum += ab[r * BS + m] * bb[m * BS + c];
                        cb[r * BS + c] += sum;
                    }
            }
            __syncwarp();
        }
    }
}

template <int BS>
void block_matmul(b2s_ctx* ctx, const BaijDev& A, const BaijDev& B, BaijDev& C)
{
    constexpr int BV = BS * BS;
    const uint32_t nr = A.nbr;
    C.bs = BS;
    C.nbr = nr;
    C.nbc = B.nbc;
    DBuf<uint32_t> cnt(nr + 1);
    C.rp.alloc(nr + 1);
    // symbolic: per-warp hash tables; rows too wide for them send the whole
    // product to the candidate-sort path
    DBuf<int> overflow(1);
    B2S_CUDA(cudaMemsetAsync(overflow.p, 0, sizeof(int), ctx->stream));
    const uint64_t hash_ctas = ((uint64_t)nr + kThreads / 32 - 1) / (kThreads / 32);
    const unsigned hash_grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(hash_ctas, (uint64_t)ctx->sm_count * 8));
    if (nr)
        B2S_LAUNCH(ctx, k_mm_hash<true>, hash_grid, kThreads, 0, nr, A.rp.p, A.ci.p, B.rp.p, B.ci.p, cnt.p,
                   (const uint32_t*)nullptr, (uint32_t*)nullptr, overflow.p);
    uint32_t nnz = exclusive_scan(ctx, cnt.p, C.rp.p, nr);
    int wide = 0;
    d2h(ctx, &wide, overflow.p, sizeof(int));
    sync(ctx);
    if (!wide)
    {
        C.ci.alloc(nnz ? nnz : 1);
        if (nr)
            B2S_LAUNCH(ctx, k_mm_hash<false>, hash_grid, kThreads, 0, nr, A.rp.p, A.ci.p, B.rp.p, B.ci.p,
                       (uint32_t*)nullptr, C.rp.p, C.ci.p, overflow.p);
    }
    else
    {
        DBuf<uint32_t> off(nr + 1);
        if (nr) B2S_LAUNCH(ctx, k_mm_ub, stream_grid(ctx, nr), kThreads, 0, nr, A.rp.p, A.ci.p, B.rp.p, cnt.p);
        const uint32_t total = exclusive_scan(ctx, cnt.p, off.p, nr);
        DBuf<uint32_t> cand(total ? total : 1), sorted(total ? total : 1);
        if (nr)
            B2S_LAUNCH(ctx, k_mm_cand, stream_grid(ctx, nr), kThreads, 0, nr, A.rp.p, A.ci.p, B.rp.p, B.ci.p, off.p,
                       cand.p);
        if (total)
        {
            size_t bytes = 0;
            B2S_CUDA(cub::DeviceSegmentedSort::SortKeys(nullptr, bytes, cand.p, sorted.p, (int64_t)total, (int64_t)nr,
                                                        off.p, off.p + 1, ctx->stream));
            DBuf<uint8_t> tmp(bytes ? bytes : 1);
            B2S_CUDA(cub::DeviceSegmentedSort::SortKeys(tmp.p, bytes, cand.p, sorted.p, (int64_t)total, (int64_t)nr,
                                                        off.p, off.p + 1, ctx->stream));
            ctx->launches += 1;
        }
        if (nr) B2S_LAUNCH(ctx, k_mm_unique_count, stream_grid(ctx, nr), kThreads, 0, nr, off.p, sorted.p, cnt.p);
        nnz = exclusive_scan(ctx, cnt.p, C.rp.p, nr);
        C.ci.alloc(nnz ? nnz : 1);
        if (nr) B2S_LAUNCH(ctx, k_mm_unique_fill, stream_grid(ctx, nr), kThreads, 0, nr, off.p, sorted.p, C.rp.p, C.ci.p);
    }
    C.v.alloc(nnz ? (size_t)nnz * BV : 1);
    if (nr)
    {
        // B's mean row length decides: warp per C row for long rows, thread per C row otherwise
        if (B.nbr && B.nnzb >= 8ull * B.nbr)
        {
            const uint64_t warps = nr, ctas = (warps + kThreads / 32 - 1) / (kThreads / 32);
            const unsigned grid = (unsigned)std::min<uint64_t>(ctas, (uint64_t)ctx->sm_count * 8);
            B2S_LAUNCH(ctx, k_mm_numeric_warp<BS>, grid, kThreads, 0, nr, A.rp.p, A.ci.p, A.v.p, B.rp.p, B.ci.p,
                       B.v.p, C.rp.p, C.ci.p, C.v.p);
        }
        else
            B2S_LAUNCH(ctx, k_mm_numeric<BS>, stream_grid(ctx, nr), kThreads, 0, nr, A.rp.p, A.ci.p, A.v.p, B.rp.p,
                       B.ci.p, B.v.p, C.rp.p, C.ci.p, C.v.p);
    }
    finish_baij(ctx, C);
}

// ------------------------------------------------------------ coarsest level

template <int BS>
__global__ void k_dense_from_baij(uint32_t nb, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                  const double* __restrict__ v, double* __restrict__ D, int sz)
{
    constexpr int BV = BS * BS;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
            for (int r = 0; r < BS; ++r)
                for (int c = 0; c < BS; ++c)
                    D[(size_t)(i * BS + r) * sz + ci[p] * BS + c] = v[(size_t)p * BV + r * BS + c];
}

// One CTA.  ref == 1: the reference's elimination (blockMatrix.hpp:962-981):
// rows swapped, pivot clamped to +-1e-14, the multiplier column eliminated
// along with the row (j from k).  ref == 0: LU with partial pivoting,
// multipliers stored below the diagonal and the permutation kept in piv.
__global__ void k_dense_factor(double* D, int sz, int ref, int* piv)
{
    __shared__ int s_pk;
    __shared__ double s_red[kThreads];
    __shared__ int s_idx[kThreads];
    for (int i = threadIdx.x; i < sz; i += blockDim.x) piv[i] = i;
    __syncthreads();
    for (int k = 0; k < sz; ++k)
    {
        // first row with the largest |D[i][k]|, i >= k (strict > keeps the earliest)
        double best = -1.0;
        int bi = k;
        for (int i = k + threadIdx.x; i < sz; i += blockDim.x)
        {
            const double a = fabs(D[(size_t)i * sz + k]);
            if (a > best)
            {
                best = a;
                bi = i;
            }
        }
        s_red[threadIdx.x] = best;
        s_idx[threadIdx.x] = bi;
        __syncthreads();
        if (threadIdx.x == 0)
        {
            // the earliest row attaining the maximum, as the sequential scan finds it
            double b = -1.0;
            int pk = k;
            for (int t = 0; t < (int)blockDim.x; ++t)
                if (s_red[t] > b || (s_red[t] == b && s_idx[t] < pk))
                {
                    b = s_red[t];
                    pk = s_idx[t];
                }
            s_pk = pk;
        }
        __syncthreads();
        const int pk = s_pk;
        if (pk != k)
        {
            for (int j = threadIdx.x; j < sz; j += blockDim.x)
            {
                const double t = D[(size_t)k * sz + j];
                D[(size_t)k * sz + j] = D[(size_t)pk * sz + j];
                D[(size_t)pk * sz + j] = t;
            }
            if (threadIdx.x == 0 && !ref)
            {
                const int t = piv[k];
                piv[k] = piv[pk];
                piv[pk] = t;
            }
        }
        __syncthreads();
        double d = D[(size_t)k * sz + k];
        if (ref)
        {
            if (fabs(d) < 1e-14) d = (d >= 0 ? 1e-14 : -1e-14);
        }
        else if (fabs(d) < 1e-300)
        {
            d = 1e-300;
            if (threadIdx.x == 0) D[(size_t)k * sz + k] = d;
        }
        for (int i = k + 1 + threadIdx.x; i < sz; i += blockDim.x)
        {
            const double f = D[(size_t)i * sz + k] / d;
            if (ref)
                for (int j = k; j < sz; ++j) D[(size_t)i * sz + j] -= f * D[(size_t)k * sz + j];
            else
            {
                D[(size_t)i * sz + k] = f;
                for (int j = k + 1; j < sz; ++j) D[(size_t)i * sz + j] -= f * D[(size_t)k * sz + j];
            }
        }
        __syncthreads();
    }
}

// coarsest solve, one thread (the row sums are sequential in the reference)
__global__ void k_dense_solve(const double* __restrict__ D, int sz, int ref, const int* __restrict__ piv,
                              const double* __restrict__ rhs, double* __restrict__ x, const int* done)
{
    if (done && *done) return;
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    // Each row's running value stays in a register while its terms are
    // subtracted in the same order as an in-place x[i] -= ... loop would.
    if (ref)
    {
        for (int i = 0; i < sz; ++i) x[i] = rhs[i];
        for (int k = 0; k < sz; ++k)
        {
            double d = D[(size_t)k * sz + k];
            if (fabs(d) < 1e-14) d = (d >= 0 ? 1e-14 : -1e-14);
            const double xk = x[k];
            for (int i = k + 1; i < sz; ++i) x[i] -= (D[(size_t)i * sz + k] / d) * xk;
        }
        for (int i = sz - 1; i >= 0; --i)
        {
            double xi = x[i];
            for (int j = i + 1; j < sz; ++j) xi -= D[(size_t)i * sz + j] * x[j];
            double d = D[(size_t)i * sz + i];
            if (fabs(d) < 1e-14) d = (d >= 0 ? 1e-14 : -1e-14);
            x[i] = xi / d;
        }
    }
    else
    {
        for (int i = 0; i < sz; ++i)
        {
            double xi = rhs[piv[i]];
            for (int j = 0; j < i; ++j) xi -= D[(size_t)i * sz + j] * x[j];
            x[i] = xi;
        }
        for (int i = sz - 1; i >= 0; --i)
        {
            double xi = x[i];
            for (int j = i + 1; j < sz; ++j) xi -= D[(size_t)i * sz + j] * x[j];
            x[i] = xi / D[(size_t)i * sz + i];
        }
    }
}

// ------------------------------------------------------------ V-cycle kernels

// pre-smoothing from zero: sol = omega * dinv * rhs   (A*0 = 0, so r = rhs)
template <int BS, typename T>
__global__ void k_smooth0(uint32_t nb, const T* __restrict__ dinv, const double* __restrict__ rhs,
                          double* __restrict__ sol, const int* done)
{
    if (done && *done) return;
    constexpr int BV = BS * BS;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
        for (int c = 0; c < BS; ++c)
        {
            double corr = 0.0;
            for (int rr = 0; rr < BS; ++rr) corr += (double)dinv[(size_t)i * BV + c * BS + rr] * rhs[(size_t)i * BS + rr];
            sol[(size_t)i * BS + c] = 0.0 + kOmega * corr;
        }
}

// Epilogues of the V-cycle's block products (baij_mv.cuh).  Each repeats the
// arithmetic of the separate vector pass it replaces, so the cycle's output is
// unchanged bit for bit.

// res = rhs - A sol
struct EpiResidual
{
    const double* rhs;
    double* res;
    template <int BS>
    __device__ __forceinline__ void put(uint32_t I, int r, double v, bool valid, uint32_t) const
    {
        if (!valid) return;
        const size_t i = (size_t)I * BS + r;
        res[i] = rhs[i] - v;
    }
};

// dst = sol + P e (coarse-grid correction)
struct EpiAddTo
{
    const double* sol;
    double* dst;
    template <int BS>
    __device__ __forceinline__ void put(uint32_t I, int r, double v, bool valid, uint32_t) const
    {
        if (!valid) return;
        const size_t i = (size_t)I * BS + r;
        dst[i] = sol[i] + v;
    }
};

// post-smoothing: sol = mid + omega * dinv * (rhs - A mid).  A block row's
// residual components come from the BS lanes of its row.
template <typename T>
struct EpiJacobi
{
    const T* dinv;
    const double* rhs;
    const double* mid;
    double* sol;
    template <int BS>
    __device__ __forceinline__ void put(uint32_t I, int r, double v, bool valid, uint32_t lane) const
    {
        constexpr int BV = BS * BS;
        const size_t i = (size_t)I * BS + r;
        const double res = valid ? rhs[i] - v : 0.0;
        double rv[BS];
        if constexpr (BS == 1)
            rv[0] = res;
        else
#pragma unroll
            for (int q = 0; q < BS; ++q) rv[q] = __shfl_sync(0xffffffffu, res, (lane / BS) * BS + q);
        if (!valid) return;
        double corr = 0.0;
#pragma unroll
        for (int q = 0; q < BS; ++q) corr += (double)dinv[(size_t)I * BV + r * BS + q] * rv[q];
        sol[i] = mid[i] + kOmega * corr;
    }
};

__global__ void k_zero(uint64_t n, double* __restrict__ x, const int* done)
{
    if (done && *done) return;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        x[i] = 0.0;
}

// ------------------------------------------------------------ hierarchy

struct Level
{
    std::unique_ptr<BaijDev> own;  // operator (null on level 0 when borrowed)
    const BaijDev* A = nullptr;
    BaijDev P, R;
    DBuf<double> dinv;
    DBuf<int32_t> agg;
    uint32_t nrows = 0;
    bool has_p = false;
    DBuf<double> tmp, r, rc, ec, sol;  // V-cycle work (rc / ec sized for the next level)
    DBuf<float> A32, P32, R32, dinv32;  // FP32 copies of the values (precision FP32)
};

__global__ void k_amg_to_f32(const double* __restrict__ a, float* __restrict__ b, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

static void amg_to_f32(b2s_ctx* ctx, const double* a, DBuf<float>& b, uint64_t n)
{
    b.alloc(n ? n : 1);
    if (n) B2S_LAUNCH(ctx, k_amg_to_f32, stream_grid(ctx, n), kThreads, 0, a, b.p, n);
}

struct PcAMG final : PcImpl
{
    int bs = 1;
    bool ref_coarse = false;
    bool fp32 = false;  // V-cycle reads FP32 copies of A, P, R and D^-1 (FP64 arithmetic and vectors)
    int aggregation = 0;  // b2s_pc_opts::amg_aggregation
    std::vector<std::unique_ptr<Level>> lv;
    std::unique_ptr<BaijDev> fine_copy;  // BS=1 copy of a CSR operator
    DBuf<double> dense;
    DBuf<int> piv;
    int sz = 0;

    template <int BS>
    void vcycle(b2s_ctx* ctx, int l, const double* rhs, double* sol, const int* done)
    {
        Level& L = *lv[l];
        const unsigned g = stream_grid(ctx, L.nrows);
        if (l == (int)lv.size() - 1)
        {
            B2S_LAUNCH(ctx, k_dense_solve, 1, 32, 0, dense.p, sz, ref_coarse ? 1 : 0, piv.p, rhs, sol, done);
            return;
        }
        // products on FP64 or FP32 values, each with its epilogue
        auto mv = [&](const BaijDev& M, const DBuf<float>& v32, const double* x, auto epi) {
            if (fp32)
                baij_mv<BS>(ctx, M, v32.p, x, epi, done);
            else
                baij_mv<BS>(ctx, M, M.v.p, x, epi, done);
        };
        // pre-smoothing from zero, residual, restriction
        if (fp32)
            B2S_LAUNCH(ctx, (k_smooth0<BS, float>), g, kThreads, 0, L.nrows, L.dinv32.p, rhs, sol, done);
        else
            B2S_LAUNCH(ctx, (k_smooth0<BS, double>), g, kThreads, 0, L.nrows, L.dinv.p, rhs, sol, done);
        mv(*L.A, L.A32, sol, EpiResidual{rhs, L.r.p});
        mv(L.R, L.R32, L.r.p, EpiStoreY{L.rc.p});
        const uint64_t nc = (uint64_t)L.R.nbr * BS;
        if (l + 1 < (int)lv.size() - 1)
            vcycle<BS>(ctx, l + 1, L.rc.p, L.ec.p, done);
        else
        {
            B2S_LAUNCH(ctx, k_zero, stream_grid(ctx, nc), kThreads, 0, nc, L.ec.p, done);
            vcycle<BS>(ctx, l + 1, L.rc.p, L.ec.p, done);
        }
        // coarse-grid correction into tmp, then post-smoothing back into sol
        mv(L.P, L.P32, L.ec.p, EpiAddTo{sol, L.tmp.p});
        if (fp32)
            mv(*L.A, L.A32, L.tmp.p, EpiJacobi<float>{L.dinv32.p, rhs, L.tmp.p, sol});
        else
            mv(*L.A, L.A32, L.tmp.p, EpiJacobi<double>{L.dinv.p, rhs, L.tmp.p, sol});
    }

    void apply(b2s_ctx* ctx, const double* r, double* z, const int* done) override
    {
        switch (bs)
        {
            case 1: vcycle<1>(ctx, 0, r, z, done); break;
            case 2: vcycle<2>(ctx, 0, r, z, done); break;
            case 3: vcycle<3>(ctx, 0, r, z, done); break;
            case 4: vcycle<4>(ctx, 0, r, z, done); break;
        }
    }

    void export_baij(b2s_ctx* ctx, const BaijDev& M, uint64_t* sizes, uint32_t* rp, uint32_t* ci, double* v)
    {
        const size_t bv = (size_t)M.bs * M.bs;
        sizes[0] = (uint64_t)M.nbr + 1;
        sizes[1] = M.nnzb;
        sizes[2] = (uint64_t)M.nnzb * bv;
        if (rp) d2h(ctx, rp, M.rp.p, (M.nbr + 1) * sizeof(uint32_t));
        if (ci) d2h(ctx, ci, M.ci.p, M.nnzb * sizeof(uint32_t));
        if (v) d2h(ctx, v, M.v.p, M.nnzb * bv * sizeof(double));
        sync(ctx);
    }

    void export_data(b2s_ctx* ctx, const std::string& what, uint64_t* sizes, uint32_t* rp, uint32_t* ci,
                     double* v) override
    {
        if (what == "amg.levels")
        {
            sizes[0] = 0;
            sizes[1] = lv.size();
            sizes[2] = 0;
            if (ci)
                for (size_t k = 0; k < lv.size(); ++k) ci[k] = lv[k]->nrows;
            return;
        }
        unsigned l = 0;
        char tail[32] = {0};
        if (std::sscanf(what.c_str(), "amg.%u.%31s", &l, tail) == 2 && l < lv.size())
        {
            Level& L = *lv[l];
            const std::string t(tail);
            if (t == "A") return export_baij(ctx, *L.A, sizes, rp, ci, v);
            if (t == "P" && L.has_p) return export_baij(ctx, L.P, sizes, rp, ci, v);
            if (t == "dinv")
            {
                sizes[0] = 0;
                sizes[1] = 0;
                sizes[2] = (uint64_t)L.nrows * bs * bs;
                if (v) d2h(ctx, v, L.dinv.p, sizes[2] * sizeof(double));
                sync(ctx);
                return;
            }
            if (t == "agg" && L.has_p)
            {
                sizes[0] = 0;
                sizes[1] = L.nrows;
                sizes[2] = 0;
                if (ci) d2h(ctx, ci, L.agg.p, L.nrows * sizeof(uint32_t));
                sync(ctx);
                return;
            }
        }
        PcImpl::export_data(ctx, what, sizes, rp, ci, v);
    }
};

template <int BS>
void build_hierarchy(b2s_ctx* ctx, PcAMG& pc, const BaijDev& A0, int max_levels, uint32_t coarse_max)
{
    constexpr int BV = BS * BS;
    const BaijDev* cur = &A0;
    std::unique_ptr<BaijDev> cur_own;
    for (int lvl = 0; lvl < max_levels; ++lvl)
    {
        auto L = std::make_unique<Level>();
        const uint32_t n = cur->nbr;
        L->nrows = n;
        L->own = std::move(cur_own);
        L->A = cur;
        L->dinv.alloc((size_t)n * BV + 1);
        if (n) B2S_LAUNCH(ctx, k_diag_inv<BS>, stream_grid(ctx, n), kThreads, 0, n, cur->v.p, cur->diag_ptr.p, L->dinv.p);
        if (n <= coarse_max)
        {
            pc.lv.push_back(std::move(L));
            cur = nullptr;
            break;
        }
        // strength
        DBuf<uint32_t> cnt(n + 1), sp(n + 1);
        B2S_LAUNCH(ctx, k_strength<BS>, stream_grid(ctx, n), kThreads, 0, n, cur->rp.p, cur->ci.p, cur->v.p,
                   (const uint32_t*)nullptr, cnt.p, (uint32_t*)nullptr);
        const uint32_t ns = exclusive_scan(ctx, cnt.p, sp.p, n);
        DBuf<uint32_t> sc(ns ? ns : 1);
        B2S_LAUNCH(ctx, k_strength<BS>, stream_grid(ctx, n), kThreads, 0, n, cur->rp.p, cur->ci.p, cur->v.p, sp.p,
                   (uint32_t*)nullptr, sc.p);
        // aggregation
        L->agg.alloc(n);
        B2S_CUDA(cudaMemsetAsync(L->agg.p, 0xFF, (size_t)n * sizeof(int32_t), ctx->stream));
        uint32_t nagg = 0;
        if (pc.aggregation == 0)
            nagg = aggregate_parallel(ctx, n, sp.p, sc.p, L->agg.p);
        else
        {
            DBuf<uint32_t> nagg_d(1);
            if (pc.aggregation == 1)
                B2S_LAUNCH(ctx, k_aggregate, 1, 32, 0, n, sp.p, sc.p, L->agg.p, nagg_d.p);
            else
            {
                DBuf<int32_t> snap(n);
                B2S_LAUNCH(ctx, k_aggregate_std, 1, 32, 0, n, sp.p, sc.p, L->agg.p, snap.p, nagg_d.p);
                sync(ctx);
            }
            d2h(ctx, &nagg, nagg_d.p, sizeof(uint32_t));
            sync(ctx);
        }
        // smoothed prolongation
        L->P.bs = BS;
        L->P.nbr = n;
        L->P.nbc = nagg;
        B2S_LAUNCH(ctx, k_p_count, stream_grid(ctx, n), kThreads, 0, n, cur->rp.p, cur->ci.p, L->agg.p, cnt.p);
        L->P.rp.alloc(n + 1);
        const uint32_t pn = exclusive_scan(ctx, cnt.p, L->P.rp.p, n);
        L->P.ci.alloc(pn ? pn : 1);
        L->P.v.alloc(pn ? (size_t)pn * BV : 1);
        B2S_LAUNCH(ctx, k_p_fill<BS>, stream_grid(ctx, n), kThreads, 0, n, cur->rp.p, cur->ci.p, cur->v.p, L->dinv.p,
                   L->agg.p, L->P.rp.p, L->P.ci.p, L->P.v.p);
        finish_baij(ctx, L->P);
        block_transpose<BS>(ctx, L->P, L->R);
        L->has_p = true;
        // Galerkin
        BaijDev AP;
        block_matmul<BS>(ctx, *cur, L->P, AP);
        cur_own = std::make_unique<BaijDev>();
        block_matmul<BS>(ctx, L->R, AP, *cur_own);
        cur = cur_own.get();
        pc.lv.push_back(std::move(L));
    }
    // work vectors
    for (size_t k = 0; k < pc.lv.size(); ++k)
    {
        Level& L = *pc.lv[k];
        const size_t nd = (size_t)L.nrows * BS + 1;
        L.tmp.alloc(nd);
        L.r.alloc(nd);
        if (L.has_p)
        {
            const size_t nc = (size_t)L.R.nbr * BS + 1;
            L.rc.alloc(nc);
            L.ec.alloc(nc);
        }
    }
    // coarsest dense operator (the last level; if max_levels was reached its P is unused)
    Level& C = *pc.lv.back();
    pc.sz = (int)(C.nrows * BS);
    pc.dense.alloc((size_t)pc.sz * pc.sz + 1);
    pc.piv.alloc(pc.sz + 1);
    B2S_CUDA(cudaMemsetAsync(pc.dense.p, 0, pc.dense.bytes(), ctx->stream));
    if (C.nrows)
        B2S_LAUNCH(ctx, k_dense_from_baij<BS>, stream_grid(ctx, C.nrows), kThreads, 0, C.nrows, C.A->rp.p, C.A->ci.p,
                   C.A->v.p, pc.dense.p, pc.sz);
    B2S_LAUNCH(ctx, k_dense_factor, 1, kThreads, 0, pc.dense.p, pc.sz, pc.ref_coarse ? 1 : 0, pc.piv.p);
    // FP32 copies of every operator the V-cycle multiplies by (the coarsest level is the dense LU, kept in FP64)
    if (pc.fp32)
        for (size_t k = 0; k + 1 < pc.lv.size(); ++k)
        {
            Level& L = *pc.lv[k];
            amg_to_f32(ctx, L.A->v.p, L.A32, (uint64_t)L.A->nnzb * BV);
            amg_to_f32(ctx, L.P.v.p, L.P32, (uint64_t)L.P.nnzb * BV);
            amg_to_f32(ctx, L.R.v.p, L.R32, (uint64_t)L.R.nnzb * BV);
            amg_to_f32(ctx, L.dinv.p, L.dinv32, (uint64_t)L.nrows * BV);
        }
    sync(ctx);
}

std::unique_ptr<PcImpl> build_amg(b2s_ctx* ctx, const BaijDev& A, const b2s_pc_opts& o,
                                  std::unique_ptr<BaijDev> owned)
{
    need(A.nbr == A.nbc, B2S_SHAPE, "block AMG needs a square block matrix");
    auto pc = std::make_unique<PcAMG>();
    pc->bs = A.bs;
    pc->ref_coarse = o.amg_ref_coarse != 0;
    pc->fp32 = o.precision != B2S_FP64;
    pc->aggregation = o.amg_aggregation;
    pc->fine_copy = std::move(owned);
    const int max_levels = o.amg_max_levels > 0 ? o.amg_max_levels : 20;
    const uint32_t coarse_max = o.amg_coarse_max > 0 ? (uint32_t)o.amg_coarse_max : 50u;
    switch (A.bs)
    {
        case 1: build_hierarchy<1>(ctx, *pc, A, max_levels, coarse_max); break;
        case 2: build_hierarchy<2>(ctx, *pc, A, max_levels, coarse_max); break;
        case 3: build_hierarchy<3>(ctx, *pc, A, max_levels, coarse_max); break;
        case 4: build_hierarchy<4>(ctx, *pc, A, max_levels, coarse_max); break;
        default: fail(B2S_UNSUPPORTED, "block size must be 1..4");
    }
    return pc;
}

}  // namespace

std::unique_ptr<PcImpl> make_pc_amg_baij(b2s_ctx* ctx, const BaijDev& A, const b2s_pc_opts& o)
{
    return build_amg(ctx, A, o, nullptr);
}

// scalar SA-AMG: BlockMatrix<double,1>::condense of the CSR operator, which
// for a block size of 1 is the same pattern and values
std::unique_ptr<PcImpl> make_pc_amg_csr(b2s_ctx* ctx, const CsrDev& A, const b2s_pc_opts& o)
{
    need(A.n == A.m, B2S_SHAPE, "AMG needs a square matrix");
    auto B = std::make_unique<BaijDev>();
    B->bs = 1;
    B->nbr = A.n;
    B->nbc = A.m;
    B->rp.alloc(A.n + 1);
    B->ci.alloc(A.nnz ? A.nnz : 1);
    B->v.alloc(A.nnz ? A.nnz : 1);
    d2d(ctx, B->rp.p, A.rp.p, (A.n + 1) * sizeof(uint32_t));
    d2d(ctx, B->ci.p, A.ci.p, A.nnz * sizeof(uint32_t));
    d2d(ctx, B->v.p, A.v.p, A.nnz * sizeof(double));
    finish_baij(ctx, *B);
    const BaijDev& ref = *B;
    return build_amg(ctx, ref, o, std::move(B));
}

// scalar (bs = 1) product and transpose for general CSR operators: the
// C ABI's b2s_csr_matmul / b2s_csr_transpose (csr.cu)
void scalar_matmul(b2s_ctx* ctx, const BaijDev& A, const BaijDev& B, BaijDev& C) { block_matmul<1>(ctx, A, B, C); }
void scalar_transpose(b2s_ctx* ctx, const BaijDev& A, BaijDev& T) { block_transpose<1>(ctx, A, T); }

}  // namespace b2s
