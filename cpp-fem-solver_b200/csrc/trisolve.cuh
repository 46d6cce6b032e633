// Level schedules of triangular dependency DAGs and the two ways of running
// a per-row operation over them (one launch per level, or one sync-free
// launch).  Shared by the scalar and block incomplete factorisations.
#pragma once
#include <cub/cub.cuh>

#include <algorithm>

#include "syncfree.cuh"

namespace b2s {

// ------------------------------------------------------------ scan / sort

static inline uint32_t exclusive_scan(b2s_ctx* ctx, const uint32_t* in, uint32_t* out, uint32_t n)
{
    // out has n+1 entries; out[n] = total
    size_t bytes = 0;
    B2S_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n + 1, ctx->stream));
    DBuf<uint8_t> tmp(bytes ? bytes : 1);
    B2S_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, bytes, in, out, n + 1, ctx->stream));
    ctx->launches += 1;
    uint32_t total = 0;
    d2h(ctx, &total, out + n, sizeof(uint32_t));
    sync(ctx);
    return total;
}

static __global__ void k_iota(uint32_t* a, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = i;
}

static __global__ void k_level_bounds(const uint32_t* __restrict__ sorted_lev, uint32_t n, uint32_t* __restrict__ lptr)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const uint32_t l = sorted_lev[i];
        if (i == 0)
            for (uint32_t k = 0; k <= l; ++k) lptr[k] = 0;
        else
        {
            const uint32_t p = sorted_lev[i - 1];
            for (uint32_t k = p + 1; k <= l; ++k) lptr[k] = i;
        }
        if (i == n - 1) lptr[l + 1] = n;
    }
}

// ------------------------------------------------------------ stable transpose order

static __global__ void k_entry_rows(uint32_t n, const uint32_t* __restrict__ rp, uint32_t* __restrict__ row_of)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p) row_of[p] = i;
}

// Entry order of a CSR pattern's transpose: after the call, perm[d] (d in
// column-major order) is the index of the d-th entry of the transpose in the
// original arrays, and row_of[p] is the row of entry p.  A stable radix sort
// by column keeps the rows of each column ascending, so the transpose rows
// come out sorted without a per-row sort.  Entries with ci[p] >= ncols are
// not expected.
static inline void transpose_order(b2s_ctx* ctx, uint32_t nrows, uint32_t ncols, const uint32_t* rp,
                                   const uint32_t* ci, uint32_t nnz, DBuf<uint32_t>& perm, DBuf<uint32_t>& row_of)
{
    perm.alloc(nnz ? nnz : 1);
    row_of.alloc(nnz ? nnz : 1);
    if (!nnz) return;
    B2S_LAUNCH(ctx, k_entry_rows, stream_grid(ctx, nrows), kThreads, 0, nrows, rp, row_of.p);
    DBuf<uint32_t> iota(nnz), keys_out(nnz);
    B2S_LAUNCH(ctx, k_iota, stream_grid(ctx, nnz), kThreads, 0, iota.p, nnz);
    int end_bit = 1;
    while (end_bit < 32 && (ncols - 1) >> end_bit) ++end_bit;
    size_t bytes = 0;
    B2S_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, ci, keys_out.p, iota.p, perm.p, (int)nnz, 0, end_bit,
                                             ctx->stream));
    DBuf<uint8_t> tmp(bytes ? bytes : 1);
    B2S_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, bytes, ci, keys_out.p, iota.p, perm.p, (int)nnz, 0, end_bit,
                                             ctx->stream));
    ctx->launches += 1;
}

// ------------------------------------------------------------ level sets

template <bool LOWER>
struct LevelOp
{
    const uint32_t *rp, *ci;
    uint32_t* level;
    __device__ bool ready(uint32_t row, const uint32_t* flags, uint32_t epoch) const
    {
        return deps_ready<LOWER>(row, rp, ci, flags, epoch);
    }
    __device__ void compute(uint32_t row) const
    {
        uint32_t l = 0;
        for (uint32_t p = __ldg(&rp[row]); p < __ldg(&rp[row + 1]); ++p)
        {
            const uint32_t j = __ldg(&ci[p]);
            if (LOWER ? (j < row) : (j > row))
            {
                const uint32_t lj = __ldcg(&level[j]) + 1;
                l = lj > l ? lj : l;
            }
        }
        level[row] = l;
    }
};

struct LevelSchedule
{
    uint32_t n = 0, nlev = 0;
    DBuf<uint32_t> level;       // level of each row
    DBuf<uint32_t> rows;        // rows sorted by (level, index)
    std::vector<uint32_t> h_ptr;  // nlev + 1

    // from levels computed on the host (compute_levels): rows sorted by (level, index)
    void build_host(b2s_ctx* ctx, const std::vector<uint32_t>& lev)
    {
        n = (uint32_t)lev.size();
        uint32_t maxl = 0;
        for (uint32_t l : lev) maxl = std::max(maxl, l);
        nlev = n ? maxl + 1 : 0;
        h_ptr.assign((size_t)nlev + 1, 0);
        for (uint32_t l : lev) h_ptr[l + 1]++;
        for (uint32_t l = 0; l < nlev; ++l) h_ptr[l + 1] += h_ptr[l];
        std::vector<uint32_t> hrows(n ? n : 1), off(h_ptr.begin(), h_ptr.end() - 1);
        for (uint32_t i = 0; i < n; ++i) hrows[off[lev[i]]++] = i;
        level = upload(ctx, lev);
        rows = upload(ctx, hrows);
    }

    void build(b2s_ctx* ctx, uint32_t nrows, const uint32_t* rp, const uint32_t* ci, bool lower)
    {
        n = nrows;
        level.alloc(n ? n : 1);
        rows.alloc(n ? n : 1);
        if (!n)
        {
            nlev = 0;
            h_ptr.assign(1, 0);
            return;
        }
        SyncFree sf;
        sf.init(ctx, n);
        if (lower)
            sf.run(ctx, nullptr, false, LevelOp<true>{rp, ci, level.p}, nullptr);
        else
            sf.run(ctx, nullptr, true, LevelOp<false>{rp, ci, level.p}, nullptr);
        if (sf.status(ctx) != 0) fail(B2S_TIMEOUT, "level-set traversal timed out");
        // stable sort rows by level
        DBuf<uint32_t> iota(n), keys_out(n);
        B2S_LAUNCH(ctx, k_iota, stream_grid(ctx, n), kThreads, 0, iota.p, n);
        size_t bytes = 0;
        B2S_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, level.p, keys_out.p, iota.p, rows.p, (int)n, 0, 32,
                                                 ctx->stream));
        DBuf<uint8_t> tmp(bytes ? bytes : 1);
        B2S_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, bytes, level.p, keys_out.p, iota.p, rows.p, (int)n, 0, 32,
                                                 ctx->stream));
        ctx->launches += 1;
        uint32_t maxl = 0;
        d2h(ctx, &maxl, keys_out.p + (n - 1), sizeof(uint32_t));
        sync(ctx);
        nlev = maxl + 1;
        DBuf<uint32_t> lptr(nlev + 1);
        B2S_LAUNCH(ctx, k_level_bounds, stream_grid(ctx, n), kThreads, 0, keys_out.p, n, lptr.p);
        h_ptr.resize(nlev + 1);
        d2h(ctx, h_ptr.data(), lptr.p, (nlev + 1) * sizeof(uint32_t));
        sync(ctx);
    }
};

template <typename Op>
__global__ void __launch_bounds__(kThreads) k_trsv_level(const uint32_t* __restrict__ rows, uint32_t count, Op op,
                                                         const int* done)
{
    if (done && *done) return;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) op.template row_compute<false>(rows[t]);
}


// Runs op over every row of a schedule: B2S_TRSV_LEVEL launches one kernel
// per level (rows of a level are independent); otherwise one sync-free
// traversal in level-sorted order.
template <typename Op>
void run_schedule(b2s_ctx* ctx, int mode, const LevelSchedule& sched, SyncFree& sf, const Op& op, const int* done)
{
    if (mode == B2S_TRSV_LEVEL)
    {
        for (uint32_t l = 0; l < sched.nlev; ++l)
        {
            const uint32_t a = sched.h_ptr[l], cnt = sched.h_ptr[l + 1] - a;
            B2S_LAUNCH(ctx, k_trsv_level<Op>, (cnt + kThreads - 1) / kThreads, kThreads, 0, sched.rows.p + a, cnt, op,
                       done);
        }
    }
    else
        sf.run(ctx, sched.rows.p, false, op, done);
}

}  // namespace b2s
