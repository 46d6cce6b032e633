// Chunked triangular solve: the default schedule of the IC(0) / ILU(0)
// solves (B2S_TRSV_CHUNK).
//
// The rows, in dependency order (natural order for a lower factor, reversed
// for an upper one), are cut into contiguous chunks that fit one CTA's shared
// memory: the chunk's slice of the factor (values, column indices, row
// offsets), its right-hand side and divisors are copied in with coalesced
// loads when the CTA starts, and the chunk's solution stays in shared memory.
// Inside a chunk the rows are ordered by their local level (the longest chain
// of dependencies inside the chunk); the CTA walks the local levels with one
// __syncthreads() between them, so a dependency inside the chunk costs a
// shared-memory read.  A dependency on an earlier chunk waits on that row's
// ready flag (bounded, B2S_TIMEOUT) and reads the value from L2.  CTAs take
// chunks from a ticket in order, so they only wait on chunks held by CTAs
// that started earlier.
//
// Every row is still summed in its column order with the reference's
// arithmetic, so the result equals the level / sync-free schedules bit for
// bit.  On a 2-D 5-point factor the 1023-level critical path then costs one
// barrier per level instead of one L2 round trip per level, except at chunk
// boundaries.
#pragma once
#include "syncfree.cuh"

namespace b2s {

constexpr int kChunkThreads = 256;
constexpr uint32_t kChunkSmemBudget = 200 * 1024;

struct ChunkArgs
{
    const uint32_t* row_lo;     // per chunk (nchunks + 1), in processing order
    const uint32_t* chunk_lvl;  // per chunk, offsets into lvl_ptr (nchunks + 1)
    const uint32_t* lvl_ptr;    // level boundaries into sorted
    const uint32_t* sorted;     // rows of every chunk, by (local level, row)
    const uint8_t* ext;         // 1 when a row of another chunk depends on the row
    uint32_t nchunks;
    uint32_t max_rows, max_nnz;
    int lower;
    SyncFreeCtl ctl;
};

// shared-memory layout for element types XT (solution), RT (rhs), VT (values)
template <typename VT, typename XT, typename RT, bool UNIT>
struct ChunkSmem
{
    static size_t bytes(uint32_t rows, uint32_t nnz)
    {
        size_t b = 0;
        b += ((size_t)rows * sizeof(XT) + 15) & ~size_t(15);
        b += ((size_t)rows * sizeof(RT) + 15) & ~size_t(15);
        if (!UNIT) b += ((size_t)rows * sizeof(VT) + 15) & ~size_t(15);
        b += ((size_t)(rows + 1) * 4 + 15) & ~size_t(15);
        b += ((size_t)nnz * sizeof(VT) + 15) & ~size_t(15);
        b += ((size_t)nnz * 4 + 15) & ~size_t(15);
        return b;
    }
};

template <bool LOWER, bool UNIT, typename VT, typename XT, typename RT>
__global__ void __launch_bounds__(kChunkThreads) k_trsv_chunk(ChunkArgs a, const uint32_t* __restrict__ rp,
                                                              const uint32_t* __restrict__ ci, const VT* __restrict__ v,
                                                              const VT* __restrict__ d, const RT* __restrict__ rhs,
                                                              XT* __restrict__ x, double* __restrict__ out64,
                                                              const int* done)
{
    if (done && *done) return;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t s_chunk;
    if (threadIdx.x == 0) s_chunk = atomicAdd(&a.ctl.ticket[0], 1u);
    __syncthreads();
    const uint32_t c = s_chunk;
    const uint32_t epoch = ld_flag(a.ctl.epoch);
    const uint32_t rlo = a.row_lo[c], rhi = a.row_lo[c + 1];
    const uint32_t lo = LOWER ? rlo : rhi, hi = LOWER ? rhi : rlo;  // row range [lo, hi)
    const uint32_t nr = hi - lo;
    const uint32_t p0 = __ldg(&rp[lo]), nz = __ldg(&rp[hi]) - p0;

    unsigned char* ptr = smem;
    auto carve = [&](size_t bytes) {
        unsigned char* r = ptr;
        ptr += (bytes + 15) & ~size_t(15);
        return r;
    };
    XT* sx = reinterpret_cast<XT*>(carve((size_t)a.max_rows * sizeof(XT)));
    RT* sr = reinterpret_cast<RT*>(carve((size_t)a.max_rows * sizeof(RT)));
    VT* sd = UNIT ? nullptr : reinterpret_cast<VT*>(carve((size_t)a.max_rows * sizeof(VT)));
    uint32_t* srp = reinterpret_cast<uint32_t*>(carve((size_t)(a.max_rows + 1) * 4));
    VT* sv = reinterpret_cast<VT*>(carve((size_t)a.max_nnz * sizeof(VT)));
    uint32_t* sc = reinterpret_cast<uint32_t*>(carve((size_t)a.max_nnz * 4));

    for (uint32_t k = threadIdx.x; k < nr; k += blockDim.x)
    {
        sr[k] = rhs[lo + k];
        if (!UNIT) sd[k] = __ldg(&d[lo + k]);
        srp[k] = __ldg(&rp[lo + k]) - p0;
    }
    if (threadIdx.x == 0) srp[nr] = nz;
    for (uint32_t q = threadIdx.x; q < nz; q += blockDim.x)
    {
        sv[q] = __ldg(&v[p0 + q]);
        sc[q] = __ldg(&ci[p0 + q]);
    }
    __syncthreads();

    const uint32_t l0 = a.chunk_lvl[c], l1 = a.chunk_lvl[c + 1];
    for (uint32_t l = l0; l < l1; ++l)
    {
        const uint32_t t1 = a.lvl_ptr[l + 1];
        for (uint32_t t = a.lvl_ptr[l] + threadIdx.x; t < t1; t += blockDim.x)
        {
            const uint32_t row = __ldg(&a.sorted[t]);
            const uint32_t k = row - lo;
            XT sum = (XT)sr[k];
            for (uint32_t q = srp[k]; q < srp[k + 1]; ++q)
            {
                const uint32_t j = sc[q];
                if (LOWER ? (j < row) : (j > row))
                {
                    XT xj;
                    if (j >= lo && j < hi)
                        xj = sx[j - lo];
                    else
                    {
                        unsigned spins = 0, backoff = 20;
                        while (ld_flag(&a.ctl.flags[j]) != epoch)
                        {
                            if (++spins > kMaxSpins)
                            {
                                atomicExch(a.ctl.err, (int)B2S_TIMEOUT);
                                break;
                            }
                            __nanosleep(backoff);
                            backoff = backoff < 320 ? backoff * 2 : 320;
                        }
                        xj = __ldcg(&x[j]);
                    }
                    sum -= (XT)sv[q] * xj;
                }
            }
            const XT r = UNIT ? sum : sum / (XT)sd[k];
            sx[k] = r;
            x[row] = r;
            if (out64) out64[row] = (double)r;
            if (a.ext[row])
            {
                __threadfence();
                st_flag_release(&a.ctl.flags[row], epoch);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        __threadfence();
        const uint32_t left = atomicAdd(&a.ctl.ticket[1], 1u);
        if (left == gridDim.x - 1)
        {
            a.ctl.ticket[0] = 0u;
            a.ctl.ticket[1] = 0u;
            __threadfence();
        }
    }
}

// Host-built chunk schedule of one triangle.
struct ChunkSchedule
{
    uint32_t n = 0, nchunks = 0, max_rows = 0, max_nnz = 0;
    bool lower = true;
    DBuf<uint32_t> row_lo, chunk_lvl, lvl_ptr, sorted;
    DBuf<uint8_t> ext;
    SyncFree sf;  // ticket / epoch / error words and per-row flags

    // pattern on the host; deps are j < i (lower) or j > i (upper)
    void build(b2s_ctx* ctx, uint32_t nrows, const std::vector<uint32_t>& h_rp, const std::vector<uint32_t>& h_ci,
               bool lo, bool unit)
    {
        n = nrows;
        lower = lo;
        std::vector<uint32_t> hrow_lo{lo ? 0u : n}, hchunk_lvl{0}, hlvl_ptr{0}, hsorted;
        hsorted.reserve(n);
        // bytes a row costs in shared memory (FP64 upper bound)
        auto row_bytes = [&](uint32_t r) { return (uint64_t)(8 + 8 + (unit ? 0 : 8) + 4) + 12ull * (h_rp[r + 1] - h_rp[r]); };
        std::vector<uint32_t> llev(n, 0), cnt;
        uint32_t pos = 0;
        while (pos < n)
        {
            // grow the chunk while it fits
            uint64_t bytes = 64;
            uint32_t end = pos;
            while (end < n)
            {
                const uint32_t r = lo ? end : n - 1 - end;
                const uint64_t b = row_bytes(r);
                if (end > pos && bytes + b > kChunkSmemBudget) break;
                bytes += b;
                ++end;
            }
            const uint32_t rlo = lo ? pos : n - end, rhi = lo ? end : n - pos;  // rows [rlo, rhi)
            // local levels in dependency order
            uint32_t maxl = 0, nnz = 0;
            for (uint32_t t = pos; t < end; ++t)
            {
                const uint32_t r = lo ? t : n - 1 - t;
                uint32_t l = 0;
                for (uint32_t p = h_rp[r]; p < h_rp[r + 1]; ++p)
                {
                    const uint32_t j = h_ci[p];
                    const bool dep = lo ? j < r : j > r;
                    if (dep && j >= rlo && j < rhi) l = std::max(l, llev[j] + 1);
                }
                llev[r] = l;
                maxl = std::max(maxl, l);
                nnz += h_rp[r + 1] - h_rp[r];
            }
            // counting sort by (level, row)
            cnt.assign(maxl + 2, 0);
            for (uint32_t r = rlo; r < rhi; ++r) cnt[llev[r] + 1]++;
            for (uint32_t l = 0; l <= maxl; ++l) cnt[l + 1] += cnt[l];
            const size_t base = hsorted.size();
            hsorted.resize(base + (rhi - rlo));
            std::vector<uint32_t> off(cnt.begin(), cnt.end() - 1);
            for (uint32_t r = rlo; r < rhi; ++r) hsorted[base + off[llev[r]]++] = r;
            for (uint32_t l = 0; l <= maxl; ++l) hlvl_ptr.push_back((uint32_t)(base + cnt[l + 1]));
            hchunk_lvl.push_back((uint32_t)hlvl_ptr.size() - 1);
            hrow_lo.push_back(lo ? end : n - end);
            max_rows = std::max(max_rows, rhi - rlo);
            max_nnz = std::max(max_nnz, nnz);
            pos = end;
        }
        nchunks = (uint32_t)hrow_lo.size() - 1;
        // rows read by a row of another chunk publish a ready flag
        std::vector<uint32_t> chunk_of(n);
        for (uint32_t c = 0; c < nchunks; ++c)
        {
            const uint32_t a = std::min(hrow_lo[c], hrow_lo[c + 1]), b = std::max(hrow_lo[c], hrow_lo[c + 1]);
            for (uint32_t r = a; r < b; ++r) chunk_of[r] = c;
        }
        std::vector<uint8_t> hext(n ? n : 1, 0);
        for (uint32_t r = 0; r < n; ++r)
            for (uint32_t p = h_rp[r]; p < h_rp[r + 1]; ++p)
            {
                const uint32_t j = h_ci[p];
                if ((lo ? j < r : j > r) && chunk_of[j] != chunk_of[r]) hext[j] = 1;
            }
        ext = upload(ctx, hext.data(), hext.size());
        row_lo = upload(ctx, hrow_lo.data(), hrow_lo.size());
        chunk_lvl = upload(ctx, hchunk_lvl.data(), hchunk_lvl.size());
        lvl_ptr = upload(ctx, hlvl_ptr.data(), hlvl_ptr.size());
        sorted = upload(ctx, hsorted.data(), hsorted.size() ? hsorted.size() : 1);
        sf.init(ctx, n);
    }

    ChunkArgs args() const
    {
        return ChunkArgs{row_lo.p, chunk_lvl.p, lvl_ptr.p, sorted.p, ext.p, nchunks, max_rows, max_nnz, lower ? 1 : 0,
                         sf.ctl()};
    }

    // shared memory a launch needs; 0 when the chunks do not fit one CTA
    template <typename VT, typename XT, typename RT, bool UNIT>
    size_t smem_bytes() const
    {
        const size_t b = ChunkSmem<VT, XT, RT, UNIT>::bytes(max_rows, max_nnz);
        return b <= 227 * 1024 ? b : 0;
    }

    template <bool LOWER, bool UNIT, typename VT, typename XT, typename RT>
    void run(b2s_ctx* ctx, const uint32_t* rp, const uint32_t* ci, const VT* v, const VT* d, const RT* rhs, XT* x,
             double* out64, const int* done)
    {
        if (!n) return;
        auto kern = k_trsv_chunk<LOWER, UNIT, VT, XT, RT>;
        const size_t smem = ChunkSmem<VT, XT, RT, UNIT>::bytes(max_rows, max_nnz);
        static thread_local size_t configured = 0;
        if (smem > configured)
        {
            B2S_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            configured = smem;
        }
        B2S_LAUNCH(ctx, k_epoch_bump, 1, 1, 0, sf.words.p + 2, done);
        B2S_LAUNCH(ctx, kern, nchunks, kChunkThreads, smem, args(), rp, ci, v, d, rhs, x, out64, done);
    }
};

}  // namespace b2s
