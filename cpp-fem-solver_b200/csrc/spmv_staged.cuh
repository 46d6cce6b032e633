// Staged CSR SpMV kernel template.
//
// One CTA owns a contiguous range of rows [blk_row[b], blk_row[b+1]) whose
// nonzeros [rp[r0], rp[r1]) are copied HBM -> shared memory with 16-byte
// vector loads (fully coalesced, each byte read once), then each thread
// forms one row's sum from shared memory in ascending column order -- the
// reference's SMatrix::spmv order (array.cpp:3418-3442), so y is bit-exact.
// x is gathered through the read-only path; for the stencil matrices here it
// stays L2-resident (x is at most 17 MB on the 128^3 grid, L2 is 126 MB).
//
// Rows whose nonzeros exceed the staging capacity get a CTA of their own and
// are summed by one thread directly from global memory (same order, slower);
// the benchmark matrices never produce such rows.
//
// An epilogue functor (Epi) sees every row's sum, writes the output and may
// accumulate NV values that are reduced grid-wide in fixed order; its last()
// runs once, on thread 0 of the last CTA, with the totals.
#pragma once
#include "b2s_internal.cuh"

namespace b2s {

__device__ __forceinline__ void stage_f64(double* s, const double* g, uint32_t cnt)
{
    uint32_t head = (((uintptr_t)g) & 15u) ? 1u : 0u;
    if (head > cnt) head = cnt;
    if (threadIdx.x == 0 && head) s[0] = __ldg(g);
    const uint32_t body = cnt - head, n2 = body >> 1;
    const double2* g2 = reinterpret_cast<const double2*>(g + head);
    for (uint32_t i = threadIdx.x; i < n2; i += blockDim.x)
    {
        const double2 t = __ldg(&g2[i]);
        s[head + 2 * i] = t.x;
        s[head + 2 * i + 1] = t.y;
    }
    if ((body & 1u) && threadIdx.x == 0) s[cnt - 1] = __ldg(&g[cnt - 1]);
}

__device__ __forceinline__ void stage_u32(uint32_t* s, const uint32_t* g, uint32_t cnt)
{
    uint32_t head = (uint32_t)(((16u - (((uintptr_t)g) & 15u)) & 15u) >> 2);
    if (head > cnt) head = cnt;
    if (threadIdx.x < head) s[threadIdx.x] = __ldg(&g[threadIdx.x]);
    const uint32_t body = cnt - head, n4 = body >> 2;
    const uint4* g4 = reinterpret_cast<const uint4*>(g + head);
    for (uint32_t i = threadIdx.x; i < n4; i += blockDim.x)
    {
        const uint4 t = __ldg(&g4[i]);
        s[head + 4 * i] = t.x;
        s[head + 4 * i + 1] = t.y;
        s[head + 4 * i + 2] = t.z;
        s[head + 4 * i + 3] = t.w;
    }
    const uint32_t tail = body & 3u;
    if (threadIdx.x < tail) s[cnt - tail + threadIdx.x] = __ldg(&g[cnt - tail + threadIdx.x]);
}

struct EpiStore
{
    static constexpr int NV = 0;
    double* y;
    __device__ void row(uint32_t r, double s, double*) const { y[r] = s; }
    __device__ void last(const double*) const {}
};

template <typename Epi>
__global__ void __launch_bounds__(kThreads) k_spmv_staged(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                                          const double* __restrict__ v,
                                                          const uint32_t* __restrict__ blk_row,
                                                          const double* __restrict__ x, const int* done, Epi epi,
                                                          double* partial, unsigned int* counter)
{
    if (done && *done) return;
    __shared__ double sv[kSpmvNnzPerCta];
    __shared__ uint32_t sc[kSpmvNnzPerCta];
    constexpr int NV = Epi::NV > 0 ? Epi::NV : 1;
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;

    const uint32_t r0 = blk_row[blockIdx.x], r1 = blk_row[blockIdx.x + 1];
    const uint32_t p0 = __ldg(&rp[r0]), p1 = __ldg(&rp[r1]);
    const uint32_t cnt = p1 - p0;
    if (cnt <= (uint32_t)kSpmvNnzPerCta)
    {
        stage_f64(sv, v + p0, cnt);
        stage_u32(sc, ci + p0, cnt);
        __syncthreads();
        for (uint32_t r = r0 + threadIdx.x; r < r1; r += blockDim.x)
        {
            const uint32_t a = __ldg(&rp[r]) - p0, b = __ldg(&rp[r + 1]) - p0;
            double sum = 0.0;
            for (uint32_t k = a; k < b; ++k) sum += sv[k] * __ldg(&x[sc[k]]);
            epi.row(r, sum, acc);
        }
    }
    else if (threadIdx.x == 0)
    {
        // one long row per CTA (partition guarantees it): sequential, same order
        for (uint32_t r = r0; r < r1; ++r)
        {
            double sum = 0.0;
            for (uint32_t k = __ldg(&rp[r]); k < __ldg(&rp[r + 1]); ++k) sum += __ldg(&v[k]) * __ldg(&x[__ldg(&ci[k])]);
            epi.row(r, sum, acc);
        }
    }
    if constexpr (Epi::NV > 0)
    {
        if (grid_reduce_last<Epi::NV>(acc, partial, counter))
            if (threadIdx.x == 0) epi.last(acc);
    }
}

// ------------------------------------------------------------------ TMA path
//
// Persistent, double-buffered form of the same computation.  Each CTA walks
// row blocks b, b + grid, ...; thread 0 issues 1-D bulk copies
// (cp.async.bulk) of block b+grid's values and column indices into the idle
// stage while the CTA sums block b out of the other stage, so HBM streams
// continuously.  Copies start on 16-byte boundaries: the value range is
// widened to even indices and the index range to multiples of four (the
// arrays carry 8 elements of padding), and the sums index from the widened
// start.  Waits on the stage barriers are bounded; on a timeout the CTA
// records B2S_TIMEOUT, waits (bounded) for its own copies and returns.

constexpr int kTmaStageVals = kSpmvNnzPerCta + 2;  // doubles per stage
constexpr int kTmaStageCols = kSpmvNnzPerCta + 8;  // uint32 per stage (range widened by up to 3 + 3)
constexpr size_t kTmaStageBytes = (size_t)kTmaStageVals * 8 + (size_t)kTmaStageCols * 4;
constexpr unsigned kTmaWaitSpins = 1u << 24;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    for (unsigned s = 0; s < kTmaWaitSpins; ++s)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// issue the copies of row block b into stage buffers (thread 0 only)
__device__ __forceinline__ void spmv_issue(uint32_t b, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                           const double* __restrict__ v, const uint32_t* __restrict__ blk_row,
                                           double* sv, uint32_t* sc, uint64_t* bar)
{
    const uint32_t r0 = blk_row[b], r1 = blk_row[b + 1];
    const uint32_t p0 = rp[r0], p1 = rp[r1];
    uint32_t bytes = 0;
    if (p1 - p0 <= (uint32_t)kSpmvNnzPerCta && p1 > p0)
    {
        const uint32_t a0 = p0 & ~1u, a1 = (p1 + 1u) & ~1u;
        const uint32_t c0 = p0 & ~3u, c1 = (p1 + 3u) & ~3u;
        bytes = (a1 - a0) * 8u + (c1 - c0) * 4u;
        mbar_arrive_expect_tx(bar, bytes);
        bulk_load(sv, v + a0, (a1 - a0) * 8u, bar);
        bulk_load(sc, ci + c0, (c1 - c0) * 4u, bar);
    }
    else
        mbar_arrive_expect_tx(bar, 0u);
}

template <typename Epi>
__global__ void __launch_bounds__(kThreads) k_spmv_tma(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                                       const double* __restrict__ v,
                                                       const uint32_t* __restrict__ blk_row, uint32_t nblk,
                                                       const double* __restrict__ x, const int* done, Epi epi,
                                                       double* partial, unsigned int* counter, int* err)
{
    if (done && *done) return;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar[2];
    double* sv[2] = {reinterpret_cast<double*>(smem), reinterpret_cast<double*>(smem + kTmaStageBytes)};
    uint32_t* sc[2] = {reinterpret_cast<uint32_t*>(smem + (size_t)kTmaStageVals * 8),
                       reinterpret_cast<uint32_t*>(smem + kTmaStageBytes + (size_t)kTmaStageVals * 8)};
    constexpr int NV = Epi::NV > 0 ? Epi::NV : 1;
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;

    if (threadIdx.x == 0)
    {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_proxy_async();
    }
    __syncthreads();
    uint32_t phase[2] = {0u, 0u};
    int stage = 0;
    bool ok = true;
    if (threadIdx.x == 0 && blockIdx.x < nblk) spmv_issue(blockIdx.x, rp, ci, v, blk_row, sv[0], sc[0], &bar[0]);
    for (uint32_t b = blockIdx.x; b < nblk; b += gridDim.x)
    {
        const uint32_t nb = b + gridDim.x;
        if (threadIdx.x == 0 && nb < nblk)
        {
            fence_proxy_async();
            spmv_issue(nb, rp, ci, v, blk_row, sv[stage ^ 1], sc[stage ^ 1], &bar[stage ^ 1]);
        }
        if (!mbar_wait(&bar[stage], phase[stage]))
        {
            ok = false;
            break;
        }
        phase[stage] ^= 1u;
        const uint32_t r0 = blk_row[b], r1 = blk_row[b + 1];
        const uint32_t p0 = __ldg(&rp[r0]), p1 = __ldg(&rp[r1]);
        if (p1 - p0 <= (uint32_t)kSpmvNnzPerCta)
        {
            // staged copies start at the widened offsets a0 = p0 & ~1, c0 = p0 & ~3
            const double* V = sv[stage];
            const uint32_t* Cc = sc[stage];
            const uint32_t a0 = p0 & ~1u, c0 = p0 & ~3u;
            for (uint32_t r = r0 + threadIdx.x; r < r1; r += blockDim.x)
            {
                const uint32_t a = __ldg(&rp[r]), e = __ldg(&rp[r + 1]);
                double sum = 0.0;
                for (uint32_t k = a; k < e; ++k) sum += V[k - a0] * __ldg(&x[Cc[k - c0]]);
                epi.row(r, sum, acc);
            }
        }
        else if (threadIdx.x == 0)
        {
            for (uint32_t r = r0; r < r1; ++r)
            {
                double sum = 0.0;
                for (uint32_t k = __ldg(&rp[r]); k < __ldg(&rp[r + 1]); ++k) sum += __ldg(&v[k]) * __ldg(&x[__ldg(&ci[k])]);
                epi.row(r, sum, acc);
            }
        }
        __syncthreads();
        stage ^= 1;
    }
    if (!ok)
    {
        // record, then wait (bounded) for this CTA's copies still in flight
        if (threadIdx.x == 0) atomicExch(err, (int)B2S_TIMEOUT);
        mbar_wait(&bar[0], phase[0]);
        mbar_wait(&bar[1], phase[1]);
        __syncthreads();
    }
    if constexpr (Epi::NV > 0)
    {
        if (grid_reduce_last<Epi::NV>(acc, partial, counter))
            if (threadIdx.x == 0) epi.last(acc);
    }
}

inline unsigned spmv_tma_grid(const b2s_ctx* ctx, uint32_t nblk)
{
    const unsigned g = (unsigned)ctx->sm_count * 2u;
    return nblk < g ? (nblk ? nblk : 1u) : g;
}

template <typename Epi>
inline void launch_spmv(b2s_ctx* ctx, const CsrDev& A, const double* x, const int* done, const Epi& epi)
{
    const unsigned grid = spmv_tma_grid(ctx, A.nblk);
    if (Epi::NV > 0) reserve_reduction(ctx, grid);
    auto kern = k_spmv_tma<Epi>;
    const size_t smem = 2 * kTmaStageBytes;
    static bool configured = false;
    if (!configured)
    {
        B2S_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured = true;
    }
    B2S_LAUNCH(ctx, kern, grid, kThreads, smem, A.rp.p, A.ci.p, A.v.p, A.blk_row.p, A.nblk, x, done, epi,
               ctx->partial.p, ctx->counter.p, ctx->errword());
}

}  // namespace b2s
