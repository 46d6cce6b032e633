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

template <typename Epi>
inline void launch_spmv(b2s_ctx* ctx, const CsrDev& A, const double* x, const int* done, const Epi& epi)
{
    if (Epi::NV > 0) reserve_reduction(ctx, A.nblk);
    B2S_LAUNCH(ctx, k_spmv_staged<Epi>, A.nblk, kThreads, 0, A.rp.p, A.ci.p, A.v.p, A.blk_row.p, x, done, epi,
               ctx->partial.p, ctx->counter.p);
}

}  // namespace b2s
