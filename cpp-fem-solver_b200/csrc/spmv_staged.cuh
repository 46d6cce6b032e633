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

// ------------------------------------------------------------- warp path
//
// The default CSR SpMV.  A warp owns 32 consecutive rows (a "row group") and
// walks their nonzeros [rp[r0], rp[r0+32]) in chunks of 256: each lane loads
// eight values and column indices (coalesced, all in flight together, not
// allocated in L1 so that L1 keeps x),
// gathers x, and writes the products to the warp's 2 KB of shared memory;
// after a __syncwarp each lane adds the products of its own row in ascending
// column order.  A product v*x rounded once and then added is exactly the
// reference's `sum += v * x` without contraction, so y is bit-exact.  There
// is no CTA-wide barrier: warps progress independently and hide each other's
// gather latency.  Groups are dealt to warps grid-stride over a fixed grid,
// so the epilogue's reductions have a fixed order.

// read-once matrix data: read-only path, not kept in L1 (which then holds x)
__device__ __forceinline__ double ld_stream(const double* p)
{
    double v;
    asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ float ld_stream(const float* p)
{
    float v;
    asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ uint32_t ld_stream(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

// The SpMV's operand x_j.  XDirect reads a vector; other operands (the PCG
// direction p = z + beta p_old, formed where it is gathered) supply at(j).
struct XDirect
{
    const double* x;
    __device__ void init() {}
    __device__ double at(uint32_t j) const { return __ldg(&x[j]); }
};

constexpr int kSpmvWarpChunk = 256;                       // products per warp per pass
constexpr int kSpmvWarpPerLane = kSpmvWarpChunk / 32;     // loads per lane per pass
constexpr int kSpmvWarpCtasPerSm = 6;

// VT: stored value type (double; float for the FP32 copies of an AMG
// hierarchy's operators), products and sums in FP64 either way.
template <typename Epi, typename Xop = XDirect, typename VT = double>
__global__ void __launch_bounds__(kThreads, kSpmvWarpCtasPerSm)
    k_spmv_warp(uint32_t n, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                const VT* __restrict__ v, Xop x, const int* done, Epi epi, double* partial,
                unsigned int* counter)
{
    if (done && *done) return;
    x.init();
    __shared__ double prod[kThreads / 32][kSpmvWarpChunk];
    constexpr int NV = Epi::NV > 0 ? Epi::NV : 1;
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    double* P = prod[wid];
    const uint32_t ngroups = (n + 31u) >> 5;
    const uint32_t warps = gridDim.x * (kThreads / 32);
    for (uint32_t g = blockIdx.x * (kThreads / 32) + wid; g < ngroups; g += warps)
    {
        const uint32_t r0 = g << 5;
        const uint32_t r = r0 + lane;
        const uint32_t rows = min(32u, n - r0);
        const bool valid = lane < rows;
        const uint32_t a = valid ? __ldg(&rp[r]) : 0u;
        const uint32_t b = valid ? __ldg(&rp[r + 1]) : 0u;
        const uint32_t p0 = __shfl_sync(0xffffffffu, a, 0);
        const uint32_t p1 = __shfl_sync(0xffffffffu, b, rows - 1);
        double sum = 0.0;
        for (uint32_t base = p0; base < p1; base += kSpmvWarpChunk)
        {
            double vv[kSpmvWarpPerLane];
            uint32_t cc[kSpmvWarpPerLane];
#pragma unroll
            for (int k = 0; k < kSpmvWarpPerLane; ++k)
            {
                const uint32_t q = base + k * 32 + lane;
                vv[k] = 0.0;
                cc[k] = 0u;
                if (q < p1)
                {
                    vv[k] = (double)ld_stream(v + q);
                    cc[k] = ld_stream(ci + q);
                }
            }
#pragma unroll
            for (int k = 0; k < kSpmvWarpPerLane; ++k)
            {
                const uint32_t q = base + k * 32 + lane;
                if (q < p1) P[k * 32 + lane] = vv[k] * x.at(cc[k]);
            }
            __syncwarp();
            const uint32_t lo = a > base ? a : base;
            const uint32_t hi = b < base + kSpmvWarpChunk ? b : base + kSpmvWarpChunk;
            for (uint32_t q = lo; q < hi; ++q) sum += P[q - base];
            __syncwarp();
        }
        if (valid) epi.row(r, sum, acc);
    }
    if constexpr (Epi::NV > 0)
    {
        if (grid_reduce_last<Epi::NV>(acc, partial, counter))
            if (threadIdx.x == 0) epi.last(acc);
    }
}

// One thread per row, for matrices of short rows whose working set stays in
// L2 (n <= kSpmvRowMaxN, rows <= kSpmvRowMaxLen): every row's loads are
// independent and the whole grid is one wave, where the warp kernel above
// would run a second, mostly idle wave of 32-row groups.  The row is summed
// from 0 in column order, as in the warp kernel, so both give the same bits.
constexpr uint32_t kSpmvRowMaxLen = 32;
constexpr uint32_t kSpmvRowMaxN = 1u << 20;

template <typename Epi, typename Xop = XDirect>
__global__ void __launch_bounds__(kThreads) k_spmv_row(uint32_t n, const uint32_t* __restrict__ rp,
                                                       const uint32_t* __restrict__ ci, const double* __restrict__ v,
                                                       Xop x, const int* done, Epi epi, double* partial,
                                                       unsigned int* counter)
{
    if (done && *done) return;
    x.init();
    constexpr int NV = Epi::NV > 0 ? Epi::NV : 1;
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n)
    {
        const uint32_t a = __ldg(&rp[r]), b = __ldg(&rp[r + 1]);
        double sum = 0.0;
        for (uint32_t q0 = a; q0 < b; q0 += 8)
        {
            double vv[8], xx[8];
#pragma unroll
            for (int k = 0; k < 8; ++k)
            {
                const uint32_t q = q0 + k;
                vv[k] = q < b ? __ldg(&v[q]) : 0.0;
                xx[k] = q < b ? x.at(__ldg(&ci[q])) : 0.0;
            }
#pragma unroll
            for (int k = 0; k < 8; ++k)
                if (q0 + k < b) sum += vv[k] * xx[k];
        }
        epi.row(r, sum, acc);
    }
    if constexpr (Epi::NV > 0)
    {
        if (grid_reduce_last<Epi::NV>(acc, partial, counter))
            if (threadIdx.x == 0) epi.last(acc);
    }
}

inline unsigned spmv_warp_grid(const b2s_ctx* ctx, uint32_t n)
{
    const uint32_t ngroups = (n + 31u) / 32u;
    const uint32_t ctas = (ngroups + kThreads / 32 - 1) / (kThreads / 32);
    const unsigned g = (unsigned)ctx->sm_count * kSpmvWarpCtasPerSm;
    return ctas < g ? (ctas ? ctas : 1u) : g;
}

inline bool spmv_by_rows(const CsrDev& A)
{
    return A.n && A.max_row && A.max_row <= kSpmvRowMaxLen && A.n <= kSpmvRowMaxN;
}

// the SpMV's grid (reduction partials to reserve before a graph capture)
inline unsigned spmv_grid(const b2s_ctx* ctx, const CsrDev& A)
{
    return spmv_by_rows(A) ? (A.n + kThreads - 1) / kThreads : spmv_warp_grid(ctx, A.n);
}

template <typename Epi, typename Xop>
inline void launch_spmv_op(b2s_ctx* ctx, const CsrDev& A, const Xop& x, const int* done, const Epi& epi)
{
    if (spmv_by_rows(A))
    {
        const unsigned grid = (A.n + kThreads - 1) / kThreads;
        if (Epi::NV > 0) reserve_reduction(ctx, grid);
        B2S_LAUNCH(ctx, (k_spmv_row<Epi, Xop>), grid, kThreads, 0, A.n, A.rp.p, A.ci.p, A.v.p, x, done, epi,
                   ctx->partial.p, ctx->counter.p);
        return;
    }
    const unsigned grid = spmv_warp_grid(ctx, A.n);
    if (Epi::NV > 0) reserve_reduction(ctx, grid);
    B2S_LAUNCH(ctx, (k_spmv_warp<Epi, Xop>), grid, kThreads, 0, A.n, A.rp.p, A.ci.p, A.v.p, x, done, epi,
               ctx->partial.p, ctx->counter.p);
}

template <typename Epi>
inline void launch_spmv(b2s_ctx* ctx, const CsrDev& A, const double* x, const int* done, const Epi& epi)
{
    launch_spmv_op(ctx, A, XDirect{x}, done, epi);
}

}  // namespace b2s
