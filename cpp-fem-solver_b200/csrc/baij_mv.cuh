// Block matvec kernels (BlockMatrix::matvec, blockMatrix.hpp:208-234) with
// an epilogue, shared by the BAIJ operator (baij.cu) and the AMG V-cycle
// (amg.cu), whose residual and smoothing updates ride on the products.
//
// Block matvec (bs >= 2): a warp owns 32/bs consecutive block rows (one lane
// per output component) and walks their blocks min(32, 256/bs^2) at a time.  The
// lanes stream the blocks' values into the warp's shared memory (coalesced,
// no L1 allocation), lane b gathers x_J of block b and forms the block's bs
// row dots with the reference's association (blk_row_dot), and the lane of
// output component (I, r) adds the dots of row I in block order -- the
// reference's order, so y is bit-exact.  No CTA-wide barrier.
#pragma once
#include "block_ops.cuh"
#include "spmv_staged.cuh"

namespace b2s {

constexpr int kBaijCtasPerSm = 4;

// VT: stored value type (double, or float for the FP32 copies of the AMG
// hierarchy); products and sums are FP64 either way.
template <int BS, typename VT, class Epi>
__global__ void __launch_bounds__(kThreads, kBaijCtasPerSm)
    k_baij_warp(uint32_t nbr, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                const VT* __restrict__ v, const double* __restrict__ x, Epi epi, const int* done)
{
    if (done && *done) return;
    constexpr int BV = BS * BS;
    constexpr int GR = 32 / BS;                        // block rows per warp group
    constexpr int NB = 256 / BV < 32 ? 256 / BV : 32;  // blocks per pass: one lane per block
    constexpr int PER = (NB * BV + 31) / 32;           // value loads per lane per pass
    __shared__ double sval[kThreads / 32][NB * BV];
    __shared__ double sdot[kThreads / 32][NB * BS];
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    double* V = sval[wid];
    double* P = sdot[wid];
    // one pass's operands in registers: its values and this lane's block column
    auto load_pass = [&](uint32_t base, uint32_t nb, double* tv, uint32_t& J) {
        const VT* vb = v + (size_t)base * BV;
#pragma unroll
        for (int k = 0; k < PER; ++k)
        {
            const uint32_t q = k * 32 + lane;
            tv[k] = q < nb * BV ? (double)ld_stream(vb + q) : 0.0;
        }
        J = lane < nb ? ld_stream(ci + base + lane) : 0u;
    };
    const uint32_t ngroups = (nbr + GR - 1) / GR;
    for (uint32_t g = blockIdx.x * (kThreads / 32) + wid; g < ngroups; g += gridDim.x * (kThreads / 32))
    {
        const uint32_t I0 = g * GR;
        const uint32_t rows = min((uint32_t)GR, nbr - I0);
        const bool out = lane < rows * BS;
        const uint32_t I = I0 + lane / BS;
        const uint32_t r = lane % BS;
        const uint32_t a = out ? __ldg(&rp[I]) : 0u, b = out ? __ldg(&rp[I + 1]) : 0u;
        const uint32_t p0 = __shfl_sync(0xffffffffu, a, 0);
        const uint32_t p1 = __shfl_sync(0xffffffffu, b, (rows - 1) * BS);
        double acc = 0.0;
        double tv[PER];
        uint32_t J = 0;
        if (p0 < p1) load_pass(p0, min((uint32_t)NB, p1 - p0), tv, J);
        for (uint32_t base = p0; base < p1; base += NB)
        {
            const uint32_t nb = min((uint32_t)NB, p1 - base);
#pragma unroll
            for (int k = 0; k < PER; ++k)
            {
                const uint32_t q = k * 32 + lane;
                if (q < nb * BV) V[q] = tv[k];
            }
            double xv[BS];
            if (lane < nb)
#pragma unroll
                for (int c = 0; c < BS; ++c) xv[c] = __ldg(&x[(size_t)J * BS + c]);
            // the next pass's operands load while this pass computes
            const uint32_t nbase = base + NB;
            if (nbase < p1) load_pass(nbase, min((uint32_t)NB, p1 - nbase), tv, J);
            __syncwarp();
            if (lane < nb)
#pragma unroll
                for (int r2 = 0; r2 < BS; ++r2) P[lane * BS + r2] = blk_row_dot<BS>(&V[lane * BV + r2 * BS], xv);
            __syncwarp();
            if (out)
            {
                const uint32_t lo = a > base ? a : base, hi = b < base + nb ? b : base + nb;
                for (uint32_t k = lo; k < hi; ++k) acc += P[(k - base) * BS + r];
            }
            __syncwarp();
        }
        epi.template put<BS>(I, r, acc, out, lane);
    }
}




// y = A x with the stored values v (A's pattern), every output component
// handed to the epilogue: epi.put<BS>(I, r, y_Ir, valid, lane).  For BS >= 2
// all 32 lanes of a warp call put together (valid false on idle lanes), so an
// epilogue may exchange a block row's components with shuffles; the lanes of
// block row I are lanes (lane / BS) * BS .. + BS - 1.  For BS = 1 a thread
// calls put for its own rows only.
// 1x1 blocks with long rows (the coarse operators and restrictions of a
// scalar AMG hierarchy, 30 to 100+ entries a row): a CTA stages a contiguous
// range of entries (the partition in A.blk_row, at most kBaijStagedCap
// entries) in shared memory and one thread per row sums its row from it.
constexpr uint32_t kBaijStagedCap = 3072;
constexpr uint32_t kBaijStagedMinRow = 16;  // mean entries per row from which the staged kernel is used

__device__ __forceinline__ void stage_vals(double* s, const double* g, uint32_t cnt) { stage_f64(s, g, cnt); }

__device__ __forceinline__ void stage_vals(float* s, const float* g, uint32_t cnt)
{
    for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) s[i] = __ldg(&g[i]);
}

template <typename VT, class Epi>
__global__ void __launch_bounds__(kThreads) k_baij_staged1(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                                           const VT* __restrict__ v,
                                                           const uint32_t* __restrict__ blk_row,
                                                           const double* __restrict__ x, Epi epi, const int* done)
{
    if (done && *done) return;
    __shared__ VT sv[kBaijStagedCap];
    __shared__ uint32_t sc[kBaijStagedCap];
    const uint32_t r0 = blk_row[blockIdx.x], r1 = blk_row[blockIdx.x + 1];
    const uint32_t p0 = __ldg(&rp[r0]), p1 = __ldg(&rp[r1]);
    const uint32_t cnt = p1 - p0;
    if (cnt <= kBaijStagedCap)
    {
        stage_vals(sv, v + p0, cnt);
        stage_u32(sc, ci + p0, cnt);
        __syncthreads();
        for (uint32_t br = r0 + threadIdx.x; br < r1; br += blockDim.x)
        {
            const uint32_t a = __ldg(&rp[br]) - p0, b = __ldg(&rp[br + 1]) - p0;
            double yr = 0.0;
            for (uint32_t k = a; k < b; ++k) yr += (double)sv[k] * __ldg(&x[sc[k]]);
            epi.template put<1>(br, 0, yr, true, 0u);
        }
    }
    else
        for (uint32_t br = r0 + threadIdx.x; br < r1; br += blockDim.x)
        {
            double yr = 0.0;
            for (uint32_t k = __ldg(&rp[br]); k < __ldg(&rp[br + 1]); ++k)
                yr += (double)__ldg(&v[k]) * __ldg(&x[__ldg(&ci[k])]);
            epi.template put<1>(br, 0, yr, true, 0u);
        }
}

// 1x1 blocks with short rows (the fine operator and the prolongation) use
// the CSR SpMV's warp kernel.  Both sum a row from 0 in column order, which
// is blk_row_dot<1>'s order, so every kernel gives the same bits.
template <class Epi>
struct EpiRowsOf
{
    static constexpr int NV = 0;
    Epi e;
    __device__ __forceinline__ void row(uint32_t r, double s, double*) const { e.template put<1>(r, 0, s, true, 0u); }
    __device__ __forceinline__ void last(const double*) const {}
};

template <int BS, typename VT, class Epi>
void baij_mv(b2s_ctx* ctx, const BaijDev& A, const VT* v, const double* x, Epi epi, const int* done)
{
    if (A.nbr == 0) return;
    if constexpr (BS == 1)
    {
        if (A.nblk)
            B2S_LAUNCH(ctx, (k_baij_staged1<VT, Epi>), A.nblk, kThreads, 0, A.rp.p, A.ci.p, v, A.blk_row.p, x, epi,
                       done);
        else
            B2S_LAUNCH(ctx, (k_spmv_warp<EpiRowsOf<Epi>, XDirect, VT>), spmv_warp_grid(ctx, A.nbr), kThreads, 0,
                       A.nbr, A.rp.p, A.ci.p, v, XDirect{x}, done, EpiRowsOf<Epi>{epi}, (double*)nullptr,
                       (unsigned int*)nullptr);
    }
    else
    {
        constexpr int GR = 32 / BS;
        const uint32_t groups = (A.nbr + GR - 1) / GR;
        const uint32_t ctas = (groups + kThreads / 32 - 1) / (kThreads / 32);
        const uint32_t cap = (uint32_t)ctx->sm_count * kBaijCtasPerSm;
        B2S_LAUNCH(ctx, (k_baij_warp<BS, VT, Epi>), ctas < cap ? ctas : cap, kThreads, 0, A.nbr, A.rp.p, A.ci.p, v,
                   x, epi, done);
    }
}

// the plain product: y[I * BS + r] = (A x)_Ir
struct EpiStoreY
{
    double* y;
    template <int BS>
    __device__ __forceinline__ void put(uint32_t I, int r, double v, bool valid, uint32_t) const
    {
        if (valid) y[(size_t)I * BS + r] = v;
    }
};

}  // namespace b2s
