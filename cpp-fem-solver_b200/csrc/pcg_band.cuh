// The whole PCG iteration in one persistent kernel, for an IC(0)-type
// preconditioner whose two FP32 triangles are applied by banded Jacobi sweeps
// (trsv_band.cuh, segments of one row, two strict entries per row).
//
// A cooperative launch of one CTA per band tile (all resident).  Each
// iteration is three phases separated by grid barriers:
//   1. p = z + beta p_old formed where it is gathered; Ap = A p and p.Ap for
//      the tile's rows (the CSR rows in column order);
//   2. the forward sweeps of the tile (its halo recomputed), with the
//      right-hand side r = r_old - alpha Ap formed as it is staged; the owned
//      rows store y, r and x += alpha p and reduce r.r;
//   3. the backward sweeps on y; the owned rows store z and reduce r.z.
// After each barrier every CTA sums the per-tile partials in tile order and
// applies the same scalar step (alpha; the convergence / NaN test; beta) to
// its own copy of the Krylov state, so all CTAs take the same decisions with
// no broadcast; CTA 0 writes the state back at the end.  Values written by
// other CTAs are read with L1-bypassing loads.  The barriers are bounded:
// after kGridBarrierPolls polls a CTA records B2S_TIMEOUT and leaves, and the
// others then give up at their next barrier, so the launch always ends.
#pragma once

#include "trsv_band.cuh"

namespace b2s {

constexpr double kPcgBreak = 1e-30;
constexpr unsigned kGridBarrierPolls = 1u << 24;
constexpr uint32_t kPcgBandThreads = 768;  // band_threads(2)

// p.Ap: the breakdown / NOT_SPD stops and alpha (array.cpp:3540-3557)
__device__ __forceinline__ void pcg_alpha(KState* st, double pAp)
{
    st->pAp = pAp;
    if (fabs(pAp) < kPcgBreak)
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

__device__ __forceinline__ unsigned ld_acquire_gpu_u32(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void red_release_gpu_add(unsigned* p, unsigned v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// All CTAs of the (cooperative) grid arrive; false after a timeout.  The
// block barrier orders the CTA's writes before thread 0's release add, and
// the acquire load that sees every arrival orders the other CTAs' writes
// before the block barrier that releases this CTA (release / acquire at gpu
// scope, cumulative through the block barriers; no separate fences).
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned target, int* err, int* s_ok)
{
    __syncthreads();
    if (threadIdx.x == 0)
    {
        red_release_gpu_add(bar, 1u);
        int ok = 1;
        for (unsigned polls = 0; ld_acquire_gpu_u32(bar) < target; ++polls)
            if (polls >= kGridBarrierPolls)
            {
                atomicExch(err, (int)B2S_TIMEOUT);
                ok = 0;
                break;
            }
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

struct PcgBandArgs
{
    uint32_t n, T, B, Rmax;
    int k;
    const uint32_t *Arp, *Aci;
    const double* Av;
    const uint16_t *loff, *uoff;  // band_off of L and of L^T
    const float *lval, *uval, *ldinv, *udinv;
    double* x;
    double* r[2];
    double* p[2];
    double *z, *Ap, *red;  // red: 3 x gridDim.x partials
    float* y32;
    KState* st;
    unsigned* bar;  // zero at launch
    int* err;
    int stall_window;  // > 0: stop when the residual has not halved for this many iterations
};

// Pass 0 and k Jacobi sweeps of the tile's extended range (two strict entries
// per row, rows in registers); returns the buffer holding pass k.  rhs(i)
// gives the FP32 right-hand side of global row i.
template <bool LOWER, typename Rhs>
__device__ __forceinline__ const float* band_jacobi(const PcgBandArgs& a, const uint16_t* __restrict__ eoff,
                                                    const float* __restrict__ eval, const float* __restrict__ dinv,
                                                    uint32_t lo, uint32_t hi, float* y0, float* y1, Rhs rhs,
                                                    uint32_t& elo_out)
{
    constexpr uint32_t NT = kPcgBandThreads, Q = kBandRowsPerThread;
    const uint32_t n = a.n, halo = (uint32_t)a.k * a.B;
    const uint32_t elo = LOWER ? (lo > halo ? lo - halo : 0u) : lo;
    const uint32_t ehi = LOWER ? hi : (uint32_t)min((uint64_t)n, (uint64_t)hi + halo);
    const uint32_t R = ehi - elo;
    const bool cut = LOWER ? elo > 0 : ehi < n;
    uint32_t off[Q][2];
    float val[Q][2], rr[Q], di[Q];
#pragma unroll
    for (uint32_t q = 0; q < Q; ++q)
    {
        const uint32_t t = threadIdx.x + NT * q;
        const bool in = t < R;
        const uint32_t i = elo + (in ? t : 0u);
#pragma unroll
        for (int e = 0; e < 2; ++e)
        {
            off[q][e] = in ? (uint32_t)__ldg(&eoff[(size_t)e * n + i]) : 0u;
            val[q][e] = in ? __ldg(&eval[(size_t)e * n + i]) : 0.f;
        }
        rr[q] = in ? rhs(i) : 0.f;
        di[q] = in ? __ldg(&dinv[i]) : 0.f;
    }
    for (int s = 0; s <= a.k; ++s)
    {
        const float* yin = (s & 1) ? y0 : y1;
        float* yout = (s & 1) ? y1 : y0;
        const uint32_t shrink = (cut && s > 0) ? (uint32_t)s * a.B : 0u;
        const uint32_t t0 = LOWER ? shrink : 0u;
        const uint32_t t1 = LOWER ? R : (R > shrink ? R - shrink : 0u);
#pragma unroll
        for (uint32_t q = 0; q < Q; ++q)
        {
            const uint32_t t = threadIdx.x + NT * q;
            if (t >= t0 && t < t1)
            {
                float sum = rr[q];
                if (s > 0)
                {
#pragma unroll
                    for (int e = 0; e < 2; ++e)
                        if (off[q][e]) sum -= val[q][e] * yin[LOWER ? t - off[q][e] : t + off[q][e]];
                }
                yout[t] = sum * di[q];
            }
        }
        __syncthreads();
    }
    elo_out = elo;
    return (a.k & 1) ? y1 : y0;
}

// sum of the per-tile partials in a fixed order (every CTA gets the same
// bits): warp 0, each lane a strided slice in tile order, then a shuffle tree;
// the result lands in *out (shared), read after the block barrier
__device__ __forceinline__ void sum_partials(const double* __restrict__ part, uint32_t ntiles, double* out)
{
    if (threadIdx.x < 32)
    {
        double t = 0.0;
        for (uint32_t b = threadIdx.x; b < ntiles; b += 32) t += __ldcg(&part[b]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) *out = t;
    }
}

struct RhsResidual  // r_old - alpha Ap, as the forward sweeps stage it
{
    const double *r, *Ap;
    double alpha;
    __device__ float operator()(uint32_t i) const { return (float)(__ldcg(&r[i]) - alpha * __ldcg(&Ap[i])); }
};

struct RhsY  // the forward result, for the backward sweeps
{
    const float* y;
    __device__ float operator()(uint32_t i) const { return __ldcg(&y[i]); }
};

__global__ void __launch_bounds__(kPcgBandThreads) k_pcg_band(PcgBandArgs a)
{
    constexpr uint32_t NT = kPcgBandThreads;
    __shared__ KState sst;
    __shared__ int s_ok;
    __shared__ double s_best, s_sum;
    __shared__ int s_best_at;
    extern __shared__ __align__(16) unsigned char smem[];
    float* const y0 = reinterpret_cast<float*>(smem);
    float* const y1 = y0 + a.Rmax;
    const uint32_t tile = blockIdx.x, ntiles = gridDim.x;
    const uint32_t lo = tile * a.T, hi = min(a.n, lo + a.T);
    if (threadIdx.x == 0)
    {
        sst = *a.st;
        s_best = HUGE_VAL;
        s_best_at = 0;
    }
    __syncthreads();
    unsigned round = 0;
    int parity = 0;
    while (!sst.done)
    {
        const double* pold = a.p[parity];
        double* pnew = a.p[parity ^ 1];
        const double* rold = a.r[parity];
        double* rnew = a.r[parity ^ 1];
        // ---- 1. p = z + beta p_old; Ap; p.Ap
        const double beta = sst.beta;
        double acc[1] = {0.0};
        // the thread's rows (T <= 3 NT) together: row pointers, then up to 4
        // entries of each, then their gathers, so the three chains overlap
        {
            constexpr int RPT = 3;
            uint32_t ra[RPT], rb[RPT];
            double sum[RPT];
#pragma unroll
            for (int k = 0; k < RPT; ++k)
            {
                const uint32_t row = lo + threadIdx.x + k * NT;
                ra[k] = row < hi ? __ldg(&a.Arp[row]) : 0u;
                rb[k] = row < hi ? __ldg(&a.Arp[row + 1]) : 0u;
                sum[k] = 0.0;
            }
            constexpr int EPC = 4;  // entries per row per round
            for (uint32_t base = 0;; base += EPC)
            {
                bool more = false;
                double vv[RPT][EPC], xx[RPT][EPC];
#pragma unroll
                for (int k = 0; k < RPT; ++k)
#pragma unroll
                    for (int e = 0; e < EPC; ++e)
                    {
                        const uint32_t q = ra[k] + base + e;
                        const bool on = q < rb[k];
                        const uint32_t j = on ? __ldg(&a.Aci[q]) : 0u;
                        vv[k][e] = on ? __ldg(&a.Av[q]) : 0.0;
                        xx[k][e] = on ? __ldcg(&a.z[j]) + beta * __ldcg(&pold[j]) : 0.0;
                    }
#pragma unroll
                for (int k = 0; k < RPT; ++k)
#pragma unroll
                    for (int e = 0; e < EPC; ++e)
                        if (ra[k] + base + e < rb[k]) sum[k] += vv[k][e] * xx[k][e];
#pragma unroll
                for (int k = 0; k < RPT; ++k) more |= ra[k] + base + EPC < rb[k];
                if (!more) break;
            }
#pragma unroll
            for (int k = 0; k < RPT; ++k)
            {
                const uint32_t row = lo + threadIdx.x + k * NT;
                if (row < hi)
                {
                    const double pr = __ldcg(&a.z[row]) + beta * __ldcg(&pold[row]);
                    pnew[row] = pr;
                    a.Ap[row] = sum[k];
                    acc[0] += pr * sum[k];
                }
            }
        }
        block_reduce<1, NT>(acc);
        if (threadIdx.x == 0) a.red[tile] = acc[0];
        if (!grid_barrier(a.bar, ntiles * ++round, a.err, &s_ok)) break;
        sum_partials(a.red, ntiles, &s_sum);
        __syncthreads();
        if (threadIdx.x == 0) pcg_alpha(&sst, s_sum);
        __syncthreads();
        if (sst.done) break;
        // ---- 2. forward sweeps on r = r_old - alpha Ap; x, r; r.r
        const double alpha = sst.alpha;
        uint32_t elo = 0;
        const float* yk =
            band_jacobi<true>(a, a.loff, a.lval, a.ldinv, lo, hi, y0, y1, RhsResidual{rold, a.Ap, alpha}, elo);
        acc[0] = 0.0;
        for (uint32_t i = lo + threadIdx.x; i < hi; i += NT)
        {
            a.y32[i] = yk[i - elo];
            a.x[i] += alpha * pnew[i];
            const double ri = __ldcg(&rold[i]) - alpha * __ldcg(&a.Ap[i]);
            rnew[i] = ri;
            acc[0] += ri * ri;
        }
        block_reduce<1, NT>(acc);
        if (threadIdx.x == 0) a.red[ntiles + tile] = acc[0];
        if (!grid_barrier(a.bar, ntiles * ++round, a.err, &s_ok)) break;
        sum_partials(a.red + ntiles, ntiles, &s_sum);
        __syncthreads();
        if (threadIdx.x == 0)
        {
            if (!pcg_check_converged(&sst, s_sum) && a.stall_window > 0)
            {
                if (sst.relres < 0.5 * s_best)
                {
                    s_best = sst.relres;
                    s_best_at = sst.it;
                }
                else if (sst.it - s_best_at >= a.stall_window)
                {
                    sst.stalled = 1;
                    sst.iters = sst.it + 1;
                    finish(&sst, B2S_OK);
                }
            }
        }
        __syncthreads();
        if (sst.done) break;
        // ---- 3. backward sweeps on y; z; r.z and beta
        yk = band_jacobi<false>(a, a.uoff, a.uval, a.udinv, lo, hi, y0, y1, RhsY{a.y32}, elo);
        acc[0] = 0.0;
        for (uint32_t i = lo + threadIdx.x; i < hi; i += NT)
        {
            const double zi = (double)yk[i - elo];
            a.z[i] = zi;
            acc[0] += rnew[i] * zi;
        }
        block_reduce<1, NT>(acc);
        if (threadIdx.x == 0) a.red[2 * ntiles + tile] = acc[0];
        if (!grid_barrier(a.bar, ntiles * ++round, a.err, &s_ok)) break;
        sum_partials(a.red + 2 * ntiles, ntiles, &s_sum);
        __syncthreads();
        if (threadIdx.x == 0) pcg_next(&sst, s_sum);
        __syncthreads();
        parity ^= 1;
    }
    if (tile == 0 && threadIdx.x == 0) *a.st = sst;
}

}  // namespace b2s
