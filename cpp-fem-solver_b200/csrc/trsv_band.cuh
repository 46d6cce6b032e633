// Sweep (B2S_TRSV_JACOBI) triangular solve of a banded triangle in one
// launch (FP32 factors whose strict entries lie within B rows of the
// diagonal -- natural-order 2-D grids, for example).
//
// Rows are grouped into segments of S consecutive rows (global index / S).
// Pass 0 solves every segment on its own (the strict entries inside the
// segment, forward substitution); each of the k sweeps then recomputes every
// row from the previous pass's values outside its segment and the current
// pass's values inside it (block Jacobi over segments, Gauss-Seidel within):
//   y_s[i] = D^-1 (rhs_i - sum_{j outside} N_ij y_{s-1}[j] - sum_{j inside} N_ij y_s[j])
// with every row's strict entries taken in column order (FP32: D^-1 is the
// reciprocal 1/d).  S = 1 is plain Jacobi (a truncated Neumann series).
// The splitting of the upper triangle is the transpose of the lower one's,
// so the apply F^T F stays symmetric positive definite; with more passes
// than the dependency depth it is the exact solve.
//
// Row i of pass s reads rows back to i - (B + S - 1) of the earlier pass
// (lower; forward for upper), so the rows [lo, hi) of pass k depend only on
// rows [lo - k Bs, hi), Bs = B rounded up to a multiple of S.  A CTA loads
// that extended range once -- each thread keeps its rows' strict entries
// (u16 offsets, FP32 values), right-hand side and reciprocal in registers --
// and runs every pass with only the pass vectors in shared memory,
// separated by __syncthreads.  At pass s it computes only the segments whose
// inputs are still exact (from the range start plus s Bs on), so nothing it
// reads is stale and rows [lo, hi) equal the one-launch-per-pass schedule
// bit for bit.  The halo is recomputed by the neighbouring tiles (redundant
// work instead of communication): no CTA waits on another.  The strict
// entries and reciprocals are packed once per factorisation (k_band_pack).
#pragma once

#include <algorithm>
#include <cstdint>

#include "b2s_internal.cuh"

namespace b2s {

constexpr uint32_t kBandRowsPerThread = 8;

// W = 2: 768 threads, W = 4: 512 (register budget: 8 rows of W offsets and
// values, rhs and reciprocal per thread)
__host__ __device__ constexpr uint32_t band_threads(uint32_t W) { return W <= 2 ? 768u : 512u; }

struct BandPlan
{
    uint32_t T = 0;      // rows per tile (0: not usable)
    uint32_t B = 0;      // bandwidth: max |i - j| over strict entries
    uint32_t W = 0;      // strict entries per row slot (2 or 4)
    uint32_t Rmax = 0;   // extended rows per tile (T + k B)
    uint32_t smem = 0;   // dynamic shared memory per CTA (two sweep vectors)
    uint32_t ntiles = 0;
};

// Host planning from the triangle's pattern (rows in CSR, column-sorted);
// lower: strict entries j < i, upper: j > i.  T is chosen so that the tiles
// fill the SMs once while each thread holds at most kBandRowsPerThread rows.
// halo rows of k passes with segments of S rows
__host__ __device__ constexpr uint32_t band_halo(uint32_t k, uint32_t B, uint32_t S)
{
    return k * ((B + S - 1) / S * S);
}

// The plan from a triangle's bandwidth B (largest |i - j| of a dependency
// entry) and widest row W (dependency entries); empty when the banded kernel
// does not apply.
inline BandPlan plan_band_from(uint32_t n, uint64_t B, uint64_t W, int k, int sm_count, uint32_t S);

inline BandPlan plan_band(uint32_t n, const uint32_t* rp, const uint32_t* ci, bool lower, int k, int sm_count,
                          uint32_t S)
{
    uint64_t B = 0, W = 0;
    for (uint32_t i = 0; i < n; ++i)
    {
        uint64_t w = 0;
        for (uint32_t q = rp[i]; q < rp[i + 1]; ++q)
        {
            const uint32_t j = ci[q];
            if (lower ? j < i : j > i)
            {
                ++w;
                B = std::max<uint64_t>(B, lower ? i - j : j - i);
            }
        }
        W = std::max(W, w);
    }
    return plan_band_from(n, B, W, k, sm_count, S);
}

// The plan of the strict transpose of a lower triangle, from the lower
// triangle's pattern: the same bandwidth, and the widest column as the
// widest row.  Equal to plan_band on the transposed pattern.
inline BandPlan plan_band_transposed(uint32_t n, const uint32_t* rp, const uint32_t* ci, int k, int sm_count,
                                     uint32_t S)
{
    uint64_t B = 0, W = 0;
    std::vector<uint32_t> cols(n, 0);
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t q = rp[i]; q < rp[i + 1]; ++q)
        {
            const uint32_t j = ci[q];
            if (j < i)
            {
                B = std::max<uint64_t>(B, i - j);
                W = std::max<uint64_t>(W, ++cols[j]);
            }
        }
    return plan_band_from(n, B, W, k, sm_count, S);
}

inline BandPlan plan_band_from(uint32_t n, uint64_t B, uint64_t W, int k, int sm_count, uint32_t S)
{
    BandPlan p;
    if (!n || k <= 0) return p;
    if (B == 0) B = 1;
    if (W > 4 || B > 65535) return p;
    const uint32_t w = W <= 2 ? 2 : 4;
    const uint64_t cap = (uint64_t)band_threads(w) * kBandRowsPerThread;
    if (S != 1 && S != kBandRowsPerThread) return p;
    const uint64_t halo = band_halo((uint32_t)k, (uint32_t)B, S);
    uint64_t T = (n + (uint64_t)sm_count - 1) / (uint64_t)sm_count;
    T = (T + 31) / 32 * 32;  // a multiple of S
    if (T < 64) T = 64;
    if (halo > 8 * T) return p;  // redundant work would dominate
    const uint64_t Rm = std::min<uint64_t>(T + halo, n);
    if (Rm > cap) return p;
    p.T = (uint32_t)T;
    p.B = (uint32_t)B;
    p.W = w;
    p.Rmax = (uint32_t)Rm;
    p.smem = (uint32_t)(2 * Rm * sizeof(float));
    p.ntiles = (uint32_t)((n + T - 1) / T);
    return p;
}

// Setup: the triangle's strict entries as W column-major slots over all rows
// (slot e of row i at e*n + i, in column order; offset 0 = no entry) and the
// FP32 reciprocal of the divisor, so a tile loads its extended range with
// independent, coalesced loads.
__global__ void k_band_pack(uint32_t n, uint32_t W, int lower, int unit, const uint32_t* __restrict__ rp,
                            const uint32_t* __restrict__ ci, const float* __restrict__ v, const float* __restrict__ d,
                            uint16_t* __restrict__ eoff, float* __restrict__ eval, float* __restrict__ dinv)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        uint32_t e = 0;
        for (uint32_t q = rp[i]; q < rp[i + 1] && e < W; ++q)
        {
            const uint32_t j = ci[q];
            if (lower ? j < i : j > i)
            {
                eoff[(size_t)e * n + i] = (uint16_t)(lower ? i - j : j - i);
                eval[(size_t)e * n + i] = v[q];
                ++e;
            }
        }
        for (; e < W; ++e)
        {
            eoff[(size_t)e * n + i] = 0;
            eval[(size_t)e * n + i] = 0.f;
        }
        dinv[i] = unit ? 1.f : 1.f / d[i];
    }
}

// PCG fusion (RZ, upper triangle of the apply): the epilogue also reduces
// r.z over the written rows (FP64, fixed order: per block, then the blocks in
// order) and the last block applies the PCG scalar step pcg_next.
struct BandRz
{
    const double* r = nullptr;
    KState* st = nullptr;
    double* partial = nullptr;
    unsigned int* counter = nullptr;
};

// PCG fusion (UPD, lower triangle of the apply): the right-hand side is the
// updated residual r_old - alpha Ap, formed for every row of the extended
// range; the owned rows also store it (r_new) and update the iterate
// (xk += alpha p), and r_new.r_new is reduced for the convergence test
// pcg_check_converged (array.cpp:3559-3573).
struct BandUpd
{
    const double* r_old = nullptr;
    const double* Ap = nullptr;
    const double* p = nullptr;
    double* xk = nullptr;
    double* r_new = nullptr;
    KState* st = nullptr;
    double* partial = nullptr;
    unsigned int* counter = nullptr;
};

template <bool LOWER, int W, int S, typename RT, bool RZ = false, bool UPD = false>
__global__ void __launch_bounds__(band_threads(W)) k_trsv_band(uint32_t n, uint32_t T, uint32_t B, uint32_t Rmax,
                                                             int k, const uint16_t* __restrict__ eoff,
                                                             const float* __restrict__ eval,
                                                             const float* __restrict__ dinv,
                                                             const RT* __restrict__ rhs, float* __restrict__ x,
                                                             double* __restrict__ out64, const int* done,
                                                             BandRz rz = BandRz(), BandUpd up = BandUpd())
{
    static_assert(!(RZ && UPD), "one fused reduction per launch");
    constexpr uint32_t NT = band_threads(W), Q = kBandRowsPerThread;
    static_assert(S == 1 || S == Q, "segments: single rows, or one segment of Q rows per thread");
    if (done && *done) return;
    double alpha = 0.0;
    if constexpr (UPD) alpha = up.st->alpha;
    extern __shared__ __align__(16) unsigned char smem[];
    float* const y0 = reinterpret_cast<float*>(smem);
    float* const y1 = y0 + Rmax;

    const uint32_t lo = blockIdx.x * T;  // < n: the grid has ceil(n / T) tiles; a multiple of S
    const uint32_t hi = min(n, lo + T);
    const uint32_t Bs = (B + S - 1) / S * S;
    const uint32_t halo = (uint32_t)k * Bs;
    const uint32_t elo = LOWER ? (lo > halo ? lo - halo : 0u) : lo;
    const uint32_t ehi = LOWER ? hi : (uint32_t)min((uint64_t)n, (uint64_t)hi + halo);
    const uint32_t R = ehi - elo;  // <= Rmax <= NT * Q by the plan
    const bool cut = LOWER ? elo > 0 : ehi < n;  // the range is truncated: the halo goes stale

    // this thread's rows: strided (S = 1) or one segment of Q consecutive rows
    auto row_of = [&](uint32_t q) -> uint32_t { return S == 1 ? threadIdx.x + NT * q : Q * threadIdx.x + q; };
    uint32_t off[Q][W];
    float val[Q][W], rr[Q], di[Q];
#pragma unroll
    for (uint32_t q = 0; q < Q; ++q)
    {
        const uint32_t t = row_of(q);
        const bool in = t < R;
        const uint32_t i = elo + (in ? t : 0u);
#pragma unroll
        for (int e = 0; e < W; ++e)
        {
            off[q][e] = in ? (uint32_t)__ldg(&eoff[(size_t)e * n + i]) : 0u;
            val[q][e] = in ? __ldg(&eval[(size_t)e * n + i]) : 0.f;
        }
        if constexpr (UPD)
            rr[q] = in ? (float)(up.r_old[i] - alpha * up.Ap[i]) : 0.f;
        else
            rr[q] = in ? (float)rhs[i] : 0.f;
        di[q] = in ? __ldg(&dinv[i]) : 0.f;
    }

    // pass s writes ybuf[s & 1]; pass 0 reads nothing outside the segments
    for (int s = 0; s <= k; ++s)
    {
        const float* yin = (s & 1) ? y0 : y1;
        float* yout = (s & 1) ? y1 : y0;
        const uint32_t shrink = (cut && s > 0) ? (uint32_t)s * Bs : 0u;
        if constexpr (S == 1)
        {
            const uint32_t t0 = LOWER ? shrink : 0u;
            const uint32_t t1 = LOWER ? R : (R > shrink ? R - shrink : 0u);
#pragma unroll
            for (uint32_t q = 0; q < Q; ++q)
            {
                const uint32_t t = row_of(q);
                if (t >= t0 && t < t1)
                {
                    float sum = rr[q];
                    if (s > 0)
                    {
#pragma unroll
                        for (int e = 0; e < W; ++e)
                            if (off[q][e]) sum -= val[q][e] * yin[LOWER ? t - off[q][e] : t + off[q][e]];
                    }
                    yout[t] = sum * di[q];
                }
            }
        }
        else
        {
            // the segment [Q tid, Q tid + Q) is computed when all of it is exact
            const uint32_t g0 = Q * threadIdx.x;
            const bool live = g0 < R && (LOWER ? g0 >= shrink : min(g0 + Q, R) + shrink <= R);
            if (live)
            {
                float prev = 0.f;  // the row before (after, upper) in this segment, this pass
#pragma unroll
                for (uint32_t u = 0; u < Q; ++u)
                {
                    const uint32_t q = LOWER ? u : Q - 1 - u;
                    const uint32_t t = g0 + q;
                    if (t >= R) continue;
                    float sum = rr[q];
#pragma unroll
                    for (int e = 0; e < W; ++e)
                    {
                        const uint32_t o = off[q][e];
                        if (!o) continue;
                        const bool inside = LOWER ? o <= q : o <= Q - 1 - q;
                        const uint32_t jj = LOWER ? t - o : t + o;
                        if (inside)
                            sum -= val[q][e] * (o == 1 ? prev : yout[jj]);
                        else if (s > 0)
                            sum -= val[q][e] * yin[jj];
                    }
                    const float yv = sum * di[q];
                    yout[t] = yv;
                    prev = yv;
                }
            }
        }
        __syncthreads();
    }

    // ---- rows [lo, hi) of pass k
    const float* yk = (k & 1) ? y1 : y0;
    double acc[1] = {0.0};
    for (uint32_t i = lo + threadIdx.x; i < hi; i += NT)
    {
        const float r = yk[i - elo];
        x[i] = r;
        if (out64) out64[i] = (double)r;
        if (RZ) acc[0] += rz.r[i] * (double)r;
        if constexpr (UPD)
        {
            up.xk[i] += alpha * up.p[i];
            const double ri = up.r_old[i] - alpha * up.Ap[i];
            up.r_new[i] = ri;
            acc[0] += ri * ri;
        }
    }
    if constexpr (RZ)
    {
        if (grid_reduce_last<1, NT>(acc, rz.partial, rz.counter))
            if (threadIdx.x == 0) pcg_next(rz.st, acc[0]);
    }
    if constexpr (UPD)
    {
        if (grid_reduce_last<1, NT>(acc, up.partial, up.counter))
            if (threadIdx.x == 0) pcg_check_converged(up.st, acc[0]);
    }
}

}  // namespace b2s
