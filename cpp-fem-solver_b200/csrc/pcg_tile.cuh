// The whole PCG loop in one persistent kernel over 2-D tiles (tile_plan.hpp),
// for an IC(0)-type preconditioner whose two FP32 triangles are applied by k
// plain Jacobi sweeps (at most two strict entries per row).
//
// A cooperative launch of one CTA per tile (all resident, one per SM).  At
// launch a CTA copies its tile's two blobs into shared memory: the global
// rows of its owned rows and halos, every extended row's two dependencies as
// local indices, the triangles' strict entries and reciprocals, and its
// owned rows of A with local columns.  Nothing static is read from global
// memory again.  Each iteration is three phases:
//   1. p = z + beta p_old staged for the SpMV's columns; Ap = A p and p.Ap
//      for the owned rows (CSR order);
//   2. the forward sweeps over the tile's lower extended set, the right-hand
//      side r_old - alpha Ap gathered for every row of it; the owned rows
//      store y, r and x += alpha p and reduce r.r;
//   3. the backward sweeps over the upper extended set on y; the owned rows
//      store z and reduce r.z.
// Sweep s computes the rows of layers 0..k-s (a prefix of the local order),
// so the owned rows equal the global sweep definition bit for bit, as the
// banded kernel's do.  The arithmetic of every row is that of k_pcg_band;
// only the association of the three per-iteration dot products differs (the
// tiles are other row sets).
//
// A phase ends with an all-reduce that is also the grid barrier: thread 0
// fences (gpu scope, after the CTA's barrier) and publishes the tile's
// partial as two 64-bit words {epoch, 32 value bits} in a line of its own;
// thread b of every CTA polls tile b's words with relaxed loads until they
// carry the phase's epoch, fences, and leaves the value in shared memory;
// after one block barrier warp 0 sums them in tile order.  Every CTA gets the
// same bits and takes the same scalar step.  Each wait is bounded
// (kGridBarrierPolls polls); a CTA that gives up records B2S_TIMEOUT and
// leaves, and the others give up at their next all-reduce, so the launch
// always ends.
#pragma once

#include "pcg_band.cuh"
#include "tile_plan.hpp"
#include "trsv_chunk.cuh"

namespace b2s {

constexpr uint32_t kTileSlotStride = 16;      // words between two tiles' all-reduce slots (128 bytes)

struct PcgTileArgs
{
    uint32_t n, ntiles, work, ystride;
    int k;
    const TileDesc* desc;
    const uint4* vals;  // value blobs
    const uint4* idx;   // index blobs
    double* x;
    double* r[2];
    double* p[2];
    double *z, *Ap;
    float* y32;
    unsigned long long* slots;  // 3 phases x ntiles x kTileSlotStride words, zero at launch
    KState* st;
    int* err;
    int stall_window;
};

__device__ __forceinline__ void st_relaxed_gpu_u64(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed_gpu_u64(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Thread 0 holds this tile's NV partials `part`.  Publishes them for `epoch`,
// waits for every tile's and returns their sums in thread 0 (tile order, the
// same association in every CTA, so the same bits); false in every thread,
// with B2S_TIMEOUT recorded, when a wait gives up.  Each tile's 2 NV words
// ({epoch, 32 value bits} per half) sit alone in a 128-byte line
// (kTileSlotStride words apart), and thread b < ntiles polls tile b's words
// only until they carry the epoch, so a tile that has arrived is not read
// again and the polls of all CTAs spread over as many lines as tiles.
template <int NV>
__device__ __forceinline__ bool tile_allreduce(unsigned long long* slots, uint32_t tile, uint32_t ntiles,
                                               uint32_t epoch, const double (&part)[NV], double (&sum)[NV], int* err,
                                               double (*s_part)[kTileMaxTiles], int* s_fail)
{
    static_assert(2 * NV <= (int)kTileSlotStride, "slot line");
    const uint32_t tid = threadIdx.x;
    if (tid == 0)
    {
        // the CTA's writes (ordered before this thread by the barrier inside
        // block_reduce) become visible before the words that announce them
        fence_acq_rel_gpu();
        const unsigned long long e = (unsigned long long)epoch << 32;
#pragma unroll
        for (int v = 0; v < NV; ++v)
        {
            const unsigned long long b = (unsigned long long)__double_as_longlong(part[v]);
            st_relaxed_gpu_u64(&slots[(size_t)kTileSlotStride * tile + 2 * v], e | (b & 0xffffffffull));
            st_relaxed_gpu_u64(&slots[(size_t)kTileSlotStride * tile + 2 * v + 1], e | (b >> 32));
        }
    }
    if (tid < ntiles)
    {
        const unsigned long long* w = &slots[(size_t)kTileSlotStride * tid];
        unsigned long long wd[2 * NV];
        bool seen = false;
        for (unsigned polls = 0; polls < kGridBarrierPolls && !seen; ++polls)
        {
            seen = true;
#pragma unroll
            for (int q = 0; q < 2 * NV; ++q)
            {
                wd[q] = ld_relaxed_gpu_u64(w + q);
                seen &= (uint32_t)(wd[q] >> 32) == epoch;
            }
        }
        if (!seen)
        {
            *s_fail = 1;
            atomicExch(err, (int)B2S_TIMEOUT);
        }
        // the words seen carry the other CTAs' fenced writes: this fence (then
        // the block barrier below) orders the CTA's later reads after them
        fence_acq_rel_gpu();
#pragma unroll
        for (int v = 0; v < NV; ++v)
            s_part[v][tid] =
                __longlong_as_double((long long)(((wd[2 * v + 1] & 0xffffffffull) << 32) | (wd[2 * v] & 0xffffffffull)));
    }
    __syncthreads();
    if (tid < 32)
    {
#pragma unroll
        for (int v = 0; v < NV; ++v)
        {
            double t = 0.0;
            for (uint32_t b = tid; b < ntiles; b += 32) t += s_part[v][b];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            sum[v] = t;
        }
    }
    return *s_fail == 0;
}

// k + 1 passes over the extended set; rows of layers 0..k-s at pass s.
// Returns the buffer holding pass k.  Branch-free over the thread's Q rows:
// every row is evaluated at every pass and only rows t < cnt[k - s] are
// stored.  An absent dependency names the spare slot `dummy` past the set,
// which holds +0 in both buffers, with a coefficient of +0, so that
// sum - 0 * 0 leaves sum unchanged (its sign included) and the stored rows
// equal the global sweep definition bit for bit.
template <uint32_t Q>
__device__ __forceinline__ const float* tile_sweeps(int k, const uint16_t* cnt, const uint32_t (&dep)[Q],
                                                    const float2 (&val)[Q], const float (&di)[Q],
                                                    const float (&rr)[Q], float* y0, float* y1, uint32_t dummy)
{
    constexpr uint32_t NT = kTileThreads;
    if (threadIdx.x == 0)
    {
        y0[dummy] = 0.f;
        y1[dummy] = 0.f;
    }
    for (int s = 0; s <= k; ++s)
    {
        const float* yin = (s & 1) ? y0 : y1;
        float* yout = (s & 1) ? y1 : y0;
        const uint32_t t1 = cnt[k - s];
        float out[Q];
        if (s == 0)
        {
#pragma unroll
            for (uint32_t q = 0; q < Q; ++q) out[q] = rr[q] * di[q];
        }
        else
        {
            float a0[Q], a1[Q];
#pragma unroll
            for (uint32_t q = 0; q < Q; ++q)
            {
                a0[q] = yin[dep[q] & 0xFFFFu];
                a1[q] = yin[dep[q] >> 16];
            }
#pragma unroll
            for (uint32_t q = 0; q < Q; ++q)
            {
                float sum = rr[q];
                sum -= val[q].x * a0[q];
                sum -= val[q].y * a1[q];
                out[q] = sum * di[q];
            }
        }
#pragma unroll
        for (uint32_t q = 0; q < Q; ++q)
        {
            const uint32_t t = threadIdx.x + NT * q;
            if (t < t1) yout[t] = out[q];
        }
        __syncthreads();
    }
    return (k & 1) ? y1 : y0;
}

// a row's two dependencies with the absent ones (kTileNoDep) sent to the spare slot
__device__ __forceinline__ uint32_t tile_dep_slots(uint32_t w, uint32_t dummy)
{
    const uint32_t d0 = w & 0xFFFFu, d1 = w >> 16;
    return (d0 == kTileNoDep ? dummy : d0) | ((d1 == kTileNoDep ? dummy : d1) << 16);
}

template <uint32_t Q, bool FUSED>
__global__ void __launch_bounds__(kTileThreads, 1) k_pcg_tile(PcgTileArgs a)
{
    constexpr uint32_t NT = kTileThreads;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ KState sst;
    __shared__ int s_fail;
    __shared__ double s_part[2][kTileMaxTiles];
    __shared__ double s_best;
    __shared__ int s_best_at;
    const uint32_t tile = blockIdx.x, ntiles = a.ntiles, tid = threadIdx.x;
    const TileDesc& Dg = a.desc[tile];
    const uint32_t n_own = Dg.n_own, n_el = Dg.n_el, n_eu = Dg.n_eu, n_ae = Dg.n_ae;
    // ---- the tile's blobs -> shared memory (16-byte copies)
    {
        const uint4* vs = a.vals + Dg.vbase / 16;
        const uint4* is = a.idx + Dg.ibase / 16;
        uint4* vd = reinterpret_cast<uint4*>(smem);
        uint4* id = reinterpret_cast<uint4*>(smem + Dg.vbytes);
        for (uint32_t i = tid; i < Dg.vbytes / 16; i += NT) cp_async16(vd + i, vs + i);
        for (uint32_t i = tid; i < Dg.ibytes / 16; i += NT) cp_async16(id + i, is + i);
        cp_async_wait_all();
    }
    __shared__ uint16_t s_lcnt[kTileMaxSweeps + 1], s_ucnt[kTileMaxSweeps + 1];
    if (tid <= (uint32_t)a.k)
    {
        s_lcnt[tid] = Dg.lcnt[tid];
        s_ucnt[tid] = Dg.ucnt[tid];
    }
    if (tid == 0)
    {
        sst = *a.st;
        s_fail = 0;
        s_best = HUGE_VAL;
        s_best_at = 0;
    }
    __syncthreads();
    const unsigned char* ib = smem + Dg.vbytes;
    const double* aval = reinterpret_cast<const double*>(smem + Dg.o_aval);
    const float2* lvals = reinterpret_cast<const float2*>(smem + Dg.o_lvals);
    const float2* uvals = reinterpret_cast<const float2*>(smem + Dg.o_uvals);
    const float* ldinv = reinterpret_cast<const float*>(smem + Dg.o_ldinv);
    const float* udinv = reinterpret_cast<const float*>(smem + Dg.o_udinv);
    const uint32_t* owned = reinterpret_cast<const uint32_t*>(ib + Dg.o_owned);
    const uint32_t* lhalo = reinterpret_cast<const uint32_t*>(ib + Dg.o_lhalo);
    const uint32_t* ldeps = reinterpret_cast<const uint32_t*>(ib + Dg.o_ldeps);
    const uint32_t* uhalo = reinterpret_cast<const uint32_t*>(ib + Dg.o_uhalo);
    const uint32_t* udeps = reinterpret_cast<const uint32_t*>(ib + Dg.o_udeps);
    const uint32_t* ahalo = reinterpret_cast<const uint32_t*>(ib + Dg.o_ahalo);
    const uint32_t* arp = reinterpret_cast<const uint32_t*>(ib + Dg.o_arp);
    const uint16_t* acol = reinterpret_cast<const uint16_t*>(ib + Dg.o_acol);
    float* const y0 = reinterpret_cast<float*>(smem + a.work);
    float* const y1 = y0 + a.ystride;
    double* const pe = reinterpret_cast<double*>(smem + a.work);  // phase 1 only (aliases y0 / y1)
    const uint32_t lbase = s_lcnt[0];  // the lower set's layer 0: the owned rows, or (fused) the upper set
    const uint32_t dummy = a.ystride - 1;  // the sweeps' spare slot (past every set)

    // the slot regions of the iteration's all-reduces (each ntiles lines)
    unsigned long long* const slot_alpha = a.slots;
    unsigned long long* const slot_rr = a.slots + (size_t)kTileSlotStride * ntiles;
    unsigned long long* const slot_rz = a.slots + (size_t)(FUSED ? 1 : 2) * kTileSlotStride * ntiles;

    // convergence test on r.r (thread 0), with the learned solve's stall guard
    auto converge = [&](double rr) {
        if (!pcg_check_converged(&sst, rr) && a.stall_window > 0)
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
    };

    uint32_t epoch = 0;
    int parity = 0;
    // The owned rows' p and x live in registers (thread's rows t = tid + NT q);
    // p is also stored each iteration (other tiles read it), x once at the end.
    double pv[Q], xv[Q];
#pragma unroll
    for (uint32_t q = 0; q < Q; ++q)
    {
        const uint32_t t = tid + NT * q;
        const uint32_t g = t < n_own ? owned[t] : 0u;
        const bool in = t < n_own;
        pv[q] = in ? a.p[0][g] : 0.0;
        xv[q] = in ? a.x[g] : 0.0;
    }
    const float* yf = y0;  // the forward sweeps' result (phase 2 -> phase 3)
    while (!sst.done)
    {
        const double* pold = a.p[parity];
        double* pnew = a.p[parity ^ 1];
        const double* rold = a.r[parity];
        double* rnew = a.r[parity ^ 1];
        // ---- 1. p = z + beta p_old at the SpMV's columns; Ap; p.Ap
        {
            const double beta = sst.beta;
#pragma unroll
            for (uint32_t q = 0; q < Q; ++q)
            {
                const uint32_t t = tid + NT * q;
                if (t < n_own) pe[t] = __ldcg(&a.z[owned[t]]) + beta * pv[q];
            }
            for (uint32_t t = n_own + tid; t < n_ae; t += NT)
            {
                const uint32_t g = ahalo[t - n_own];
                pe[t] = __ldcg(&a.z[g]) + beta * __ldcg(&pold[g]);
            }
            __syncthreads();
            double acc[1] = {0.0};
#pragma unroll
            for (uint32_t q = 0; q < Q; ++q)
            {
                const uint32_t t = tid + NT * q;
                if (t < n_own)
                {
                    double sum = 0.0;
                    for (uint32_t e = arp[t]; e < arp[t + 1]; ++e) sum += aval[e] * pe[acol[e]];
                    const double pr = pe[t];
                    const uint32_t g = owned[t];
                    pnew[g] = pr;
                    a.Ap[g] = sum;
                    acc[0] += pr * sum;
                    pv[q] = pr;
                }
            }
            block_reduce<1, NT>(acc);
            double tot[1];
            if (!tile_allreduce<1>(slot_alpha, tile, ntiles, ++epoch, acc, tot, a.err, s_part, &s_fail)) break;
            if (tid == 0) pcg_alpha(&sst, tot[0]);
            __syncthreads();
            if (sst.done) break;
        }
        // ---- 2. forward sweeps on r = r_old - alpha Ap; x, r; r.r
        double rr_acc = 0.0;
        {
            const double alpha = sst.alpha;
            uint32_t dep[Q];
            float2 val[Q];
            float di[Q], rr[Q];
#pragma unroll
            for (uint32_t q = 0; q < Q; ++q)
            {
                const uint32_t t = tid + NT * q;
                const bool in = t < n_el;
                const uint32_t g = !in ? 0u : t < n_own ? owned[t] : t < lbase ? uhalo[t - n_own] : lhalo[t - lbase];
                dep[q] = tile_dep_slots(in ? ldeps[t] : 0xFFFFFFFFu, dummy);
                val[q] = in ? lvals[t] : make_float2(0.f, 0.f);
                di[q] = in ? ldinv[t] : 0.f;
                const double rv = in ? __ldcg(&rold[g]) - alpha * __ldcg(&a.Ap[g]) : 0.0;
                rr[q] = (float)rv;
                if (t < n_own)  // the owned rows' r, r.r and x now, before the sweeps
                {
                    rnew[g] = rv;
                    rr_acc += rv * rv;
                    xv[q] += alpha * pv[q];
                }
            }
            yf = tile_sweeps<Q>(a.k, s_lcnt, dep, val, di, rr, y0, y1, dummy);
            if constexpr (!FUSED)
            {
                // other tiles read y at this tile's rows after the grid-wide exchange
#pragma unroll
                for (uint32_t q = 0; q < Q; ++q)
                {
                    const uint32_t t = tid + NT * q;
                    if (t < n_own) a.y32[owned[t]] = yf[t];
                }
                double acc[1] = {rr_acc}, tot[1];
                block_reduce<1, NT>(acc);
                if (!tile_allreduce<1>(slot_rr, tile, ntiles, ++epoch, acc, tot, a.err, s_part, &s_fail)) break;
                if (tid == 0) converge(tot[0]);
                __syncthreads();
                if (sst.done) break;
            }
        }
        // ---- 3. backward sweeps on y; z; r.z and beta (fused: with r.r and the test)
        {
            uint32_t dep[Q];
            float2 val[Q];
            float di[Q], rr[Q];
#pragma unroll
            for (uint32_t q = 0; q < Q; ++q)
            {
                const uint32_t t = tid + NT * q;
                const bool in = t < n_eu;
                dep[q] = tile_dep_slots(in ? udeps[t] : 0xFFFFFFFFu, dummy);
                val[q] = in ? uvals[t] : make_float2(0.f, 0.f);
                di[q] = in ? udinv[t] : 0.f;
                // this thread's own forward results (read before its sweeps write):
                // every row of the upper set when fused, else the owned rows
                if constexpr (FUSED)
                    rr[q] = in ? yf[t] : 0.f;
                else
                    rr[q] = t < n_own ? yf[t] : in ? __ldcg(&a.y32[uhalo[t - n_own]]) : 0.f;
            }
            const float* yk = tile_sweeps<Q>(a.k, s_ucnt, dep, val, di, rr, y0, y1, dummy);
            double acc[2] = {0.0, 0.0};
#pragma unroll
            for (uint32_t q = 0; q < Q; ++q)
            {
                const uint32_t t = tid + NT * q;
                if (t < n_own)
                {
                    const uint32_t g = owned[t];
                    const double zi = (double)yk[t];
                    a.z[g] = zi;
                    acc[1] += rnew[g] * zi;  // (this thread's own store of phase 2)
                }
            }
            if constexpr (FUSED)
            {
                acc[0] = rr_acc;
                double tot[2];
                block_reduce<2, NT>(acc);
                if (!tile_allreduce<2>(slot_rz, tile, ntiles, ++epoch, acc, tot, a.err, s_part, &s_fail)) break;
                if (tid == 0)
                {
                    converge(tot[0]);
                    if (!sst.done) pcg_next(&sst, tot[1]);
                }
            }
            else
            {
                double one[1] = {acc[1]}, tot[1];
                block_reduce<1, NT>(one);
                if (!tile_allreduce<1>(slot_rz, tile, ntiles, ++epoch, one, tot, a.err, s_part, &s_fail)) break;
                if (tid == 0) pcg_next(&sst, tot[0]);
            }
            __syncthreads();
        }
        parity ^= 1;
    }
#pragma unroll
    for (uint32_t q = 0; q < Q; ++q)
    {
        const uint32_t t = tid + NT * q;
        if (t < n_own) a.x[owned[t]] = xv[q];
    }
    if (tile == 0 && tid == 0) *a.st = sst;
}

// Builds the index blobs of a 5-point grid's tiles (tile_plan.hpp,
// grid5_build_elem / grid5_build_dep): block t builds tile t, one thread per
// blob element, then one per extended row for the dependencies once the
// halos are written.  *bad = 1 when an index falls outside its segment.
__global__ void __launch_bounds__(kThreads) k_tile_build_grid5(const TileDesc* __restrict__ desc,
                                                               const TileGeom* __restrict__ geom,
                                                               uint8_t* __restrict__ idx, uint32_t B, uint32_t ny,
                                                               uint32_t K, bool fused, int* bad)
{
    __shared__ TileDesc D;
    __shared__ TileGeom G;
    if (threadIdx.x == 0)
    {
        D = desc[blockIdx.x];
        G = geom[blockIdx.x];
    }
    __syncthreads();
    uint8_t* ib = idx + D.ibase;
    const uint32_t ne = grid5_elements(D, G, B, ny, K, fused);
    for (uint32_t e = threadIdx.x; e < ne; e += blockDim.x)
        if (!grid5_build_elem(D, G, B, ny, K, fused, e, ib)) atomicExch(bad, 1);
    __syncthreads();  // the halos, read back below
    for (uint32_t t = threadIdx.x; t < D.n_el; t += blockDim.x) grid5_build_dep(D, G, B, ny, K, true, fused, t, ib);
    for (uint32_t t = threadIdx.x; t < D.n_eu; t += blockDim.x) grid5_build_dep(D, G, B, ny, K, false, fused, t, ib);
}

// Fills the value blobs after factorisation: A's values for the owned rows
// (checking that A's row holds exactly the planned columns), the triangles'
// strict entries and reciprocals from the banded sweep arrays (slot e of row
// g at e*n + g, checking the planned dependency's offset).  *bad = 1 when A's
// pattern or the factor's differs from the plan.
__global__ void k_tile_pack(const TileDesc* __restrict__ desc, const uint8_t* __restrict__ idx,
                            uint8_t* __restrict__ vals, uint32_t n, int k, const uint32_t* __restrict__ Arp,
                            const uint32_t* __restrict__ Aci, const double* __restrict__ Av,
                            const uint16_t* __restrict__ loff, const float* __restrict__ lval,
                            const float* __restrict__ ldinv, const uint16_t* __restrict__ uoff,
                            const float* __restrict__ uval, const float* __restrict__ udinv, int* bad)
{
    const TileDesc D = desc[blockIdx.x];
    const uint8_t* ib = idx + D.ibase;
    uint8_t* vb = vals + D.vbase;
    const uint32_t* owned = reinterpret_cast<const uint32_t*>(ib + D.o_owned);
    const uint32_t* lhalo = reinterpret_cast<const uint32_t*>(ib + D.o_lhalo);
    const uint32_t* ldeps = reinterpret_cast<const uint32_t*>(ib + D.o_ldeps);
    const uint32_t* uhalo = reinterpret_cast<const uint32_t*>(ib + D.o_uhalo);
    const uint32_t* udeps = reinterpret_cast<const uint32_t*>(ib + D.o_udeps);
    const uint32_t* ahalo = reinterpret_cast<const uint32_t*>(ib + D.o_ahalo);
    const uint32_t* arp = reinterpret_cast<const uint32_t*>(ib + D.o_arp);
    const uint16_t* acol = reinterpret_cast<const uint16_t*>(ib + D.o_acol);
    double* aval = reinterpret_cast<double*>(vb + D.o_aval);
    float2* lv = reinterpret_cast<float2*>(vb + D.o_lvals);
    float2* uv = reinterpret_cast<float2*>(vb + D.o_uvals);
    float* ld = reinterpret_cast<float*>(vb + D.o_ldinv);
    float* ud = reinterpret_cast<float*>(vb + D.o_udinv);
    auto ae_global = [&](uint32_t c) { return c < D.n_own ? owned[c] : ahalo[c - D.n_own]; };
    for (uint32_t q = threadIdx.x; q < D.n_own; q += blockDim.x)
    {
        const uint32_t g = owned[q];
        const uint32_t a0 = Arp[g], cntA = Arp[g + 1] - a0, e0 = arp[q], cntP = arp[q + 1] - e0;
        if (cntA != cntP)
        {
            atomicExch(bad, 1);
            continue;
        }
        for (uint32_t e = 0; e < cntP; ++e)
        {
            if (Aci[a0 + e] != ae_global(acol[e0 + e])) atomicExch(bad, 1);
            aval[e0 + e] = Av[a0 + e];
        }
    }
    // one triangle's extended rows: values and reciprocal from the band slots;
    // rows of layers below k (computed by the sweeps) must have every factor
    // entry planned (a missing entry shows as a planned "none" over a band slot)
    // (a fused plan's lower set: the upper set's rows first, then its own halo from base on)
    auto tri = [&](uint32_t ne, uint32_t below_k, uint32_t base, const uint32_t* halo, const uint32_t* deps,
                   const uint16_t* off, const float* val, const float* dinv, float2* outv, float* outd, bool lower) {
        auto glob = [&](uint32_t t) {
            return t < D.n_own ? owned[t] : t < base ? uhalo[t - D.n_own] : halo[t - base];
        };
        for (uint32_t t = threadIdx.x; t < ne; t += blockDim.x)
        {
            const uint32_t g = glob(t);
            const uint32_t dp[2] = {deps[t] & 0xFFFFu, deps[t] >> 16};
            float v2[2];
            for (int e = 0; e < 2; ++e)
            {
                const uint32_t o = off[(size_t)e * n + g];
                v2[e] = val[(size_t)e * n + g];
                if (dp[e] != kTileNoDep)  // (an entry of a layer-k row may point outside the set: never read)
                {
                    const uint32_t j = glob(dp[e]);
                    if (o != (lower ? g - j : j - g)) atomicExch(bad, 1);
                }
                else
                {
                    if (o != 0 && t < below_k) atomicExch(bad, 1);
                    v2[e] = 0.f;  // (read against the sweeps' +0 spare slot; layer-k rows never read it)
                }
            }
            outv[t] = make_float2(v2[0], v2[1]);
            outd[t] = dinv[g];
        }
    };
    tri(D.n_el, k > 0 ? D.lcnt[k - 1] : 0u, D.lcnt[0], lhalo, ldeps, loff, lval, ldinv, lv, ld, true);
    tri(D.n_eu, k > 0 ? D.ucnt[k - 1] : 0u, D.n_own, uhalo, udeps, uoff, uval, udinv, uv, ud, false);
}

}  // namespace b2s
