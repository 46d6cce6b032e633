// Chunked triangular solve: the default schedule of the IC(0) / ILU(0) and
// block ILU(0) solves (B2S_TRSV_CHUNK).  Planning (chunks, positions, slots,
// blob layout) is in trsv_plan.hpp.
//
// One CTA per chunk; CTAs take chunks from a ticket in order, so a CTA only
// waits on chunks held by CTAs that started before it.  A CTA:
//   1. copies its chunk's value blob and metadata blob (16-byte cp.async) and
//      its slice of the right-hand side (element cp.async) into shared memory;
//   2. splits into compute warps and one producer warp.  The producer's
//      lanes serve the chunk's slots in the order they are needed: each polls
//      its slot's row in the exchange array until the row carries this
//      traversal's epoch, and hands the value over in shared memory (release
//      at CTA scope).  The compute warps walk the local levels; a level is a
//      contiguous run of positions, separated by __syncwarp (one compute
//      warp) or a named barrier over the compute warps.  Every operand of a
//      row is in shared memory, so a level costs a few shared-memory round
//      trips, a divide and a barrier.
//   3. publishes each row that another chunk reads, right after computing
//      it, into the exchange array: one 64-bit word per 32-bit half of each
//      value, {epoch, bits}, written with a relaxed store (every row reaches
//      x only after the traversal, copied from shared memory).  A 64-bit access
//      is single-copy atomic, so a reader that sees the epoch in a word also
//      sees that word's value bits: one L2 round trip per slot and no fence
//      on the publishing side.
// The last CTA to finish resets the tickets and advances the epoch, so the
// exchange array never needs clearing and the launch can be replayed from a
// CUDA graph.  Waits spin without sleeping for a bounded number of polls (a
// dependency normally resolves in well under a microsecond), then back off
// with 1 us sleeps, and give up with B2S_TIMEOUT after a fixed bound.
//
// Every row is summed in its column order with the reference's arithmetic
// (sum = rhs; sum -= v * x_j; x = sum / d), so in FP64 the result equals the
// level / sync-free schedules bit for bit.  The FP32 solves multiply by a
// reciprocal of d packed once per factorisation (one extra rounding).
#pragma once
#include "syncfree.cuh"
#include "trsv_plan.hpp"

namespace b2s {

// default wait bounds (b2s_ctx_set_wait_limits changes them per context):
// polls of one slot without sleeping, and polls with a 1 us sleep that one
// lane may spend over a whole launch
constexpr unsigned kChunkFastPolls = 1u << 20;
constexpr unsigned kChunkSlowPolls = 1u << 20;

struct ChunkArgs
{
    const ChunkDesc* desc;
    const uint4* meta;
    const uint4* vals;
    const uint32_t* slot_row;
    unsigned long long* xch;  // exchange words, 2 per value component
    SyncFreeCtl ctl;          // ticket, epoch, error word (the context's)
    unsigned fast_polls;      // polls of one slot without sleeping
    unsigned slow_polls;      // sleeping polls per lane and launch
};

__device__ __forceinline__ int ld_err(const int* p)
{
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async16(void* dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

template <int BYTES>
__device__ __forceinline__ void cp_async_elem(void* dst, const void* src)
{
    static_assert(BYTES == 4 || BYTES == 8, "element size");
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ uint32_t ld_acquire_cta_shared(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.acquire.cta.shared::cta.u32 %0, [%1];" : "=r"(v) : "r"(smem_u32(p)) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_cta_shared(uint32_t* p, uint32_t v)
{
    asm volatile("st.release.cta.shared::cta.u32 [%0], %1;" ::"r"(smem_u32(p)), "r"(v) : "memory");
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// publish one value component: words w[0], w[1] = {epoch, low bits}, {epoch, high bits}
template <typename XT>
__device__ __forceinline__ void xch_put(unsigned long long* w, XT v, uint32_t epoch)
{
    const unsigned long long e = (unsigned long long)epoch << 32;
    if constexpr (sizeof(XT) == 4)
        st_relaxed_u64(w, e | __float_as_uint(v));
    else
    {
        const unsigned long long b = (unsigned long long)__double_as_longlong(v);
        st_relaxed_u64(w, e | (b & 0xffffffffull));
        st_relaxed_u64(w + 1, e | (b >> 32));
    }
}

// read one value component; false while the words do not carry `epoch`
template <typename XT>
__device__ __forceinline__ bool xch_get(const unsigned long long* w, uint32_t epoch, XT& v)
{
    if constexpr (sizeof(XT) == 4)
    {
        const unsigned long long a = ld_relaxed_u64(w);
        v = __uint_as_float((uint32_t)a);
        return (uint32_t)(a >> 32) == epoch;
    }
    else
    {
        const unsigned long long a = ld_relaxed_u64(w), b = ld_relaxed_u64(w + 1);
        v = __longlong_as_double((long long)(((b & 0xffffffffull) << 32) | (a & 0xffffffffull)));
        return (uint32_t)(a >> 32) == epoch && (uint32_t)(b >> 32) == epoch;
    }
}

// The producer warp: lane l serves slots l, l+32, ... in order.  The loop is
// warp-uniform: every pass, each lane with a pending slot polls it once (all
// lanes' polls in flight together) and hands it over as soon as its words
// carry this traversal's epoch, so no lane waits for another lane's slot.
// A slot is polled fast_polls times without sleeping, then with 1 us sleeps
// drawn from the lane's budget of slow_polls for the whole launch.  A lane
// gives up when that budget is spent or when another wait of the launch has
// already given up (the error word is set): it records B2S_TIMEOUT, hands
// over what it read, and from then on hands over its remaining slots without
// waiting, so a launch that fails ends within one budget.
template <int BS, typename XT>
__device__ __forceinline__ void produce_slots(const ChunkArgs& a, const ChunkDesc& D, uint32_t epoch, uint32_t lane,
                                              XT* xv, uint32_t* xr)
{
    uint32_t s = lane;
    uint32_t j = s < D.ns ? __ldg(&a.slot_row[D.slot + s]) : 0u;
    unsigned polls = 0, slept = 0;
    bool gave_up = false;
    while (__any_sync(0xffffffffu, s < D.ns))
    {
        if (s < D.ns)
        {
            XT val[BS];
            bool ok = true;
#pragma unroll
            for (int c = 0; c < BS; ++c) ok &= xch_get<XT>(a.xch + ((size_t)j * BS + c) * 2, epoch, val[c]);
            if (!ok && (gave_up || ++polls >= a.fast_polls))
            {
                if (!gave_up && (slept >= a.slow_polls || ld_err(a.ctl.err) != 0))
                {
                    atomicCAS(a.ctl.err, 0, (int)B2S_TIMEOUT);
                    gave_up = true;
                }
                if (gave_up)
                    ok = true;
                else
                {
                    ++slept;
                    __nanosleep(1000);
                }
            }
            if (ok)
            {
#pragma unroll
                for (int c = 0; c < BS; ++c) xv[s * BS + c] = val[c];
                st_release_cta_shared(&xr[s], 1u);
                s += 32;
                if (s < D.ns) j = __ldg(&a.slot_row[D.slot + s]);
                polls = 0;
            }
        }
    }
}

// compute warp: wait until the producer has filled slot s.  8 x fast_polls
// polls without sleeping, then 1 us sleeps from the thread's budget of
// slow_polls for the whole launch; gives up (B2S_TIMEOUT) when the budget is
// spent or another wait of the launch has given up.
__device__ __forceinline__ void slot_wait(const uint32_t* xr, uint32_t s, const ChunkArgs& a, unsigned& slept)
{
    for (unsigned polls = 0; ld_acquire_cta_shared(&xr[s]) == 0u; ++polls)
    {
        if (polls >= 8 * a.fast_polls)
        {
            if (slept >= a.slow_polls || ld_err(a.ctl.err) != 0)
            {
                atomicCAS(a.ctl.err, 0, (int)B2S_TIMEOUT);
                slept = a.slow_polls;
                return;
            }
            ++slept;
            __nanosleep(1000);
        }
    }
}

template <int NW>
__device__ __forceinline__ void compute_barrier()
{
    if constexpr (NW == 1)
        __syncwarp();
    else
        asm volatile("bar.sync 1, %0;" ::"n"(NW * 32) : "memory");
}

template <int NW>
constexpr int chunk_block() { return (NW + 1) * 32 > 256 ? (NW + 1) * 32 : 256; }

template <bool LOWER, bool UNIT, int NW, typename VT, typename XT, typename RT, int MAXQ>
__global__ void __launch_bounds__(chunk_block<NW>()) k_trsv_chunk(ChunkArgs a, const RT* __restrict__ rhs,
                                                                   XT* __restrict__ x, double* __restrict__ out64,
                                                                   const int* done)
{
    if (done && *done) return;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t s_chunk;
    const uint32_t tid = threadIdx.x;
    if (tid == 0) s_chunk = atomicAdd(&a.ctl.ticket[0], 1u);
    __syncthreads();
    const ChunkDesc D = a.desc[s_chunk];
    const uint32_t epoch = ld_flag(a.ctl.epoch) + 1u;
    const SmemLayout L = smem_layout(D.nr, D.nd, D.nl, D.ns, sizeof(VT), sizeof(XT), sizeof(RT), 1, UNIT ? 0 : 1);

    // ---- 1. stage the chunk
    {
        const uint4* vsrc = a.vals + (sizeof(VT) == 8 ? D.v64 : D.v32);
        const uint4* msrc = a.meta + D.meta;
        uint4* vdst = reinterpret_cast<uint4*>(smem + L.sv);
        uint4* mdst = reinterpret_cast<uint4*>(smem + L.meta);
        for (uint32_t i = tid; i < L.vals / 16; i += blockDim.x) cp_async16(vdst + i, vsrc + i);
        for (uint32_t i = tid; i < L.m.bytes / 16; i += blockDim.x) cp_async16(mdst + i, msrc + i);
        RT* sr = reinterpret_cast<RT*>(smem + L.sr);
        for (uint32_t k = tid; k < D.nr; k += blockDim.x) cp_async_elem<sizeof(RT)>(sr + k, rhs + D.lo + k);
        uint32_t* xr = reinterpret_cast<uint32_t*>(smem + L.xr);
        for (uint32_t s = tid; s < D.ns; s += blockDim.x) xr[s] = 0u;
        if (tid == 0) reinterpret_cast<XT*>(smem + L.sx)[D.nr] = XT(0);  // the zero of absent entries
        cp_async_wait_all();
    }
    __syncthreads();

    const uint32_t warp = tid >> 5, lane = tid & 31u;
    XT* xv = reinterpret_cast<XT*>(smem + L.xv);
    uint32_t* xr = reinterpret_cast<uint32_t*>(smem + L.xr);

    if (warp == (uint32_t)NW)
    {
        // ---- 2a. producer: values of earlier chunks, in the order they are needed
        produce_slots<1, XT>(a, D, epoch, lane, xv, xr);
        return;
    }
    if (warp > (uint32_t)NW) return;  // helpers only stage

    // ---- 2b. compute warps
    // Everything a row needs except its operands' values is fixed before the
    // traversal: its record, column entries, coefficients, right-hand side
    // and divisor.  The warp reads those for the next level while it solves
    // the current one, so a level's critical path is the operand loads, the
    // products, one divide and the barrier.
    const VT* sv = reinterpret_cast<const VT*>(smem + L.sv);
    const VT* sd = reinterpret_cast<const VT*>(smem + L.sd);
    const uint16_t* slc = reinterpret_cast<const uint16_t*>(smem + L.meta + L.m.slc);
    const uint2* rec = reinterpret_cast<const uint2*>(smem + L.meta + L.m.rec);
    const uint16_t* slv = reinterpret_cast<const uint16_t*>(smem + L.meta + L.m.slv);
    XT* sx = reinterpret_cast<XT*>(smem + L.sx);
    const RT* sr = reinterpret_cast<const RT*>(smem + L.sr);
    // A row with at most MAXQ entries is solved with straight-line code: its
    // absent entries read the zero at sx[nr] with a zero coefficient (sum -
    // 0 * 0 leaves sum, its sign included, unchanged), and the record's slot
    // mask says which entries are values of other chunks.  Longer rows loop.
    const uint32_t zero_pos = D.nr;
    struct Ops
    {
        uint32_t pr = 0, e0 = 0, e1 = 0, smask = 0;
        uint32_t m[MAXQ];
        VT vv[MAXQ];
        XT rhs = XT(0), dv = XT(1);
    };
    unsigned slept = 0;  // this thread's sleeping polls in slot waits (bounded per launch)
    // a position's record (zero past the level's end), then everything else it
    // needs, read through that record: the two steps run a level apart
    auto rec_at = [&](uint32_t t, uint32_t tend) { return t < tend ? rec[t] : make_uint2(0u, 0u); };
    auto fetch_ops = [&](uint2 rw, bool valid, uint32_t t, Ops& o) {
        o.pr = rec_perm(rw.x);
        o.e0 = rec_e0(rw.x);
        o.e1 = rec_e1(rw.y);
        o.smask = rw.y >> 16;
        o.rhs = valid ? (XT)sr[o.pr & 0x7fffu] : XT(0);
        if (!UNIT) o.dv = valid ? (XT)sd[t] : XT(1);
#pragma unroll
        for (int q = 0; q < MAXQ; ++q)
        {
            const bool on = o.e0 + q < o.e1;
            o.m[q] = on ? (uint32_t)slc[o.e0 + q] : zero_pos;
            o.vv[q] = on ? sv[o.e0 + q] : VT(0);
        }
    };
    auto fetch = [&](uint32_t t, uint32_t tend, Ops& o) { fetch_ops(rec_at(t, tend), t < tend, t, o); };
    auto solve_row = [&](uint32_t t, const Ops& o) -> XT {
        XT sum = o.rhs;
        if (o.e1 - o.e0 <= MAXQ)
        {
            XT xj[MAXQ];
            if (o.smask == 0)
            {
#pragma unroll
                for (int q = 0; q < MAXQ; ++q) xj[q] = sx[o.m[q]];
            }
            else
            {
#pragma unroll
                for (int q = 0; q < MAXQ; ++q)
                {
                    const bool slot = (o.smask >> q) & 1u;
                    if (slot) slot_wait(xr, o.m[q] & 0x7fffu, a, slept);
                    xj[q] = (slot ? xv : sx)[o.m[q] & 0x7fffu];
                }
            }
#pragma unroll
            for (int q = 0; q < MAXQ; ++q) sum -= (XT)o.vv[q] * xj[q];
        }
        else
        {
            for (uint32_t e = o.e0; e < o.e1; ++e)
            {
                const uint32_t m = slc[e];
                XT xj;
                if (m & 0x8000u)
                {
                    const uint32_t s = m & 0x7fffu;
                    slot_wait(xr, s, a, slept);
                    xj = xv[s];
                }
                else
                    xj = sx[m];
                sum -= (XT)sv[e] * xj;
            }
        }
        // FP64 divides, as the reference; FP32 multiplies by the packed reciprocal
        const XT r = UNIT ? sum : (sizeof(XT) == 4 ? sum * o.dv : sum / o.dv);
        sx[t] = r;
        // rows other chunks read are published now; every row reaches x after the traversal
        if (o.pr & 0x8000u) xch_put<XT>(a.xch + (size_t)(D.lo + (o.pr & 0x7fffu)) * 2, r, epoch);
        return r;
    };
    // Software-pipelined over levels: while level l is solved, the operands'
    // metadata of level l + 1 (read through records loaded one level earlier)
    // and the records of level l + 2 are in flight; none of them is consumed
    // before the next iteration.
    uint32_t t0 = 0, t1 = slv[1];
    uint32_t t2 = D.nl >= 2 ? slv[2] : t1;
    Ops cur;
    fetch(tid, t1, cur);
    uint2 rnext = rec_at(t1 + tid, t2);
    for (uint32_t l = 0; l < D.nl; ++l)
    {
        const uint32_t t3 = l + 3 <= D.nl ? slv[l + 3] : t2;  // the end of level l + 2
        const uint2 rnn = rec_at(t2 + tid, t3);
        Ops nxt;
        fetch_ops(rnext, t1 + tid < t2, t1 + tid, nxt);
        if (t0 + tid < t1) solve_row(t0 + tid, cur);
        for (uint32_t t = t0 + tid + NW * 32; t < t1; t += NW * 32)
        {
            Ops o;
            fetch(t, t1, o);
            solve_row(t, o);
        }
        compute_barrier<NW>();
        cur = nxt;
        rnext = rnn;
        t0 = t1;
        t1 = t2;
        t2 = t3;
    }
    // the chunk's values, from shared memory to x (and out64) in position order
    for (uint32_t t = tid; t < D.nr; t += NW * 32)
    {
        const uint32_t row = D.lo + (rec_perm(rec[t].x) & 0x7fffu);
        const XT r = sx[t];
        x[row] = r;
        if (out64) out64[row] = (double)r;
    }

    // ---- 3. the last CTA to finish resets the tickets and advances the epoch
    if (tid == 0)
    {
        __threadfence();
        const uint32_t left = atomicAdd(&a.ctl.ticket[1], 1u);
        if (left == gridDim.x - 1)
        {
            a.ctl.ticket[0] = 0u;
            a.ctl.ticket[1] = 0u;
            *a.ctl.epoch = epoch;
            __threadfence();
        }
    }
}

// Value blob of one chunk: dependency values (bs*bs per entry), then the
// divisors by position (dv per row: none, a scalar or an inverse block).
// recip: store 1/d, rounded once from FP64, instead of d (the FP32 scalar
// solves multiply by it).
template <typename VT>
__global__ void __launch_bounds__(kThreads) k_chunk_pack(const ChunkDesc* __restrict__ desc,
                                                         const uint4* __restrict__ meta,
                                                         const uint32_t* __restrict__ src, const VT* __restrict__ v,
                                                         const VT* __restrict__ d, uint4* __restrict__ vals,
                                                         uint32_t bs, uint32_t dv, int recip)
{
    const ChunkDesc D = desc[blockIdx.x];
    const SmemLayout L = smem_layout(D.nr, D.nd, D.nl, D.ns, sizeof(VT), sizeof(VT), sizeof(VT), bs, dv);
    const uint32_t bv = bs * bs;
    unsigned char* out = reinterpret_cast<unsigned char*>(vals + (sizeof(VT) == 8 ? D.v64 : D.v32));
    VT* sv = reinterpret_cast<VT*>(out + L.sv);
    const uint32_t nv = (L.sd - L.sv) / sizeof(VT);  // values with padding
    for (uint32_t e = threadIdx.x; e < nv; e += blockDim.x)
        sv[e] = e < D.nd * bv ? v[(size_t)src[D.dep + e / bv] * bv + e % bv] : VT(0);
    if (dv)
    {
        VT* sd = reinterpret_cast<VT*>(out + L.sd);
        const uint32_t* recw = reinterpret_cast<const uint32_t*>(reinterpret_cast<const unsigned char*>(meta + D.meta) +
                                                                 L.m.rec);
        const uint32_t nd = (L.vals - L.sd) / sizeof(VT);
        for (uint32_t e = threadIdx.x; e < nd; e += blockDim.x)
        {
            const uint32_t t = e / dv;
            const VT dd = t < D.nr ? d[(size_t)(D.lo + (rec_perm(recw[2 * t]) & 0x7fffu)) * dv + e % dv] : VT(0);
            sd[e] = (recip && t < D.nr) ? (VT)(1.0 / (double)dd) : dd;
        }
    }
}

// Block rows (BAIJ, bs x bs): the block forward substitution of a unit lower
// factor (x_I = t_I) or the block back substitution times the cached inverse
// of the diagonal block (x_I = inv_I t_I), with
//     t_I = rhs_I - sum_J  V_IJ x_J,   (V_IJ x_J)_r = sum_c V_IJ[r][c] x_J[c],
// each component r accumulated in the reference's order (blockMatrix.hpp:
// 584-621).  A group of BS lanes takes one position, lane r of the group
// component r; the upper solve gathers t across the group with shuffles.
// Staging, producer warp, slots, levels and publication are those of
// k_trsv_chunk.
template <bool LOWER, int BS, int NW, typename VT, typename XT, typename RT>
__global__ void __launch_bounds__(chunk_block<NW>()) k_btrsv_chunk(ChunkArgs a, const RT* __restrict__ rhs,
                                                                    XT* __restrict__ x, double* __restrict__ out64,
                                                                    const int* done)
{
    constexpr int BV = BS * BS;
    constexpr uint32_t DV = LOWER ? 0 : BV;
    constexpr uint32_t GPW = 32 / BS;  // position groups per warp
    if (done && *done) return;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t s_chunk;
    const uint32_t tid = threadIdx.x;
    if (tid == 0) s_chunk = atomicAdd(&a.ctl.ticket[0], 1u);
    __syncthreads();
    const ChunkDesc D = a.desc[s_chunk];
    const uint32_t epoch = ld_flag(a.ctl.epoch) + 1u;
    const SmemLayout L = smem_layout(D.nr, D.nd, D.nl, D.ns, sizeof(VT), sizeof(XT), sizeof(RT), BS, DV);
    {
        const uint4* vsrc = a.vals + (sizeof(VT) == 8 ? D.v64 : D.v32);
        const uint4* msrc = a.meta + D.meta;
        uint4* vdst = reinterpret_cast<uint4*>(smem + L.sv);
        uint4* mdst = reinterpret_cast<uint4*>(smem + L.meta);
        for (uint32_t i = tid; i < L.vals / 16; i += blockDim.x) cp_async16(vdst + i, vsrc + i);
        for (uint32_t i = tid; i < L.m.bytes / 16; i += blockDim.x) cp_async16(mdst + i, msrc + i);
        RT* sr = reinterpret_cast<RT*>(smem + L.sr);
        const RT* rsrc = rhs + (size_t)D.lo * BS;
        for (uint32_t k = tid; k < D.nr * BS; k += blockDim.x) cp_async_elem<sizeof(RT)>(sr + k, rsrc + k);
        uint32_t* xr = reinterpret_cast<uint32_t*>(smem + L.xr);
        for (uint32_t s = tid; s < D.ns; s += blockDim.x) xr[s] = 0u;
        cp_async_wait_all();
    }
    __syncthreads();

    const uint32_t warp = tid >> 5, lane = tid & 31u;
    XT* xv = reinterpret_cast<XT*>(smem + L.xv);
    uint32_t* xr = reinterpret_cast<uint32_t*>(smem + L.xr);
    if (warp == (uint32_t)NW)
    {
        produce_slots<BS, XT>(a, D, epoch, lane, xv, xr);
        return;
    }
    if (warp > (uint32_t)NW) return;

    const VT* sv = reinterpret_cast<const VT*>(smem + L.sv);
    const VT* sd = reinterpret_cast<const VT*>(smem + L.sd);
    const uint16_t* slc = reinterpret_cast<const uint16_t*>(smem + L.meta + L.m.slc);
    const uint2* rec = reinterpret_cast<const uint2*>(smem + L.meta + L.m.rec);
    const uint16_t* slv = reinterpret_cast<const uint16_t*>(smem + L.meta + L.m.slv);
    XT* sx = reinterpret_cast<XT*>(smem + L.sx);
    const RT* sr = reinterpret_cast<const RT*>(smem + L.sr);
    const uint32_t grp = lane / BS, r = lane % BS;
    const uint32_t gbase = grp * BS;
    const bool lane_ok = grp < GPW;
    unsigned slept = 0;  // this thread's sleeping polls in slot waits (bounded per launch)
    uint32_t t0 = 0, t1 = slv[1];
    for (uint32_t l = 0; l < D.nl; ++l)
    {
        const uint32_t tn = l + 2 <= D.nl ? slv[l + 2] : t1;  // the next level's end, read ahead
        // uniform trip count across the warp: shuffles below need every lane
        for (uint32_t tb = t0; tb < t1; tb += NW * GPW)
        {
            const uint32_t t = tb + warp * GPW + grp;
            const bool act = lane_ok && t < t1;
            XT tr = 0;
            uint32_t pr = 0;
            if (act)
            {
                const uint2 rw = rec[t];
                pr = rec_perm(rw.x);
                const uint32_t k = pr & 0x7fffu;
                tr = (XT)sr[k * BS + r];
                const uint32_t e1 = rec_e1(rw.y);
                for (uint32_t e = rec_e0(rw.x); e < e1; ++e)
                {
                    const uint32_t m = slc[e];
                    const XT* xj;
                    if (m & 0x8000u)
                    {
                        const uint32_t s = m & 0x7fffu;
                        slot_wait(xr, s, a, slept);
                        xj = xv + s * BS;
                    }
                    else
                        xj = sx + m * BS;
                    const VT* blk = sv + (size_t)e * BV + r * BS;
                    XT acc = 0;
#pragma unroll
                    for (int c = 0; c < BS; ++c) acc += (XT)blk[c] * xj[c];
                    tr -= acc;
                }
            }
            XT xr_ = tr;
            if constexpr (!LOWER)
            {
                XT tc[BS];
#pragma unroll
                for (int c = 0; c < BS; ++c) tc[c] = __shfl_sync(0xffffffffu, tr, (gbase + c) & 31u);
                if (act)
                {
                    const VT* inv = sd + (size_t)t * BV + r * BS;
                    XT acc = 0;
#pragma unroll
                    for (int c = 0; c < BS; ++c) acc += (XT)inv[c] * tc[c];
                    xr_ = acc;
                }
            }
            // the group leader stores and publishes the whole row
            XT xc[BS];
#pragma unroll
            for (int c = 0; c < BS; ++c) xc[c] = __shfl_sync(0xffffffffu, xr_, (gbase + c) & 31u);
            if (act)
            {
                sx[t * BS + r] = xr_;
                if (r == 0)
                {
                    const uint32_t row = D.lo + (pr & 0x7fffu);
#pragma unroll
                    for (int c = 0; c < BS; ++c)
                    {
                        x[(size_t)row * BS + c] = xc[c];
                        if (out64) out64[(size_t)row * BS + c] = (double)xc[c];
                    }
                    if (pr & 0x8000u)
#pragma unroll
                        for (int c = 0; c < BS; ++c) xch_put<XT>(a.xch + ((size_t)row * BS + c) * 2, xc[c], epoch);
                }
            }
        }
        compute_barrier<NW>();
        t0 = t1;
        t1 = tn;
    }
    if (tid == 0)
    {
        __threadfence();
        const uint32_t left = atomicAdd(&a.ctl.ticket[1], 1u);
        if (left == gridDim.x - 1)
        {
            a.ctl.ticket[0] = 0u;
            a.ctl.ticket[1] = 0u;
            *a.ctl.epoch = epoch;
            __threadfence();
        }
    }
}

// Device copy of a triangle's chunk plan plus its packed values.
struct ChunkSchedule
{
    uint32_t n = 0, nchunks = 0;
    bool lower = true;
    uint32_t bs = 1, dv = 1;  // block size; divisor values per row (0: unit)
    int nw = 1;
    int maxq = 4;          // scalar rows: straight-line entries per row (2, 3 or 4; longer rows loop)
    uint32_t plan_vs = 8;  // value size the chunks were sized for
    DBuf<ChunkDesc> desc;
    DBuf<uint4> meta, vals;
    DBuf<uint32_t> slot_row, src;
    DBuf<unsigned long long> xch;  // exchange words: 2 per value component
    std::vector<ChunkDesc> h_desc;
    SyncFree sf;  // ticket / epoch / error words
    const void* packed_v = nullptr;
    const void* packed_d = nullptr;
    uint32_t packed_vs = 0;

    // pattern on the host; chunks sized for values of vs bytes (8 FP64, 4 FP32)
    bool build(b2s_ctx* ctx, uint32_t nrows, const std::vector<uint32_t>& h_rp, const std::vector<uint32_t>& h_ci,
               bool lo, uint32_t divisor_values, uint32_t vs, uint32_t block = 1)
    {
        return load(ctx, plan_chunks(nrows, h_rp.data(), h_ci.data(), lo, divisor_values, vs, vs, 8, kChunkSmemBudget,
                                     block),
                    vs);
    }

    // a plan made on the host (plan_chunks with xs = vs, rs = 8) -> device
    bool load(b2s_ctx* ctx, const ChunkPlan& P, uint32_t vs)
    {
        n = P.n;
        lower = P.lower;
        bs = P.bs;
        dv = P.dv;
        plan_vs = vs;
        if (!P.ok) return false;
        nchunks = (uint32_t)P.desc.size();
        // one compute warp while a level needs at most two passes of it
        const uint32_t per_warp = 32 / bs;
        nw = P.max_level_rows <= 2 * per_warp ? 1 : 8;
        maxq = P.max_row_deps <= 2 ? 2 : P.max_row_deps == 3 ? 3 : 4;
        h_desc = P.desc;
        desc = upload(ctx, P.desc);
        meta = upload(ctx, reinterpret_cast<const uint4*>(P.meta.data()), P.meta.size() / 16);
        slot_row = upload(ctx, P.slot_row);
        src = upload(ctx, P.src);
        vals.alloc(std::max<uint64_t>(vs == 8 ? P.v64_units : P.v32_units, 1));
        xch.alloc((size_t)n * bs * 2);
        B2S_CUDA(cudaMemsetAsync(xch.p, 0, xch.bytes(), ctx->stream));
        sf.init(ctx, 0);
        return true;
    }

    template <typename VT, typename XT, typename RT>
    size_t smem_bytes() const
    {
        size_t b = 0;
        for (const ChunkDesc& d : h_desc)
            b = std::max<size_t>(b, smem_layout(d.nr, d.nd, d.nl, d.ns, sizeof(VT), sizeof(XT), sizeof(RT), bs, dv).total);
        return b;
    }

    // true when a launch with these element types fits shared memory and the value blob
    template <typename VT, typename XT, typename RT>
    bool usable() const
    {
        return nchunks && sizeof(VT) <= plan_vs && smem_bytes<VT, XT, RT>() <= kChunkSmemLimit;
    }

    // gather the factor values (and divisors) into the chunk layout
    template <typename VT>
    void pack(b2s_ctx* ctx, const VT* v, const VT* d)
    {
        if (!nchunks) return;
        const int recip = sizeof(VT) == 4 && bs == 1 && dv == 1;
        B2S_LAUNCH(ctx, k_chunk_pack<VT>, nchunks, kThreads, 0, desc.p, meta.p, src.p, v, d, vals.p, bs, dv, recip);
        packed_v = v;
        packed_d = d;
        packed_vs = sizeof(VT);
    }

    template <typename Kern, typename RT, typename XT>
    void go(b2s_ctx* ctx, Kern kern, int threads, size_t smem, const RT* rhs, XT* x, double* out64, const int* done)
    {
        static thread_local std::vector<std::pair<const void*, size_t>> configured;
        size_t* have = nullptr;
        for (auto& c : configured)
            if (c.first == reinterpret_cast<const void*>(kern)) have = &c.second;
        if (!have)
        {
            configured.emplace_back(reinterpret_cast<const void*>(kern), 0);
            have = &configured.back().second;
        }
        if (smem > *have)
        {
            B2S_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            *have = smem;
        }
        SyncFreeCtl c = sf.ctl();
        c.err = ctx->errword();  // read back by check_device_error at the next synchronisation
        const ChunkArgs a{desc.p, meta.p, vals.p, slot_row.p, xch.p, c, ctx->wait_fast_polls, ctx->wait_slow_polls};
        B2S_LAUNCH(ctx, kern, nchunks, threads, smem, a, rhs, x, out64, done);
    }

    // scalar rows
    template <bool LOWER, bool UNIT, typename VT, typename XT, typename RT>
    void run(b2s_ctx* ctx, const VT* v, const VT* d, const RT* rhs, XT* x, double* out64, const int* done)
    {
        if (!n) return;
        if (packed_v != v || packed_d != d || packed_vs != sizeof(VT)) pack<VT>(ctx, v, d);
        const size_t smem = smem_bytes<VT, XT, RT>();
        if (nw == 1 && maxq == 2)
            go(ctx, k_trsv_chunk<LOWER, UNIT, 1, VT, XT, RT, 2>, chunk_block<1>(), smem, rhs, x, out64, done);
        else if (nw == 1 && maxq == 3)
            go(ctx, k_trsv_chunk<LOWER, UNIT, 1, VT, XT, RT, 3>, chunk_block<1>(), smem, rhs, x, out64, done);
        else if (nw == 1)
            go(ctx, k_trsv_chunk<LOWER, UNIT, 1, VT, XT, RT, 4>, chunk_block<1>(), smem, rhs, x, out64, done);
        else
            go(ctx, k_trsv_chunk<LOWER, UNIT, 8, VT, XT, RT, 4>, chunk_block<8>(), smem, rhs, x, out64, done);
    }

    // block rows: unit lower, or upper times the cached inverse blocks (d)
    template <bool LOWER, int BS, typename VT, typename XT, typename RT>
    void run_block(b2s_ctx* ctx, const VT* v, const VT* d, const RT* rhs, XT* x, double* out64, const int* done)
    {
        if (!n) return;
        if (packed_v != v || packed_d != d || packed_vs != sizeof(VT)) pack<VT>(ctx, v, d);
        const size_t smem = smem_bytes<VT, XT, RT>();
        if (nw == 1)
            go(ctx, k_btrsv_chunk<LOWER, BS, 1, VT, XT, RT>, chunk_block<1>(), smem, rhs, x, out64, done);
        else
            go(ctx, k_btrsv_chunk<LOWER, BS, 8, VT, XT, RT>, chunk_block<8>(), smem, rhs, x, out64, done);
    }
};

}  // namespace b2s
