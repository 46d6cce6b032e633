// Exact triangular solves of 5-point grid factors (IC(0) / ILU(0) of a
// natural-order 5-point stencil).
//
// Row i = y * B + x of a lower factor depends on (x, y - 1) and (x - 1, y);
// of an upper one on (x + 1, y) and (x, y + 1).  Walking an upper factor from
// the far corner (k = B - 1 - x, line = ny - 1 - y) gives it the lower shape,
// so both are described in solve order (k along a line, line across).  Lane j
// of warp w owns line 32 w + j and walks it one point per step, lane j at step
// s on point k = s - j: the line's previous point is the lane's own last value
// (a register) and the point of the neighbouring line is the lane below's
// value from the previous step (one shuffle).  Each warp is a CTA of its own,
// one per SM (the dynamic shared memory is sized for that), so no warp shares
// an issue slot.  Lane 0 takes the neighbouring line from warp w - 1's lane 31
// through epoch-tagged 64-bit words in global memory ({epoch, 32 value bits}:
// one store publishes a value, no fence), published at the end of each group
// of kGrid5Group steps, read a group (FP32) or half a group (FP64) ahead and
// checked when the group starts.  A level (anti-diagonal) costs one step: a
// shuffle, two products, two differences and the divisor -- no shared-memory
// round trip and no barrier.
//
// Each row is summed in its column order with the reference's arithmetic
// (FP32 multiplies by a reciprocal rounded once from FP64, as the chunked
// solve does; FP64 forms the correctly rounded quotient from the correctly
// rounded reciprocal, g5_quotient, and divides where that is not exact), so
// the result equals the other schedules bit for bit.  The step body is
// branch-free: the write-back of the previous group's results (runs of eight
// consecutive points, through shared memory) is predicated stores interleaved
// with the steps, and the hand-over predicated stores after them.
//
// The coefficients are packed at set-up in the order the warps consume them:
// slot (w, s, j) holds lane j's point of step s as {c_y, c_x, divisor, 1 / d}
// (c_y the coefficient of the neighbouring line's point, c_x of the line's
// previous point), so one step of a warp reads 32 consecutive slots -- one
// coalesced 16-byte (FP32) or two 16-byte (FP64) loads per lane -- issued
// kGrid5Group steps ahead.  Slots off the grid (before a line starts, after
// it ends, past the last line) hold {0, 0, 1, 1}.  Used when the grid has at
// most kGrid5MaxLines lines; otherwise the chunked schedule runs.
#pragma once
#include "trsv_chunk.cuh"

namespace b2s {

constexpr int kGrid5Group = 8;                   // steps between a warp's hand-overs and checks
constexpr uint32_t kGrid5MaxLines = 4096;        // 128 CTAs
constexpr uint32_t kGrid5MinSmem = 120u << 10;   // one CTA per SM

// polls of one group's hand-over words before a grid schedule's warp gives
// up (B2S_TIMEOUT): the context's wait bounds (b2s_ctx_set_wait_limits), spin
// and sleep budgets together, as the grid schedules never sleep
inline unsigned grid_polls(const b2s_ctx* ctx)
{
    const uint64_t p = (uint64_t)ctx->wait_fast_polls + ctx->wait_slow_polls;
    return (unsigned)std::min<uint64_t>(std::max<uint64_t>(p, 1), 0xffffffffu);
}

// one packed slot: the point's two coefficients, its divisor (d; the
// reciprocal rounded once from FP64 for an FP32 factor; 1 for a unit
// diagonal) and, for FP64, the correctly rounded reciprocal 1 / d
template <typename VT>
struct alignas(4 * sizeof(VT)) G5Slot
{
    VT cy, cx, dv, rc;
};

// packed steps per warp: B + 31 steps, rounded up to whole groups, plus the
// group the last one prefetches
inline uint32_t grid5_steps(uint32_t B) { return (B + 31u + kGrid5Group - 1u) / kGrid5Group * kGrid5Group + kGrid5Group; }

template <typename VT>
__global__ void __launch_bounds__(kThreads) k_grid5_pack(uint32_t B, uint32_t ny, uint32_t SP, bool lower, bool unit,
                                                         const uint32_t* __restrict__ rp,
                                                         const uint32_t* __restrict__ ci, const VT* __restrict__ v,
                                                         const VT* __restrict__ d, G5Slot<VT>* __restrict__ slot)
{
    const uint32_t nw = (ny + 31u) / 32u;
    const size_t total = (size_t)nw * SP * 32u;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x)
    {
        const uint32_t j = (uint32_t)(q % 32u);
        const size_t ws = q / 32u;
        const uint32_t s = (uint32_t)(ws % SP), w = (uint32_t)(ws / SP);
        const uint32_t line = w * 32u + j, k = s - j;  // k wraps before the line starts
        G5Slot<VT> P{VT(0), VT(0), VT(1), VT(1)};
        if (line < ny && k < B)
        {
            const uint32_t xx = lower ? k : B - 1u - k, yy = lower ? line : ny - 1u - line, i = yy * B + xx;
            for (uint32_t e = rp[i]; e < rp[i + 1]; ++e)
            {
                const uint32_t c = ci[e];
                if (lower ? c + B == i : c == i + B) P.cy = v[e];
                if (lower ? c + 1 == i : c == i + 1) P.cx = v[e];
            }
            if (!unit)
            {
                if constexpr (sizeof(VT) == 4)
                {
                    P.dv = (VT)(1.0 / (double)d[i]);
                    P.rc = VT(0);
                }
                else
                {
                    P.dv = d[i];
                    P.rc = 1.0 / d[i];
                }
            }
        }
        slot[q] = P;
    }
}

__device__ __forceinline__ void g5_st_if(bool p, unsigned long long* a, unsigned long long v)
{
    asm volatile(
        "{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t@q st.relaxed.gpu.global.u64 [%0], %1;\n\t}" ::"l"(a), "l"(v),
        "r"((unsigned)p));
}
__device__ __forceinline__ void g5_stx_if(bool p, float* a, float v)
{
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t@q st.global.f32 [%0], %1;\n\t}" ::"l"(a), "f"(v),
                 "r"((unsigned)p));
}
__device__ __forceinline__ void g5_stx_if(bool p, double* a, double v)
{
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t@q st.global.f64 [%0], %1;\n\t}" ::"l"(a), "d"(v),
                 "r"((unsigned)p));
}
__device__ __forceinline__ unsigned long long g5_ld(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ G5Slot<float> g5_slot(const G5Slot<float>* p)
{
    const float4 q = __ldg(reinterpret_cast<const float4*>(p));
    return {q.x, q.y, q.z, q.w};
}
__device__ __forceinline__ G5Slot<double> g5_slot(const G5Slot<double>* p)
{
    const double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return {a.x, a.y, b.x, b.y};
}

// sum / d rounded to nearest from the correctly rounded reciprocal y = 1 / d:
// q0 = sum * y is within 1.5 ulp of the quotient; one correction
// q1 = q0 + (sum - d q0) y (residual by FMA) is faithful, and a second
// correction from the exact residual of q1 is the correctly rounded quotient
// (P. Markstein, IBM J. Res. Develop. 34(1), 1990: a quotient within one ulp
// and a reciprocal within half an ulp give the correctly rounded result after
// one such step).  A zero dividend gives q0, whose sign is the quotient's.
// `bad` is set where a residual could underflow or a product overflow; the
// caller then divides instead.
__device__ __forceinline__ double g5_quotient(double sum, double d, double y, bool active, bool& bad)
{
    const double q0 = sum * y;
    const double q1 = fma(fma(-q0, d, sum), y, q0);
    const double q = fma(fma(-q1, d, sum), y, q1);
    const double as = fabs(sum), aq = fabs(q0);
    const bool zero = sum == 0.0;
    bad |= active && !(zero || (as >= 0x1p-900 && as <= 0x1p+900 && aq >= 0x1p-900 && aq <= 0x1p+900));
    return zero ? q0 : q;
}

// One warp per CTA; CTA w (by ticket, so it only waits on a CTA that started
// before it) owns lines 32 w .. 32 w + 31.  ctl: [0] epoch, [1] exit count,
// [2] ticket (the last CTA to leave resets [1], [2] and advances [0], so the
// launch can be replayed).  ew: each warp's last line as epoch-tagged 64-bit
// words by k (one per FP32 value, two per FP64 value: {epoch, 32 value bits}).
template <bool LOWER, bool UNIT, typename VT, typename XT, typename RT>
__global__ void __launch_bounds__(32, 1) k_trsv_grid5(uint32_t B, uint32_t ny, uint32_t SP,
                                                      const G5Slot<VT>* __restrict__ slot,
                                                      const RT* __restrict__ rhs, XT* __restrict__ x,
                                                      double* __restrict__ out64, const int* done,
                                                      unsigned long long* ew, uint32_t* ctl, int* err,
                                                      unsigned polls_max)
{
    if (done && *done) return;
    constexpr int G = kGrid5Group;
    constexpr int WPV = sizeof(XT) == 8 ? 2 : 1;  // exchange words per value
    constexpr bool MARK = sizeof(XT) == 8 && !UNIT;
    // FP64 reads warp w - 1's words of the next group half way through a group,
    // FP32 right after the check (each the faster on 512^2, measured)
    constexpr bool NB_LATE = sizeof(XT) == 8;
    extern __shared__ __align__(16) unsigned long long g5_sm[];  // two groups of results
    XT* const stg = reinterpret_cast<XT*>(g5_sm);
    const uint32_t lane = threadIdx.x, nw = gridDim.x;
    uint32_t w = 0;
    if (lane == 0) w = atomicAdd(&ctl[2], 1u);
    w = __shfl_sync(0xffffffffu, w, 0);
    const uint32_t epoch = ld_flag(&ctl[0]) + 1u;
    const uint32_t line = w * 32u + lane;
    const bool valid = line < ny;
    const uint32_t n = B * ny, S = B + 31u;  // lane j is busy for steps s in [j, j + B)
    const uint32_t k0 = valid ? 0u - lane : B;  // k of step 0 (an invalid lane's never falls in [0, B))
    const bool has_pred = w > 0;
    const bool pub = lane == 31u && w + 1u < nw;  // lane 31 hands its line to warp w + 1
    unsigned long long* pw = ew + (size_t)w * B * WPV;
    const unsigned long long* nbg = ew + (size_t)(w ? w - 1u : 0u) * B * WPV;
    const unsigned long long etag = (unsigned long long)epoch << 32;
    // the operands of step s, G steps ahead; the slots are padded, the
    // right-hand side is read on the grid only
    struct Op
    {
        G5Slot<VT> c;
        RT r;
    };
    const G5Slot<VT>* ps = slot + (size_t)w * SP * 32u + lane;
    uint32_t lk = k0, li = line * B - lane;  // k and solve-order index line * B + k of the step being loaded
    auto load_next = [&](Op& o) {
        o.c = g5_slot(ps);
        o.r = lk < B ? __ldg(&rhs[LOWER ? li : n - 1u - li]) : RT(0);
        ps += 32;
        ++lk;
        ++li;
    };
    // warp w - 1's words for the group starting at s0.  FP64 reads them in
    // every lane (one broadcast request per word) and checks them with
    // warp-uniform branches; FP32 in lane 0 alone (each the faster on 512^2,
    // measured)
    constexpr bool UNIFORM = sizeof(XT) == 8;
    unsigned long long nbw[G * WPV];
    auto load_nb = [&](uint32_t s0) {
        if ((UNIFORM || lane == 0) && has_pred)
#pragma unroll
            for (int u = 0; u < G; ++u)
#pragma unroll
                for (int c = 0; c < WPV; ++c)
                    nbw[u * WPV + c] = s0 + u < B ? g5_ld(nbg + (size_t)(s0 + u) * WPV + c) : 0ull;
    };
    // pass p of a finished group's write-back: thread t stores point u = t % 8
    // of line 4 p + t / 8, so one store covers four lines' runs of eight points
    double* o64 = out64 ? out64 : reinterpret_cast<double*>(x);
    const bool w64 = out64 != nullptr;
    auto write_back = [&](int pass, uint32_t sg, const XT* buf) {
        const uint32_t l = (uint32_t)pass * (32u / G) + lane / G, u = lane % G;
        const uint32_t k = sg + u - l, ln = w * 32u + l;
        const bool p = ln < ny && k < B;
        const uint32_t i = ln * B + k, ii = LOWER ? i : n - 1u - i;
        const XT r = buf[u * 32u + l];
        // FP32 given out64: the FP64 copy is the result and x is not written
        // (FP64 keeps the unconditional store, the faster code there, measured)
        if constexpr (sizeof(XT) == 4)
            g5_stx_if(p && !w64, x + ii, r);
        else
            g5_stx_if(p, x + ii, r);
        g5_stx_if(p && w64, o64 + ii, (double)r);
    };
    // The row's entries in column order: lower (x, y-1) then (x-1, y), upper
    // (x+1, y) then (x, y+1).  An absent neighbour has a +0 coefficient and a
    // +0 value (a line's first point, the first line), and s - (+0 * +0) is s,
    // its sign included.
    auto row_sum = [&](RT r, VT cy, VT cx, XT nb, XT pv) -> XT {
        XT sum = (XT)r;
        if (LOWER)
        {
            sum -= (XT)cy * nb;
            sum -= (XT)cx * pv;
        }
        else
        {
            sum -= (XT)cx * pv;
            sum -= (XT)cy * nb;
        }
        return sum;
    };
    Op ops[G];
#pragma unroll
    for (int u = 0; u < G; ++u) load_next(ops[u]);
    load_nb(0);
    XT prev = XT(0);  // this line's value at the previous step
    uint32_t s0 = 0, g = 0;
    bool failed = false;
    for (; s0 < S; s0 += G, ++g)
    {
        // every word of this group must carry the epoch; the stale ones are read again
        XT nbv[G];
#pragma unroll
        for (int u = 0; u < G; ++u) nbv[u] = XT(0);
        if (has_pred)
        {
            auto fresh = [&]() {
                bool all = true;
#pragma unroll
                for (int u = 0; u < G; ++u)
#pragma unroll
                    for (int c = 0; c < WPV; ++c)
                        all &= s0 + u >= B || (uint32_t)(nbw[u * WPV + c] >> 32) == epoch;
                return all;
            };
            auto reread = [&]() {
#pragma unroll
                for (int u = 0; u < G; ++u)
#pragma unroll
                    for (int c = 0; c < WPV; ++c)
                        if (s0 + u < B && (uint32_t)(nbw[u * WPV + c] >> 32) != epoch)
                            nbw[u * WPV + c] = g5_ld(nbg + (size_t)(s0 + u) * WPV + c);
            };
            if constexpr (UNIFORM)
            {
                if (!__all_sync(0xffffffffu, fresh()))
                    for (unsigned polls = 0;; ++polls)
                    {
                        reread();
                        if (__all_sync(0xffffffffu, fresh())) break;
                        if (__any_sync(0xffffffffu, polls >= polls_max || ld_err(err) != 0))
                        {
                            if (lane == 0) atomicCAS(err, 0, (int)B2S_TIMEOUT);
                            failed = true;
                            break;
                        }
                    }
            }
            else
            {
                int fail = 0;
                if (lane == 0)
                    for (unsigned polls = 0;; ++polls)
                    {
                        bool all = true;
#pragma unroll
                        for (int u = 0; u < G; ++u)
#pragma unroll
                            for (int c = 0; c < WPV; ++c)
                                if (s0 + u < B && (uint32_t)(nbw[u * WPV + c] >> 32) != epoch)
                                {
                                    all = false;
                                    nbw[u * WPV + c] = g5_ld(nbg + (size_t)(s0 + u) * WPV + c);
                                }
                        if (all) break;
                        if (polls >= polls_max || ld_err(err) != 0)
                        {
                            fail = 1;
                            atomicCAS(err, 0, (int)B2S_TIMEOUT);
                            break;
                        }
                    }
                failed = __shfl_sync(0xffffffffu, fail, 0) != 0;
            }
            if (failed) break;
#pragma unroll
            for (int u = 0; u < G; ++u)
            {
                if constexpr (WPV == 1)
                    nbv[u] = (XT)__uint_as_float((uint32_t)nbw[u]);
                else
                    nbv[u] = (XT)__longlong_as_double(
                        (long long)(((nbw[2 * u + 1] & 0xffffffffull) << 32) | (nbw[2 * u] & 0xffffffffull)));
            }
            if constexpr (!NB_LATE) load_nb(s0 + G);  // the next group's words, checked when it starts
        }
        __syncwarp();  // the previous group's results are in stg for every lane
        XT* cur = stg + (g & 1u) * (G * 32);
        const XT* old = stg + ((g & 1u) ^ 1u) * (G * 32);
        const uint32_t kg = k0 + s0;
        const XT prev0 = prev;
        bool bad = false;
#pragma unroll
        for (int u = 0; u < G; ++u)
        {
            const uint32_t k = kg + (uint32_t)u;
            const bool active = k < B;
            // the neighbouring line's point: the lane below's previous value, or warp w - 1's
            XT nb = __shfl_up_sync(0xffffffffu, prev, 1);
            if (lane == 0) nb = nbv[u];
            const Op o = ops[u];
            load_next(ops[u]);
            const XT sum = row_sum(o.r, o.c.cy, o.c.cx, nb, prev);
            XT r;
            if constexpr (UNIT)
                r = sum;
            else if constexpr (sizeof(XT) == 4)
                r = sum * (XT)o.c.dv;
            else
                r = g5_quotient(sum, o.c.dv, o.c.rc, active, bad);
            prev = active ? r : prev;  // inactive lanes compute garbage and keep prev
            cur[u * 32 + lane] = r;
            write_back(u, s0 - G, old);  // the previous group (none before the first: k falls off)
            if constexpr (NB_LATE)
                if (u == G / 2 - 1) load_nb(s0 + G);
        }
        if constexpr (MARK)
        {
            // a quotient outside the range of g5_quotient's steps: the group again, dividing
            if (__any_sync(0xffffffffu, bad))
            {
                prev = prev0;
#pragma unroll
                for (int u = 0; u < G; ++u)
                {
                    const uint32_t k = kg + (uint32_t)u;
                    const bool active = k < B;
                    XT nb = __shfl_up_sync(0xffffffffu, prev, 1);
                    if (lane == 0) nb = nbv[u];
                    const G5Slot<VT> c = g5_slot(slot + ((size_t)w * SP + s0 + u) * 32u + lane);
                    const uint32_t i = line * B + k;
                    const RT rr = active ? rhs[LOWER ? i : n - 1u - i] : RT(0);
                    const XT r = row_sum(rr, c.cy, c.cx, nb, prev) / c.dv;
                    prev = active ? r : prev;
                    cur[u * 32 + lane] = r;
                }
            }
        }
        // lane 31: the group's values of the last line to warp w + 1
#pragma unroll
        for (int u = 0; u < G; ++u)
        {
            const uint32_t k = kg + (uint32_t)u;
            const bool p = pub && k < B;
            const XT r = cur[u * 32 + 31];
            if constexpr (WPV == 1)
                g5_st_if(p, pw + k, etag | __float_as_uint((float)r));
            else
            {
                const unsigned long long bits = (unsigned long long)__double_as_longlong((double)r);
                g5_st_if(p, pw + 2 * (size_t)k, etag | (bits & 0xffffffffull));
                g5_st_if(p, pw + 2 * (size_t)k + 1, etag | (bits >> 32));
            }
        }
    }
    if (!failed && g)
    {
        __syncwarp();
#pragma unroll
        for (int pass = 0; pass < G; ++pass) write_back(pass, s0 - G, stg + ((g - 1u) & 1u) * (G * 32));
    }
    // the last CTA to leave resets the counters and advances the epoch
    if (lane == 0)
    {
        __threadfence();
        if (atomicAdd(&ctl[1], 1u) == nw - 1u)
        {
            ctl[1] = 0u;
            ctl[2] = 0u;
            ctl[0] = epoch;
            __threadfence();
        }
    }
}

// One triangle's 5-point grid schedule: the packed slots per precision and
// the launch.
struct Grid5Tri
{
    bool on = false;
    uint32_t B = 0, ny = 0;
    DBuf<G5Slot<double>> s64;
    DBuf<G5Slot<float>> s32;
    const void* packed_v = nullptr;
    uint32_t packed_vs = 0;

    DBuf<unsigned long long> ew;  // exchange words: each warp's last line, 2 per value
    DBuf<uint32_t> ctl;           // epoch, exit count, ticket

    static bool fits(uint32_t B, uint32_t ny) { return B && ny && ny <= kGrid5MaxLines; }
    void enable(uint32_t grid_b, uint32_t lines)
    {
        B = grid_b;
        ny = lines;
        on = fits(B, ny);
    }
    template <typename VT, typename XT>
    bool usable() const
    {
        return on && packed_v && packed_vs == sizeof(VT) && ctl.p;
    }
    template <typename VT>
    void pack(b2s_ctx* ctx, const uint32_t* rp, const uint32_t* ci, const VT* v, const VT* d, bool lower, bool unit)
    {
        if (!on) return;
        const uint32_t nw = (ny + 31) / 32, SP = grid5_steps(B);
        const size_t slots = (size_t)nw * SP * 32;
        DBuf<G5Slot<VT>>* c;
        if constexpr (sizeof(VT) == 8)
            c = &s64;
        else
            c = &s32;
        if (c->n < slots) c->alloc(slots);
        if (!ctl.p)
        {
            ew.alloc((size_t)nw * B * 2);
            ctl.alloc(3);
            B2S_CUDA(cudaMemsetAsync(ew.p, 0, ew.bytes(), ctx->stream));
            B2S_CUDA(cudaMemsetAsync(ctl.p, 0, ctl.bytes(), ctx->stream));
        }
        B2S_LAUNCH(ctx, k_grid5_pack<VT>, stream_grid(ctx, slots), kThreads, 0, B, ny, SP, lower, unit, rp, ci, v, d,
                   c->p);
        packed_v = v;
        packed_vs = sizeof(VT);
    }
    template <bool LOWER, bool UNIT, typename VT, typename XT, typename RT>
    void run(b2s_ctx* ctx, const RT* rhs, XT* x, double* out64, const int* done)
    {
        const G5Slot<VT>* c;
        if constexpr (sizeof(VT) == 8)
            c = s64.p;
        else
            c = s32.p;
        const uint32_t nw = (ny + 31) / 32;
        auto kern = k_trsv_grid5<LOWER, UNIT, VT, XT, RT>;
        static bool attr = false;
        if (!attr)
        {
            B2S_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGrid5MinSmem));
            attr = true;
        }
        B2S_LAUNCH(ctx, kern, nw, 32, kGrid5MinSmem, B, ny, grid5_steps(B), c, rhs, x, out64, done, ew.p, ctl.p,
                   ctx->errword(), grid_polls(ctx));
    }
};

// Host checks of the patterns: a lower triangle whose strict entries are
// {i - B if y > 0, i - 1 if x > 0} (column order), and an upper one whose are
// {i + 1 if x + 1 < B, i + B if y + 1 < ny}; the diagonal may be stored anywhere.
inline bool grid5_triangle(uint32_t n, const uint32_t* rp, const uint32_t* ci, uint32_t B, bool lower)
{
    if (!B || n % B) return false;
    const uint32_t ny = n / B;
    for (uint32_t i = 0; i < n; ++i)
    {
        const uint32_t x = i % B, y = i / B;
        uint32_t want[2], nw = 0;
        if (lower)
        {
            if (y > 0) want[nw++] = i - B;
            if (x > 0) want[nw++] = i - 1;
        }
        else
        {
            if (x + 1 < B) want[nw++] = i + 1;
            if (y + 1 < ny) want[nw++] = i + B;
        }
        uint32_t got = 0;
        for (uint32_t e = rp[i]; e < rp[i + 1]; ++e)
        {
            const uint32_t j = ci[e];
            if (j == i) continue;
            if (got >= nw || j != want[got]) return false;
            ++got;
        }
        if (got != nw) return false;
    }
    return true;
}

}  // namespace b2s
