// Exact triangular solves of 5-point grid factors (IC(0) / ILU(0) of a
// natural-order 5-point stencil), one CTA for the whole triangle.
//
// Row i = y * B + x of a lower factor depends on (x, y - 1) and (x - 1, y);
// of an upper one on (x + 1, y) and (x, y + 1).  Lane j of a warp owns grid
// line y = 32 w + j (counted from the far end for an upper factor) and walks
// it one point per step, lane j at step s on point x = s - j: the line's
// previous point is the lane's own last value (a register) and the point of
// the neighbouring line is the lane below's value from the previous step (one
// shuffle).  Each warp is a CTA of its own (on its own SM, so no warp shares
// an issue slot); lane 0 takes the neighbouring line from warp w - 1's lane
// 31 through epoch-tagged 64-bit words in global memory ({epoch, 32 value
// bits}: one store publishes a value, no fence), read a group of
// kGrid5Group steps ahead and checked when the group starts, so warp w runs
// about 32 + kGrid5Group steps behind warp w - 1.  A level (anti-diagonal)
// then costs one step: a shuffle, two products, two differences and the
// divisor -- no shared-memory round trip and no barrier.  Each row is summed
// in its column order with the reference's arithmetic (FP64 divides; FP32
// multiplies by a reciprocal rounded once from FP64, as the chunked solve
// does), so the result equals the other schedules bit for bit.  Results go
// out a group at a time through shared memory, as runs of consecutive points.
//
// The coefficients are laid out line-major at set-up (point (x, y) at
// x * ny + y), so a warp's loads of one step are contiguous; they are issued
// kGrid5Group steps ahead.  Used when the grid has at most kGrid5MaxLines
// lines; otherwise the chunked schedule runs.
#pragma once
#include "trsv_chunk.cuh"

namespace b2s {

constexpr int kGrid5Group = 8;                // steps between a warp's progress reports
constexpr uint32_t kGrid5MaxLines = 4096;     // 128 CTAs of one warp
constexpr unsigned kGrid5Polls = 1u << 20;    // polls of a group's words before giving up

// per point, line-major: c_y (the coefficient of the neighbouring line's point),
// c_x (of the line's previous point), the divisor (d, its reciprocal, or none)
template <typename VT>
__global__ void __launch_bounds__(kThreads) k_grid5_pack(uint32_t B, uint32_t ny, bool lower, bool unit, int recip,
                                                         const uint32_t* __restrict__ rp,
                                                         const uint32_t* __restrict__ ci, const VT* __restrict__ v,
                                                         const VT* __restrict__ d, VT* __restrict__ cy,
                                                         VT* __restrict__ cx, VT* __restrict__ dv)
{
    const uint32_t n = B * ny;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const uint32_t x = i % B, y = i / B, t = x * ny + y;
        VT a = VT(0), b = VT(0);
        for (uint32_t e = rp[i]; e < rp[i + 1]; ++e)
        {
            const uint32_t j = ci[e];
            if (lower ? j + B == i : j == i + B) a = v[e];
            if (lower ? j + 1 == i : j == i + 1) b = v[e];
        }
        cy[t] = a;
        cx[t] = b;
        if (!unit) dv[t] = recip ? (VT)(1.0 / (double)d[i]) : d[i];
    }
}

__device__ __forceinline__ void g5_st(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long g5_ld(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// One warp per CTA; CTA w (by ticket, so it only waits on a CTA that started
// before it) owns lines 32 w .. 32 w + 31.  ctl: [0] epoch, [1] exit count,
// [2] ticket (the last CTA to leave resets [1], [2] and advances [0], so the
// launch can be replayed).  ew: each warp's last line as epoch-tagged 64-bit
// words (one per FP32 value, two per FP64 value: {epoch, 32 value bits}).
template <bool LOWER, bool UNIT, typename VT, typename XT, typename RT>
__global__ void __launch_bounds__(32) k_trsv_grid5(uint32_t B, uint32_t ny, const VT* __restrict__ cy,
                                                   const VT* __restrict__ cx, const VT* __restrict__ dv,
                                                   const RT* __restrict__ rhs, XT* __restrict__ x,
                                                   double* __restrict__ out64, const int* done,
                                                   unsigned long long* ew, uint32_t* ctl, int* err)
{
    if (done && *done) return;
    constexpr int G = kGrid5Group;
    constexpr int WPV = sizeof(XT) == 8 ? 2 : 1;  // exchange words per value
    __shared__ XT stg[G][32];                      // a group's results
    __shared__ uint32_t s_w;
    const uint32_t lane = threadIdx.x, nw = gridDim.x;
    if (lane == 0) s_w = atomicAdd(&ctl[2], 1u);
    __syncwarp();
    const uint32_t w = s_w;
    const uint32_t epoch = ld_flag(&ctl[0]) + 1u;
    const uint32_t line = w * 32u + lane;  // counted from the far end for an upper factor
    const bool valid = line < ny;
    const uint32_t y = LOWER ? line : ny - 1u - line;
    const uint32_t S = B + 31u;  // steps of a warp: lane j is busy for s in [j, j + B)
    // the operands of step s, G steps ahead
    struct Op
    {
        VT cy, cx, dv;
        RT r;
    };
    // the point of step s is k = s - lane along the line; the loads of a step
    // advance running offsets (coefficients by ny, the right-hand side by 1)
    const long long dt = LOWER ? (long long)ny : -(long long)ny, dr = LOWER ? 1 : -1;
    long long lt = LOWER ? -(long long)lane * ny + y : (long long)(B - 1u + lane) * ny + y;  // step 0
    long long lr = (long long)y * B + (LOWER ? -(long long)lane : (long long)(B - 1u + lane));
    uint32_t lk = 0u - lane;  // k of the step being loaded
    auto load_next = [&](Op& o) {
        if (valid && lk < B)
        {
            o.cy = __ldg(&cy[lt]);
            o.cx = __ldg(&cx[lt]);
            if (!UNIT) o.dv = __ldg(&dv[lt]);
            o.r = __ldg(&rhs[lr]);
        }
        lt += dt;
        lr += dr;
        ++lk;
    };
    // lane 0's neighbouring-line values of the group starting at s0 (words of warp w - 1)
    auto nb_word = [&](uint32_t s, int c) -> const unsigned long long* {
        const uint32_t xx = LOWER ? s : B - 1u - s;
        return ew + ((size_t)(w - 1) * B + xx) * WPV + c;
    };
    auto load_nb = [&](uint32_t s0, unsigned long long (&wd)[G * WPV]) {
        if (lane == 0 && w > 0)
#pragma unroll
            for (int u = 0; u < G; ++u)
#pragma unroll
                for (int c = 0; c < WPV; ++c)
                    wd[u * WPV + c] = s0 + u < B ? g5_ld(nb_word(s0 + u, c)) : 0ull;
    };
    Op ops[G];
#pragma unroll
    for (int u = 0; u < G; ++u) load_next(ops[u]);
    unsigned long long nbw[G * WPV];
    load_nb(0, nbw);
    XT prev = XT(0);  // this line's value at the previous step
    for (uint32_t s0 = 0; s0 < S; s0 += G)
    {
        // lane 0: every word of this group must carry the epoch; re-read the others
        XT nbv[G];
#pragma unroll
        for (int u = 0; u < G; ++u) nbv[u] = XT(0);
        if (w > 0)
        {
            int fail = 0;
            if (lane == 0)
            {
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
                                nbw[u * WPV + c] = g5_ld(nb_word(s0 + u, c));
                            }
                    if (all) break;
                    if (polls >= kGrid5Polls || ld_err(err) != 0)
                    {
                        fail = 1;
                        atomicCAS(err, 0, (int)B2S_TIMEOUT);
                        break;
                    }
                }
#pragma unroll
                for (int u = 0; u < G; ++u)
                {
                    if constexpr (WPV == 1)
                        nbv[u] = (XT)__uint_as_float((uint32_t)nbw[u]);
                    else
                        nbv[u] = (XT)__longlong_as_double(
                            (long long)(((nbw[2 * u + 1] & 0xffffffffull) << 32) | (nbw[2 * u] & 0xffffffffull)));
                }
            }
            if (__shfl_sync(0xffffffffu, fail, 0)) break;
            load_nb(s0 + G, nbw);  // the next group's words, checked when it starts
        }
#pragma unroll
        for (int u = 0; u < G; ++u)
        {
            const uint32_t s = s0 + (uint32_t)u;
            const uint32_t k = s - lane;  // (wraps while s < lane)
            const bool active = valid && k < B;
            const uint32_t xx = LOWER ? k : B - 1u - k;
            // the neighbouring line's point: the lane below's previous value, or warp w - 1's
            XT nb = __shfl_up_sync(0xffffffffu, prev, 1);
            if (lane == 0) nb = nbv[u];
            const Op o = ops[u];
            load_next(ops[u]);
            // The row's entries in column order: lower (x, y-1) then (x-1, y), upper
            // (x+1, y) then (x, y+1).  An absent neighbour has a +0 coefficient and a
            // +0 value (a line's first point, the first line), and s - (+0 * +0)
            // is s, its sign included.  Inactive lanes compute garbage and keep prev.
            XT sum = (XT)o.r;
            if (LOWER)
            {
                sum -= (XT)o.cy * nb;
                sum -= (XT)o.cx * prev;
            }
            else
            {
                sum -= (XT)o.cx * prev;
                sum -= (XT)o.cy * nb;
            }
            XT r;
            if constexpr (UNIT)
                r = sum;
            else if constexpr (sizeof(XT) == 4)
                r = sum * (XT)o.dv;
            else
                r = sum / (XT)o.dv;
            prev = active ? r : prev;
            stg[u][lane] = r;
            if (lane == 31u && w + 1u < nw && active)
            {
                unsigned long long* wd = ew + ((size_t)w * B + xx) * WPV;
                const unsigned long long e = (unsigned long long)epoch << 32;
                if constexpr (WPV == 1)
                    g5_st(wd, e | __float_as_uint((float)r));
                else
                {
                    const unsigned long long bits = (unsigned long long)__double_as_longlong((double)r);
                    g5_st(wd, e | (bits & 0xffffffffull));
                    g5_st(wd + 1, e | (bits >> 32));
                }
            }
        }
        __syncwarp();
        // the group's results to x: thread t writes point u = t % 8 of line t / 8
        // (+ 4 per pass), so one store instruction covers four lines' runs of
        // eight consecutive points instead of 32 scattered points
#pragma unroll
        for (int pass = 0; pass < 8; ++pass)
        {
            const uint32_t l = (uint32_t)pass * 4u + (lane >> 3), u = lane & 7u;
            const uint32_t s = s0 + u, k = s - l, ln = w * 32u + l;
            if (ln < ny && s >= l && k < B && s < S)
            {
                const uint32_t yy = LOWER ? ln : ny - 1u - ln, xx = LOWER ? k : B - 1u - k;
                const XT r = stg[u][l];
                const size_t i = (size_t)yy * B + xx;
                x[i] = r;
                if (out64) out64[i] = (double)r;
            }
        }
        __syncwarp();
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

// One triangle's 5-point grid schedule: the line-major coefficients per
// precision and the launch.
struct Grid5Tri
{
    bool on = false;
    uint32_t B = 0, ny = 0;
    DBuf<double> c64[3];
    DBuf<float> c32[3];
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
        const size_t n = (size_t)B * ny;
        DBuf<VT>* c;
        if constexpr (sizeof(VT) == 8)
            c = c64;
        else
            c = c32;
        for (int q = 0; q < 3; ++q)
            if (c[q].n < n) c[q].alloc(n);
        if (!ctl.p)
        {
            const uint32_t nw = (ny + 31) / 32;
            ew.alloc((size_t)nw * B * 2);
            ctl.alloc(3);
            B2S_CUDA(cudaMemsetAsync(ew.p, 0, ew.bytes(), ctx->stream));
            B2S_CUDA(cudaMemsetAsync(ctl.p, 0, ctl.bytes(), ctx->stream));
        }
        const int recip = sizeof(VT) == 4 && !unit;
        B2S_LAUNCH(ctx, k_grid5_pack<VT>, stream_grid(ctx, n), kThreads, 0, B, ny, lower, unit, recip, rp, ci, v, d,
                   c[0].p, c[1].p, c[2].p);
        packed_v = v;
        packed_vs = sizeof(VT);
    }
    template <bool LOWER, bool UNIT, typename VT, typename XT, typename RT>
    void run(b2s_ctx* ctx, const RT* rhs, XT* x, double* out64, const int* done)
    {
        const DBuf<VT>* c;
        if constexpr (sizeof(VT) == 8)
            c = c64;
        else
            c = c32;
        const uint32_t nw = (ny + 31) / 32;
        B2S_LAUNCH(ctx, (k_trsv_grid5<LOWER, UNIT, VT, XT, RT>), nw, 32, 0, B, ny, c[0].p, c[1].p, c[2].p, rhs, x,
                   out64, done, ew.p, ctl.p, ctx->errword());
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
