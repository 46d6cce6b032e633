// Exact triangular solves of 7-point grid factors (IC(0) / ILU(0) of a
// natural-order 7-point stencil on a B x ny x nz grid), the 3-D form of the
// 5-point grid schedule in trsv_grid5.cuh.
//
// Row i = (z ny + y) B + x of a lower factor depends on (x, y, z - 1),
// (x, y - 1, z) and (x - 1, y, z), in that column order; an upper one on
// (x + 1, y, z), (x, y + 1, z) and (x, y, z + 1).  In solve order (the upper
// factor walked from the far corner) both have the lower shape.  Lane j of
// warp w = z nyb + yb (nyb = ceil(ny / 32)) owns line (yb 32 + j, z) and
// walks it one point per step, lane j at step s on point k = s - j, as in the
// 5-point schedule: the line's previous point in a register, the
// neighbouring line of the same plane from the lane below (one shuffle; lane
// 0 from warp w - 1's lane 31 through epoch-tagged words, published at the
// end of each group), and the same line of the previous plane from warp
// w - nyb, which writes every step's value of every lane as an epoch-tagged
// word at [step][lane] -- so a warp's step is one coalesced store, and the
// next plane's warp reads the same words at the same step, one coalesced
// load per lane, a group ahead, and checks them with warp-uniform branches.
// Warps take tickets in (plane, block) order, so each waits only on warps
// that started before it; the critical path is about
// B + 31 + (nyb - 1) (block hand-over) + (nz - 1) (plane hand-over) steps.
//
// The arithmetic is the reference's (column order; FP32 multiplies by the
// reciprocal rounded once from FP64; FP64 forms the correctly rounded
// quotient from the correctly rounded reciprocal, g5_quotient, and redoes a
// group with the division where that is not exact), so the results equal the
// other schedules bit for bit.  The coefficients are packed at set-up in
// consumption order: slot (w, s, j) = {c_z, c_y, c_x, divisor[, 1 / d, 0]}
// (16 bytes FP32, 48 bytes FP64), padded off the grid with {0, 0, 0, 1, 1}.
#pragma once
#include "trsv_grid5.cuh"

namespace b2s {

constexpr uint32_t kGrid7MaxWarps = 1u << 16;  // ny / 32 * nz line warps
constexpr uint32_t kGrid7Ring = 32;            // steps of operands in flight (shared-memory ring)

// packed steps per warp: B + 31 steps, rounded up to whole groups, plus the
// steps the operand ring copies ahead of the last one
inline uint32_t grid7_steps(uint32_t B)
{
    return (B + 31u + kGrid5Group - 1u) / kGrid5Group * kGrid5Group + kGrid7Ring;
}

template <typename VT>
struct G7Slot;
template <>
struct alignas(16) G7Slot<float>
{
    float cz, cy, cx, dv;
};
template <>
struct alignas(16) G7Slot<double>
{
    double cz, cy, cx, dv, rc, pad;
};

__device__ __forceinline__ G7Slot<float> g7_slot(const G7Slot<float>* p)
{
    const float4 q = __ldg(reinterpret_cast<const float4*>(p));
    return {q.x, q.y, q.z, q.w};
}
__device__ __forceinline__ G7Slot<double> g7_slot(const G7Slot<double>* p)
{
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
    return {a.x, a.y, b.x, b.y, c.x, 0.0};
}
__device__ __forceinline__ void g7_st2_if(bool q, unsigned long long* p, unsigned long long a, unsigned long long b)
{
    asm volatile(
        "{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %3, 0;\n\t@q st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};\n\t}" ::"l"(p),
        "l"(a), "l"(b), "r"((unsigned)q));
}
__device__ __forceinline__ void g7_ld2(const unsigned long long* p, unsigned long long& a, unsigned long long& b)
{
    asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p));
}
__device__ __forceinline__ void g7_cp16(uint32_t dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
// BYTES (4 or 8) of src, zero-filled where src_bytes is 0
template <int BYTES>
__device__ __forceinline__ void g7_cp_small(uint32_t dst, const void* src, uint32_t src_bytes)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(dst), "l"(src), "n"(BYTES), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void g7_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void g7_cp_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <typename VT>
__global__ void __launch_bounds__(kThreads) k_grid7_pack(uint32_t B, uint32_t ny, uint32_t nz, uint32_t SP, bool lower,
                                                         bool unit, const uint32_t* __restrict__ rp,
                                                         const uint32_t* __restrict__ ci, const VT* __restrict__ v,
                                                         const VT* __restrict__ d, G7Slot<VT>* __restrict__ slot)
{
    const uint32_t nyb = (ny + 31u) / 32u, P = B * ny, n = P * nz;
    const size_t total = (size_t)nyb * nz * SP * 32u;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x)
    {
        const uint32_t j = (uint32_t)(q % 32u);
        const size_t ws = q / 32u;
        const uint32_t s = (uint32_t)(ws % SP), w = (uint32_t)(ws / SP);
        const uint32_t zs = w / nyb, ys = (w % nyb) * 32u + j, k = s - j;  // solve order; k wraps before the line
        G7Slot<VT> P7{};
        P7.dv = VT(1);
        if constexpr (sizeof(VT) == 8) P7.rc = 1.0;
        if (ys < ny && k < B)
        {
            const uint32_t ii = (zs * ny + ys) * B + k, i = lower ? ii : n - 1u - ii;
            for (uint32_t e = rp[i]; e < rp[i + 1]; ++e)
            {
                const uint32_t c = ci[e];
                if (lower ? c + P == i : c == i + P) P7.cz = v[e];
                if (lower ? c + B == i : c == i + B) P7.cy = v[e];
                if (lower ? c + 1 == i : c == i + 1) P7.cx = v[e];
            }
            if (!unit)
            {
                if constexpr (sizeof(VT) == 4)
                    P7.dv = (VT)(1.0 / (double)d[i]);
                else
                {
                    P7.dv = d[i];
                    P7.rc = 1.0 / d[i];
                }
            }
        }
        slot[q] = P7;
    }
}

// ctl: [0] epoch, [1] exit count, [2] ticket (the last CTA to leave resets
// [1], [2] and advances [0], so the launch can be replayed).  ew: each warp's
// last line by k (one word per FP32 value, two per FP64 value); zw: each
// warp's values of every step and lane, [step][lane] (same word format).
template <bool LOWER, bool UNIT, typename VT, typename XT, typename RT>
__global__ void __launch_bounds__(32, 1) k_trsv_grid7(uint32_t B, uint32_t ny, uint32_t nz, uint32_t SP,
                                                      const G7Slot<VT>* __restrict__ slot,
                                                      const RT* __restrict__ rhs, XT* __restrict__ x,
                                                      double* __restrict__ out64, const int* done,
                                                      unsigned long long* ew, unsigned long long* zw, uint32_t* ctl,
                                                      int* err, unsigned polls_max)
{
    if (done && *done) return;
    constexpr int G = kGrid5Group;
    constexpr int WPV = sizeof(XT) == 8 ? 2 : 1;  // exchange words per value
    constexpr bool MARK = sizeof(XT) == 8 && !UNIT;
    // FP32 reads the next group's words half way through a group, FP64 right
    // after the check (each the faster on 128^3, measured)
    constexpr bool NB_LATE = sizeof(XT) == 4;
    extern __shared__ __align__(16) unsigned long long g7_sm[];  // two groups of results (4 KB), the operand ring
    XT* const stg = reinterpret_cast<XT*>(g7_sm);
    const uint32_t lane = threadIdx.x, nw = gridDim.x;
    uint32_t w = 0;
    if (lane == 0) w = atomicAdd(&ctl[2], 1u);
    w = __shfl_sync(0xffffffffu, w, 0);
    const uint32_t epoch = ld_flag(&ctl[0]) + 1u;
    const uint32_t nyb = (ny + 31u) / 32u, zs = w / nyb, yb = w % nyb;
    const uint32_t ys = yb * 32u + lane, L = zs * ny + ys;  // this lane's line in solve order
    const bool valid = ys < ny;
    const uint32_t n = B * ny * nz, S = B + 31u;
    const uint32_t k0 = valid ? 0u - lane : B;
    const bool has_y = yb > 0, has_z = zs > 0;  // warp w - 1 (same plane), warp w - nyb (previous plane)
    const bool pub_y = lane == 31u && yb + 1u < nyb;
    const bool pub_z = zs + 1u < nz;
    unsigned long long* pw = ew + (size_t)w * B * WPV;
    const unsigned long long* nbg = ew + (size_t)(has_y ? w - 1u : 0u) * B * WPV;
    unsigned long long* zo = zw + (size_t)w * SP * 32u * WPV + lane * WPV;
    const unsigned long long* zi = zw + (size_t)(has_z ? w - nyb : 0u) * SP * 32u * WPV + lane * WPV;
    const unsigned long long etag = (unsigned long long)epoch << 32;
    struct Op
    {
        G7Slot<VT> c;
        RT r;
    };
    const G7Slot<VT>* ps = slot + (size_t)w * SP * 32u + lane;
    uint32_t lk = k0, li = L * B - lane, lq = 0;  // k, solve-order index and ring entry of the step being fetched
    // registers, a group ahead (FP64 with a divisor: its long steps hide the
    // latency) ...
    auto load_next = [&](Op& o) {
        o.c = g7_slot(ps);
        o.r = lk < B ? __ldg(&rhs[LOWER ? li : n - 1u - li]) : RT(0);
        ps += 32;
        ++lk;
        ++li;
    };
    // ... or a shared-memory ring of kGrid7Ring steps copied asynchronously
    // kGrid7Ring - 1 steps ahead (FP32 and unit triangles, whose short steps
    // would wait on operands that 128^3 streams from DRAM): step s reads entry
    // s % kGrid7Ring, and its copy for step s + kGrid7Ring - 1 refills the
    // entry that step s - 1 read
    constexpr bool RING = sizeof(VT) == 4 || UNIT;
    constexpr uint32_t D = kGrid7Ring;
    const uint32_t ring_c = (uint32_t)__cvta_generic_to_shared(g7_sm) + 4096u;
    const uint32_t ring_r = ring_c + D * 32u * (uint32_t)sizeof(G7Slot<VT>);
    const G7Slot<VT>* ring_cp =
        reinterpret_cast<const G7Slot<VT>*>(reinterpret_cast<const unsigned char*>(g7_sm) + 4096);
    const RT* ring_rp = reinterpret_cast<const RT*>(ring_cp + D * 32u);
    auto copy_next = [&]() {
        const uint32_t e = lq * 32u + lane;
#pragma unroll
        for (uint32_t c = 0; c < sizeof(G7Slot<VT>) / 16; ++c)
            g7_cp16(ring_c + e * (uint32_t)sizeof(G7Slot<VT>) + 16u * c,
                    reinterpret_cast<const unsigned char*>(ps) + 16u * c);
        const bool on = lk < B;
        g7_cp_small<sizeof(RT)>(ring_r + e * (uint32_t)sizeof(RT), on ? &rhs[LOWER ? li : n - 1u - li] : rhs,
                                on ? (uint32_t)sizeof(RT) : 0u);
        g7_cp_commit();
        ps += 32;
        ++lk;
        ++li;
        lq = lq + 1u == D ? 0u : lq + 1u;
    };
    // warp w - 1's last-line words (every lane reads them) and warp w - nyb's
    // words of this lane, for the group starting at s0
    unsigned long long nbw[G * WPV], zbw[G * WPV];
    auto load_nb = [&](uint32_t s0) {
        if (has_y)
#pragma unroll
            for (int u = 0; u < G; ++u)
#pragma unroll
                for (int c = 0; c < WPV; ++c)
                    nbw[u * WPV + c] = s0 + u < B ? g5_ld(nbg + (size_t)(s0 + u) * WPV + c) : 0ull;
        if (has_z)
#pragma unroll
            for (int u = 0; u < G; ++u)
            {
                if constexpr (WPV == 1)
                    zbw[u] = g5_ld(zi + (size_t)(s0 + u) * 32u);
                else
                    g7_ld2(zi + (size_t)(s0 + u) * 64u, zbw[2 * u], zbw[2 * u + 1]);
            }
    };
    double* o64 = out64 ? out64 : reinterpret_cast<double*>(x);
    const bool w64 = out64 != nullptr;
    auto write_back = [&](int pass, uint32_t sg, const XT* buf) {
        const uint32_t l = (uint32_t)pass * (32u / G) + lane / G, u = lane % G;
        const uint32_t k = sg + u - l, yl = yb * 32u + l;
        const bool p = yl < ny && k < B;
        const uint32_t i = (zs * ny + yl) * B + k, ii = LOWER ? i : n - 1u - i;
        const XT r = buf[u * 32u + l];
        g5_stx_if(p && !w64, x + ii, r);  // given out64, the FP64 copy is the result and x is not written
        g5_stx_if(p && w64, o64 + ii, (double)r);
    };
    // the row's entries in column order: lower (z-1), (y-1), (x-1); upper
    // (x+1), (y+1), (z+1); absent ones have +0 coefficients and +0 values
    auto row_sum = [&](RT r, const G7Slot<VT>& c, XT zb, XT nb, XT pv) -> XT {
        XT sum = (XT)r;
        if (LOWER)
        {
            sum -= (XT)c.cz * zb;
            sum -= (XT)c.cy * nb;
            sum -= (XT)c.cx * pv;
        }
        else
        {
            sum -= (XT)c.cx * pv;
            sum -= (XT)c.cy * nb;
            sum -= (XT)c.cz * zb;
        }
        return sum;
    };
    auto word_value = [](const unsigned long long* wd) -> XT {
        if constexpr (WPV == 1)
            return (XT)__uint_as_float((uint32_t)wd[0]);
        else
            return (XT)__longlong_as_double(
                (long long)(((wd[1] & 0xffffffffull) << 32) | (wd[0] & 0xffffffffull)));
    };
    Op ops[RING ? 1 : G];
    if constexpr (RING)
        for (uint32_t q = 0; q + 1 < D; ++q) copy_next();
    else
#pragma unroll
        for (int u = 0; u < G; ++u) load_next(ops[u]);
    load_nb(0);
    XT prev = XT(0);
    uint32_t s0 = 0, g = 0;
    bool failed = false;
    for (; s0 < S; s0 += G, ++g)
    {
        // the group's words from warps w - 1 and w - nyb must carry the epoch;
        // stale ones are read again (warp-uniform branches)
        auto fresh = [&]() {
            bool all = true;
#pragma unroll
            for (int u = 0; u < G; ++u)
#pragma unroll
                for (int c = 0; c < WPV; ++c)
                {
                    all &= !has_y || s0 + u >= B || (uint32_t)(nbw[u * WPV + c] >> 32) == epoch;
                    all &= !has_z || (uint32_t)(zbw[u * WPV + c] >> 32) == epoch;
                }
            return all;
        };
        if ((has_y || has_z) && !__all_sync(0xffffffffu, fresh()))
            for (unsigned polls = 0;; ++polls)
            {
#pragma unroll
                for (int u = 0; u < G; ++u)
#pragma unroll
                    for (int c = 0; c < WPV; ++c)
                    {
                        if (has_y && s0 + u < B && (uint32_t)(nbw[u * WPV + c] >> 32) != epoch)
                            nbw[u * WPV + c] = g5_ld(nbg + (size_t)(s0 + u) * WPV + c);
                        if (has_z && (uint32_t)(zbw[u * WPV + c] >> 32) != epoch)
                            zbw[u * WPV + c] = g5_ld(zi + (size_t)(s0 + u) * 32u * WPV + c);
                    }
                if (__all_sync(0xffffffffu, fresh())) break;
                if (__any_sync(0xffffffffu, polls >= polls_max || ld_err(err) != 0))
                {
                    if (lane == 0) atomicCAS(err, 0, (int)B2S_TIMEOUT);
                    failed = true;
                    break;
                }
            }
        if (failed) break;
        XT nbv[G], zbv[G];
#pragma unroll
        for (int u = 0; u < G; ++u)
        {
            nbv[u] = has_y ? word_value(&nbw[u * WPV]) : XT(0);
            zbv[u] = has_z ? word_value(&zbw[u * WPV]) : XT(0);
        }
        if constexpr (!NB_LATE) load_nb(s0 + G);  // the next group's words, checked when it starts
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
            XT nb = __shfl_up_sync(0xffffffffu, prev, 1);
            if (lane == 0) nb = nbv[u];
            Op o;
            if constexpr (RING)
            {
                g7_cp_wait<D - 2>();  // this step's copies have landed
                const uint32_t e = ((s0 % D) + (uint32_t)u) * 32u + lane;
                o.c = ring_cp[e];
                o.r = ring_rp[e];
                copy_next();
            }
            else
            {
                o = ops[u];
                load_next(ops[u]);
            }
            const XT sum = row_sum(o.r, o.c, zbv[u], nb, prev);
            XT r;
            if constexpr (UNIT)
                r = sum;
            else if constexpr (sizeof(XT) == 4)
                r = sum * (XT)o.c.dv;
            else
                r = g5_quotient(sum, o.c.dv, o.c.rc, active, bad);
            prev = active ? r : prev;
            cur[u * 32 + lane] = r;
            write_back(u, s0 - G, old);
            if constexpr (NB_LATE)
                if (u == G / 2 - 1) load_nb(s0 + G);
            // this step's value to the next plane's warp ([step][lane]); with the
            // FP64 quotient only while no lane of the group has needed the
            // division yet (a redo keeps the earlier steps' values: both
            // roundings are correct), the rest after the group
            bool pz = pub_z;
            if constexpr (MARK) pz = pz && !__any_sync(0xffffffffu, bad);
            if constexpr (WPV == 1)
                g5_st_if(pz, zo + (size_t)(s0 + u) * 32u, etag | __float_as_uint((float)r));
            else
            {
                const unsigned long long bits = (unsigned long long)__double_as_longlong((double)r);
                g7_st2_if(pz, zo + (size_t)(s0 + u) * 64u, etag | (bits & 0xffffffffull), etag | (bits >> 32));
            }
        }
        if constexpr (MARK)
        {
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
                    const G7Slot<VT> c = g7_slot(slot + ((size_t)w * SP + s0 + u) * 32u + lane);
                    const uint32_t i = L * B + k;
                    const RT rr = active ? rhs[LOWER ? i : n - 1u - i] : RT(0);
                    const XT r = row_sum(rr, c, zbv[u], nb, prev) / c.dv;
                    prev = active ? r : prev;
                    cur[u * 32 + lane] = r;
                }
                // the group's values to the next plane's warp (the steps already
                // handed over get the same values again)
#pragma unroll
                for (int u = 0; u < G; ++u)
                {
                    const unsigned long long bits =
                        (unsigned long long)__double_as_longlong((double)cur[u * 32 + lane]);
                    g7_st2_if(pub_z, zo + (size_t)(s0 + u) * 64u, etag | (bits & 0xffffffffull), etag | (bits >> 32));
                }
            }
        }
        // lane 31: the group's values of the last line to warp w + 1
#pragma unroll
        for (int u = 0; u < G; ++u)
        {
            const uint32_t k = kg + (uint32_t)u;
            const bool p = pub_y && k < B;
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
    if constexpr (RING) g7_cp_wait<0>();  // no copy into shared memory outlives the CTA
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

// One triangle's 7-point grid schedule: packed slots per precision, the
// exchange words and the launch.
struct Grid7Tri
{
    bool on = false;
    uint32_t B = 0, ny = 0, nz = 0;
    DBuf<G7Slot<double>> s64;
    DBuf<G7Slot<float>> s32;
    const void* packed_v = nullptr;
    uint32_t packed_vs = 0;
    DBuf<unsigned long long> ew, zw;
    DBuf<uint32_t> ctl;

    uint32_t warps() const { return (ny + 31) / 32 * nz; }
    static bool fits(uint32_t b, uint32_t y, uint32_t z)
    {
        return b >= 2 && y >= 2 && z >= 2 && (uint64_t)(y + 31) / 32 * z <= kGrid7MaxWarps;
    }
    void enable(uint32_t b, uint32_t y, uint32_t z)
    {
        B = b;
        ny = y;
        nz = z;
        on = fits(B, ny, nz);
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
        const uint32_t nw = warps(), SP = grid7_steps(B);
        const size_t slots = (size_t)nw * SP * 32;
        DBuf<G7Slot<VT>>* c;
        if constexpr (sizeof(VT) == 8)
            c = &s64;
        else
            c = &s32;
        if (c->n < slots) c->alloc(slots);
        if (!ctl.p)
        {
            ew.alloc((size_t)nw * B * 2);
            zw.alloc(slots * 2);
            ctl.alloc(3);
            B2S_CUDA(cudaMemsetAsync(ew.p, 0, ew.bytes(), ctx->stream));
            B2S_CUDA(cudaMemsetAsync(zw.p, 0, zw.bytes(), ctx->stream));
            B2S_CUDA(cudaMemsetAsync(ctl.p, 0, ctl.bytes(), ctx->stream));
        }
        B2S_LAUNCH(ctx, k_grid7_pack<VT>, stream_grid(ctx, slots), kThreads, 0, B, ny, nz, SP, lower, unit, rp, ci, v,
                   d, c->p);
        packed_v = v;
        packed_vs = sizeof(VT);
    }
    template <bool LOWER, bool UNIT, typename VT, typename XT, typename RT>
    void run(b2s_ctx* ctx, const RT* rhs, XT* x, double* out64, const int* done)
    {
        const G7Slot<VT>* c;
        if constexpr (sizeof(VT) == 8)
            c = s64.p;
        else
            c = s32.p;
        auto kern = k_trsv_grid7<LOWER, UNIT, VT, XT, RT>;
        static bool attr = false;
        if (!attr)
        {
            B2S_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGrid5MinSmem));
            attr = true;
        }
        B2S_LAUNCH(ctx, kern, warps(), 32, kGrid5MinSmem, B, ny, nz, grid7_steps(B), c, rhs, x, out64, done, ew.p,
                   zw.p, ctl.p, ctx->errword(), grid_polls(ctx));
    }
};

// Host checks: the dimensions of a lower triangle that is a natural-order
// 7-point grid's (B >= 2, ny >= 2, nz >= 2; strict entries {i - B ny if
// z > 0, i - B if y > 0, i - 1 if x > 0} in column order), and the same test
// for either triangle at given dimensions (the diagonal may be stored anywhere).
inline bool grid7_triangle(uint32_t n, const uint32_t* rp, const uint32_t* ci, uint32_t B, uint32_t ny, bool lower)
{
    if (B < 2 || ny < 2 || n % (B * ny) || n / (B * ny) < 2) return false;
    const uint32_t P = B * ny, nz = n / P;
    for (uint32_t i = 0; i < n; ++i)
    {
        const uint32_t x = i % B, y = (i / B) % ny, z = i / P;
        uint32_t want[3], nwant = 0;
        if (lower)
        {
            if (z > 0) want[nwant++] = i - P;
            if (y > 0) want[nwant++] = i - B;
            if (x > 0) want[nwant++] = i - 1;
        }
        else
        {
            if (x + 1 < B) want[nwant++] = i + 1;
            if (y + 1 < ny) want[nwant++] = i + B;
            if (z + 1 < nz) want[nwant++] = i + P;
        }
        uint32_t got = 0;
        for (uint32_t e = rp[i]; e < rp[i + 1]; ++e)
        {
            const uint32_t j = ci[e];
            if (j == i) continue;
            if (got >= nwant || j != want[got]) return false;
            ++got;
        }
        if (got != nwant) return false;
    }
    return true;
}

// {B, ny, nz} of a lower triangle with the 7-point grid pattern, else zeros:
// B is the first row with an entry farther than one column back, B ny the
// first with an entry farther than B back.
inline void grid7_dims(uint32_t n, const uint32_t* rp, const uint32_t* ci, uint32_t* dims)
{
    dims[0] = dims[1] = dims[2] = 0;
    uint32_t B = 0, P = 0;
    for (uint32_t i = 0; i < n && !P; ++i)
        for (uint32_t e = rp[i]; e < rp[i + 1]; ++e)
        {
            const uint32_t j = ci[e];
            if (j >= i) continue;
            if (!B && i - j > 1) B = i - j;
            else if (B && i - j > B) P = i - j;
        }
    if (!B || !P || P % B || n % P) return;
    if (!grid7_triangle(n, rp, ci, B, P / B, true)) return;
    dims[0] = B;
    dims[1] = P / B;
    dims[2] = n / P;
}

}  // namespace b2s
