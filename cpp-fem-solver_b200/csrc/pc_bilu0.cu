// Block ILU(0) on BAIJ matrices (make_block_ilu0_preconditioner,
// blockMatrix.hpp:455-623).
//
// Setup: the block pattern is split into L (J < I) and U (J >= I), the level
// sets of L's dependency DAG are computed, and the factor runs one launch per
// level with one warp per block row, repeating the reference's block
// arithmetic exactly (left sum L_IJ U_JK found by binary search, right
// multiplication by inv(U_KK), update of row I's U blocks, Gauss-Jordan
// inverse of the diagonal block) -- bit-equal factors.
// Apply: block forward substitution and block back substitution times the
// cached inverse, in FP64 or FP32: chunked (default, trsv_chunk.cuh), per
// level or sync-free.
#include "block_ops.cuh"
#include "trisolve.cuh"
#include "trsv_chunk.cuh"

#include <exception>
#include <thread>

namespace b2s {

namespace {

struct BCsr
{
    uint32_t nb = 0, nnzb = 0;
    DBuf<uint32_t> rp, ci;
    DBuf<double> v;
    DBuf<float> v32;
};

__global__ void k_bsplit_count(uint32_t nb, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci, int upper,
                               uint32_t* __restrict__ cnt)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
    {
        uint32_t c = 0;
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p) c += upper ? (ci[p] >= i) : (ci[p] < i);
        cnt[i] = c;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt[nb] = 0;
}

__global__ void k_bsplit_fill(uint32_t nb, int bv, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                              const double* __restrict__ v, int upper, const uint32_t* __restrict__ orp,
                              uint32_t* __restrict__ oci, double* __restrict__ ov, uint32_t* __restrict__ udiag,
                              int* missing)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
    {
        uint32_t d = orp[i];
        bool has = false;
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
        {
            const uint32_t j = ci[p];
            if (upper ? (j < i) : (j >= i)) continue;
            if (upper && j == i)
            {
                udiag[i] = d;
                has = true;
            }
            oci[d] = j;
            for (int k = 0; k < bv; ++k) ov[(size_t)d * bv + k] = v[(size_t)p * bv + k];
            ++d;
        }
        if (upper && !has) atomicMin(missing, (int)i);
    }
}

__device__ __forceinline__ uint32_t bfind(const uint32_t* rp, const uint32_t* ci, uint32_t row, uint32_t col)
{
    uint32_t lo = rp[row], hi = rp[row + 1];
    while (lo < hi)
    {
        const uint32_t mid = lo + (hi - lo) / 2;
        const uint32_t c = ci[mid];
        if (c == col) return mid;
        if (c < col)
            lo = mid + 1;
        else
            hi = mid;
    }
    return 0xFFFFFFFFu;
}

// Block row I of the factor (blockMatrix.hpp:528-575), one warp per block
// row of the level.  Lane e < BS*BS owns entry
// (e / BS, e % BS) of the block L_IK being formed and accumulates it in the
// reference's order (left products L_IJ U_JK by ascending J, then the right
// multiplication by inv(U_KK)), so every entry is rounded exactly as in the
// one-thread form.  The row update spreads row I's U blocks over the lanes:
// each lane finds its block's column in row K by binary search and applies
// the block product, which the reference applies in the same per-block
// arithmetic.  Rows with at most kBiluPairRows L blocks look up all their
// U_JK positions up front, in parallel, into shared memory.
constexpr uint32_t kBiluPairRows = 32;

template <int BS>
__global__ void __launch_bounds__(kThreads) k_bilu0_level_warp(const uint32_t* __restrict__ rows, uint32_t count,
                                                               const uint32_t* __restrict__ Lrp,
                                                               const uint32_t* __restrict__ Lci, double* Lv,
                                                               const uint32_t* __restrict__ Urp,
                                                               const uint32_t* __restrict__ Uci, double* Uv,
                                                               const uint32_t* __restrict__ Udiag, double* inv,
                                                               int* singular)
{
    constexpr int BV = BS * BS;
    constexpr uint32_t NONE = 0xFFFFFFFFu;
    __shared__ uint32_t spair[kThreads / 32][kBiluPairRows * (kBiluPairRows - 1) / 2];
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= count) return;  // the whole warp
    uint32_t* pair = spair[threadIdx.x >> 5];
    const uint32_t I = rows[w];
    const uint32_t Ls = Lrp[I], Le = Lrp[I + 1], Us = Urp[I], Ue = Urp[I + 1];
    const uint32_t m = Le - Ls;
    const bool cached = m <= kBiluPairRows;
    if (cached)
        for (uint32_t a = 1; a < m; ++a)
            for (uint32_t b = lane; b < a; b += 32) pair[a * (a - 1) / 2 + b] = bfind(Urp, Uci, Lci[Ls + b], Lci[Ls + a]);
    __syncwarp();
    const uint32_t e = lane < (uint32_t)BV ? lane : 0u;  // lanes past BV shadow entry 0
    const int r = (int)e / BS, c = (int)e % BS;
    for (uint32_t a = 0; a < m; ++a)
    {
        const uint32_t pL = Ls + a, K = Lci[pL];
        double lik = Lv[(size_t)pL * BV + e];
        for (uint32_t b = 0; b < a; ++b)
        {
            const uint32_t pJK = cached ? pair[a * (a - 1) / 2 + b] : bfind(Urp, Uci, Lci[Ls + b], K);
            if (pJK == NONE) continue;
            const double* A = Lv + (size_t)(Ls + b) * BV + r * BS;
            const double* B = Uv + (size_t)pJK * BV + c;
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < BS; ++k) s += A[k] * B[k * BS];
            lik -= s;
        }
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < BS; ++k) s += __shfl_sync(0xffffffffu, lik, r * BS + k) * inv[(size_t)K * BV + k * BS + c];
        lik = s;
        if (lane < (uint32_t)BV) Lv[(size_t)pL * BV + e] = lik;
        double Lb[BV];
#pragma unroll
        for (int q = 0; q < BV; ++q) Lb[q] = __shfl_sync(0xffffffffu, lik, q);
        for (uint32_t pi = Us + lane; pi < Ue; pi += 32)
        {
            const uint32_t pk = bfind(Urp, Uci, K, Uci[pi]);
            if (pk != NONE) blk_mma<BS>(Lb, &Uv[(size_t)pk * BV], &Uv[(size_t)pi * BV]);
        }
        __syncwarp();  // L_IK and row I's U blocks are visible to every lane
    }
    if (lane == 0)
    {
        double Mi[BV];
        if (!blk_inv<BS>(&Uv[(size_t)Udiag[I] * BV], Mi))
        {
            atomicMin(singular, (int)I);
            for (int k = 0; k < BV; ++k) Mi[k] = 0.0;
        }
        for (int k = 0; k < BV; ++k) inv[(size_t)I * BV + k] = Mi[k];
    }
}

// block forward / backward substitution rows (blockMatrix.hpp:584-621)
template <int BS, bool LOWER, typename VT, typename XT, typename RT>
struct BTrsvOp
{
    const uint32_t *rp, *ci;
    const VT* v;
    const VT* inv;  // backward only
    const RT* rhs;
    XT* x;
    double* out64;
    __device__ bool ready(uint32_t row, const uint32_t* flags, uint32_t epoch) const
    {
        return deps_ready<LOWER>(row, rp, ci, flags, epoch);
    }
    template <bool SYNCFREE>
    __device__ __forceinline__ void row_compute(uint32_t I) const
    {
        constexpr int BV = BS * BS;
        XT t[BS];
#pragma unroll
        for (int c = 0; c < BS; ++c) t[c] = (XT)rhs[(size_t)I * BS + c];
        for (uint32_t p = __ldg(&rp[I]); p < __ldg(&rp[I + 1]); ++p)
        {
            const uint32_t J = __ldg(&ci[p]);
            if (LOWER ? !(J < I) : !(J > I)) continue;
            XT xJ[BS];
#pragma unroll
            for (int c = 0; c < BS; ++c) xJ[c] = SYNCFREE ? __ldcg(&x[(size_t)J * BS + c]) : x[(size_t)J * BS + c];
#pragma unroll
            for (int r = 0; r < BS; ++r)
            {
                XT s = 0;
#pragma unroll
                for (int c = 0; c < BS; ++c) s += (XT)__ldg(&v[(size_t)p * BV + r * BS + c]) * xJ[c];
                t[r] -= s;
            }
        }
        if (LOWER)
        {
#pragma unroll
            for (int c = 0; c < BS; ++c)
            {
                x[(size_t)I * BS + c] = t[c];
                if (out64) out64[(size_t)I * BS + c] = (double)t[c];
            }
        }
        else
        {
#pragma unroll
            for (int r = 0; r < BS; ++r)
            {
                XT s = 0;
#pragma unroll
                for (int c = 0; c < BS; ++c) s += (XT)__ldg(&inv[(size_t)I * BV + r * BS + c]) * t[c];
                x[(size_t)I * BS + r] = s;
                if (out64) out64[(size_t)I * BS + r] = (double)s;
            }
        }
    }
    __device__ void compute(uint32_t row) const { row_compute<true>(row); }
};

__global__ void k_to32(const double* __restrict__ a, float* __restrict__ b, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

struct PcBILU0 final : PcImpl
{
    int bs = 3;
    uint32_t nb = 0;
    int mode = B2S_TRSV_SYNCFREE;
    bool fp32 = false;
    BCsr L, U;
    DBuf<uint32_t> udiag;
    DBuf<double> inv, y;
    DBuf<float> inv32, y32, z32;
    LevelSchedule sl, su;
    SyncFree sfl, sfu;
    ChunkSchedule csl, csu;
    bool chunks = false;

    template <int BS>
    void apply_t(b2s_ctx* ctx, const double* r, double* z, const int* done)
    {
        if (chunks)
        {
            if (!fp32)
            {
                csl.run_block<true, BS, double, double, double>(ctx, L.v.p, nullptr, r, y.p, nullptr, done);
                csu.run_block<false, BS, double, double, double>(ctx, U.v.p, inv.p, y.p, z, nullptr, done);
            }
            else
            {
                csl.run_block<true, BS, float, float, double>(ctx, L.v32.p, nullptr, r, y32.p, nullptr, done);
                csu.run_block<false, BS, float, float, float>(ctx, U.v32.p, inv32.p, y32.p, z32.p, z, done);
            }
            return;
        }
        if (!fp32)
        {
            run_schedule(ctx, mode, sl, sfl,
                         BTrsvOp<BS, true, double, double, double>{L.rp.p, L.ci.p, L.v.p, nullptr, r, y.p, nullptr}, done);
            run_schedule(ctx, mode, su, sfu,
                         BTrsvOp<BS, false, double, double, double>{U.rp.p, U.ci.p, U.v.p, inv.p, y.p, z, nullptr}, done);
        }
        else
        {
            run_schedule(ctx, mode, sl, sfl,
                         BTrsvOp<BS, true, float, float, double>{L.rp.p, L.ci.p, L.v32.p, nullptr, r, y32.p, nullptr},
                         done);
            run_schedule(ctx, mode, su, sfu,
                         BTrsvOp<BS, false, float, float, float>{U.rp.p, U.ci.p, U.v32.p, inv32.p, y32.p, z32.p, z},
                         done);
        }
    }

    void apply(b2s_ctx* ctx, const double* r, double* z, const int* done) override
    {
        switch (bs)
        {
            case 1: apply_t<1>(ctx, r, z, done); break;
            case 2: apply_t<2>(ctx, r, z, done); break;
            case 3: apply_t<3>(ctx, r, z, done); break;
            case 4: apply_t<4>(ctx, r, z, done); break;
        }
    }

    void export_data(b2s_ctx* ctx, const std::string& what, uint64_t* sizes, uint32_t* rp, uint32_t* ci,
                     double* v) override
    {
        const size_t bv = (size_t)bs * bs;
        const BCsr* m = what == "bilu0.L" ? &L : what == "bilu0.U" ? &U : nullptr;
        if (m)
        {
            sizes[0] = (uint64_t)nb + 1;
            sizes[1] = m->nnzb;
            sizes[2] = (uint64_t)m->nnzb * bv;
            if (rp) d2h(ctx, rp, m->rp.p, (nb + 1) * sizeof(uint32_t));
            if (ci) d2h(ctx, ci, m->ci.p, m->nnzb * sizeof(uint32_t));
            if (v) d2h(ctx, v, m->v.p, m->nnzb * bv * sizeof(double));
            sync(ctx);
            return;
        }
        if (what == "bilu0.inv")
        {
            sizes[0] = 0;
            sizes[1] = nb;
            sizes[2] = (uint64_t)nb * bv;
            if (ci) d2h(ctx, ci, udiag.p, nb * sizeof(uint32_t));
            if (v) d2h(ctx, v, inv.p, nb * bv * sizeof(double));
            sync(ctx);
            return;
        }
        PcImpl::export_data(ctx, what, sizes, rp, ci, v);
    }
};

template <int BS>
void bilu0_factor(b2s_ctx* ctx, PcBILU0& pc, int* singular)
{
    for (uint32_t l = 0; l < pc.sl.nlev; ++l)
    {
        const uint32_t a = pc.sl.h_ptr[l], cnt = pc.sl.h_ptr[l + 1] - a;
        B2S_LAUNCH(ctx, k_bilu0_level_warp<BS>, (cnt + kThreads / 32 - 1) / (kThreads / 32), kThreads, 0,
                   pc.sl.rows.p + a, cnt, pc.L.rp.p, pc.L.ci.p, pc.L.v.p, pc.U.rp.p, pc.U.ci.p, pc.U.v.p,
                   pc.udiag.p, pc.inv.p, singular);
    }
}

}  // namespace

std::unique_ptr<PcImpl> make_pc_bilu0(b2s_ctx* ctx, const BaijDev& A, const b2s_pc_opts& o)
{
    need(A.nbr == A.nbc, B2S_SHAPE, "Block-ILU(0) needs a square block matrix");
    auto pc = std::make_unique<PcBILU0>();
    const uint32_t nb = A.nbr;
    const int bs = A.bs, bv = bs * bs;
    pc->bs = bs;
    pc->nb = nb;
    need(o.trsv != B2S_TRSV_JACOBI, B2S_UNSUPPORTED, "block ILU(0): Jacobi-sweep triangular solves are not provided");
    pc->mode = o.trsv == B2S_TRSV_AUTO ? B2S_TRSV_CHUNK : o.trsv;
    pc->fp32 = o.precision != B2S_FP64;
    pc->udiag.alloc(nb ? nb : 1);
    DBuf<int> flags(2);
    const int big[2] = {0x7fffffff, 0x7fffffff};
    h2d(ctx, flags.p, big, sizeof(big));
    for (int upper = 0; upper < 2; ++upper)
    {
        BCsr& M = upper ? pc->U : pc->L;
        DBuf<uint32_t> cnt(nb + 1);
        B2S_LAUNCH(ctx, k_bsplit_count, stream_grid(ctx, nb), kThreads, 0, nb, A.rp.p, A.ci.p, upper, cnt.p);
        M.nb = nb;
        M.rp.alloc(nb + 1);
        M.nnzb = exclusive_scan(ctx, cnt.p, M.rp.p, nb);
        M.ci.alloc(M.nnzb ? M.nnzb : 1);
        M.v.alloc(M.nnzb ? (size_t)M.nnzb * bv : 1);
        B2S_LAUNCH(ctx, k_bsplit_fill, stream_grid(ctx, nb), kThreads, 0, nb, bv, A.rp.p, A.ci.p, A.v.p, upper, M.rp.p,
                   M.ci.p, M.v.p, pc->udiag.p, flags.p);
    }
    int h[2];
    d2h(ctx, h, flags.p, sizeof(h));
    sync(ctx);
    if (h[0] != big[0])
        fail(B2S_MISSING_DIAG, "Block-ILU(0) failed: block row " + std::to_string(h[0]) + " has no diagonal block");
    // host analysis: block levels of L here (for the factorisation); the chunk
    // plans on a host thread while the device factorises
    const uint32_t vs = pc->fp32 ? 4 : 8;
    std::vector<uint32_t> lrp(nb + 1), lci(pc->L.nnzb ? pc->L.nnzb : 1), urp(nb + 1), uci(pc->U.nnzb ? pc->U.nnzb : 1);
    d2h(ctx, lrp.data(), pc->L.rp.p, (nb + 1) * sizeof(uint32_t));
    d2h(ctx, lci.data(), pc->L.ci.p, pc->L.nnzb * sizeof(uint32_t));
    d2h(ctx, urp.data(), pc->U.rp.p, (nb + 1) * sizeof(uint32_t));
    d2h(ctx, uci.data(), pc->U.ci.p, pc->U.nnzb * sizeof(uint32_t));
    sync(ctx);
    std::vector<uint32_t> llev, ulev;
    compute_levels(nb, lrp.data(), lci.data(), true, llev);
    if (nb) pc->sl.build_host(ctx, llev);
    const bool chunked = pc->mode == B2S_TRSV_CHUNK && nb;
    ChunkPlan lplan, uplan;
    std::exception_ptr perr;
    std::thread th([&] {
        try
        {
            // the two triangles' plans run side by side
            plan_parallel(2, 2, [&](uint32_t side, unsigned) {
                if (side == 0)
                {
                    if (chunked)
                        lplan = plan_chunks(nb, lrp.data(), lci.data(), true, 0, vs, vs, 8, kChunkSmemBudget,
                                            (uint32_t)bs, &llev);
                    return;
                }
                compute_levels(nb, urp.data(), uci.data(), false, ulev);
                if (chunked)
                    uplan = plan_chunks(nb, urp.data(), uci.data(), false, (uint32_t)bv, vs, vs, 8, kChunkSmemBudget,
                                        (uint32_t)bs, &ulev);
            });
        }
        catch (...)
        {
            perr = std::current_exception();
        }
    });
    struct Join
    {
        std::thread& t;
        ~Join()
        {
            if (t.joinable()) t.join();
        }
    } join{th};
    pc->inv.alloc((size_t)nb * bv + 1);
    switch (bs)
    {
        case 1: bilu0_factor<1>(ctx, *pc, flags.p + 1); break;
        case 2: bilu0_factor<2>(ctx, *pc, flags.p + 1); break;
        case 3: bilu0_factor<3>(ctx, *pc, flags.p + 1); break;
        case 4: bilu0_factor<4>(ctx, *pc, flags.p + 1); break;
    }
    d2h(ctx, h, flags.p, sizeof(h));
    sync(ctx);
    if (h[1] != big[1])
        fail(B2S_SINGULAR_BLOCK, "Block-ILU(0) breakdown: diagonal block " + std::to_string(h[1]) + " is singular");
    th.join();
    if (perr) std::rethrow_exception(perr);
    if (chunked) pc->chunks = pc->csl.load(ctx, lplan, vs) && pc->csu.load(ctx, uplan, vs);
    if (!pc->chunks)
    {
        if (pc->mode == B2S_TRSV_CHUNK) pc->mode = B2S_TRSV_SYNCFREE;
        if (nb) pc->su.build_host(ctx, ulev);
        pc->sfl.init(ctx, nb);
        pc->sfu.init(ctx, nb);
    }
    pc->y.alloc((size_t)nb * bs + 1);
    if (pc->fp32)
    {
        auto cvt = [&](const DBuf<double>& a, DBuf<float>& b, uint64_t n) {
            b.alloc(n ? n : 1);
            if (n) B2S_LAUNCH(ctx, k_to32, stream_grid(ctx, n), kThreads, 0, a.p, b.p, n);
        };
        cvt(pc->L.v, pc->L.v32, (uint64_t)pc->L.nnzb * bv);
        cvt(pc->U.v, pc->U.v32, (uint64_t)pc->U.nnzb * bv);
        cvt(pc->inv, pc->inv32, (uint64_t)nb * bv);
        pc->y32.alloc((size_t)nb * bs + 1);
        pc->z32.alloc((size_t)nb * bs + 1);
    }
    if (pc->chunks)
    {
        if (pc->fp32)
        {
            pc->csl.pack<float>(ctx, pc->L.v32.p, nullptr);
            pc->csu.pack<float>(ctx, pc->U.v32.p, pc->inv32.p);
        }
        else
        {
            pc->csl.pack<double>(ctx, pc->L.v.p, nullptr);
            pc->csu.pack<double>(ctx, pc->U.v.p, pc->inv.p);
        }
    }
    sync(ctx);
    return pc;
}

}  // namespace b2s
