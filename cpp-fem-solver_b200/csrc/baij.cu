// BAIJ (block CSR) handles, block matvec and block Jacobi.
//   BlockMatrix storage / cache_diag / matvec: blockMatrix.hpp:139-234
//   BlockMatrix::gmres "blockjacobi":         blockMatrix.hpp:714-733
//
// Block matvec (bs >= 2): a warp owns 32/bs consecutive block rows (one lane
// per output component) and walks their blocks min(32, 256/bs^2) at a time.  The
// lanes stream the blocks' values into the warp's shared memory (coalesced,
// no L1 allocation), lane b gathers x_J of block b and forms the block's bs
// row dots with the reference's association (blk_row_dot), and the lane of
// output component (I, r) adds the dots of row I in block order -- the
// reference's order, so y is bit-exact.  No CTA-wide barrier.  bs = 1 (the
// scalar AMG levels, whose coarse rows are long) keeps the staged kernel.
#include "block_ops.cuh"
#include "spmv_staged.cuh"

namespace b2s {

template <int BS>
struct BaijCap
{
    static constexpr int value = BS == 1 ? 3072 : BS == 2 ? 1024 : BS == 3 ? 512 : 256;
};

constexpr int kBaijCtasPerSm = 4;

// VT: stored value type (double, or float for the FP32 copies of the AMG
// hierarchy); products and sums are FP64 either way.
template <int BS, typename VT>
__global__ void __launch_bounds__(kThreads, kBaijCtasPerSm)
    k_baij_warp(uint32_t nbr, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                const VT* __restrict__ v, const double* __restrict__ x, double* __restrict__ y, const int* done)
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
        if (out) y[(size_t)I * BS + r] = acc;
    }
}

template <int BS, typename VT>
static void launch_baij(b2s_ctx* ctx, const BaijDev& A, const VT* v, const double* x, double* y, const int* done)
{
    constexpr int GR = 32 / BS;
    const uint32_t groups = (A.nbr + GR - 1) / GR;
    const uint32_t ctas = (groups + kThreads / 32 - 1) / (kThreads / 32);
    const uint32_t cap = (uint32_t)ctx->sm_count * kBaijCtasPerSm;
    B2S_LAUNCH(ctx, (k_baij_warp<BS, VT>), ctas < cap ? ctas : cap, kThreads, 0, A.nbr, A.rp.p, A.ci.p, v, x, y, done);
}

__device__ __forceinline__ void stage_vals(double* s, const double* g, uint32_t cnt) { stage_f64(s, g, cnt); }

__device__ __forceinline__ void stage_vals(float* s, const float* g, uint32_t cnt)
{
    for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) s[i] = __ldg(&g[i]);
}

// 1x1 blocks (the AMG hierarchies' operators, rows of 7 to 100+ entries): a CTA
// stages a contiguous block range in shared memory and one thread per row sums it.
template <int BS, typename VT>
__global__ void __launch_bounds__(kThreads) k_baij_staged(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                                          const VT* __restrict__ v,
                                                          const uint32_t* __restrict__ blk_row,
                                                          const double* __restrict__ x, double* __restrict__ y,
                                                          const int* done)
{
    if (done && *done) return;
    constexpr int BV = BS * BS, CAP = BaijCap<BS>::value;
    __shared__ VT sv[CAP * BV];
    __shared__ uint32_t sc[CAP];
    const uint32_t r0 = blk_row[blockIdx.x], r1 = blk_row[blockIdx.x + 1];
    const uint32_t p0 = __ldg(&rp[r0]), p1 = __ldg(&rp[r1]);
    const uint32_t cnt = p1 - p0;
    const uint32_t nthr = (r1 - r0) * BS;
    if (cnt <= (uint32_t)CAP)
    {
        stage_vals(sv, v + (size_t)p0 * BV, cnt * BV);
        stage_u32(sc, ci + p0, cnt);
        __syncthreads();
        for (uint32_t t = threadIdx.x; t < nthr; t += blockDim.x)
        {
            const uint32_t br = r0 + t / BS;
            const int r = (int)(t % BS);
            const uint32_t a = __ldg(&rp[br]) - p0, b = __ldg(&rp[br + 1]) - p0;
            double yr = 0.0;
            for (uint32_t k = a; k < b; ++k)
            {
                const double* xj = x + (size_t)sc[k] * BS;
                double xv[BS], brow[BS];
#pragma unroll
                for (int c = 0; c < BS; ++c)
                {
                    xv[c] = __ldg(&xj[c]);
                    brow[c] = (double)sv[(size_t)k * BV + r * BS + c];
                }
                yr += blk_row_dot<BS>(brow, xv);
            }
            y[(size_t)br * BS + r] = yr;
        }
    }
    else
    {
        for (uint32_t t = threadIdx.x; t < nthr; t += blockDim.x)
        {
            const uint32_t br = r0 + t / BS;
            const int r = (int)(t % BS);
            double yr = 0.0;
            for (uint32_t k = __ldg(&rp[br]); k < __ldg(&rp[br + 1]); ++k)
            {
                const double* xj = x + (size_t)__ldg(&ci[k]) * BS;
                double xv[BS], brow[BS];
#pragma unroll
                for (int c = 0; c < BS; ++c)
                {
                    xv[c] = __ldg(&xj[c]);
                    brow[c] = (double)__ldg(&v[(size_t)k * BV + r * BS + c]);
                }
                yr += blk_row_dot<BS>(brow, xv);
            }
            y[(size_t)br * BS + r] = yr;
        }
    }
}


template <typename VT>
static void baij_matvec_t(b2s_ctx* ctx, const BaijDev& A, const VT* v, const double* x, double* y, const int* done)
{
    if (A.nbr == 0) return;
    switch (A.bs)
    {
        case 1:
            B2S_LAUNCH(ctx, (k_baij_staged<1, VT>), A.nblk, kThreads, 0, A.rp.p, A.ci.p, v, A.blk_row.p, x, y, done);
            break;
        case 2: launch_baij<2, VT>(ctx, A, v, x, y, done); break;
        case 3: launch_baij<3, VT>(ctx, A, v, x, y, done); break;
        case 4: launch_baij<4, VT>(ctx, A, v, x, y, done); break;
        default: fail(B2S_UNSUPPORTED, "block size must be 1..4");
    }
}

void baij_matvec(b2s_ctx* ctx, const BaijDev& A, const double* x, double* y, const int* done)
{
    baij_matvec_t<double>(ctx, A, A.v.p, x, y, done);
}

void baij_matvec_f32(b2s_ctx* ctx, const BaijDev& A, const float* v32, const double* x, double* y, const int* done)
{
    baij_matvec_t<float>(ctx, A, v32, x, y, done);
}

static uint32_t baij_cap(int bs)
{
    switch (bs)
    {
        case 1: return BaijCap<1>::value;
        case 2: return BaijCap<2>::value;
        case 3: return BaijCap<3>::value;
        default: return BaijCap<4>::value;
    }
}

// ------------------------------------------------------------ block Jacobi

template <int BS>
__global__ void k_bjacobi_setup(uint32_t nb, const double* __restrict__ v, const uint32_t* __restrict__ dptr,
                                double* __restrict__ inv, int* bad)
{
    constexpr int BV = BS * BS;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
    {
        double M[BV], Mi[BV];
        const uint32_t p = dptr[i];
        if (p == 0xFFFFFFFFu)
        {
            atomicMin(bad, (int)i);
            continue;
        }
        for (int k = 0; k < BV; ++k) M[k] = v[(size_t)p * BV + k];
        if (!blk_inv<BS>(M, Mi))
            for (int k = 0; k < BV; ++k) Mi[k] = 0.0;
        for (int k = 0; k < BV; ++k) inv[(size_t)i * BV + k] = Mi[k];
    }
}

template <int BS>
__global__ void k_bjacobi_apply(uint32_t nb, const double* __restrict__ inv, const double* __restrict__ r,
                                double* __restrict__ z, const int* done)
{
    if (done && *done) return;
    constexpr int BV = BS * BS;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
    {
        double M[BV], t[BS], o[BS];
        for (int k = 0; k < BV; ++k) M[k] = inv[(size_t)i * BV + k];
        for (int c = 0; c < BS; ++c) t[c] = r[(size_t)i * BS + c];
        blk_mv<BS>(M, t, o);
        for (int c = 0; c < BS; ++c) z[(size_t)i * BS + c] = o[c];
    }
}

namespace {

struct PcBJacobi final : PcImpl
{
    int bs;
    uint32_t nb;
    DBuf<double> inv;
    void apply(b2s_ctx* ctx, const double* r, double* z, const int* done) override
    {
        const unsigned g = stream_grid(ctx, nb);
        switch (bs)
        {
            case 1: B2S_LAUNCH(ctx, k_bjacobi_apply<1>, g, kThreads, 0, nb, inv.p, r, z, done); break;
            case 2: B2S_LAUNCH(ctx, k_bjacobi_apply<2>, g, kThreads, 0, nb, inv.p, r, z, done); break;
            case 3: B2S_LAUNCH(ctx, k_bjacobi_apply<3>, g, kThreads, 0, nb, inv.p, r, z, done); break;
            case 4: B2S_LAUNCH(ctx, k_bjacobi_apply<4>, g, kThreads, 0, nb, inv.p, r, z, done); break;
        }
    }
};

}  // namespace

std::unique_ptr<PcImpl> make_pc_bjacobi(b2s_ctx* ctx, const BaijDev& A)
{
    auto pc = std::make_unique<PcBJacobi>();
    pc->bs = A.bs;
    pc->nb = A.nbr;
    pc->inv.alloc((size_t)A.nbr * A.bs * A.bs);
    DBuf<int> bad(1);
    const int big = 0x7fffffff;
    h2d(ctx, bad.p, &big, sizeof(int));
    const unsigned g = stream_grid(ctx, A.nbr);
    switch (A.bs)
    {
        case 1: B2S_LAUNCH(ctx, k_bjacobi_setup<1>, g, kThreads, 0, A.nbr, A.v.p, A.diag_ptr.p, pc->inv.p, bad.p); break;
        case 2: B2S_LAUNCH(ctx, k_bjacobi_setup<2>, g, kThreads, 0, A.nbr, A.v.p, A.diag_ptr.p, pc->inv.p, bad.p); break;
        case 3: B2S_LAUNCH(ctx, k_bjacobi_setup<3>, g, kThreads, 0, A.nbr, A.v.p, A.diag_ptr.p, pc->inv.p, bad.p); break;
        case 4: B2S_LAUNCH(ctx, k_bjacobi_setup<4>, g, kThreads, 0, A.nbr, A.v.p, A.diag_ptr.p, pc->inv.p, bad.p); break;
    }
    int h = 0;
    d2h(ctx, &h, bad.p, sizeof(int));
    sync(ctx);
    if (h != big) fail(B2S_MISSING_DIAG, "block Jacobi: block row " + std::to_string(h) + " has no diagonal block");
    return pc;
}

}  // namespace b2s

using namespace b2s;

extern "C" {

b2s_status b2s_baij_create(b2s_ctx* ctx, int bs, uint32_t nbr, uint32_t nbc, const uint32_t* row_ptr,
                           const uint32_t* col_idx, const double* values, b2s_baij** out)
{
    if (!ctx || !out || !row_ptr) return B2S_INVALID_ARG;
    if (bs < 1 || bs > 4) return B2S_UNSUPPORTED;
    *out = nullptr;
    b2s_baij* A = new b2s_baij();
    A->ctx = ctx;
    b2s_status st = guarded(ctx, [&] {
        B2S_CUDA(cudaSetDevice(ctx->device));
        need(row_ptr[0] == 0, B2S_INVALID_ARG, "row_ptr[0] must be 0");
        for (uint32_t i = 0; i < nbr; ++i) need(row_ptr[i + 1] >= row_ptr[i], B2S_INVALID_ARG, "row_ptr must be non-decreasing");
        const uint32_t nnzb = row_ptr[nbr];
        need(nnzb == 0 || (col_idx && values), B2S_INVALID_ARG, "null col_idx / values");
        BaijDev& d = A->d;
        d.bs = bs;
        d.nbr = nbr;
        d.nbc = nbc;
        d.nnzb = nnzb;
        d.h_rp.assign(row_ptr, row_ptr + nbr + 1);
        d.h_ci.assign(col_idx, col_idx + nnzb);
        d.h_v.assign(values, values + (size_t)nnzb * bs * bs);
        d.h_diag.assign(nbr, 0xFFFFFFFFu);
        for (uint32_t i = 0; i < nbr; ++i)
            for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
            {
                need(col_idx[k] < nbc, B2S_INVALID_ARG, "block column index out of range");
                need(k == row_ptr[i] || col_idx[k] > col_idx[k - 1], B2S_INVALID_ARG,
                     "block columns must be strictly ascending within a row");
                if (col_idx[k] == i && d.h_diag[i] == 0xFFFFFFFFu) d.h_diag[i] = k;
            }
        d.rp = upload(ctx, row_ptr, (size_t)nbr + 1);
        d.ci = upload(ctx, col_idx, nnzb);
        d.v = upload(ctx, values, (size_t)nnzb * bs * bs);
        d.diag_ptr = upload(ctx, d.h_diag.data(), nbr);
        std::vector<uint32_t> blk;
        build_row_blocks(row_ptr, nbr, 1, (uint32_t)(kThreads / bs), baij_cap(bs), blk);
        d.nblk = (uint32_t)blk.size() - 1;
        d.blk_row = upload(ctx, blk.data(), blk.size());
        sync(ctx);
    });
    if (st != B2S_OK)
    {
        delete A;
        return st;
    }
    *out = A;
    return B2S_OK;
}

b2s_status b2s_baij_destroy(b2s_baij* A)
{
    if (!A) return B2S_INVALID_ARG;
    cudaSetDevice(A->ctx->device);
    delete A;
    return B2S_OK;
}

b2s_status b2s_baij_info(const b2s_baij* A, int* bs, uint32_t* nbr, uint32_t* nbc, uint32_t* nnzb)
{
    if (!A) return B2S_INVALID_ARG;
    if (bs) *bs = A->d.bs;
    if (nbr) *nbr = A->d.nbr;
    if (nbc) *nbc = A->d.nbc;
    if (nnzb) *nnzb = A->d.nnzb;
    return B2S_OK;
}

b2s_status b2s_baij_matvec_device(b2s_ctx* ctx, const b2s_baij* A, const double* d_x, double* d_y)
{
    if (!ctx || !A) return B2S_INVALID_ARG;
    return guarded(ctx, [&] { baij_matvec(ctx, A->d, d_x, d_y); });
}

b2s_status b2s_baij_matvec(b2s_ctx* ctx, const b2s_baij* A, const double* x, double* y)
{
    if (!ctx || !A) return B2S_INVALID_ARG;
    return guarded(ctx, [&] {
        const size_t nx = (size_t)A->d.nbc * A->d.bs, ny = (size_t)A->d.nbr * A->d.bs;
        need((!nx || x) && (!ny || y), B2S_INVALID_ARG, "null vector");
        DBuf<double> dx(nx), dy(ny);
        h2d(ctx, dx.p, x, dx.bytes());
        baij_matvec(ctx, A->d, dx.p, dy.p);
        d2h(ctx, y, dy.p, dy.bytes());
        sync(ctx);
    });
}

}  // extern "C"
