// BAIJ (block CSR) handles, block matvec and block Jacobi.
//   BlockMatrix storage / cache_diag / matvec: blockMatrix.hpp:139-234
//   BlockMatrix::gmres "blockjacobi":         blockMatrix.hpp:714-733
//
// The block matvec kernels are in baij_mv.cuh.
#include "baij_mv.cuh"

namespace b2s {

template <typename VT>
static void baij_matvec_t(b2s_ctx* ctx, const BaijDev& A, const VT* v, const double* x, double* y, const int* done)
{
    switch (A.bs)
    {
        case 1: baij_mv<1>(ctx, A, v, x, EpiStoreY{y}, done); break;
        case 2: baij_mv<2>(ctx, A, v, x, EpiStoreY{y}, done); break;
        case 3: baij_mv<3>(ctx, A, v, x, EpiStoreY{y}, done); break;
        case 4: baij_mv<4>(ctx, A, v, x, EpiStoreY{y}, done); break;
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

void baij_partition(b2s_ctx* ctx, BaijDev& M, const uint32_t* h_rp)
{
    M.nblk = 0;
    if (M.bs != 1 || M.nbr == 0 || M.nnzb < (uint64_t)kBaijStagedMinRow * M.nbr) return;
    std::vector<uint32_t> blk;
    build_row_blocks(h_rp, M.nbr, 1, kThreads, kBaijStagedCap, blk);
    M.nblk = (uint32_t)blk.size() - 1;
    M.blk_row = upload(ctx, blk.data(), blk.size());
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
        std::vector<uint32_t> diag(nbr, 0xFFFFFFFFu);
        for (uint32_t i = 0; i < nbr; ++i)
            for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
            {
                need(col_idx[k] < nbc, B2S_INVALID_ARG, "block column index out of range");
                need(k == row_ptr[i] || col_idx[k] > col_idx[k - 1], B2S_INVALID_ARG,
                     "block columns must be strictly ascending within a row");
                if (col_idx[k] == i && diag[i] == 0xFFFFFFFFu) diag[i] = k;
            }
        d.rp = upload(ctx, row_ptr, (size_t)nbr + 1);
        d.ci = upload(ctx, col_idx, nnzb);
        d.v = upload(ctx, values, (size_t)nnzb * bs * bs);
        d.diag_ptr = upload(ctx, diag.data(), nbr);
        baij_partition(ctx, d, row_ptr);
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
