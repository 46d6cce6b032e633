// Compositions of device preconditioners:
//   * the block-triangular saddle-point (Schur-complement) preconditioner of
//     make_schur_preconditioner (blockMatrix.hpp:637-685), for r = [r_u; r_p]:
//       1  w_u  = A^-1 r_u
//       2  w_p  = B w_u                3  r_p' = w_p - r_p
//       4  z_p  = S^-1 r_p'
//       5  w_bt = B^T z_p              6  r_u' = r_u - w_bt
//       7  z_u  = A^-1 r_u'
//     Every step runs on the device, on the context's stream: A^-1 and S^-1
//     are preconditioners of the same context, steps 2-3 and 5-6 are each one
//     SpMV with the difference formed in its epilogue, and the halves of r and
//     z are addressed in place.  The SpMVs sum each row in column order and
//     the differences are elementwise, so with bit-exact sub-preconditioners
//     an apply equals the reference's composition bit for bit.
//   * a scaled preconditioner z = alpha M^-1 r (the reference's 3-D Stokes
//     test scales its pressure AMG by the velocity diagonal,
//     test_BlockMatrix_schur3d.cpp:150-160).
#include "spmv_staged.cuh"

namespace b2s {

namespace {

// r_p' = B w_u - r_p, per row of B
struct EpiMinusR
{
    static constexpr int NV = 0;
    double* out;
    const double* r;
    __device__ void row(uint32_t i, double s, double*) const { out[i] = s - r[i]; }
    __device__ void last(const double*) const {}
};

// r_u' = r_u - B^T z_p, per row of B^T
struct EpiRMinus
{
    static constexpr int NV = 0;
    double* out;
    const double* r;
    __device__ void row(uint32_t i, double s, double*) const { out[i] = r[i] - s; }
    __device__ void last(const double*) const {}
};

struct PcSchur final : PcImpl
{
    uint64_t nv = 0, np = 0;
    const CsrDev* B = nullptr;
    const CsrDev* Bt = nullptr;
    PcImpl* A = nullptr;
    PcImpl* S = nullptr;  // null: identity
    DBuf<double> wu, rpm, rum;
    void apply(b2s_ctx* ctx, const double* r, double* z, const int* done) override
    {
        const double* ru = r;
        const double* rp = r + nv;
        double* zu = z;
        double* zp = z + nv;
        A->apply(ctx, ru, wu.p, done);                             // 1
        launch_spmv(ctx, *B, wu.p, done, EpiMinusR{rpm.p, rp});     // 2-3
        if (S)
            S->apply(ctx, rpm.p, zp, done);                        // 4
        else
            copy(ctx, zp, rpm.p, np, done);
        launch_spmv(ctx, *Bt, zp, done, EpiRMinus{rum.p, ru});     // 5-6
        A->apply(ctx, rum.p, zu, done);                            // 7
    }
    bool is_host() const override { return A->is_host() || (S && S->is_host()); }
};

__global__ void k_scale(uint64_t n, double alpha, double* __restrict__ z, const int* done)
{
    if (done && *done) return;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        z[i] = alpha * z[i];
}

struct PcScaled final : PcImpl
{
    uint64_t n = 0;
    double alpha = 1.0;
    PcImpl* inner = nullptr;
    void apply(b2s_ctx* ctx, const double* r, double* z, const int* done) override
    {
        inner->apply(ctx, r, z, done);
        if (n) B2S_LAUNCH(ctx, k_scale, stream_grid(ctx, n), kThreads, 0, n, alpha, z, done);
    }
    bool is_host() const override { return inner->is_host(); }
};

}  // namespace

}  // namespace b2s

using namespace b2s;

extern "C" {

b2s_status b2s_pc_create_schur(b2s_ctx* ctx, uint64_t n_vel, uint64_t n_pres, const b2s_csr* B, const b2s_csr* Bt,
                               b2s_pc* A_pc, b2s_pc* S_pc, b2s_pc** out)
{
    if (!ctx || !B || !Bt || !A_pc || !out) return B2S_INVALID_ARG;
    *out = nullptr;
    b2s_pc* pc = new b2s_pc();
    pc->ctx = ctx;
    pc->kind = B2S_PC_SCHUR;
    pc->n = n_vel + n_pres;
    const b2s_status st = guarded(ctx, [&] {
        need(B->d.n == n_pres && B->d.m == n_vel, B2S_SHAPE, "Schur: B must be n_pres x n_vel");
        need(Bt->d.n == n_vel && Bt->d.m == n_pres, B2S_SHAPE, "Schur: B^T must be n_vel x n_pres");
        need(A_pc->n == n_vel, B2S_SHAPE, "Schur: the velocity preconditioner must have n_vel rows");
        need(!S_pc || S_pc->n == n_pres, B2S_SHAPE, "Schur: the pressure preconditioner must have n_pres rows");
        need(A_pc->ctx == ctx && (!S_pc || S_pc->ctx == ctx) && B->ctx == ctx && Bt->ctx == ctx, B2S_INVALID_ARG,
             "Schur: every part must belong to this context");
        auto impl = std::make_unique<PcSchur>();
        impl->nv = n_vel;
        impl->np = n_pres;
        impl->B = &B->d;
        impl->Bt = &Bt->d;
        impl->A = A_pc->impl.get();
        impl->S = S_pc ? S_pc->impl.get() : nullptr;
        impl->wu.alloc(n_vel ? n_vel : 1);
        impl->rum.alloc(n_vel ? n_vel : 1);
        impl->rpm.alloc(n_pres ? n_pres : 1);
        pc->impl = std::move(impl);
    });
    if (st != B2S_OK)
    {
        delete pc;
        return st;
    }
    *out = pc;
    return B2S_OK;
}

b2s_status b2s_pc_create_scaled(b2s_ctx* ctx, b2s_pc* inner, double alpha, b2s_pc** out)
{
    if (!ctx || !inner || !out) return B2S_INVALID_ARG;
    *out = nullptr;
    b2s_pc* pc = new b2s_pc();
    pc->ctx = ctx;
    pc->kind = B2S_PC_SCALED;
    pc->n = inner->n;
    const b2s_status st = guarded(ctx, [&] {
        need(inner->ctx == ctx, B2S_INVALID_ARG, "scaled preconditioner: the inner one belongs to another context");
        auto impl = std::make_unique<PcScaled>();
        impl->n = inner->n;
        impl->alpha = alpha;
        impl->inner = inner->impl.get();
        pc->impl = std::move(impl);
    });
    if (st != B2S_OK)
    {
        delete pc;
        return st;
    }
    *out = pc;
    return B2S_OK;
}

}  // extern "C"
