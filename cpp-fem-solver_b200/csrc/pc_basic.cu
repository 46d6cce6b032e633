// Identity, diagonal (Jacobi) and host-callback preconditioners, and the
// preconditioner half of the C ABI.
//   make_diag_preconditioner: array.cpp:2450-2508
//   preconditioner name tables: array.cpp:3482-3515 (pcg), 3637-3673
//   (bicgstab), 4212-4242 (gmres); blockMatrix.hpp:710-744 (block gmres)
#include "b2s_internal.cuh"

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>

namespace b2s {

namespace {

struct PcIdentity final : PcImpl
{
    uint64_t n;
    explicit PcIdentity(uint64_t n_) : n(n_) {}
    void apply(b2s_ctx* ctx, const double* r, double* z, const int* done) override { copy(ctx, z, r, n, done); }
    bool is_identity() const override { return true; }
};

__global__ void k_diag_apply(uint64_t n, const double* __restrict__ r, const double* __restrict__ d,
                             double* __restrict__ z, const int* done)
{
    if (done && *done) return;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        z[i] = r[i] / d[i];
}

struct PcDiag final : PcImpl
{
    uint64_t n;
    DBuf<double> d;
    void apply(b2s_ctx* ctx, const double* r, double* z, const int* done) override
    {
        B2S_LAUNCH(ctx, k_diag_apply, stream_grid(ctx, n), kThreads, 0, n, r, d.p, z, done);
    }
    const double* fused_diag() const override { return d.p; }
};

struct PcHost final : PcImpl
{
    uint64_t n;
    b2s_host_pc_fn fn;
    void* user;
    std::vector<double> hr, hz;
    void apply(b2s_ctx* ctx, const double* r, double* z, const int* done) override
    {
        if (done)
        {
            int h = 0;
            d2h(ctx, &h, done, sizeof(int));
            sync(ctx);
            if (h) return;
        }
        hr.resize(n);
        hz.assign(n, 0.0);
        d2h(ctx, hr.data(), r, n * sizeof(double));
        sync(ctx);
        const int rc = fn(user, hr.data(), hz.data(), n);
        if (rc != 0) fail(B2S_BREAKDOWN, "host preconditioner callback failed (code " + std::to_string(rc) + ")");
        h2d(ctx, z, hz.data(), n * sizeof(double));
        sync(ctx);
    }
    bool is_host() const override { return true; }
};

}  // namespace

std::unique_ptr<PcImpl> make_pc_identity(uint64_t n) { return std::make_unique<PcIdentity>(n); }

std::unique_ptr<PcImpl> make_pc_diag(b2s_ctx* ctx, const CsrDev& A)
{
    need(A.n == A.m, B2S_SHAPE, "diag preconditioner needs a square matrix");
    auto pc = std::make_unique<PcDiag>();
    pc->n = A.n;
    pc->d.alloc(A.n);
    copy(ctx, pc->d.p, A.diag.p, A.n);
    std::vector<double> h(A.n);
    d2h(ctx, h.data(), A.diag.p, A.n * sizeof(double));
    sync(ctx);
    for (uint32_t i = 0; i < A.n; ++i)
    {
        if (std::fabs(h[i]) < 1e-14)
            fail(B2S_ZERO_PIVOT, "diag preconditioner: zero or tiny diagonal entry at row " + std::to_string(i));
        if (h[i] <= 0.0)
            fail(B2S_NOT_SPD, "diag preconditioner: diagonal must be positive (row " + std::to_string(i) + ")");
    }
    return pc;
}

std::unique_ptr<PcImpl> make_pc_host(uint64_t n, b2s_host_pc_fn fn, void* user)
{
    auto pc = std::make_unique<PcHost>();
    pc->n = n;
    pc->fn = fn;
    pc->user = user;
    return pc;
}

}  // namespace b2s

using namespace b2s;

namespace {

double now_ms()
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

extern "C" {

b2s_status b2s_pc_create(b2s_ctx* ctx, const b2s_csr* A, b2s_pc_kind kind, const b2s_pc_opts* opts, b2s_pc** out)
{
    if (!ctx || !A || !out) return B2S_INVALID_ARG;
    *out = nullptr;
    b2s_pc_opts o;
    b2s_pc_opts_default(&o);
    if (opts) o = *opts;
    b2s_pc* pc = new b2s_pc();
    pc->ctx = ctx;
    pc->kind = kind;
    pc->n = A->d.n;
    b2s_status st = guarded(ctx, [&] {
        B2S_CUDA(cudaSetDevice(ctx->device));
        need(A->d.n == A->d.m, B2S_SHAPE, "preconditioner needs a square matrix");
        need(o.precision == B2S_FP64 || o.precision == B2S_FP32, B2S_UNSUPPORTED,
             "preconditioner precision: only B2S_FP64 and B2S_FP32 storage exist");
        const double t0 = now_ms();
        switch (kind)
        {
            case B2S_PC_NONE: pc->impl = make_pc_identity(A->d.n); break;
            case B2S_PC_DIAG: pc->impl = make_pc_diag(ctx, A->d); break;
            case B2S_PC_IC0: pc->impl = make_pc_ic0(ctx, A->d, o); break;
            case B2S_PC_ILU0: pc->impl = make_pc_ilu0(ctx, A->d, o); break;
            case B2S_PC_SSOR: pc->impl = make_pc_ssor(ctx, A->d, o); break;
            case B2S_PC_SA_AMG: pc->impl = make_pc_amg_csr(ctx, A->d, o); break;
            case B2S_PC_LEARNED_IC0: pc->impl = make_pc_learned_ic0(ctx, A->d, o); break;
            default: fail(B2S_INVALID_ARG, "preconditioner kind not valid for a CSR matrix");
        }
        sync(ctx);
        check_device_error(ctx, "a device-side wait gave up during the set-up");
        pc->setup_ms = now_ms() - t0;
    });
    if (st != B2S_OK)
    {
        delete pc;
        return st;
    }
    *out = pc;
    return B2S_OK;
}

b2s_status b2s_pc_create_baij(b2s_ctx* ctx, const b2s_baij* A, b2s_pc_kind kind, const b2s_pc_opts* opts,
                              b2s_pc** out)
{
    if (!ctx || !A || !out) return B2S_INVALID_ARG;
    *out = nullptr;
    b2s_pc_opts o;
    b2s_pc_opts_default(&o);
    if (opts) o = *opts;
    b2s_pc* pc = new b2s_pc();
    pc->ctx = ctx;
    pc->kind = kind;
    pc->n = (uint64_t)A->d.nbr * A->d.bs;
    b2s_status st = guarded(ctx, [&] {
        B2S_CUDA(cudaSetDevice(ctx->device));
        need(A->d.nbr == A->d.nbc, B2S_SHAPE, "block preconditioner needs a square block matrix");
        need(o.precision == B2S_FP64 || o.precision == B2S_FP32, B2S_UNSUPPORTED,
             "preconditioner precision: only B2S_FP64 and B2S_FP32 storage exist");
        const double t0 = now_ms();
        switch (kind)
        {
            case B2S_PC_NONE: pc->impl = make_pc_identity(pc->n); break;
            case B2S_PC_BJACOBI: pc->impl = make_pc_bjacobi(ctx, A->d); break;
            case B2S_PC_BILU0: pc->impl = make_pc_bilu0(ctx, A->d, o); break;
            case B2S_PC_BSA_AMG:
            case B2S_PC_SA_AMG: pc->impl = make_pc_amg_baij(ctx, A->d, o); break;
            default: fail(B2S_INVALID_ARG, "preconditioner kind not valid for a BAIJ matrix");
        }
        sync(ctx);
        check_device_error(ctx, "a device-side wait gave up during the set-up");
        pc->setup_ms = now_ms() - t0;
    });
    if (st != B2S_OK)
    {
        delete pc;
        return st;
    }
    *out = pc;
    return B2S_OK;
}

b2s_status b2s_pc_create_host(b2s_ctx* ctx, uint64_t n, b2s_host_pc_fn fn, void* user, b2s_pc** out)
{
    if (!ctx || !fn || !out) return B2S_INVALID_ARG;
    b2s_pc* pc = new b2s_pc();
    pc->ctx = ctx;
    pc->kind = B2S_PC_NONE;
    pc->n = n;
    pc->impl = make_pc_host(n, fn, user);
    *out = pc;
    return B2S_OK;
}

b2s_status b2s_pc_destroy(b2s_pc* pc)
{
    if (!pc) return B2S_INVALID_ARG;
    cudaSetDevice(pc->ctx->device);
    delete pc;
    return B2S_OK;
}

b2s_status b2s_pc_apply_device(b2s_ctx* ctx, b2s_pc* pc, const double* d_r, double* d_z)
{
    if (!ctx || !pc) return B2S_INVALID_ARG;
    return guarded(ctx, [&] { pc->impl->apply(ctx, d_r, d_z, nullptr); });
}

b2s_status b2s_pc_apply(b2s_ctx* ctx, b2s_pc* pc, const double* r, double* z)
{
    if (!ctx || !pc || (pc->n && (!r || !z))) return B2S_INVALID_ARG;
    return guarded(ctx, [&] {
        DBuf<double> dr(pc->n), dz(pc->n);
        h2d(ctx, dr.p, r, dr.bytes());
        pc->impl->apply(ctx, dr.p, dz.p, nullptr);
        d2h(ctx, z, dz.p, dz.bytes());
        sync(ctx);
        check_device_error(ctx, "a triangular-solve wait gave up during the apply");
    });
}

b2s_status b2s_pc_export(b2s_ctx* ctx, b2s_pc* pc, const char* what, uint64_t* sizes, uint32_t* rp, uint32_t* ci,
                         double* v)
{
    if (!ctx || !pc || !what || !sizes) return B2S_INVALID_ARG;
    return guarded(ctx, [&] { pc->impl->export_data(ctx, what, sizes, rp, ci, v); });
}

b2s_status b2s_pc_kind_from_name(int method, const char* name, b2s_pc_kind* kind)
{
    if (!name || !kind) return B2S_INVALID_ARG;
    std::string s(name);
    if (method == B2S_BLOCK_GMRES)
    {
        // BlockMatrix::gmres compares the raw string (no to_lower)
        if (s == "none" || s == "identity") *kind = B2S_PC_NONE;
        else if (s == "blockjacobi") *kind = B2S_PC_BJACOBI;
        else if (s == "blockilu" || s == "blockilu0") *kind = B2S_PC_BILU0;
        else return B2S_INVALID_ARG;
        return B2S_OK;
    }
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    if (s == "none" || s == "identity" || s == "noprecond" || (method == B2S_PCG && s == "cg")) *kind = B2S_PC_NONE;
    else if (s == "diag" || s == "diagonal" || s == "jacobi") *kind = B2S_PC_DIAG;
    else if (s == "ic" || s == "ic0" || s == "ichol" || (method != B2S_GMRES && method != B2S_FGMRES && s == "incomplete_cholesky"))
        *kind = B2S_PC_IC0;
    else if (s == "ilu" || s == "ilu0") *kind = B2S_PC_ILU0;
    else if (s == "sor" || s == "ssor") *kind = B2S_PC_SSOR;
    else if (s == "amg") *kind = B2S_PC_SA_AMG;
    else return B2S_INVALID_ARG;
    return B2S_OK;
}

}  // extern "C"
