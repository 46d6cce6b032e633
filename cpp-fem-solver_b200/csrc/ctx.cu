// Context, status names and matrix handles of the b2s C ABI.
#include "b2s_internal.cuh"

#include <algorithm>

using namespace b2s;

extern "C" {

b2s_status b2s_ctx_create(int device, b2s_ctx** out)
{
    if (!out) return B2S_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
    {
        cudaGetLastError();
        return B2S_NO_DEVICE;
    }
    if (device < 0 || device >= count) return B2S_INVALID_ARG;
    b2s_ctx* ctx = new b2s_ctx();
    b2s_status st = guarded(ctx, [&] {
        ctx->device = device;
        B2S_CUDA(cudaSetDevice(device));
        cudaDeviceProp prop;
        B2S_CUDA(cudaGetDeviceProperties(&prop, device));
        if (prop.major < 10) fail(B2S_UNSUPPORTED, "b2s is built for sm_100a (B200); device is sm_" +
                                                       std::to_string(prop.major) + std::to_string(prop.minor));
        ctx->sm_count = prop.multiProcessorCount;
        B2S_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        ctx->partial.alloc((size_t)ctx->sm_count * 8 * kMaxRedValues);
        ctx->counter.alloc(64);
        B2S_CUDA(cudaMemset(ctx->counter.p, 0, ctx->counter.bytes()));
        ctx->kstate.alloc(1);
        B2S_CUDA(cudaMallocHost(&ctx->h_kstate, sizeof(KState)));
        B2S_CUDA(cudaMallocHost(&ctx->h_scalar, 64 * sizeof(double)));
        B2S_CUDA(cudaEventCreate(&ctx->ev0));
        B2S_CUDA(cudaEventCreate(&ctx->ev1));
        B2S_CUDA(cudaDeviceSynchronize());
    });
    if (st != B2S_OK)
    {
        b2s_ctx_destroy(ctx);
        return st;
    }
    *out = ctx;
    return B2S_OK;
}

b2s_status b2s_ctx_destroy(b2s_ctx* ctx)
{
    if (!ctx) return B2S_INVALID_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->partial.release();
    ctx->counter.release();
    ctx->kstate.release();
    if (ctx->h_kstate) cudaFreeHost(ctx->h_kstate);
    if (ctx->h_scalar) cudaFreeHost(ctx->h_scalar);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return B2S_OK;
}

const char* b2s_last_error(const b2s_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

const char* b2s_status_name(b2s_status st)
{
    switch (st)
    {
        case B2S_OK: return "B2S_OK";
        case B2S_INVALID_ARG: return "B2S_INVALID_ARG";
        case B2S_SHAPE: return "B2S_SHAPE";
        case B2S_NOT_SPD: return "B2S_NOT_SPD";
        case B2S_BREAKDOWN: return "B2S_BREAKDOWN";
        case B2S_ZERO_PIVOT: return "B2S_ZERO_PIVOT";
        case B2S_MISSING_DIAG: return "B2S_MISSING_DIAG";
        case B2S_SINGULAR_BLOCK: return "B2S_SINGULAR_BLOCK";
        case B2S_DIVERGED: return "B2S_DIVERGED";
        case B2S_TIMEOUT: return "B2S_TIMEOUT";
        case B2S_CUDA_ERROR: return "B2S_CUDA_ERROR";
        case B2S_NO_DEVICE: return "B2S_NO_DEVICE";
        case B2S_OUT_OF_MEMORY: return "B2S_OUT_OF_MEMORY";
        case B2S_UNSUPPORTED: return "B2S_UNSUPPORTED";
    }
    return "B2S_UNKNOWN";
}

void* b2s_ctx_stream(b2s_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

b2s_status b2s_ctx_synchronize(b2s_ctx* ctx)
{
    if (!ctx) return B2S_INVALID_ARG;
    return guarded(ctx, [&] { sync(ctx); });
}

uint64_t b2s_ctx_kernel_launches(const b2s_ctx* ctx) { return ctx ? ctx->launches : 0; }

void b2s_pc_opts_default(b2s_pc_opts* o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->omega = 1.2;
    o->precision = B2S_FP64;
    o->trsv = B2S_TRSV_AUTO;
    o->amg_ref_coarse = 0;
    o->amg_max_levels = 0;
    o->amg_coarse_max = 0;
    o->amg_aggregation = 0;
    o->learned_weights = nullptr;
}

void b2s_solve_opts_default(b2s_solve_opts* o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->tol = 1e-10;
    o->maxit = 2000;
    o->restart = 30;
    o->orth = B2S_ORTH_MGS;
    o->ir_steps = 0;
    o->ir_inner_tol = 0.0;
    o->check_every = 0;
    o->use_graphs = 1;
}

}  // extern "C"
