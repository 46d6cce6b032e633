// Context, status names and matrix handles of the b2s C ABI.
#include <mutex>
#include <unordered_map>
#include <unordered_set>

#include "b2s_internal.cuh"

#include <algorithm>

using namespace b2s;

namespace b2s {
namespace mem {

namespace {
std::mutex g_mu;
std::unordered_set<cudaStream_t> g_live;          // streams of live contexts
std::unordered_map<int, cudaStream_t> g_alloc;    // per-device allocation stream

cudaStream_t alloc_stream_of(int dev)
{
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_alloc.find(dev);
    if (it != g_alloc.end()) return it->second;
    cudaStream_t s = nullptr;
    cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreateWithFlags (allocation stream)");
    // keep freed memory in the pool rather than returning it at every synchronisation
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess)
    {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    g_alloc[dev] = s;
    return s;
}

bool live(cudaStream_t s)
{
    std::lock_guard<std::mutex> lock(g_mu);
    return g_live.count(s) != 0;
}
}  // namespace

cudaStream_t& current_stream()
{
    static thread_local cudaStream_t s = nullptr;
    return s;
}

void register_stream(cudaStream_t s)
{
    std::lock_guard<std::mutex> lock(g_mu);
    g_live.insert(s);
}

void unregister_stream(cudaStream_t s)
{
    std::lock_guard<std::mutex> lock(g_mu);
    g_live.erase(s);
}

Block alloc(size_t bytes)
{
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    Block b;
    b.alloc_stream = alloc_stream_of(dev);
    b.owner = current_stream();
    cudaError_t e = cudaMallocAsync(&b.p, bytes, b.alloc_stream);
    if (e == cudaErrorMemoryAllocation)
    {
        // give the pool's cached memory back to the device and try once more
        cudaGetLastError();
        cudaMemPool_t pool;
        cudaStreamSynchronize(b.alloc_stream);
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
        e = cudaMallocAsync(&b.p, bytes, b.alloc_stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(b.alloc_stream);
    if (e != cudaSuccess)
    {
        b.p = nullptr;
        cuda_check(e, ("device allocation of " + std::to_string(bytes) + " bytes").c_str());
    }
    return b;
}

void free(const Block& b)
{
    if (!b.p) return;
    if (b.owner && live(b.owner))
    {
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        cudaEvent_t ev = nullptr;
        if (cudaStreamIsCapturing(b.owner, &cap) == cudaSuccess && cap == cudaStreamCaptureStatusNone &&
            cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess)
        {
            const bool ok = cudaEventRecord(ev, b.owner) == cudaSuccess &&
                            cudaStreamWaitEvent(b.alloc_stream, ev, 0) == cudaSuccess &&
                            cudaFreeAsync(b.p, b.alloc_stream) == cudaSuccess;
            cudaEventDestroy(ev);
            if (ok) return;
        }
        cudaGetLastError();
    }
    cudaFree(b.p);  // synchronous
    cudaGetLastError();
}

}  // namespace mem
}  // namespace b2s

namespace b2s {

void check_device_error(b2s_ctx* ctx, const char* where)
{
    int h = 0;
    B2S_CUDA(cudaMemcpyAsync(&h, ctx->errword(), sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    if (h)
    {
        B2S_CUDA(cudaMemsetAsync(ctx->errword(), 0, sizeof(int), ctx->stream));
        sync(ctx);
        fail((b2s_status)h, where);
    }
}

}  // namespace b2s

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
        mem::register_stream(ctx->stream);
        mem::current_stream() = ctx->stream;
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
    if (ctx->stream)
    {
        mem::unregister_stream(ctx->stream);
        cudaStreamDestroy(ctx->stream);
    }
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
    // asynchronous entry points (b2s_dense_bf16_device, b2s_pc_apply_device)
    // report a bounded device wait that gave up through the error word
    return guarded(ctx, [&] { check_device_error(ctx, "a device-side wait gave up"); });
}

b2s_status b2s_ctx_set_wait_limits(b2s_ctx* ctx, uint32_t spin_polls, uint32_t sleep_polls)
{
    if (!ctx) return B2S_INVALID_ARG;
    ctx->wait_fast_polls = spin_polls ? spin_polls : (1u << 20);
    ctx->wait_slow_polls = (spin_polls || sleep_polls) ? sleep_polls : (1u << 20);
    return B2S_OK;
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
