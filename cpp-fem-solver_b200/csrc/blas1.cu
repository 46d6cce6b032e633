// Vector kernels: dot (SMatrix::dot, array.cpp:3401-3416), fill, copy.
#include "b2s_internal.cuh"

namespace b2s {

__global__ void __launch_bounds__(kThreads) k_dot(uint64_t n, const double* __restrict__ a, const double* __restrict__ b,
                                                  double* out, const int* done, double* partial, unsigned int* counter)
{
    if (done && *done) return;
    double acc[1] = {0.0};
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        acc[0] += a[i] * b[i];
    if (grid_reduce_last<1>(acc, partial, counter))
        if (threadIdx.x == 0) *out = acc[0];
}

__global__ void k_fill(double* x, double v, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) x[i] = v;
}

__global__ void k_copy(double* __restrict__ d, const double* __restrict__ s, uint64_t n, const int* done)
{
    if (done && *done) return;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) d[i] = s[i];
}

void dot_dev(b2s_ctx* ctx, uint64_t n, const double* a, const double* b, double* out, const int* done)
{
    const unsigned g = stream_grid(ctx, n);
    reserve_reduction(ctx, g);
    B2S_LAUNCH(ctx, k_dot, g, kThreads, 0, n, a, b, out, done, ctx->partial.p, ctx->counter.p);
}

double dot_host(b2s_ctx* ctx, uint64_t n, const double* a, const double* b)
{
    DBuf<double> out(1);
    dot_dev(ctx, n, a, b, out.p);
    d2h(ctx, ctx->h_scalar, out.p, sizeof(double));
    sync(ctx);
    return ctx->h_scalar[0];
}

void fill(b2s_ctx* ctx, double* x, double v, uint64_t n)
{
    if (!n) return;
    B2S_LAUNCH(ctx, k_fill, stream_grid(ctx, n), kThreads, 0, x, v, n);
}

void copy(b2s_ctx* ctx, double* dst, const double* src, uint64_t n, const int* done)
{
    if (!n) return;
    B2S_LAUNCH(ctx, k_copy, stream_grid(ctx, n), kThreads, 0, dst, src, n, done);
}

}  // namespace b2s

using namespace b2s;

extern "C" {

b2s_status b2s_dot_device(b2s_ctx* ctx, uint64_t n, const double* d_a, const double* d_b, double* out)
{
    if (!ctx || !out) return B2S_INVALID_ARG;
    return guarded(ctx, [&] { *out = dot_host(ctx, n, d_a, d_b); });
}

b2s_status b2s_dot(b2s_ctx* ctx, uint64_t n, const double* a, const double* b, double* out)
{
    if (!ctx || !out || (n && (!a || !b))) return B2S_INVALID_ARG;
    return guarded(ctx, [&] {
        DBuf<double> da(n), db(n);
        h2d(ctx, da.p, a, da.bytes());
        h2d(ctx, db.p, b, db.bytes());
        *out = dot_host(ctx, n, da.p, db.p);
    });
}

}  // extern "C"
