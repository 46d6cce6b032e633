// Sync-free traversal of a triangular dependency DAG in one launch.
//
// Rows are visited in a fixed "position" order in which every row's
// dependencies sit at earlier positions (natural order for a lower factor,
// reversed order for an upper one, or any level-sorted order).  A CTA takes
// the next chunk of kThreads positions from a global ticket when it starts,
// so a CTA only ever waits on positions owned by CTAs that started before it
// (resident or finished): no CTA waits on one that cannot run.  Inside a warp
// the lanes advance in lockstep: on each pass every unfinished lane checks
// its dependencies' ready flags and, when all are set, computes its row and
// publishes it; a lane never spins while a lane it depends on is parked in
// the same warp.  Every wait is bounded: after kMaxSpins passes the lane sets
// the error word (B2S_TIMEOUT) and publishes its row anyway, so the kernel
// always ends and the host reads the status.
//
// Ready flags hold an epoch number kept in device memory and bumped before
// each traversal, so flags never need clearing and a captured CUDA graph can
// replay the traversal.
#pragma once
#include "b2s_internal.cuh"

namespace b2s {

constexpr unsigned kMaxSpins = 1u << 22;

// acquire: loads of a dependency's value issued after a flag read observe the
// value its producer wrote before the matching release store
__device__ __forceinline__ uint32_t ld_flag(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_flag_release(uint32_t* p, uint32_t v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

struct SyncFreeCtl
{
    uint32_t* ticket;   // [0] chunk ticket, [1] exit counter
    uint32_t* epoch;    // current epoch (device)
    uint32_t* flags;    // per row
    int* err;           // B2S_TIMEOUT on a wait that gave up
};

static __global__ void k_epoch_bump(uint32_t* epoch, const int* done)
{
    if (done && *done) return;
    *epoch += 1u;
}

// Op must provide:
//   __device__ bool ready(uint32_t row, const uint32_t* flags, uint32_t epoch) const
//   __device__ void compute(uint32_t row) const
template <typename Op>
__global__ void __launch_bounds__(kThreads) k_syncfree(uint32_t n, const uint32_t* __restrict__ order, int reverse,
                                                       SyncFreeCtl ctl, Op op, const int* done)
{
    if (done && *done) return;
    __shared__ uint32_t s_chunk;
    if (threadIdx.x == 0) s_chunk = atomicAdd(&ctl.ticket[0], 1u);
    __syncthreads();
    const uint32_t epoch = ld_flag(ctl.epoch);
    const uint32_t pos = s_chunk * blockDim.x + threadIdx.x;
    const bool active = pos < n;
    uint32_t row = 0;
    if (active) row = order ? __ldg(&order[pos]) : (reverse ? n - 1 - pos : pos);
    bool fin = !active;
    unsigned spins = 0, backoff = 32;
    for (;;)
    {
        const unsigned pending = __ballot_sync(0xffffffffu, !fin);
        if (!pending) break;
        bool advanced = false;
        if (!fin)
        {
            if (op.ready(row, ctl.flags, epoch))
            {
                op.compute(row);
                __threadfence();
                st_flag_release(&ctl.flags[row], epoch);
                fin = true;
                advanced = true;
            }
            else if (++spins > kMaxSpins)
            {
                atomicExch(ctl.err, (int)B2S_TIMEOUT);
                st_flag_release(&ctl.flags[row], epoch);
                fin = true;
            }
        }
        // a warp that made no progress backs off (bounded exponential sleep) so
        // that waiting warps do not flood L2 with flag polls
        if (__ballot_sync(0xffffffffu, advanced))
            backoff = 32;
        else
        {
            __nanosleep(backoff);
            backoff = backoff < 1024 ? backoff * 2 : 1024;
        }
        __syncwarp();
    }
    // the last CTA to leave resets the ticket for the next launch
    __syncthreads();
    if (threadIdx.x == 0)
    {
        __threadfence();
        const uint32_t left = atomicAdd(&ctl.ticket[1], 1u);
        if (left == gridDim.x - 1)
        {
            ctl.ticket[0] = 0u;
            ctl.ticket[1] = 0u;
            __threadfence();
        }
    }
}

// all dependencies j (j < row for a lower DAG, j > row for an upper one) published?
template <bool LOWER>
__device__ __forceinline__ bool deps_ready(uint32_t row, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                           const uint32_t* flags, uint32_t epoch)
{
    const uint32_t a = __ldg(&rp[row]), b = __ldg(&rp[row + 1]);
    for (uint32_t p = a; p < b; ++p)
    {
        const uint32_t j = __ldg(&ci[p]);
        if (LOWER ? (j < row) : (j > row))
            if (ld_flag(&flags[j]) != epoch) return false;
    }
    return true;
}

// Holder of the control words of one traversal schedule.
struct SyncFree
{
    DBuf<uint32_t> words;  // ticket[2], epoch[1], err (as int) [1]
    DBuf<uint32_t> flags;
    uint32_t n = 0;
    void init(b2s_ctx* ctx, uint32_t rows)
    {
        n = rows;
        words.alloc(4);
        flags.alloc(rows ? rows : 1);
        B2S_CUDA(cudaMemsetAsync(words.p, 0, words.bytes(), ctx->stream));
        B2S_CUDA(cudaMemsetAsync(flags.p, 0, flags.bytes(), ctx->stream));
    }
    SyncFreeCtl ctl() const { return SyncFreeCtl{words.p, words.p + 2, flags.p, reinterpret_cast<int*>(words.p + 3)}; }
    template <typename Op>
    void run(b2s_ctx* ctx, const uint32_t* order, bool reverse, const Op& op, const int* done)
    {
        if (!n) return;
        B2S_LAUNCH(ctx, k_epoch_bump, 1, 1, 0, words.p + 2, done);
        const unsigned grid = (n + kThreads - 1) / kThreads;
        B2S_LAUNCH(ctx, k_syncfree<Op>, grid, kThreads, 0, n, order, reverse ? 1 : 0, ctl(), op, done);
    }
    // B2S_OK or B2S_TIMEOUT (synchronises)
    int status(b2s_ctx* ctx) const
    {
        int e = 0;
        d2h(ctx, &e, words.p + 3, sizeof(int));
        sync(ctx);
        return e;
    }
};

}  // namespace b2s
