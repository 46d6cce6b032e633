// Internal definitions shared by the b2s CUDA sources (sm_100a only).
//
// Layout in HBM: every operator and factor is device resident for the life of
// its handle.  CSR uses uint32 row_ptr / col_idx and FP64 values (plus an
// optional FP32 copy for mixed-precision preconditioners); BAIJ stores blocks
// row-major, contiguous per block.  Vectors are plain FP64 arrays.
//
// Numerics: the library is compiled with -fmad=false, so every a*b+c is a
// rounded multiply followed by a rounded add, as in the reference compiled
// with ISO C++17 (no contraction).  Per-row sums run in ascending column
// order, so SpMV and triangular-solve rows equal the reference bit for bit.
// Reductions (dots, norms) use a fixed-order two-level tree: block partials in
// a fixed grid, combined by the last block to arrive; the result is identical
// from run to run.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "b2s.h"

namespace b2s {

// ----------------------------------------------------------------- errors

struct Error : std::runtime_error
{
    b2s_status status;
    Error(b2s_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

[[noreturn]] inline void fail(b2s_status s, const std::string& m) { throw Error(s, m); }

inline void cuda_check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess)
    {
        // clear the runtime's last-error state so a recoverable error is not
        // reported again by the next launch check
        cudaGetLastError();
        if (e == cudaErrorMemoryAllocation) fail(B2S_OUT_OF_MEMORY, std::string(what) + ": " + cudaGetErrorString(e));
        fail(B2S_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

#define B2S_CUDA(call) ::b2s::cuda_check((call), #call)

// ---------------------------------------------------------- device memory
//
// Device memory comes from the device's stream-ordered pool and goes back to
// it, so repeated set-ups reuse memory instead of paying for cudaMalloc and
// for cudaFree's device-wide synchronisation (ctx.cu).  Allocations run on a
// per-device allocation stream that is synchronised at once, so the memory is
// ready for any stream.  A buffer remembers the stream of the context whose
// API call allocated it, and its free is ordered after the work already on
// that stream (an event the allocation stream waits on); when that stream is
// gone the free is synchronous.
namespace mem {
struct Block
{
    void* p = nullptr;
    cudaStream_t alloc_stream = nullptr;  // the pool's allocation stream of the block's device
    cudaStream_t owner = nullptr;         // stream of the allocating context, or null
};
Block alloc(size_t bytes);  // throws Error on failure
void free(const Block& b);
cudaStream_t& current_stream();  // thread-local: the stream of the API call in progress
void register_stream(cudaStream_t s);
void unregister_stream(cudaStream_t s);
}  // namespace mem

template <typename T>
struct DBuf
{
    T* p = nullptr;
    size_t n = 0;
    mem::Block blk;
    DBuf() = default;
    explicit DBuf(size_t count) { alloc(count); }
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), blk(o.blk)
    {
        o.p = nullptr;
        o.n = 0;
        o.blk = mem::Block{};
    }
    DBuf& operator=(DBuf&& o) noexcept
    {
        if (this != &o)
        {
            release();
            p = o.p;
            n = o.n;
            blk = o.blk;
            o.p = nullptr;
            o.n = 0;
            o.blk = mem::Block{};
        }
        return *this;
    }
    ~DBuf() { release(); }
    void alloc(size_t count)
    {
        release();
        if (count)
        {
            blk = mem::alloc(count * sizeof(T));
            p = static_cast<T*>(blk.p);
            n = count;
        }
    }
    // grows (never shrinks); contents are not preserved
    void reserve(size_t count)
    {
        if (count > n) alloc(count);
    }
    void release()
    {
        if (p) mem::free(blk);
        p = nullptr;
        n = 0;
        blk = mem::Block{};
    }
    size_t bytes() const { return n * sizeof(T); }
};

// --------------------------------------------------------------- constants

constexpr int kThreads = 256;          // block size of streaming / reduction kernels
constexpr int kMaxRedValues = 8;       // values reduced together by one kernel
constexpr int kSpmvRowsPerCta = 256;   // staged SpMV: at most this many rows per CTA
constexpr int kSpmvNnzPerCta = 3072;   // staged SpMV: nnz staged in shared memory per CTA

// Device-side solver state: the scalars of one Krylov iteration.  Kernels read
// it at entry, the last block of each reduction kernel updates it.
struct KState
{
    double normb, tol;
    double rz_old, pAp, alpha, beta, normr, omega, rho_old, rho_new;
    double relres;
    double aux[8];
    int it;       // iteration index in progress
    int it_end;   // the reference's returned count
    int maxit;
    int done;     // 1 once converged / failed / stopped
    int status;   // b2s_status
    int iters;    // iterations executed (SpMVs in the loop)
    int stalled;  // 1: a device-side stall guard stopped the solve
    int pad;
};

}  // namespace b2s

// ------------------------------------------------------------------ handles

struct b2s_ctx
{
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    std::string err;
    uint64_t launches = 0;
    // reduction scratch: partial sums (kMaxRedValues per block) + arrival counter
    b2s::DBuf<double> partial;
    b2s::DBuf<unsigned int> counter;
    // general device scratch and pinned host staging
    b2s::DBuf<b2s::KState> kstate;
    b2s::DBuf<double> ws;             // Krylov workspace, grown on demand
    b2s::DBuf<double> small;          // Hessenberg / Givens scratch
    b2s::KState* h_kstate = nullptr;  // pinned mirror
    double* h_scalar = nullptr;       // pinned, 64 doubles
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // device error word (B2S_TIMEOUT from a bounded wait); counter[32..]
    int* errword() { return reinterpret_cast<int*>(counter.p + 32); }
    // bounds of the chunked triangular solves' waits (b2s_ctx_set_wait_limits)
    unsigned wait_fast_polls = 1u << 20;
    unsigned wait_slow_polls = 1u << 20;
};

namespace b2s {
// Reads the context's device error word (synchronises); a set word is
// cleared and raised as its status (B2S_TIMEOUT: a bounded wait gave up).
void check_device_error(b2s_ctx* ctx, const char* where);
}

namespace b2s {

struct CsrDev
{
    uint32_t n = 0, m = 0, nnz = 0;
    DBuf<uint32_t> rp, ci;
    DBuf<double> v;
    DBuf<float> v32;            // FP32 copy, created on demand
    DBuf<uint32_t> blk_row;     // staged-SpMV row partition (nblk+1)
    uint32_t nblk = 0;
    uint32_t max_row = 0;       // longest row (nonzeros); 0 = not known
    DBuf<double> diag;          // diagonal entries (0 where missing)
    // host copy of the pattern, made on demand by the setup code that needs it
    mutable std::vector<uint32_t> h_rp, h_ci;
    void host_pattern(b2s_ctx* ctx) const;
    void ensure_fp32(b2s_ctx* ctx);
};

struct BaijDev
{
    int bs = 3;
    uint32_t nbr = 0, nbc = 0, nnzb = 0;
    DBuf<uint32_t> rp, ci;
    DBuf<double> v;
    DBuf<uint32_t> diag_ptr;    // UINT32_MAX when missing
    DBuf<uint32_t> blk_row;     // bs = 1 with long rows: staged-matvec row partition (nblk + 1)
    uint32_t nblk = 0;          // 0: the matvec needs no partition
};

// Row partition of a bs = 1 BAIJ with long rows for its staged matvec
// (nothing for other operators); h_rp: the host row pointers.
void baij_partition(b2s_ctx* ctx, BaijDev& M, const uint32_t* h_rp);

// Preconditioner implementation.  apply() enqueues z = M^-1 r on ctx->stream
// (device pointers).  `done` (device, may be null) lets the Krylov drivers
// replay work after convergence: every kernel returns at once when *done != 0.
struct PcImpl
{
    virtual ~PcImpl() = default;
    virtual void apply(b2s_ctx* ctx, const double* r, double* z, const int* done) = 0;
    // diagonal scaling that the PCG update kernel can fuse (null if none)
    virtual const double* fused_diag() const { return nullptr; }
    virtual bool is_identity() const { return false; }
    virtual bool is_host() const { return false; }
    virtual void export_data(b2s_ctx*, const std::string& what, uint64_t* sizes, uint32_t* rp, uint32_t* ci,
                             double* v)
    {
        fail(B2S_UNSUPPORTED, "export '" + what + "' not available for this preconditioner");
    }
    // PCG fusion: z = M^-1 r, then rz = r.z and the PCG scalar step
    // (pcg_next) on the device, in the apply's own launches; false (nothing
    // enqueued) when the preconditioner cannot fuse them
    virtual bool apply_rz(b2s_ctx*, const double* r, double* z, KState* st, const int* done)
    {
        (void)r, (void)z, (void)st, (void)done;
        return false;
    }
    // PCG fusion of a whole iteration after the SpMV (given Ap and alpha in
    // st): x += alpha p, r_new = r_old - alpha Ap with the convergence test,
    // z = M^-1 r_new, r_new.z and the scalar step
    virtual bool can_fuse_pcg() const { return false; }
    virtual void pcg_update_apply(b2s_ctx*, double* x, const double* p, const double* Ap, const double* r_old,
                                  double* r_new, double* z, KState* st, const int* done)
    {
        (void)x, (void)p, (void)Ap, (void)r_old, (void)r_new, (void)z, (void)st, (void)done;
        fail(B2S_UNSUPPORTED, "this preconditioner does not fuse the PCG update");
    }
    // The whole PCG loop in one persistent launch (from the state after
    // the first z = M^-1 r, p = z, rz_old): r, p in two buffers each, x
    // updated in place, st on exit as the iteration-by-iteration loop would
    // leave it (st->stalled when the stall guard stopped it).  which: the
    // b2s_solve_opts.persistent choice.  False, with nothing enqueued, when
    // the preconditioner cannot run it.
    virtual bool pcg_persistent(b2s_ctx*, const CsrDev& A, double* x, double* r0, double* r1, double* p0,
                                double* p1, double* z, double* Ap, KState* st, int stall_window, int which)
    {
        (void)A, (void)x, (void)r0, (void)r1, (void)p0, (void)p1, (void)z, (void)Ap, (void)st, (void)stall_window;
        (void)which;
        return false;
    }
    // one triangle of a factored preconditioner M = L L^T (FP64 storage):
    // out = L^{-1} in (upper = false) or L^{-T} in (upper = true)
    virtual void solve_factor(b2s_ctx*, bool upper, const double* in, double* out, const int* done)
    {
        (void)upper, (void)in, (void)out, (void)done;
        fail(B2S_UNSUPPORTED, "no triangular factor solve for this preconditioner");
    }
};

}  // namespace b2s

struct b2s_csr
{
    b2s_ctx* ctx = nullptr;
    b2s::CsrDev d;
};

namespace b2s {
// set_halo state of a BAIJ that holds one rank's block rows with global block
// columns (BlockMatrix::set_halo, blockMatrix.hpp:317-348)
struct HaloDev
{
    bool set = false;
    uint32_t n_owned = 0, n_ghost = 0, n_send = 0, start = 0;
    DBuf<uint32_t> lci;         // local column of every block: owned g - start, ghost n_owned + k
    DBuf<uint32_t> send_local;  // owned block rows that other ranks read, grouped by destination
    std::vector<int> recv_procs, recv_cnts, send_procs, send_cnts;
};
}  // namespace b2s

struct b2s_baij
{
    b2s_ctx* ctx = nullptr;
    b2s::BaijDev d;
    b2s::HaloDev halo;
};

struct b2s_pc
{
    b2s_ctx* ctx = nullptr;
    b2s_pc_kind kind = B2S_PC_NONE;
    uint64_t n = 0;
    double setup_ms = 0.0;
    std::unique_ptr<b2s::PcImpl> impl;
};

namespace b2s {

// ------------------------------------------------------------ API guarding

template <typename F>
b2s_status guarded(b2s_ctx* ctx, F&& f)
{
    // device buffers allocated by this call belong to the context's stream
    struct StreamScope
    {
        cudaStream_t saved;
        explicit StreamScope(cudaStream_t s) : saved(mem::current_stream()) { mem::current_stream() = s; }
        ~StreamScope() { mem::current_stream() = saved; }
    } scope(ctx ? ctx->stream : nullptr);
    try
    {
        f();
        return B2S_OK;
    }
    catch (const Error& e)
    {
        if (ctx) ctx->err = e.what();
        return e.status;
    }
    catch (const std::bad_alloc&)
    {
        if (ctx) ctx->err = "host allocation failed";
        return B2S_OUT_OF_MEMORY;
    }
    catch (const std::exception& e)
    {
        if (ctx) ctx->err = e.what();
        return B2S_CUDA_ERROR;
    }
}

inline void need(bool cond, b2s_status s, const char* msg)
{
    if (!cond) fail(s, msg);
}

inline void note_launch(b2s_ctx* ctx, const char* what)
{
    ctx->launches++;
#ifdef B2S_DEBUG_SYNC
    B2S_CUDA(cudaStreamSynchronize(ctx->stream));
#endif
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) cuda_check(cudaGetLastError(), what);
}

#define B2S_LAUNCH(ctx, kernel, grid, block, smem, ...)                                    \
    do                                                                                     \
    {                                                                                      \
        kernel<<<(grid), (block), (smem), (ctx)->stream>>>(__VA_ARGS__);                   \
        ::b2s::note_launch((ctx), #kernel);                                                \
    } while (0)

inline unsigned stream_grid(const b2s_ctx* ctx, uint64_t n)
{
    uint64_t g = (n + kThreads - 1) / kThreads;
    uint64_t cap = (uint64_t)ctx->sm_count * 8;
    if (g > cap) g = cap;
    return g ? (unsigned)g : 1u;
}

// reserve reduction scratch for `blocks` blocks
inline void reserve_reduction(b2s_ctx* ctx, unsigned blocks)
{
    ctx->partial.reserve((size_t)blocks * kMaxRedValues);
}

// --------------------------------------------------- device-side reductions

// Fixed-order block reduction of NV values (all threads receive the result);
// NT = the block's thread count (a multiple of 32, at most 1024).
template <int NV, int NT = kThreads>
__device__ __forceinline__ void block_reduce(double (&v)[NV])
{
    static_assert(NT % 32 == 0 && NT <= 1024, "block size");
    __shared__ double sred[NV][NT / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k)
    {
        double a = v[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) a += __shfl_down_sync(0xffffffffu, a, off);
        if (lane == 0) sred[k][warp] = a;
    }
    __syncthreads();
    if (warp == 0)
    {
#pragma unroll
        for (int k = 0; k < NV; ++k)
        {
            double a = lane < (NT / 32) ? sred[k][lane] : 0.0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) a += __shfl_down_sync(0xffffffffu, a, off);
            if (lane == 0) sred[k][0] = a;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = sred[k][0];
    __syncthreads();
}

// Grid-wide deterministic reduction: every block contributes v; returns true
// in the last block to arrive, where v then holds the grid total (summed over
// block partials in block order).  Must be called by all threads of every
// block exactly once per kernel.
template <int NV, int NT = kThreads>
__device__ __forceinline__ bool grid_reduce_last(double (&v)[NV], double* partial, unsigned int* counter)
{
    __shared__ bool s_last;
    block_reduce<NV, NT>(v);
    if (threadIdx.x == 0)
    {
#pragma unroll
        for (int k = 0; k < NV; ++k) partial[(size_t)k * gridDim.x + blockIdx.x] = v[k];
        __threadfence();
        const unsigned t = atomicAdd(counter, 1u);
        s_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    // every value's partials summed in block order as before, but the NV loads of
    // one stride issued together (one L2 round trip per stride, not NV)
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = 0.0;
#pragma unroll 2
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
    {
        double p[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) p[k] = __ldcg(&partial[(size_t)k * gridDim.x + b]);
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] += p[k];
    }
    block_reduce<NV, NT>(v);
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

// ------------------------------------------------- PCG scalar steps (device)

__device__ __forceinline__ void finish(KState* st, int status)
{
    st->status = status;
    st->done = 1;
}

// rr = r.r after the update: relative residual, the tolerance and NaN / Inf
// stops (array.cpp:3560-3573)
__device__ __forceinline__ bool pcg_check_converged(KState* st, double rr)
{
    const double normr = sqrt(rr);
    st->normr = normr;
    st->relres = normr / st->normb;
    if (st->relres < st->tol)
    {
        st->it_end = st->it > 0 ? st->it - 1 : 0;
        st->iters = st->it + 1;
        finish(st, B2S_OK);
        return true;
    }
    if (!(normr == normr) || isinf(normr))
    {
        st->iters = st->it + 1;
        st->it_end = st->maxit - 1;
        finish(st, B2S_DIVERGED);
        return true;
    }
    return false;
}

// rz_new = r.z: beta, the iteration counters and the NOT_SPD / maxit stops
// (array.cpp:3575-3593)
__device__ __forceinline__ void pcg_next(KState* st, double rz_new)
{
    if (rz_new <= 0.0)
    {
        st->iters = st->it + 1;
        finish(st, B2S_NOT_SPD);
        return;
    }
    st->beta = rz_new / st->rz_old;
    st->rz_old = rz_new;
    st->it_end = st->it;
    st->it += 1;
    st->iters = st->it;
    if (st->it >= st->maxit) finish(st, B2S_OK);
}

// ---------------------------------------------------------- host helpers

inline void h2d(b2s_ctx* ctx, void* dst, const void* src, size_t bytes)
{
    if (bytes) B2S_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
}
inline void d2h(b2s_ctx* ctx, void* dst, const void* src, size_t bytes)
{
    if (bytes) B2S_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
}
inline void d2d(b2s_ctx* ctx, void* dst, const void* src, size_t bytes)
{
    if (bytes) B2S_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
}
inline void sync(b2s_ctx* ctx) { B2S_CUDA(cudaStreamSynchronize(ctx->stream)); }

template <typename T>
DBuf<T> upload(b2s_ctx* ctx, const T* src, size_t count)
{
    DBuf<T> b(count);
    h2d(ctx, b.p, src, count * sizeof(T));
    return b;
}

// a device copy of a host vector; an empty vector gets one uninitialised element
template <typename T>
DBuf<T> upload(b2s_ctx* ctx, const std::vector<T>& src)
{
    DBuf<T> b(src.empty() ? 1 : src.size());
    if (!src.empty()) h2d(ctx, b.p, src.data(), src.size() * sizeof(T));
    return b;
}

// ------------------------------------------- kernels shared across files

// y = A x, staged CSR (csr.cu)
void spmv(b2s_ctx* ctx, const CsrDev& A, const double* x, double* y, const int* done = nullptr);
// dot product into *out (device), deterministic (blas1.cu)
void dot_dev(b2s_ctx* ctx, uint64_t n, const double* a, const double* b, double* out, const int* done = nullptr);
double dot_host(b2s_ctx* ctx, uint64_t n, const double* a, const double* b);
void fill(b2s_ctx* ctx, double* x, double v, uint64_t n);
void copy(b2s_ctx* ctx, double* dst, const double* src, uint64_t n, const int* done = nullptr);
// BAIJ matvec (baij.cu)
void baij_matvec(b2s_ctx* ctx, const BaijDev& A, const double* x, double* y, const int* done = nullptr);
// the same product with A's pattern and FP32 values v32 (FP64 arithmetic)
void baij_matvec_f32(b2s_ctx* ctx, const BaijDev& A, const float* v32, const double* x, double* y,
                     const int* done = nullptr);
// row partition for staged kernels (csr.cu)
void build_row_blocks(const uint32_t* rp, uint32_t nrows, uint32_t unit, uint32_t max_rows, uint32_t max_units,
                      std::vector<uint32_t>& out);

// Changes IC(0) factor values in place after the factorisation (the learned
// preconditioner): L holds rows with the diagonal last, diag the diagonal.
struct Ic0Correction
{
    virtual ~Ic0Correction() = default;
    virtual void correct(b2s_ctx* ctx, const CsrDev& A, const uint32_t* Lrp, const uint32_t* Lci, uint32_t Lnnz,
                         double* Lv, double* diag) = 0;
};
std::unique_ptr<PcImpl> make_pc_ic0_ex(b2s_ctx* ctx, const CsrDev& A, const b2s_pc_opts& o, Ic0Correction* corr);

// preconditioner factories (one per file)
std::unique_ptr<PcImpl> make_pc_diag(b2s_ctx* ctx, const CsrDev& A);
std::unique_ptr<PcImpl> make_pc_identity(uint64_t n);
std::unique_ptr<PcImpl> make_pc_ic0(b2s_ctx* ctx, const CsrDev& A, const b2s_pc_opts& o);

// The reference's colouring and colour-by-colour renumbering of a square
// CSR matrix (multicolour SSOR and red-black SOR): colour c owns the new rows
// [h_cptr[c], h_cptr[c+1]); row ni of A2 is row perm[ni] of A with columns
// new_id[] sorted; d2 its diagonal (MISSING_DIAG when absent or < 1e-300).
struct RedBlack
{
    uint32_t n = 0, ncolor = 0;
    std::vector<uint32_t> h_cptr, h_new_id;
    DBuf<uint32_t> perm, new_id, rp2, ci2;
    DBuf<double> v2, d2;
};
void build_redblack(b2s_ctx* ctx, const CsrDev& A, RedBlack& rb, const char* what);
std::unique_ptr<PcImpl> make_pc_ilu0(b2s_ctx* ctx, const CsrDev& A, const b2s_pc_opts& o);
std::unique_ptr<PcImpl> make_pc_ssor(b2s_ctx* ctx, const CsrDev& A, const b2s_pc_opts& o);
std::unique_ptr<PcImpl> make_pc_amg_csr(b2s_ctx* ctx, const CsrDev& A, const b2s_pc_opts& o);
// C = A B and T = A^T for bs = 1 operators on the device (amg.cu): sorted
// columns, sums in the reference's order (SMatrix::operator*,
// array.cpp:2336-2447; SMatrix::transpose, array.cpp:2201-2234)
void scalar_matmul(b2s_ctx* ctx, const BaijDev& A, const BaijDev& B, BaijDev& C);
void scalar_transpose(b2s_ctx* ctx, const BaijDev& A, BaijDev& T);

std::unique_ptr<PcImpl> make_pc_amg_baij(b2s_ctx* ctx, const BaijDev& A, const b2s_pc_opts& o);
std::unique_ptr<PcImpl> make_pc_bjacobi(b2s_ctx* ctx, const BaijDev& A);
std::unique_ptr<PcImpl> make_pc_bilu0(b2s_ctx* ctx, const BaijDev& A, const b2s_pc_opts& o);
std::unique_ptr<PcImpl> make_pc_learned_ic0(b2s_ctx* ctx, const CsrDev& A, const b2s_pc_opts& o);
std::unique_ptr<PcImpl> make_pc_host(uint64_t n, b2s_host_pc_fn fn, void* user);

}  // namespace b2s
