// IC(0) and ILU(0) preconditioners: factorisation and triangular solves on the
// GPU.
//   make_ic0_preconditioner  array.cpp:2522-2732
//   make_ilu0_preconditioner array.cpp:2744-2934
//
// Setup (all on the device):
//   1. split the pattern of A (L incl. diagonal for IC(0); strict L and U incl.
//      diagonal for ILU(0)) with a count / scan / fill;
//   2. level sets of the factor's dependency DAG: level[i] = 1 + max level of
//      the rows row i reads, computed by one sync-free traversal, then rows
//      sorted by (level, index) with a stable radix sort;
//   3. the factorisation, one launch per level, one thread per row, each row
//      computed with exactly the reference's loop (two-pointer merges, same
//      order of operations) -- the factors equal the reference's bit for bit;
//   4. IC(0): L^T (strict part) by a device transpose whose rows are then
//      sorted, and the level sets of the upper solve.
// Apply: forward and backward substitution, either one launch per level
// (B2S_TRSV_LEVEL) or one sync-free launch per triangle (B2S_TRSV_SYNCFREE);
// both evaluate every row in the reference's order, so the FP64 apply equals
// the reference's bit for bit.  With B2S_FP32 the factor values and the
// intermediate vectors are FP32 (FP32 accumulation); the factorisation itself
// stays FP64.
#include <algorithm>

#include "trisolve.cuh"
#include "trsv_chunk.cuh"
#include "trsv_band.cuh"
#include "pcg_band.cuh"
#include "pcg_tile.cuh"
#include "trsv_grid5.cuh"
#include "trsv_grid7.cuh"

#include <cstdlib>
#include <cstring>
#include <exception>
#include <thread>

namespace b2s {

// ------------------------------------------------------------ pattern split

// mode 0: keep j <= i (IC(0) L); mode 1: j < i (ILU(0) L); mode 2: j >= i (ILU(0) U)
__global__ void k_split_count(uint32_t n, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci, int mode,
                              uint32_t* __restrict__ cnt)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        uint32_t c = 0;
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
        {
            const uint32_t j = ci[p];
            c += mode == 0 ? (j <= i) : mode == 1 ? (j < i) : (j >= i);
        }
        cnt[i] = c;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt[n] = 0;
}

__global__ void k_split_fill(uint32_t n, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                             const double* __restrict__ v, int mode, const uint32_t* __restrict__ orp,
                             uint32_t* __restrict__ oci, double* __restrict__ ov, uint32_t* __restrict__ dpos,
                             unsigned long long* err)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        uint32_t d = orp[i];
        bool has_diag = false;
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
        {
            const uint32_t j = ci[p];
            const bool keep = mode == 0 ? (j <= i) : mode == 1 ? (j < i) : (j >= i);
            if (!keep) continue;
            if (j == i)
            {
                has_diag = true;
                if (dpos) dpos[i] = d;
            }
            oci[d] = j;
            ov[d] = v[p];
            ++d;
        }
        if (mode != 1 && !has_diag) atomicMin(err, ((unsigned long long)i << 8) | B2S_MISSING_DIAG);
    }
}

struct Csr32
{
    uint32_t n = 0, nnz = 0;
    DBuf<uint32_t> rp, ci;
    DBuf<double> v;
    DBuf<float> v32;
    std::vector<uint32_t> h_rp;
};

static void split(b2s_ctx* ctx, const CsrDev& A, int mode, Csr32& out, uint32_t* dpos, unsigned long long* err)
{
    const uint32_t n = A.n;
    DBuf<uint32_t> cnt(n + 1);
    B2S_LAUNCH(ctx, k_split_count, stream_grid(ctx, n), kThreads, 0, n, A.rp.p, A.ci.p, mode, cnt.p);
    out.n = n;
    out.rp.alloc(n + 1);
    out.nnz = exclusive_scan(ctx, cnt.p, out.rp.p, n);
    out.ci.alloc(out.nnz ? out.nnz : 1);
    out.v.alloc(out.nnz ? out.nnz : 1);
    B2S_LAUNCH(ctx, k_split_fill, stream_grid(ctx, n), kThreads, 0, n, A.rp.p, A.ci.p, A.v.p, mode, out.rp.p,
               out.ci.p, out.v.p, dpos, err);
}

static void check_err(b2s_ctx* ctx, DBuf<unsigned long long>& err, const char* what)
{
    unsigned long long e = 0;
    d2h(ctx, &e, err.p, sizeof(e));
    sync(ctx);
    if (e != ~0ull)
    {
        const uint32_t row = (uint32_t)(e >> 8);
        const b2s_status st = (b2s_status)(e & 0xff);
        std::string msg = std::string(what) + ": ";
        switch (st)
        {
            case B2S_MISSING_DIAG: msg += "missing diagonal entry"; break;
            case B2S_NOT_SPD: msg += "matrix may not be SPD (pivot <= 1e-14)"; break;
            case B2S_ZERO_PIVOT: msg += "breakdown: U_kk close to zero"; break;
            default: msg += b2s_status_name(st);
        }
        fail(st, msg + " at row " + std::to_string(row));
    }
}

// ------------------------------------------------------------ factorisation

// IC(0) row, array.cpp:2577-2655
// IC(0) of row i in place (array.cpp:2560-2660): l_ij = (a_ij - sum_k l_ik l_jk) / l_jj
// for the strict entries in column order, then l_ii = sqrt(a_ii - sum_k l_ik^2);
// rows j < i must be final.  A missing diagonal or a pivot <= 1e-14 records
// (i << 8 | status) in *err (the smallest row wins) and leaves diag[i] = 1.
__device__ __forceinline__ void ic0_row(uint32_t i, const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Lci,
                                        double* Lv, double* diag, unsigned long long* err)
{
    const uint32_t rs = Lrp[i], re = Lrp[i + 1];
    for (uint32_t p = rs; p < re; ++p)
    {
        const uint32_t j = Lci[p];
        if (j >= i) break;
        double sum = 0.0;
        uint32_t pi = rs, pj = Lrp[j];
        const uint32_t ej = Lrp[j + 1];
        while (pi < p && pj < ej)
        {
            const uint32_t ki = Lci[pi], kj = Lci[pj];
            if (ki == kj)
            {
                sum += Lv[pi] * Lv[pj];
                ++pi;
                ++pj;
            }
            else if (ki < kj)
                ++pi;
            else
                ++pj;
        }
        Lv[p] = (Lv[p] - sum) / diag[j];
    }
    uint32_t dp = re;
    for (uint32_t p = rs; p < re; ++p)
        if (Lci[p] == i)
        {
            dp = p;
            break;
        }
    if (dp == re)
    {
        atomicMin(err, ((unsigned long long)i << 8) | B2S_MISSING_DIAG);
        diag[i] = 1.0;
        return;
    }
    double sd = 0.0;
    for (uint32_t p = rs; p < dp; ++p) sd += Lv[p] * Lv[p];
    const double dv = Lv[dp] - sd;
    if (!(dv > 1e-14))
    {
        atomicMin(err, ((unsigned long long)i << 8) | B2S_NOT_SPD);
        diag[i] = 1.0;
        return;
    }
    Lv[dp] = sqrt(dv);
    diag[i] = Lv[dp];
}

__global__ void k_ic0_level(const uint32_t* __restrict__ rows, uint32_t count, const uint32_t* __restrict__ Lrp,
                            const uint32_t* __restrict__ Lci, double* Lv, double* diag, unsigned long long* err)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    ic0_row(rows[t], Lrp, Lci, Lv, diag, err);
}

// Fixed-point IC(0) (Chow and Patel, "Fine-grained parallel incomplete LU
// factorization", SIAM J. Sci. Comput. 37 (2015)): every entry of L is
// recomputed from the previous sweep's values,
//   l_ij = (a_ij - sum_{k<j} l_ik l_jk) / l_jj   (j < i),
//   l_ii = sqrt(a_ii - sum_{k<i} l_ik^2),
// the sums over the common columns in column order (the exact row
// factorisation's arithmetic, so a sweep count above the dependency depth
// reproduces it bit for bit).  Sweep 0 starts from l_ij = a_ij / sqrt(a_jj),
// l_ii = sqrt(a_ii).  Rows hold the diagonal last (tril of a matrix with a
// full diagonal; checked by k_ic0_par_init).
__global__ void k_ic0_par_init(uint32_t n, const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Lci,
                               const double* __restrict__ a, double* __restrict__ l, unsigned long long* err)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const uint32_t rs = Lrp[i], re = Lrp[i + 1];
        if (re == rs || Lci[re - 1] != i)
        {
            atomicMin(err, ((unsigned long long)i << 8) | B2S_MISSING_DIAG);
            for (uint32_t p = rs; p < re; ++p) l[p] = 0.0;
            continue;
        }
        for (uint32_t p = rs; p < re; ++p)
        {
            const uint32_t j = Lci[p];
            const double ajj = a[Lrp[j + 1] - 1];
            l[p] = j == i ? sqrt(fabs(a[p])) : a[p] / sqrt(fabs(ajj));
        }
    }
}

__global__ void k_ic0_par_sweep(uint32_t n, const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Lci,
                                const double* __restrict__ a, const double* __restrict__ lin,
                                double* __restrict__ lout)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const uint32_t rs = Lrp[i], re = Lrp[i + 1];
        for (uint32_t p = rs; p < re; ++p)
        {
            const uint32_t j = Lci[p];
            if (j < i)
            {
                double sum = 0.0;
                uint32_t pi = rs, pj = Lrp[j];
                const uint32_t ej = Lrp[j + 1];
                while (pi < p && pj < ej)
                {
                    const uint32_t ki = Lci[pi], kj = Lci[pj];
                    if (ki == kj)
                    {
                        sum += lin[pi] * lin[pj];
                        ++pi;
                        ++pj;
                    }
                    else if (ki < kj)
                        ++pi;
                    else
                        ++pj;
                }
                lout[p] = (a[p] - sum) / lin[ej - 1];
            }
            else
            {
                double sd = 0.0;
                for (uint32_t q = rs; q < p; ++q) sd += lin[q] * lin[q];
                const double dv = a[p] - sd;
                lout[p] = dv > 0.0 ? sqrt(dv) : 0.0;  // a non-positive pivot is caught after the last sweep
            }
        }
    }
}

// after the last sweep: diag[i] = l_ii, a pivot <= 1e-14 (or NaN) is NOT_SPD
__global__ void k_ic0_par_finish(uint32_t n, const uint32_t* __restrict__ Lrp, const double* __restrict__ l,
                                 double* __restrict__ diag, unsigned long long* err)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const double d = l[Lrp[i + 1] - 1];
        if (!(d * d > 1e-14))
        {
            atomicMin(err, ((unsigned long long)i << 8) | B2S_NOT_SPD);
            diag[i] = 1.0;
        }
        else
            diag[i] = d;
    }
}

// The whole factorisation in one CTA when every level is narrow: the CTA
// walks the levels in order, its threads take a level's rows, and a
// __syncthreads separates the levels (the block barrier orders the global
// writes of one level before the reads of the next).  No launch per level
// and no cross-CTA waits.
constexpr uint32_t kIc0OneCtaThreads = 1024;
constexpr uint32_t kIc0OneCtaMaxWidth = 4 * kIc0OneCtaThreads;

__global__ void __launch_bounds__(kIc0OneCtaThreads) k_ic0_one_cta(const uint32_t* __restrict__ rows,
                                                                  const uint32_t* __restrict__ lptr, uint32_t nlev,
                                                                  const uint32_t* __restrict__ Lrp,
                                                                  const uint32_t* __restrict__ Lci, double* Lv,
                                                                  double* diag, unsigned long long* err)
{
    for (uint32_t l = 0; l < nlev; ++l)
    {
        const uint32_t a = lptr[l], b = lptr[l + 1];
        for (uint32_t t = a + threadIdx.x; t < b; t += blockDim.x) ic0_row(rows[t], Lrp, Lci, Lv, diag, err);
        __syncthreads();
    }
}

// ILU(0) row, array.cpp:2840-2898 (IKJ; fill-in dropped)
__global__ void k_ilu0_level(const uint32_t* __restrict__ rows, uint32_t count, const uint32_t* __restrict__ Lrp,
                             const uint32_t* __restrict__ Lci, double* Lv, const uint32_t* __restrict__ Urp,
                             const uint32_t* __restrict__ Uci, double* Uv, const uint32_t* __restrict__ dix,
                             unsigned long long* err)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const uint32_t i = rows[t];
    const uint32_t us = Urp[i], ue = Urp[i + 1];
    for (uint32_t pl = Lrp[i]; pl < Lrp[i + 1]; ++pl)
    {
        const uint32_t k = Lci[pl];
        const double ukk = Uv[dix[k]];
        if (fabs(ukk) < 1e-30)
        {
            atomicMin(err, ((unsigned long long)i << 8) | B2S_ZERO_PIVOT);
            return;
        }
        Lv[pl] /= ukk;
        uint32_t pi = us, pk = Urp[k];
        const uint32_t ek = Urp[k + 1];
        while (pi < ue && pk < ek)
        {
            const uint32_t ji = Uci[pi], jk = Uci[pk];
            if (ji == jk)
            {
                Uv[pi] -= Lv[pl] * Uv[pk];
                ++pi;
                ++pk;
            }
            else if (ji < jk)
                ++pi;
            else
                ++pk;
        }
    }
}

// ------------------------------------------------------------ transpose

__global__ void k_tr_count(uint32_t n, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                           uint32_t* __restrict__ cnt)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
            if (ci[p] < i) atomicAdd(&cnt[ci[p]], 1u);
}

// strict lower part of L -> its transpose (strict upper) as sorted CSR: a
// stable sort of L's strict entries by column gives each row of the transpose
// its columns in ascending order
__global__ void k_strict_flag(uint32_t n, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                              uint32_t* __restrict__ key)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p) key[p] = ci[p] < i ? ci[p] : n;  // diagonal entries sort last
}

__global__ void k_tr_gather(uint32_t nnz, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ row_of,
                            const double* __restrict__ v, uint32_t* __restrict__ tci, double* __restrict__ tv)
{
    for (uint32_t d = blockIdx.x * blockDim.x + threadIdx.x; d < nnz; d += gridDim.x * blockDim.x)
    {
        const uint32_t p = perm[d];
        tci[d] = row_of[p];
        tv[d] = v[p];
    }
}

static void transpose_strict(b2s_ctx* ctx, const Csr32& L, Csr32& T)
{
    const uint32_t n = L.n;
    DBuf<uint32_t> cnt(n + 1);
    B2S_CUDA(cudaMemsetAsync(cnt.p, 0, cnt.bytes(), ctx->stream));
    B2S_LAUNCH(ctx, k_tr_count, stream_grid(ctx, n), kThreads, 0, n, L.rp.p, L.ci.p, cnt.p);
    T.n = n;
    T.rp.alloc(n + 1);
    T.nnz = exclusive_scan(ctx, cnt.p, T.rp.p, n);
    T.ci.alloc(T.nnz ? T.nnz : 1);
    T.v.alloc(T.nnz ? T.nnz : 1);
    if (!T.nnz) return;
    // sort keys: the column of a strict entry, n for a diagonal one (those land after all strict entries)
    DBuf<uint32_t> key(L.nnz ? L.nnz : 1), perm, row_of;
    B2S_LAUNCH(ctx, k_strict_flag, stream_grid(ctx, n), kThreads, 0, n, L.rp.p, L.ci.p, key.p);
    transpose_order(ctx, n, n + 1, L.rp.p, key.p, L.nnz, perm, row_of);
    B2S_LAUNCH(ctx, k_tr_gather, stream_grid(ctx, T.nnz), kThreads, 0, T.nnz, perm.p, row_of.p, L.v.p, T.ci.p, T.v.p);
}

// ------------------------------------------------------------ triangular solves

template <typename T>
__device__ __forceinline__ T ld_dep(const T* p)
{
    return __ldcg(p);
}

// One row of a triangular solve:  x_i = (rhs_i - sum_{deps j} V_ij x_j) [/ d_i]
// in the row's column order.  VT: factor storage, XT: solution / accumulation
// type, RT: right-hand-side type.  out64 (optional) receives x as FP64.
template <bool LOWER, bool UNIT, typename VT, typename XT, typename RT>
struct TrsvOp
{
    const uint32_t *rp, *ci;
    const VT* v;
    const VT* d;
    const RT* rhs;
    XT* x;
    double* out64;
    __device__ bool ready(uint32_t row, const uint32_t* flags, uint32_t epoch) const
    {
        return deps_ready<LOWER>(row, rp, ci, flags, epoch);
    }
    template <bool SYNCFREE>
    __device__ __forceinline__ void row_compute(uint32_t row) const
    {
        XT sum = (XT)rhs[row];
        const uint32_t a = __ldg(&rp[row]), b = __ldg(&rp[row + 1]);
        for (uint32_t p = a; p < b; ++p)
        {
            const uint32_t j = __ldg(&ci[p]);
            if (LOWER ? (j < row) : (j > row))
            {
                const XT xj = SYNCFREE ? ld_dep(&x[j]) : x[j];
                sum -= (XT)__ldg(&v[p]) * xj;
            }
        }
        const XT r = UNIT ? sum : sum / (XT)__ldg(&d[row]);
        x[row] = r;
        if (out64) out64[row] = (double)r;
    }
    __device__ void compute(uint32_t row) const { row_compute<true>(row); }
};

// D^-1 a in a Jacobi sweep: FP64 divides (the exact solves' arithmetic, so
// enough sweeps reproduce them bit for bit); FP32 multiplies by the FP32
// reciprocal 1/d, the value the banded kernel packs.
template <typename XT>
__device__ __forceinline__ XT jacobi_scale(XT a, XT d)
{
    if constexpr (sizeof(XT) == 4)
        return a * (1.f / d);
    else
        return a / d;
}

// One pass of the sweep schedule (B2S_TRSV_JACOBI) over a triangle T = D + N,
// one thread per segment of S consecutive rows (global index / S), rows in
// dependency order inside the segment:
//   y[i] = D^-1 (rhs_i - sum_{j in segment} N_ij y[j] - sum_{j outside} N_ij yin[j]),
// the strict entries in column order; pass 0 has no yin (each segment solved
// on its own), passes 1..k are the sweeps.  S = 1 is plain Jacobi.
template <bool LOWER, bool UNIT, typename VT, typename XT, typename RT>
__global__ void __launch_bounds__(kThreads) k_trsv_sweep(uint32_t n, uint32_t S, int pass,
                                                         const uint32_t* __restrict__ rp,
                                                         const uint32_t* __restrict__ ci, const VT* __restrict__ v,
                                                         const VT* __restrict__ d, const RT* __restrict__ rhs,
                                                         const XT* __restrict__ yin, XT* yout,
                                                         double* __restrict__ out64, const int* done)
{
    if (done && *done) return;
    const uint32_t nseg = (n + S - 1) / S;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < nseg; g += gridDim.x * blockDim.x)
    {
        const uint32_t a = g * S, b = min(n, a + S);
        for (uint32_t u = 0; u < b - a; ++u)
        {
            const uint32_t row = LOWER ? a + u : b - 1 - u;
            XT sum = (XT)rhs[row];
            const uint32_t p0 = __ldg(&rp[row]), p1 = __ldg(&rp[row + 1]);
            for (uint32_t p = p0; p < p1; ++p)
            {
                const uint32_t j = __ldg(&ci[p]);
                if (!(LOWER ? (j < row) : (j > row))) continue;
                XT xj;
                if (j >= a && j < b)
                    xj = yout[j];  // this pass, written above by this thread
                else if (pass > 0)
                    xj = yin[j];
                else
                    continue;
                sum -= (XT)__ldg(&v[p]) * xj;
            }
            const XT r = UNIT ? sum : jacobi_scale<XT>(sum, (XT)__ldg(&d[row]));
            yout[row] = r;
            if (out64) out64[row] = (double)r;
        }
    }
}

// A triangular factor ready for solves: CSR rows + divisor + schedule.
struct Tri
{
    bool lower = true, unit = false;
    uint32_t n = 0;
    const Csr32* m = nullptr;
    const double* d64 = nullptr;
    const float* d32 = nullptr;
    LevelSchedule sched;
    SyncFree sf;
    ChunkSchedule cs;
    Grid5Tri g5;  // 5-point grid factors: the exact solve with a lane per grid line
    Grid7Tri g7;  // 7-point grid factors: the same with planes handed on
    bool has_chunks = false, sched_ready = false;
    std::vector<uint32_t> h_level;  // host copy of the rows' levels (compute_levels), when known
    int sweeps = 8;                 // B2S_TRSV_JACOBI: sweeps after pass 0
    uint32_t segment = 8;           // rows per Gauss-Seidel segment
    DBuf<double> jw64[2];           // sweep ping-pong buffers, made at setup
    DBuf<float> jw32[2];
    BandPlan band;                  // FP32 banded triangles: all sweeps in one launch
    DBuf<uint16_t> band_off;        // packed strict entries and reciprocals (k_band_pack)
    DBuf<float> band_val, band_dinv;

    // plan: the triangle's band plan (plan_band), usable for FP32 factors
    void prepare_sweeps(b2s_ctx* ctx, int k, uint32_t seg, bool fp32, const BandPlan* plan)
    {
        sweeps = k;
        segment = seg;
        if (fp32 && plan) band = *plan;
        if (band.T)
        {
            reserve_reduction(ctx, band.ntiles);  // the fused r.z of apply_rz
            band_off.alloc((size_t)band.W * n);
            band_val.alloc((size_t)band.W * n);
            band_dinv.alloc(n);
            return;
        }
        for (int b = 0; b < 2; ++b)
        {
            if (fp32)
                jw32[b].alloc(n ? n : 1);
            else
                jw64[b].alloc(n ? n : 1);
        }
    }

    template <bool LOWER, typename RT, bool RZ = false, bool UPD = false>
    void run_band(b2s_ctx* ctx, const RT* rhs, float* x, double* out64, const int* done, BandRz rz = BandRz(),
                  BandUpd up = BandUpd())
    {
        if (band.W == 2)
        {
            auto kern = segment == 1 ? k_trsv_band<LOWER, 2, 1, RT, RZ, UPD> : k_trsv_band<LOWER, 2, 8, RT, RZ, UPD>;
            B2S_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)band.smem));
            B2S_LAUNCH(ctx, kern, band.ntiles, band_threads(2), band.smem, n, band.T, band.B, band.Rmax, sweeps,
                       band_off.p, band_val.p, band_dinv.p, rhs, x, out64, done, rz, up);
        }
        else
        {
            auto kern = segment == 1 ? k_trsv_band<LOWER, 4, 1, RT, RZ, UPD> : k_trsv_band<LOWER, 4, 8, RT, RZ, UPD>;
            B2S_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)band.smem));
            B2S_LAUNCH(ctx, kern, band.ntiles, band_threads(4), band.smem, n, band.T, band.B, band.Rmax, sweeps,
                       band_off.p, band_val.p, band_dinv.p, rhs, x, out64, done, rz, up);
        }
    }

    template <bool LOWER, bool UNIT, typename VT, typename XT, typename RT>
    void run_sweeps(b2s_ctx* ctx, const VT* v, const VT* d, const RT* rhs, XT* x, double* out64, const int* done)
    {
        if constexpr (sizeof(VT) == 4 && sizeof(XT) == 4)
        {
            if (band.T)
            {
                if (n) run_band<LOWER, RT>(ctx, rhs, x, out64, done);
                return;
            }
        }
        XT* buf[2];
        if constexpr (sizeof(XT) == 4)
            buf[0] = jw32[0].p, buf[1] = jw32[1].p;
        else
            buf[0] = jw64[0].p, buf[1] = jw64[1].p;
        need(buf[0] && buf[1], B2S_INVALID_ARG, "Jacobi triangular solve: sweep buffers not prepared");
        const unsigned g = stream_grid(ctx, ((uint64_t)n + segment - 1) / segment);
        for (int s = 0; s <= sweeps; ++s)
        {
            const bool last = s == sweeps;
            XT* out = last ? x : buf[s & 1];
            double* o64 = last ? out64 : nullptr;
            const XT* in = s ? buf[(s - 1) & 1] : nullptr;
            B2S_LAUNCH(ctx, (k_trsv_sweep<LOWER, UNIT, VT, XT, RT>), g, kThreads, 0, n, segment, s, m->rp.p, m->ci.p,
                       v, d, rhs, in, out, o64, done);
        }
    }

    template <bool LOWER, bool UNIT, typename VT, typename XT, typename RT>
    void run_t(b2s_ctx* ctx, int mode, const VT* v, const VT* d, const RT* rhs, XT* x, double* out64, const int* done)
    {
        if (mode == B2S_TRSV_JACOBI)
            run_sweeps<LOWER, UNIT, VT, XT, RT>(ctx, v, d, rhs, x, out64, done);
        else if (mode == B2S_TRSV_CHUNK && g5.usable<VT, XT>() && g5.packed_v == (const void*)v)
            g5.run<LOWER, UNIT, VT, XT, RT>(ctx, rhs, x, out64, done);
        else if (mode == B2S_TRSV_CHUNK && g7.usable<VT, XT>() && g7.packed_v == (const void*)v)
            g7.run<LOWER, UNIT, VT, XT, RT>(ctx, rhs, x, out64, done);
        else if (mode == B2S_TRSV_CHUNK && has_chunks && cs.usable<VT, XT, RT>())
            cs.run<LOWER, UNIT, VT, XT, RT>(ctx, v, d, rhs, x, out64, done);
        else
            run_schedule(ctx, mode == B2S_TRSV_LEVEL ? B2S_TRSV_LEVEL : B2S_TRSV_SYNCFREE, sched, sf,
                         TrsvOp<LOWER, UNIT, VT, XT, RT>{m->rp.p, m->ci.p, v, d, rhs, x, out64}, done);
    }

    // x = T^-1 rhs; precision per the type parameters.  With out64 the results
    // also go there in FP64, and the grid schedules then leave x unwritten
    // (an FP32 x is scratch for every caller that passes out64)
    template <typename VT, typename XT, typename RT>
    void solve(b2s_ctx* ctx, int mode, const VT* v, const VT* d, const RT* rhs, XT* x, double* out64, const int* done)
    {
        if (lower && unit)
            run_t<true, true, VT, XT, RT>(ctx, mode, v, d, rhs, x, out64, done);
        else if (lower)
            run_t<true, false, VT, XT, RT>(ctx, mode, v, d, rhs, x, out64, done);
        else if (unit)
            run_t<false, true, VT, XT, RT>(ctx, mode, v, d, rhs, x, out64, done);
        else
            run_t<false, false, VT, XT, RT>(ctx, mode, v, d, rhs, x, out64, done);
    }

    void init(const Csr32& mat, bool lo, bool un)
    {
        m = &mat;
        lower = lo;
        unit = un;
        n = mat.n;
    }

    // level schedule: the factorisation, the level / sync-free solves and export use it
    void ensure_sched(b2s_ctx* ctx)
    {
        if (sched_ready) return;
        if (h_level.size() == n && n)
            sched.build_host(ctx, h_level);
        else
            sched.build(ctx, n, m->rp.p, m->ci.p, lower);
        sf.init(ctx, n);
        sched_ready = true;
    }

    // a host chunk plan -> device; falls back to the level schedule when no plan is usable
    void load_chunks(b2s_ctx* ctx, int mode, const ChunkPlan* plan, uint32_t vs)
    {
        has_chunks = mode == B2S_TRSV_CHUNK && n && plan && cs.load(ctx, *plan, vs);
        if (!has_chunks && mode != B2S_TRSV_JACOBI) ensure_sched(ctx);
    }

    // lay the final factor values out for the chunk schedule (no-op otherwise)
    template <typename VT>
    void pack(b2s_ctx* ctx, const VT* v, const VT* d)
    {
        if (has_chunks && sizeof(VT) <= cs.plan_vs) cs.pack<VT>(ctx, v, d);
        g5.pack<VT>(ctx, m->rp.p, m->ci.p, v, d, lower, unit);
        g7.pack<VT>(ctx, m->rp.p, m->ci.p, v, d, lower, unit);
        if constexpr (sizeof(VT) == 4)
        {
            if (band.T && n)
                B2S_LAUNCH(ctx, k_band_pack, stream_grid(ctx, n), kThreads, 0, n, band.W, lower ? 1 : 0,
                           unit ? 1 : 0, m->rp.p, m->ci.p, v, d, band_off.p, band_val.p, band_dinv.p);
        }
    }
};

// Host analysis of a factor pair, run on a host thread while the device
// factorises: the levels of the upper triangle and, for the chunk schedule,
// the chunk plans of both triangles.
struct HostAnalysis
{
    std::vector<uint32_t> up_rp, up_ci;  // upper pattern when it is derived on the host
    std::vector<uint32_t> up_level;
    ChunkPlan lo_plan, up_plan;
    BandPlan lo_band, up_band;
    TilePlan tiles;  // the tiled persistent PCG kernel's plan (sweep schedule, FP32)
    bool tiles_grid5 = false;        // a 5-point grid: the index blobs are built on the device
    std::vector<TileGeom> tile_geom;
    bool chunked = false;
    std::exception_ptr error;
    std::thread th;
    ~HostAnalysis()
    {
        if (th.joinable()) th.join();
    }
    void wait()
    {
        if (th.joinable()) th.join();
        if (error) std::rethrow_exception(error);
    }
};

// What the sweep schedules need of a lower factor's pattern (diagonal last in
// each row), computed on the device: the bandwidth B (largest i - j), the
// widest row and the widest column of the strict part, and whether the pattern
// is a 5-point grid's of row length B (is_grid5 in tile_plan.hpp).
struct PatternStats
{
    uint32_t B = 0, w_row = 0, w_col = 0;
    bool grid5 = false;
};

__global__ void k_pattern_stats(uint32_t n, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                uint32_t* __restrict__ colcnt, uint32_t* __restrict__ out)
{
    uint32_t B = 0, w = 0, wc = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        uint32_t c = 0;
        for (uint32_t q = rp[i]; q < rp[i + 1]; ++q)
        {
            const uint32_t j = ci[q];
            if (j < i)
            {
                ++c;
                B = max(B, i - j);
                wc = max(wc, atomicAdd(&colcnt[j], 1u) + 1u);
            }
        }
        w = max(w, c);
    }
    if (B) atomicMax(&out[0], B);
    if (w) atomicMax(&out[1], w);
    if (wc) atomicMax(&out[2], wc);
}

__global__ void k_pattern_grid5(uint32_t n, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                uint32_t B, uint32_t* __restrict__ bad)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const uint32_t x = i % B, y = i / B;
        const uint32_t e0 = rp[i], e1 = rp[i + 1];
        const uint32_t want = (y > 0) + (x > 0) + 1u;
        bool ok = e1 - e0 == want && ci[e1 - 1] == i;
        uint32_t e = e0;
        if (ok && y > 0) ok = ci[e++] == i - B;
        if (ok && x > 0) ok = ci[e] == i - 1;
        if (!ok) atomicExch(bad, 1u);
    }
}

static PatternStats pattern_stats(b2s_ctx* ctx, const Csr32& L)
{
    PatternStats ps;
    const uint32_t n = L.n;
    if (!n) return ps;
    DBuf<uint32_t> colcnt(n), out(4);
    B2S_CUDA(cudaMemsetAsync(colcnt.p, 0, colcnt.bytes(), ctx->stream));
    B2S_CUDA(cudaMemsetAsync(out.p, 0, out.bytes(), ctx->stream));
    const unsigned g = stream_grid(ctx, n);
    B2S_LAUNCH(ctx, k_pattern_stats, g, kThreads, 0, n, L.rp.p, L.ci.p, colcnt.p, out.p);
    uint32_t h[4] = {0, 0, 0, 0};
    d2h(ctx, h, out.p, 3 * sizeof(uint32_t));
    sync(ctx);
    ps.B = h[0];
    ps.w_row = h[1];
    ps.w_col = h[2];
    if (ps.B && n % ps.B == 0)
    {
        B2S_LAUNCH(ctx, k_pattern_grid5, g, kThreads, 0, n, L.rp.p, L.ci.p, ps.B, out.p + 3);
        d2h(ctx, h + 3, out.p + 3, sizeof(uint32_t));
        sync(ctx);
        ps.grid5 = h[3] == 0;
    }
    return ps;
}

// "trsv.grid5": sizes = {grid row length B (0: the grid schedule is off), lines, 1 when
// both triangles' coefficients are packed}
static void export_grid5(const Tri& fwd, const Tri& bwd, uint64_t* sizes)
{
    const bool on = fwd.g5.on && bwd.g5.on;
    sizes[0] = on ? fwd.g5.B : 0;
    sizes[1] = on ? fwd.g5.ny : 0;
    sizes[2] = on && fwd.g5.packed_v && bwd.g5.packed_v ? 1 : 0;
}

// "trsv.grid7": sizes = {B, ny, nz} of the 7-point grid schedule when both
// triangles take it (packed), else zeros
static void export_grid7(const Tri& fwd, const Tri& bwd, uint64_t* sizes)
{
    const bool on = fwd.g7.on && bwd.g7.on && fwd.g7.packed_v && bwd.g7.packed_v;
    sizes[0] = on ? fwd.g7.B : 0;
    sizes[1] = on ? fwd.g7.ny : 0;
    sizes[2] = on ? fwd.g7.nz : 0;
}

// the grid row length B of a lower triangle that is a 5-point grid's, else 0
static uint32_t grid5_lower_b(uint32_t n, const std::vector<uint32_t>& rp, const std::vector<uint32_t>& ci)
{
    uint32_t B = 0;
    for (uint32_t i = 0; i < n; ++i)
        if (rp[i + 1] > rp[i] && ci[rp[i]] < i) B = std::max(B, i - ci[rp[i]]);
    return B && grid5_triangle(n, rp.data(), ci.data(), B, true) ? B : 0u;
}

// The grid schedule that the exact solves of a factor take, found from L's
// pattern before any planning (a factor that takes one needs no chunk plans);
// ILU(0) passes U's pattern to be checked too (IC(0)'s L^T is the grid's).
struct GridShape
{
    uint32_t b5 = 0, d7[3] = {0, 0, 0};
    bool any() const { return b5 || d7[0]; }
};
static GridShape grid_shape(uint32_t n, const std::vector<uint32_t>& lrp, const std::vector<uint32_t>& lci,
                            const std::vector<uint32_t>* urp, const std::vector<uint32_t>* uci)
{
    GridShape g;
    if (!n) return g;
    if (const uint32_t B = grid5_lower_b(n, lrp, lci))
    {
        if (Grid5Tri::fits(B, n / B) && (!urp || grid5_triangle(n, urp->data(), uci->data(), B, false))) g.b5 = B;
        return g;
    }
    uint32_t d[3];
    grid7_dims(n, lrp.data(), lci.data(), d);
    if (d[0] && Grid7Tri::fits(d[0], d[1], d[2]) &&
        (!urp || grid7_triangle(n, urp->data(), uci->data(), d[0], d[1], false)))
        std::copy(d, d + 3, g.d7);
    return g;
}
static void enable_grid(Tri& fwd, Tri& bwd, const GridShape& g, uint32_t n)
{
    if (g.b5)
    {
        fwd.g5.enable(g.b5, n / g.b5);
        bwd.g5.enable(g.b5, n / g.b5);
    }
    else if (g.d7[0])
    {
        fwd.g7.enable(g.d7[0], g.d7[1], g.d7[2]);
        bwd.g7.enable(g.d7[0], g.d7[1], g.d7[2]);
    }
}

static void copy_pattern(b2s_ctx* ctx, const Csr32& M, std::vector<uint32_t>& rp, std::vector<uint32_t>& ci)
{
    rp.resize((size_t)M.n + 1);
    ci.resize(M.nnz ? M.nnz : 1);
    d2h(ctx, rp.data(), M.rp.p, ((size_t)M.n + 1) * sizeof(uint32_t));
    d2h(ctx, ci.data(), M.ci.p, (size_t)M.nnz * sizeof(uint32_t));
    sync(ctx);
}

__global__ void k_f64_to_f32(const double* __restrict__ a, float* __restrict__ b, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

static void to_f32(b2s_ctx* ctx, const DBuf<double>& a, DBuf<float>& b, uint64_t n)
{
    b.alloc(n ? n : 1);
    if (n) B2S_LAUNCH(ctx, k_f64_to_f32, stream_grid(ctx, n), kThreads, 0, a.p, b.p, n);
}

// B2S_TRSV_JACOBI defaults: 8 sweeps of plain Jacobi (segments of one row).
// On the 512^2 benchmark systems 8-row Gauss-Seidel segments needed fewer
// sweeps for the same iterations but cost more per pass (a chain of dependent
// rows per thread), and were slower end to end.
static int sweep_count(const b2s_pc_opts& o) { return o.trsv_sweeps > 0 ? o.trsv_sweeps : 8; }
static uint32_t sweep_segment(const b2s_pc_opts& o) { return o.trsv_segment > 0 ? (uint32_t)o.trsv_segment : 1u; }

static int pick_trsv(const b2s_pc_opts& o)
{
    need(o.trsv >= B2S_TRSV_AUTO && o.trsv <= B2S_TRSV_JACOBI, B2S_INVALID_ARG, "unknown triangular-solve schedule");
    need(o.trsv_sweeps >= 0 && o.trsv_sweeps <= 1024, B2S_INVALID_ARG, "trsv_sweeps must be 0..1024");
    need(o.trsv_segment >= 0 && o.trsv_segment <= 32, B2S_INVALID_ARG, "trsv_segment must be 0..32");
    need(o.factor_sweeps >= 0 && o.factor_sweeps <= 1024, B2S_INVALID_ARG, "factor_sweeps must be 0..1024");
    return o.trsv == B2S_TRSV_AUTO ? B2S_TRSV_CHUNK : o.trsv;
}

static void export_csr(b2s_ctx* ctx, const Csr32& m, uint64_t* sizes, uint32_t* rp, uint32_t* ci, double* v)
{
    sizes[0] = (uint64_t)m.n + 1;
    sizes[1] = m.nnz;
    sizes[2] = m.nnz;
    if (rp) d2h(ctx, rp, m.rp.p, (m.n + 1) * sizeof(uint32_t));
    if (ci) d2h(ctx, ci, m.ci.p, m.nnz * sizeof(uint32_t));
    if (v) d2h(ctx, v, m.v.p, m.nnz * sizeof(double));
    sync(ctx);
}

static void export_levels(b2s_ctx* ctx, Tri& t, uint64_t* sizes, uint32_t* ci)
{
    t.ensure_sched(ctx);
    const LevelSchedule& s = t.sched;
    sizes[0] = 0;
    sizes[1] = s.n;
    sizes[2] = 0;
    if (ci) d2h(ctx, ci, s.level.p, s.n * sizeof(uint32_t));
    sync(ctx);
}

// ------------------------------------------------------------ IC(0)

namespace {

struct PcIC0 final : PcImpl
{
    uint32_t n = 0;
    int mode = B2S_TRSV_SYNCFREE;
    bool fp32 = false;
    Csr32 L, LT;
    DBuf<double> diag, y;
    DBuf<float> diag32, y32, z32;
    Tri fwd, bwd;

    void apply(b2s_ctx* ctx, const double* r, double* z, const int* done) override
    {
        if (!fp32)
        {
            fwd.solve<double, double, double>(ctx, mode, L.v.p, diag.p, r, y.p, nullptr, done);
            bwd.solve<double, double, double>(ctx, mode, LT.v.p, diag.p, y.p, z, nullptr, done);
        }
        else
        {
            fwd.solve<float, float, double>(ctx, mode, L.v32.p, diag32.p, r, y32.p, nullptr, done);
            bwd.solve<float, float, float>(ctx, mode, LT.v32.p, diag32.p, y32.p, z32.p, z, done);
        }
    }

    bool can_fuse_pcg() const override { return fp32 && mode == B2S_TRSV_JACOBI && fwd.band.T && bwd.band.T; }

    DBuf<unsigned> pcg_ctl;  // grid-barrier counter, error word

    // the tiled persistent PCG kernel (pcg_tile.cuh), when its plan was made
    // and A's pattern matched it
    bool tiles_ready = false;
    uint32_t tile_n = 0, tile_count = 0, tile_Q = 0, tile_smem = 0, tile_work = 0, tile_ystride = 0;
    bool tile_fused = false;  // the forward set grown from the upper set: two all-reduces per iteration
    DBuf<TileDesc> tile_desc;
    DBuf<uint8_t> tile_idx, tile_vals;
    DBuf<unsigned long long> tile_slots;

    // uploads the plan (a 5-point grid's index blobs are built on the device)
    // and packs the value blobs from A and the band arrays
    void load_tiles(b2s_ctx* ctx, const CsrDev& A, const TilePlan& P, const std::vector<TileGeom>* grid5)
    {
        tiles_ready = false;
        if (!P.ok || A.n != n) return;
        tile_desc = upload(ctx, P.desc);
        DBuf<int> bad(1);
        DBuf<TileGeom> geom;  // (held until the set-up's sync)
        B2S_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream));
        if (grid5)
        {
            const uint32_t B = P.B, ny = n / P.B;
            tile_idx.alloc(P.ibytes ? P.ibytes : 16);
            B2S_CUDA(cudaMemsetAsync(tile_idx.p, 0, tile_idx.bytes(), ctx->stream));  // the segments' padding
            geom = upload(ctx, *grid5);
            B2S_LAUNCH(ctx, k_tile_build_grid5, P.ntiles, kThreads, 0, tile_desc.p, geom.p, tile_idx.p, B, ny, P.k,
                       P.fused, bad.p);
        }
        else
            tile_idx = upload(ctx, P.idx.data(), P.idx.size());
        tile_vals.alloc(P.vbytes ? P.vbytes : 16);
        tile_slots.alloc(3ull * kTileSlotStride * P.ntiles);
        B2S_LAUNCH(ctx, k_tile_pack, P.ntiles, kThreads, 0, tile_desc.p, tile_idx.p, tile_vals.p, n, (int)P.k,
                   A.rp.p, A.ci.p, A.v.p, fwd.band_off.p, fwd.band_val.p, fwd.band_dinv.p, bwd.band_off.p,
                   bwd.band_val.p, bwd.band_dinv.p, bad.p);
        int hb = 0;
        d2h(ctx, &hb, bad.p, sizeof(int));
        sync(ctx);
        if (hb) return;  // A is not the structurally symmetric matrix of L's pattern: the banded kernel runs
        tile_n = n;
        tile_count = P.ntiles;
        tile_Q = P.Q;
        tile_smem = P.smem;
        tile_work = P.work;
        tile_ystride = ::b2s::tile_ystride(P.max_ext);
        tile_fused = P.fused;
        tiles_ready = true;
    }

    template <uint32_t Q, bool FUSED>
    bool launch_tiles(b2s_ctx* ctx, PcgTileArgs& a)
    {
        B2S_CUDA(cudaFuncSetAttribute(k_pcg_tile<Q, FUSED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)tile_smem));
        void* params[] = {&a};
        const cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_pcg_tile<Q, FUSED>, dim3(tile_count),
                                                          dim3(kTileThreads), params, tile_smem, ctx->stream);
        if (e == cudaErrorCooperativeLaunchTooLarge || e == cudaErrorNotSupported)
        {
            cudaGetLastError();
            return false;
        }
        B2S_CUDA(e);
        note_launch(ctx, "k_pcg_tile");
        return true;
    }

    // the whole PCG loop as one k_pcg_tile launch; false (nothing enqueued) when it cannot run
    bool pcg_tiles(b2s_ctx* ctx, const CsrDev& A, double* x, double* r0, double* r1, double* p0, double* p1,
                   double* z, double* Ap, KState* st, int stall_window)
    {
        if (!tiles_ready || A.n != tile_n || A.rp.p == nullptr || fwd.sweeps != bwd.sweeps) return false;
        if (!pcg_ctl.p) pcg_ctl.alloc(2);
        B2S_CUDA(cudaMemsetAsync(pcg_ctl.p, 0, 2 * sizeof(unsigned), ctx->stream));
        B2S_CUDA(cudaMemsetAsync(tile_slots.p, 0, tile_slots.bytes(), ctx->stream));
        PcgTileArgs a{};
        a.n = n;
        a.ntiles = tile_count;
        a.work = tile_work;
        a.ystride = tile_ystride;
        a.k = fwd.sweeps;
        a.desc = tile_desc.p;
        a.vals = reinterpret_cast<const uint4*>(tile_vals.p);
        a.idx = reinterpret_cast<const uint4*>(tile_idx.p);
        a.x = x;
        a.r[0] = r0;
        a.r[1] = r1;
        a.p[0] = p0;
        a.p[1] = p1;
        a.z = z;
        a.Ap = Ap;
        a.y32 = y32.p;
        a.slots = tile_slots.p;
        a.st = st;
        a.err = reinterpret_cast<int*>(pcg_ctl.p + 1);
        a.stall_window = stall_window;
        bool ok = false;
        switch (tile_Q * 2 + (tile_fused ? 1 : 0))
        {
            case 2: ok = launch_tiles<1, false>(ctx, a); break;
            case 3: ok = launch_tiles<1, true>(ctx, a); break;
            case 4: ok = launch_tiles<2, false>(ctx, a); break;
            case 5: ok = launch_tiles<2, true>(ctx, a); break;
            case 6: ok = launch_tiles<3, false>(ctx, a); break;
            case 7: ok = launch_tiles<3, true>(ctx, a); break;
            case 8: ok = launch_tiles<4, false>(ctx, a); break;
            case 9: ok = launch_tiles<4, true>(ctx, a); break;
            default: return false;
        }
        if (!ok) return false;
        int err = 0;
        d2h(ctx, &err, pcg_ctl.p + 1, sizeof(int));
        sync(ctx);
        if (err) fail(B2S_TIMEOUT, "persistent PCG: a tile's all-reduce wait gave up");
        return true;
    }

    bool pcg_persistent(b2s_ctx* ctx, const CsrDev& A, double* x, double* r0, double* r1, double* p0, double* p1,
                        double* z, double* Ap, KState* st, int stall_window, int which) override
    {
        if (can_fuse_pcg() && which == 0 && pcg_tiles(ctx, A, x, r0, r1, p0, p1, z, Ap, st, stall_window))
            return true;
        const BandPlan &lb = fwd.band, &ub = bwd.band;
        if (!(can_fuse_pcg() && fwd.segment == 1 && bwd.segment == 1 && lb.W == 2 && ub.W == 2 && lb.T == ub.T &&
              lb.B == ub.B && lb.Rmax == ub.Rmax && lb.ntiles == ub.ntiles && fwd.sweeps == bwd.sweeps &&
              A.n == n && n > 0 && lb.ntiles <= (uint32_t)ctx->sm_count && lb.T <= 3 * kPcgBandThreads))
            return false;
        if (!pcg_ctl.p) pcg_ctl.alloc(2);
        B2S_CUDA(cudaMemsetAsync(pcg_ctl.p, 0, 2 * sizeof(unsigned), ctx->stream));
        reserve_reduction(ctx, 3 * lb.ntiles);
        PcgBandArgs a{};
        a.n = n;
        a.T = lb.T;
        a.B = lb.B;
        a.Rmax = lb.Rmax;
        a.k = fwd.sweeps;
        a.Arp = A.rp.p;
        a.Aci = A.ci.p;
        a.Av = A.v.p;
        a.loff = fwd.band_off.p;
        a.lval = fwd.band_val.p;
        a.ldinv = fwd.band_dinv.p;
        a.uoff = bwd.band_off.p;
        a.uval = bwd.band_val.p;
        a.udinv = bwd.band_dinv.p;
        a.x = x;
        a.r[0] = r0;
        a.r[1] = r1;
        a.p[0] = p0;
        a.p[1] = p1;
        a.z = z;
        a.Ap = Ap;
        a.red = ctx->partial.p;
        a.y32 = y32.p;
        a.st = st;
        a.bar = pcg_ctl.p;
        a.err = reinterpret_cast<int*>(pcg_ctl.p + 1);
        a.stall_window = stall_window;
        const size_t smem = 2 * (size_t)lb.Rmax * sizeof(float);
        B2S_CUDA(cudaFuncSetAttribute(k_pcg_band, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        void* params[] = {&a};
        const cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_pcg_band, dim3(lb.ntiles),
                                                          dim3(kPcgBandThreads), params, smem, ctx->stream);
        if (e == cudaErrorCooperativeLaunchTooLarge || e == cudaErrorNotSupported)
        {
            cudaGetLastError();  // the CTAs could not all be resident: the caller iterates launch by launch
            return false;
        }
        B2S_CUDA(e);
        note_launch(ctx, "k_pcg_band");
        int err = 0;
        d2h(ctx, &err, pcg_ctl.p + 1, sizeof(int));
        sync(ctx);
        if (err) fail(B2S_TIMEOUT, "persistent PCG: a grid barrier wait gave up");
        return true;
    }

    void pcg_update_apply(b2s_ctx* ctx, double* x, const double* p, const double* Ap, const double* r_old,
                          double* r_new, double* z, KState* st, const int* done) override
    {
        fwd.run_band<true, double, false, true>(
            ctx, r_old, y32.p, nullptr, done, BandRz(),
            BandUpd{r_old, Ap, p, x, r_new, st, ctx->partial.p, ctx->counter.p});
        bwd.run_band<false, float, true>(ctx, y32.p, z32.p, z, done, BandRz{r_new, st, ctx->partial.p, ctx->counter.p});
    }

    bool apply_rz(b2s_ctx* ctx, const double* r, double* z, KState* st, const int* done) override
    {
        if (!(fp32 && mode == B2S_TRSV_JACOBI && fwd.band.T && bwd.band.T)) return false;
        fwd.run_band<true, double>(ctx, r, y32.p, nullptr, done);
        bwd.run_band<false, float, true>(ctx, y32.p, z32.p, z, done, BandRz{r, st, ctx->partial.p, ctx->counter.p});
        return true;
    }

    void solve_factor(b2s_ctx* ctx, bool upper, const double* in, double* out, const int* done) override
    {
        need(!fp32, B2S_UNSUPPORTED, "triangular factor solves need an FP64 IC(0)");
        if (upper)
            bwd.solve<double, double, double>(ctx, mode, LT.v.p, diag.p, in, out, nullptr, done);
        else
            fwd.solve<double, double, double>(ctx, mode, L.v.p, diag.p, in, out, nullptr, done);
    }

    void export_data(b2s_ctx* ctx, const std::string& what, uint64_t* sizes, uint32_t* rp, uint32_t* ci,
                     double* v) override
    {
        if (what == "ic0.L") return export_csr(ctx, L, sizes, rp, ci, v);
        if (what == "ic0.LT") return export_csr(ctx, LT, sizes, rp, ci, v);
        if (what == "ic0.diag")
        {
            sizes[0] = 0;
            sizes[1] = 0;
            sizes[2] = n;
            if (v) d2h(ctx, v, diag.p, n * sizeof(double));
            sync(ctx);
            return;
        }
        if (what == "levels.L") return export_levels(ctx, fwd, sizes, ci);
        if (what == "levels.U") return export_levels(ctx, bwd, sizes, ci);
        if (what == "trsv.grid5") return export_grid5(fwd, bwd, sizes);
        if (what == "trsv.grid7") return export_grid7(fwd, bwd, sizes);
        if (what == "pcg.tiles")  // the tiled persistent PCG kernel: tiles (0: not planned), rows per thread, smem
        {
            sizes[0] = tiles_ready ? tile_count : 0;
            sizes[1] = tiles_ready ? tile_Q : 0;
            sizes[2] = tiles_ready ? tile_smem : 0;
            return;
        }
        if (what == "pcg.tiles.idx")  // the tiles' index blobs as 32-bit words (ci)
        {
            sizes[0] = 0;
            sizes[1] = tiles_ready ? tile_idx.n / 4 : 0;
            sizes[2] = 0;
            if (ci && sizes[1]) d2h(ctx, ci, tile_idx.p, sizes[1] * 4);
            sync(ctx);
            return;
        }
        PcImpl::export_data(ctx, what, sizes, rp, ci, v);
    }
};

}  // namespace

// factor IC(0) on the pattern of tril(A) with values Lv (already placed);
// shared with the learned preconditioner, which factors corrected values.
// Narrow levels (at most kIc0OneCtaMaxWidth rows each): one CTA walks them
// all; otherwise one launch per level.  Every row is computed by ic0_row in
// level order either way, so the factor is the same bits.
void ic0_factor_inplace(b2s_ctx* ctx, const LevelSchedule& s, const uint32_t* Lrp, const uint32_t* Lci, double* Lv,
                        double* diag, const char* what)
{
    DBuf<unsigned long long> err(1);
    const unsigned long long none = ~0ull;
    h2d(ctx, err.p, &none, sizeof(none));
    uint32_t width = 0;
    for (uint32_t l = 0; l < s.nlev; ++l) width = std::max(width, s.h_ptr[l + 1] - s.h_ptr[l]);
    if (s.nlev && width <= kIc0OneCtaMaxWidth)
    {
        auto lptr = upload(ctx, s.h_ptr);
        B2S_LAUNCH(ctx, k_ic0_one_cta, 1, kIc0OneCtaThreads, 0, s.rows.p, lptr.p, s.nlev, Lrp, Lci, Lv, diag, err.p);
        check_err(ctx, err, what);  // synchronises before lptr is released
        return;
    }
    for (uint32_t l = 0; l < s.nlev; ++l)
    {
        const uint32_t a = s.h_ptr[l], cnt = s.h_ptr[l + 1] - a;
        B2S_LAUNCH(ctx, k_ic0_level, (cnt + kThreads - 1) / kThreads, kThreads, 0, s.rows.p + a, cnt, Lrp, Lci, Lv,
                   diag, err.p);
    }
    check_err(ctx, err, what);
}

// k fixed-point sweeps on L (values: tril(A) in, the approximate factor
// out).  False when a pivot failed (the caller then factors exactly from the
// saved tril(A)); other failures throw like the exact factorisation.
static bool ic0_factor_fixed_point(b2s_ctx* ctx, Csr32& L, double* diag, int k, const DBuf<double>& a)
{
    const uint32_t n = L.n;
    DBuf<unsigned long long> err(1);
    const unsigned long long none = ~0ull;
    h2d(ctx, err.p, &none, sizeof(none));
    DBuf<double> tmp(L.nnz ? L.nnz : 1);
    const unsigned g = stream_grid(ctx, n);
    // ping-pong so that the last sweep lands in L.v
    double* buf[2] = {L.v.p, tmp.p};
    int cur = (k & 1) ? 1 : 0;
    B2S_LAUNCH(ctx, k_ic0_par_init, g, kThreads, 0, n, L.rp.p, L.ci.p, a.p, buf[cur], err.p);
    for (int s = 0; s < k; ++s)
    {
        B2S_LAUNCH(ctx, k_ic0_par_sweep, g, kThreads, 0, n, L.rp.p, L.ci.p, a.p, buf[cur], buf[cur ^ 1]);
        cur ^= 1;
    }
    B2S_LAUNCH(ctx, k_ic0_par_finish, g, kThreads, 0, n, L.rp.p, L.v.p, diag, err.p);
    unsigned long long e = 0;
    d2h(ctx, &e, err.p, sizeof(e));
    sync(ctx);
    if (e == ~0ull) return true;
    if ((e & 0xff) == B2S_NOT_SPD) return false;
    check_err(ctx, err, "IC(0) failed");  // MISSING_DIAG: the exact factorisation's error
    return false;
}

std::unique_ptr<PcImpl> make_pc_ic0_ex(b2s_ctx* ctx, const CsrDev& A, const b2s_pc_opts& o, Ic0Correction* corr)
{
    need(A.n == A.m, B2S_SHAPE, "IC(0) needs a square matrix");
    auto pc = std::make_unique<PcIC0>();
    const uint32_t n = A.n;
    pc->n = n;
    pc->mode = pick_trsv(o);
    pc->fp32 = o.precision != B2S_FP64;
    const uint32_t vs = pc->fp32 ? 4 : 8;
    DBuf<unsigned long long> err(1);
    const unsigned long long none = ~0ull;
    h2d(ctx, err.p, &none, sizeof(none));
    split(ctx, A, 0, pc->L, nullptr, err.p);
    check_err(ctx, err, "IC(0) failed");
    pc->diag.alloc(n ? n : 1);
    // Host analysis of L.  The exact schedules need the levels of both
    // triangles (and the chunk plans); the sweep schedule needs only the band
    // plans.  What the factorisation does not need runs on a host thread
    // while the device factorises.
    const bool sweeps = pc->mode == B2S_TRSV_JACOBI;
    const int nsweeps = sweep_count(o);
    const uint32_t seg = sweep_segment(o);
    const int fsweeps = o.factor_sweeps;
    // The host copy of L's pattern feeds the level schedules and the chunk and
    // breadth-first tile planners.  The sweep schedule over a fixed-point factor
    // needs none of them: its band plans and the 5-point grid test come from
    // statistics reduced on the device (a few words back instead of the pattern).
    std::vector<uint32_t> hrp, hci;
    bool have_pattern = false;
    auto need_pattern = [&] {
        if (!have_pattern) copy_pattern(ctx, pc->L, hrp, hci);
        have_pattern = true;
    };
    pc->fwd.init(pc->L, true, false);
    // the levels of L order the exact factorisation and the exact solves
    auto levels = [&] {
        need_pattern();
        compute_levels(n, hrp.data(), hci.data(), true, pc->fwd.h_level);
        pc->fwd.ensure_sched(ctx);
    };
    const bool sweep_only = sweeps && fsweeps > 0;
    if (!sweep_only) levels();
    HostAnalysis ha;
    ha.chunked = pc->mode == B2S_TRSV_CHUNK && n;
    const int sm_count = ctx->sm_count;
    const bool fp32 = pc->fp32;
    int smem_optin = 0;
    B2S_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    const uint32_t tile_smem = smem_optin > 4096 ? (uint32_t)smem_optin - 4096u : 0u;  // static shared memory aside
    PatternStats ps;
    bool bfs = false;
    if (sweeps)
    {
        ps = pattern_stats(ctx, pc->L);
        const char* planner = std::getenv("B2S_TILE_PLANNER");  // "bfs": the general planner
        bfs = (planner && std::strcmp(planner, "bfs") == 0) || !ps.grid5;
        if (fp32 && bfs && n <= kTilePlanHostMaxRows) need_pattern();
    }
    else
        need_pattern();
    GridShape gs;
    if (ha.chunked && have_pattern)
    {
        gs = grid_shape(n, hrp, hci, nullptr, nullptr);
        if (gs.any()) ha.chunked = false;  // the grid schedule takes the exact solves
    }
    ha.th = std::thread([&ha, &hrp, &hci, &pc, ps, bfs, n, vs, sweeps, nsweeps, seg, sm_count, fp32, tile_smem] {
        try
        {
            if (sweeps)
            {
                // both band plans from L's statistics (L^T's pattern is not needed on the host)
                if (fp32)
                {
                    ha.lo_band = plan_band_from(n, ps.B, ps.w_row, nsweeps, sm_count, seg);
                    ha.up_band = plan_band_from(n, ps.B, ps.w_col, nsweeps, sm_count, seg);
                }
                // the tiled persistent PCG kernel: plain Jacobi, two strict entries per row.
                // A 5-point grid is laid out from closed forms (its blobs are built on the
                // device); other patterns take the breadth-first planner while it is cheap.
                if (fp32 && seg == 1 && ha.lo_band.T && ha.up_band.T && ha.lo_band.W == 2 && ha.up_band.W == 2 &&
                    nsweeps <= kTileMaxSweeps)
                {
                    if (!bfs)
                    {
                        ha.tiles = plan_tiles_grid5(n, ps.B, nsweeps, sm_count, tile_smem, ha.tile_geom);
                        ha.tiles_grid5 = true;
                    }
                    else if (n <= kTilePlanHostMaxRows)
                    {
                        std::vector<uint32_t> lrp, lci, urp, uci;
                        strict_lower(n, hrp.data(), hci.data(), lrp, lci);
                        strict_transpose(n, hrp.data(), hci.data(), true, urp, uci);
                        ha.tiles = plan_tiles(n, lrp.data(), lci.data(), urp.data(), uci.data(), nsweeps, sm_count,
                                              tile_smem, 8);
                    }
                }
                return;
            }
            strict_transpose(n, hrp.data(), hci.data(), true, ha.up_rp, ha.up_ci);
            // the two triangles' plans run side by side
            plan_parallel(2, 2, [&](uint32_t side, unsigned) {
                if (side == 0)
                {
                    if (ha.chunked)
                        ha.lo_plan = plan_chunks(n, hrp.data(), hci.data(), true, 1, vs, vs, 8, kChunkSmemBudget, 1,
                                                 &pc->fwd.h_level);
                    return;
                }
                compute_levels(n, ha.up_rp.data(), ha.up_ci.data(), false, ha.up_level);
                if (ha.chunked)
                    ha.up_plan = plan_chunks(n, ha.up_rp.data(), ha.up_ci.data(), false, 1, vs, vs, 8,
                                             kChunkSmemBudget, 1, &ha.up_level);
            });
        }
        catch (...)
        {
            ha.error = std::current_exception();
        }
    });
    pc->fwd.d64 = pc->diag.p;
    bool factored = false;
    if (fsweeps > 0)
    {
        DBuf<double> a(pc->L.nnz ? pc->L.nnz : 1);  // tril(A), the sweeps' right-hand side
        d2d(ctx, a.p, pc->L.v.p, (size_t)pc->L.nnz * sizeof(double));
        factored = ic0_factor_fixed_point(ctx, pc->L, pc->diag.p, fsweeps, a);
        if (!factored)  // a pivot failed: the exact factorisation decides (and reports)
        {
            d2d(ctx, pc->L.v.p, a.p, (size_t)pc->L.nnz * sizeof(double));
            if (!pc->fwd.sched_ready) levels();
        }
    }
    if (!factored)
        ic0_factor_inplace(ctx, pc->fwd.sched, pc->L.rp.p, pc->L.ci.p, pc->L.v.p, pc->diag.p, "IC(0) failed");
    if (corr) corr->correct(ctx, A, pc->L.rp.p, pc->L.ci.p, pc->L.nnz, pc->L.v.p, pc->diag.p);
    transpose_strict(ctx, pc->L, pc->LT);
    pc->y.alloc(n ? n : 1);
    if (pc->fp32)
    {
        to_f32(ctx, pc->L.v, pc->L.v32, pc->L.nnz);
        to_f32(ctx, pc->LT.v, pc->LT.v32, pc->LT.nnz);
        to_f32(ctx, pc->diag, pc->diag32, n);
        pc->y32.alloc(n ? n : 1);
        pc->z32.alloc(n ? n : 1);
    }
    ha.wait();
    pc->bwd.init(pc->LT, false, false);
    pc->bwd.h_level = std::move(ha.up_level);
    pc->fwd.load_chunks(ctx, pc->mode, ha.chunked ? &ha.lo_plan : nullptr, vs);
    pc->bwd.load_chunks(ctx, pc->mode, ha.chunked ? &ha.up_plan : nullptr, vs);
    enable_grid(pc->fwd, pc->bwd, gs, n);
    if (sweeps)
    {
        pc->fwd.prepare_sweeps(ctx, nsweeps, seg, pc->fp32, &ha.lo_band);
        pc->bwd.prepare_sweeps(ctx, nsweeps, seg, pc->fp32, &ha.up_band);
    }
    if (pc->fp32)
    {
        pc->fwd.pack<float>(ctx, pc->L.v32.p, pc->diag32.p);
        pc->bwd.pack<float>(ctx, pc->LT.v32.p, pc->diag32.p);
        if (sweeps && ha.tiles.ok && pc->fwd.band.T && pc->bwd.band.T)
            pc->load_tiles(ctx, A, ha.tiles, ha.tiles_grid5 ? &ha.tile_geom : nullptr);
    }
    else
    {
        pc->fwd.pack<double>(ctx, pc->L.v.p, pc->diag.p);
        pc->bwd.pack<double>(ctx, pc->LT.v.p, pc->diag.p);
    }
    sync(ctx);
    return pc;
}

std::unique_ptr<PcImpl> make_pc_ic0(b2s_ctx* ctx, const CsrDev& A, const b2s_pc_opts& o)
{
    return make_pc_ic0_ex(ctx, A, o, nullptr);
}

// ------------------------------------------------------------ ILU(0)

namespace {

struct PcILU0 final : PcImpl
{
    uint32_t n = 0;
    int mode = B2S_TRSV_SYNCFREE;
    bool fp32 = false;
    Csr32 L, U;
    DBuf<uint32_t> dix;
    DBuf<double> udiag, y;
    DBuf<float> udiag32, y32, z32;
    Tri fwd, bwd;

    void apply(b2s_ctx* ctx, const double* r, double* z, const int* done) override
    {
        if (!fp32)
        {
            fwd.solve<double, double, double>(ctx, mode, L.v.p, (const double*)nullptr, r, y.p, nullptr, done);
            bwd.solve<double, double, double>(ctx, mode, U.v.p, udiag.p, y.p, z, nullptr, done);
        }
        else
        {
            fwd.solve<float, float, double>(ctx, mode, L.v32.p, (const float*)nullptr, r, y32.p, nullptr, done);
            bwd.solve<float, float, float>(ctx, mode, U.v32.p, udiag32.p, y32.p, z32.p, z, done);
        }
    }

    void export_data(b2s_ctx* ctx, const std::string& what, uint64_t* sizes, uint32_t* rp, uint32_t* ci,
                     double* v) override
    {
        if (what == "ilu0.L") return export_csr(ctx, L, sizes, rp, ci, v);
        if (what == "ilu0.U") return export_csr(ctx, U, sizes, rp, ci, v);
        if (what == "trsv.grid5") return export_grid5(fwd, bwd, sizes);
        if (what == "trsv.grid7") return export_grid7(fwd, bwd, sizes);
        if (what == "levels.L") return export_levels(ctx, fwd, sizes, ci);
        if (what == "levels.U") return export_levels(ctx, bwd, sizes, ci);
        PcImpl::export_data(ctx, what, sizes, rp, ci, v);
    }
};

__global__ void k_gather_diag(uint32_t n, const double* __restrict__ Uv, const uint32_t* __restrict__ dix,
                              double* __restrict__ d)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d[i] = Uv[dix[i]];
}

}  // namespace

std::unique_ptr<PcImpl> make_pc_ilu0(b2s_ctx* ctx, const CsrDev& A, const b2s_pc_opts& o)
{
    need(A.n == A.m, B2S_SHAPE, "ILU(0) needs a square matrix");
    auto pc = std::make_unique<PcILU0>();
    const uint32_t n = A.n;
    pc->n = n;
    pc->mode = pick_trsv(o);
    pc->fp32 = o.precision != B2S_FP64;
    const uint32_t vs = pc->fp32 ? 4 : 8;
    DBuf<unsigned long long> err(1);
    const unsigned long long none = ~0ull;
    h2d(ctx, err.p, &none, sizeof(none));
    pc->dix.alloc(n ? n : 1);
    split(ctx, A, 1, pc->L, nullptr, err.p);
    split(ctx, A, 2, pc->U, pc->dix.p, err.p);
    check_err(ctx, err, "ILU(0) failed");
    // host analysis: levels of L here (for the factorisation), the rest on a thread
    std::vector<uint32_t> lrp, lci, urp, uci;
    copy_pattern(ctx, pc->L, lrp, lci);
    copy_pattern(ctx, pc->U, urp, uci);
    pc->fwd.init(pc->L, true, true);
    compute_levels(n, lrp.data(), lci.data(), true, pc->fwd.h_level);
    pc->fwd.ensure_sched(ctx);
    HostAnalysis ha;
    ha.chunked = pc->mode == B2S_TRSV_CHUNK && n;
    GridShape gs;
    if (ha.chunked)
    {
        gs = grid_shape(n, lrp, lci, &urp, &uci);
        if (gs.any()) ha.chunked = false;  // the grid schedule takes the exact solves
    }
    ha.th = std::thread([&ha, &lrp, &lci, &urp, &uci, &pc, n, vs] {
        try
        {
            // the two triangles' plans run side by side
            plan_parallel(2, 2, [&](uint32_t side, unsigned) {
                if (side == 0)
                {
                    if (ha.chunked)
                        ha.lo_plan = plan_chunks(n, lrp.data(), lci.data(), true, 0, vs, vs, 8, kChunkSmemBudget, 1,
                                                 &pc->fwd.h_level);
                    return;
                }
                compute_levels(n, urp.data(), uci.data(), false, ha.up_level);
                if (ha.chunked)
                    ha.up_plan = plan_chunks(n, urp.data(), uci.data(), false, 1, vs, vs, 8, kChunkSmemBudget, 1,
                                             &ha.up_level);
            });
        }
        catch (...)
        {
            ha.error = std::current_exception();
        }
    });
    // factor, level by level
    for (uint32_t l = 0; l < pc->fwd.sched.nlev; ++l)
    {
        const uint32_t a = pc->fwd.sched.h_ptr[l], cnt = pc->fwd.sched.h_ptr[l + 1] - a;
        B2S_LAUNCH(ctx, k_ilu0_level, (cnt + kThreads - 1) / kThreads, kThreads, 0, pc->fwd.sched.rows.p + a, cnt,
                   pc->L.rp.p, pc->L.ci.p, pc->L.v.p, pc->U.rp.p, pc->U.ci.p, pc->U.v.p, pc->dix.p, err.p);
    }
    check_err(ctx, err, "ILU(0) failed");
    pc->udiag.alloc(n ? n : 1);
    if (n) B2S_LAUNCH(ctx, k_gather_diag, stream_grid(ctx, n), kThreads, 0, n, pc->U.v.p, pc->dix.p, pc->udiag.p);
    pc->y.alloc(n ? n : 1);
    if (pc->fp32)
    {
        to_f32(ctx, pc->L.v, pc->L.v32, pc->L.nnz);
        to_f32(ctx, pc->U.v, pc->U.v32, pc->U.nnz);
        to_f32(ctx, pc->udiag, pc->udiag32, n);
        pc->y32.alloc(n ? n : 1);
        pc->z32.alloc(n ? n : 1);
    }
    ha.wait();
    pc->bwd.init(pc->U, false, false);
    pc->bwd.h_level = std::move(ha.up_level);
    pc->fwd.load_chunks(ctx, pc->mode, ha.chunked ? &ha.lo_plan : nullptr, vs);
    pc->bwd.load_chunks(ctx, pc->mode, ha.chunked ? &ha.up_plan : nullptr, vs);
    enable_grid(pc->fwd, pc->bwd, gs, n);
    if (pc->mode == B2S_TRSV_JACOBI)
    {
        const int k = sweep_count(o);
        const uint32_t seg = sweep_segment(o);
        BandPlan lo, up;
        if (pc->fp32)
        {
            lo = plan_band(n, lrp.data(), lci.data(), true, k, ctx->sm_count, seg);
            up = plan_band(n, urp.data(), uci.data(), false, k, ctx->sm_count, seg);
        }
        pc->fwd.prepare_sweeps(ctx, k, seg, pc->fp32, &lo);
        pc->bwd.prepare_sweeps(ctx, k, seg, pc->fp32, &up);
    }
    if (pc->fp32)
    {
        pc->fwd.pack<float>(ctx, pc->L.v32.p, (const float*)nullptr);
        pc->bwd.pack<float>(ctx, pc->U.v32.p, pc->udiag32.p);
    }
    else
    {
        pc->fwd.pack<double>(ctx, pc->L.v.p, (const double*)nullptr);
        pc->bwd.pack<double>(ctx, pc->U.v.p, pc->udiag.p);
    }
    sync(ctx);
    return pc;
}

}  // namespace b2s
