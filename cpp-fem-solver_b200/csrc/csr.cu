// CSR handles and SpMV (SMatrix::spmv, array.cpp:3418-3442).
#include "spmv_staged.cuh"

#include <algorithm>

namespace b2s {

// Greedy row partition: a block closes when it holds max_rows rows or when
// the next row would push it past max_units units (nnz or nonzero blocks); a
// row that alone exceeds max_units gets a block of its own.
void build_row_blocks(const uint32_t* rp, uint32_t nrows, uint32_t unit, uint32_t max_rows, uint32_t max_units,
                      std::vector<uint32_t>& out)
{
    (void)unit;
    out.clear();
    out.push_back(0);
    uint32_t start = 0;
    while (start < nrows)
    {
        uint32_t r = start;
        const uint32_t base = rp[start];
        while (r < nrows && r - start < max_rows && rp[r + 1] - base <= max_units) ++r;
        if (r == start) r = start + 1;  // a single oversized row
        out.push_back(r);
        start = r;
    }
}

__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

void CsrDev::host_pattern(b2s_ctx* ctx) const
{
    if (h_rp.size() == (size_t)n + 1) return;
    h_rp.resize((size_t)n + 1);
    h_ci.resize(nnz ? nnz : 1);
    d2h(ctx, h_rp.data(), rp.p, ((size_t)n + 1) * sizeof(uint32_t));
    if (nnz) d2h(ctx, h_ci.data(), ci.p, (size_t)nnz * sizeof(uint32_t));
    sync(ctx);
}

void CsrDev::ensure_fp32(b2s_ctx* ctx)
{
    if (v32.p || nnz == 0) return;
    v32.alloc(nnz);
    B2S_LAUNCH(ctx, k_to_f32, stream_grid(ctx, nnz), kThreads, 0, v.p, v32.p, (uint64_t)nnz);
}

__global__ void k_extract_diag(uint32_t n, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                               const double* __restrict__ v, double* __restrict__ d)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        double di = 0.0;
        for (uint32_t k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i)
            {
                di = v[k];
                break;
            }
        d[i] = di;
    }
}

// A device-built pattern (row pointers on the device) becomes a CSR handle's
// storage: padded copies of the columns and values, the host-side row
// partition of the SpMV, the longest row and the diagonal -- what
// b2s_csr_create derives from host arrays.
static void csr_adopt(b2s_ctx* ctx, CsrDev& d, uint32_t n, uint32_t m, DBuf<uint32_t>&& rp, const uint32_t* ci,
                      const double* v)
{
    std::vector<uint32_t> h_rp((size_t)n + 1);
    d2h(ctx, h_rp.data(), rp.p, h_rp.size() * sizeof(uint32_t));
    sync(ctx);
    const uint32_t nnz = h_rp[n];
    uint32_t max_row = 0;
    for (uint32_t i = 0; i < n; ++i) max_row = std::max(max_row, h_rp[i + 1] - h_rp[i]);
    d.n = n;
    d.m = m;
    d.nnz = nnz;
    d.max_row = max_row;
    d.rp = std::move(rp);
    d.ci.alloc((size_t)nnz + 8);
    d.v.alloc((size_t)nnz + 8);
    B2S_CUDA(cudaMemsetAsync(d.ci.p, 0, d.ci.bytes(), ctx->stream));
    B2S_CUDA(cudaMemsetAsync(d.v.p, 0, d.v.bytes(), ctx->stream));
    d2d(ctx, d.ci.p, ci, (size_t)nnz * sizeof(uint32_t));
    d2d(ctx, d.v.p, v, (size_t)nnz * sizeof(double));
    std::vector<uint32_t> blk;
    build_row_blocks(h_rp.data(), n, 1, kSpmvRowsPerCta, kSpmvNnzPerCta, blk);
    d.nblk = (uint32_t)blk.size() - 1;
    d.blk_row = upload(ctx, blk.data(), blk.size());
    if (n == m && n > 0)
    {
        d.diag.alloc(n);
        B2S_LAUNCH(ctx, k_extract_diag, stream_grid(ctx, n), kThreads, 0, n, d.rp.p, d.ci.p, d.v.p, d.diag.p);
    }
    sync(ctx);
}

// a bs = 1 block view of a CSR handle (device copies)
static void csr_as_scalar_blocks(b2s_ctx* ctx, const CsrDev& A, BaijDev& B)
{
    B.bs = 1;
    B.nbr = A.n;
    B.nbc = A.m;
    B.nnzb = A.nnz;
    B.rp.alloc((size_t)A.n + 1);
    B.ci.alloc(A.nnz ? A.nnz : 1);
    B.v.alloc(A.nnz ? A.nnz : 1);
    d2d(ctx, B.rp.p, A.rp.p, ((size_t)A.n + 1) * sizeof(uint32_t));
    d2d(ctx, B.ci.p, A.ci.p, (size_t)A.nnz * sizeof(uint32_t));
    d2d(ctx, B.v.p, A.v.p, (size_t)A.nnz * sizeof(double));
}

void spmv(b2s_ctx* ctx, const CsrDev& A, const double* x, double* y, const int* done)
{
    if (A.n == 0) return;
    launch_spmv(ctx, A, x, done, EpiStore{y});
}

}  // namespace b2s

using namespace b2s;

extern "C" {

b2s_status b2s_csr_create(b2s_ctx* ctx, uint32_t n, uint32_t m, const uint32_t* row_ptr, const uint32_t* col_idx,
                          const double* values, b2s_csr** out)
{
    if (!ctx || !out || !row_ptr) return B2S_INVALID_ARG;
    *out = nullptr;
    b2s_csr* A = new b2s_csr();
    A->ctx = ctx;
    b2s_status st = guarded(ctx, [&] {
        B2S_CUDA(cudaSetDevice(ctx->device));
        need(row_ptr[0] == 0, B2S_INVALID_ARG, "row_ptr[0] must be 0");
        const uint32_t nnz = row_ptr[n];
        need(nnz == 0 || (col_idx && values), B2S_INVALID_ARG, "null col_idx / values");
        // one pass: row pointers non-decreasing, columns in range and strictly ascending
        uint32_t max_row = 0;
        bool ok_rp = true, ok_range = true, ok_order = true;
        for (uint32_t i = 0; i < n && ok_rp; ++i)
        {
            const uint32_t a = row_ptr[i], b = row_ptr[i + 1];
            if (b < a || b > nnz)
            {
                ok_rp = false;
                break;
            }
            max_row = std::max(max_row, b - a);
            uint32_t prev = 0;
            for (uint32_t k = a; k < b; ++k)
            {
                const uint32_t c = col_idx[k];
                ok_range &= c < m;
                ok_order &= k == a || c > prev;
                prev = c;
            }
        }
        need(ok_rp, B2S_INVALID_ARG, "row_ptr must be non-decreasing");
        need(ok_range, B2S_INVALID_ARG, "column index out of range");
        need(ok_order, B2S_INVALID_ARG, "columns must be strictly ascending within a row");
        CsrDev& d = A->d;
        d.n = n;
        d.m = m;
        d.nnz = nnz;
        d.max_row = max_row;
        d.rp = upload(ctx, row_ptr, (size_t)n + 1);
        // 8 elements of padding: the bulk copies of the SpMV start and end on
        // 16-byte boundaries and may read a few elements past the last nonzero
        d.ci.alloc((size_t)nnz + 8);
        d.v.alloc((size_t)nnz + 8);
        B2S_CUDA(cudaMemsetAsync(d.ci.p, 0, d.ci.bytes(), ctx->stream));
        B2S_CUDA(cudaMemsetAsync(d.v.p, 0, d.v.bytes(), ctx->stream));
        h2d(ctx, d.ci.p, col_idx, (size_t)nnz * sizeof(uint32_t));
        h2d(ctx, d.v.p, values, (size_t)nnz * sizeof(double));
        std::vector<uint32_t> blk;
        build_row_blocks(row_ptr, n, 1, kSpmvRowsPerCta, kSpmvNnzPerCta, blk);
        d.nblk = (uint32_t)blk.size() - 1;
        d.blk_row = upload(ctx, blk.data(), blk.size());
        if (n == m && n > 0)
        {
            d.diag.alloc(n);
            B2S_LAUNCH(ctx, k_extract_diag, stream_grid(ctx, n), kThreads, 0, n, d.rp.p, d.ci.p, d.v.p, d.diag.p);
        }
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

b2s_status b2s_csr_destroy(b2s_csr* A)
{
    if (!A) return B2S_INVALID_ARG;
    cudaSetDevice(A->ctx->device);
    delete A;
    return B2S_OK;
}

b2s_status b2s_csr_info(const b2s_csr* A, uint32_t* n, uint32_t* m, uint32_t* nnz)
{
    if (!A) return B2S_INVALID_ARG;
    if (n) *n = A->d.n;
    if (m) *m = A->d.m;
    if (nnz) *nnz = A->d.nnz;
    return B2S_OK;
}

b2s_status b2s_spmv_device(b2s_ctx* ctx, const b2s_csr* A, const double* d_x, double* d_y)
{
    if (!ctx || !A) return B2S_INVALID_ARG;
    return guarded(ctx, [&] { spmv(ctx, A->d, d_x, d_y); });
}

b2s_status b2s_spmv(b2s_ctx* ctx, const b2s_csr* A, const double* x, double* y)
{
    if (!ctx || !A || (!x && A->d.m) || (!y && A->d.n)) return B2S_INVALID_ARG;
    return guarded(ctx, [&] {
        DBuf<double> dx(A->d.m), dy(A->d.n);
        h2d(ctx, dx.p, x, dx.bytes());
        spmv(ctx, A->d, dx.p, dy.p);
        d2h(ctx, y, dy.p, dy.bytes());
        sync(ctx);
    });
}

b2s_status b2s_csr_matmul(b2s_ctx* ctx, const b2s_csr* A, const b2s_csr* B, b2s_csr** out)
{
    if (!ctx || !A || !B || !out) return B2S_INVALID_ARG;
    *out = nullptr;
    b2s_csr* C = new b2s_csr();
    C->ctx = ctx;
    const b2s_status st = guarded(ctx, [&] {
        B2S_CUDA(cudaSetDevice(ctx->device));
        need(A->d.m == B->d.n, B2S_SHAPE, "matmul: columns of A differ from rows of B");
        BaijDev a, b, c;
        csr_as_scalar_blocks(ctx, A->d, a);
        csr_as_scalar_blocks(ctx, B->d, b);
        scalar_matmul(ctx, a, b, c);
        csr_adopt(ctx, C->d, A->d.n, B->d.m, std::move(c.rp), c.ci.p, c.v.p);
    });
    if (st != B2S_OK)
    {
        delete C;
        return st;
    }
    *out = C;
    return B2S_OK;
}

b2s_status b2s_csr_transpose(b2s_ctx* ctx, const b2s_csr* A, b2s_csr** out)
{
    if (!ctx || !A || !out) return B2S_INVALID_ARG;
    *out = nullptr;
    b2s_csr* T = new b2s_csr();
    T->ctx = ctx;
    const b2s_status st = guarded(ctx, [&] {
        B2S_CUDA(cudaSetDevice(ctx->device));
        BaijDev a, t;
        csr_as_scalar_blocks(ctx, A->d, a);
        scalar_transpose(ctx, a, t);
        csr_adopt(ctx, T->d, A->d.m, A->d.n, std::move(t.rp), t.ci.p, t.v.p);
    });
    if (st != B2S_OK)
    {
        delete T;
        return st;
    }
    *out = T;
    return B2S_OK;
}

b2s_status b2s_csr_export(b2s_ctx* ctx, const b2s_csr* A, uint32_t* row_ptr, uint32_t* col_idx, double* values)
{
    if (!ctx || !A) return B2S_INVALID_ARG;
    return guarded(ctx, [&] {
        if (row_ptr) d2h(ctx, row_ptr, A->d.rp.p, ((size_t)A->d.n + 1) * sizeof(uint32_t));
        if (col_idx) d2h(ctx, col_idx, A->d.ci.p, (size_t)A->d.nnz * sizeof(uint32_t));
        if (values) d2h(ctx, values, A->d.v.p, (size_t)A->d.nnz * sizeof(double));
        sync(ctx);
    });
}

}  // extern "C"
