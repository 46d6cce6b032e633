/* b2s_oracle.c -- CPU restatement of the reference's sparse solver path.
 *
 * TEST INFRASTRUCTURE ONLY (see b2s_oracle.h).  Every function names the
 * reference function it restates as file:line under ode-solver/.  Loops run in
 * the reference's order with FP contraction off, so at one thread the results
 * agree bit for bit with the reference compiled from source. */
#include "b2s_oracle.h"

#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORC_NONE 0xFFFFFFFFu

static void set_err(char* err, int errlen, const char* msg)
{
    if (err && errlen > 0)
    {
        strncpy(err, msg, (size_t)errlen - 1);
        err[errlen - 1] = 0;
    }
}

static void* xcalloc(size_t n, size_t sz)
{
    void* p = calloc(n ? n : 1, sz);
    if (!p)
    {
        fprintf(stderr, "oracle: out of memory\n");
        abort();
    }
    return p;
}

/* ======================================================================
 * CSR container
 * ====================================================================== */

typedef struct
{
    uint32_t i, j;
    double v;
    uint64_t k; /* original position: makes the sort deterministic */
} coo_entry;

static int coo_cmp(const void* a, const void* b)
{
    const coo_entry* x = (const coo_entry*)a;
    const coo_entry* y = (const coo_entry*)b;
    if (x->i != y->i) return x->i < y->i ? -1 : 1;
    if (x->j != y->j) return x->j < y->j ? -1 : 1;
    return x->k < y->k ? -1 : (x->k > y->k);
}

/* SMatrix COO constructor, array.cpp:2072-2182: drop zeros, sort by (i,j),
 * merge duplicates by summation, drop merged zeros, build CSR.  Duplicates are
 * summed in input order (the reference's std::sort leaves their order
 * unspecified). */
orc_csr* orc_csr_from_coo(uint32_t n, uint32_t m, uint64_t nnz, const double* v, const uint32_t* r,
                          const uint32_t* c, int* st)
{
    *st = ORC_OK;
    coo_entry* e = (coo_entry*)xcalloc(nnz, sizeof(coo_entry));
    uint64_t ne = 0;
    for (uint64_t k = 0; k < nnz; ++k)
    {
        if (r[k] >= n || c[k] >= m)
        {
            free(e);
            *st = ORC_INVALID_ARG;
            return NULL;
        }
        if (v[k] != 0.0)
        {
            e[ne].i = r[k];
            e[ne].j = c[k];
            e[ne].v = v[k];
            e[ne].k = k;
            ++ne;
        }
    }
    qsort(e, ne, sizeof(coo_entry), coo_cmp);
    uint64_t nm = 0;
    for (uint64_t k = 0; k < ne; ++k)
    {
        if (nm > 0 && e[nm - 1].i == e[k].i && e[nm - 1].j == e[k].j)
            e[nm - 1].v += e[k].v;
        else
            e[nm++] = e[k];
    }
    uint64_t nz = 0;
    for (uint64_t k = 0; k < nm; ++k)
        if (e[k].v != 0.0) e[nz++] = e[k];

    orc_csr* A = (orc_csr*)xcalloc(1, sizeof(orc_csr));
    A->n = n;
    A->m = m;
    A->rp = (uint32_t*)xcalloc((size_t)n + 1, 4);
    A->ci = (uint32_t*)xcalloc(nz, 4);
    A->v = (double*)xcalloc(nz, 8);
    for (uint64_t k = 0; k < nz; ++k) A->rp[e[k].i + 1]++;
    for (uint32_t i = 0; i < n; ++i) A->rp[i + 1] += A->rp[i];
    for (uint64_t k = 0; k < nz; ++k)
    {
        A->ci[k] = e[k].j; /* already in row-major order */
        A->v[k] = e[k].v;
    }
    free(e);
    return A;
}

/* SMatrix CSR constructor, array.cpp:2183-2189 (arrays taken as given). */
orc_csr* orc_csr_copy(uint32_t n, uint32_t m, const uint32_t* rp, const uint32_t* ci, const double* v)
{
    orc_csr* A = (orc_csr*)xcalloc(1, sizeof(orc_csr));
    A->n = n;
    A->m = m;
    A->rp = (uint32_t*)xcalloc((size_t)n + 1, 4);
    memcpy(A->rp, rp, 4 * ((size_t)n + 1));
    A->ci = (uint32_t*)xcalloc(rp[n], 4);
    A->v = (double*)xcalloc(rp[n], 8);
    memcpy(A->ci, ci, 4 * (size_t)rp[n]);
    memcpy(A->v, v, 8 * (size_t)rp[n]);
    return A;
}

void orc_csr_free(orc_csr* A)
{
    if (!A) return;
    free(A->rp);
    free(A->ci);
    free(A->v);
    free(A);
}

uint32_t orc_csr_nnz(const orc_csr* A) { return A->rp[A->n]; }

void orc_csr_export(const orc_csr* A, uint32_t* rp, uint32_t* ci, double* v)
{
    memcpy(rp, A->rp, 4 * ((size_t)A->n + 1));
    memcpy(ci, A->ci, 4 * (size_t)A->rp[A->n]);
    memcpy(v, A->v, 8 * (size_t)A->rp[A->n]);
}

/* SMatrix::transpose, array.cpp:2202-2235: count, prefix, scatter in row order. */
orc_csr* orc_csr_transpose(const orc_csr* A)
{
    const uint32_t n = A->n, m = A->m, nnz = A->rp[n];
    orc_csr* T = (orc_csr*)xcalloc(1, sizeof(orc_csr));
    T->n = m;
    T->m = n;
    T->rp = (uint32_t*)xcalloc((size_t)m + 1, 4);
    T->ci = (uint32_t*)xcalloc(nnz, 4);
    T->v = (double*)xcalloc(nnz, 8);
    for (uint32_t p = 0; p < nnz; ++p) T->rp[A->ci[p] + 1]++;
    for (uint32_t i = 0; i < m; ++i) T->rp[i + 1] += T->rp[i];
    uint32_t* off = (uint32_t*)xcalloc((size_t)m + 1, 4);
    memcpy(off, T->rp, 4 * ((size_t)m + 1));
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t p = A->rp[i]; p < A->rp[i + 1]; ++p)
        {
            const uint32_t j = A->ci[p];
            T->ci[off[j]] = i;
            T->v[off[j]++] = A->v[p];
        }
    free(off);
    return T;
}

static int u32_cmp(const void* a, const void* b)
{
    const uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return x < y ? -1 : (x > y);
}

/* SMatrix::operator*, array.cpp:2336-2447: per-row sparse accumulator,
 * products accumulated in (p, q) order, columns sorted, zeros kept. */
orc_csr* orc_csr_matmul(const orc_csr* A, const orc_csr* B)
{
    const uint32_t n = A->n, m = B->m;
    int32_t* marker = (int32_t*)xcalloc(m, 4);
    double* accum = (double*)xcalloc(m, 8);
    for (uint32_t k = 0; k < m; ++k) marker[k] = -1;
    uint32_t* rp = (uint32_t*)xcalloc((size_t)n + 1, 4);
    for (uint32_t i = 0; i < n; ++i)
    {
        uint32_t c = 0;
        for (uint32_t p = A->rp[i]; p < A->rp[i + 1]; ++p)
        {
            const uint32_t j = A->ci[p];
            for (uint32_t q = B->rp[j]; q < B->rp[j + 1]; ++q)
                if (marker[B->ci[q]] != (int32_t)i)
                {
                    marker[B->ci[q]] = (int32_t)i;
                    ++c;
                }
        }
        rp[i + 1] = c;
    }
    for (uint32_t i = 0; i < n; ++i) rp[i + 1] += rp[i];
    for (uint32_t k = 0; k < m; ++k) marker[k] = -1;
    uint32_t* ci = (uint32_t*)xcalloc(rp[n], 4);
    double* vv = (double*)xcalloc(rp[n], 8);
    uint32_t* cols = (uint32_t*)xcalloc(m, 4);
    for (uint32_t i = 0; i < n; ++i)
    {
        uint32_t nc = 0;
        for (uint32_t p = A->rp[i]; p < A->rp[i + 1]; ++p)
        {
            const uint32_t j = A->ci[p];
            const double a = A->v[p];
            for (uint32_t q = B->rp[j]; q < B->rp[j + 1]; ++q)
            {
                const uint32_t k = B->ci[q];
                if (marker[k] != (int32_t)i)
                {
                    marker[k] = (int32_t)i;
                    cols[nc++] = k;
                }
                accum[k] += a * B->v[q];
            }
        }
        qsort(cols, nc, 4, u32_cmp);
        uint32_t w = rp[i];
        for (uint32_t t = 0; t < nc; ++t)
        {
            ci[w] = cols[t];
            vv[w] = accum[cols[t]];
            accum[cols[t]] = 0.0;
            ++w;
        }
    }
    free(cols);
    free(marker);
    free(accum);
    orc_csr* C = (orc_csr*)xcalloc(1, sizeof(orc_csr));
    C->n = n;
    C->m = m;
    C->rp = rp;
    C->ci = ci;
    C->v = vv;
    return C;
}

/* ======================================================================
 * Kernels
 * ====================================================================== */

/* SMatrix::spmv, array.cpp:3418-3442: ascending-k sum per row. */
void orc_spmv(const orc_csr* A, const double* x, double* y)
{
    for (uint32_t i = 0; i < A->n; ++i)
    {
        double sum = 0.0;
        for (uint32_t k = A->rp[i]; k < A->rp[i + 1]; ++k) sum += A->v[k] * x[A->ci[k]];
        y[i] = sum;
    }
}

/* SMatrix::dot, array.cpp:3401-3416 (one thread: ascending order). */
double orc_dot(uint64_t n, const double* a, const double* b)
{
    double sum = 0.0;
    for (uint64_t i = 0; i < n; ++i) sum += a[i] * b[i];
    return sum;
}

/* ======================================================================
 * Block helpers (blockMatrix.hpp:37-118), runtime block size
 * ====================================================================== */

/* blk_matmat_accum: C -= A*B */
static void blk_mma(int bs, const double* A, const double* B, double* C)
{
    for (int r = 0; r < bs; ++r)
        for (int c = 0; c < bs; ++c)
        {
            double s = 0.0;
            for (int k = 0; k < bs; ++k) s += A[r * bs + k] * B[k * bs + c];
            C[r * bs + c] -= s;
        }
}

/* blk_right_mul: C := C*B */
static void blk_rmul(int bs, double* C, const double* B)
{
    double tmp[64];
    for (int r = 0; r < bs; ++r)
        for (int c = 0; c < bs; ++c)
        {
            double s = 0.0;
            for (int k = 0; k < bs; ++k) s += C[r * bs + k] * B[k * bs + c];
            tmp[r * bs + c] = s;
        }
    for (int t = 0; t < bs * bs; ++t) C[t] = tmp[t];
}

/* blk_matvec: y = M*x */
static void blk_mv(int bs, const double* M, const double* x, double* y)
{
    for (int r = 0; r < bs; ++r)
    {
        double s = 0.0;
        for (int c = 0; c < bs; ++c) s += M[r * bs + c] * x[c];
        y[r] = s;
    }
}

/* blk_invert: Gauss elimination with partial pivoting on [M | I]. */
static int blk_inv(int bs, const double* M, double* Minv)
{
    double aug[8][16];
    for (int i = 0; i < bs; ++i)
        for (int j = 0; j < bs; ++j)
        {
            aug[i][j] = M[i * bs + j];
            aug[i][bs + j] = (i == j) ? 1.0 : 0.0;
        }
    for (int k = 0; k < bs; ++k)
    {
        int piv = k;
        for (int i = k + 1; i < bs; ++i)
            if (fabs(aug[i][k]) > fabs(aug[piv][k])) piv = i;
        if (fabs(aug[piv][k]) < 1e-300) return 0;
        if (piv != k)
            for (int j = 0; j < 2 * bs; ++j)
            {
                double t = aug[k][j];
                aug[k][j] = aug[piv][j];
                aug[piv][j] = t;
            }
        for (int i = k + 1; i < bs; ++i)
        {
            const double f = aug[i][k] / aug[k][k];
            for (int j = k; j < 2 * bs; ++j) aug[i][j] -= f * aug[k][j];
        }
    }
    for (int i = bs - 1; i >= 0; --i)
    {
        for (int j = i + 1; j < bs; ++j)
            for (int c = 0; c < bs; ++c) aug[i][bs + c] -= aug[i][j] * aug[j][bs + c];
        for (int c = 0; c < bs; ++c) aug[i][bs + c] /= aug[i][i];
    }
    for (int i = 0; i < bs; ++i)
        for (int j = 0; j < bs; ++j) Minv[i * bs + j] = aug[i][bs + j];
    return 1;
}

/* blk_find_col: binary search of a block column in a sorted row */
static uint32_t blk_find(const uint32_t* rp, const uint32_t* ci, uint32_t row, uint32_t col)
{
    uint32_t lo = rp[row], hi = rp[row + 1];
    while (lo < hi)
    {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (ci[mid] == col) return mid;
        if (ci[mid] < col)
            lo = mid + 1;
        else
            hi = mid;
    }
    return ORC_NONE;
}

/* blk_fro_norm, blockMatrix.hpp:874-880 */
static double blk_fro(int bs, const double* b)
{
    double s = 0.0;
    for (int i = 0; i < bs * bs; ++i) s += b[i] * b[i];
    return sqrt(s);
}

/* ======================================================================
 * BlockMatrix
 * ====================================================================== */

static void blk_cache_diag(orc_blk* A)
{
    A->diag_ptr = (uint32_t*)xcalloc(A->nbr, 4);
    for (uint32_t bi = 0; bi < A->nbr; ++bi)
    {
        A->diag_ptr[bi] = ORC_NONE;
        for (uint32_t p = A->rp[bi]; p < A->rp[bi + 1]; ++p)
            if (A->ci[p] == bi)
            {
                A->diag_ptr[bi] = p;
                break;
            }
    }
}

static orc_blk* blk_take(int bs, uint32_t nbr, uint32_t nbc, uint32_t* rp, uint32_t* ci, double* v)
{
    orc_blk* A = (orc_blk*)xcalloc(1, sizeof(orc_blk));
    A->bs = bs;
    A->nbr = nbr;
    A->nbc = nbc;
    A->rp = rp;
    A->ci = ci;
    A->v = v;
    blk_cache_diag(A);
    return A;
}

/* BlockMatrix constructor + cache_diag, blockMatrix.hpp:175-207 */
orc_blk* orc_blk_create(int bs, uint32_t nbr, uint32_t nbc, const uint32_t* rp, const uint32_t* ci,
                        const double* v)
{
    const size_t bv = (size_t)bs * bs, nnzb = rp[nbr];
    uint32_t* r = (uint32_t*)xcalloc((size_t)nbr + 1, 4);
    uint32_t* c = (uint32_t*)xcalloc(nnzb, 4);
    double* vv = (double*)xcalloc(nnzb * bv, 8);
    memcpy(r, rp, 4 * ((size_t)nbr + 1));
    memcpy(c, ci, 4 * nnzb);
    memcpy(vv, v, 8 * nnzb * bv);
    return blk_take(bs, nbr, nbc, r, c, vv);
}

void orc_blk_free(orc_blk* A)
{
    if (!A) return;
    free(A->rp);
    free(A->ci);
    free(A->v);
    free(A->diag_ptr);
    free(A);
}

uint32_t orc_blk_nnzb(const orc_blk* A) { return A->rp[A->nbr]; }
uint32_t orc_blk_rows(const orc_blk* A) { return A->nbr; }

void orc_blk_export(const orc_blk* A, uint32_t* rp, uint32_t* ci, double* v)
{
    memcpy(rp, A->rp, 4 * ((size_t)A->nbr + 1));
    memcpy(ci, A->ci, 4 * (size_t)A->rp[A->nbr]);
    memcpy(v, A->v, 8 * (size_t)A->rp[A->nbr] * A->bs * A->bs);
}

/* BlockMatrix::matvec, blockMatrix.hpp:208-234: per block a row GEMV whose
 * partial sum is added into y.  The reference marks the row sum
 * `#pragma omp simd reduction(+:acc)`; compiled by GCC 13 at -O3 for x86-64-v3
 * that 3-term sum becomes (p0 + p2) + p1 (two lanes, then a lane reduction),
 * which tests/test_oracle_pin.py confirms against the compiled reference; other
 * block sizes sum in ascending order. */
void orc_blk_matvec(const orc_blk* A, const double* x, double* y)
{
    const int bs = A->bs, bv = bs * bs;
    for (uint32_t bi = 0; bi < A->nbr; ++bi)
    {
        double* yi = &y[(size_t)bi * bs];
        for (int r = 0; r < bs; ++r) yi[r] = 0.0;
        for (uint32_t p = A->rp[bi]; p < A->rp[bi + 1]; ++p)
        {
            const double* B = &A->v[(size_t)p * bv];
            const double* xj = &x[(size_t)A->ci[p] * bs];
            for (int r = 0; r < bs; ++r)
            {
                double acc;
                if (bs == 3)
                {
                    const double p0 = B[r * 3 + 0] * xj[0], p1 = B[r * 3 + 1] * xj[1], p2 = B[r * 3 + 2] * xj[2];
                    acc = (p0 + p2) + p1;
                }
                else
                {
                    acc = 0.0;
                    for (int c = 0; c < bs; ++c) acc += B[r * bs + c] * xj[c];
                }
                yi[r] += acc;
            }
        }
    }
}

/* BlockMatrix::distributed_matvec with MPI, blockMatrix.hpp:351-437, after
 * the halo exchange: one rank's block rows with local columns (lci: an owned
 * column j < n_owned, a ghost column n_owned + k), x_full = [owned | ghosts].
 * y starts at zero; pass 1 adds the owned columns' blocks in row order, pass
 * 2 the ghost columns'; each block contributes acc = sum_c B[r][c] x_j[c]
 * summed in c order (this loop carries no omp simd, unlike matvec). */
void orc_blk_dist_matvec(int bs, uint32_t nbr, const uint32_t* rp, const uint32_t* lci, const double* v,
                         uint32_t n_owned, const double* x_full, double* y)
{
    const int bv = bs * bs;
    for (size_t i = 0; i < (size_t)nbr * bs; ++i) y[i] = 0.0;
    for (int pass = 0; pass < 2; ++pass)
        for (uint32_t bi = 0; bi < nbr; ++bi)
        {
            double* yi = &y[(size_t)bi * bs];
            for (uint32_t p = rp[bi]; p < rp[bi + 1]; ++p)
            {
                if ((lci[p] >= n_owned) != (pass == 1)) continue;
                const double* B = &v[(size_t)p * bv];
                const double* xj = &x_full[(size_t)lci[p] * bs];
                for (int r = 0; r < bs; ++r)
                {
                    double acc = 0.0;
                    for (int c = 0; c < bs; ++c) acc += B[r * bs + c] * xj[c];
                    yi[r] += acc;
                }
            }
        }
}

/* BlockMatrix::transpose, blockMatrix.hpp:237-267 */
orc_blk* orc_blk_transpose(const orc_blk* A)
{
    const int bs = A->bs, bv = bs * bs;
    const uint32_t nnzb = A->rp[A->nbr];
    uint32_t* trp = (uint32_t*)xcalloc((size_t)A->nbc + 1, 4);
    for (uint32_t p = 0; p < nnzb; ++p) trp[A->ci[p] + 1]++;
    for (uint32_t i = 0; i < A->nbc; ++i) trp[i + 1] += trp[i];
    uint32_t* tci = (uint32_t*)xcalloc(nnzb, 4);
    uint32_t* off = (uint32_t*)xcalloc((size_t)A->nbc + 1, 4);
    memcpy(off, trp, 4 * ((size_t)A->nbc + 1));
    for (uint32_t i = 0; i < A->nbr; ++i)
        for (uint32_t p = A->rp[i]; p < A->rp[i + 1]; ++p) tci[off[A->ci[p]]++] = i;
    free(off);
    double* tv = (double*)xcalloc((size_t)nnzb * bv, 8);
    for (uint32_t j = 0; j < A->nbc; ++j)
        for (uint32_t q = trp[j]; q < trp[j + 1]; ++q)
        {
            const uint32_t i = tci[q];
            uint32_t p = A->rp[i];
            while (A->ci[p] != j) ++p;
            const double* B = &A->v[(size_t)p * bv];
            double* C = &tv[(size_t)q * bv];
            for (int r = 0; r < bs; ++r)
                for (int c = 0; c < bs; ++c) C[r * bs + c] = B[c * bs + r];
        }
    return blk_take(bs, A->nbc, A->nbr, trp, tci, tv);
}

/* BlockMatrix::condense, blockMatrix.hpp:269-315: scalar CSR -> BAIJ. */
orc_blk* orc_blk_condense(int bs, const orc_csr* A, uint32_t nbr, uint32_t nbc)
{
    const int bv = bs * bs;
    uint32_t* rp = (uint32_t*)xcalloc((size_t)nbr + 1, 4);
    uint32_t** cols = (uint32_t**)xcalloc(nbr, sizeof(uint32_t*));
    for (uint32_t bi = 0; bi < nbr; ++bi)
    {
        uint32_t cnt = 0;
        for (uint32_t i = bi * bs; i < (bi + 1) * bs; ++i) cnt += A->rp[i + 1] - A->rp[i];
        uint32_t* out = (uint32_t*)xcalloc(cnt, 4);
        uint32_t k = 0;
        for (uint32_t i = bi * bs; i < (bi + 1) * bs; ++i)
            for (uint32_t p = A->rp[i]; p < A->rp[i + 1]; ++p) out[k++] = A->ci[p] / bs;
        qsort(out, k, 4, u32_cmp);
        uint32_t u = 0;
        for (uint32_t t = 0; t < k; ++t)
            if (u == 0 || out[u - 1] != out[t]) out[u++] = out[t];
        cols[bi] = out;
        rp[bi + 1] = u;
    }
    for (uint32_t bi = 0; bi < nbr; ++bi) rp[bi + 1] += rp[bi];
    uint32_t* ci = (uint32_t*)xcalloc(rp[nbr], 4);
    double* vv = (double*)xcalloc((size_t)rp[nbr] * bv, 8);
    for (uint32_t bi = 0; bi < nbr; ++bi)
    {
        const uint32_t cnt = rp[bi + 1] - rp[bi];
        for (uint32_t k = 0; k < cnt; ++k) ci[rp[bi] + k] = cols[bi][k];
        for (uint32_t i = bi * bs; i < (bi + 1) * bs; ++i)
        {
            const int r = (int)(i % bs);
            for (uint32_t p = A->rp[i]; p < A->rp[i + 1]; ++p)
            {
                const uint32_t bj = A->ci[p] / bs, c = A->ci[p] % bs;
                uint32_t lo = 0, hi = cnt; /* lower_bound */
                while (lo < hi)
                {
                    uint32_t mid = (lo + hi) / 2;
                    if (cols[bi][mid] < bj)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                const uint32_t boff = rp[bi] + lo;
                vv[(size_t)boff * bv + (size_t)r * bs + c] += A->v[p];
            }
        }
        free(cols[bi]);
    }
    free(cols);
    return blk_take(bs, nbr, nbc, rp, ci, vv);
}

/* blk_matmul, blockMatrix.hpp:883-932: dense-accumulator block SpGEMM,
 * columns sorted per row. */
orc_blk* orc_blk_matmul(const orc_blk* A, const orc_blk* B)
{
    const int bs = A->bs, bv = bs * bs;
    const uint32_t nr = A->nbr, nc = B->nbc;
    uint32_t* rp = (uint32_t*)xcalloc((size_t)nr + 1, 4);
    double* accum = (double*)xcalloc((size_t)nc * bv, 8);
    char* hit = (char*)xcalloc(nc, 1);
    uint32_t* hl = (uint32_t*)xcalloc(nc, 4);
    size_t cap = 1024, used = 0;
    uint32_t* ci = (uint32_t*)xcalloc(cap, 4);
    double* val = (double*)xcalloc(cap * bv, 8);
    for (uint32_t i = 0; i < nr; ++i)
    {
        uint32_t nh = 0;
        for (uint32_t pa = A->rp[i]; pa < A->rp[i + 1]; ++pa)
        {
            const uint32_t k = A->ci[pa];
            const double* ab = &A->v[(size_t)pa * bv];
            for (uint32_t pb = B->rp[k]; pb < B->rp[k + 1]; ++pb)
            {
                const uint32_t j = B->ci[pb];
                const double* bb = &B->v[(size_t)pb * bv];
                if (!hit[j])
                {
                    hit[j] = 1;
                    hl[nh++] = j;
                    memset(&accum[(size_t)j * bv], 0, 8 * (size_t)bv);
                }
                double* cb = &accum[(size_t)j * bv];
                for (int r = 0; r < bs; ++r)
                    for (int c = 0; c < bs; ++c)
                    {
                        double s = 0.0;
                        for (int m = 0; m < bs; ++m) s += ab[r * bs + m] * bb[m * bs + c];
                        cb[r * bs + c] += s;
                    }
            }
        }
        qsort(hl, nh, 4, u32_cmp);
        rp[i + 1] = nh;
        if (used + nh > cap)
        {
            while (used + nh > cap) cap *= 2;
            ci = (uint32_t*)realloc(ci, cap * 4);
            val = (double*)realloc(val, cap * bv * 8);
        }
        for (uint32_t t = 0; t < nh; ++t)
        {
            const uint32_t j = hl[t];
            ci[used] = j;
            memcpy(&val[used * bv], &accum[(size_t)j * bv], 8 * (size_t)bv);
            ++used;
            hit[j] = 0;
        }
    }
    for (uint32_t i = 0; i < nr; ++i) rp[i + 1] += rp[i];
    free(accum);
    free(hit);
    free(hl);
    return blk_take(bs, nr, nc, rp, ci, val);
}

/* ======================================================================
 * Preconditioners
 * ====================================================================== */

enum
{
    PC_NONE,
    PC_DIAG,
    PC_IC0,
    PC_ILU0,
    PC_SSOR,
    PC_BJACOBI,
    PC_BILU0,
    PC_AMG
};

typedef struct
{
    orc_blk* A;
    orc_blk* P;
    orc_blk* R;
    double* diag_inv;
    int32_t* agg;
    uint32_t nrows;
} amg_level;

struct orc_pc
{
    int kind;
    uint32_t n;      /* scalar length of r and z */
    int bs;
    /* diag */
    double* diag;
    /* IC0 / ILU0 (scalar) */
    uint32_t *Lrp, *Lci, *Urp, *Uci, *diag_idx;
    double *Lv, *Uv;
    /* SSOR */
    orc_csr* A2;
    uint32_t ncolor;
    uint32_t *color_ptr, *new_id, *perm;
    double *diag2, *f, *w, *z2;
    double omega;
    /* block Jacobi / block ILU0 */
    const orc_blk* Ablk; /* not owned (block Jacobi) */
    double* inv_diag;
    uint32_t* Udiag;
    /* AMG */
    amg_level* lv;
    int nlev;
    int exact_coarse;
    orc_blk* owned_blk; /* BS=1 condensed copy for scalar SA-AMG */
    double* coarse_lu;
    uint32_t* coarse_piv;
};

static orc_pc* pc_new(int kind, uint32_t n)
{
    orc_pc* pc = (orc_pc*)xcalloc(1, sizeof(orc_pc));
    pc->kind = kind;
    pc->n = n;
    return pc;
}

uint32_t orc_pc_n(const orc_pc* pc) { return pc->n; }

/* make_diag_preconditioner, array.cpp:2450-2508 */
static orc_pc* pc_diag(const orc_csr* A, int* st, char* err, int errlen)
{
    const uint32_t n = A->n;
    if (A->n != A->m)
    {
        *st = ORC_INVALID_ARG;
        set_err(err, errlen, "diag preconditioner needs a square matrix");
        return NULL;
    }
    orc_pc* pc = pc_new(PC_DIAG, n);
    pc->diag = (double*)xcalloc(n, 8);
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t k = A->rp[i]; k < A->rp[i + 1]; ++k)
            if (A->ci[k] == i)
            {
                pc->diag[i] = A->v[k];
                break;
            }
    for (uint32_t i = 0; i < n; ++i)
    {
        if (fabs(pc->diag[i]) < 1e-14 || pc->diag[i] <= 0.0)
        {
            *st = ORC_BREAKDOWN;
            set_err(err, errlen,
                    fabs(pc->diag[i]) < 1e-14 ? "diag preconditioner: zero or tiny diagonal entry"
                                              : "diag preconditioner: diagonal must be positive");
            orc_pc_free(pc);
            return NULL;
        }
    }
    return pc;
}

/* make_ic0_preconditioner, array.cpp:2522-2698 */
static orc_pc* pc_ic0(const orc_csr* A, int* st, char* err, int errlen)
{
    if (A->n != A->m)
    {
        *st = ORC_INVALID_ARG;
        set_err(err, errlen, "IC(0) needs a square matrix");
        return NULL;
    }
    const uint32_t n = A->n;
    orc_pc* pc = pc_new(PC_IC0, n);
    uint32_t* Lrp = pc->Lrp = (uint32_t*)xcalloc((size_t)n + 1, 4);
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t p = A->rp[i]; p < A->rp[i + 1]; ++p)
            if (A->ci[p] <= i) Lrp[i + 1]++;
    for (uint32_t i = 0; i < n; ++i) Lrp[i + 1] += Lrp[i];
    const uint32_t Lnnz = Lrp[n];
    uint32_t* Lci = pc->Lci = (uint32_t*)xcalloc(Lnnz, 4);
    double* Lv = pc->Lv = (double*)xcalloc(Lnnz, 8);
    for (uint32_t i = 0, d = 0; i < n; ++i)
        for (uint32_t p = A->rp[i]; p < A->rp[i + 1]; ++p)
            if (A->ci[p] <= i)
            {
                Lci[d] = A->ci[p];
                Lv[d] = A->v[p];
                ++d;
            }
    double* diag = pc->diag = (double*)xcalloc(n, 8);
    for (uint32_t i = 0; i < n; ++i)
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
            *st = ORC_BREAKDOWN;
            set_err(err, errlen, "IC(0) failed: missing diagonal entry");
            orc_pc_free(pc);
            return NULL;
        }
        double sd = 0.0;
        for (uint32_t p = rs; p < dp; ++p) sd += Lv[p] * Lv[p];
        const double dv = Lv[dp] - sd;
        if (dv <= 1e-14)
        {
            *st = ORC_BREAKDOWN;
            set_err(err, errlen, "IC(0) failed: matrix may not be SPD (non-positive pivot)");
            orc_pc_free(pc);
            return NULL;
        }
        Lv[dp] = sqrt(dv);
        diag[i] = Lv[dp];
    }
    /* L^T (strict part) as CSR, array.cpp:2659-2695 */
    uint32_t* Urp = pc->Urp = (uint32_t*)xcalloc((size_t)n + 1, 4);
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t p = Lrp[i]; p < Lrp[i + 1]; ++p)
            if (Lci[p] < i) Urp[Lci[p] + 1]++;
    for (uint32_t i = 0; i < n; ++i) Urp[i + 1] += Urp[i];
    pc->Uci = (uint32_t*)xcalloc(Urp[n], 4);
    pc->Uv = (double*)xcalloc(Urp[n], 8);
    uint32_t* off = (uint32_t*)xcalloc((size_t)n + 1, 4);
    memcpy(off, Urp, 4 * ((size_t)n + 1));
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t p = Lrp[i]; p < Lrp[i + 1]; ++p)
        {
            const uint32_t j = Lci[p];
            if (j < i)
            {
                const uint32_t d = off[j]++;
                pc->Uci[d] = i;
                pc->Uv[d] = Lv[p];
            }
        }
    free(off);
    return pc;
}

/* IC(0) apply, array.cpp:2700-2731 */
static void apply_ic0(orc_pc* pc, const double* rhs, double* z)
{
    const uint32_t n = pc->n;
    double* y = (double*)xcalloc(n, 8);
    for (uint32_t i = 0; i < n; ++i)
    {
        double sum = rhs[i];
        for (uint32_t p = pc->Lrp[i]; p < pc->Lrp[i + 1]; ++p)
        {
            const uint32_t j = pc->Lci[p];
            if (j >= i) break;
            sum -= pc->Lv[p] * y[j];
        }
        y[i] = sum / pc->diag[i];
    }
    for (uint32_t ii = n; ii-- > 0;)
    {
        double sum = y[ii];
        for (uint32_t p = pc->Urp[ii]; p < pc->Urp[ii + 1]; ++p) sum -= pc->Uv[p] * z[pc->Uci[p]];
        z[ii] = sum / pc->diag[ii];
    }
    free(y);
}

/* make_ilu0_preconditioner, array.cpp:2744-2900 */
static orc_pc* pc_ilu0(const orc_csr* A, int* st, char* err, int errlen)
{
    if (A->n != A->m)
    {
        *st = ORC_INVALID_ARG;
        set_err(err, errlen, "ILU(0) needs a square matrix");
        return NULL;
    }
    const uint32_t n = A->n;
    orc_pc* pc = pc_new(PC_ILU0, n);
    uint32_t* Lrp = pc->Lrp = (uint32_t*)xcalloc((size_t)n + 1, 4);
    uint32_t* Urp = pc->Urp = (uint32_t*)xcalloc((size_t)n + 1, 4);
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t p = A->rp[i]; p < A->rp[i + 1]; ++p)
        {
            if (A->ci[p] < i)
                Lrp[i + 1]++;
            else
                Urp[i + 1]++;
        }
    for (uint32_t i = 0; i < n; ++i)
    {
        Lrp[i + 1] += Lrp[i];
        Urp[i + 1] += Urp[i];
    }
    uint32_t* Lci = pc->Lci = (uint32_t*)xcalloc(Lrp[n], 4);
    double* Lv = pc->Lv = (double*)xcalloc(Lrp[n], 8);
    uint32_t* Uci = pc->Uci = (uint32_t*)xcalloc(Urp[n], 4);
    double* Uv = pc->Uv = (double*)xcalloc(Urp[n], 8);
    uint32_t* dix = pc->diag_idx = (uint32_t*)xcalloc(n, 4);
    char* has = (char*)xcalloc(n, 1);
    for (uint32_t i = 0, dl = 0, du = 0; i < n; ++i)
        for (uint32_t p = A->rp[i]; p < A->rp[i + 1]; ++p)
        {
            const uint32_t j = A->ci[p];
            if (j < i)
            {
                Lci[dl] = j;
                Lv[dl] = A->v[p];
                ++dl;
            }
            else
            {
                Uci[du] = j;
                Uv[du] = A->v[p];
                if (j == i)
                {
                    dix[i] = du;
                    has[i] = 1;
                }
                ++du;
            }
        }
    for (uint32_t i = 0; i < n; ++i)
        if (!has[i])
        {
            free(has);
            *st = ORC_BREAKDOWN;
            set_err(err, errlen, "ILU(0) failed: missing diagonal entry");
            orc_pc_free(pc);
            return NULL;
        }
    free(has);
    for (uint32_t i = 0; i < n; ++i)
    {
        const uint32_t us = Urp[i], ue = Urp[i + 1];
        for (uint32_t pl = Lrp[i]; pl < Lrp[i + 1]; ++pl)
        {
            const uint32_t k = Lci[pl];
            const uint32_t dk = dix[k];
            if (fabs(Uv[dk]) < 1e-30)
            {
                *st = ORC_BREAKDOWN;
                set_err(err, errlen, "ILU(0) breakdown: U_kk close to zero");
                orc_pc_free(pc);
                return NULL;
            }
            Lv[pl] /= Uv[dk];
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
    return pc;
}

/* ILU(0) apply, array.cpp:2902-2933 */
static void apply_ilu0(orc_pc* pc, const double* rhs, double* z)
{
    const uint32_t n = pc->n;
    double* y = (double*)xcalloc(n, 8);
    for (uint32_t i = 0; i < n; ++i)
    {
        double sum = rhs[i];
        for (uint32_t p = pc->Lrp[i]; p < pc->Lrp[i + 1]; ++p) sum -= pc->Lv[p] * y[pc->Lci[p]];
        y[i] = sum;
    }
    for (uint32_t ii = n; ii-- > 0;)
    {
        double sum = y[ii];
        for (uint32_t p = pc->Urp[ii]; p < pc->Urp[ii + 1]; ++p)
        {
            const uint32_t j = pc->Uci[p];
            if (j == ii) continue;
            sum -= pc->Uv[p] * z[j];
        }
        z[ii] = sum / pc->Uv[pc->diag_idx[ii]];
    }
    free(y);
}

/* make_redblack_data, array.cpp:2947-3067: colouring of the graph of A+A^T
 * (BFS 2-colouring, else greedy first-fit in natural order), colour-major
 * renumbering, A2 = P A P^T through the COO constructor, diag2. */
static int build_colouring(orc_pc* pc, const orc_csr* A, char* err, int errlen)
{
    const uint32_t n = A->n, nnz = A->rp[n];
    uint32_t* ATp = (uint32_t*)xcalloc((size_t)n + 1, 4);
    for (uint32_t p = 0; p < nnz; ++p) ATp[A->ci[p] + 1]++;
    for (uint32_t i = 0; i < n; ++i) ATp[i + 1] += ATp[i];
    uint32_t* ATr = (uint32_t*)xcalloc(nnz, 4);
    {
        uint32_t* off = (uint32_t*)xcalloc((size_t)n + 1, 4);
        memcpy(off, ATp, 4 * ((size_t)n + 1));
        for (uint32_t i = 0; i < n; ++i)
            for (uint32_t p = A->rp[i]; p < A->rp[i + 1]; ++p) ATr[off[A->ci[p]]++] = i;
        free(off);
    }
    int* color = (int*)xcalloc(n, sizeof(int));
    for (uint32_t i = 0; i < n; ++i) color[i] = -1;
    int bip = 1;
    uint32_t* queue = (uint32_t*)xcalloc(n, 4);
    for (uint32_t seed = 0; seed < n && bip; ++seed)
    {
        if (color[seed] != -1) continue;
        color[seed] = 0;
        uint32_t qn = 0;
        queue[qn++] = seed;
        for (uint32_t head = 0; head < qn && bip; ++head)
        {
            const uint32_t i = queue[head];
            for (int pass = 0; pass < 2; ++pass)
            {
                const uint32_t* ptr = pass == 0 ? A->rp : ATp;
                const uint32_t* idx = pass == 0 ? A->ci : ATr;
                for (uint32_t p = ptr[i]; p < ptr[i + 1]; ++p)
                {
                    const uint32_t j = idx[p];
                    if (j == i) continue;
                    if (color[j] == -1)
                    {
                        color[j] = 1 - color[i];
                        queue[qn++] = j;
                    }
                    else if (color[j] == color[i])
                        bip = 0;
                }
            }
        }
    }
    free(queue);
    if (!bip)
    {
        for (uint32_t i = 0; i < n; ++i) color[i] = -1;
        char* used = (char*)xcalloc((size_t)n + 1, 1);
        uint32_t* touched = (uint32_t*)xcalloc((size_t)n + 1, 4);
        for (uint32_t i = 0; i < n; ++i)
        {
            uint32_t nt = 0;
            for (int pass = 0; pass < 2; ++pass)
            {
                const uint32_t* ptr = pass == 0 ? A->rp : ATp;
                const uint32_t* idx = pass == 0 ? A->ci : ATr;
                for (uint32_t p = ptr[i]; p < ptr[i + 1]; ++p)
                {
                    const uint32_t j = idx[p];
                    if (j == i) continue;
                    const int c = color[j];
                    if (c >= 0 && !used[c])
                    {
                        used[c] = 1;
                        touched[nt++] = (uint32_t)c;
                    }
                }
            }
            int c = 0;
            while (used[c]) ++c;
            color[i] = c;
            for (uint32_t t = 0; t < nt; ++t) used[touched[t]] = 0;
        }
        free(used);
        free(touched);
    }
    free(ATp);
    free(ATr);
    uint32_t nc = 0;
    for (uint32_t i = 0; i < n; ++i)
        if ((uint32_t)color[i] + 1 > nc) nc = (uint32_t)color[i] + 1;
    pc->ncolor = nc;
    pc->color_ptr = (uint32_t*)xcalloc((size_t)nc + 1, 4);
    for (uint32_t i = 0; i < n; ++i) pc->color_ptr[color[i] + 1]++;
    for (uint32_t c = 0; c < nc; ++c) pc->color_ptr[c + 1] += pc->color_ptr[c];
    pc->new_id = (uint32_t*)xcalloc(n, 4);
    {
        uint32_t* off = (uint32_t*)xcalloc((size_t)nc + 1, 4);
        memcpy(off, pc->color_ptr, 4 * ((size_t)nc + 1));
        for (uint32_t i = 0; i < n; ++i) pc->new_id[i] = off[color[i]]++;
        free(off);
    }
    free(color);
    pc->perm = (uint32_t*)xcalloc(n, 4);
    for (uint32_t i = 0; i < n; ++i) pc->perm[pc->new_id[i]] = i;
    double* v2 = (double*)xcalloc(nnz, 8);
    uint32_t* r2 = (uint32_t*)xcalloc(nnz, 4);
    uint32_t* c2 = (uint32_t*)xcalloc(nnz, 4);
    uint32_t k = 0;
    for (uint32_t ni = 0; ni < n; ++ni)
    {
        const uint32_t i = pc->perm[ni];
        for (uint32_t p = A->rp[i]; p < A->rp[i + 1]; ++p)
        {
            r2[k] = ni;
            c2[k] = pc->new_id[A->ci[p]];
            v2[k] = A->v[p];
            ++k;
        }
    }
    int st = 0;
    pc->A2 = orc_csr_from_coo(n, n, nnz, v2, r2, c2, &st);
    free(v2);
    free(r2);
    free(c2);
    pc->diag2 = (double*)xcalloc(n, 8);
    for (uint32_t ni = 0; ni < n; ++ni)
    {
        int found = 0;
        for (uint32_t p = pc->A2->rp[ni]; p < pc->A2->rp[ni + 1]; ++p)
            if (pc->A2->ci[p] == ni)
            {
                pc->diag2[ni] = pc->A2->v[p];
                found = 1;
                break;
            }
        if (!found || fabs(pc->diag2[ni]) < 1e-300)
        {
            set_err(err, errlen, "SSOR/red-black failed: missing nonzero diagonal");
            return ORC_BREAKDOWN;
        }
    }
    pc->f = (double*)xcalloc(n, 8);
    pc->w = (double*)xcalloc(n, 8);
    pc->z2 = (double*)xcalloc(n, 8);
    return ORC_OK;
}

/* make_ssor_preconditioner, array.cpp:3068-3091 */
static orc_pc* pc_ssor(const orc_csr* A, double omega, int* st, char* err, int errlen)
{
    if (A->n != A->m)
    {
        *st = ORC_INVALID_ARG;
        set_err(err, errlen, "SSOR needs a square matrix");
        return NULL;
    }
    if (!(omega > 0.0 && omega < 2.0))
    {
        *st = ORC_INVALID_ARG;
        set_err(err, errlen, "SSOR: relaxation factor must satisfy 0 < omega < 2");
        return NULL;
    }
    orc_pc* pc = pc_new(PC_SSOR, A->n);
    pc->omega = omega;
    int s = build_colouring(pc, A, err, errlen);
    if (s != ORC_OK)
    {
        *st = s;
        orc_pc_free(pc);
        return NULL;
    }
    return pc;
}

/* SSOR apply, array.cpp:3093-3163 */
static void apply_ssor(orc_pc* pc, const double* rhs, double* z)
{
    const uint32_t n = pc->n;
    const double omega = pc->omega, fw = omega * (2.0 - omega);
    const uint32_t *r2 = pc->A2->rp, *c2 = pc->A2->ci;
    const double *v2 = pc->A2->v, *d2 = pc->diag2;
    double *f = pc->f, *w = pc->w, *z2 = pc->z2;
    for (uint32_t i = 0; i < n; ++i) f[i] = rhs[pc->perm[i]];
    for (uint32_t c = 0; c < pc->ncolor; ++c)
        for (uint32_t ii = pc->color_ptr[c]; ii < pc->color_ptr[c + 1]; ++ii)
        {
            double sigma = fw * f[ii];
            for (uint32_t p = r2[ii]; p < r2[ii + 1]; ++p)
                if (c2[p] < ii) sigma -= omega * v2[p] * w[c2[p]];
            w[ii] = sigma / d2[ii];
        }
    for (uint32_t cc = pc->ncolor; cc-- > 0;)
        for (uint32_t ii = pc->color_ptr[cc]; ii < pc->color_ptr[cc + 1]; ++ii)
        {
            double sigma = 0.0;
            for (uint32_t p = r2[ii]; p < r2[ii + 1]; ++p)
                if (c2[p] > ii) sigma += v2[p] * z2[c2[p]];
            z2[ii] = w[ii] - (omega / d2[ii]) * sigma;
        }
    for (uint32_t i = 0; i < n; ++i) z[i] = z2[pc->new_id[i]];
}

/* ---------------- block Jacobi (BlockMatrix::gmres "blockjacobi", blockMatrix.hpp:714-733) */
static void apply_bjacobi(orc_pc* pc, const double* r, double* z)
{
    const orc_blk* A = pc->Ablk;
    const int bs = A->bs, bv = bs * bs;
    for (uint32_t bi = 0; bi < A->nbr; ++bi)
    {
        double tmp[8], Minv[64];
        for (int c = 0; c < bs; ++c) tmp[c] = r[(size_t)bi * bs + c];
        blk_inv(bs, &A->v[(size_t)A->diag_ptr[bi] * bv], Minv);
        blk_mv(bs, Minv, tmp, &z[(size_t)bi * bs]);
    }
}

/* ---------------- block ILU(0) (make_block_ilu0_preconditioner, blockMatrix.hpp:455-576) */
static orc_pc* pc_bilu0(const orc_blk* A, int* st, char* err, int errlen)
{
    if (A->nbr != A->nbc)
    {
        *st = ORC_INVALID_ARG;
        set_err(err, errlen, "Block-ILU(0) needs a square block matrix");
        return NULL;
    }
    const uint32_t nb = A->nbr;
    const int bs = A->bs, bv = bs * bs;
    orc_pc* pc = pc_new(PC_BILU0, nb * (uint32_t)bs);
    pc->bs = bs;
    uint32_t* Lrp = pc->Lrp = (uint32_t*)xcalloc((size_t)nb + 1, 4);
    uint32_t* Urp = pc->Urp = (uint32_t*)xcalloc((size_t)nb + 1, 4);
    for (uint32_t I = 0; I < nb; ++I)
        for (uint32_t p = A->rp[I]; p < A->rp[I + 1]; ++p)
        {
            if (A->ci[p] < I)
                Lrp[I + 1]++;
            else
                Urp[I + 1]++;
        }
    for (uint32_t I = 0; I < nb; ++I)
    {
        Lrp[I + 1] += Lrp[I];
        Urp[I + 1] += Urp[I];
    }
    uint32_t* Lci = pc->Lci = (uint32_t*)xcalloc(Lrp[nb], 4);
    double* Lv = pc->Lv = (double*)xcalloc((size_t)Lrp[nb] * bv, 8);
    uint32_t* Uci = pc->Uci = (uint32_t*)xcalloc(Urp[nb], 4);
    double* Uv = pc->Uv = (double*)xcalloc((size_t)Urp[nb] * bv, 8);
    uint32_t* Ud = pc->Udiag = (uint32_t*)xcalloc(nb, 4);
    for (uint32_t I = 0; I < nb; ++I) Ud[I] = ORC_NONE;
    for (uint32_t I = 0, dl = 0, du = 0; I < nb; ++I)
        for (uint32_t p = A->rp[I]; p < A->rp[I + 1]; ++p)
        {
            const uint32_t J = A->ci[p];
            const double* src = &A->v[(size_t)p * bv];
            if (J < I)
            {
                Lci[dl] = J;
                memcpy(&Lv[(size_t)dl * bv], src, 8 * (size_t)bv);
                ++dl;
            }
            else
            {
                Uci[du] = J;
                memcpy(&Uv[(size_t)du * bv], src, 8 * (size_t)bv);
                if (J == I) Ud[I] = du;
                ++du;
            }
        }
    for (uint32_t I = 0; I < nb; ++I)
        if (Ud[I] == ORC_NONE)
        {
            *st = ORC_BREAKDOWN;
            set_err(err, errlen, "Block-ILU(0) failed: missing diagonal block");
            orc_pc_free(pc);
            return NULL;
        }
    double* inv = pc->inv_diag = (double*)xcalloc((size_t)nb * bv, 8);
    for (uint32_t I = 0; I < nb; ++I)
    {
        const uint32_t Ls = Lrp[I], Le = Lrp[I + 1], Us = Urp[I], Ue = Urp[I + 1];
        for (uint32_t pL = Ls; pL < Le; ++pL)
        {
            const uint32_t K = Lci[pL];
            double* LIK = &Lv[(size_t)pL * bv];
            for (uint32_t q = Ls; q < pL; ++q)
            {
                const uint32_t J = Lci[q];
                const uint32_t pJK = blk_find(Urp, Uci, J, K);
                if (pJK != ORC_NONE) blk_mma(bs, &Lv[(size_t)q * bv], &Uv[(size_t)pJK * bv], LIK);
            }
            blk_rmul(bs, LIK, &inv[(size_t)K * bv]);
            uint32_t pi = Us, pk = Urp[K];
            const uint32_t ek = Urp[K + 1];
            while (pi < Ue && pk < ek)
            {
                if (Uci[pi] == Uci[pk])
                {
                    blk_mma(bs, LIK, &Uv[(size_t)pk * bv], &Uv[(size_t)pi * bv]);
                    ++pi;
                    ++pk;
                }
                else if (Uci[pi] < Uci[pk])
                    ++pi;
                else
                    ++pk;
            }
        }
        if (!blk_inv(bs, &Uv[(size_t)Ud[I] * bv], &inv[(size_t)I * bv]))
        {
            *st = ORC_BREAKDOWN;
            set_err(err, errlen, "Block-ILU(0) breakdown: singular diagonal block");
            orc_pc_free(pc);
            return NULL;
        }
    }
    pc->f = (double*)xcalloc(pc->n, 8); /* y buffer */
    return pc;
}

/* Block ILU(0) apply, blockMatrix.hpp:578-622 */
static void apply_bilu0(orc_pc* pc, const double* rhs, double* z)
{
    const int bs = pc->bs, bv = bs * bs;
    const uint32_t nb = pc->n / (uint32_t)bs;
    double* y = pc->f;
    for (uint32_t I = 0; I < nb; ++I)
    {
        double* yI = &y[(size_t)I * bs];
        for (int c = 0; c < bs; ++c) yI[c] = rhs[(size_t)I * bs + c];
        for (uint32_t p = pc->Lrp[I]; p < pc->Lrp[I + 1]; ++p)
        {
            const double* LIJ = &pc->Lv[(size_t)p * bv];
            const double* yJ = &y[(size_t)pc->Lci[p] * bs];
            for (int r = 0; r < bs; ++r)
            {
                double s = 0.0;
                for (int c = 0; c < bs; ++c) s += LIJ[r * bs + c] * yJ[c];
                yI[r] -= s;
            }
        }
    }
    for (uint32_t II = nb; II-- > 0;)
    {
        double tmp[8];
        for (int c = 0; c < bs; ++c) tmp[c] = y[(size_t)II * bs + c];
        for (uint32_t p = pc->Urp[II]; p < pc->Urp[II + 1]; ++p)
        {
            const uint32_t J = pc->Uci[p];
            if (J == II) continue;
            const double* UIJ = &pc->Uv[(size_t)p * bv];
            const double* zJ = &z[(size_t)J * bs];
            for (int r = 0; r < bs; ++r)
            {
                double s = 0.0;
                for (int c = 0; c < bs; ++c) s += UIJ[r * bs + c] * zJ[c];
                tmp[r] -= s;
            }
        }
        blk_mv(bs, &pc->inv_diag[(size_t)II * bv], tmp, &z[(size_t)II * bs]);
    }
}

/* Parallel aggregation rule of the library (no reference counterpart),
 * restated serially with the same snapshots: distance-2 independent roots
 * chosen in rounds by a fixed per-row key, then neighbour assignment, then
 * singletons.  Each round reads only the previous round's state. */
static uint64_t agg_key(uint32_t i)
{
    uint32_t x = i;
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return ((uint64_t)x << 32) | (uint64_t)(i + 1u);
}

static int32_t aggregate_mis(uint32_t n, const uint32_t* sp, const uint32_t* sc, int32_t* agg)
{
    enum { UND = 0, ROOT = 1, OUT = 2 };
    uint8_t* st = (uint8_t*)xcalloc(n ? n : 1, 1);
    uint8_t* c1 = (uint8_t*)xcalloc(n ? n : 1, 1);
    uint64_t* m1 = (uint64_t*)xcalloc(n ? n : 1, 8);
    uint32_t left = n;
    while (left)
    {
        for (uint32_t i = 0; i < n; ++i)
        {
            uint64_t m = st[i] == UND ? agg_key(i) : 0;
            for (uint32_t p = sp[i]; p < sp[i + 1]; ++p)
                if (st[sc[p]] == UND && agg_key(sc[p]) > m) m = agg_key(sc[p]);
            m1[i] = m;
        }
        for (uint32_t i = 0; i < n; ++i)
        {
            if (st[i] != UND) continue;
            uint64_t m = m1[i];
            for (uint32_t p = sp[i]; p < sp[i + 1]; ++p)
                if (m1[sc[p]] > m) m = m1[sc[p]];
            if (m == agg_key(i)) st[i] = ROOT; /* reads only m1: the order of i does not matter */
        }
        for (uint32_t i = 0; i < n; ++i)
        {
            int c = st[i] == ROOT;
            for (uint32_t p = sp[i]; p < sp[i + 1] && !c; ++p) c = st[sc[p]] == ROOT;
            c1[i] = (uint8_t)c;
        }
        left = 0;
        for (uint32_t i = 0; i < n; ++i)
        {
            if (st[i] != UND) continue;
            int c = c1[i];
            for (uint32_t p = sp[i]; p < sp[i + 1] && !c; ++p) c = c1[sc[p]];
            if (c)
                st[i] = OUT;
            else
                ++left;
        }
    }
    int32_t nroots = 0;
    int32_t* rank = (int32_t*)xcalloc(n ? n : 1, 4);
    for (uint32_t i = 0; i < n; ++i)
        if (st[i] == ROOT) rank[i] = nroots++;
    for (uint32_t i = 0; i < n; ++i)
    {
        if (st[i] == ROOT)
        {
            agg[i] = rank[i];
            continue;
        }
        uint64_t best = 0;
        int32_t g = -1;
        for (uint32_t p = sp[i]; p < sp[i + 1]; ++p)
            if (st[sc[p]] == ROOT && agg_key(sc[p]) > best)
            {
                best = agg_key(sc[p]);
                g = rank[sc[p]];
            }
        agg[i] = g;
    }
    int32_t* snap = (int32_t*)xcalloc(n ? n : 1, 4);
    memcpy(snap, agg, 4 * (size_t)n);
    for (uint32_t i = 0; i < n; ++i)
    {
        if (snap[i] >= 0) continue;
        uint64_t best = 0;
        int32_t g = -1;
        for (uint32_t p = sp[i]; p < sp[i + 1]; ++p)
            if (snap[sc[p]] >= 0 && agg_key(sc[p]) > best)
            {
                best = agg_key(sc[p]);
                g = snap[sc[p]];
            }
        agg[i] = g;
    }
    int32_t nagg = nroots;
    for (uint32_t i = 0; i < n; ++i)
        if (agg[i] < 0) agg[i] = nagg++;
    free(st);
    free(c1);
    free(m1);
    free(rank);
    free(snap);
    return nagg;
}

/* ---------------- block SA-AMG (make_block_amg_preconditioner, blockMatrix.hpp:1051-1179)
 * agg_mode: 0 the reference's capped greedy rule, 1 sequential three-phase
 * rule, 2 the library's parallel rule (aggregate_mis). */
static orc_pc* pc_amg(const orc_blk* A0, int exact, int agg_mode, int* st, char* err, int errlen)
{
    if (A0->nbr != A0->nbc)
    {
        *st = ORC_INVALID_ARG;
        set_err(err, errlen, "Block AMG needs a square block matrix");
        return NULL;
    }
    const int bs = A0->bs, bv = bs * bs;
    const double theta = 0.25, omega = 2.0 / 3.0;
    const int max_levels = 20, max_agg = 4;
    const uint32_t coarse_max = 50;
    orc_pc* pc = pc_new(PC_AMG, A0->nbr * (uint32_t)bs);
    pc->bs = bs;
    pc->exact_coarse = exact;
    pc->lv = (amg_level*)xcalloc((size_t)max_levels, sizeof(amg_level));
    orc_blk* cur = orc_blk_create(bs, A0->nbr, A0->nbc, A0->rp, A0->ci, A0->v);
    for (int lvl = 0; lvl < max_levels; ++lvl)
    {
        const uint32_t n = cur->nbr;
        amg_level* L = &pc->lv[pc->nlev];
        L->A = cur;
        L->nrows = n;
        L->diag_inv = (double*)xcalloc((size_t)n * bv, 8);
        for (uint32_t i = 0; i < n; ++i)
            blk_inv(bs, &cur->v[(size_t)cur->diag_ptr[i] * bv], &L->diag_inv[(size_t)i * bv]);
        if (n <= coarse_max)
        {
            pc->nlev++;
            cur = NULL;
            break;
        }
        /* 1. strength by block Frobenius norm, blockMatrix.hpp:1084-1099 */
        uint32_t* sp = (uint32_t*)xcalloc((size_t)n + 1, 4);
        uint32_t* sc = (uint32_t*)xcalloc(cur->rp[n], 4);
        for (uint32_t i = 0; i < n; ++i)
        {
            double mx = 0.0;
            for (uint32_t p = cur->rp[i]; p < cur->rp[i + 1]; ++p)
                if (cur->ci[p] != i)
                {
                    const double fn = blk_fro(bs, &cur->v[(size_t)p * bv]);
                    mx = mx < fn ? fn : mx; /* std::max(mx, fn) */
                }
            const double thr = theta * mx;
            sp[i + 1] = sp[i];
            for (uint32_t p = cur->rp[i]; p < cur->rp[i + 1]; ++p)
                if (cur->ci[p] != i && blk_fro(bs, &cur->v[(size_t)p * bv]) >= thr) sc[sp[i + 1]++] = cur->ci[p];
        }
        int32_t* agg = L->agg = (int32_t*)xcalloc(n, 4);
        for (uint32_t i = 0; i < n; ++i) agg[i] = -1;
        int32_t nagg = 0;
        if (agg_mode == 2)
            nagg = aggregate_mis(n, sp, sc, agg);
        else if (agg_mode == 0)
        {
            /* 2. greedy aggregation, natural order, <= max_agg, blockMatrix.hpp:1101-1111 */
            for (uint32_t i = 0; i < n; ++i)
            {
                if (agg[i] != -1) continue;
                agg[i] = nagg;
                int sz = 1;
                for (uint32_t p = sp[i]; p < sp[i + 1]; ++p)
                {
                    const uint32_t j = sc[p];
                    if (agg[j] == -1 && sz < max_agg)
                    {
                        agg[j] = nagg;
                        ++sz;
                    }
                }
                ++nagg;
            }
        }
        else
        {
            /* standard smoothed-aggregation rule (no reference counterpart; the
             * reference's capped greedy rule stalls on 3-D problems):
             * 1. a row whose strong neighbours are all free becomes a root and
             *    takes them all; 2. a free row joins the phase-1 aggregate of
             *    its first aggregated strong neighbour; 3. the remaining rows
             *    group with their free strong neighbours. */
            for (uint32_t i = 0; i < n; ++i)
            {
                if (agg[i] != -1) continue;
                int free_all = 1;
                for (uint32_t p = sp[i]; p < sp[i + 1]; ++p)
                    if (agg[sc[p]] != -1)
                    {
                        free_all = 0;
                        break;
                    }
                if (!free_all) continue;
                agg[i] = nagg;
                for (uint32_t p = sp[i]; p < sp[i + 1]; ++p) agg[sc[p]] = nagg;
                ++nagg;
            }
            int32_t* snap = (int32_t*)xcalloc(n, 4);
            memcpy(snap, agg, 4 * (size_t)n);
            for (uint32_t i = 0; i < n; ++i)
            {
                if (snap[i] != -1) continue;
                for (uint32_t p = sp[i]; p < sp[i + 1]; ++p)
                    if (snap[sc[p]] != -1)
                    {
                        agg[i] = snap[sc[p]];
                        break;
                    }
            }
            free(snap);
            for (uint32_t i = 0; i < n; ++i)
            {
                if (agg[i] != -1) continue;
                agg[i] = nagg;
                for (uint32_t p = sp[i]; p < sp[i + 1]; ++p)
                    if (agg[sc[p]] == -1) agg[sc[p]] = nagg;
                ++nagg;
            }
        }
        free(sp);
        free(sc);
        /* 3-4. smoothed prolongation P = (I - omega D^-1 A) P_t, blockMatrix.hpp:1113-1164.
         * Row i of P has one block per distinct aggregate among {agg[i]} and
         * {agg[k] : k in row i of A}, columns ascending (std::map order). */
        uint32_t* prp = (uint32_t*)xcalloc((size_t)n + 1, 4);
        size_t cap = (size_t)cur->rp[n] + n, used = 0;
        uint32_t* pci = (uint32_t*)xcalloc(cap, 4);
        double* pv = (double*)xcalloc(cap * bv, 8);
        uint32_t* gl = (uint32_t*)xcalloc((size_t)(cur->rp[n] + 1), 4);
        double* blks = (double*)xcalloc(((size_t)cur->rp[n] + 1) * bv, 8);
        for (uint32_t i = 0; i < n; ++i)
        {
            uint32_t ng = 0;
            /* identity term at agg[i] */
            gl[ng] = (uint32_t)agg[i];
            memset(&blks[0], 0, 8 * (size_t)bv);
            for (int r = 0; r < bs; ++r) blks[r * bs + r] = 1.0;
            ng = 1;
            const double* dinv = &L->diag_inv[(size_t)i * bv];
            for (uint32_t p = cur->rp[i]; p < cur->rp[i + 1]; ++p)
            {
                const uint32_t g = (uint32_t)agg[cur->ci[p]];
                const double* ab = &cur->v[(size_t)p * bv];
                uint32_t slot = ng;
                for (uint32_t t = 0; t < ng; ++t)
                    if (gl[t] == g)
                    {
                        slot = t;
                        break;
                    }
                if (slot == ng)
                {
                    gl[ng] = g;
                    memset(&blks[(size_t)ng * bv], 0, 8 * (size_t)bv);
                    ++ng;
                }
                double* dst = &blks[(size_t)slot * bv];
                for (int r = 0; r < bs; ++r)
                    for (int c = 0; c < bs; ++c)
                    {
                        double s = 0.0;
                        for (int m = 0; m < bs; ++m) s += dinv[r * bs + m] * ab[m * bs + c];
                        dst[r * bs + c] -= omega * s;
                    }
            }
            /* emit in ascending aggregate order */
            for (uint32_t e = 0; e < ng; ++e)
            {
                uint32_t best = ORC_NONE, bt = 0;
                for (uint32_t t = 0; t < ng; ++t)
                {
                    if (gl[t] == ORC_NONE) continue;
                    if (best == ORC_NONE || gl[t] < best)
                    {
                        best = gl[t];
                        bt = t;
                    }
                }
                pci[used] = best;
                memcpy(&pv[used * bv], &blks[(size_t)bt * bv], 8 * (size_t)bv);
                ++used;
                gl[bt] = ORC_NONE;
            }
            prp[i + 1] = (uint32_t)used;
        }
        free(gl);
        free(blks);
        L->P = blk_take(bs, n, (uint32_t)nagg, prp, pci, pv);
        L->R = orc_blk_transpose(L->P);
        pc->nlev++;
        /* 5. Galerkin A_c = R (A P), blockMatrix.hpp:1169-1170 */
        orc_blk* AP = orc_blk_matmul(cur, L->P);
        cur = orc_blk_matmul(L->R, AP);
        orc_blk_free(AP);
    }
    if (cur) orc_blk_free(cur); /* max_levels reached: last Galerkin product is unused */
    if (exact)
    {
        /* correct coarsest solve: dense LU with partial pivoting, RHS permuted */
        amg_level* L = &pc->lv[pc->nlev - 1];
        const int sz = (int)(L->nrows * (uint32_t)bs);
        double* d = pc->coarse_lu = (double*)xcalloc((size_t)sz * sz, 8);
        uint32_t* piv = pc->coarse_piv = (uint32_t*)xcalloc((size_t)sz, 4);
        for (uint32_t i = 0; i < L->nrows; ++i)
            for (uint32_t p = L->A->rp[i]; p < L->A->rp[i + 1]; ++p)
            {
                const uint32_t j = L->A->ci[p];
                for (int r = 0; r < bs; ++r)
                    for (int c = 0; c < bs; ++c)
                        d[(size_t)(i * bs + r) * sz + j * bs + c] = L->A->v[(size_t)p * bv + r * bs + c];
            }
        for (int i = 0; i < sz; ++i) piv[i] = (uint32_t)i;
        for (int k = 0; k < sz; ++k)
        {
            int pk = k;
            for (int i = k + 1; i < sz; ++i)
                if (fabs(d[(size_t)i * sz + k]) > fabs(d[(size_t)pk * sz + k])) pk = i;
            if (pk != k)
            {
                for (int j = 0; j < sz; ++j)
                {
                    double t = d[(size_t)k * sz + j];
                    d[(size_t)k * sz + j] = d[(size_t)pk * sz + j];
                    d[(size_t)pk * sz + j] = t;
                }
                uint32_t t = piv[k];
                piv[k] = piv[pk];
                piv[pk] = t;
            }
            if (fabs(d[(size_t)k * sz + k]) < 1e-300) d[(size_t)k * sz + k] = 1e-300;
            for (int i = k + 1; i < sz; ++i)
            {
                const double f = d[(size_t)i * sz + k] / d[(size_t)k * sz + k];
                d[(size_t)i * sz + k] = f;
                for (int j = k + 1; j < sz; ++j) d[(size_t)i * sz + j] -= f * d[(size_t)k * sz + j];
            }
        }
    }
    return pc;
}

/* coarsest level, reference form: blockMatrix.hpp:958-1000 (row swaps not
 * applied to the RHS; the forward sweep reads multipliers that elimination
 * already zeroed, so it does nothing). */
static void coarse_ref(const amg_level* L, int bs, const double* rhs, double* sol)
{
    const int bv = bs * bs, sz = (int)(L->nrows * (uint32_t)bs);
    double* d = (double*)xcalloc((size_t)sz * sz, 8);
    for (uint32_t i = 0; i < L->nrows; ++i)
        for (uint32_t p = L->A->rp[i]; p < L->A->rp[i + 1]; ++p)
        {
            const uint32_t j = L->A->ci[p];
            for (int r = 0; r < bs; ++r)
                for (int c = 0; c < bs; ++c)
                    d[(size_t)(i * bs + r) * sz + j * bs + c] = L->A->v[(size_t)p * bv + r * bs + c];
        }
    for (int k = 0; k < sz; ++k)
    {
        int pk = k;
        for (int i = k + 1; i < sz; ++i)
            if (fabs(d[(size_t)i * sz + k]) > fabs(d[(size_t)pk * sz + k])) pk = i;
        if (pk != k)
            for (int j = 0; j < sz; ++j)
            {
                double t = d[(size_t)k * sz + j];
                d[(size_t)k * sz + j] = d[(size_t)pk * sz + j];
                d[(size_t)pk * sz + j] = t;
            }
        double dk = d[(size_t)k * sz + k];
        if (fabs(dk) < 1e-14) dk = (dk >= 0 ? 1e-14 : -1e-14);
        for (int i = k + 1; i < sz; ++i)
        {
            const double f = d[(size_t)i * sz + k] / dk;
            for (int j = k; j < sz; ++j) d[(size_t)i * sz + j] -= f * d[(size_t)k * sz + j];
        }
    }
    double* x = (double*)xcalloc((size_t)sz, 8);
    memcpy(x, rhs, 8 * (size_t)sz);
    for (int k = 0; k < sz; ++k)
    {
        double dk = d[(size_t)k * sz + k];
        if (fabs(dk) < 1e-14) dk = (dk >= 0 ? 1e-14 : -1e-14);
        for (int i = k + 1; i < sz; ++i) x[i] -= (d[(size_t)i * sz + k] / dk) * x[k];
    }
    for (int i = sz - 1; i >= 0; --i)
    {
        for (int j = i + 1; j < sz; ++j) x[i] -= d[(size_t)i * sz + j] * x[j];
        double di = d[(size_t)i * sz + i];
        if (fabs(di) < 1e-14) di = (di >= 0 ? 1e-14 : -1e-14);
        x[i] /= di;
    }
    memcpy(sol, x, 8 * (size_t)sz);
    free(x);
    free(d);
}

static void coarse_exact(const orc_pc* pc, int sz, const double* rhs, double* sol)
{
    const double* d = pc->coarse_lu;
    for (int i = 0; i < sz; ++i) sol[i] = rhs[pc->coarse_piv[i]];
    for (int i = 0; i < sz; ++i)
        for (int j = 0; j < i; ++j) sol[i] -= d[(size_t)i * sz + j] * sol[j];
    for (int i = sz - 1; i >= 0; --i)
    {
        for (int j = i + 1; j < sz; ++j) sol[i] -= d[(size_t)i * sz + j] * sol[j];
        sol[i] /= d[(size_t)i * sz + i];
    }
}

static void amg_smooth(const amg_level* L, int bs, double omega, const double* rhs, double* sol, double* tmp,
                       double* r)
{
    const int bv = bs * bs;
    const uint32_t n = L->nrows, ndof = n * (uint32_t)bs;
    orc_blk_matvec(L->A, sol, tmp);
    for (uint32_t i = 0; i < ndof; ++i) r[i] = rhs[i] - tmp[i];
    for (uint32_t i = 0; i < n; ++i)
    {
        const double* dinv = &L->diag_inv[(size_t)i * bv];
        for (int c = 0; c < bs; ++c)
        {
            double corr = 0.0;
            for (int rr = 0; rr < bs; ++rr) corr += dinv[c * bs + rr] * r[i * bs + rr];
            sol[i * bs + c] += omega * corr;
        }
    }
}

/* blk_amg_vcycle, blockMatrix.hpp:946-1046 (sol enters as zeros) */
static void amg_vcycle(const orc_pc* pc, int lvl, const double* rhs, double* sol)
{
    const int bs = pc->bs;
    const amg_level* L = &pc->lv[lvl];
    const uint32_t ndof = L->nrows * (uint32_t)bs;
    const double omega = 2.0 / 3.0;
    if (lvl == pc->nlev - 1)
    {
        if (pc->exact_coarse)
            coarse_exact(pc, (int)ndof, rhs, sol);
        else
            coarse_ref(L, bs, rhs, sol);
        return;
    }
    double* tmp = (double*)xcalloc(ndof, 8);
    double* r = (double*)xcalloc(ndof, 8);
    amg_smooth(L, bs, omega, rhs, sol, tmp, r);
    orc_blk_matvec(L->A, sol, tmp);
    for (uint32_t i = 0; i < ndof; ++i) r[i] = rhs[i] - tmp[i];
    const uint32_t nc = L->R->nbr * (uint32_t)bs;
    double* rc = (double*)xcalloc(nc, 8);
    double* ec = (double*)xcalloc(nc, 8);
    orc_blk_matvec(L->R, r, rc);
    amg_vcycle(pc, lvl + 1, rc, ec);
    orc_blk_matvec(L->P, ec, tmp);
    for (uint32_t i = 0; i < ndof; ++i) sol[i] += tmp[i];
    amg_smooth(L, bs, omega, rhs, sol, tmp, r);
    free(rc);
    free(ec);
    free(tmp);
    free(r);
}

void orc_pc_apply(orc_pc* pc, const double* r, double* z)
{
    switch (pc->kind)
    {
        case PC_NONE: memcpy(z, r, 8 * (size_t)pc->n); break;
        case PC_DIAG:
            for (uint32_t i = 0; i < pc->n; ++i) z[i] = r[i] / pc->diag[i];
            break;
        case PC_IC0: apply_ic0(pc, r, z); break;
        case PC_ILU0: apply_ilu0(pc, r, z); break;
        case PC_SSOR: apply_ssor(pc, r, z); break;
        case PC_BJACOBI: apply_bjacobi(pc, r, z); break;
        case PC_BILU0: apply_bilu0(pc, r, z); break;
        case PC_AMG:
            memset(z, 0, 8 * (size_t)pc->n);
            amg_vcycle(pc, 0, r, z);
            break;
    }
}

void orc_pc_free(orc_pc* pc)
{
    if (!pc) return;
    free(pc->diag);
    free(pc->Lrp);
    free(pc->Lci);
    free(pc->Lv);
    free(pc->Urp);
    free(pc->Uci);
    free(pc->Uv);
    free(pc->diag_idx);
    orc_csr_free(pc->A2);
    free(pc->color_ptr);
    free(pc->new_id);
    free(pc->perm);
    free(pc->diag2);
    free(pc->f);
    free(pc->w);
    free(pc->z2);
    free(pc->inv_diag);
    free(pc->Udiag);
    for (int l = 0; l < pc->nlev; ++l)
    {
        orc_blk_free(pc->lv[l].A);
        orc_blk_free(pc->lv[l].P);
        orc_blk_free(pc->lv[l].R);
        free(pc->lv[l].diag_inv);
        free(pc->lv[l].agg);
    }
    free(pc->lv);
    orc_blk_free(pc->owned_blk);
    free(pc->coarse_lu);
    free(pc->coarse_piv);
    free(pc);
}

orc_pc* orc_pc_create(const orc_csr* A, const char* kind, double omega, int* st, char* err, int errlen)
{
    *st = ORC_OK;
    if (!strcmp(kind, "none")) return pc_new(PC_NONE, A->n);
    if (!strcmp(kind, "diag")) return pc_diag(A, st, err, errlen);
    if (!strcmp(kind, "ic0")) return pc_ic0(A, st, err, errlen);
    if (!strcmp(kind, "ilu0")) return pc_ilu0(A, st, err, errlen);
    if (!strcmp(kind, "ssor")) return pc_ssor(A, omega, st, err, errlen);
    if (!strcmp(kind, "sa_amg") || !strcmp(kind, "sa_amg_exact") || !strcmp(kind, "sa_amg_std") ||
        !strcmp(kind, "sa_amg_mis"))
    {
        if (A->n != A->m)
        {
            *st = ORC_INVALID_ARG;
            set_err(err, errlen, "AMG needs a square matrix");
            return NULL;
        }
        orc_blk* B = orc_blk_condense(1, A, A->n, A->m);
        const int mode = !strcmp(kind, "sa_amg_std") ? 1 : !strcmp(kind, "sa_amg_mis") ? 2 : 0;
        orc_pc* pc = pc_amg(B, strcmp(kind, "sa_amg") != 0, mode, st, err, errlen);
        if (pc)
            pc->owned_blk = B;
        else
            orc_blk_free(B);
        return pc;
    }
    *st = ORC_INVALID_ARG;
    set_err(err, errlen, "unknown preconditioner kind");
    return NULL;
}

orc_pc* orc_blk_pc_create(const orc_blk* A, const char* kind, int* st, char* err, int errlen)
{
    *st = ORC_OK;
    if (!strcmp(kind, "jacobi"))
    {
        orc_pc* pc = pc_new(PC_BJACOBI, A->nbr * (uint32_t)A->bs);
        pc->bs = A->bs;
        pc->Ablk = A;
        return pc;
    }
    if (!strcmp(kind, "ilu0")) return pc_bilu0(A, st, err, errlen);
    if (!strcmp(kind, "amg")) return pc_amg(A, 0, 0, st, err, errlen);
    if (!strcmp(kind, "amg_exact")) return pc_amg(A, 1, 0, st, err, errlen);
    if (!strcmp(kind, "amg_std")) return pc_amg(A, 1, 1, st, err, errlen);
    if (!strcmp(kind, "amg_mis")) return pc_amg(A, 1, 2, st, err, errlen);
    *st = ORC_INVALID_ARG;
    set_err(err, errlen, "unknown block preconditioner kind");
    return NULL;
}

int orc_ic0_export(orc_pc* pc, uint32_t* sizes, uint32_t* Lrp, uint32_t* Lci, double* Lv, uint32_t* LTrp,
                   uint32_t* LTci, double* LTv, double* diag)
{
    if (pc->kind != PC_IC0) return -1;
    const uint32_t n = pc->n;
    sizes[0] = pc->Lrp[n];
    sizes[1] = pc->Urp[n];
    if (!Lrp) return 0;
    memcpy(Lrp, pc->Lrp, 4 * ((size_t)n + 1));
    memcpy(Lci, pc->Lci, 4 * (size_t)sizes[0]);
    memcpy(Lv, pc->Lv, 8 * (size_t)sizes[0]);
    memcpy(LTrp, pc->Urp, 4 * ((size_t)n + 1));
    memcpy(LTci, pc->Uci, 4 * (size_t)sizes[1]);
    memcpy(LTv, pc->Uv, 8 * (size_t)sizes[1]);
    memcpy(diag, pc->diag, 8 * (size_t)n);
    return 0;
}

int orc_ilu0_export(orc_pc* pc, uint32_t* sizes, uint32_t* Lrp, uint32_t* Lci, double* Lv, uint32_t* Urp,
                    uint32_t* Uci, double* Uv, uint32_t* diag_idx)
{
    if (pc->kind != PC_ILU0) return -1;
    const uint32_t n = pc->n;
    sizes[0] = pc->Lrp[n];
    sizes[1] = pc->Urp[n];
    if (!Lrp) return 0;
    memcpy(Lrp, pc->Lrp, 4 * ((size_t)n + 1));
    memcpy(Lci, pc->Lci, 4 * (size_t)sizes[0]);
    memcpy(Lv, pc->Lv, 8 * (size_t)sizes[0]);
    memcpy(Urp, pc->Urp, 4 * ((size_t)n + 1));
    memcpy(Uci, pc->Uci, 4 * (size_t)sizes[1]);
    memcpy(Uv, pc->Uv, 8 * (size_t)sizes[1]);
    memcpy(diag_idx, pc->diag_idx, 4 * (size_t)n);
    return 0;
}

int orc_colour_export(orc_pc* pc, uint32_t* ncolor, uint32_t* color_ptr, uint32_t* new_id, uint32_t* perm,
                      double* diag2)
{
    if (pc->kind != PC_SSOR) return -1;
    *ncolor = pc->ncolor;
    memcpy(color_ptr, pc->color_ptr, 4 * ((size_t)pc->ncolor + 1));
    memcpy(new_id, pc->new_id, 4 * (size_t)pc->n);
    memcpy(perm, pc->perm, 4 * (size_t)pc->n);
    memcpy(diag2, pc->diag2, 8 * (size_t)pc->n);
    return 0;
}

int orc_blk_ilu0_export(orc_pc* pc, uint32_t* sizes, uint32_t* Lrp, uint32_t* Lci, double* Lv, uint32_t* Urp,
                        uint32_t* Uci, double* Uv, uint32_t* Udiag, double* inv_diag)
{
    if (pc->kind != PC_BILU0) return -1;
    const int bv = pc->bs * pc->bs;
    const uint32_t nb = pc->n / (uint32_t)pc->bs;
    sizes[0] = pc->Lrp[nb];
    sizes[1] = pc->Urp[nb];
    if (!Lrp) return 0;
    memcpy(Lrp, pc->Lrp, 4 * ((size_t)nb + 1));
    memcpy(Lci, pc->Lci, 4 * (size_t)sizes[0]);
    memcpy(Lv, pc->Lv, 8 * (size_t)sizes[0] * bv);
    memcpy(Urp, pc->Urp, 4 * ((size_t)nb + 1));
    memcpy(Uci, pc->Uci, 4 * (size_t)sizes[1]);
    memcpy(Uv, pc->Uv, 8 * (size_t)sizes[1] * bv);
    memcpy(Udiag, pc->Udiag, 4 * (size_t)nb);
    memcpy(inv_diag, pc->inv_diag, 8 * (size_t)nb * bv);
    return 0;
}

int orc_blk_amg_export(orc_pc* pc, int level, uint32_t* sizes, uint32_t* Arp, uint32_t* Aci, double* Av,
                       uint32_t* Prp, uint32_t* Pci, double* Pv, double* diag_inv)
{
    if (pc->kind != PC_AMG) return -1;
    if (level < 0) return pc->nlev;
    if (level >= pc->nlev) return -1;
    const amg_level* L = &pc->lv[level];
    const int bv = pc->bs * pc->bs;
    sizes[0] = L->nrows;
    sizes[1] = L->A->rp[L->nrows];
    sizes[2] = L->P ? L->P->nbc : 0;
    sizes[3] = L->P ? L->P->rp[L->P->nbr] : 0;
    if (!Arp) return 0;
    orc_blk_export(L->A, Arp, Aci, Av);
    if (L->P) orc_blk_export(L->P, Prp, Pci, Pv);
    memcpy(diag_inv, L->diag_inv, 8 * (size_t)L->nrows * bv);
    return 0;
}

int orc_blk_amg_aggregates(orc_pc* pc, int level, int32_t* agg)
{
    if (pc->kind != PC_AMG || level < 0 || level >= pc->nlev || !pc->lv[level].agg) return -1;
    memcpy(agg, pc->lv[level].agg, 4 * (size_t)pc->lv[level].nrows);
    return 0;
}

uint32_t orc_levels(uint32_t n, const uint32_t* rp, const uint32_t* ci, int upper, uint32_t* level)
{
    uint32_t nlev = 0;
    if (!upper)
    {
        for (uint32_t i = 0; i < n; ++i)
        {
            uint32_t l = 0;
            for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
                if (ci[p] < i && level[ci[p]] + 1 > l) l = level[ci[p]] + 1;
            level[i] = l;
            if (l + 1 > nlev) nlev = l + 1;
        }
    }
    else
    {
        for (uint32_t i = n; i-- > 0;)
        {
            uint32_t l = 0;
            for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
                if (ci[p] > i && level[ci[p]] + 1 > l) l = level[ci[p]] + 1;
            level[i] = l;
            if (l + 1 > nlev) nlev = l + 1;
        }
    }
    return nlev;
}

/* ======================================================================
 * Krylov solvers (operator + preconditioner callbacks)
 * ====================================================================== */

typedef void (*matvec_fn)(const void* A, const double* x, double* y);

static void mv_csr(const void* A, const double* x, double* y) { orc_spmv((const orc_csr*)A, x, y); }
static void mv_blk(const void* A, const double* x, double* y) { orc_blk_matvec((const orc_blk*)A, x, y); }

static void pc_apply_or_copy(orc_pc* pc, uint32_t n, const double* r, double* z)
{
    if (pc)
        orc_pc_apply(pc, r, z);
    else
        memcpy(z, r, 8 * (size_t)n);
}

/* SMatrix::pcg main loop, array.cpp:3518-3600 (after the shape checks,
 * normb / initial-residual early returns and the factory). Returned it is the
 * index of the last fully completed iteration. */
static int krylov_pcg(const void* A, matvec_fn mv, uint32_t n, orc_pc* pc, const double* b, double tol, int maxit,
                      double* x, int* itout, char* err, int errlen)
{
    double* r = (double*)xcalloc(n, 8);
    double* z = (double*)xcalloc(n, 8);
    double* p = (double*)xcalloc(n, 8);
    double* Ap = (double*)xcalloc(n, 8);
    int st = ORC_OK;
    const double normb = sqrt(orc_dot(n, b, b));
    memset(x, 0, 8 * (size_t)n);
    *itout = 0;
    if (normb < 1e-300) goto done;
    memcpy(r, b, 8 * (size_t)n);
    if (sqrt(orc_dot(n, r, r)) / normb < tol) goto done;
    pc_apply_or_copy(pc, n, r, z);
    memcpy(p, z, 8 * (size_t)n);
    double rz_old = orc_dot(n, r, z);
    if (rz_old <= 0.0)
    {
        st = ORC_BREAKDOWN;
        set_err(err, errlen, "PCG failed: r^T M^-1 r <= 0, preconditioner may not be SPD");
        goto done;
    }
    int it_end = 0;
    for (int it = 0; it < maxit; ++it)
    {
        mv(A, p, Ap);
        const double pAp = orc_dot(n, p, Ap);
        if (fabs(pAp) < 1e-30)
        {
            st = ORC_BREAKDOWN;
            set_err(err, errlen, "PCG breakdown: p^T A p too small");
            goto done;
        }
        if (pAp <= 0.0)
        {
            st = ORC_BREAKDOWN;
            set_err(err, errlen, "PCG failed: p^T A p <= 0, A may not be SPD");
            goto done;
        }
        const double alpha = rz_old / pAp;
        for (uint32_t i = 0; i < n; ++i)
        {
            x[i] += alpha * p[i];
            r[i] -= alpha * Ap[i];
        }
        if (sqrt(orc_dot(n, r, r)) / normb < tol) break;
        pc_apply_or_copy(pc, n, r, z);
        const double rz_new = orc_dot(n, r, z);
        if (rz_new <= 0.0)
        {
            st = ORC_BREAKDOWN;
            set_err(err, errlen, "PCG failed: r^T M^-1 r <= 0, preconditioner may not be SPD");
            goto done;
        }
        const double beta = rz_new / rz_old;
        for (uint32_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        rz_old = rz_new;
        it_end = it;
    }
    *itout = it_end;
done:
    free(r);
    free(z);
    free(p);
    free(Ap);
    return st;
}

/* SMatrix::bicgstab main loop, array.cpp:3675-3841 (right preconditioning,
 * shadow residual r0, true-residual check with residual replacement). */
static int krylov_bicgstab(const void* A, matvec_fn mv, uint32_t n, orc_pc* pc, const double* b, double tol,
                           int maxit, double* x, int* itout, char* err, int errlen)
{
    double* r = (double*)xcalloc(n, 8);
    double* rt = (double*)xcalloc(n, 8);
    double* p = (double*)xcalloc(n, 8);
    double* v = (double*)xcalloc(n, 8);
    double* y = (double*)xcalloc(n, 8);
    double* z = (double*)xcalloc(n, 8);
    double* s = (double*)xcalloc(n, 8);
    double* t = (double*)xcalloc(n, 8);
    double* Ax = (double*)xcalloc(n, 8);
    int st = ORC_OK;
    const double normb = sqrt(orc_dot(n, b, b));
    memset(x, 0, 8 * (size_t)n);
    *itout = 0;
    if (normb < 1e-300) goto done;
    memcpy(r, b, 8 * (size_t)n);
    if (sqrt(orc_dot(n, r, r)) / normb < tol) goto done;
    memcpy(rt, r, 8 * (size_t)n);
    double rho_old = 1.0, alpha = 1.0, omega = 1.0;
    const double bt = 1e-30;
    int it_end = 0;
    for (int it = 0; it < maxit; ++it)
    {
        const double rho_new = orc_dot(n, rt, r);
        if (fabs(rho_new) < bt || fabs(rho_old) < bt || fabs(omega) < bt)
        {
            st = ORC_BREAKDOWN;
            set_err(err, errlen,
                    fabs(rho_new) < bt   ? "BiCGSTAB breakdown: rho_{k+1} too small"
                    : fabs(rho_old) < bt ? "BiCGSTAB breakdown: rho_k too small"
                                         : "BiCGSTAB breakdown: omega_k = 0");
            goto done;
        }
        const double beta = (rho_new / rho_old) * (alpha / omega);
        for (uint32_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        pc_apply_or_copy(pc, n, p, y);
        mv(A, y, v);
        const double rhat_v = orc_dot(n, rt, v);
        if (fabs(rhat_v) < bt)
        {
            st = ORC_BREAKDOWN;
            set_err(err, errlen, "BiCGSTAB breakdown: r0^T v too small");
            goto done;
        }
        alpha = rho_new / rhat_v;
        for (uint32_t i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
        pc_apply_or_copy(pc, n, s, z);
        mv(A, z, t);
        const double tt = orc_dot(n, t, t);
        if (tt < bt)
        {
            st = ORC_BREAKDOWN;
            set_err(err, errlen, "BiCGSTAB breakdown: t^T t too small");
            goto done;
        }
        omega = orc_dot(n, t, s) / tt;
        for (uint32_t i = 0; i < n; ++i)
        {
            x[i] += alpha * y[i] + omega * z[i];
            r[i] = s[i] - omega * t[i];
        }
        const double normr = sqrt(orc_dot(n, r, r));
        it_end = it;
        int converged = 0;
        if (normr / normb < tol)
        {
            mv(A, x, Ax);
            double tr = 0.0;
            for (uint32_t i = 0; i < n; ++i)
            {
                const double d = b[i] - Ax[i];
                tr += d * d;
            }
            if (sqrt(tr) / normb < tol)
                converged = 1;
            else
            {
                for (uint32_t i = 0; i < n; ++i) r[i] = b[i] - Ax[i];
                const double rc = orc_dot(n, rt, r);
                if (fabs(rc) < bt)
                    converged = 1;
                else
                {
                    rho_old = rc;
                    continue;
                }
            }
        }
        else
            rho_old = rho_new;
        if (converged) break;
    }
    *itout = it_end;
done:
    free(r);
    free(rt);
    free(p);
    free(v);
    free(y);
    free(z);
    free(s);
    free(t);
    free(Ax);
    return st;
}

/* SMatrix::gmres, array.cpp:4244-4400 (and the std::function overload
 * 4402-4533, BlockMatrix::gmres blockMatrix.hpp:747-866): restarted,
 * right-preconditioned, MGS Arnoldi, Givens, back substitution,
 * x += M^-1 (V y). */
static int krylov_gmres(const void* A, matvec_fn mv, uint32_t n, orc_pc* pc, const double* b, int m, double tol,
                        int maxit, double* x, int* itout, char* err, int errlen)
{
    int st = ORC_OK;
    memset(x, 0, 8 * (size_t)n);
    *itout = 0;
    const double normb = sqrt(orc_dot(n, b, b));
    if (normb < 1e-300) return ORC_OK;
    double* V = (double*)xcalloc((size_t)(m + 1) * n, 8);
    double* H = (double*)xcalloc((size_t)(m + 1) * m, 8);
    double* cs = (double*)xcalloc((size_t)m, 8);
    double* sn = (double*)xcalloc((size_t)m, 8);
    double* g = (double*)xcalloc((size_t)m + 1, 8);
    double* y = (double*)xcalloc((size_t)m, 8);
    double* w = (double*)xcalloc(n, 8);
    double* wt = (double*)xcalloc(n, 8);
    double* z = (double*)xcalloc(n, 8);
    double* dz = (double*)xcalloc(n, 8);
    const double bt = 1e-30;
#define HV(i, j) H[(size_t)(i) * m + (j)]
    int total = 0, it_end = 0, converged = 0;
    while (total < maxit && !converged)
    {
        double beta;
        if (total == 0)
        {
            beta = normb;
            for (uint32_t i = 0; i < n; ++i) V[i] = b[i] / beta;
        }
        else
        {
            mv(A, x, w);
            double rr = 0.0;
            for (uint32_t i = 0; i < n; ++i)
            {
                const double ri = b[i] - w[i];
                V[i] = ri;
                rr += ri * ri;
            }
            beta = sqrt(rr);
            if (beta / normb < tol)
            {
                converged = 1;
                break;
            }
            for (uint32_t i = 0; i < n; ++i) V[i] /= beta;
        }
        memset(g, 0, 8 * ((size_t)m + 1));
        g[0] = beta;
        memset(H, 0, 8 * (size_t)(m + 1) * m);
        int j_used = 0;
        for (int j = 0; j < m && total < maxit; ++j)
        {
            pc_apply_or_copy(pc, n, &V[(size_t)j * n], wt);
            mv(A, wt, w);
            for (int i = 0; i <= j; ++i)
            {
                HV(i, j) = orc_dot(n, w, &V[(size_t)i * n]);
                const double hij = HV(i, j);
                const double* Vi = &V[(size_t)i * n];
                for (uint32_t t = 0; t < n; ++t) w[t] -= hij * Vi[t];
            }
            HV(j + 1, j) = sqrt(orc_dot(n, w, w));
            if (HV(j + 1, j) > bt)
            {
                const double inv = 1.0 / HV(j + 1, j);
                double* Vn = &V[(size_t)(j + 1) * n];
                for (uint32_t t = 0; t < n; ++t) Vn[t] = w[t] * inv;
            }
            for (int i = 0; i < j; ++i)
            {
                const double t1 = cs[i] * HV(i, j) + sn[i] * HV(i + 1, j);
                const double t2 = -sn[i] * HV(i, j) + cs[i] * HV(i + 1, j);
                HV(i, j) = t1;
                HV(i + 1, j) = t2;
            }
            const double den = hypot(HV(j, j), HV(j + 1, j));
            if (den < bt)
            {
                st = ORC_BREAKDOWN;
                set_err(err, errlen, "GMRES breakdown: Hessenberg pivot too small");
                goto done;
            }
            cs[j] = HV(j, j) / den;
            sn[j] = HV(j + 1, j) / den;
            HV(j, j) = cs[j] * HV(j, j) + sn[j] * HV(j + 1, j);
            HV(j + 1, j) = 0.0;
            const double g1 = cs[j] * g[j] + sn[j] * g[j + 1];
            const double g2 = -sn[j] * g[j] + cs[j] * g[j + 1];
            g[j] = g1;
            g[j + 1] = g2;
            j_used = j + 1;
            it_end = total;
            ++total;
            if (fabs(g[j + 1]) / normb < tol)
            {
                converged = 1;
                break;
            }
        }
        for (int i = j_used - 1; i >= 0; --i)
        {
            double sum = g[i];
            for (int k = i + 1; k < j_used; ++k) sum -= HV(i, k) * y[k];
            if (fabs(HV(i, i)) < bt)
            {
                st = ORC_BREAKDOWN;
                set_err(err, errlen, "GMRES breakdown: upper triangular pivot too small");
                goto done;
            }
            y[i] = sum / HV(i, i);
        }
        for (uint32_t t = 0; t < n; ++t)
        {
            double acc = 0.0;
            for (int i = 0; i < j_used; ++i) acc += y[i] * V[(size_t)i * n + t];
            z[t] = acc;
        }
        pc_apply_or_copy(pc, n, z, dz);
        for (uint32_t t = 0; t < n; ++t) x[t] += dz[t];
    }
#undef HV
    *itout = it_end;
done:
    free(V);
    free(H);
    free(cs);
    free(sn);
    free(g);
    free(y);
    free(w);
    free(wt);
    free(z);
    free(dz);
    return st;
}

static void lower(const char* s, char* out, size_t cap)
{
    size_t i = 0;
    for (; s[i] && i + 1 < cap; ++i) out[i] = (char)tolower((unsigned char)s[i]);
    out[i] = 0;
}

/* Preconditioner alias tables: pcg array.cpp:3482-3515, bicgstab 3637-3673,
 * gmres 4212-4242.  Returns the canonical kind or NULL when unknown. */
static const char* resolve_precond(int method, const char* name)
{
    char s[64];
    lower(name, s, sizeof s);
    if (!strcmp(s, "none") || !strcmp(s, "identity") || !strcmp(s, "noprecond")) return "none";
    if (method == 0 && !strcmp(s, "cg")) return "none";
    if (!strcmp(s, "diag") || !strcmp(s, "diagonal") || !strcmp(s, "jacobi")) return "diag";
    if (!strcmp(s, "ic") || !strcmp(s, "ic0") || !strcmp(s, "ichol")) return "ic0";
    if (method != 2 && !strcmp(s, "incomplete_cholesky")) return "ic0";
    if (!strcmp(s, "ilu") || !strcmp(s, "ilu0")) return "ilu0";
    if (!strcmp(s, "sor") || !strcmp(s, "ssor")) return "ssor";
    if (!strcmp(s, "amg")) return "sa_amg_mis";
    return NULL;
}

/* SMatrix::amg main loop, array.cpp:4534-4563, with the preconditioner given
 * (one V-cycle from zero per correction when it is an AMG): from x = 0, at
 * index k: r = b - A x, rr summed in row order; stop with it = k when
 * sqrt(rr) / ||b|| < tol, else x += M^-1 r.  Running out leaves it = maxit - 1. */
static int stationary(const void* A, matvec_fn mv, uint32_t n, orc_pc* pc, const double* b, double tol, int maxit,
                      double* x, int* itout)
{
    memset(x, 0, 8 * (size_t)n);
    *itout = 0;
    const double normb = sqrt(orc_dot(n, b, b));
    if (normb < 1e-300) return ORC_OK;
    double* r = (double*)xcalloc(n, 8);
    double* d = (double*)xcalloc(n, 8);
    double* Ax = (double*)xcalloc(n, 8);
    int it_end = 0;
    for (int k = 0; k < maxit; ++k)
    {
        mv(A, x, Ax);
        double rr = 0.0;
        for (uint32_t i = 0; i < n; ++i)
        {
            r[i] = b[i] - Ax[i];
            rr += r[i] * r[i];
        }
        it_end = k;
        if (sqrt(rr) / normb < tol) break;
        pc_apply_or_copy(pc, n, r, d);
        for (uint32_t i = 0; i < n; ++i) x[i] += d[i];
    }
    *itout = it_end;
    free(r);
    free(d);
    free(Ax);
    return ORC_OK;
}

static int run_method(const void* A, matvec_fn mv, uint32_t n, int method, orc_pc* pc, int restart, double tol,
                      int maxit, const double* b, double* x, int* it, char* err, int errlen)
{
    if (method == 5) return stationary(A, mv, n, pc, b, tol, maxit, x, it);
    if (method == 0) return krylov_pcg(A, mv, n, pc, b, tol, maxit, x, it, err, errlen);
    if (method == 1) return krylov_bicgstab(A, mv, n, pc, b, tol, maxit, x, it, err, errlen);
    return krylov_gmres(A, mv, n, pc, b, restart, tol, maxit, x, it, err, errlen);
}

int orc_solve(const orc_csr* A, int method, const char* precond, int restart, double tol, int maxit,
              const double* b, double* x, int* it, char* err, int errlen)
{
    *it = 0;
    if (A->n != A->m)
    {
        set_err(err, errlen, "solver needs a square matrix");
        return ORC_INVALID_ARG;
    }
    const uint32_t n = A->n;
    memset(x, 0, 8 * (size_t)n);
    const double normb = sqrt(orc_dot(n, b, b));
    if (normb < 1e-300) return ORC_OK;
    /* pcg and bicgstab return before the factory when r0 = b already passes */
    if (method != 2 && sqrt(orc_dot(n, b, b)) / normb < tol) return ORC_OK;
    const char* kind = resolve_precond(method, precond);
    if (!kind)
    {
        set_err(err, errlen, "unknown preconditioner type");
        return ORC_INVALID_ARG;
    }
    int st = ORC_OK;
    orc_pc* pc = orc_pc_create(A, kind, 1.2, &st, err, errlen);
    if (!pc) return st;
    st = run_method(A, mv_csr, n, method, pc, restart, tol, maxit, b, x, it, err, errlen);
    orc_pc_free(pc);
    return st;
}

int orc_solve_pc(const orc_csr* A, int method, orc_pc* pc, int restart, double tol, int maxit, const double* b,
                 double* x, int* it, char* err, int errlen)
{
    *it = 0;
    if (A->n != A->m)
    {
        set_err(err, errlen, "solver needs a square matrix");
        return ORC_INVALID_ARG;
    }
    return run_method(A, mv_csr, A->n, method, pc, restart, tol, maxit, b, x, it, err, errlen);
}

int orc_blk_gmres(const orc_blk* A, const double* b, const char* precond, double tol, int maxit, int restart,
                  double* x, int* it, char* err, int errlen)
{
    const uint32_t n = A->nbr * (uint32_t)A->bs;
    *it = 0;
    memset(x, 0, 8 * (size_t)n);
    if (sqrt(orc_dot(n, b, b)) < 1e-300) return ORC_OK;
    int st = ORC_OK;
    orc_pc* pc = NULL;
    if (!strcmp(precond, "none") || !strcmp(precond, "identity"))
        pc = NULL;
    else if (!strcmp(precond, "blockjacobi"))
        pc = orc_blk_pc_create(A, "jacobi", &st, err, errlen);
    else if (!strcmp(precond, "blockilu") || !strcmp(precond, "blockilu0"))
    {
        pc = orc_blk_pc_create(A, "ilu0", &st, err, errlen);
        if (!pc) return st;
    }
    else
    {
        set_err(err, errlen, "BlockMatrix::gmres: unknown preconditioner type");
        return ORC_INVALID_ARG;
    }
    st = krylov_gmres(A, mv_blk, n, pc, b, restart, tol, maxit, x, it, err, errlen);
    orc_pc_free(pc);
    return st;
}

int orc_blk_solve_pc(const orc_blk* A, int method, orc_pc* pc, int restart, double tol, int maxit,
                     const double* b, double* x, int* it, char* err, int errlen)
{
    *it = 0;
    const uint32_t n = A->nbr * (uint32_t)A->bs;
    return run_method(A, mv_blk, n, method, pc, restart, tol, maxit, b, x, it, err, errlen);
}
