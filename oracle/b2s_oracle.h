/* b2s_oracle.h -- CPU restatement of the sparse iterative-solver path of
 * xuyinshen/cpp-FEM-solver (ode-solver/src/math/array.cpp and
 * ode-solver/include/math/blockMatrix.hpp).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load this library, and only as the checker
 * or the timed CPU baseline; the product never links or calls it.
 *
 * Each function restates one reference function in plain C, keeping its
 * operation order (serial loops, ascending index, no contraction) so that at
 * one thread it agrees bit for bit with the reference compiled from source
 * (oracle/_ref/libref.so); tests/test_oracle_pin.py pins that.  Parity is
 * pinned against the compiled reference, not against stored golden vectors:
 * the reference ships none.
 *
 * Status codes: 0 ok, 1 invalid argument (std::invalid_argument /
 * std::out_of_range in the reference), 2 numerical breakdown
 * (std::runtime_error in the reference). */
#pragma once
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_OK = 0, ORC_INVALID_ARG = 1, ORC_BREAKDOWN = 2 };

typedef struct orc_csr
{
    uint32_t n, m;
    uint32_t* rp;  /* n+1 */
    uint32_t* ci;  /* nnz */
    double* v;     /* nnz */
} orc_csr;

typedef struct orc_blk
{
    int bs;
    uint32_t nbr, nbc;
    uint32_t* rp;        /* nbr+1 */
    uint32_t* ci;        /* nnzb */
    double* v;           /* nnzb*bs*bs, row-major per block */
    uint32_t* diag_ptr;  /* nbr, UINT32_MAX when missing */
} orc_blk;

typedef struct orc_pc orc_pc;

/* ---- CSR container (array.cpp:2072-2235, 2336-2447) ---- */
orc_csr* orc_csr_from_coo(uint32_t n, uint32_t m, uint64_t nnz, const double* v, const uint32_t* r,
                          const uint32_t* c, int* st);
orc_csr* orc_csr_copy(uint32_t n, uint32_t m, const uint32_t* rp, const uint32_t* ci, const double* v);
void orc_csr_free(orc_csr* A);
uint32_t orc_csr_nnz(const orc_csr* A);
void orc_csr_export(const orc_csr* A, uint32_t* rp, uint32_t* ci, double* v);
orc_csr* orc_csr_transpose(const orc_csr* A);
orc_csr* orc_csr_matmul(const orc_csr* A, const orc_csr* B);

/* ---- kernels (array.cpp:3401-3442) ---- */
void orc_spmv(const orc_csr* A, const double* x, double* y);
double orc_dot(uint64_t n, const double* a, const double* b);

/* ---- preconditioners (array.cpp:2450-3164; blockMatrix.hpp:455-623, 1051-1179) ----
 * scalar kinds: "none", "diag", "ic0", "ilu0", "ssor", "sa_amg" (block SA-AMG
 * with BS=1 via condense, reference coarsest solve), "sa_amg_exact" (same
 * hierarchy, coarsest level solved by a correct pivoted LU), "sa_amg_std"
 * (sequential three-phase aggregation + correct LU), "sa_amg_mis" (the
 * library's parallel aggregation rule + correct LU; the library's "amg"). */
orc_pc* orc_pc_create(const orc_csr* A, const char* kind, double omega, int* st, char* err, int errlen);
void orc_pc_apply(orc_pc* pc, const double* r, double* z);
void orc_pc_free(orc_pc* pc);
uint32_t orc_pc_n(const orc_pc* pc);

int orc_ic0_export(orc_pc* pc, uint32_t* sizes, uint32_t* Lrp, uint32_t* Lci, double* Lv, uint32_t* LTrp,
                   uint32_t* LTci, double* LTv, double* diag);
int orc_ilu0_export(orc_pc* pc, uint32_t* sizes, uint32_t* Lrp, uint32_t* Lci, double* Lv, uint32_t* Urp,
                    uint32_t* Uci, double* Uv, uint32_t* diag_idx);
int orc_colour_export(orc_pc* pc, uint32_t* ncolor, uint32_t* color_ptr, uint32_t* new_id, uint32_t* perm,
                      double* diag2);

/* Topological levels of a triangular DAG: for upper==0 row i depends on the
 * columns j<i of its row, for upper!=0 on the columns j>i.  level[i] is the
 * longest dependency chain ending at i (0 for independent rows). Returns the
 * level count. */
uint32_t orc_levels(uint32_t n, const uint32_t* rp, const uint32_t* ci, int upper, uint32_t* level);

/* ---- solvers (array.cpp:3445-3842, 4190-4533) ----
 * method: 0 pcg, 1 bicgstab, 2 gmres, 5 the stationary loop of SMatrix::amg
 * (array.cpp:4534-4563: x += M^-1 (b - A x) from x = 0 with the true residual
 * checked before every correction).  The preconditioner string follows each
 * solver's own alias table; "amg" maps to "sa_amg_mis". */
int orc_solve(const orc_csr* A, int method, const char* precond, int restart, double tol, int maxit,
              const double* b, double* x, int* it, char* err, int errlen);
/* Same solvers with an explicit preconditioner object (the std::function
 * overload of gmres, array.cpp:4402-4533; pcg/bicgstab with a functor are
 * extensions with the same algorithm). pc may be NULL for identity. */
int orc_solve_pc(const orc_csr* A, int method, orc_pc* pc, int restart, double tol, int maxit,
                 const double* b, double* x, int* it, char* err, int errlen);

/* ---- distributed BlockMatrix (blockMatrix.hpp:317-437) ----
 * distributed_matvec after the halo exchange on one rank's rows: local
 * columns (owned < n_owned, ghosts after), owned pass then ghost pass. */
void orc_blk_dist_matvec(int bs, uint32_t nbr, const uint32_t* rp, const uint32_t* lci, const double* v,
                         uint32_t n_owned, const double* x_full, double* y);

/* ---- BlockMatrix (blockMatrix.hpp:139-315) ---- */
orc_blk* orc_blk_create(int bs, uint32_t nbr, uint32_t nbc, const uint32_t* rp, const uint32_t* ci,
                        const double* v);
orc_blk* orc_blk_condense(int bs, const orc_csr* A, uint32_t nbr, uint32_t nbc);
orc_blk* orc_blk_transpose(const orc_blk* A);
orc_blk* orc_blk_matmul(const orc_blk* A, const orc_blk* B);
void orc_blk_free(orc_blk* A);
uint32_t orc_blk_nnzb(const orc_blk* A);
uint32_t orc_blk_rows(const orc_blk* A);
void orc_blk_export(const orc_blk* A, uint32_t* rp, uint32_t* ci, double* v);
void orc_blk_matvec(const orc_blk* A, const double* x, double* y);

/* block kinds: "jacobi", "ilu0", "amg" (reference aggregation and coarsest
 * solve), "amg_exact" (reference aggregation, correct coarsest LU), "amg_std"
 * (sequential three-phase aggregation, correct coarsest LU), "amg_mis" (the
 * library's default parallel aggregation, correct coarsest LU; no reference
 * counterpart) */
orc_pc* orc_blk_pc_create(const orc_blk* A, const char* kind, int* st, char* err, int errlen);
int orc_blk_ilu0_export(orc_pc* pc, uint32_t* sizes, uint32_t* Lrp, uint32_t* Lci, double* Lv, uint32_t* Urp,
                        uint32_t* Uci, double* Uv, uint32_t* Udiag, double* inv_diag);
int orc_blk_amg_export(orc_pc* pc, int level, uint32_t* sizes, uint32_t* Arp, uint32_t* Aci, double* Av,
                       uint32_t* Prp, uint32_t* Pci, double* Pv, double* diag_inv);
/* aggregate id of each block row of level `level` (not the coarsest) */
int orc_blk_amg_aggregates(orc_pc* pc, int level, int32_t* agg);

/* BlockMatrix::gmres (blockMatrix.hpp:688-866), argument order as the reference */
int orc_blk_gmres(const orc_blk* A, const double* b, const char* precond, double tol, int maxit, int restart,
                  double* x, int* it, char* err, int errlen);
/* Krylov solve of a block operator with a preconditioner object; method as orc_solve_pc */
int orc_blk_solve_pc(const orc_blk* A, int method, orc_pc* pc, int restart, double tol, int maxit,
                     const double* b, double* x, int* it, char* err, int errlen);

#ifdef __cplusplus
}
#endif
