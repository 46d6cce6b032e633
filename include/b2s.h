/* b2s.h -- C ABI of the B200-native sparse iterative-solver library.
 *
 * This is the drop-in boundary for the sparse solver path of
 * xuyinshen/cpp-FEM-solver: every solver and preconditioner that the
 * reference exposes as a static member of sparse::SMatrix
 * (ode-solver/include/math/array.hpp:266-373) or as a member / free function
 * of block::BlockMatrix (ode-solver/include/math/blockMatrix.hpp:139-452)
 * maps onto one entry point here.  The C++ drop-in headers
 * include/b2s/math/array.hpp and include/b2s/math/blockMatrix.hpp re-expose
 * the reference's own call surface on top of it.
 *
 * Conventions
 *   - Plain pointers and sizes only.  Index arrays are uint32 (as in the
 *     reference), values FP64.  Functions without a _device suffix take HOST
 *     pointers and copy in/out; _device variants take device pointers already
 *     resident on the context's GPU and enqueue on the context's stream.
 *   - Every function returns b2s_status.  b2s_last_error(ctx) gives the
 *     message of the last failure on that context.
 *   - Handles belong to one context (one device, one CUDA stream).  Calls on
 *     one context must be serialised by the caller; distinct contexts are
 *     independent.
 *   - Nothing here falls back to the CPU: without a usable GPU the context
 *     cannot be created (B2S_NO_DEVICE) and no solver runs.
 */
#ifndef B2S_H
#define B2S_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B2S_VERSION_MAJOR 0
#define B2S_VERSION_MINOR 1

typedef enum b2s_status
{
    B2S_OK = 0,
    B2S_INVALID_ARG = 1,     /* std::invalid_argument in the reference */
    B2S_SHAPE = 2,           /* std::invalid_argument (dimension mismatch) */
    B2S_NOT_SPD = 3,         /* std::runtime_error: pAp <= 0, rz <= 0, IC(0) pivot <= 1e-14, diag <= 0 */
    B2S_BREAKDOWN = 4,       /* std::runtime_error: Krylov breakdown below 1e-30 */
    B2S_ZERO_PIVOT = 5,      /* std::runtime_error: ILU(0) |U_kk| < 1e-30, diag |d| < 1e-14 */
    B2S_MISSING_DIAG = 6,    /* std::runtime_error: a row without diagonal entry */
    B2S_SINGULAR_BLOCK = 7,  /* std::runtime_error: a singular diagonal block */
    B2S_DIVERGED = 8,        /* NaN / Inf in a residual */
    B2S_TIMEOUT = 9,         /* a bounded device-side wait gave up */
    B2S_CUDA_ERROR = 10,
    B2S_NO_DEVICE = 11,
    B2S_OUT_OF_MEMORY = 12,
    B2S_UNSUPPORTED = 13
} b2s_status;

typedef struct b2s_ctx b2s_ctx;
typedef struct b2s_csr b2s_csr;
typedef struct b2s_baij b2s_baij;
typedef struct b2s_pc b2s_pc;

/* ------------------------------------------------------------------ context */

/* Creates a context on CUDA device `device` with its own non-blocking stream. */
b2s_status b2s_ctx_create(int device, b2s_ctx** out);
b2s_status b2s_ctx_destroy(b2s_ctx* ctx);
/* Message of the last failure on ctx (static storage inside ctx). */
const char* b2s_last_error(const b2s_ctx* ctx);
/* Name of a status code. */
const char* b2s_status_name(b2s_status st);
/* The context's cudaStream_t, for callers that enqueue their own work. */
void* b2s_ctx_stream(b2s_ctx* ctx);
b2s_status b2s_ctx_synchronize(b2s_ctx* ctx);
/* Number of this library's kernels launched on ctx since creation. */
uint64_t b2s_ctx_kernel_launches(const b2s_ctx* ctx);
/* Bounds of the device-side waits of the chunked triangular solves on ctx
 * (IC(0) / ILU(0) / block ILU(0) with B2S_TRSV_CHUNK, the default): a wait
 * polls spin_polls times without sleeping, then sleeps 1 us per poll, drawing
 * on a budget of sleep_polls per thread for the whole launch.  The 5- and
 * 7-point grid schedules of the same solves poll a group's hand-over words
 * up to spin_polls + sleep_polls times (at least once) without sleeping.  A
 * wait that runs out, and every later wait of the same launch, gives up at
 * once and the call reports B2S_TIMEOUT (the synchronous calls at their end, the _device
 * ones at the next b2s_ctx_synchronize or solve).  (0, 0) restores the
 * defaults (2^20 and 2^20, about one second).  No counterpart in the
 * reference (its solves are sequential). */
b2s_status b2s_ctx_set_wait_limits(b2s_ctx* ctx, uint32_t spin_polls, uint32_t sleep_polls);

/* ---------------------------------------------------------------- matrices */

/* CSR matrix from host arrays (SMatrix CSR constructor, array.cpp:2183-2189).
 * Columns must be sorted ascending within each row (the SMatrix COO
 * constructor, array.cpp:2072-2182, guarantees this).  The arrays are copied
 * to the device; the handle owns the copy. */
b2s_status b2s_csr_create(b2s_ctx* ctx, uint32_t n, uint32_t m, const uint32_t* row_ptr, const uint32_t* col_idx,
                          const double* values, b2s_csr** out);
b2s_status b2s_csr_destroy(b2s_csr* A);
b2s_status b2s_csr_info(const b2s_csr* A, uint32_t* n, uint32_t* m, uint32_t* nnz);

/* C = A B on the device (SMatrix::operator*, array.cpp:2336-2447): columns
 * ascending in every row, each entry the sum of its products in the
 * reference's order (A's row entries ascending, then B's), so the values equal
 * the reference's bit for bit; entries that sum to zero are kept, as the
 * reference keeps them.  One difference: a product column that only one row
 * of A B touches is kept here, while the reference leaves that slot as
 * (column 0, value 0) because its marker array is not reset between its
 * symbolic and numeric passes (array.cpp:2357-2443). */
b2s_status b2s_csr_matmul(b2s_ctx* ctx, const b2s_csr* A, const b2s_csr* B, b2s_csr** out);
/* T = A^T on the device (SMatrix::transpose, array.cpp:2201-2234): every row
 * of T lists its entries in ascending column order, values copied. */
b2s_status b2s_csr_transpose(b2s_ctx* ctx, const b2s_csr* A, b2s_csr** out);
/* Copies a handle's arrays to host memory: row_ptr (n+1), col_idx and values
 * (nnz each); a NULL array is skipped. */
b2s_status b2s_csr_export(b2s_ctx* ctx, const b2s_csr* A, uint32_t* row_ptr, uint32_t* col_idx, double* values);

/* Block-CSR (BAIJ) matrix, BlockMatrix<double,BS> constructor
 * (blockMatrix.hpp:175-186).  bs in {1, 2, 3, 4}.  values holds
 * nnzb*bs*bs doubles, row-major inside each block; vectors are node-major. */
b2s_status b2s_baij_create(b2s_ctx* ctx, int bs, uint32_t nbr, uint32_t nbc, const uint32_t* row_ptr,
                           const uint32_t* col_idx, const double* values, b2s_baij** out);
b2s_status b2s_baij_destroy(b2s_baij* A);
b2s_status b2s_baij_info(const b2s_baij* A, int* bs, uint32_t* nbr, uint32_t* nbc, uint32_t* nnzb);

/* --------------------------------------------------------------- operators */

/* y = A x.  SMatrix::spmv (array.cpp:3418-3442).  Each row is summed in
 * ascending column order, so the result equals the reference bit for bit. */
b2s_status b2s_spmv(b2s_ctx* ctx, const b2s_csr* A, const double* x, double* y);
b2s_status b2s_spmv_device(b2s_ctx* ctx, const b2s_csr* A, const double* d_x, double* d_y);

/* SMatrix::dot (array.cpp:3401-3416), deterministic fixed-order reduction. */
b2s_status b2s_dot(b2s_ctx* ctx, uint64_t n, const double* a, const double* b, double* out);
b2s_status b2s_dot_device(b2s_ctx* ctx, uint64_t n, const double* d_a, const double* d_b, double* out);

/* Dot product for callers that cannot allocate device memory (no reference
 * counterpart): device pointers in and out, enqueued on `stream` (NULL = the
 * default stream), no b2s context, no cudaMalloc / cudaFree -- the reduction
 * scratch is a fixed 32 KiB __device__ array per device.  n above
 * B2S_DOT_NOALLOC_MAX_N returns B2S_INVALID_ARG.  Every call shares that
 * array: calls that overlap on the GPU race, so serialise them.  The first
 * call on a device looks up the array's address (make it before any stream
 * capture). */
#define B2S_DOT_NOALLOC_MAX_N 8388608ull
b2s_status b2s_dot_noalloc(const double* d_a, const double* d_b, uint64_t n, double* d_out, void* stream);

/* BlockMatrix::matvec (blockMatrix.hpp:208-234); distributed_matvec
 * (blockMatrix.hpp:351-442) on one device-resident matrix is the same call. */
b2s_status b2s_baij_matvec(b2s_ctx* ctx, const b2s_baij* A, const double* x, double* y);
b2s_status b2s_baij_matvec_device(b2s_ctx* ctx, const b2s_baij* A, const double* d_x, double* d_y);

/* ------------------------------------------------- row-partitioned BAIJ
 * One rank's block rows of a matrix partitioned by contiguous block rows
 * (the BAIJ handle holds nbr local rows and nbc = the GLOBAL block column
 * count, columns in global numbering).  BlockMatrix::set_halo
 * (blockMatrix.hpp:317-348), same arguments: the ghost columns this rank
 * receives, grouped by source rank (recv_global, sum(recv_cnts) entries),
 * the owned rows it sends, grouped by destination (send_local, local
 * numbering), and the global number of its first row.  A block column that
 * is neither owned nor listed is rejected (B2S_INVALID_ARG). */
b2s_status b2s_baij_set_halo(b2s_ctx* ctx, b2s_baij* A, int nrecv, const int* recv_procs, const int* recv_cnts,
                             const uint32_t* recv_global, int nsend, const int* send_procs, const int* send_cnts,
                             const uint32_t* send_local, uint32_t owned_global_start);
b2s_status b2s_baij_halo_info(const b2s_baij* A, uint32_t* n_owned, uint32_t* n_ghost, uint32_t* n_send);
/* The device steps of BlockMatrix::distributed_matvec (blockMatrix.hpp:
 * 351-437) around the caller's exchange (NCCL, MPI, ...), on the context's
 * stream.  x_full = [x_owned (n_owned*bs) | ghosts (n_ghost*bs, recv order)].
 *   pack:  send_buf = x_owned rows listed in send_local (n_send*bs values)
 *   owned: y  = the owned columns' blocks times x_full (reads no ghost)
 *   ghost: y += the ghost columns' blocks times x_full
 * Sums as the reference's MPI branch: y from zero, owned blocks in row order,
 * then the ghost blocks, each block component summed in column order. */
b2s_status b2s_baij_halo_pack_device(b2s_ctx* ctx, const b2s_baij* A, const double* d_x_owned, double* d_send_buf);
b2s_status b2s_baij_dist_matvec_owned_device(b2s_ctx* ctx, const b2s_baij* A, const double* d_x_full, double* d_y);
b2s_status b2s_baij_dist_matvec_ghost_device(b2s_ctx* ctx, const b2s_baij* A, const double* d_x_full, double* d_y);

/* --------------------------------------------------------- preconditioners */

typedef enum b2s_pc_kind
{
    B2S_PC_NONE = 0,        /* identity: "none", "identity", "noprecond", ("cg" for pcg) */
    B2S_PC_DIAG = 1,        /* make_diag_preconditioner, array.cpp:2450-2508 */
    B2S_PC_IC0 = 2,         /* make_ic0_preconditioner, array.cpp:2522-2732 */
    B2S_PC_ILU0 = 3,        /* make_ilu0_preconditioner, array.cpp:2744-2934 */
    B2S_PC_SSOR = 4,        /* make_ssor_preconditioner, array.cpp:3068-3164 */
    B2S_PC_SA_AMG = 5,      /* smoothed aggregation: make_block_amg_preconditioner on the
                               BS=1 condensed matrix, blockMatrix.hpp:1051-1179 */
    B2S_PC_LEARNED_IC0 = 6, /* IC(0) pattern with values from the message-passing network */
    B2S_PC_BJACOBI = 7,     /* BlockMatrix::gmres "blockjacobi", blockMatrix.hpp:714-733 */
    B2S_PC_BILU0 = 8,       /* make_block_ilu0_preconditioner, blockMatrix.hpp:455-623 */
    B2S_PC_BSA_AMG = 9,     /* make_block_amg_preconditioner on a BAIJ matrix */
    B2S_PC_SCHUR = 10,      /* make_schur_preconditioner (b2s_pc_create_schur) */
    B2S_PC_SCALED = 11      /* alpha times another preconditioner (b2s_pc_create_scaled) */
} b2s_pc_kind;

/* Storage / arithmetic precision of a preconditioner. */
typedef enum b2s_precision
{
    B2S_FP64 = 0,
    B2S_FP32 = 1, /* IC(0)/ILU(0)/block ILU(0)/learned IC(0): factors stored FP32, solves
                     accumulate in FP32; SA-AMG: FP32 copies of A, P, R and D^-1 on every level,
                     FP64 vectors and arithmetic, the coarsest dense LU in FP64; the diagonal,
                     block-Jacobi and SSOR preconditioners ignore it */
    B2S_BF16 = 2  /* reserved: no preconditioner stores BF16 values, so b2s_pc_create* returns
                     B2S_UNSUPPORTED (FP32 AMG values already left the V-cycle time unchanged) */
} b2s_precision;

/* Triangular-solve schedule for IC(0)/ILU(0)/block ILU(0). */
typedef enum b2s_trsv
{
    B2S_TRSV_AUTO = 0,
    B2S_TRSV_LEVEL = 1,    /* one launch per level of the dependency DAG */
    B2S_TRSV_SYNCFREE = 2, /* one launch; rows wait on bounded per-row ready flags */
    B2S_TRSV_CHUNK = 3,    /* one launch; row chunks staged in shared memory, local levels split by
                              barriers, bounded flags between chunks (the AUTO choice) */
    B2S_TRSV_JACOBI = 4    /* inexact: rows grouped into segments of trsv_segment consecutive rows;
                              each segment solved on its own, then trsv_sweeps block-Jacobi sweeps
                              (Gauss-Seidel inside a segment, the previous sweep's values outside);
                              segment 1 is plain Jacobi, a truncated Neumann series.  Fully
                              parallel passes; the IC(0) apply stays symmetric positive definite
                              (M^-1 = F^T F) but is no longer the exact factor solve */
} b2s_trsv;

typedef struct b2s_pc_opts
{
    double omega;        /* SSOR relaxation (reference default 1.2) */
    int precision;       /* b2s_precision */
    int trsv;            /* b2s_trsv */
    int amg_ref_coarse;  /* 1: reproduce the reference's coarsest-level elimination
                            (blockMatrix.hpp:958-1000) bit for bit; 0: correct pivoted LU */
    int amg_max_levels;  /* 0: reference default 20 */
    int amg_coarse_max;  /* 0: reference default 50 block rows */
    int amg_aggregation; /* 0: parallel rule (default): distance-2 independent roots chosen in
                               rounds by a fixed per-row key, then neighbour assignment;
                            1: the reference's capped greedy rule (blockMatrix.hpp:1101-1111),
                               which stalls on 3-D problems and serves parity tests;
                            2: sequential three-phase smoothed-aggregation rule */
    const char* learned_weights; /* B2S_PC_LEARNED_IC0: path of a weight file, NULL = built-in init */
    int trsv_sweeps;     /* B2S_TRSV_JACOBI: sweeps per triangle after the segment solve (0: 8) */
    int trsv_segment;    /* B2S_TRSV_JACOBI: rows per segment, 1..32 (0: 1, plain Jacobi) */
    int factor_sweeps;   /* IC(0): 0 = the exact factorisation (level order, the reference's values);
                            k > 0 = k fixed-point sweeps over all entries at once (Chow-Patel), an
                            approximate factor; a failed pivot falls back to the exact factorisation */
} b2s_pc_opts;

/* Fills opts with the reference's defaults. */
void b2s_pc_opts_default(b2s_pc_opts* opts);

b2s_status b2s_pc_create(b2s_ctx* ctx, const b2s_csr* A, b2s_pc_kind kind, const b2s_pc_opts* opts, b2s_pc** out);
b2s_status b2s_pc_create_baij(b2s_ctx* ctx, const b2s_baij* A, b2s_pc_kind kind, const b2s_pc_opts* opts,
                              b2s_pc** out);
/* Preconditioner that calls back into host code (a user's std::function).
 * The solver copies r to host, calls fn(user, r, z, n) and copies z back. */
typedef int (*b2s_host_pc_fn)(void* user, const double* r, double* z, uint64_t n);
b2s_status b2s_pc_create_host(b2s_ctx* ctx, uint64_t n, b2s_host_pc_fn fn, void* user, b2s_pc** out);
b2s_status b2s_pc_destroy(b2s_pc* pc);
/* Block-triangular saddle-point preconditioner, make_schur_preconditioner
 * (blockMatrix.hpp:637-685), on the device.  For r = [r_u (n_vel); r_p (n_pres)]:
 *   w_u = A^-1 r_u;  r_p' = B w_u - r_p;  z_p = S^-1 r_p';
 *   r_u' = r_u - B^T z_p;  z_u = A^-1 r_u';  z = [z_u; z_p]
 * A_pc (n_vel rows) and S_pc (n_pres rows; NULL = identity) are preconditioners
 * of this context, B (n_pres x n_vel) and Bt (n_vel x n_pres) its CSR handles;
 * all of them must outlive the Schur preconditioner.  Every step stays on the
 * device (no host round trip per apply); each step's arithmetic is the
 * reference's, so with bit-exact parts the apply equals the reference's bit
 * for bit. */
b2s_status b2s_pc_create_schur(b2s_ctx* ctx, uint64_t n_vel, uint64_t n_pres, const b2s_csr* B, const b2s_csr* Bt,
                               b2s_pc* A_pc, b2s_pc* S_pc, b2s_pc** out);
/* z = alpha * M^-1 r for a preconditioner M of this context (which must
 * outlive it): the scaled pressure AMG of the reference's 3-D Stokes test
 * (test_BlockMatrix_schur3d.cpp:150-160, z[i] = scale * w[i]). */
b2s_status b2s_pc_create_scaled(b2s_ctx* ctx, b2s_pc* inner, double alpha, b2s_pc** out);

/* z = M^-1 r (the functor returned by the reference factories). */
b2s_status b2s_pc_apply(b2s_ctx* ctx, b2s_pc* pc, const double* r, double* z);
b2s_status b2s_pc_apply_device(b2s_ctx* ctx, b2s_pc* pc, const double* d_r, double* d_z);
/* Factor / hierarchy inspection (for parity tests).  what:
 *   "ic0.L"  rp,ci,v of L incl. diagonal;   "ic0.diag"  diag (vals only)
 *   "ilu0.L" strict L;  "ilu0.U" U incl. diagonal
 *   "levels.L" / "levels.U": level of each row (ci holds levels, rp/v unused)
 *   "ssor.colour": rp = color_ptr (ncolor+1), ci = new_id (n); v = diag2
 *   "bilu0.L" / "bilu0.U" / "bilu0.inv": block factors (v = nnzb*bs*bs)
 *   "amg.N.A", "amg.N.P": level N operator / prolongation; "amg.N.agg": aggregates in ci
 *   "pcg.tiles": sizes = {tiles of the tiled persistent PCG kernel (0: none), rows per thread,
 *                shared memory per CTA}; no arrays
 *   "pcg.tiles.idx": the tiles' index blobs as 32-bit words in ci.  A 5-point grid's blobs are
 *                built on the device from closed forms; with the environment variable
 *                B2S_TILE_PLANNER=bfs at set-up the general breadth-first planner (host) lays them
 *                out instead, for grids up to 65536 rows (it gives the same bytes)
 *   "trsv.grid5": sizes = {points per grid line B (0: the exact solves do not take the 5-point
 *                grid schedule), grid lines, 1 if the factor's values are packed for it}; no
 *                arrays (IC(0) and ILU(0) with the chunk schedule)
 * Query sizes with NULL arrays: sizes[0] = rows (+1 for rp), sizes[1] = nnz, sizes[2] = values. */
b2s_status b2s_pc_export(b2s_ctx* ctx, b2s_pc* pc, const char* what, uint64_t* sizes, uint32_t* rp, uint32_t* ci,
                         double* v);

/* Maps a preconditioner name to a kind with the reference's alias tables:
 * method B2S_PCG array.cpp:3482-3515, B2S_BICGSTAB 3637-3673, B2S_GMRES
 * 4212-4242 (to_lower first); block GMRES blockMatrix.hpp:710-744 (exact
 * match).  "amg" maps to B2S_PC_SA_AMG.  Unknown names: B2S_INVALID_ARG. */
b2s_status b2s_pc_kind_from_name(int method, const char* name, b2s_pc_kind* kind);

/* ------------------------------------------------------ learned IC(0) net
 * A message-passing network over the graph of A (3 layers, 64 hidden,
 * BF16 weights, FP32 accumulation) that corrects the IC(0) factor values on
 * the unchanged pattern (no counterpart in the reference).  Training runs on
 * the GPU with this library's own forward and backward kernels. */
typedef struct b2s_learner b2s_learner;

/* New network: hidden weights from `seed`, output layer zero (the untrained
 * network reproduces IC(0)). */
b2s_status b2s_learner_create(b2s_ctx* ctx, uint64_t seed, b2s_learner** out);
b2s_status b2s_learner_destroy(b2s_learner* L);
/* Weight file: "B2SLRN01", uint32 version 1, uint32 count, float[count],
 * uint64 FNV-1a checksum of the floats. */
b2s_status b2s_learner_load(b2s_learner* L, const char* path);
b2s_status b2s_learner_save(b2s_learner* L, const char* path);
/* FP32 master parameters: get (set == 0) or set (set == 1); *count in/out. */
b2s_status b2s_learner_params(b2s_learner* L, float* params, uint64_t* count, int set);
/* Training loss of b2s_learner_step, over probe vectors w: */
#define B2S_LOSS_PRECOND 0 /* preconditioned residual mean_w ||w - (L~L~^T)^{-1} A w||^2 / ||w||^2 (default) */
#define B2S_LOSS_FACTOR 1  /* factorisation residual mean_w ||(L~L~^T - A) w||^2 / ||A w||^2 */
#define B2S_LOSS_SWEEPS 2  /* preconditioned residual with the deployed sweep apply: M^-1 = F^T F, F the
                              trsv_sweeps Jacobi sweeps of L~ (B2S_TRSV_JACOBI's operator) */
b2s_status b2s_learner_set_loss(b2s_learner* L, int kind);
/* B2S_LOSS_SWEEPS: Jacobi sweeps per triangle (default 6); every loss: the base factor the network
 * corrects, 0 = the exact IC(0) (default), k > 0 = k fixed-point sweeps (b2s_pc_opts.factor_sweeps),
 * as the preconditioner that deploys the network is built. */
b2s_status b2s_learner_set_sweeps(b2s_learner* L, int trsv_sweeps, int factor_sweeps);
/* One training step on A (SPD, structurally symmetric) with the learner's
 * loss over nprobes probes (generated from seed, every second one
 * Jacobi-smoothed; or taken from `probes`, host, nprobes * n, when not NULL).
 * update = 1 applies one Adam step with learning rate lr.  loss and grad
 * (host, count floats) are optional. */
b2s_status b2s_learner_step(b2s_ctx* ctx, b2s_learner* L, const b2s_csr* A, int nprobes, uint64_t seed,
                            const double* probes, double lr, int update, double* loss, float* grad);
/* IC(0) corrected by this network (the same kernels as B2S_PC_LEARNED_IC0). */
b2s_status b2s_pc_create_learned(b2s_ctx* ctx, const b2s_csr* A, b2s_learner* L, const b2s_pc_opts* opts,
                                 b2s_pc** out);
/* The network's hidden dense layer on the tensor cores (tcgen05, BF16 x BF16,
 * FP32 accumulation), device pointers on the context's stream:
 * d_y (n x no, FP32, row-major) = bf16(d_x) (n x k, FP32, row-major) W^T
 * [+ d_bias], W (no x k, BF16 bits, row-major); bf16() rounds to nearest even.
 * Supported: k = 64, no = 128 (the message-passing layers' [W_s; W_m]) and
 * k = 64, no = 64; other shapes return B2S_UNSUPPORTED.  All pointers 16-byte
 * aligned; d_bias may be NULL.  No counterpart in the reference. */
b2s_status b2s_dense_bf16_device(b2s_ctx* ctx, uint64_t n, int k, int no, const float* d_x, const uint16_t* d_w,
                                 const float* d_bias, float* d_y);

/* ----------------------------------------------------------------- solvers */

typedef enum b2s_method
{
    B2S_PCG = 0,       /* SMatrix::pcg, array.cpp:3445-3601 */
    B2S_BICGSTAB = 1,  /* SMatrix::bicgstab, array.cpp:3602-3842 */
    B2S_GMRES = 2,     /* SMatrix::gmres, array.cpp:4190-4533; BlockMatrix::gmres */
    B2S_FGMRES = 3,    /* flexible GMRES (Z stored), for variable / low-precision preconditioners */
    B2S_BLOCK_GMRES = 4, /* name table of BlockMatrix::gmres for b2s_pc_kind_from_name only */
    B2S_STATIONARY = 5   /* x += M^-1 (b - A x) from x = 0 with the true residual checked before every
                            correction: SMatrix::amg (array.cpp:4534-4563) when M is an AMG
                            preconditioner (one V-cycle per correction); it = index of the last check,
                            max_iter - 1 when the loop runs out */
} b2s_method;

/* Gram-Schmidt variant for (F)GMRES. */
typedef enum b2s_orth
{
    B2S_ORTH_MGS = 0, /* modified Gram-Schmidt, the reference's order */
    B2S_ORTH_CGS2 = 1 /* classical Gram-Schmidt applied twice: two batched passes */
} b2s_orth;

typedef struct b2s_solve_opts
{
    double tol;      /* relative residual target (reference default 1e-10) */
    int maxit;       /* reference default 2000 */
    int restart;     /* GMRES restart length m */
    int orth;        /* b2s_orth */
    int ir_steps;    /* >0: iterative refinement sweeps around the solve (outer FP64 residual) */
    double ir_inner_tol; /* relative tolerance of each refinement solve (0: 1e-4) */
    int check_every; /* host polls convergence every this many iterations (0: auto) */
    int use_graphs;  /* 1: replay iteration bodies as CUDA graphs */
    int stall_window; /* B2S_PC_LEARNED_IC0: the solve counts as stalled when the recursive
                         residual has not halved within this many iterations (0: 200,
                         < 0: never); a stalled, broken-down or unconverged learned solve
                         continues with plain FP64 IC(0) from its iterate (b2s_stats.fallbacks) */
    int persistent;   /* PCG with an FP32 IC(0)-type preconditioner applied by plain Jacobi sweeps:
                         0 = the whole loop in one launch, over 2-D tiles when they can be planned,
                         else over row strips; 1 = row strips only; 2 = three launches per iteration */
} b2s_solve_opts;

void b2s_solve_opts_default(b2s_solve_opts* opts);

typedef struct b2s_stats
{
    int it;               /* the reference's returned iteration count (its own convention) */
    int iterations;       /* Krylov iterations executed (SpMVs in the loop) */
    int spmvs;            /* operator applications incl. true-residual checks */
    int pc_applies;       /* preconditioner applications */
    int restarts;         /* GMRES restarts / refinement sweeps */
    int status;           /* b2s_status of the solve */
    double relres;        /* final recursive (or Givens) relative residual */
    double relres_true;   /* ||b - A x|| / ||b|| recomputed in FP64 on exit */
    double setup_ms;      /* preconditioner setup inside this call (0 when given one) */
    double solve_ms;      /* iteration time, device events */
    int fallbacks;        /* 1 when a learned IC(0) solve handed over to plain IC(0) */
    int stalled_at;       /* iterations run with the learned preconditioner before that */
} b2s_stats;

/* Solves A x = b from x0 = 0.  pc may be NULL (identity).  Host pointers. */
b2s_status b2s_solve(b2s_ctx* ctx, const b2s_csr* A, b2s_pc* pc, b2s_method method, const b2s_solve_opts* opts,
                     const double* b, double* x, b2s_stats* stats);
b2s_status b2s_solve_device(b2s_ctx* ctx, const b2s_csr* A, b2s_pc* pc, b2s_method method,
                            const b2s_solve_opts* opts, const double* d_b, double* d_x, b2s_stats* stats);
/* SMatrix::sor (array.cpp:3843-3945), red_black = 0, and SMatrix::sor_rb
 * (array.cpp:3946-4189), red_black = 1: SOR sweeps from x0 = 0 until
 * ||b - A x|| / ||b|| < tol or maxit sweeps; stats->it is the reference's
 * returned index of the last sweep.  Natural order follows the reference's
 * sequential Gauss-Seidel order (one sync-free traversal per sweep);
 * red-black uses its colouring and renumbering.  Iterates equal the
 * reference's bit for bit.  Errors as the reference: a non-square matrix
 * (B2S_SHAPE), 0 < omega < 2 violated (B2S_INVALID_ARG, checked after a zero
 * right-hand side returns x = 0), a missing or zero diagonal
 * (B2S_MISSING_DIAG), NaN/Inf in the residual (B2S_DIVERGED). */
b2s_status b2s_sor(b2s_ctx* ctx, const b2s_csr* A, int red_black, double omega, double tol, int maxit, const double* b,
                   double* x, b2s_stats* stats);
b2s_status b2s_sor_device(b2s_ctx* ctx, const b2s_csr* A, int red_black, double omega, double tol, int maxit,
                          const double* d_b, double* d_x, b2s_stats* stats);
/* Same on a BAIJ operator (BlockMatrix::gmres; block PCG is an extension). */
b2s_status b2s_solve_baij(b2s_ctx* ctx, const b2s_baij* A, b2s_pc* pc, b2s_method method, const b2s_solve_opts* opts,
                          const double* b, double* x, b2s_stats* stats);
b2s_status b2s_solve_baij_device(b2s_ctx* ctx, const b2s_baij* A, b2s_pc* pc, b2s_method method,
                                 const b2s_solve_opts* opts, const double* d_b, double* d_x, b2s_stats* stats);

/* ------------------------------------------------------------- generators
 * Host-side problem generators for the benchmark configurations.  Two-step:
 * call with NULL arrays to get n and nnz, then with arrays of that size.
 * Output is CSR (sorted columns) or BAIJ. */

/* 2-D 5-point Poisson on an N x N interior grid, Dirichlet by elimination
 * (diagonal 4, off-diagonal -1; test_SMatrix_pcg.cpp:70-99). */
b2s_status b2s_gen_poisson2d(uint32_t N, uint32_t* n, uint32_t* nnz, uint32_t* rp, uint32_t* ci, double* v);
/* 3-D 7-point Poisson on N^3 (diagonal 6, off-diagonal -1). */
b2s_status b2s_gen_poisson3d(uint32_t N, uint32_t* n, uint32_t* nnz, uint32_t* rp, uint32_t* ci, double* v);
/* 3-D convection-diffusion, central diffusion + first-order upwind for a
 * constant velocity (vx, vy, vz) >= 0: diagonal 6 + vx + vy + vz, upwind
 * neighbours -1 - v_d, downwind -1. */
b2s_status b2s_gen_convdiff3d(uint32_t N, double vx, double vy, double vz, uint32_t* n, uint32_t* nnz, uint32_t* rp,
                              uint32_t* ci, double* v);
/* Q1 hexahedral linear elasticity on an NE^3-element unit cube, E, nu,
 * 2x2x2 Gauss quadrature, nodes on the x=0 face clamped (their block rows and
 * columns eliminated).  BAIJ with bs=3, node-major. */
b2s_status b2s_gen_elasticity_q1(uint32_t NE, double E, double nu, uint32_t* nbr, uint32_t* nnzb, uint32_t* rp,
                                 uint32_t* ci, double* v);
/* -div(k grad u) on an N x N grid, 5-point finite volume, harmonic-mean face
 * coefficients, Dirichlet (zero) boundary; log k is a Gaussian random field
 * with squared-exponential covariance (correlation length corr, variance var)
 * sampled by FFT circulant embedding from `seed`.  kfield (N*N, optional)
 * receives k. */
b2s_status b2s_gen_grf_diffusion(uint32_t N, double corr, double var, uint64_t seed, uint32_t* n, uint32_t* nnz,
                                 uint32_t* rp, uint32_t* ci, double* v, double* kfield);
/* Uniform[-1,1] vector from a counter-based generator: element i is
 * splitmix64(seed * 0x9E3779B97F4A7C15 + i) mapped to [-1, 1). */
b2s_status b2s_gen_uniform(uint64_t seed, uint64_t n, double* out);

#ifdef __cplusplus
}
#endif

#endif /* B2S_H */
