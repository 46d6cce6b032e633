// C harness around the reference library (xuyinshen/cpp-FEM-solver), compiled
// in place from the reference sources by oracle/Makefile into oracle/_ref/.
//
// TEST INFRASTRUCTURE ONLY.  The product never links, loads or calls this:
// only tests/, __graft_entry__.smoke() and bench.py's reference/cpu_baseline
// legs use it, as the checker and as the timed CPU baseline.
//
// The translation unit includes ode-solver/src/math/array.cpp textually (it is
// not copied), which exposes the file-static internals (make_redblack_data,
// the IC0/ILU0/RB data structs, make_amg_data) next to the public API.
// blockMatrix.hpp is header-only and must live in exactly one TU, which is
// this one.
//
// Factor data captured inside the reference's std::function preconditioners
// is read back through the functor's storage: with libstdc++ a lambda that
// holds a std::shared_ptr is heap-stored and the first word of the
// std::function is the lambda's address; GCC lays captures out in
// capture-list order, so the shared_ptr named first in the capture list sits
// at offset 0.  Every export checks the recovered object's sizes against the
// matrix before using it.
#include "src/math/array.cpp"
#include "math/blockMatrix.hpp"

#include <cstring>
#include <string>
#ifdef CPPNUM_HAVE_OPENMP
#include <omp.h>
#endif

using sparse::SMatrix;
using PC = std::function<void(const std::vector<double>&, std::vector<double>&)>;

namespace {

int fail(char* err, int errlen, const char* msg)
{
    if (err && errlen > 0)
    {
        std::strncpy(err, msg, (size_t)errlen - 1);
        err[errlen - 1] = 0;
    }
    return 0;
}

// 0 ok, 1 std::invalid_argument / std::out_of_range, 2 std::runtime_error, 3 other
template <typename F>
int guarded(char* err, int errlen, F&& f)
{
    try
    {
        f();
        return 0;
    }
    catch (const std::invalid_argument& e) { fail(err, errlen, e.what()); return 1; }
    catch (const std::out_of_range& e)     { fail(err, errlen, e.what()); return 1; }
    catch (const std::runtime_error& e)    { fail(err, errlen, e.what()); return 2; }
    catch (const std::exception& e)        { fail(err, errlen, e.what()); return 3; }
}

template <typename T>
std::shared_ptr<T>& captured_data(PC& f)
{
    void* lam = *reinterpret_cast<void**>(&f);
    return *reinterpret_cast<std::shared_ptr<T>*>(lam);
}

struct RefPC
{
    PC f;
    std::string kind;
    uint32_t n = 0;
};

struct RefBlk
{
    int bs;
    void* m;   // block::BlockMatrix<double, bs>*
};

template <int BS>
block::BlockMatrix<double, BS>& blk(RefBlk* b) { return *static_cast<block::BlockMatrix<double, BS>*>(b->m); }

}  // namespace

extern "C" {

void ref_set_threads(int t)
{
#ifdef CPPNUM_HAVE_OPENMP
    omp_set_num_threads(t);
#else
    (void)t;
#endif
}

int ref_max_threads(void)
{
#ifdef CPPNUM_HAVE_OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// ---------------- CSR (array.cpp:2072-2235) ----------------
void* ref_csr_coo(uint32_t n, uint32_t m, uint64_t nnz, const double* v, const uint32_t* r,
                  const uint32_t* c, char* err, int errlen)
{
    SMatrix* out = nullptr;
    int st = guarded(err, errlen, [&] {
        std::vector<double> vv(v, v + nnz);
        std::vector<uint32_t> rr(r, r + nnz), cc(c, c + nnz);
        out = new SMatrix(n, m, vv, rr, cc);
    });
    return st == 0 ? out : nullptr;
}

void* ref_csr_direct(uint32_t n, uint32_t m, const uint32_t* rp, const uint32_t* ci, const double* v)
{
    const uint32_t nnz = rp[n];
    return new SMatrix(n, m, std::vector<uint32_t>(rp, rp + n + 1), std::vector<uint32_t>(ci, ci + nnz),
                       std::vector<double>(v, v + nnz));
}

void ref_csr_free(void* A) { delete static_cast<SMatrix*>(A); }
uint32_t ref_csr_rows(void* A) { return static_cast<SMatrix*>(A)->rows(); }
uint32_t ref_csr_cols(void* A) { return static_cast<SMatrix*>(A)->cols(); }
uint32_t ref_csr_nnz(void* A) { return static_cast<SMatrix*>(A)->nnz(); }

void ref_csr_export(void* A, uint32_t* rp, uint32_t* ci, double* v)
{
    const SMatrix& M = *static_cast<SMatrix*>(A);
    std::memcpy(rp, M.row_ptr().data(), sizeof(uint32_t) * (M.rows() + 1));
    std::memcpy(ci, M.col_idx().data(), sizeof(uint32_t) * M.nnz());
    std::memcpy(v, M.values().data(), sizeof(double) * M.nnz());
}

void* ref_csr_transpose(void* A) { return new SMatrix(static_cast<SMatrix*>(A)->transpose()); }
void* ref_csr_matmul(void* A, void* B) { return new SMatrix(*static_cast<SMatrix*>(A) * *static_cast<SMatrix*>(B)); }

void ref_spmv(void* A, const double* x, double* y)
{
    const SMatrix& M = *static_cast<SMatrix*>(A);
    std::vector<double> xv(x, x + M.cols());
    std::vector<double> yv = SMatrix::spmv(M, xv);
    std::memcpy(y, yv.data(), sizeof(double) * yv.size());
}

double ref_dot(const double* a, const double* b, uint64_t n)
{
    return SMatrix::dot(std::vector<double>(a, a + n), std::vector<double>(b, b + n));
}

// ---------------- Solvers (array.cpp:3445-4563) ----------------
// method: 0 pcg, 1 bicgstab, 2 gmres (string overload), 3 amg (stand-alone)
int ref_solve(void* A, int method, const char* precond, int restart, double tol, int maxit,
              const double* b, double* x, int* it, char* err, int errlen)
{
    const SMatrix& M = *static_cast<SMatrix*>(A);
    return guarded(err, errlen, [&] {
        std::vector<double> bv(b, b + M.rows());
        std::tuple<std::vector<double>, int> res;
        switch (method)
        {
            case 0: res = SMatrix::pcg(M, bv, precond, tol, maxit); break;
            case 1: res = SMatrix::bicgstab(M, bv, precond, tol, maxit); break;
            case 2: res = SMatrix::gmres(M, bv, std::string(precond), restart, tol, maxit); break;
            case 3: res = SMatrix::amg(M, bv, tol, maxit); break;
            default: throw std::invalid_argument("ref_solve: unknown method");
        }
        std::memcpy(x, std::get<0>(res).data(), sizeof(double) * M.rows());
        *it = std::get<1>(res);
    });
}

// ---------------- SOR solvers (array.cpp:3843-4189) ----------------
int ref_sor(void* A, int red_black, double omega, double tol, int maxit, const double* b, double* x, int* it,
            char* err, int errlen)
{
    const SMatrix& M = *static_cast<SMatrix*>(A);
    return guarded(err, errlen, [&] {
        std::vector<double> bv(b, b + M.rows());
        auto res = red_black ? SMatrix::sor_rb(M, bv, omega, tol, maxit) : SMatrix::sor(M, bv, omega, tol, maxit);
        std::memcpy(x, std::get<0>(res).data(), sizeof(double) * M.rows());
        *it = std::get<1>(res);
    });
}

// ---------------- Preconditioner factories (array.cpp:2450-3398) ----------------
void* ref_pc_create(void* A, const char* kind, double omega, char* err, int errlen)
{
    const SMatrix& M = *static_cast<SMatrix*>(A);
    RefPC* pc = new RefPC();
    pc->kind = kind;
    pc->n = M.rows();
    int st = guarded(err, errlen, [&] {
        if (pc->kind == "diag") pc->f = SMatrix::make_diag_preconditioner(M);
        else if (pc->kind == "ic0") pc->f = SMatrix::make_ic0_preconditioner(M);
        else if (pc->kind == "ilu0") pc->f = SMatrix::make_ilu0_preconditioner(M);
        else if (pc->kind == "ssor") pc->f = SMatrix::make_ssor_preconditioner(M, omega);
        else if (pc->kind == "amg") pc->f = SMatrix::make_amg_preconditioner(M);
        else throw std::invalid_argument("ref_pc_create: unknown kind");
    });
    if (st != 0) { delete pc; return nullptr; }
    return pc;
}

void ref_pc_apply(void* p, const double* r, double* z)
{
    RefPC* pc = static_cast<RefPC*>(p);
    std::vector<double> rv(r, r + pc->n), zv;
    pc->f(rv, zv);
    std::memcpy(z, zv.data(), sizeof(double) * pc->n);
}

void ref_pc_free(void* p) { delete static_cast<RefPC*>(p); }

int ref_gmres_pc(void* A, void* p, int restart, double tol, int maxit, const double* b, double* x,
                 int* it, char* err, int errlen)
{
    const SMatrix& M = *static_cast<SMatrix*>(A);
    RefPC* pc = static_cast<RefPC*>(p);
    return guarded(err, errlen, [&] {
        std::vector<double> bv(b, b + M.rows());
        auto res = SMatrix::gmres(M, bv, pc->f, restart, tol, maxit);
        std::memcpy(x, std::get<0>(res).data(), sizeof(double) * M.rows());
        *it = std::get<1>(res);
    });
}

// make_schur_preconditioner (blockMatrix.hpp:637-685) over the reference's
// own SMatrix::spmv of B and B^T, with the velocity preconditioner A_pc and
// the pressure preconditioner S_pc scaled by s_scale (z[i] = s_scale * w[i],
// the S_pre of test_BlockMatrix_schur3d.cpp:150-160), or the identity
// (z = r, test_BlockMatrix_schur.cpp:95) when S_pc is null.
void* ref_schur_create(uint32_t n_vel, uint32_t n_pres, void* B, void* Bt, void* A_pc, void* S_pc, double s_scale)
{
    const SMatrix Bm = *static_cast<SMatrix*>(B), Btm = *static_cast<SMatrix*>(Bt);
    block::SaddlePointSystem sys;
    sys.n_vel = n_vel;
    sys.n_pres = n_pres;
    sys.spmv_B = [Bm](const std::vector<double>& x, std::vector<double>& y) { y = SMatrix::spmv(Bm, x); };
    sys.spmv_Bt = [Btm](const std::vector<double>& x, std::vector<double>& y) { y = SMatrix::spmv(Btm, x); };
    PC Sf;
    if (S_pc)
    {
        const PC inner = static_cast<RefPC*>(S_pc)->f;
        Sf = [inner, s_scale](const std::vector<double>& r, std::vector<double>& z) {
            std::vector<double> w;
            inner(r, w);
            z.resize(r.size());
            for (size_t i = 0; i < r.size(); ++i) z[i] = s_scale * w[i];
        };
    }
    else
        Sf = [](const std::vector<double>& r, std::vector<double>& z) { z = r; };
    RefPC* pc = new RefPC();
    pc->kind = "schur";
    pc->n = n_vel + n_pres;
    pc->f = block::make_schur_preconditioner(sys, static_cast<RefPC*>(A_pc)->f, Sf);
    return pc;
}

// IC(0) factor of a "ic0" preconditioner (IC0_Data, array.cpp:2510-2521).
// sizes[0] = nnz(L) incl. diagonal, sizes[1] = nnz(L^T strict).  Pass null
// arrays to query sizes.  Returns 0 on success, -1 if the object is not IC0.
int ref_ic0_export(void* p, uint32_t* sizes, uint32_t* Lrp, uint32_t* Lci, double* Lv, uint32_t* LTrp,
                   uint32_t* LTci, double* LTv, double* diag)
{
    RefPC* pc = static_cast<RefPC*>(p);
    if (pc->kind != "ic0") return -1;
    auto& d = captured_data<sparse::IC0_Data>(pc->f);
    if (!d || d->diag.size() != pc->n || d->L_row_ptr.size() != pc->n + 1) return -1;
    sizes[0] = d->L_row_ptr[pc->n];
    sizes[1] = d->LT_row_ptr[pc->n];
    if (!Lrp) return 0;
    std::memcpy(Lrp, d->L_row_ptr.data(), 4 * (pc->n + 1));
    std::memcpy(Lci, d->L_col_idx.data(), 4 * sizes[0]);
    std::memcpy(Lv, d->L_values.data(), 8 * sizes[0]);
    std::memcpy(LTrp, d->LT_row_ptr.data(), 4 * (pc->n + 1));
    std::memcpy(LTci, d->LT_col_idx.data(), 4 * sizes[1]);
    std::memcpy(LTv, d->LT_values.data(), 8 * sizes[1]);
    std::memcpy(diag, d->diag.data(), 8 * pc->n);
    return 0;
}

// ILU(0) factor (ILU0_Data, array.cpp:2733-2743).  sizes = {nnz(L), nnz(U)}.
int ref_ilu0_export(void* p, uint32_t* sizes, uint32_t* Lrp, uint32_t* Lci, double* Lv, uint32_t* Urp,
                    uint32_t* Uci, double* Uv, uint32_t* diag_idx)
{
    RefPC* pc = static_cast<RefPC*>(p);
    if (pc->kind != "ilu0") return -1;
    auto& d = captured_data<sparse::ILU0_Data>(pc->f);
    if (!d || d->diag_U_idx.size() != pc->n || d->L_row_ptr.size() != pc->n + 1) return -1;
    sizes[0] = d->L_row_ptr[pc->n];
    sizes[1] = d->U_row_ptr[pc->n];
    if (!Lrp) return 0;
    std::memcpy(Lrp, d->L_row_ptr.data(), 4 * (pc->n + 1));
    std::memcpy(Lci, d->L_col_idx.data(), 4 * sizes[0]);
    std::memcpy(Lv, d->L_values.data(), 8 * sizes[0]);
    std::memcpy(Urp, d->U_row_ptr.data(), 4 * (pc->n + 1));
    std::memcpy(Uci, d->U_col_idx.data(), 4 * sizes[1]);
    std::memcpy(Uv, d->U_values.data(), 8 * sizes[1]);
    std::memcpy(diag_idx, d->diag_U_idx.data(), 4 * pc->n);
    return 0;
}

// Multicolour data (make_redblack_data, array.cpp:2947-3067).
// Writes ncolor, color_ptr[ncolor+1] (capacity n+1), new_id[n], perm[n], diag2[n].
int ref_redblack(void* A, uint32_t* ncolor, uint32_t* color_ptr, uint32_t* new_id, uint32_t* perm,
                 double* diag2, char* err, int errlen)
{
    const SMatrix& M = *static_cast<SMatrix*>(A);
    return guarded(err, errlen, [&] {
        auto d = sparse::make_redblack_data(M);
        *ncolor = d->ncolor;
        std::memcpy(color_ptr, d->color_ptr.data(), 4 * (d->ncolor + 1));
        std::memcpy(new_id, d->new_id.data(), 4 * M.rows());
        std::memcpy(perm, d->perm.data(), 4 * M.rows());
        std::memcpy(diag2, d->diag2.data(), 8 * M.rows());
    });
}

// ---------------- BlockMatrix (blockMatrix.hpp), BS in {1, 3} ----------------
void* ref_blk_create(int bs, uint32_t nbr, uint32_t nbc, const uint32_t* rp, const uint32_t* ci,
                     const double* v)
{
    const uint32_t nnzb = rp[nbr];
    std::vector<uint32_t> r(rp, rp + nbr + 1), c(ci, ci + nnzb);
    RefBlk* b = new RefBlk{bs, nullptr};
    if (bs == 1)
        b->m = new block::BlockMatrix<double, 1>(nbr, nbc, r, c, std::vector<double>(v, v + nnzb));
    else if (bs == 3)
        b->m = new block::BlockMatrix<double, 3>(nbr, nbc, r, c, std::vector<double>(v, v + (size_t)nnzb * 9));
    else { delete b; return nullptr; }
    return b;
}

void* ref_blk_condense(int bs, void* A, uint32_t nbr, uint32_t nbc)
{
    const SMatrix& M = *static_cast<SMatrix*>(A);
    RefBlk* b = new RefBlk{bs, nullptr};
    if (bs == 1) b->m = new block::BlockMatrix<double, 1>(block::BlockMatrix<double, 1>::condense(M, nbr, nbc));
    else if (bs == 3) b->m = new block::BlockMatrix<double, 3>(block::BlockMatrix<double, 3>::condense(M, nbr, nbc));
    else { delete b; return nullptr; }
    return b;
}

void ref_blk_free(void* p)
{
    RefBlk* b = static_cast<RefBlk*>(p);
    if (b->bs == 1) delete &blk<1>(b);
    else delete &blk<3>(b);
    delete b;
}

uint32_t ref_blk_nnzb(void* p)
{
    RefBlk* b = static_cast<RefBlk*>(p);
    return b->bs == 1 ? (uint32_t)blk<1>(b).nnz_blocks() : (uint32_t)blk<3>(b).nnz_blocks();
}

uint32_t ref_blk_rows(void* p)
{
    RefBlk* b = static_cast<RefBlk*>(p);
    return b->bs == 1 ? blk<1>(b).block_rows() : blk<3>(b).block_rows();
}

extern "C++" {
template <int BS>
static void blk_export_t(block::BlockMatrix<double, BS>& M, uint32_t* rp, uint32_t* ci, double* v)
{
    std::memcpy(rp, M.block_row_ptr().data(), 4 * (M.block_rows() + 1));
    std::memcpy(ci, M.block_col_idx().data(), 4 * M.nnz_blocks());
    std::memcpy(v, M.values().data(), 8 * M.nnz_blocks() * BS * BS);
}
}  // extern "C++"

void ref_blk_export(void* p, uint32_t* rp, uint32_t* ci, double* v)
{
    RefBlk* b = static_cast<RefBlk*>(p);
    if (b->bs == 1) blk_export_t(blk<1>(b), rp, ci, v);
    else blk_export_t(blk<3>(b), rp, ci, v);
}

void* ref_blk_transpose(void* p)
{
    RefBlk* b = static_cast<RefBlk*>(p);
    RefBlk* t = new RefBlk{b->bs, nullptr};
    if (b->bs == 1) t->m = new block::BlockMatrix<double, 1>(blk<1>(b).transpose());
    else t->m = new block::BlockMatrix<double, 3>(blk<3>(b).transpose());
    return t;
}

void ref_blk_matvec(void* p, const double* x, double* y)
{
    RefBlk* b = static_cast<RefBlk*>(p);
    std::vector<double> yv;
    if (b->bs == 1)
    {
        auto& M = blk<1>(b);
        M.matvec(std::vector<double>(x, x + M.cols()), yv);
    }
    else
    {
        auto& M = blk<3>(b);
        M.matvec(std::vector<double>(x, x + M.cols()), yv);
    }
    std::memcpy(y, yv.data(), 8 * yv.size());
}

// kind: "ilu0" (make_block_ilu0_preconditioner) or "amg" (make_block_amg_preconditioner)
void* ref_blk_pc_create(void* p, const char* kind, char* err, int errlen)
{
    RefBlk* b = static_cast<RefBlk*>(p);
    RefPC* pc = new RefPC();
    pc->kind = std::string("blk_") + kind;
    int st = guarded(err, errlen, [&] {
        if (b->bs == 1)
        {
            auto& M = blk<1>(b);
            pc->n = M.rows();
            if (std::string(kind) == "ilu0") pc->f = block::make_block_ilu0_preconditioner(M);
            else if (std::string(kind) == "amg") pc->f = block::make_block_amg_preconditioner(M);
            else throw std::invalid_argument("unknown block preconditioner");
        }
        else
        {
            auto& M = blk<3>(b);
            pc->n = M.rows();
            if (std::string(kind) == "ilu0") pc->f = block::make_block_ilu0_preconditioner(M);
            else if (std::string(kind) == "amg") pc->f = block::make_block_amg_preconditioner(M);
            else throw std::invalid_argument("unknown block preconditioner");
        }
    });
    if (st != 0) { delete pc; return nullptr; }
    return pc;
}

// Block ILU(0) factor (BlockILU0_Data, blockMatrix.hpp:121-131).
// sizes = {nnzb(L), nnzb(U)}; values are BS*BS per block.
extern "C++" {
template <int BS>
static int blk_ilu0_export_t(RefPC* pc, uint32_t* sizes, uint32_t* Lrp, uint32_t* Lci, double* Lv,
                             uint32_t* Urp, uint32_t* Uci, double* Uv, uint32_t* Udiag, double* inv_diag)
{
    auto& d = captured_data<block::BlockILU0_Data<BS>>(pc->f);
    const uint32_t nb = pc->n / BS;
    if (!d || d->U_diag_ptr.size() != nb || d->L_row_ptr.size() != nb + 1) return -1;
    sizes[0] = d->L_row_ptr[nb];
    sizes[1] = d->U_row_ptr[nb];
    if (!Lrp) return 0;
    std::memcpy(Lrp, d->L_row_ptr.data(), 4 * (nb + 1));
    std::memcpy(Lci, d->L_col_idx.data(), 4 * sizes[0]);
    std::memcpy(Lv, d->L_values.data(), 8 * (size_t)sizes[0] * BS * BS);
    std::memcpy(Urp, d->U_row_ptr.data(), 4 * (nb + 1));
    std::memcpy(Uci, d->U_col_idx.data(), 4 * sizes[1]);
    std::memcpy(Uv, d->U_values.data(), 8 * (size_t)sizes[1] * BS * BS);
    std::memcpy(Udiag, d->U_diag_ptr.data(), 4 * nb);
    std::memcpy(inv_diag, d->inv_diag.data(), 8 * (size_t)nb * BS * BS);
    return 0;
}
}  // extern "C++"

int ref_blk_ilu0_export(void* p, int bs, uint32_t* sizes, uint32_t* Lrp, uint32_t* Lci, double* Lv,
                        uint32_t* Urp, uint32_t* Uci, double* Uv, uint32_t* Udiag, double* inv_diag)
{
    RefPC* pc = static_cast<RefPC*>(p);
    if (pc->kind != "blk_ilu0") return -1;
    if (bs == 1) return blk_ilu0_export_t<1>(pc, sizes, Lrp, Lci, Lv, Urp, Uci, Uv, Udiag, inv_diag);
    if (bs == 3) return blk_ilu0_export_t<3>(pc, sizes, Lrp, Lci, Lv, Urp, Uci, Uv, Udiag, inv_diag);
    return -1;
}

// Block SA-AMG hierarchy (BlockAMGLevel, blockMatrix.hpp:935-943).
// info(level=-1) returns the level count.  For level k, sizes =
// {nrows, nnzb(A), ncols(P), nnzb(P)} (P is empty on the coarsest level);
// arrays may be null to query sizes.
extern "C++" {
template <int BS>
static int blk_amg_export_t(RefPC* pc, int level, uint32_t* sizes, uint32_t* Arp, uint32_t* Aci, double* Av,
                            uint32_t* Prp, uint32_t* Pci, double* Pv, double* diag_inv)
{
    auto& lv = captured_data<std::vector<block::BlockAMGLevel<double, BS>>>(pc->f);
    if (!lv || lv->empty() || (*lv)[0].nrows * BS != pc->n) return -1;
    if (level < 0) return (int)lv->size();
    if (level >= (int)lv->size()) return -1;
    auto& L = (*lv)[level];
    sizes[0] = L.nrows;
    sizes[1] = (uint32_t)L.A.nnz_blocks();
    sizes[2] = L.P.block_cols();
    sizes[3] = (uint32_t)L.P.nnz_blocks();
    if (!Arp) return 0;
    blk_export_t(const_cast<block::BlockMatrix<double, BS>&>(L.A), Arp, Aci, Av);
    if (sizes[3] > 0) blk_export_t(const_cast<block::BlockMatrix<double, BS>&>(L.P), Prp, Pci, Pv);
    std::memcpy(diag_inv, L.diag_inv.data(), 8 * (size_t)L.nrows * BS * BS);
    return 0;
}
}  // extern "C++"

int ref_blk_amg_export(void* p, int bs, int level, uint32_t* sizes, uint32_t* Arp, uint32_t* Aci, double* Av,
                       uint32_t* Prp, uint32_t* Pci, double* Pv, double* diag_inv)
{
    RefPC* pc = static_cast<RefPC*>(p);
    if (pc->kind != "blk_amg") return -1;
    if (bs == 1) return blk_amg_export_t<1>(pc, level, sizes, Arp, Aci, Av, Prp, Pci, Pv, diag_inv);
    if (bs == 3) return blk_amg_export_t<3>(pc, level, sizes, Arp, Aci, Av, Prp, Pci, Pv, diag_inv);
    return -1;
}

// BlockMatrix::gmres (blockMatrix.hpp:688-866)
int ref_blk_gmres(void* p, const double* b, const char* precond, double tol, int maxit, int restart,
                  double* x, int* it, char* err, int errlen)
{
    RefBlk* B = static_cast<RefBlk*>(p);
    return guarded(err, errlen, [&] {
        std::tuple<std::vector<double>, int> res;
        size_t n;
        if (B->bs == 1)
        {
            auto& M = blk<1>(B);
            n = M.rows();
            res = block::BlockMatrix<double, 1>::gmres(M, std::vector<double>(b, b + n), precond, tol, maxit, restart);
        }
        else
        {
            auto& M = blk<3>(B);
            n = M.rows();
            res = block::BlockMatrix<double, 3>::gmres(M, std::vector<double>(b, b + n), precond, tol, maxit, restart);
        }
        std::memcpy(x, std::get<0>(res).data(), 8 * n);
        *it = std::get<1>(res);
    });
}

}  // extern "C"
