// sparse::SMatrix drop-in (include/b2s/math/array.hpp) over the b2s C ABI.
//   constructors / accessors: array.cpp:2072-2198; transpose / operator*
//   (on the device): array.cpp:2201-2447
//   factories: array.cpp:2450-3398; solvers: array.cpp:3445-4533
// Host-side containers keep the reference's CSR semantics; every solve runs
// on the GPU against a device copy uploaded once per matrix.
#include "math/array.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <tuple>

namespace sparse
{
    namespace detail
    {
        b2s_ctx* context()
        {
            static std::once_flag once;
            static b2s_ctx* ctx = nullptr;
            static b2s_status st = B2S_OK;
            std::call_once(once, [] {
                const char* d = std::getenv("B2S_DEVICE");
                st = b2s_ctx_create(d ? std::atoi(d) : 0, &ctx);
            });
            if (!ctx) throw std::runtime_error(std::string("b2s: no GPU context (") + b2s_status_name(st) + ")");
            return ctx;
        }

        void raise(b2s_status st, const std::string& where)
        {
            const std::string msg = where + ": " + b2s_status_name(st) + ": " + b2s_last_error(context());
            if (st == B2S_INVALID_ARG || st == B2S_SHAPE) throw std::invalid_argument(msg);
            throw std::runtime_error(msg);
        }

        void DevicePrecond::operator()(const std::vector<double>& r, std::vector<double>& z) const
        {
            z.resize(r.size());
            check(b2s_pc_apply(context(), pc.get(), r.data(), z.data()), "preconditioner apply");
        }

        static int host_trampoline(void* user, const double* r, double* z, uint64_t n)
        {
            try
            {
                const Precond& f = *static_cast<const Precond*>(user);
                std::vector<double> rv(r, r + n), zv;
                f(rv, zv);
                if (zv.size() != n) return 2;
                std::copy(zv.begin(), zv.end(), z);
                return 0;
            }
            catch (...)
            {
                return 1;
            }
        }

        std::tuple<std::vector<double>, int> solve_op(b2s_csr* csr, b2s_baij* baij, uint64_t n,
                                                      const std::vector<double>& b, b2s_method m, b2s_pc* pc,
                                                      const Precond* fn, int restart, double tol, int max_iter)
        {
            b2s_ctx* ctx = context();
            std::shared_ptr<b2s_pc> hostpc;
            if (!pc && fn && *fn)
            {
                if (const DevicePrecond* d = fn->target<DevicePrecond>())
                    pc = d->pc.get();
                else
                {
                    b2s_pc* h = nullptr;
                    check(b2s_pc_create_host(ctx, n, host_trampoline, const_cast<Precond*>(fn), &h), "preconditioner");
                    hostpc.reset(h, [](b2s_pc* p) { b2s_pc_destroy(p); });
                    pc = h;
                }
            }
            b2s_solve_opts o;
            b2s_solve_opts_default(&o);
            o.tol = tol;
            o.maxit = max_iter;
            o.restart = restart;
            std::vector<double> x(n, 0.0);
            b2s_stats st;
            const b2s_status s = csr ? b2s_solve(ctx, csr, pc, m, &o, b.data(), x.data(), &st)
                                     : b2s_solve_baij(ctx, baij, pc, m, &o, b.data(), x.data(), &st);
            if (s != B2S_OK) raise(s, "solve");
            if (st.status == B2S_DIVERGED) return {x, max_iter - 1};  // the reference runs on with NaN to max_iter
            return {x, st.it};
        }

        std::tuple<std::vector<double>, int> solve_csr(const SMatrix& A, const std::vector<double>& b, b2s_method m,
                                                       const std::string* name, const Precond* fn, int restart,
                                                       double tol, int max_iter)
        {
            if (A.rows() != A.cols()) throw std::invalid_argument("solver needs a square matrix");
            if (A.cols() != b.size()) throw std::invalid_argument("matrix columns differ from vector length");
            const uint32_t n = A.rows();
            double nb = 0.0;
            for (double v : b) nb += v * v;
            const double normb = std::sqrt(nb);
            if (normb < 1e-300) return {std::vector<double>(n, 0.0), 0};
            if (m != B2S_GMRES && 1.0 < tol) return {std::vector<double>(n, 0.0), 0};
            std::shared_ptr<b2s_pc> pc;
            if (name)
            {
                b2s_pc_kind kind;
                if (b2s_pc_kind_from_name(m, name->c_str(), &kind) != B2S_OK)
                    throw std::invalid_argument("unknown preconditioner type: " + *name);
                if (kind != B2S_PC_NONE)
                {
                    b2s_pc* h = nullptr;
                    check(b2s_pc_create(context(), A.device(), kind, nullptr, &h), "preconditioner");
                    pc.reset(h, [](b2s_pc* p) { b2s_pc_destroy(p); });
                }
            }
            return solve_op(A.device(), nullptr, n, b, m, pc.get(), fn, restart, tol, max_iter);
        }
    }

    SMatrix::SMatrix() : rows_(0), cols_(0), row_ptr_(1, 0) {}

    SMatrix::SMatrix(uint32_t rows, uint32_t cols, const std::vector<double>& values,
                     const std::vector<uint32_t>& rowlist, const std::vector<uint32_t>& collist)
        : rows_(rows), cols_(cols)
    {
        if (values.size() != rowlist.size() || values.size() != collist.size())
            throw std::invalid_argument("COO input error: values, rowlist, collist differ in length");
        struct E
        {
            uint32_t i, j;
            double v;
            size_t k;
        };
        std::vector<E> e;
        e.reserve(values.size());
        for (size_t k = 0; k < values.size(); ++k)
        {
            if (rowlist[k] >= rows || collist[k] >= cols) throw std::out_of_range("COO input error: index out of range");
            if (values[k] != 0.0) e.push_back({rowlist[k], collist[k], values[k], k});
        }
        std::sort(e.begin(), e.end(), [](const E& a, const E& b) {
            return a.i != b.i ? a.i < b.i : a.j != b.j ? a.j < b.j : a.k < b.k;
        });
        std::vector<E> m;
        m.reserve(e.size());
        for (const E& x : e)
        {
            if (!m.empty() && m.back().i == x.i && m.back().j == x.j)
                m.back().v += x.v;
            else
                m.push_back(x);
        }
        row_ptr_.assign(rows + 1, 0);
        for (const E& x : m)
            if (x.v != 0.0) row_ptr_[x.i + 1]++;
        for (uint32_t i = 0; i < rows; ++i) row_ptr_[i + 1] += row_ptr_[i];
        for (const E& x : m)
            if (x.v != 0.0)
            {
                col_idx_.push_back(x.j);
                values_.push_back(x.v);
            }
    }

    SMatrix::SMatrix(uint32_t rows, uint32_t cols, std::vector<uint32_t> row_ptr, std::vector<uint32_t> col_idx,
                     std::vector<double> values)
        : rows_(rows), cols_(cols), row_ptr_(std::move(row_ptr)), col_idx_(std::move(col_idx)),
          values_(std::move(values))
    {
    }

    uint32_t SMatrix::rows() const { return rows_; }
    uint32_t SMatrix::cols() const { return cols_; }
    uint32_t SMatrix::nnz() const { return (uint32_t)values_.size(); }
    const std::vector<double>& SMatrix::values() const { return values_; }
    const std::vector<uint32_t>& SMatrix::row_ptr() const { return row_ptr_; }
    const std::vector<uint32_t>& SMatrix::col_idx() const { return col_idx_; }

    b2s_csr* SMatrix::device() const
    {
        if (!dev_)
        {
            b2s_csr* h = nullptr;
            detail::check(b2s_csr_create(detail::context(), rows_, cols_, row_ptr_.data(), col_idx_.data(),
                                         values_.data(), &h),
                          "SMatrix upload");
            dev_.reset(h, [](b2s_csr* p) { b2s_csr_destroy(p); });
        }
        return dev_.get();
    }

    namespace detail
    {
        // a device-built CSR handle back into host vectors
        static SMatrix from_device(b2s_csr* h, uint32_t rows, uint32_t cols)
        {
            std::shared_ptr<b2s_csr> keep(h, [](b2s_csr* p) { b2s_csr_destroy(p); });
            uint32_t n = 0, m = 0, nnz = 0;
            check(b2s_csr_info(h, &n, &m, &nnz), "matrix info");
            std::vector<uint32_t> rp((size_t)rows + 1), ci(nnz);
            std::vector<double> vv(nnz);
            check(b2s_csr_export(context(), h, rp.data(), ci.data(), vv.data()), "matrix download");
            return SMatrix(rows, cols, std::move(rp), std::move(ci), std::move(vv));
        }
    }

    SMatrix SMatrix::transpose() const
    {
        b2s_csr* t = nullptr;
        detail::check(b2s_csr_transpose(detail::context(), device(), &t), "transpose");
        return detail::from_device(t, cols_, rows_);
    }

    SMatrix SMatrix::operator*(const SMatrix& B) const
    {
        if (cols_ != B.rows_) throw std::invalid_argument("matrix product: columns of A differ from rows of B");
        b2s_csr* c = nullptr;
        detail::check(b2s_csr_matmul(detail::context(), device(), B.device(), &c), "matrix product");
        return detail::from_device(c, rows_, B.cols_);
    }

    double SMatrix::dot(const std::vector<double>& a, const std::vector<double>& b)
    {
        if (a.size() != b.size()) throw std::invalid_argument("dot: vector lengths differ");
        double out = 0.0;
        detail::check(b2s_dot(detail::context(), a.size(), a.data(), b.data(), &out), "dot");
        return out;
    }

    std::vector<double> SMatrix::spmv(const SMatrix& A, const std::vector<double>& x)
    {
        if (A.cols_ != x.size()) throw std::invalid_argument("spmv: matrix columns differ from vector length");
        std::vector<double> y(A.rows_, 0.0);
        detail::check(b2s_spmv(detail::context(), A.device(), x.data(), y.data()), "spmv");
        return y;
    }

    Precond SMatrix::make_preconditioner(const SMatrix& A, b2s_pc_kind kind, const b2s_pc_opts* opts)
    {
        if (A.rows() != A.cols()) throw std::invalid_argument("preconditioner needs a square matrix");
        b2s_pc* h = nullptr;
        detail::check(b2s_pc_create(detail::context(), A.device(), kind, opts, &h), "preconditioner");
        detail::DevicePrecond d;
        d.pc.reset(h, [](b2s_pc* p) { b2s_pc_destroy(p); });
        d.n = A.rows();
        return Precond(d);
    }

    Precond SMatrix::make_diag_preconditioner(const SMatrix& A) { return make_preconditioner(A, B2S_PC_DIAG); }
    Precond SMatrix::make_ic0_preconditioner(const SMatrix& A) { return make_preconditioner(A, B2S_PC_IC0); }
    Precond SMatrix::make_ilu0_preconditioner(const SMatrix& A) { return make_preconditioner(A, B2S_PC_ILU0); }
    Precond SMatrix::make_amg_preconditioner(const SMatrix& A) { return make_preconditioner(A, B2S_PC_SA_AMG); }
    Precond SMatrix::make_ssor_preconditioner(const SMatrix& A, double omega)
    {
        if (!(omega > 0.0 && omega < 2.0))
            throw std::invalid_argument("SSOR: relaxation factor must satisfy 0 < omega < 2");
        b2s_pc_opts o;
        b2s_pc_opts_default(&o);
        o.omega = omega;
        return make_preconditioner(A, B2S_PC_SSOR, &o);
    }

    std::tuple<std::vector<double>, int> SMatrix::pcg(const SMatrix& A, const std::vector<double>& b,
                                                      const std::string& precond, double tol, int max_iter)
    {
        return detail::solve_csr(A, b, B2S_PCG, &precond, nullptr, 30, tol, max_iter);
    }

    std::tuple<std::vector<double>, int> SMatrix::bicgstab(const SMatrix& A, const std::vector<double>& b,
                                                           const std::string& precond, double tol, int max_iter)
    {
        return detail::solve_csr(A, b, B2S_BICGSTAB, &precond, nullptr, 30, tol, max_iter);
    }

    std::tuple<std::vector<double>, int> SMatrix::gmres(const SMatrix& A, const std::vector<double>& b,
                                                        const std::string& precond, int restart, double tol,
                                                        int max_iter)
    {
        return detail::solve_csr(A, b, B2S_GMRES, &precond, nullptr, restart, tol, max_iter);
    }

    std::tuple<std::vector<double>, int> SMatrix::gmres(const SMatrix& A, const std::vector<double>& b,
                                                        const Precond& solveM, int restart, double tol, int max_iter)
    {
        return detail::solve_csr(A, b, B2S_GMRES, nullptr, &solveM, restart, tol, max_iter);
    }

    std::tuple<std::vector<double>, int> SMatrix::pcg(const SMatrix& A, const std::vector<double>& b,
                                                      const Precond& solveM, double tol, int max_iter)
    {
        return detail::solve_csr(A, b, B2S_PCG, nullptr, &solveM, 30, tol, max_iter);
    }

    std::tuple<std::vector<double>, int> SMatrix::bicgstab(const SMatrix& A, const std::vector<double>& b,
                                                           const Precond& solveM, double tol, int max_iter)
    {
        return detail::solve_csr(A, b, B2S_BICGSTAB, nullptr, &solveM, 30, tol, max_iter);
    }

    namespace detail
    {
        std::tuple<std::vector<double>, int> sor_csr(const SMatrix& A, const std::vector<double>& b, int red_black,
                                                     double omega, double tol, int max_iter)
        {
            if (A.rows() != A.cols())
                throw std::invalid_argument(red_black ? "red-black SOR needs a square matrix" : "SOR needs a square matrix");
            if (A.cols() != b.size()) throw std::invalid_argument("SOR: matrix columns differ from vector length");
            std::vector<double> x(A.rows(), 0.0);
            b2s_stats st;
            check(b2s_sor(context(), A.device(), red_black, omega, tol, max_iter, b.data(), x.data(), &st),
                  red_black ? "red-black SOR" : "SOR");
            return {x, st.it};
        }
    }

    std::tuple<std::vector<double>, int> SMatrix::sor(const SMatrix& A, const std::vector<double>& b, double omega,
                                                      double tol, int max_iter)
    {
        return detail::sor_csr(A, b, 0, omega, tol, max_iter);
    }

    std::tuple<std::vector<double>, int> SMatrix::sor_rb(const SMatrix& A, const std::vector<double>& b, double omega,
                                                         double tol, int max_iter)
    {
        return detail::sor_csr(A, b, 1, omega, tol, max_iter);
    }

    std::tuple<std::vector<double>, int> SMatrix::amg(const SMatrix& A, const std::vector<double>& b, double tol,
                                                      int max_iter)
    {
        if (A.rows() != A.cols()) throw std::invalid_argument("AMG needs a square matrix");
        if (A.cols() != b.size()) throw std::invalid_argument("AMG: matrix columns differ from vector length");
        const uint32_t n = A.rows();
        double nb = 0.0;
        for (double v : b) nb += v * v;
        if (std::sqrt(nb) < 1e-300) return {std::vector<double>(n, 0.0), 0};
        b2s_pc* h = nullptr;
        detail::check(b2s_pc_create(detail::context(), A.device(), B2S_PC_SA_AMG, nullptr, &h), "AMG setup");
        std::shared_ptr<b2s_pc> pc(h, [](b2s_pc* p) { b2s_pc_destroy(p); });
        return detail::solve_op(A.device(), nullptr, n, b, B2S_STATIONARY, pc.get(), nullptr, 30, tol, max_iter);
    }
}
