// Drop-in replacement for the sparse part of xuyinshen/cpp-FEM-solver's
// ode-solver/include/math/array.hpp (namespace sparse, class SMatrix,
// array.hpp:264-373), running every solver on a B200 through the b2s C ABI
// (include/b2s.h).
//
// Use: put include/b2s (this directory's parent) ahead of the reference's
// include directory, so `#include "math/array.hpp"` resolves here, and link
// libb2s.so.  The dense array::Matrix / Tensor types of the reference are not
// part of this header.
//
// Same surface as the reference:
//   constructors (COO uint32 vectors: sorted, duplicates merged, zeros
//   dropped; CSR vectors taken as given), rows/cols/nnz/values/row_ptr/
//   col_idx, transpose, operator*, dot, spmv, the make_*_preconditioner
//   factories, pcg / bicgstab / gmres (both overloads) / sor / sor_rb / amg
//   returning std::tuple<std::vector<double>, int> with the reference's
//   iteration counts, and the same exception types (std::invalid_argument for
//   argument and shape errors, std::runtime_error for numerical breakdown).
// Differences, by design:
//   - "amg" is smoothed aggregation (the reference's classical C/F AMG
//     produces NaN at the benchmark sizes), in the "amg" preconditioner string,
//     make_amg_preconditioner and the stand-alone amg solver alike.
//   - transpose and operator* run on the GPU; operator* keeps every product
//     column (the reference's drops a column that only one row of the product
//     touches, because its marker array is not reset between its passes).
//   - Extensions: pcg and bicgstab also accept a std::function preconditioner;
//     a preconditioner returned by a make_* factory here runs on the GPU even
//     when passed through std::function to gmres/pcg.
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../b2s.h"

namespace sparse
{
    using Precond = std::function<void(const std::vector<double>&, std::vector<double>&)>;

    namespace detail
    {
        // process-wide context on device B2S_DEVICE (default 0)
        b2s_ctx* context();
        [[noreturn]] void raise(b2s_status st, const std::string& where);
        inline void check(b2s_status st, const std::string& where)
        {
            if (st != B2S_OK) raise(st, where);
        }
        // a GPU preconditioner wrapped as a std::function target
        struct DevicePrecond
        {
            std::shared_ptr<b2s_pc> pc;
            std::shared_ptr<void> keep;  // keeps the matrix handle alive
            uint64_t n = 0;
            void operator()(const std::vector<double>& r, std::vector<double>& z) const;
        };
    }

    class SMatrix
    {
        private:
            uint32_t rows_ = 0, cols_ = 0;
            std::vector<uint32_t> row_ptr_;
            std::vector<uint32_t> col_idx_;
            std::vector<double> values_;
            mutable std::shared_ptr<b2s_csr> dev_;  // device copy, created on first use

        public:
            SMatrix();
            SMatrix(uint32_t rows, uint32_t cols, const std::vector<double>& values,
                    const std::vector<uint32_t>& rowlist, const std::vector<uint32_t>& collist);
            SMatrix(uint32_t rows, uint32_t cols, std::vector<uint32_t> row_ptr, std::vector<uint32_t> col_idx,
                    std::vector<double> values);

            static double dot(const std::vector<double>& a, const std::vector<double>& b);

            uint32_t rows() const;
            uint32_t cols() const;
            uint32_t nnz() const;

            const std::vector<double>& values() const;
            const std::vector<uint32_t>& row_ptr() const;
            const std::vector<uint32_t>& col_idx() const;

            SMatrix transpose() const;
            SMatrix operator*(const SMatrix& B) const;

            // the device-resident copy (b2s_csr), uploaded once and cached
            b2s_csr* device() const;

            static Precond make_diag_preconditioner(const SMatrix& A);
            static Precond make_ic0_preconditioner(const SMatrix& A);
            static Precond make_ilu0_preconditioner(const SMatrix& A);
            static Precond make_ssor_preconditioner(const SMatrix& A, double omega = 1.2);
            static Precond make_amg_preconditioner(const SMatrix& A);
            // extension: any b2s preconditioner kind with options
            static Precond make_preconditioner(const SMatrix& A, b2s_pc_kind kind, const b2s_pc_opts* opts = nullptr);

            static std::vector<double> spmv(const SMatrix& A, const std::vector<double>& x);

            static std::tuple<std::vector<double>, int> pcg(const SMatrix& A, const std::vector<double>& b,
                                                            const std::string& precond = "none", double tol = 1e-10,
                                                            int max_iter = 2000);
            static std::tuple<std::vector<double>, int> bicgstab(const SMatrix& A, const std::vector<double>& b,
                                                                 const std::string& precond, double tol = 1e-10,
                                                                 int max_iter = 2000);
            static std::tuple<std::vector<double>, int> gmres(const SMatrix& A, const std::vector<double>& b,
                                                              const std::string& precond, int restart,
                                                              double tol = 1e-10, int max_iter = 2000);
            static std::tuple<std::vector<double>, int> gmres(const SMatrix& A, const std::vector<double>& b,
                                                              const Precond& solveM, int restart, double tol = 1e-10,
                                                              int max_iter = 2000);
            // SOR, natural order and red-black (array.hpp:351-365)
            static std::tuple<std::vector<double>, int> sor(const SMatrix& A, const std::vector<double>& b,
                                                            double omega, double tol = 1e-10, int max_iter = 2000);
            static std::tuple<std::vector<double>, int> sor_rb(const SMatrix& A, const std::vector<double>& b,
                                                               double omega, double tol = 1e-10, int max_iter = 2000);
            // stand-alone AMG (array.hpp:367-372, array.cpp:4534-4563): from x = 0,
            // x += one V-cycle of the residual until ||b - A x|| / ||b|| < tol;
            // returns the index of the last residual check
            static std::tuple<std::vector<double>, int> amg(const SMatrix& A, const std::vector<double>& b,
                                                            double tol = 1e-10, int max_iter = 2000);
            // extensions with a functor preconditioner
            static std::tuple<std::vector<double>, int> pcg(const SMatrix& A, const std::vector<double>& b,
                                                            const Precond& solveM, double tol = 1e-10,
                                                            int max_iter = 2000);
            static std::tuple<std::vector<double>, int> bicgstab(const SMatrix& A, const std::vector<double>& b,
                                                                 const Precond& solveM, double tol = 1e-10,
                                                                 int max_iter = 2000);
    };

    // Runs `method` on a device operator with a string or functor
    // preconditioner; shared by SMatrix and block::BlockMatrix.
    namespace detail
    {
        std::tuple<std::vector<double>, int> solve_csr(const SMatrix& A, const std::vector<double>& b, b2s_method m,
                                                       const std::string* name, const Precond* fn, int restart,
                                                       double tol, int max_iter);
        std::tuple<std::vector<double>, int> solve_op(b2s_csr* csr, b2s_baij* baij, uint64_t n,
                                                      const std::vector<double>& b, b2s_method m, b2s_pc* pc,
                                                      const Precond* fn, int restart, double tol, int max_iter);
    }
}
