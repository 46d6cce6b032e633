// Drop-in replacement for xuyinshen/cpp-FEM-solver's
// ode-solver/include/math/blockMatrix.hpp (namespace block), running on a
// B200 through the b2s C ABI.  Same call surface: BlockMatrix<T,BS>
// (blockMatrix.hpp:139-452) with matvec / transpose / condense / set_halo /
// distributed_matvec / gmres(A, b, precond, tol, max_iter, restart), the free
// factories make_block_ilu0_preconditioner, make_block_amg_preconditioner and
// make_schur_preconditioner (blockMatrix.hpp:455-685, 1051-1179), and
// SaddlePointSystem.
//
// One device holds the whole matrix: set_halo is accepted and recorded but no
// rows are ghosts (owned_rows() == block_rows()), and distributed_matvec is
// matvec -- the reference's own behaviour without MPI (blockMatrix.hpp:439-441).
// Only T = double is supported; BS in {1, 2, 3, 4}.
// Extension: BlockMatrix::pcg (block conjugate gradients with the same
// convention as SMatrix::pcg).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "math/array.hpp"

using namespace sparse;

namespace block
{
    template <typename T, int BS>
    class BlockMatrix
    {
        static_assert(std::is_same<T, double>::value, "b2s BlockMatrix supports T = double");
        static_assert(BS >= 1 && BS <= 4, "b2s BlockMatrix supports 1 <= BS <= 4");

        private:
            uint32_t nbr_ = 0, nbc_ = 0;
            std::vector<uint32_t> row_ptr_{0};
            std::vector<uint32_t> col_idx_;
            std::vector<T> values_;
            std::vector<uint32_t> diag_ptr_;
            // halo description (recorded; one device needs no exchange)
            std::vector<int> recv_procs_, recv_cnts_, send_procs_, send_cnts_;
            std::vector<uint32_t> recv_global_, send_local_;
            mutable std::shared_ptr<b2s_baij> dev_;

        public:
            static constexpr int kBlock = BS;
            static constexpr int kBlockVals = BS * BS;

            BlockMatrix() = default;
            BlockMatrix(uint32_t nbr, uint32_t nbc, std::vector<uint32_t> row_ptr, std::vector<uint32_t> col_idx,
                        std::vector<T> values)
                : nbr_(nbr), nbc_(nbc), row_ptr_(std::move(row_ptr)), col_idx_(std::move(col_idx)),
                  values_(std::move(values))
            {
                cache_diag();
            }

            uint32_t block_rows() const { return nbr_; }
            uint32_t block_cols() const { return nbc_; }
            uint32_t rows() const { return nbr_ * BS; }
            uint32_t cols() const { return nbc_ * BS; }
            size_t nnz_blocks() const { return col_idx_.size(); }
            size_t nnz() const { return col_idx_.size() * (size_t)kBlockVals; }
            const std::vector<uint32_t>& block_row_ptr() const { return row_ptr_; }
            const std::vector<uint32_t>& block_col_idx() const { return col_idx_; }
            const std::vector<T>& values() const { return values_; }
            const T* block(uint32_t p) const { return &values_[(size_t)p * kBlockVals]; }
            const T* diag_block(uint32_t bi) const { return &values_[(size_t)diag_ptr_[bi] * kBlockVals]; }

            void cache_diag()
            {
                diag_ptr_.assign(nbr_, UINT32_MAX);
                for (uint32_t bi = 0; bi < nbr_; ++bi)
                    for (uint32_t p = row_ptr_[bi]; p < row_ptr_[bi + 1]; ++p)
                        if (col_idx_[p] == bi)
                        {
                            diag_ptr_[bi] = p;
                            break;
                        }
            }

            // device-resident copy, uploaded once
            b2s_baij* device() const
            {
                if (!dev_)
                {
                    b2s_baij* h = nullptr;
                    sparse::detail::check(b2s_baij_create(sparse::detail::context(), BS, nbr_, nbc_, row_ptr_.data(),
                                                          col_idx_.data(), values_.data(), &h),
                                          "BlockMatrix upload");
                    dev_.reset(h, [](b2s_baij* p) { b2s_baij_destroy(p); });
                }
                return dev_.get();
            }

            void matvec(const std::vector<T>& x, std::vector<T>& y) const
            {
                if (x.size() != cols()) throw std::invalid_argument("BlockMatrix::matvec: size mismatch");
                y.assign(rows(), T(0));
                sparse::detail::check(b2s_baij_matvec(sparse::detail::context(), device(), x.data(), y.data()),
                                      "BlockMatrix::matvec");
            }

            BlockMatrix<T, BS> transpose() const
            {
                std::vector<uint32_t> trp(nbc_ + 1, 0);
                for (size_t p = 0; p < col_idx_.size(); ++p) trp[col_idx_[p] + 1]++;
                for (uint32_t i = 0; i < nbc_; ++i) trp[i + 1] += trp[i];
                std::vector<uint32_t> tci(col_idx_.size()), off(trp.begin(), trp.end() - 1);
                std::vector<T> tv(values_.size());
                for (uint32_t i = 0; i < nbr_; ++i)
                    for (uint32_t p = row_ptr_[i]; p < row_ptr_[i + 1]; ++p)
                    {
                        const uint32_t q = off[col_idx_[p]]++;
                        tci[q] = i;
                        for (int r = 0; r < BS; ++r)
                            for (int c = 0; c < BS; ++c)
                                tv[(size_t)q * kBlockVals + r * BS + c] = values_[(size_t)p * kBlockVals + c * BS + r];
                    }
                return BlockMatrix(nbc_, nbr_, std::move(trp), std::move(tci), std::move(tv));
            }

            static BlockMatrix<T, BS> condense(const SMatrix& A, uint32_t nbr, uint32_t nbc)
            {
                const auto& Ap = A.row_ptr();
                const auto& Ac = A.col_idx();
                const auto& Av = A.values();
                std::vector<uint32_t> rp(nbr + 1, 0), ci;
                std::vector<std::vector<uint32_t>> cols(nbr);
                for (uint32_t bi = 0; bi < nbr; ++bi)
                {
                    auto& out = cols[bi];
                    for (uint32_t i = bi * BS; i < (bi + 1) * BS; ++i)
                        for (uint32_t p = Ap[i]; p < Ap[i + 1]; ++p) out.push_back(Ac[p] / BS);
                    std::sort(out.begin(), out.end());
                    out.erase(std::unique(out.begin(), out.end()), out.end());
                    rp[bi + 1] = rp[bi] + (uint32_t)out.size();
                }
                ci.resize(rp[nbr]);
                std::vector<T> vv((size_t)rp[nbr] * kBlockVals, T(0));
                for (uint32_t bi = 0; bi < nbr; ++bi)
                {
                    std::copy(cols[bi].begin(), cols[bi].end(), ci.begin() + rp[bi]);
                    for (uint32_t i = bi * BS; i < (bi + 1) * BS; ++i)
                        for (uint32_t p = Ap[i]; p < Ap[i + 1]; ++p)
                        {
                            const uint32_t bj = Ac[p] / BS, c = Ac[p] % BS;
                            const auto it = std::lower_bound(cols[bi].begin(), cols[bi].end(), bj);
                            const uint32_t boff = rp[bi] + (uint32_t)(it - cols[bi].begin());
                            vv[(size_t)boff * kBlockVals + (size_t)(i % BS) * BS + c] += Av[p];
                        }
                }
                return BlockMatrix(nbr, nbc, std::move(rp), std::move(ci), std::move(vv));
            }

            void set_halo(std::vector<int> recv_procs, std::vector<int> recv_cnts, std::vector<uint32_t> recv_global,
                          std::vector<int> send_procs, std::vector<int> send_cnts, std::vector<uint32_t> send_local,
                          uint32_t owned_global_start = 0)
            {
                (void)owned_global_start;
                recv_procs_ = std::move(recv_procs);
                recv_cnts_ = std::move(recv_cnts);
                recv_global_ = std::move(recv_global);
                send_procs_ = std::move(send_procs);
                send_cnts_ = std::move(send_cnts);
                send_local_ = std::move(send_local);
            }
            uint32_t owned_rows() const { return nbr_; }

            void distributed_matvec(const std::vector<T>& x_owned, std::vector<T>& y_owned) const
            {
                matvec(x_owned, y_owned);
            }

            static std::tuple<std::vector<T>, int> gmres(const BlockMatrix& A, const std::vector<T>& b,
                                                         const std::string& precond, double tol, int max_iter,
                                                         int restart)
            {
                b2s_pc_kind kind;
                double nb = 0;
                for (double v : b) nb += v * v;
                if (std::sqrt(nb) < 1e-300) return {std::vector<T>(b.size(), T(0)), 0};
                if (b2s_pc_kind_from_name(B2S_BLOCK_GMRES, precond.c_str(), &kind) != B2S_OK)
                    throw std::invalid_argument("BlockMatrix::gmres unknown preconditioner type: " + precond);
                std::shared_ptr<b2s_pc> pc;
                if (kind != B2S_PC_NONE)
                {
                    b2s_pc* h = nullptr;
                    sparse::detail::check(b2s_pc_create_baij(sparse::detail::context(), A.device(), kind, nullptr, &h),
                                          "BlockMatrix::gmres preconditioner");
                    pc.reset(h, [](b2s_pc* p) { b2s_pc_destroy(p); });
                }
                return sparse::detail::solve_op(nullptr, A.device(), A.rows(), b, B2S_GMRES, pc.get(), nullptr,
                                                restart, tol, max_iter);
            }

            // extension: block CG with a functor preconditioner (a factory
            // result from this header runs on the GPU)
            static std::tuple<std::vector<T>, int> pcg(const BlockMatrix& A, const std::vector<T>& b,
                                                       const sparse::Precond& solveM, double tol = 1e-10,
                                                       int max_iter = 2000)
            {
                return sparse::detail::solve_op(nullptr, A.device(), A.rows(), b, B2S_PCG, nullptr, &solveM, 30, tol,
                                                max_iter);
            }
    };

    template <typename T, int BS>
    sparse::Precond make_block_preconditioner_(const BlockMatrix<T, BS>& A, b2s_pc_kind kind, const char* what)
    {
        if (A.block_rows() != A.block_cols()) throw std::invalid_argument(std::string(what) + " needs a square block matrix");
        b2s_pc* h = nullptr;
        sparse::detail::check(b2s_pc_create_baij(sparse::detail::context(), A.device(), kind, nullptr, &h), what);
        sparse::detail::DevicePrecond d;
        d.pc.reset(h, [](b2s_pc* p) { b2s_pc_destroy(p); });
        d.n = A.rows();
        return sparse::Precond(d);
    }

    template <typename T, int BS>
    sparse::Precond make_block_ilu0_preconditioner(const BlockMatrix<T, BS>& A)
    {
        return make_block_preconditioner_(A, B2S_PC_BILU0, "Block-ILU(0)");
    }

    template <typename T, int BS>
    sparse::Precond make_block_amg_preconditioner(const BlockMatrix<T, BS>& A)
    {
        return make_block_preconditioner_(A, B2S_PC_BSA_AMG, "Block AMG");
    }

    // blockMatrix.hpp:628-634
    struct SaddlePointSystem
    {
        size_t n_vel;
        size_t n_pres;
        std::function<void(const std::vector<double>&, std::vector<double>&)> spmv_A;
        std::function<void(const std::vector<double>&, std::vector<double>&)> spmv_B;
        std::function<void(const std::vector<double>&, std::vector<double>&)> spmv_Bt;
    };

    // Block-triangular saddle-point preconditioner (blockMatrix.hpp:637-685):
    //   w_u = A^-1 r_u;  z_p = S^-1 (B w_u - r_p);  z_u = A^-1 (r_u - B^T z_p)
    inline sparse::Precond make_schur_preconditioner(const SaddlePointSystem& sys, sparse::Precond A_precond,
                                                     sparse::Precond S_precond)
    {
        struct Work
        {
            std::vector<double> r_u, r_p, w_u, w_p, r_p_mod, z_p, w_bt, r_u_mod, z_u;
        };
        auto work = std::make_shared<Work>();
        return [sys, A_precond, S_precond, work](const std::vector<double>& r, std::vector<double>& z) {
            Work& k = *work;
            const size_t nv = sys.n_vel, np = sys.n_pres;
            k.r_u.assign(r.begin(), r.begin() + nv);
            k.r_p.assign(r.begin() + nv, r.begin() + nv + np);
            A_precond(k.r_u, k.w_u);
            sys.spmv_B(k.w_u, k.w_p);
            k.r_p_mod.resize(np);
            for (size_t i = 0; i < np; ++i) k.r_p_mod[i] = k.w_p[i] - k.r_p[i];
            S_precond(k.r_p_mod, k.z_p);
            sys.spmv_Bt(k.z_p, k.w_bt);
            k.r_u_mod.resize(nv);
            for (size_t i = 0; i < nv; ++i) k.r_u_mod[i] = k.r_u[i] - k.w_bt[i];
            A_precond(k.r_u_mod, k.z_u);
            z.resize(nv + np);
            std::copy(k.z_u.begin(), k.z_u.end(), z.begin());
            std::copy(k.z_p.begin(), k.z_p.end(), z.begin() + nv);
        };
    }

    // Extension: the same composition resident on the device, given B and
    // B^T as matrices.  A_precond must come from this library's factories
    // (make_*_preconditioner); an empty S_precond is the identity.  No step of
    // an apply leaves the GPU (b2s_pc_create_schur), and the result equals the
    // composition above bit for bit.
    inline sparse::Precond make_schur_preconditioner(const SaddlePointSystem& sys, const sparse::SMatrix& B,
                                                     const sparse::SMatrix& Bt, const sparse::Precond& A_precond,
                                                     const sparse::Precond& S_precond = sparse::Precond())
    {
        using sparse::detail::DevicePrecond;
        const DevicePrecond* Ad = A_precond.target<DevicePrecond>();
        const DevicePrecond* Sd = S_precond ? S_precond.target<DevicePrecond>() : nullptr;
        if (!Ad || (S_precond && !Sd))
            throw std::invalid_argument("device Schur preconditioner: A_precond and S_precond must be device "
                                        "preconditioners from the make_*_preconditioner factories");
        b2s_pc* h = nullptr;
        sparse::detail::check(b2s_pc_create_schur(sparse::detail::context(), sys.n_vel, sys.n_pres, B.device(),
                                                  Bt.device(), Ad->pc.get(), Sd ? Sd->pc.get() : nullptr, &h),
                              "Schur preconditioner");
        DevicePrecond d;
        d.pc.reset(h, [](b2s_pc* p) { b2s_pc_destroy(p); });
        d.n = sys.n_vel + sys.n_pres;
        // the parts stay alive as long as the composition
        d.keep = std::make_shared<std::tuple<sparse::Precond, sparse::Precond, sparse::SMatrix, sparse::SMatrix>>(
            A_precond, S_precond, B, Bt);
        return sparse::Precond(d);
    }

    // Extension: z = alpha M^-1 r for a device preconditioner M (the scaled
    // pressure AMG of the reference's 3-D Stokes test), on the device.
    inline sparse::Precond make_scaled_preconditioner(const sparse::Precond& M, double alpha)
    {
        using sparse::detail::DevicePrecond;
        const DevicePrecond* Md = M.target<DevicePrecond>();
        if (!Md) throw std::invalid_argument("scaled preconditioner: M must be a device preconditioner");
        b2s_pc* h = nullptr;
        sparse::detail::check(b2s_pc_create_scaled(sparse::detail::context(), Md->pc.get(), alpha, &h),
                              "scaled preconditioner");
        DevicePrecond d;
        d.pc.reset(h, [](b2s_pc* p) { b2s_pc_destroy(p); });
        d.n = Md->n;
        d.keep = std::make_shared<sparse::Precond>(M);
        return sparse::Precond(d);
    }
}
