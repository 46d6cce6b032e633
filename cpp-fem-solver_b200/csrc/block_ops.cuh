// Small dense block helpers on the device: the arithmetic of
// blk_matmat_accum / blk_right_mul / blk_matvec / blk_invert
// (blockMatrix.hpp:37-103), operation for operation, so block factors match
// the reference bit for bit (the library builds with -fmad=false).
#pragma once
#include <cuda_runtime.h>

namespace b2s {

// C -= A*B
template <int BS>
__host__ __device__ __forceinline__ void blk_mma(const double* A, const double* B, double* C)
{
#pragma unroll
    for (int r = 0; r < BS; ++r)
#pragma unroll
        for (int c = 0; c < BS; ++c)
        {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < BS; ++k) s += A[r * BS + k] * B[k * BS + c];
            C[r * BS + c] -= s;
        }
}

// C := C*B
template <int BS>
__host__ __device__ __forceinline__ void blk_rmul(double* C, const double* B)
{
    double tmp[BS * BS];
#pragma unroll
    for (int r = 0; r < BS; ++r)
#pragma unroll
        for (int c = 0; c < BS; ++c)
        {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < BS; ++k) s += C[r * BS + k] * B[k * BS + c];
            tmp[r * BS + c] = s;
        }
#pragma unroll
    for (int t = 0; t < BS * BS; ++t) C[t] = tmp[t];
}

// y = M x
template <int BS>
__host__ __device__ __forceinline__ void blk_mv(const double* M, const double* x, double* y)
{
#pragma unroll
    for (int r = 0; r < BS; ++r)
    {
        double s = 0.0;
#pragma unroll
        for (int c = 0; c < BS; ++c) s += M[r * BS + c] * x[c];
        y[r] = s;
    }
}

// Minv = M^-1 by elimination with partial pivoting on [M | I]; false if a
// pivot is below 1e-300 (Minv then untouched).
template <int BS>
__host__ __device__ __forceinline__ bool blk_inv(const double* M, double* Minv)
{
    double aug[BS][2 * BS];
    for (int i = 0; i < BS; ++i)
        for (int j = 0; j < BS; ++j)
        {
            aug[i][j] = M[i * BS + j];
            aug[i][BS + j] = (i == j) ? 1.0 : 0.0;
        }
    for (int k = 0; k < BS; ++k)
    {
        int piv = k;
        for (int i = k + 1; i < BS; ++i)
            if (fabs(aug[i][k]) > fabs(aug[piv][k])) piv = i;
        if (fabs(aug[piv][k]) < 1e-300) return false;
        if (piv != k)
            for (int j = 0; j < 2 * BS; ++j)
            {
                const double t = aug[k][j];
                aug[k][j] = aug[piv][j];
                aug[piv][j] = t;
            }
        for (int i = k + 1; i < BS; ++i)
        {
            const double f = aug[i][k] / aug[k][k];
            for (int j = k; j < 2 * BS; ++j) aug[i][j] -= f * aug[k][j];
        }
    }
    for (int i = BS - 1; i >= 0; --i)
    {
        for (int j = i + 1; j < BS; ++j)
            for (int c = 0; c < BS; ++c) aug[i][BS + c] -= aug[i][j] * aug[j][BS + c];
        for (int c = 0; c < BS; ++c) aug[i][BS + c] /= aug[i][i];
    }
    for (int i = 0; i < BS; ++i)
        for (int j = 0; j < BS; ++j) Minv[i * BS + j] = aug[i][BS + j];
    return true;
}

// One row of BlockMatrix::matvec's block GEMV (blockMatrix.hpp:218-231): the
// reference's `omp simd` row sum, which GCC turns into (p0 + p2) + p1 for a
// 3-wide block; other widths sum in ascending order.
template <int BS>
__host__ __device__ __forceinline__ double blk_row_dot(const double* Brow, const double* x)
{
    if constexpr (BS == 3)
    {
        const double p0 = Brow[0] * x[0], p1 = Brow[1] * x[1], p2 = Brow[2] * x[2];
        return (p0 + p2) + p1;
    }
    else
    {
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < BS; ++c) acc += Brow[c] * x[c];
        return acc;
    }
}

}  // namespace b2s
