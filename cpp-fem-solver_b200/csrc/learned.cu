// Learned IC(0): a message-passing network over the graph of A that corrects
// the IC(0) factor values on the unchanged pattern (no counterpart in the
// reference; its IC(0) is make_ic0_preconditioner, array.cpp:2522-2732).
//
// Network (26,502 parameters, FP32 master copy, BF16 copy used in the
// forward pass, FP32 accumulation everywhere):
//   node features f_i (8): scale-free statistics of row i -- mean / min / max
//     of log(|a_ij| / a_ii) over the neighbours, log of the off-diagonal row
//     sum over a_ii, degree / 4, and log(a_ii / mean_j a_jj)
//   edge features e_ij (4): log(|a_ij|/a_ii), log(|a_ij|/a_jj),
//     log(a_jj/a_ii), +1 for j < i / -1 for j > i
//   h0 = relu(W_in f + b_in)                                   (64)
//   3 layers:  [s | m] = h [W_s | W_m]^T ;  g_ij = sigmoid(W_g e_ij + b_g)
//              h' = relu(s_i + b + (1/deg_i) sum_j g_ij * m_j) + h
//   head:      c_ij = u.h_i + v.h_j + w.e_ij + b_o   (j < i)
//              c_ii = d.h_i + b_d
//   L~_ij = L_ij exp(0.5 tanh c_ij); the diagonal is kept >= 1e-3 sqrt(a_ii)
//   (positive-pivot guard), so L~ L~^T stays SPD.
// The output layer starts at zero: an untrained network returns IC(0).
//
// Training losses on probe vectors w (half standard normal, half smoothed by
// ten 2/3-Jacobi sweeps, the modes IC(0) resolves worst):
//   preconditioned residual (B2S_LOSS_PRECOND, the default):
//     loss = mean_w ||w - M^{-1} A w||^2 / ||w||^2,   M = L~ L~^T
//     y = L~^{-1} A w, z = L~^{-T} y, g = -2 (w - z) / (P ||w||^2),
//     a = L~^{-1} g, b = L~^{-T} a:  dloss/dL~_ij = -(z_i a_j + b_i y_j)
//     (four triangular solves per probe, on the FP64 chunk schedules)
//   factorisation residual (B2S_LOSS_FACTOR):
//     loss = mean_w ||(L~ L~^T - A) w||^2 / ||A w||^2
//     whose gradient needs only products with L~ and L~^T:
//     dloss/dL~_ij = 2 (v_i u_j + w_i q_j) / ||Aw||^2,  u = L~^T w,
//     v = L~ u - A w,  q = L~^T v.
//   preconditioned residual through the deployed sweep apply
//   (B2S_LOSS_SWEEPS): the same loss with M^-1 = F^T F, F = k Jacobi sweeps
//   of L~ (y_0 = D^-1 r, y_s = D^-1 (r - N y_{s-1}); D, N the diagonal and
//   strict part of L~) and F^T the k sweeps of L~^T -- the operator the
//   B2S_TRSV_JACOBI preconditioner applies.  Its gradient runs the adjoint
//   recursions back through both sweep sequences (every sweep state kept):
//   with h = D^-1 gbar_s, dL~_ii -= h_i y_s[i], dN_ij -= h_i y_{s-1}[j] and
//   gbar_{s-1} = -N^T h (lower) or -N h (upper), the upper sweeps' h summed
//   into the adjoint of their right-hand side.
// All parameter gradients are reduced in a fixed order (per-CTA partials,
// then one ordered sum), so training is deterministic.
#include <cuda_bf16.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <dlfcn.h>

#include <fstream>

#include "b2s_internal.cuh"
#include "tc_linear.cuh"

struct b2s_learner;

namespace b2s {

namespace {

constexpr int H = 64, FIN = 8, FE = 4, NL = 3;
constexpr float kScale = 0.5f;

// parameter layout
constexpr int OFF_WIN = 0, OFF_BIN = OFF_WIN + H * FIN;
constexpr int LAYER0 = OFF_BIN + H;
constexpr int L_WS = 0, L_WM = H * H, L_WG = 2 * H * H, L_BG = L_WG + H * FE, L_B = L_BG + H, L_SIZE = L_B + H;
constexpr int OFF_OUT = LAYER0 + NL * L_SIZE;
constexpr int O_U = 0, O_V = H, O_W = 2 * H, O_BO = 2 * H + FE, O_D = O_BO + 1, O_BD = O_D + H, O_SIZE = O_BD + 1;
constexpr int NPARAM = OFF_OUT + O_SIZE;
static_assert(NPARAM == 26502, "parameter count");

__device__ __forceinline__ float sigm(float x) { return 1.0f / (1.0f + expf(-x)); }

// ------------------------------------------------------------ graph setup

// rev[p] = position of (j, i) in row j for the entry (i, j) at p; UINT32_MAX if absent
__global__ void k_rev(uint32_t n, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci, uint32_t* rev,
                      int* nonsym)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
        {
            const uint32_t j = ci[p];
            uint32_t lo = rp[j], hi = rp[j + 1], f = 0xFFFFFFFFu;
            while (lo < hi)
            {
                const uint32_t mid = (lo + hi) / 2;
                if (ci[mid] == i)
                {
                    f = mid;
                    break;
                }
                if (ci[mid] < i)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            rev[p] = f;
            if (f == 0xFFFFFFFFu) atomicExch(nonsym, 1);
        }
}

// node features F (n x 8), edge features EF (nnz x 4), inverse degree
__global__ void k_features(uint32_t n, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                           const double* __restrict__ v, const double* __restrict__ diag, double mean_logd,
                           float* __restrict__ F, float* __restrict__ EF, float* __restrict__ invdeg)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const double aii = diag[i];
        const double la = log(fabs(aii) + 1e-300);
        double s = 0, mn = 1e300, mx = -1e300, off = 0;
        int deg = 0;
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
        {
            const uint32_t j = ci[p];
            if (j == i) continue;
            const double a = fabs(v[p]) + 1e-300;
            const double t = log(a) - la;
            s += t;
            mn = fmin(mn, t);
            mx = fmax(mx, t);
            off += a;
            ++deg;
            const double lj = log(fabs(diag[j]) + 1e-300);
            EF[(size_t)p * FE + 0] = (float)t;
            EF[(size_t)p * FE + 1] = (float)(log(a) - lj);
            EF[(size_t)p * FE + 2] = (float)(lj - la);
            EF[(size_t)p * FE + 3] = j < i ? 1.0f : -1.0f;
        }
        float* f = F + (size_t)i * FIN;
        f[0] = deg ? (float)(s / deg) : 0.f;
        f[1] = deg ? (float)mn : 0.f;
        f[2] = deg ? (float)mx : 0.f;
        f[3] = (float)log(off / fabs(aii) + 1e-30);
        f[4] = deg / 4.0f;
        f[5] = (float)(la - mean_logd);
        f[6] = 0.f;
        f[7] = 0.f;
        invdeg[i] = deg ? 1.0f / deg : 0.f;
    }
}

__global__ void k_logdiag_sum(uint32_t n, const double* __restrict__ d, double* out, double* partial, unsigned* counter)
{
    double acc[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc[0] += log(fabs(d[i]) + 1e-300);
    if (grid_reduce_last<1>(acc, partial, counter))
        if (threadIdx.x == 0) *out = acc[0] / (n ? n : 1);
}

// ------------------------------------------------------------ dense layers

// Y (n x NO) = act(X (n x K) W^T + b), W (NO x K) in BF16, FP32 accumulation.
// Optionally stores the pre-activation; RES adds X (K == NO) after the activation.
constexpr int kFwdRows = 32, kBwdRows = 16;

template <int K, int NO, bool RELU>
__global__ void __launch_bounds__(256) k_linear(uint32_t n, const float* __restrict__ X,
                                                const __nv_bfloat16* __restrict__ W, const float* __restrict__ bias,
                                                float* __restrict__ Y, float* __restrict__ pre)
{
    constexpr int ROWS = kFwdRows, TPR = 256 / ROWS, CPT = NO / TPR;
    __shared__ float Ws[K][NO + 1];
    __shared__ float Xs[ROWS][K + 1];
    for (int t = threadIdx.x; t < K * NO; t += blockDim.x)
    {
        const int o = t / K, k = t % K;
        Ws[k][o] = __bfloat162float(W[t]);
    }
    const uint32_t r0 = blockIdx.x * ROWS;
    for (int t = threadIdx.x; t < ROWS * K; t += blockDim.x)
    {
        const int r = t / K, k = t % K;
        Xs[r][k] = (r0 + r < n) ? X[(size_t)(r0 + r) * K + k] : 0.f;
    }
    __syncthreads();
    const int r = threadIdx.x / TPR, cg = threadIdx.x % TPR;
    float acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = bias ? bias[cg + c * TPR] : 0.f;
#pragma unroll 8
    for (int k = 0; k < K; ++k)
    {
        const float x = Xs[r][k];
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] += x * Ws[k][cg + c * TPR];
    }
    if (r0 + r < n)
    {
#pragma unroll
        for (int c = 0; c < CPT; ++c)
        {
            const int o = cg + c * TPR;
            if (pre) pre[(size_t)(r0 + r) * NO + o] = acc[c];
            Y[(size_t)(r0 + r) * NO + o] = RELU ? fmaxf(acc[c], 0.f) : acc[c];
        }
    }
}

// dX (n x K) [+]= dY (n x NO) W (NO x K)
template <int K, int NO>
__global__ void __launch_bounds__(256) k_linear_bwd_data(uint32_t n, const float* __restrict__ dY,
                                                         const __nv_bfloat16* __restrict__ W, float* __restrict__ dX,
                                                         int accumulate)
{
    constexpr int ROWS = kBwdRows, TPR = 256 / ROWS, CPT = K / TPR;
    __shared__ float Ws[NO][K + 1];
    __shared__ float Ds[ROWS][NO + 1];
    for (int t = threadIdx.x; t < K * NO; t += blockDim.x)
    {
        const int o = t / K, k = t % K;
        Ws[o][k] = __bfloat162float(W[t]);
    }
    const uint32_t r0 = blockIdx.x * ROWS;
    for (int t = threadIdx.x; t < ROWS * NO; t += blockDim.x)
    {
        const int r = t / NO, o = t % NO;
        Ds[r][o] = (r0 + r < n) ? dY[(size_t)(r0 + r) * NO + o] : 0.f;
    }
    __syncthreads();
    const int r = threadIdx.x / TPR, cg = threadIdx.x % TPR;
    float acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = 0.f;
#pragma unroll 8
    for (int o = 0; o < NO; ++o)
    {
        const float d = Ds[r][o];
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] += d * Ws[o][cg + c * TPR];
    }
    if (r0 + r < n)
#pragma unroll
        for (int c = 0; c < CPT; ++c)
        {
            const size_t idx = (size_t)(r0 + r) * K + cg + c * TPR;
            dX[idx] = accumulate ? dX[idx] + acc[c] : acc[c];
        }
}

// per-CTA partial of dW (NO x K) = dY^T X and db = sum dY over a row chunk;
// RX: X rounded to BF16 first, the operand the tensor-core forward multiplied
template <int K, int NO, bool RX>
__global__ void __launch_bounds__(256) k_linear_bwd_weight(uint32_t n, uint32_t rows_per_cta, const float* __restrict__ dY,
                                                           const float* __restrict__ X, float* __restrict__ partial)
{
    constexpr int PAIRS = NO * K, PPT = (PAIRS + 255) / 256, TILE = 32;
    __shared__ float Ds[TILE][NO];
    __shared__ float Xs[TILE][K];
    float acc[PPT];
    float bacc = 0.f;
#pragma unroll
    for (int q = 0; q < PPT; ++q) acc[q] = 0.f;
    const uint32_t r_begin = blockIdx.x * rows_per_cta;
    const uint32_t r_end = min(n, r_begin + rows_per_cta);
    for (uint32_t t0 = r_begin; t0 < r_end; t0 += TILE)
    {
        __syncthreads();
        for (int t = threadIdx.x; t < TILE * NO; t += blockDim.x)
        {
            const int rr = t / NO, o = t % NO;
            Ds[rr][o] = (t0 + rr < r_end) ? dY[(size_t)(t0 + rr) * NO + o] : 0.f;
        }
        for (int t = threadIdx.x; t < TILE * K; t += blockDim.x)
        {
            const int rr = t / K, k = t % K;
            const float x = (t0 + rr < r_end) ? X[(size_t)(t0 + rr) * K + k] : 0.f;
            Xs[rr][k] = RX ? __bfloat162float(__float2bfloat16_rn(x)) : x;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < PPT; ++q)
        {
            const int pr = threadIdx.x + q * 256;
            if (pr < PAIRS)
            {
                const int o = pr / K, k = pr % K;
                float a = acc[q];
                for (int rr = 0; rr < TILE; ++rr) a += Ds[rr][o] * Xs[rr][k];
                acc[q] = a;
            }
        }
        if (threadIdx.x < NO)
            for (int rr = 0; rr < TILE; ++rr) bacc += Ds[rr][threadIdx.x];
    }
    float* out = partial + (size_t)blockIdx.x * (PAIRS + NO);
#pragma unroll
    for (int q = 0; q < PPT; ++q)
    {
        const int pr = threadIdx.x + q * 256;
        if (pr < PAIRS) out[pr] = acc[q];
    }
    if (threadIdx.x < NO) out[PAIRS + threadIdx.x] = bacc;
}

// out[j] (+)= sum over b of partial[b * stride + j], in block order
__global__ void k_reduce_partials(uint32_t nblocks, uint32_t stride, uint32_t count, const float* __restrict__ partial,
                                  float* __restrict__ out, int accumulate)
{
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x)
    {
        float s = 0.f;
        for (uint32_t b = 0; b < nblocks; ++b) s += partial[(size_t)b * stride + j];
        out[j] = accumulate ? out[j] + s : s;
    }
}

// ------------------------------------------------------------ message passing

// SM = [s | m] (n x 128).  pre_i = s_i + b + invdeg_i sum_j g_ij m_j ;  Hn = relu(pre) + H
__global__ void __launch_bounds__(256) k_aggregate(uint32_t n, const uint32_t* __restrict__ rp, const uint32_t* __restrict__ ci,
                                                   const float* __restrict__ EF, const float* __restrict__ invdeg,
                                                   const float* __restrict__ SM, const __nv_bfloat16* __restrict__ Wl,
                                                   const float* __restrict__ Hin, float* __restrict__ pre,
                                                   float* __restrict__ Hout)
{
    // one warp per node, 2 channels per lane
    __shared__ float wg[H][FE], bg[H], bl[H];
    for (int t = threadIdx.x; t < H * FE; t += blockDim.x) wg[t / FE][t % FE] = __bfloat162float(Wl[L_WG + t]);
    for (int t = threadIdx.x; t < H; t += blockDim.x)
    {
        bg[t] = __bfloat162float(Wl[L_BG + t]);
        bl[t] = __bfloat162float(Wl[L_B + t]);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int c0 = lane, c1 = lane + 32;
    // grid-stride over nodes, so the weights above are staged once per CTA
    for (uint32_t i = blockIdx.x * 8 + (threadIdx.x >> 5); i < n; i += gridDim.x * 8)
    {
        float a0 = 0.f, a1 = 0.f;
        // neighbours eight at a time: their indices, edge features and messages
        // are all in flight before the gates are formed (same summation order)
        const uint32_t pa = rp[i], pe = rp[i + 1];
        for (uint32_t pb = pa; pb < pe; pb += 8)
        {
            uint32_t jj[8];
            float4 ee[8];
            float m0[8], m1[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) jj[k] = pb + k < pe ? ci[pb + k] : i;
#pragma unroll
            for (int k = 0; k < 8; ++k)
            {
                const bool on = jj[k] != i;
                ee[k] = on ? *reinterpret_cast<const float4*>(EF + (size_t)(pb + k) * FE) : make_float4(0.f, 0.f, 0.f, 0.f);
                m0[k] = on ? SM[(size_t)jj[k] * 2 * H + H + c0] : 0.f;
                m1[k] = on ? SM[(size_t)jj[k] * 2 * H + H + c1] : 0.f;
            }
#pragma unroll
            for (int k = 0; k < 8; ++k)
            {
                if (jj[k] == i) continue;
                const float4 e = ee[k];
                const float g0 = sigm(bg[c0] + wg[c0][0] * e.x + wg[c0][1] * e.y + wg[c0][2] * e.z + wg[c0][3] * e.w);
                const float g1 = sigm(bg[c1] + wg[c1][0] * e.x + wg[c1][1] * e.y + wg[c1][2] * e.z + wg[c1][3] * e.w);
                a0 += g0 * m0[k];
                a1 += g1 * m1[k];
            }
        }
        const float id = invdeg[i];
        const float p0 = SM[(size_t)i * 2 * H + c0] + bl[c0] + id * a0;
        const float p1 = SM[(size_t)i * 2 * H + c1] + bl[c1] + id * a1;
        if (pre)  // kept for the backward pass (training only)
        {
            pre[(size_t)i * H + c0] = p0;
            pre[(size_t)i * H + c1] = p1;
        }
        Hout[(size_t)i * H + c0] = fmaxf(p0, 0.f) + Hin[(size_t)i * H + c0];
        Hout[(size_t)i * H + c1] = fmaxf(p1, 0.f) + Hin[(size_t)i * H + c1];
    }
}

// backward of k_aggregate for one layer.
//   dpre = dHout * (pre > 0);  dHin = dHout (residual, written here);
//   dSM[:, :64] = dpre;  dSM[j, 64:] = sum_{i in N(j)} invdeg_i g_ij dpre_i
//   per-CTA partials of dW_g (64x4), db_g (64), db (64)
__global__ void __launch_bounds__(256) k_aggregate_bwd(uint32_t n, const uint32_t* __restrict__ rp,
                                                       const uint32_t* __restrict__ ci, const uint32_t* __restrict__ rev,
                                                       const float* __restrict__ EF, const float* __restrict__ invdeg,
                                                       const float* __restrict__ SM, const __nv_bfloat16* __restrict__ Wl,
                                                       const float* __restrict__ pre, const float* __restrict__ dHout,
                                                       float* __restrict__ dSM, float* __restrict__ dHin,
                                                       float* __restrict__ partial)
{
    __shared__ float wg[H][FE], bg[H];
    __shared__ float pw[8][H][FE + 2];  // per warp: dW_g (4), db_g, db
    for (int t = threadIdx.x; t < H * FE; t += blockDim.x) wg[t / FE][t % FE] = __bfloat162float(Wl[L_WG + t]);
    for (int t = threadIdx.x; t < H; t += blockDim.x) bg[t] = __bfloat162float(Wl[L_BG + t]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int t = lane; t < H * (FE + 2); t += 32) pw[warp][t / (FE + 2)][t % (FE + 2)] = 0.f;
    __syncthreads();
    const uint32_t j = blockIdx.x * 8 + warp;
    if (j < n)
    {
        for (int h = 0; h < 2; ++h)
        {
            const int c = lane + 32 * h;
            const float dp = pre[(size_t)j * H + c] > 0.f ? dHout[(size_t)j * H + c] : 0.f;
            dSM[(size_t)j * 2 * H + c] = dp;
            dHin[(size_t)j * H + c] = dHout[(size_t)j * H + c];
            pw[warp][c][FE + 1] += dp;
            // gather over neighbours i of j: edge (i, j) at rev[p] in row i
            float dm = 0.f;
            for (uint32_t p = rp[j]; p < rp[j + 1]; ++p)
            {
                const uint32_t i = ci[p];
                if (i == j) continue;
                const uint32_t q = rev[p];
                const float* e = EF + (size_t)q * FE;
                const float z = bg[c] + wg[c][0] * e[0] + wg[c][1] * e[1] + wg[c][2] * e[2] + wg[c][3] * e[3];
                const float g = sigm(z);
                const float dpi = pre[(size_t)i * H + c] > 0.f ? dHout[(size_t)i * H + c] : 0.f;
                const float w = invdeg[i] * dpi;
                dm += w * g;
            }
            dSM[(size_t)j * 2 * H + H + c] = dm;
            // gate gradient for the edges (j, k) of row j (owned by node j)
            const float dpj = dp * invdeg[j];
            for (uint32_t p = rp[j]; p < rp[j + 1]; ++p)
            {
                const uint32_t k = ci[p];
                if (k == j) continue;
                const float* e = EF + (size_t)p * FE;
                const float z = bg[c] + wg[c][0] * e[0] + wg[c][1] * e[1] + wg[c][2] * e[2] + wg[c][3] * e[3];
                const float g = sigm(z);
                const float dz = dpj * SM[(size_t)k * 2 * H + H + c] * g * (1.f - g);
                pw[warp][c][0] += dz * e[0];
                pw[warp][c][1] += dz * e[1];
                pw[warp][c][2] += dz * e[2];
                pw[warp][c][3] += dz * e[3];
                pw[warp][c][FE] += dz;
            }
        }
    }
    __syncthreads();
    // fixed-order sum over the 8 warps, then one partial per CTA
    float* out = partial + (size_t)blockIdx.x * (H * (FE + 2));
    for (int t = threadIdx.x; t < H * (FE + 2); t += blockDim.x)
    {
        float s = 0.f;
        for (int w = 0; w < 8; ++w) s += pw[w][t / (FE + 2)][t % (FE + 2)];
        out[t] = s;
    }
}

// ------------------------------------------------------------ output head

// Lv <- L0 * exp(s tanh c) on the pattern of L (rows with diagonal last).  The
// head uses FP32 parameters (Pf) rounded to BF16 by the caller.  C receives c.
// Per-node projections of the head: proj[3i..3i+2] = (u.h_i, v.h_i, d.h_i).
// Half a warp per node, four features per lane, a fixed shuffle tree: the
// sums do not depend on the launch.
__global__ void k_head_proj(uint32_t n, const float* __restrict__ Hf, const float* __restrict__ Pf,
                            float* __restrict__ proj)
{
    const uint32_t lane = threadIdx.x & 15u;
    // u and v start on 16-byte boundaries; d (at O_D = 133) does not
    static_assert(((OFF_OUT + O_U) % 4) == 0 && ((OFF_OUT + O_V) % 4) == 0, "u, v alignment");
    const float4 u = *reinterpret_cast<const float4*>(Pf + OFF_OUT + O_U + 4 * lane);
    const float4 v = *reinterpret_cast<const float4*>(Pf + OFF_OUT + O_V + 4 * lane);
    const float* dp = Pf + OFF_OUT + O_D + 4 * lane;
    const float4 dd = make_float4(dp[0], dp[1], dp[2], dp[3]);
    const uint32_t stride = (gridDim.x * blockDim.x) >> 4;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; i < n; i += stride)
    {
        const float4 h = *reinterpret_cast<const float4*>(Hf + (size_t)i * H + 4 * lane);
        float a = u.x * h.x + u.y * h.y + u.z * h.z + u.w * h.w;
        float b = v.x * h.x + v.y * h.y + v.z * h.z + v.w * h.w;
        float c = dd.x * h.x + dd.y * h.y + dd.z * h.z + dd.w * h.w;
#pragma unroll
        for (int o = 8; o > 0; o >>= 1)
        {
            // the two half-warps may run different trip counts: each shuffles alone
            const unsigned half = 0xFFFFu << (threadIdx.x & 16u);
            a += __shfl_xor_sync(half, a, o, 16);
            b += __shfl_xor_sync(half, b, o, 16);
            c += __shfl_xor_sync(half, c, o, 16);
        }
        if (lane == 0)
        {
            proj[3 * (size_t)i] = a;
            proj[3 * (size_t)i + 1] = b;
            proj[3 * (size_t)i + 2] = c;
        }
    }
}

// c_ij = b_o + u.h_i + v.h_j + w.e_ij (j < i),  c_ii = b_d + d.h_i, from the
// node projections; Lv <- L0 * exp(s tanh c) on the pattern of L (rows with
// diagonal last).  The head uses FP32 parameters (Pf) rounded to BF16 by the
// caller.  C receives c.
__global__ void k_head(uint32_t n, const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Lci,
                       const uint32_t* __restrict__ Arp, const double* __restrict__ Adiag, const float* __restrict__ EF,
                       const float* __restrict__ proj, const float* __restrict__ Pf, const double* __restrict__ L0,
                       double* __restrict__ Lv, float* __restrict__ C, double* __restrict__ diag_out)
{
    const float bo = Pf[OFF_OUT + O_BO], bd = Pf[OFF_OUT + O_BD];
    float w[FE];
#pragma unroll
    for (int k = 0; k < FE; ++k) w[k] = Pf[OFF_OUT + O_W + k];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const float ai = proj[3 * (size_t)i], di = proj[3 * (size_t)i + 2];
        for (uint32_t q = Lrp[i]; q < Lrp[i + 1]; ++q)
        {
            const uint32_t j = Lci[q];
            float c;
            if (j == i)
                c = bd + di;
            else
            {
                const uint32_t pA = Arp[i] + (q - Lrp[i]);  // L row i is a prefix of A row i
                const float4 e = *reinterpret_cast<const float4*>(EF + (size_t)pA * FE);
                c = bo + ai + proj[3 * (size_t)j + 1];
                c += w[0] * e.x + w[1] * e.y + w[2] * e.z + w[3] * e.w;
            }
            C[q] = c;
            double val = L0[q] * exp((double)(kScale * tanhf(c)));
            if (j == i)
            {
                const double lo = 1e-3 * sqrt(fabs(Adiag[i]));
                if (val < lo) val = lo;
                if (diag_out) diag_out[i] = val;
            }
            Lv[q] = val;
        }
    }
}

// dc from dL~ : dc = dL * L~ * s (1 - tanh^2 c), 0 where the guard clamped
__global__ void k_head_dc(uint32_t nnz, const double* __restrict__ dL, const double* __restrict__ Lv,
                          const double* __restrict__ L0, const float* __restrict__ C, float* __restrict__ dC)
{
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += gridDim.x * blockDim.x)
    {
        const float t = tanhf(C[q]);
        const double expected = L0[q] * exp((double)(kScale * t));
        const bool clamped = fabs(Lv[q] - expected) > 1e-12 * fabs(expected);
        dC[q] = clamped ? 0.f : (float)(dL[q] * Lv[q] * kScale * (1.f - t * t));
    }
}

// head backward: dH_i += sum_row dc_q u (+ dc_ii d) ; dH_j += sum_{col j} dc_q v ;
// per-CTA partials of du, dv, dw, dbo, dd, dbd
__global__ void __launch_bounds__(256) k_head_bwd(uint32_t n, const uint32_t* __restrict__ Lrp,
                                                  const uint32_t* __restrict__ Lci, const uint32_t* __restrict__ Trp,
                                                  const uint32_t* __restrict__ Tpos, const uint32_t* __restrict__ Arp,
                                                  const float* __restrict__ EF, const float* __restrict__ Hf,
                                                  const float* __restrict__ Pf, const float* __restrict__ dC,
                                                  float* __restrict__ dH, float* __restrict__ partial)
{
    __shared__ float pw[8][O_SIZE];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int t = lane; t < O_SIZE; t += 32) pw[warp][t] = 0.f;
    __syncwarp();
    const uint32_t i = blockIdx.x * 8 + warp;
    if (i < n)
    {
        for (int h = 0; h < 2; ++h)
        {
            const int c = lane + 32 * h;
            float dh = 0.f;
            const float hic = Hf[(size_t)i * H + c];
            for (uint32_t q = Lrp[i]; q < Lrp[i + 1]; ++q)
            {
                const uint32_t j = Lci[q];
                const float d = dC[q];
                if (j == i)
                {
                    dh += d * Pf[OFF_OUT + O_D + c];
                    pw[warp][O_D + c] += d * hic;
                    if (c == 0) pw[warp][O_BD] += d;
                }
                else
                {
                    dh += d * Pf[OFF_OUT + O_U + c];
                    pw[warp][O_U + c] += d * hic;
                    pw[warp][O_V + c] += d * Hf[(size_t)j * H + c];
                    if (c < FE) pw[warp][O_W + c] += d * EF[(size_t)(Arp[i] + (q - Lrp[i])) * FE + c];
                    if (c == 0) pw[warp][O_BO] += d;
                }
            }
            // column part: entries (k, i) with k > i, listed in row i of L^T
            for (uint32_t t = Trp[i]; t < Trp[i + 1]; ++t) dh += dC[Tpos[t]] * Pf[OFF_OUT + O_V + c];
            dH[(size_t)i * H + c] = dh;
        }
    }
    __syncthreads();
    float* out = partial + (size_t)blockIdx.x * O_SIZE;
    for (int t = threadIdx.x; t < O_SIZE; t += blockDim.x)
    {
        float s = 0.f;
        for (int w = 0; w < 8; ++w) s += pw[w][t];
        out[t] = s;
    }
}

// ------------------------------------------------------------ loss

// u = L~^T w : u_j = L~_jj w_j + sum_{i>j} L~_ij w_i  (via L^T rows: Trp / Tpos)
__global__ void k_ltmul(uint32_t n, const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Trp,
                        const uint32_t* __restrict__ Tci, const uint32_t* __restrict__ Tpos,
                        const double* __restrict__ Lv, const double* __restrict__ w, double* __restrict__ u)
{
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    {
        double s = Lv[Lrp[j + 1] - 1] * w[j];
        for (uint32_t t = Trp[j]; t < Trp[j + 1]; ++t) s += Lv[Tpos[t]] * w[Tci[t]];
        u[j] = s;
    }
}

// v = L~ u - Aw ; acc += v.v
__global__ void k_lmul_res(uint32_t n, const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Lci,
                           const double* __restrict__ Lv, const double* __restrict__ u, const double* __restrict__ Aw,
                           double* __restrict__ v, double* out, double* partial, unsigned* counter)
{
    double acc[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        double s = 0.0;
        for (uint32_t q = Lrp[i]; q < Lrp[i + 1]; ++q) s += Lv[q] * u[Lci[q]];
        const double vi = s - Aw[i];
        v[i] = vi;
        acc[0] += vi * vi;
    }
    if (grid_reduce_last<1>(acc, partial, counter))
        if (threadIdx.x == 0) *out = acc[0];
}

// dL_q += scale (v_i u_j + w_i q_j)
__global__ void k_dL(uint32_t n, const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Lci,
                     const double* __restrict__ v, const double* __restrict__ u, const double* __restrict__ w,
                     const double* __restrict__ qv, const double* __restrict__ scale, double* __restrict__ dL)
{
    const double s = *scale;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (uint32_t q = Lrp[i]; q < Lrp[i + 1]; ++q)
        {
            const uint32_t j = Lci[q];
            dL[q] += s * (v[i] * u[j] + w[i] * qv[j]);
        }
}

// preconditioned-residual loss: e = w - z
__global__ void k_sub(uint32_t n, const double* __restrict__ w, const double* __restrict__ z, double* __restrict__ e)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) e[i] = w[i] - z[i];
}

// g = -scale * e
__global__ void k_neg_scale(uint32_t n, const double* __restrict__ e, const double* __restrict__ scale,
                            double* __restrict__ g)
{
    const double s = *scale;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) g[i] = -s * e[i];
}

// dL~_ij -= z_i a_j + b_i y_j
__global__ void k_dL_pc(uint32_t n, const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Lci,
                        const double* __restrict__ z, const double* __restrict__ a, const double* __restrict__ b,
                        const double* __restrict__ y, double* __restrict__ dL)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (uint32_t q = Lrp[i]; q < Lrp[i + 1]; ++q)
        {
            const uint32_t j = Lci[q];
            dL[q] -= z[i] * a[j] + b[i] * y[j];
        }
}

// ---- the sweep apply and its adjoint (B2S_LOSS_SWEEPS), FP64
// L~ rows hold the strict entries in column order, then the diagonal.

// lower sweep: yout_i = (r_i - sum_{j<i} L_ij yin_j) / L_ii (pass 0: yin null)
__global__ void k_sw_lo(uint32_t n, const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Lci,
                        const double* __restrict__ Lv, const double* __restrict__ r, const double* __restrict__ yin,
                        double* __restrict__ yout)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const uint32_t d = Lrp[i + 1] - 1;
        double t = r[i];
        if (yin)
            for (uint32_t q = Lrp[i]; q < d; ++q) t -= Lv[q] * yin[Lci[q]];
        yout[i] = t / Lv[d];
    }
}

// upper sweep over L~^T rows (Trp / Tci / Tpos): zout_i = (u_i - sum_{j>i} L_ji zin_j) / L_ii
__global__ void k_sw_up(uint32_t n, const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Trp,
                        const uint32_t* __restrict__ Tci, const uint32_t* __restrict__ Tpos,
                        const double* __restrict__ Lv, const double* __restrict__ u, const double* __restrict__ zin,
                        double* __restrict__ zout)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        double t = u[i];
        if (zin)
            for (uint32_t q = Trp[i]; q < Trp[i + 1]; ++q) t -= Lv[Tpos[q]] * zin[Tci[q]];
        zout[i] = t / Lv[Lrp[i + 1] - 1];
    }
}

// adjoint step, diagonal part: h = gbar / L_ii; dL_ii -= h_i state_i; acc += h (when acc is given)
__global__ void k_sw_h(uint32_t n, const uint32_t* __restrict__ Lrp, const double* __restrict__ Lv,
                       const double* __restrict__ gbar, const double* __restrict__ state, double* __restrict__ h,
                       double* __restrict__ acc, double* __restrict__ dL)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const uint32_t d = Lrp[i + 1] - 1;
        const double hi = gbar[i] / Lv[d];
        h[i] = hi;
        if (acc) acc[i] += hi;
        dL[d] -= hi * state[i];
    }
}

// upper adjoint, strict part (rows j of L~): dL_ji -= h_i zprev_j; gnext_j = -sum_{i<j} L_ji h_i
__global__ void k_sw_up_adj(uint32_t n, const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Lci,
                            const double* __restrict__ Lv, const double* __restrict__ h,
                            const double* __restrict__ zprev, double* __restrict__ gnext, double* __restrict__ dL)
{
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    {
        double g = 0.0;
        const double zj = zprev[j];
        for (uint32_t q = Lrp[j]; q < Lrp[j + 1] - 1; ++q)
        {
            const double hi = h[Lci[q]];
            g -= Lv[q] * hi;
            dL[q] -= hi * zj;
        }
        gnext[j] = g;
    }
}

// lower adjoint, strict part (rows j of L~^T): dL_ij -= h_i yprev_j; gnext_j = -sum_{i>j} L_ij h_i
__global__ void k_sw_lo_adj(uint32_t n, const uint32_t* __restrict__ Trp, const uint32_t* __restrict__ Tci,
                            const uint32_t* __restrict__ Tpos, const double* __restrict__ Lv,
                            const double* __restrict__ h, const double* __restrict__ yprev,
                            double* __restrict__ gnext, double* __restrict__ dL)
{
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    {
        double g = 0.0;
        const double yj = yprev[j];
        for (uint32_t t = Trp[j]; t < Trp[j + 1]; ++t)
        {
            const uint32_t q = Tpos[t];
            const double hi = h[Tci[t]];
            g -= Lv[q] * hi;
            dL[q] -= hi * yj;
        }
        gnext[j] = g;
    }
}

// diag[i] = L_ii, the last entry of row i of L (columns ascending, j <= i)
__global__ void k_diag_from_rows(uint32_t n, const uint32_t* __restrict__ Lrp, const double* __restrict__ Lv,
                                 double* __restrict__ diag)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        diag[i] = Lv[Lrp[i + 1] - 1];
}

// scale = 2 / (P ||Aw||^2), loss += ||v||^2 / (P ||Aw||^2)
__global__ void k_loss_scale(const double* vv, const double* aw2, int nprobes, double* scale, double* loss)
{
    const double d = (*aw2 > 0 ? *aw2 : 1.0) * nprobes;
    *scale = 2.0 / d;
    *loss += *vv / d;
}

// Jacobi smoothing of a probe: w <- w - (2/3) D^-1 (A w)
__global__ void k_jacobi_probe(uint32_t n, const double* __restrict__ Aw, const double* __restrict__ d,
                               double* __restrict__ w)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        w[i] -= (2.0 / 3.0) * Aw[i] / d[i];
}

__global__ void k_normal(uint64_t seed, uint32_t n, double* __restrict__ w)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        auto mix = [](uint64_t z) {
            z += 0x9E3779B97F4A7C15ull;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            return z ^ (z >> 31);
        };
        const double u1 = ((mix(seed * 0x9E3779B97F4A7C15ull + 2ull * i) >> 11) + 1.0) * (1.0 / 9007199254740993.0);
        const double u2 = (mix(seed * 0x9E3779B97F4A7C15ull + 2ull * i + 1) >> 11) * (1.0 / 9007199254740992.0);
        w[i] = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    }
}

// ------------------------------------------------------------ optimiser

__global__ void k_adam(uint32_t np, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                       __nv_bfloat16* __restrict__ pb)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x)
    {
        const float gk = g[k];
        const float mk = b1 * m[k] + (1.f - b1) * gk;
        const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
        m[k] = mk;
        v[k] = vk;
        const float pk = p[k] - lr * (mk / c1) / (sqrtf(vk / c2) + eps);
        p[k] = pk;
        pb[k] = __float2bfloat16(pk);
    }
}

__global__ void k_to_bf16(uint32_t np, const float* __restrict__ p, __nv_bfloat16* __restrict__ pb,
                          float* __restrict__ pr)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x)
    {
        pb[k] = __float2bfloat16(p[k]);
        pr[k] = __bfloat162float(pb[k]);
    }
}

__global__ void k_lt_positions(uint32_t n, const uint32_t* __restrict__ Trp, const uint32_t* __restrict__ Tci,
                               const uint32_t* __restrict__ Lrp, const uint32_t* __restrict__ Lci,
                               uint32_t* __restrict__ Tpos)
{
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
        for (uint32_t t = Trp[j]; t < Trp[j + 1]; ++t)
        {
            const uint32_t i = Tci[t];
            uint32_t lo = Lrp[i], hi = Lrp[i + 1];
            while (lo < hi)
            {
                const uint32_t mid = (lo + hi) / 2;
                if (Lci[mid] < j)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            Tpos[t] = lo;
        }
}

// dpre0 = dH0 * (pre0 > 0)
__global__ void k_relu_mask(uint64_t n, const float* __restrict__ pre, const float* __restrict__ dH, float* __restrict__ d)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        d[i] = pre[i] > 0.f ? dH[i] : 0.f;
}

// reduced gate partials [c][0..3 dW_g, 4 db_g, 5 db] -> layer gradient layout
__global__ void k_gate_grads(const float* __restrict__ red, float* __restrict__ gl)
{
    for (int c = threadIdx.x; c < H; c += blockDim.x)
    {
        for (int e = 0; e < FE; ++e) gl[L_WG + c * FE + e] = red[c * (FE + 2) + e];
        gl[L_BG + c] = red[c * (FE + 2) + FE];
        gl[L_B + c] = red[c * (FE + 2) + FE + 1];
    }
}

}  // namespace

// ------------------------------------------------------------ network state

// Y = bf16(X) W^T [+ bias] on the tensor cores (tc_linear.cuh)
template <int K, int NO>
static void linear_tc(b2s_ctx* ctx, uint32_t n, const float* X, const __nv_bfloat16* W, const float* bias, float* Y,
                      int* err)
{
    using S = tc::LinearShape<K, NO>;
    if (!n) return;
    need((((uintptr_t)X | (uintptr_t)W | (uintptr_t)Y | (uintptr_t)bias) & 15) == 0, B2S_INVALID_ARG,
         "tensor-core layer: operands must be 16-byte aligned");
    B2S_CUDA(cudaFuncSetAttribute(tc::k_linear_tc<K, NO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::kSmem));
    const uint32_t tiles = (n + tc::kTileRows - 1) / tc::kTileRows;
    const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)ctx->sm_count * S::kCtasPerSm);
    B2S_LAUNCH(ctx, (tc::k_linear_tc<K, NO>), grid, tc::kThreadsTc, S::kSmem, n, X, W, bias, Y, err);
}

struct Gnn
{
    DBuf<float> p;                 // FP32 master parameters
    DBuf<__nv_bfloat16> pb;        // BF16 copy (forward)
    DBuf<float> pr;                // BF16-rounded values as FP32 (head)
    DBuf<float> m, v, g;           // Adam moments, gradient
    int step = 0;

    void init(b2s_ctx* ctx, uint64_t seed)
    {
        p.alloc(NPARAM);
        pb.alloc(NPARAM);
        pr.alloc(NPARAM);
        m.alloc(NPARAM);
        v.alloc(NPARAM);
        g.alloc(NPARAM);
        std::vector<float> h(NPARAM, 0.f);
        uint64_t s = seed * 0x9E3779B97F4A7C15ull + 12345;
        auto rnd = [&]() {
            s += 0x9E3779B97F4A7C15ull;
            uint64_t z = s;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            z ^= z >> 31;
            return (float)((z >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
        };
        const float sin_ = std::sqrt(6.f / (FIN + H)), sh = std::sqrt(6.f / (2 * H)), sg = std::sqrt(6.f / (FE + H));
        for (int k = 0; k < H * FIN; ++k) h[OFF_WIN + k] = sin_ * rnd();
        for (int l = 0; l < NL; ++l)
        {
            float* L = &h[LAYER0 + l * L_SIZE];
            for (int k = 0; k < H * H; ++k) L[L_WS + k] = 0.5f * sh * rnd();
            for (int k = 0; k < H * H; ++k) L[L_WM + k] = 0.5f * sh * rnd();
            for (int k = 0; k < H * FE; ++k) L[L_WG + k] = sg * rnd();
        }
        // output head zero: the untrained network returns IC(0)
        set(ctx, h.data());
    }
    void set(b2s_ctx* ctx, const float* host)
    {
        h2d(ctx, p.p, host, NPARAM * sizeof(float));
        B2S_CUDA(cudaMemsetAsync(m.p, 0, m.bytes(), ctx->stream));
        B2S_CUDA(cudaMemsetAsync(v.p, 0, v.bytes(), ctx->stream));
        step = 0;
        refresh(ctx);
    }
    void refresh(b2s_ctx* ctx)
    {
        B2S_LAUNCH(ctx, k_to_bf16, stream_grid(ctx, NPARAM), kThreads, 0, (uint32_t)NPARAM, p.p, pb.p, pr.p);
    }
};

// graph-derived state of one matrix + the activations of one forward pass
struct GnnGraph
{
    uint32_t n = 0, nnz = 0;
    DBuf<uint32_t> rev;
    DBuf<float> F, EF, invdeg;
    // Activations.  Training keeps every layer's (Hs[0..NL], SM, pre, pre0)
    // for the backward pass; inference keeps two node-state buffers and one
    // [s | m] buffer, reused layer after layer.
    DBuf<float> Hs[NL + 1], SM[NL], pre[NL], pre0;
    DBuf<double> logd;
    DBuf<int> err;  // B2S_TIMEOUT from the tensor-core layer's bounded wait
    bool training = false;

    const float* state(int l) const { return training ? Hs[l].p : Hs[l & 1].p; }
    float* state_mut(int l) { return training ? Hs[l].p : Hs[l & 1].p; }
    float* sm(int l) { return training ? SM[l].p : SM[0].p; }

    void build(b2s_ctx* ctx, const CsrDev& A, bool train = false)
    {
        training = train;
        n = A.n;
        nnz = A.nnz;
        err.alloc(1);
        B2S_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), ctx->stream));
        rev.alloc(nnz ? nnz : 1);
        DBuf<int> nonsym(1);
        B2S_CUDA(cudaMemsetAsync(nonsym.p, 0, sizeof(int), ctx->stream));
        B2S_LAUNCH(ctx, k_rev, stream_grid(ctx, n), kThreads, 0, n, A.rp.p, A.ci.p, rev.p, nonsym.p);
        int h = 0;
        d2h(ctx, &h, nonsym.p, sizeof(int));
        sync(ctx);
        if (h) fail(B2S_UNSUPPORTED, "learned IC(0) needs a structurally symmetric matrix");
        F.alloc((size_t)n * FIN);
        EF.alloc((size_t)nnz * FE);
        B2S_CUDA(cudaMemsetAsync(EF.p, 0, EF.bytes(), ctx->stream));
        invdeg.alloc(n);
        logd.alloc(1);
        reserve_reduction(ctx, stream_grid(ctx, n));
        B2S_LAUNCH(ctx, k_logdiag_sum, stream_grid(ctx, n), kThreads, 0, n, A.diag.p, logd.p, ctx->partial.p,
                   ctx->counter.p);
        double mean = 0;
        d2h(ctx, &mean, logd.p, sizeof(double));
        sync(ctx);
        B2S_LAUNCH(ctx, k_features, stream_grid(ctx, n), kThreads, 0, n, A.rp.p, A.ci.p, A.v.p, A.diag.p, mean, F.p,
                   EF.p, invdeg.p);
        if (training)
        {
            for (int l = 0; l <= NL; ++l) Hs[l].alloc((size_t)n * H);
            for (int l = 0; l < NL; ++l)
            {
                SM[l].alloc((size_t)n * 2 * H);
                pre[l].alloc((size_t)n * H);
            }
            pre0.alloc((size_t)n * H);
        }
        else
        {
            Hs[0].alloc((size_t)n * H);
            Hs[1].alloc((size_t)n * H);
            SM[0].alloc((size_t)n * 2 * H);
        }
    }

    void forward(b2s_ctx* ctx, const Gnn& net, const CsrDev& A)
    {
        const unsigned g64 = (n + kFwdRows - 1) / kFwdRows;
        const unsigned gw = std::min<unsigned>((n + 7) / 8, (unsigned)ctx->sm_count * 8);
        B2S_LAUNCH(ctx, (k_linear<FIN, H, true>), g64, 256, 0, n, F.p, net.pb.p + OFF_WIN, net.pr.p + OFF_BIN,
                   state_mut(0), training ? pre0.p : (float*)nullptr);
        for (int l = 0; l < NL; ++l)
        {
            const __nv_bfloat16* Wl = net.pb.p + LAYER0 + l * L_SIZE;
            // [W_s ; W_m] are contiguous: one 128 x 64 weight, on the tensor cores
            linear_tc<H, 2 * H>(ctx, n, state(l), Wl + L_WS, nullptr, sm(l), err.p);
            B2S_LAUNCH(ctx, k_aggregate, gw, 256, 0, n, A.rp.p, A.ci.p, EF.p, invdeg.p, sm(l), Wl, state(l),
                       training ? pre[l].p : (float*)nullptr, state_mut(l + 1));
        }
    }

    // the output head on the final node states
    void head(b2s_ctx* ctx, const Gnn& net, const CsrDev& A, const uint32_t* Lrp, const uint32_t* Lci,
              const double* L0, double* Lv, float* C, double* diag)
    {
        DBuf<float> proj((size_t)3 * n + 1);
        const unsigned gp = (unsigned)std::min<uint64_t>(((uint64_t)n * 16 + 255) / 256, (uint64_t)ctx->sm_count * 8);
        B2S_LAUNCH(ctx, k_head_proj, gp ? gp : 1u, 256, 0, n, state(NL), net.pr.p, proj.p);
        B2S_LAUNCH(ctx, k_head, stream_grid(ctx, n), kThreads, 0, n, Lrp, Lci, A.rp.p, A.diag.p, EF.p, proj.p,
                   net.pr.p, L0, Lv, C, diag);
    }

    // after a synchronisation: fail with B2S_TIMEOUT if a layer's wait gave up
    void check(b2s_ctx* ctx)
    {
        int h = 0;
        d2h(ctx, &h, err.p, sizeof(int));
        sync(ctx);
        if (h) fail(B2S_TIMEOUT, "tensor-core layer: wait for the MMA completion gave up");
    }
};

// IC(0) factor values -> corrected values (inference)
struct LearnedCorrection final : Ic0Correction
{
    const Gnn* net;
    explicit LearnedCorrection(const Gnn* g) : net(g) {}
    void correct(b2s_ctx* ctx, const CsrDev& A, const uint32_t* Lrp, const uint32_t* Lci, uint32_t Lnnz, double* Lv,
                 double* diag) override
    {
        GnnGraph G;
        G.build(ctx, A);
        G.forward(ctx, *net, A);
        DBuf<double> L0(Lnnz ? Lnnz : 1);
        d2d(ctx, L0.p, Lv, Lnnz * sizeof(double));
        DBuf<float> C(Lnnz ? Lnnz : 1);
        G.head(ctx, *net, A, Lrp, Lci, L0.p, Lv, C.p, diag);
        G.check(ctx);
    }
};

// a factor computed elsewhere (the training step's L~) placed into an IC(0)
// preconditioner on the same pattern, so its triangular solves can be reused
struct GivenFactor final : Ic0Correction
{
    const double* src;
    explicit GivenFactor(const double* s) : src(s) {}
    void correct(b2s_ctx* ctx, const CsrDev& A, const uint32_t* Lrp, const uint32_t*, uint32_t Lnnz, double* Lv,
                 double* diag) override
    {
        d2d(ctx, Lv, src, Lnnz * sizeof(double));
        B2S_LAUNCH(ctx, k_diag_from_rows, stream_grid(ctx, A.n), kThreads, 0, A.n, Lrp, Lv, diag);
    }
};

}  // namespace b2s

// ------------------------------------------------------------ learner handle

struct b2s_learner
{
    b2s_ctx* ctx = nullptr;
    b2s::Gnn net;
    int loss = B2S_LOSS_PRECOND;
    int trsv_sweeps = 6;    // B2S_LOSS_SWEEPS: sweeps per triangle
    int factor_sweeps = 0;  // base factor: 0 exact IC(0), k > 0 k fixed-point sweeps
};

namespace b2s {

static const char kMagic[8] = {'B', '2', 'S', 'L', 'R', 'N', '0', '1'};

static uint64_t fnv1a(const void* data, size_t bytes)
{
    const unsigned char* p = static_cast<const unsigned char*>(data);
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < bytes; ++i)
    {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}

static void load_weights(b2s_ctx* ctx, Gnn& net, const char* path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) fail(B2S_INVALID_ARG, std::string("cannot open weight file ") + path);
    char magic[8];
    uint32_t ver = 0, count = 0;
    f.read(magic, 8);
    f.read(reinterpret_cast<char*>(&ver), 4);
    f.read(reinterpret_cast<char*>(&count), 4);
    if (!f || std::memcmp(magic, kMagic, 8) != 0 || ver != 1 || count != (uint32_t)NPARAM)
        fail(B2S_INVALID_ARG, std::string("not a learned IC(0) weight file: ") + path);
    std::vector<float> h(NPARAM);
    uint64_t sum = 0;
    f.read(reinterpret_cast<char*>(h.data()), NPARAM * sizeof(float));
    f.read(reinterpret_cast<char*>(&sum), 8);
    if (!f || sum != fnv1a(h.data(), NPARAM * sizeof(float)))
        fail(B2S_INVALID_ARG, std::string("weight file checksum mismatch: ") + path);
    net.set(ctx, h.data());
}

// default weights shipped next to the library: <dir of libb2s.so>/weights/learned_ic0.bin
static std::string default_weight_path()
{
    Dl_info info;
    if (dladdr(reinterpret_cast<void*>(&default_weight_path), &info) && info.dli_fname)
    {
        std::string p(info.dli_fname);
        const size_t s = p.rfind('/');
        return (s == std::string::npos ? std::string(".") : p.substr(0, s)) + "/weights/learned_ic0.bin";
    }
    return "";
}

static void save_weights(b2s_ctx* ctx, const Gnn& net, const char* path)
{
    std::vector<float> h(NPARAM);
    d2h(ctx, h.data(), net.p.p, NPARAM * sizeof(float));
    sync(ctx);
    std::ofstream f(path, std::ios::binary);
    if (!f) fail(B2S_INVALID_ARG, std::string("cannot write ") + path);
    const uint32_t ver = 1, count = NPARAM;
    const uint64_t sum = fnv1a(h.data(), NPARAM * sizeof(float));
    f.write(kMagic, 8);
    f.write(reinterpret_cast<const char*>(&ver), 4);
    f.write(reinterpret_cast<const char*>(&count), 4);
    f.write(reinterpret_cast<const char*>(h.data()), NPARAM * sizeof(float));
    f.write(reinterpret_cast<const char*>(&sum), 8);
    if (!f) fail(B2S_INVALID_ARG, std::string("write failed: ") + path);
}

std::unique_ptr<PcImpl> make_pc_learned_with(b2s_ctx* ctx, const CsrDev& A, const b2s_pc_opts& o, const Gnn& net)
{
    LearnedCorrection corr(&net);
    b2s_pc_opts oo = o;
    return make_pc_ic0_ex(ctx, A, oo, &corr);
}

std::unique_ptr<PcImpl> make_pc_learned_ic0(b2s_ctx* ctx, const CsrDev& A, const b2s_pc_opts& o)
{
    Gnn net;
    net.init(ctx, 0);
    std::string path = o.learned_weights ? std::string(o.learned_weights) : default_weight_path();
    if (!path.empty())
    {
        std::ifstream probe(path, std::ios::binary);
        if (probe.good() || o.learned_weights) load_weights(ctx, net, path.c_str());
    }
    return make_pc_learned_with(ctx, A, o, net);
}

// ------------------------------------------------------------ one training step

struct TrainBuffers
{
    DBuf<double> w, Aw, u, vres, qv, dL, scal;  // scal: [vv, aw2, scale, loss]
};

static void train_step(b2s_ctx* ctx, Gnn& net, const CsrDev& A, int nprobes, uint64_t seed, const double* host_probes,
                       double lr, bool update, double* loss_out, float* grad_out, int loss_kind, int ksweeps,
                       int fsweeps)
{
    need(nprobes > 0 && nprobes <= 64, B2S_INVALID_ARG, "nprobes must be 1..64");
    const uint32_t n = A.n;
    // base IC(0) factor (FP64; exact, or fsweeps fixed-point sweeps as deployed), its L^T structure
    b2s_pc_opts o;
    b2s_pc_opts_default(&o);
    o.factor_sweeps = fsweeps;
    if (fsweeps > 0) o.trsv = B2S_TRSV_JACOBI;  // the fixed-point factor comes with the sweep schedule
    auto base = make_pc_ic0(ctx, A, o);
    uint64_t sz[3];
    base->export_data(ctx, "ic0.L", sz, nullptr, nullptr, nullptr);
    const uint32_t Lnnz = (uint32_t)sz[1];
    std::vector<uint32_t> hLrp(n + 1), hLci(Lnnz);
    std::vector<double> hL0(Lnnz);
    base->export_data(ctx, "ic0.L", sz, hLrp.data(), hLci.data(), hL0.data());
    base->export_data(ctx, "ic0.LT", sz, nullptr, nullptr, nullptr);
    const uint32_t Tnnz = (uint32_t)sz[1];
    std::vector<uint32_t> hTrp(n + 1), hTci(Tnnz ? Tnnz : 1);
    std::vector<double> hTv(Tnnz ? Tnnz : 1);
    base->export_data(ctx, "ic0.LT", sz, hTrp.data(), hTci.data(), hTv.data());
    auto Lrp = upload(ctx, hLrp.data(), n + 1), Lci = upload(ctx, hLci.data(), Lnnz);
    auto L0 = upload(ctx, hL0.data(), Lnnz);
    auto Trp = upload(ctx, hTrp.data(), n + 1), Tci = upload(ctx, hTci.data(), hTci.size());
    DBuf<uint32_t> Tpos(hTci.size());
    B2S_LAUNCH(ctx, k_lt_positions, stream_grid(ctx, n), kThreads, 0, n, Trp.p, Tci.p, Lrp.p, Lci.p, Tpos.p);

    GnnGraph G;
    G.build(ctx, A, true);
    G.forward(ctx, net, A);
    DBuf<double> Lv(Lnnz), dL(Lnnz);
    DBuf<float> C(Lnnz), dC(Lnnz);
    G.head(ctx, net, A, Lrp.p, Lci.p, L0.p, Lv.p, C.p, (double*)nullptr);
    B2S_CUDA(cudaMemsetAsync(dL.p, 0, dL.bytes(), ctx->stream));

    TrainBuffers T;
    T.w.alloc(n);
    T.Aw.alloc(n);
    T.u.alloc(n);
    T.vres.alloc(n);
    T.qv.alloc(n);
    T.scal.alloc(4);
    // preconditioned-residual loss: M = L~ L~^T as an FP64 IC(0) on the same
    // pattern (its chunk-scheduled triangular solves), two more work vectors
    std::unique_ptr<PcImpl> M;
    DBuf<double> ya, yb;
    if (loss_kind == B2S_LOSS_PRECOND)
    {
        b2s_pc_opts o64;
        b2s_pc_opts_default(&o64);
        GivenFactor gf(Lv.p);
        M = make_pc_ic0_ex(ctx, A, o64, &gf);
        ya.alloc(n);
        yb.alloc(n);
    }
    // sweep loss: the k + 1 states of each sweep sequence and the adjoint work vectors
    std::vector<DBuf<double>> ys, zs;
    DBuf<double> hb, gb, gb2, ub;
    if (loss_kind == B2S_LOSS_SWEEPS)
    {
        need(ksweeps >= 0 && ksweeps <= 64, B2S_INVALID_ARG, "sweep loss: 0..64 sweeps");
        for (int s = 0; s <= ksweeps; ++s)
        {
            ys.emplace_back(n);
            zs.emplace_back(n);
        }
        hb.alloc(n);
        gb.alloc(n);
        gb2.alloc(n);
        ub.alloc(n);
    }
    B2S_CUDA(cudaMemsetAsync(T.scal.p, 0, T.scal.bytes(), ctx->stream));
    const unsigned gn = stream_grid(ctx, n);
    reserve_reduction(ctx, gn);
    for (int k = 0; k < nprobes; ++k)
    {
        if (host_probes)
            h2d(ctx, T.w.p, host_probes + (size_t)k * n, n * sizeof(double));
        else
        {
            B2S_LAUNCH(ctx, k_normal, gn, kThreads, 0, seed * 131 + k, n, T.w.p);
            if (k % 2 == 1)
                for (int s = 0; s < 10; ++s)
                {
                    spmv(ctx, A, T.w.p, T.Aw.p);
                    B2S_LAUNCH(ctx, k_jacobi_probe, gn, kThreads, 0, n, T.Aw.p, A.diag.p, T.w.p);
                }
        }
        spmv(ctx, A, T.w.p, T.Aw.p);
        if (loss_kind == B2S_LOSS_SWEEPS)
        {
            const int K = ksweeps;
            // y = F Aw (k sweeps of L~), z = F^T y (k sweeps of L~^T), e = w - z
            for (int s = 0; s <= K; ++s)
                B2S_LAUNCH(ctx, k_sw_lo, gn, kThreads, 0, n, Lrp.p, Lci.p, Lv.p, T.Aw.p,
                           s ? ys[s - 1].p : (const double*)nullptr, ys[s].p);
            for (int s = 0; s <= K; ++s)
                B2S_LAUNCH(ctx, k_sw_up, gn, kThreads, 0, n, Lrp.p, Trp.p, Tci.p, Tpos.p, Lv.p, ys[K].p,
                           s ? zs[s - 1].p : (const double*)nullptr, zs[s].p);
            B2S_LAUNCH(ctx, k_sub, gn, kThreads, 0, n, T.w.p, zs[K].p, T.vres.p);
            dot_dev(ctx, n, T.vres.p, T.vres.p, T.scal.p);
            dot_dev(ctx, n, T.w.p, T.w.p, T.scal.p + 1);
            B2S_LAUNCH(ctx, k_loss_scale, 1, 1, 0, T.scal.p, T.scal.p + 1, nprobes, T.scal.p + 2, T.scal.p + 3);
            // adjoint of z_K: g = -scale e; back through the upper sweeps (ub collects the rhs adjoint)
            B2S_LAUNCH(ctx, k_neg_scale, gn, kThreads, 0, n, T.vres.p, T.scal.p + 2, gb.p);
            B2S_CUDA(cudaMemsetAsync(ub.p, 0, ub.bytes(), ctx->stream));
            for (int s = K; s >= 0; --s)
            {
                B2S_LAUNCH(ctx, k_sw_h, gn, kThreads, 0, n, Lrp.p, Lv.p, gb.p, zs[s].p, hb.p, ub.p, dL.p);
                if (s == 0) break;
                B2S_LAUNCH(ctx, k_sw_up_adj, gn, kThreads, 0, n, Lrp.p, Lci.p, Lv.p, hb.p, zs[s - 1].p, gb2.p, dL.p);
                std::swap(gb, gb2);
            }
            // back through the lower sweeps from y_K's adjoint ub (Aw is a constant)
            for (int s = K; s >= 0; --s)
            {
                B2S_LAUNCH(ctx, k_sw_h, gn, kThreads, 0, n, Lrp.p, Lv.p, ub.p, ys[s].p, hb.p, (double*)nullptr, dL.p);
                if (s == 0) break;
                B2S_LAUNCH(ctx, k_sw_lo_adj, gn, kThreads, 0, n, Trp.p, Tci.p, Tpos.p, Lv.p, hb.p, ys[s - 1].p,
                           gb2.p, dL.p);
                std::swap(ub, gb2);
            }
            continue;
        }
        if (loss_kind == B2S_LOSS_PRECOND)
        {
            // y = L~^-1 Aw (u), z = L~^-T y (qv), e = w - z (vres)
            M->solve_factor(ctx, false, T.Aw.p, T.u.p, nullptr);
            M->solve_factor(ctx, true, T.u.p, T.qv.p, nullptr);
            B2S_LAUNCH(ctx, k_sub, gn, kThreads, 0, n, T.w.p, T.qv.p, T.vres.p);
            dot_dev(ctx, n, T.vres.p, T.vres.p, T.scal.p);
            dot_dev(ctx, n, T.w.p, T.w.p, T.scal.p + 1);
            B2S_LAUNCH(ctx, k_loss_scale, 1, 1, 0, T.scal.p, T.scal.p + 1, nprobes, T.scal.p + 2, T.scal.p + 3);
            // g = -scale e (Aw is free now), a = L~^-1 g, b = L~^-T a
            B2S_LAUNCH(ctx, k_neg_scale, gn, kThreads, 0, n, T.vres.p, T.scal.p + 2, T.Aw.p);
            M->solve_factor(ctx, false, T.Aw.p, ya.p, nullptr);
            M->solve_factor(ctx, true, ya.p, yb.p, nullptr);
            B2S_LAUNCH(ctx, k_dL_pc, gn, kThreads, 0, n, Lrp.p, Lci.p, T.qv.p, ya.p, yb.p, T.u.p, dL.p);
            continue;
        }
        dot_dev(ctx, n, T.Aw.p, T.Aw.p, T.scal.p + 1);
        B2S_LAUNCH(ctx, k_ltmul, gn, kThreads, 0, n, Lrp.p, Trp.p, Tci.p, Tpos.p, Lv.p, T.w.p, T.u.p);
        B2S_LAUNCH(ctx, k_lmul_res, gn, kThreads, 0, n, Lrp.p, Lci.p, Lv.p, T.u.p, T.Aw.p, T.vres.p, T.scal.p,
                   ctx->partial.p, ctx->counter.p);
        B2S_LAUNCH(ctx, k_loss_scale, 1, 1, 0, T.scal.p, T.scal.p + 1, nprobes, T.scal.p + 2, T.scal.p + 3);
        B2S_LAUNCH(ctx, k_ltmul, gn, kThreads, 0, n, Lrp.p, Trp.p, Tci.p, Tpos.p, Lv.p, T.vres.p, T.qv.p);
        B2S_LAUNCH(ctx, k_dL, gn, kThreads, 0, n, Lrp.p, Lci.p, T.vres.p, T.u.p, T.w.p, T.qv.p, T.scal.p + 2, dL.p);
    }
    B2S_LAUNCH(ctx, k_head_dc, stream_grid(ctx, Lnnz), kThreads, 0, Lnnz, dL.p, Lv.p, L0.p, C.p, dC.p);

    // backward
    const unsigned gw = (n + 7) / 8, g64 = (n + kBwdRows - 1) / kBwdRows;
    B2S_CUDA(cudaMemsetAsync(net.g.p, 0, net.g.bytes(), ctx->stream));
    DBuf<float> dH(n * (size_t)H), dH2(n * (size_t)H), dSM(n * (size_t)2 * H), part;
    part.alloc((size_t)std::max<unsigned>(gw, 1) * (H * (FE + 2) > O_SIZE ? H * (FE + 2) : O_SIZE) + 16);
    B2S_LAUNCH(ctx, k_head_bwd, gw, 256, 0, n, Lrp.p, Lci.p, Trp.p, Tpos.p, A.rp.p, G.EF.p, G.Hs[NL].p, net.pr.p,
               dC.p, dH.p, part.p);
    B2S_LAUNCH(ctx, k_reduce_partials, 1, 256, 0, gw, (uint32_t)O_SIZE, (uint32_t)O_SIZE, part.p, net.g.p + OFF_OUT, 0);
    const uint32_t rows_per = 2048;
    const unsigned gwb = (n + rows_per - 1) / rows_per;
    DBuf<float> wpart((size_t)gwb * (2 * H * H + 2 * H) + 16), red(H * (FE + 2));
    for (int l = NL - 1; l >= 0; --l)
    {
        const __nv_bfloat16* Wl = net.pb.p + LAYER0 + l * L_SIZE;
        float* gl = net.g.p + LAYER0 + l * L_SIZE;
        // dH (wrt H_{l+1}) -> dpre, dSM, residual into dH2
        B2S_LAUNCH(ctx, k_aggregate_bwd, gw, 256, 0, n, A.rp.p, A.ci.p, G.rev.p, G.EF.p, G.invdeg.p, G.SM[l].p, Wl,
                   G.pre[l].p, dH.p, dSM.p, dH2.p, part.p);
        // per-CTA gate partials -> ordered sum -> layer layout
        B2S_LAUNCH(ctx, k_reduce_partials, 2, 256, 0, gw, (uint32_t)(H * (FE + 2)), (uint32_t)(H * (FE + 2)), part.p,
                   red.p, 0);
        B2S_LAUNCH(ctx, k_gate_grads, 1, 64, 0, red.p, gl);
        // weights [W_s; W_m] (128 x 64): dW = dSM^T H_l ; dH_l += dSM W
        B2S_LAUNCH(ctx, (k_linear_bwd_weight<H, 2 * H, true>), gwb, 256, 0, n, rows_per, dSM.p, G.Hs[l].p, wpart.p);
        B2S_LAUNCH(ctx, k_reduce_partials, 64, 256, 0, gwb, (uint32_t)(2 * H * H + 2 * H), (uint32_t)(2 * H * H),
                   wpart.p, gl + L_WS, 0);
        B2S_LAUNCH(ctx, (k_linear_bwd_data<H, 2 * H>), g64, 256, 0, n, dSM.p, Wl + L_WS, dH2.p, 1);
        std::swap(dH, dH2);
    }
    // input layer: dpre0 = dH0 * (pre0 > 0) ; dW_in = dpre0^T F ; db_in
    B2S_LAUNCH(ctx, k_relu_mask, stream_grid(ctx, (uint64_t)n * H), kThreads, 0, (uint64_t)n * H, G.pre0.p, dH.p,
               dSM.p);
    B2S_LAUNCH(ctx, (k_linear_bwd_weight<FIN, H, false>), gwb, 256, 0, n, rows_per, dSM.p, G.F.p, wpart.p);
    B2S_LAUNCH(ctx, k_reduce_partials, 4, 256, 0, gwb, (uint32_t)(H * FIN + H), (uint32_t)(H * FIN + H), wpart.p,
               net.g.p + OFF_WIN, 0);

    double lossv = 0;
    d2h(ctx, &lossv, T.scal.p + 3, sizeof(double));
    if (grad_out) d2h(ctx, grad_out, net.g.p, NPARAM * sizeof(float));
    G.check(ctx);
    if (loss_out) *loss_out = lossv;
    if (update)
    {
        net.step += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - std::pow(b1, (float)net.step), c2 = 1.f - std::pow(b2, (float)net.step);
        B2S_LAUNCH(ctx, k_adam, stream_grid(ctx, NPARAM), kThreads, 0, (uint32_t)NPARAM, net.p.p, net.g.p, net.m.p,
                   net.v.p, (float)lr, b1, b2, 1e-8f, c1, c2, net.pb.p);
        B2S_LAUNCH(ctx, k_to_bf16, stream_grid(ctx, NPARAM), kThreads, 0, (uint32_t)NPARAM, net.p.p, net.pb.p, net.pr.p);
        sync(ctx);
    }
}

}  // namespace b2s

using namespace b2s;

extern "C" {

b2s_status b2s_learner_create(b2s_ctx* ctx, uint64_t seed, b2s_learner** out)
{
    if (!ctx || !out) return B2S_INVALID_ARG;
    *out = nullptr;
    b2s_learner* L = new b2s_learner();
    L->ctx = ctx;
    b2s_status st = guarded(ctx, [&] {
        B2S_CUDA(cudaSetDevice(ctx->device));
        L->net.init(ctx, seed);
        sync(ctx);
    });
    if (st != B2S_OK)
    {
        delete L;
        return st;
    }
    *out = L;
    return B2S_OK;
}

b2s_status b2s_learner_destroy(b2s_learner* L)
{
    if (!L) return B2S_INVALID_ARG;
    cudaSetDevice(L->ctx->device);
    delete L;
    return B2S_OK;
}

b2s_status b2s_learner_load(b2s_learner* L, const char* path)
{
    if (!L || !path) return B2S_INVALID_ARG;
    return guarded(L->ctx, [&] { load_weights(L->ctx, L->net, path); sync(L->ctx); });
}

b2s_status b2s_learner_save(b2s_learner* L, const char* path)
{
    if (!L || !path) return B2S_INVALID_ARG;
    return guarded(L->ctx, [&] { save_weights(L->ctx, L->net, path); });
}

b2s_status b2s_learner_params(b2s_learner* L, float* params, uint64_t* count, int set)
{
    if (!L || !count) return B2S_INVALID_ARG;
    if (!params)
    {
        *count = NPARAM;
        return B2S_OK;
    }
    if (*count != (uint64_t)NPARAM) return B2S_SHAPE;
    return guarded(L->ctx, [&] {
        if (set)
            L->net.set(L->ctx, params);
        else
            d2h(L->ctx, params, L->net.p.p, NPARAM * sizeof(float));
        sync(L->ctx);
    });
}

b2s_status b2s_learner_step(b2s_ctx* ctx, b2s_learner* L, const b2s_csr* A, int nprobes, uint64_t seed,
                            const double* probes, double lr, int update, double* loss, float* grad)
{
    if (!ctx || !L || !A) return B2S_INVALID_ARG;
    return guarded(ctx, [&] {
        need(A->d.n == A->d.m, B2S_SHAPE, "learned IC(0) needs a square matrix");
        train_step(ctx, L->net, A->d, nprobes, seed, probes, lr, update != 0, loss, grad, L->loss, L->trsv_sweeps,
                   L->factor_sweeps);
        check_device_error(ctx, "a triangular-solve wait gave up during the training step");
    });
}

b2s_status b2s_learner_set_loss(b2s_learner* L, int kind)
{
    if (!L || (kind != B2S_LOSS_PRECOND && kind != B2S_LOSS_FACTOR && kind != B2S_LOSS_SWEEPS))
        return B2S_INVALID_ARG;
    L->loss = kind;
    return B2S_OK;
}

b2s_status b2s_learner_set_sweeps(b2s_learner* L, int trsv_sweeps, int factor_sweeps)
{
    if (!L || trsv_sweeps < 0 || trsv_sweeps > 64 || factor_sweeps < 0 || factor_sweeps > 1024)
        return B2S_INVALID_ARG;
    L->trsv_sweeps = trsv_sweeps;
    L->factor_sweeps = factor_sweeps;
    return B2S_OK;
}

b2s_status b2s_dense_bf16_device(b2s_ctx* ctx, uint64_t n, int k, int no, const float* d_x, const uint16_t* d_w,
                                 const float* d_bias, float* d_y)
{
    if (!ctx) return B2S_INVALID_ARG;
    if (n && (!d_x || !d_w || !d_y)) return B2S_INVALID_ARG;
    if (n > UINT32_MAX - tc::kTileRows) return B2S_UNSUPPORTED;
    return guarded(ctx, [&] {
        const auto* w = reinterpret_cast<const __nv_bfloat16*>(d_w);
        if (k == 64 && no == 128)
            linear_tc<64, 128>(ctx, (uint32_t)n, d_x, w, d_bias, d_y, ctx->errword());
        else if (k == 64 && no == 64)
            linear_tc<64, 64>(ctx, (uint32_t)n, d_x, w, d_bias, d_y, ctx->errword());
        else
            fail(B2S_UNSUPPORTED, "dense layer: supported shapes are k = 64 with no = 128 or 64");
    });
}

b2s_status b2s_pc_create_learned(b2s_ctx* ctx, const b2s_csr* A, b2s_learner* L, const b2s_pc_opts* opts,
                                 b2s_pc** out)
{
    if (!ctx || !A || !L || !out) return B2S_INVALID_ARG;
    *out = nullptr;
    b2s_pc_opts o;
    b2s_pc_opts_default(&o);
    if (opts) o = *opts;
    b2s_pc* pc = new b2s_pc();
    pc->ctx = ctx;
    pc->kind = B2S_PC_LEARNED_IC0;
    pc->n = A->d.n;
    b2s_status st = guarded(ctx, [&] {
        need(A->d.n == A->d.m, B2S_SHAPE, "learned IC(0) needs a square matrix");
        pc->impl = make_pc_learned_with(ctx, A->d, o, L->net);
        sync(ctx);
        check_device_error(ctx, "a device-side wait gave up during the set-up");
    });
    if (st != B2S_OK)
    {
        delete pc;
        return st;
    }
    *out = pc;
    return B2S_OK;
}

}  // extern "C"
