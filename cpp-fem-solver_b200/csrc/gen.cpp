// Host-side problem generators for the benchmark configurations and tests.
//
// All generators are deterministic: the same arguments give the same
// matrices bit for bit.  Random numbers come from splitmix64 used as a
// counter-based generator (Steele, Lea & Flood 2014): value i of stream `seed`
// is splitmix64(seed * 0x9E3779B97F4A7C15 + i), mapped to [0, 1) through its
// top 53 bits.  Normal deviates use the Box-Muller transform.
//
// The 2-D Poisson and convection-diffusion stencils follow the reference's
// test generators (test_SMatrix_pcg.cpp:70-99, test_SMatrix_gmres.cpp:75-112);
// the 3-D, elasticity and random-coefficient generators have no counterpart
// in the reference.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

#include "b2s.h"

namespace {

inline uint64_t splitmix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

inline double u01(uint64_t seed, uint64_t i)
{
    return (double)(splitmix64(seed * 0x9E3779B97F4A7C15ull + i) >> 11) * (1.0 / 9007199254740992.0);
}

// CSR builder from per-row sorted (col, val) lists
struct CsrOut
{
    uint32_t* n;
    uint32_t* nnz;
    uint32_t* rp;
    uint32_t* ci;
    double* v;
};

template <typename RowFn>
b2s_status emit_csr(uint32_t n, CsrOut o, RowFn&& row)
{
    // row(i, cols, vals, &cnt) fills up to 16 sorted entries
    uint32_t cols[32];
    double vals[32];
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; ++i)
    {
        uint32_t cnt = 0;
        row(i, cols, vals, cnt);
        total += cnt;
    }
    if (total > 0xFFFFFFFFull) return B2S_UNSUPPORTED;
    *o.n = n;
    *o.nnz = (uint32_t)total;
    if (!o.rp) return B2S_OK;
    uint32_t k = 0;
    o.rp[0] = 0;
    for (uint32_t i = 0; i < n; ++i)
    {
        uint32_t cnt = 0;
        row(i, cols, vals, cnt);
        for (uint32_t t = 0; t < cnt; ++t)
        {
            o.ci[k] = cols[t];
            o.v[k] = vals[t];
            ++k;
        }
        o.rp[i + 1] = k;
    }
    return B2S_OK;
}

// in-place iterative radix-2 complex FFT (forward: sign -1)
void fft1d(std::complex<double>* a, size_t n, int sign)
{
    for (size_t i = 1, j = 0; i < n; ++i)
    {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (size_t len = 2; len <= n; len <<= 1)
    {
        const double ang = sign * 2.0 * M_PI / (double)len;
        for (size_t i = 0; i < n; i += len)
            for (size_t k = 0; k < len / 2; ++k)
            {
                const std::complex<double> w(std::cos(ang * (double)k), std::sin(ang * (double)k));
                const std::complex<double> u = a[i + k], t = w * a[i + k + len / 2];
                a[i + k] = u + t;
                a[i + k + len / 2] = u - t;
            }
    }
}

void fft2d(std::vector<std::complex<double>>& a, size_t M, int sign)
{
    for (size_t r = 0; r < M; ++r) fft1d(&a[r * M], M, sign);
    std::vector<std::complex<double>> col(M);
    for (size_t c = 0; c < M; ++c)
    {
        for (size_t r = 0; r < M; ++r) col[r] = a[r * M + c];
        fft1d(col.data(), M, sign);
        for (size_t r = 0; r < M; ++r) a[r * M + c] = col[r];
    }
}

// 24x24 stiffness of a cube element of edge h (trilinear Q1, isotropic,
// 2x2x2 Gauss).  Local node a = (ax, ay, az) in {0,1}^3, index ax + 2 ay + 4 az;
// dof 3a + d.
void q1_element(double h, double E, double nu, double Ke[24][24])
{
    const double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = E / (2.0 * (1.0 + nu));
    double D[6][6] = {};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) D[i][j] = lam;
    for (int i = 0; i < 3; ++i) D[i][i] += 2.0 * mu;
    for (int i = 3; i < 6; ++i) D[i][i] = mu;
    std::memset(Ke, 0, sizeof(double) * 24 * 24);
    const double gp = 1.0 / std::sqrt(3.0);
    for (int gz = 0; gz < 2; ++gz)
        for (int gy = 0; gy < 2; ++gy)
            for (int gx = 0; gx < 2; ++gx)
            {
                const double xi[3] = {gx ? gp : -gp, gy ? gp : -gp, gz ? gp : -gp};
                // shape-function gradients in physical coordinates (Jacobian h/2 I)
                double dN[8][3];
                for (int a = 0; a < 8; ++a)
                {
                    const double s[3] = {(a & 1) ? 1.0 : -1.0, (a & 2) ? 1.0 : -1.0, (a & 4) ? 1.0 : -1.0};
                    for (int d = 0; d < 3; ++d)
                    {
                        double g = 0.125 * s[d];
                        for (int e = 0; e < 3; ++e)
                            if (e != d) g *= (1.0 + s[e] * xi[e]);
                        dN[a][d] = g * (2.0 / h);
                    }
                }
                double B[6][24] = {};
                for (int a = 0; a < 8; ++a)
                {
                    B[0][3 * a + 0] = dN[a][0];
                    B[1][3 * a + 1] = dN[a][1];
                    B[2][3 * a + 2] = dN[a][2];
                    B[3][3 * a + 0] = dN[a][1];
                    B[3][3 * a + 1] = dN[a][0];
                    B[4][3 * a + 1] = dN[a][2];
                    B[4][3 * a + 2] = dN[a][1];
                    B[5][3 * a + 0] = dN[a][2];
                    B[5][3 * a + 2] = dN[a][0];
                }
                const double w = (h / 2.0) * (h / 2.0) * (h / 2.0);  // det J, Gauss weights 1
                double DB[6][24];
                for (int i = 0; i < 6; ++i)
                    for (int j = 0; j < 24; ++j)
                    {
                        double s = 0.0;
                        for (int k = 0; k < 6; ++k) s += D[i][k] * B[k][j];
                        DB[i][j] = s;
                    }
                for (int i = 0; i < 24; ++i)
                    for (int j = 0; j < 24; ++j)
                    {
                        double s = 0.0;
                        for (int k = 0; k < 6; ++k) s += B[k][i] * DB[k][j];
                        Ke[i][j] += w * s;
                    }
            }
}

}  // namespace

extern "C" {

b2s_status b2s_gen_uniform(uint64_t seed, uint64_t n, double* out)
{
    if (n && !out) return B2S_INVALID_ARG;
    for (uint64_t i = 0; i < n; ++i) out[i] = 2.0 * u01(seed, i) - 1.0;
    return B2S_OK;
}

b2s_status b2s_gen_poisson2d(uint32_t N, uint32_t* n, uint32_t* nnz, uint32_t* rp, uint32_t* ci, double* v)
{
    if (!n || !nnz || N == 0 || (uint64_t)N * N > 0xFFFFFFFFull) return B2S_INVALID_ARG;
    return emit_csr(N * N, CsrOut{n, nnz, rp, ci, v}, [&](uint32_t idx, uint32_t* c, double* val, uint32_t& k) {
        const uint32_t i = idx / N, j = idx % N;
        if (i > 0) { c[k] = idx - N; val[k++] = -1.0; }
        if (j > 0) { c[k] = idx - 1; val[k++] = -1.0; }
        c[k] = idx; val[k++] = 4.0;
        if (j < N - 1) { c[k] = idx + 1; val[k++] = -1.0; }
        if (i < N - 1) { c[k] = idx + N; val[k++] = -1.0; }
    });
}

b2s_status b2s_gen_convdiff3d(uint32_t N, double vx, double vy, double vz, uint32_t* n, uint32_t* nnz, uint32_t* rp,
                              uint32_t* ci, double* v)
{
    if (!n || !nnz || N == 0 || (uint64_t)N * N * N > 0xFFFFFFFFull) return B2S_INVALID_ARG;
    const uint32_t NN = N * N;
    return emit_csr(NN * N, CsrOut{n, nnz, rp, ci, v}, [&](uint32_t idx, uint32_t* c, double* val, uint32_t& k) {
        const uint32_t i = idx % N, j = (idx / N) % N, kk = idx / NN;
        if (kk > 0) { c[k] = idx - NN; val[k++] = -1.0 - vz; }
        if (j > 0) { c[k] = idx - N; val[k++] = -1.0 - vy; }
        if (i > 0) { c[k] = idx - 1; val[k++] = -1.0 - vx; }
        c[k] = idx; val[k++] = 6.0 + vx + vy + vz;
        if (i < N - 1) { c[k] = idx + 1; val[k++] = -1.0; }
        if (j < N - 1) { c[k] = idx + N; val[k++] = -1.0; }
        if (kk < N - 1) { c[k] = idx + NN; val[k++] = -1.0; }
    });
}

b2s_status b2s_gen_poisson3d(uint32_t N, uint32_t* n, uint32_t* nnz, uint32_t* rp, uint32_t* ci, double* v)
{
    return b2s_gen_convdiff3d(N, 0.0, 0.0, 0.0, n, nnz, rp, ci, v);
}

b2s_status b2s_gen_elasticity_q1(uint32_t NE, double E, double nu, uint32_t* nbr, uint32_t* nnzb, uint32_t* rp,
                                 uint32_t* ci, double* v)
{
    if (!nbr || !nnzb || NE == 0 || NE > 1000) return B2S_INVALID_ARG;
    const uint32_t P = NE + 1;  // nodes per direction
    static thread_local double Ke[24][24];
    q1_element(1.0 / NE, E, nu, Ke);
    // free nodes: ix > 0 (the x = 0 face is clamped); node-major numbering
    auto free_id = [&](uint32_t ix, uint32_t iy, uint32_t iz) -> uint32_t {
        return (iz * P + iy) * NE + (ix - 1);
    };
    const uint32_t nb = NE * P * P;
    uint64_t total = 0;
    if (rp) rp[0] = 0;
    uint32_t k = 0;
    for (uint32_t iz = 0; iz < P; ++iz)
        for (uint32_t iy = 0; iy < P; ++iy)
            for (uint32_t ix = 1; ix < P; ++ix)
            {
                // neighbours in ascending free-id order: dz, dy, dx loops
                for (int dz = -1; dz <= 1; ++dz)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dx = -1; dx <= 1; ++dx)
                        {
                            const int jx = (int)ix + dx, jy = (int)iy + dy, jz = (int)iz + dz;
                            if (jx < 1 || jy < 0 || jz < 0 || jx >= (int)P || jy >= (int)P || jz >= (int)P) continue;
                            ++total;
                            if (!rp) continue;
                            ci[k] = free_id(jx, jy, jz);
                            double* blk = v + (size_t)k * 9;
                            for (int t = 0; t < 9; ++t) blk[t] = 0.0;
                            // elements containing both nodes: min corner e in [max(i,j)-1, min(i,j)]
                            for (int ez = std::max((int)iz, jz) - 1; ez <= std::min((int)iz, jz); ++ez)
                                for (int ey = std::max((int)iy, jy) - 1; ey <= std::min((int)iy, jy); ++ey)
                                    for (int ex = std::max((int)ix, jx) - 1; ex <= std::min((int)ix, jx); ++ex)
                                    {
                                        if (ex < 0 || ey < 0 || ez < 0 || ex >= (int)NE || ey >= (int)NE ||
                                            ez >= (int)NE)
                                            continue;
                                        const int la = ((int)ix - ex) + 2 * ((int)iy - ey) + 4 * ((int)iz - ez);
                                        const int lb = (jx - ex) + 2 * (jy - ey) + 4 * (jz - ez);
                                        for (int r = 0; r < 3; ++r)
                                            for (int c = 0; c < 3; ++c) blk[r * 3 + c] += Ke[3 * la + r][3 * lb + c];
                                    }
                            ++k;
                        }
                if (rp) rp[free_id(ix, iy, iz) + 1] = k;
            }
    if (total > 0xFFFFFFFFull) return B2S_UNSUPPORTED;
    *nbr = nb;
    *nnzb = (uint32_t)total;
    return B2S_OK;
}

b2s_status b2s_gen_grf_diffusion(uint32_t N, double corr, double var, uint64_t seed, uint32_t* n, uint32_t* nnz,
                                 uint32_t* rp, uint32_t* ci, double* v, double* kfield)
{
    if (!n || !nnz || N < 2 || N > 8192 || !(corr > 0) || !(var >= 0)) return B2S_INVALID_ARG;
    const uint32_t NN = N * N;
    *n = NN;
    *nnz = 5 * NN - 4 * N;
    if (!rp && !kfield) return B2S_OK;
    // log k on cell centres: circulant embedding on a 2N-periodic torus
    size_t M = 1;
    while (M < 2 * (size_t)N) M <<= 1;
    const double h = 1.0 / N;
    std::vector<std::complex<double>> c(M * M);
    for (size_t p = 0; p < M; ++p)
        for (size_t q = 0; q < M; ++q)
        {
            const double dx = (double)std::min(p, M - p) * h, dy = (double)std::min(q, M - q) * h;
            c[p * M + q] = var * std::exp(-(dx * dx + dy * dy) / (2.0 * corr * corr));
        }
    fft2d(c, M, -1);  // eigenvalues of the circulant covariance
    std::vector<std::complex<double>> w(M * M);
    for (size_t t = 0; t < M * M; ++t)
    {
        const double lam = std::max(c[t].real(), 0.0);
        const double u1 = std::max(u01(seed ^ 0x5DEECE66Dull, 2 * t), 1e-300), u2 = u01(seed ^ 0x5DEECE66Dull, 2 * t + 1);
        const double rad = std::sqrt(-2.0 * std::log(u1)), th = 2.0 * M_PI * u2;
        w[t] = std::sqrt(lam / (double)(M * M)) * std::complex<double>(rad * std::cos(th), rad * std::sin(th));
    }
    fft2d(w, M, -1);
    std::vector<double> kc(NN);
    for (uint32_t i = 0; i < N; ++i)
        for (uint32_t j = 0; j < N; ++j) kc[(size_t)i * N + j] = std::exp(w[(size_t)i * M + j].real());
    if (kfield) std::memcpy(kfield, kc.data(), sizeof(double) * NN);
    if (!rp) return B2S_OK;
    auto face = [](double a, double b) { return 2.0 * a * b / (a + b); };
    uint32_t k = 0;
    rp[0] = 0;
    for (uint32_t idx = 0; idx < NN; ++idx)
    {
        const uint32_t i = idx / N, j = idx % N;
        const double kp = kc[idx];
        double diag = 0.0;
        double fs = 0, fw = 0, fe = 0, fn = 0;
        fs = i > 0 ? face(kp, kc[idx - N]) : 2.0 * kp;
        fw = j > 0 ? face(kp, kc[idx - 1]) : 2.0 * kp;
        fe = j < N - 1 ? face(kp, kc[idx + 1]) : 2.0 * kp;
        fn = i < N - 1 ? face(kp, kc[idx + N]) : 2.0 * kp;
        diag = ((fs + fw) + fe) + fn;
        if (i > 0) { ci[k] = idx - N; v[k++] = -fs; }
        if (j > 0) { ci[k] = idx - 1; v[k++] = -fw; }
        ci[k] = idx; v[k++] = diag;
        if (j < N - 1) { ci[k] = idx + 1; v[k++] = -fe; }
        if (i < N - 1) { ci[k] = idx + N; v[k++] = -fn; }
        rp[idx + 1] = k;
    }
    return B2S_OK;
}

}  // extern "C"
