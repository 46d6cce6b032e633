// CPU replay of the tiled persistent PCG kernel's index arithmetic
// (cpp-fem-solver_b200/csrc/pcg_tile.cuh) over plans made by plan_tiles
// (tile_plan.hpp).  For 5-point patterns on N x N grids (the kernel's target)
// and for a general banded pattern, every tile's sweeps are replayed with
// bounds-checked local reads exactly as the kernel orders them, and the
// owned rows must equal the global sweep definition bit for bit (FP32, no
// contraction); the SpMV over local columns must equal the CSR product in
// column order (FP64); every blob segment and work buffer must lie inside
// the planned shared memory.  Exit status 0 when every check holds.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "../../cpp-fem-solver_b200/csrc/tile_plan.hpp"

using namespace b2s;

static int fails = 0;
#define CHECK(c, ...)                \
    do                               \
    {                                \
        if (!(c))                    \
        {                            \
            std::printf(__VA_ARGS__); \
            std::printf("\n");       \
            if (++fails > 20) std::exit(1); \
        }                            \
    } while (0)

struct Pattern
{
    uint32_t n;
    std::vector<uint32_t> lrp, lci, urp, uci;  // strict lower / strict upper (transpose)
};

static Pattern five_point(uint32_t N, uint32_t M = 0)
{
    if (!M) M = N;  // N columns, M grid rows
    Pattern P;
    P.n = N * M;
    P.lrp.assign(P.n + 1, 0);
    for (uint32_t i = 0; i < P.n; ++i)
    {
        const uint32_t x = i % N, y = i / N;
        if (y > 0) P.lci.push_back(i - N);
        if (x > 0) P.lci.push_back(i - 1);
        P.lrp[i + 1] = (uint32_t)P.lci.size();
    }
    strict_transpose(P.n, P.lrp.data(), P.lci.data(), true, P.urp, P.uci);
    return P;
}

// rows with up to two strict lower entries at offsets 1..B (random), a band
static Pattern banded(uint32_t n, uint32_t B, unsigned seed)
{
    Pattern P;
    P.n = n;
    std::mt19937 g(seed);
    P.lrp.assign(n + 1, 0);
    for (uint32_t i = 0; i < n; ++i)
    {
        std::vector<uint32_t> c;
        for (int e = 0; e < 2; ++e)
        {
            const uint32_t o = 1 + g() % B;
            if (o <= i && std::find(c.begin(), c.end(), i - o) == c.end()) c.push_back(i - o);
        }
        std::sort(c.begin(), c.end());
        for (uint32_t j : c) P.lci.push_back(j);
        P.lrp[i + 1] = (uint32_t)P.lci.size();
    }
    strict_transpose(n, P.lrp.data(), P.lci.data(), true, P.urp, P.uci);
    return P;
}

// global sweeps: pass 0 y = rhs * dinv, pass s y = (rhs - sum v yprev) * dinv
static std::vector<float> sweeps(const std::vector<uint32_t>& rp, const std::vector<uint32_t>& ci,
                                 const std::vector<float>& v, const std::vector<float>& dinv,
                                 const std::vector<float>& rhs, int k)
{
    const uint32_t n = (uint32_t)rhs.size();
    std::vector<float> y(n), yn(n);
    for (uint32_t i = 0; i < n; ++i) y[i] = rhs[i] * dinv[i];
    for (int s = 1; s <= k; ++s)
    {
        for (uint32_t i = 0; i < n; ++i)
        {
            float sum = rhs[i];
            for (uint32_t e = rp[i]; e < rp[i + 1]; ++e) sum -= v[e] * y[ci[e]];
            yn[i] = sum * dinv[i];
        }
        y.swap(yn);
    }
    return y;
}

static void check_plan(const char* name, const Pattern& P, int k, int sms, uint32_t smem_limit, bool expect_ok)
{
    const uint32_t n = P.n;
    TilePlan T = plan_tiles(n, P.lrp.data(), P.lci.data(), P.urp.data(), P.uci.data(), k, sms, smem_limit, 4);
    std::printf("%-22s n=%u k=%d: ok=%d fused=%d tiles=%u (%ux%u) B=%u Q=%u max_ext=%u smem=%u\n", name, n, k, T.ok,
                T.fused, T.ntiles, T.tiles_x, T.tiles_y, T.B, T.Q, T.max_ext, T.smem);
    CHECK(T.ok == expect_ok, "%s: plan ok=%d, expected %d", name, T.ok, expect_ok);
    if (!T.ok) return;
    CHECK(T.ntiles <= (uint32_t)sms && T.ntiles <= (uint32_t)kTileMaxTiles, "%s: too many tiles", name);
    CHECK(T.smem <= smem_limit && T.Q >= 1 && T.Q <= kTileMaxQ, "%s: smem/Q", name);
    CHECK((size_t)T.Q * kTileThreads >= T.max_ext, "%s: Q too small", name);
    std::mt19937 g(7);
    std::uniform_real_distribution<float> U(-0.5f, 0.5f);
    std::vector<float> lv(P.lci.size()), uv(P.uci.size()), ld(n), ud(n), r(n);
    for (auto& x : lv) x = U(g);
    for (auto& x : uv) x = U(g);
    for (uint32_t i = 0; i < n; ++i)
    {
        ld[i] = 1.0f / (2.0f + U(g));
        ud[i] = 1.0f / (2.0f + U(g));
        r[i] = U(g);
    }
    const std::vector<float> yl = sweeps(P.lrp, P.lci, lv, ld, r, k);
    const std::vector<float> yu = sweeps(P.urp, P.uci, uv, ud, yl, k);
    // A = [strict lower | diag | strict upper] in column order, FP64
    std::vector<double> pg(n);
    for (auto& x : pg) x = (double)U(g);
    std::vector<uint32_t> seen(n, 0);
    const uint32_t ystride = tile_ystride(T.max_ext);
    CHECK(ystride > T.max_ext, "%s: no spare sweep slot", name);
    for (uint32_t t = 0; t < T.ntiles; ++t)
    {
        const TileDesc& D = T.desc[t];
        const uint8_t* ib = T.idx.data() + D.ibase;
        // the blobs and the work buffers inside the planned shared memory
        CHECK(D.vbytes % 16 == 0 && D.ibytes % 16 == 0 && D.vbase % 16 == 0 && D.ibase % 16 == 0, "align");
        CHECK(D.vbytes + D.ibytes <= T.work, "%s tile %u: blobs past the work buffers", name, t);
        CHECK(T.work + 8ull * ystride <= T.smem && T.work + 8ull * D.n_ae <= T.smem, "%s: work buffers", name);
        CHECK(D.o_aval + 8ull * D.nnz <= D.vbytes && D.o_udinv + 4ull * D.n_eu <= D.vbytes, "value segments");
        CHECK(D.o_acol + 2ull * D.nnz <= D.ibytes && D.o_arp + 4ull * (D.n_own + 1) <= D.ibytes, "index segments");
        CHECK(D.ibase + D.ibytes <= T.idx.size(), "index blob inside");
        auto u32 = [&](uint32_t off, uint32_t i) {
            uint32_t v;
            std::memcpy(&v, ib + off + 4ull * i, 4);
            return v;
        };
        auto u16 = [&](uint32_t off, uint32_t i) {
            uint16_t v;
            std::memcpy(&v, ib + off + 2ull * i, 2);
            return (uint32_t)v;
        };
        for (uint32_t q = 0; q < D.n_own; ++q) seen[u32(D.o_owned, q)]++;
        // one triangle's sweeps as the kernel runs them (local buffers, prefix per
        // pass); local_rhs: the right-hand side of rows t < its size taken from
        // the CTA (a fused plan's backward sweeps), not from the global vector
        auto replay = [&](bool lower, uint32_t ne, const uint16_t* cnt, uint32_t o_halo, uint32_t o_deps,
                          const std::vector<uint32_t>& rp, const std::vector<uint32_t>& ci, const std::vector<float>& v,
                          const std::vector<float>& dinv, const std::vector<float>& rhs, const std::vector<float>& want,
                          uint32_t check_rows, const std::vector<float>* local_rhs) {
            const uint32_t base = lower ? cnt[0] : D.n_own;  // rows of the layer-0 set
            CHECK(cnt[0] == (lower && T.fused ? D.n_eu : D.n_own) && cnt[k] == ne, "%s: layer counts", name);
            auto glob = [&](uint32_t tl) {
                return tl < D.n_own ? u32(D.o_owned, tl) : tl < base ? u32(D.o_uhalo, tl - D.n_own) : u32(o_halo, tl - base);
            };
            std::vector<float> y0(ystride, NAN), y1(ystride, NAN);
            for (int s = 0; s <= k; ++s)
            {
                const std::vector<float>& yin = (s & 1) ? y0 : y1;
                std::vector<float>& yout = (s & 1) ? y1 : y0;
                const uint32_t t1 = cnt[k - s];
                for (uint32_t tl = 0; tl < t1; ++tl)
                {
                    const uint32_t gr = glob(tl);
                    float sum = local_rhs && tl < local_rhs->size() ? (*local_rhs)[tl] : rhs[gr];
                    const uint32_t w = u32(o_deps, tl);
                    const uint32_t d[2] = {w & 0xFFFFu, w >> 16};
                    // the planned dependencies are the row's strict entries in column order
                    uint32_t e = rp[gr];
                    for (int q = 0; q < 2; ++q)
                    {
                        if (e < rp[gr + 1])
                        {
                            if (d[q] != kTileNoDep) CHECK(glob(d[q]) == ci[e], "%s: dependency column", name);
                            else CHECK(s == 0 || tl >= cnt[k - 1], "%s: missing dependency of a computed row", name);
                        }
                        else
                            CHECK(d[q] == kTileNoDep, "%s: extra dependency", name);
                        if (s > 0 && d[q] != kTileNoDep)
                        {
                            CHECK(d[q] < cnt[k - s + 1], "%s: reads a row the previous pass did not compute", name);
                            CHECK(d[q] < ystride, "%s: dependency outside the sweep buffer", name);
                            sum -= v[e] * yin[d[q]];
                        }
                        if (e < rp[gr + 1]) ++e;
                    }
                    yout[tl] = sum * dinv[gr];
                }
            }
            const std::vector<float>& yk = (k & 1) ? y1 : y0;
            for (uint32_t tl = 0; tl < check_rows; ++tl)
            {
                const uint32_t gr = glob(tl);
                CHECK(std::memcmp(&yk[tl], &want[gr], 4) == 0, "%s tile %u row %u (%s): %g vs %g", name, t, gr,
                      lower ? "lower" : "upper", yk[tl], want[gr]);
            }
            return std::vector<float>(yk.begin(), yk.begin() + check_rows);
        };
        // fused: the forward sweeps must give every row of the upper set, which
        // the backward sweeps then take from the CTA
        const std::vector<float> yloc = replay(true, D.n_el, D.lcnt, D.o_lhalo, D.o_ldeps, P.lrp, P.lci, lv, ld, r, yl,
                                               T.fused ? D.n_eu : D.n_own, nullptr);
        replay(false, D.n_eu, D.ucnt, D.o_uhalo, D.o_udeps, P.urp, P.uci, uv, ud, yl, yu, D.n_own,
               T.fused ? &yloc : nullptr);
        // SpMV over local columns against the CSR rows [lower | diag | upper]
        std::vector<double> pe(D.n_ae);
        for (uint32_t c = 0; c < D.n_ae; ++c) pe[c] = pg[c < D.n_own ? u32(D.o_owned, c) : u32(D.o_ahalo, c - D.n_own)];
        for (uint32_t q = 0; q < D.n_own; ++q)
        {
            const uint32_t gr = u32(D.o_owned, q);
            double sum = 0.0, want = 0.0;
            uint32_t e = u32(D.o_arp, q);
            const uint32_t e1 = u32(D.o_arp, q + 1);
            CHECK(e1 - e == (P.lrp[gr + 1] - P.lrp[gr]) + 1 + (P.urp[gr + 1] - P.urp[gr]), "%s: row length", name);
            std::vector<uint32_t> cols;
            for (uint32_t a = P.lrp[gr]; a < P.lrp[gr + 1]; ++a) cols.push_back(P.lci[a]);
            cols.push_back(gr);
            for (uint32_t a = P.urp[gr]; a < P.urp[gr + 1]; ++a) cols.push_back(P.uci[a]);
            for (size_t m = 0; m < cols.size() && e < e1; ++m, ++e)
            {
                const uint32_t c = u16(D.o_acol, e);
                CHECK(c < D.n_ae, "%s: local column outside the staged p", name);
                const double w = 1.0 + 0.25 * (double)(m + 1);
                sum += w * pe[c];
                want += w * pg[cols[m]];
            }
            CHECK(sum == want, "%s: SpMV row %u", name, gr);
        }
    }
    for (uint32_t i = 0; i < n; ++i) CHECK(seen[i] == 1, "%s: row %u owned %u times", name, i, seen[i]);
}

// the closed-form 5-point planner and builder against the breadth-first planner:
// the same descriptors and the same index blobs, byte for byte, for the fused
// layout (tried first) and the separate one
static void check_grid5(const char* name, uint32_t N, uint32_t M, int k, int sms)
{
    const Pattern P = five_point(N, M);
    for (int fused_first = 1; fused_first >= 0; --fused_first)
    {
        const TilePlan T = plan_tiles(P.n, P.lrp.data(), P.lci.data(), P.urp.data(), P.uci.data(), k, sms, 228352, 4,
                                      fused_first != 0);
        std::vector<TileGeom> geom;
        const TilePlan G = plan_tiles_grid5(P.n, N, k, sms, 228352, geom, fused_first != 0);
        std::printf("%-22s grid5 ok=%d fused=%d (BFS ok=%d fused=%d) tiles=%u Q=%u smem=%u\n", name, G.ok, G.fused, T.ok,
                    T.fused, G.ntiles, G.Q, G.smem);
        CHECK(is_grid5(P.n, P.lrp.data(), P.lci.data(), N, false), "%s: not recognised as a 5-point grid", name);
        CHECK(G.ok == T.ok, "%s: grid5 ok %d vs %d", name, G.ok, T.ok);
        if (!G.ok || !T.ok) continue;
        CHECK(G.fused == T.fused, "%s: fused %d vs %d", name, G.fused, T.fused);
        CHECK(G.ntiles == T.ntiles && G.smem == T.smem && G.work == T.work && G.Q == T.Q &&
                  G.ibytes == T.idx.size() && G.vbytes == T.vbytes,
              "%s: plan sizes differ", name);
        // the element-at-a-time builder (one device thread per element, then the
        // dependencies once the halos are in place), in reverse element order
        std::vector<uint8_t> blob(G.ibytes, 0);
        for (uint32_t t = 0; t < G.ntiles; ++t)
        {
            const TileDesc& D = G.desc[t];
            CHECK(std::memcmp(&D, &T.desc[t], sizeof(TileDesc)) == 0, "%s tile %u: descriptor differs", name, t);
            uint8_t* ib = blob.data() + D.ibase;
            const uint32_t ne = grid5_elements(D, geom[t], N, M, (uint32_t)k, G.fused);
            for (uint32_t e = ne; e-- > 0;)
                CHECK(grid5_build_elem(D, geom[t], N, M, (uint32_t)k, G.fused, e, ib),
                      "%s tile %u element %u: build failed", name, t, e);
            for (uint32_t r = D.n_el; r-- > 0;) grid5_build_dep(D, geom[t], N, M, (uint32_t)k, true, G.fused, r, ib);
            for (uint32_t r = D.n_eu; r-- > 0;) grid5_build_dep(D, geom[t], N, M, (uint32_t)k, false, G.fused, r, ib);
        }
        CHECK(blob == T.idx, "%s: index blobs differ", name);
    }
    // a pattern that is not a 5-point grid is not taken for one
    Pattern Q = P;
    if (Q.lci.size() > 2) std::swap(Q.lci[Q.lrp[N + 1]], Q.lci[Q.lrp[N + 1] + 1]);
    CHECK(!is_grid5(Q.n, Q.lrp.data(), Q.lci.data(), N, false), "%s: a perturbed pattern passed the check", name);
}

int main()
{
    check_grid5("grid5 512^2 k=6", 512, 512, 6, 148);
    check_grid5("grid5 512^2 k=8", 512, 512, 8, 148);
    check_grid5("grid5 600x200 k=6", 600, 200, 6, 148);
    check_grid5("grid5 100x3000 k=6", 100, 3000, 6, 148);
    check_grid5("grid5 64^2 k=3", 64, 64, 3, 148);
    check_grid5("grid5 37^2 k=16", 37, 37, 16, 148);
    check_grid5("grid5 512^2 132 SMs", 512, 512, 6, 132);
    check_plan("5-point 512^2, k=6", five_point(512), 6, 148, 228352, true);
    check_plan("5-point 512^2, k=8", five_point(512), 8, 148, 228352, true);
    check_plan("5-point 256^2, k=6", five_point(256), 6, 148, 228352, true);
    check_plan("5-point 64^2, k=3", five_point(64), 3, 148, 228352, true);
    check_plan("5-point 37^2, k=16", five_point(37), 16, 148, 228352, true);
    check_plan("5-point 512^2, 10 SMs", five_point(512), 6, 10, 228352, false);  // tiles too large
    check_plan("5-point 600x200, k=6", five_point(600, 200), 6, 148, 228352, true);
    check_plan("5-point 100x3000, k=6", five_point(100, 3000), 6, 148, 228352, true);
    check_plan("5-point 513x511, k=7", five_point(513, 511), 7, 148, 228352, true);
    check_plan("5-point 512^2, 132 SMs", five_point(512), 6, 132, 228352, true);
    // random offsets give L^T rows with more than two entries: not the kernel's pattern
    check_plan("banded 20000, B=40", banded(20000, 40, 3), 5, 148, 228352, false);
    std::printf(fails ? "FAILED (%d)\n" : "ALL PASSED\n", fails);
    return fails ? 1 : 0;
}
