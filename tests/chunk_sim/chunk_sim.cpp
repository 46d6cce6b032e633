// CPU model of the chunked triangular solves (scalar and block rows).
//
// Plans triangles with trsv_plan.hpp, packs the value blobs the way
// k_chunk_pack does, then replays the index arithmetic of k_trsv_chunk
// (bs = 1) or k_btrsv_chunk (bs > 1) chunk by chunk on a byte array the size
// of the CTA's shared memory, with every access checked against its segment.
// The result must equal a plain serial solve bit for bit.  Used by
// tests/test_chunk_plan.py (no GPU needed).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>

#include "../../cpp-fem-solver_b200/csrc/trsv_plan.hpp"

using namespace b2s;

#define CHECK(c)                                                                      \
    do                                                                                \
    {                                                                                 \
        if (!(c))                                                                     \
        {                                                                             \
            std::fprintf(stderr, "CHECK failed %s:%d: %s\n", __FILE__, __LINE__, #c); \
            std::exit(1);                                                             \
        }                                                                             \
    } while (0)

struct Tri
{
    uint32_t n;
    std::vector<uint32_t> rp, ci;
    std::vector<double> v, d;  // v: nnz * bs*bs, d: n * dv
};

// 2-D 5-point, 3-D 7-point or 3-D 27-point stencil pattern restricted to one triangle
static Tri stencil(uint32_t nx, uint32_t ny, uint32_t nz, bool lower, bool with_diag, bool box = false)
{
    Tri T;
    T.n = nx * ny * nz;
    T.rp.push_back(0);
    for (uint32_t k = 0; k < nz; ++k)
        for (uint32_t j = 0; j < ny; ++j)
            for (uint32_t i = 0; i < nx; ++i)
            {
                const uint32_t r = (k * ny + j) * nx + i;
                std::vector<uint32_t> cols;
                for (int dk = -1; dk <= 1; ++dk)
                    for (int dj = -1; dj <= 1; ++dj)
                        for (int di = -1; di <= 1; ++di)
                        {
                            const int nnzd = (di != 0) + (dj != 0) + (dk != 0);
                            if (!box && nnzd > 1) continue;
                            const int64_t ii = (int64_t)i + di, jj = (int64_t)j + dj, kk = (int64_t)k + dk;
                            if (ii < 0 || jj < 0 || kk < 0 || ii >= nx || jj >= ny || kk >= nz) continue;
                            cols.push_back((uint32_t)((kk * ny + jj) * nx + ii));
                        }
                std::sort(cols.begin(), cols.end());
                for (uint32_t c : cols)
                    if ((lower ? c < r : c > r) || (with_diag && c == r)) T.ci.push_back(c);
                T.rp.push_back((uint32_t)T.ci.size());
            }
    return T;
}

// random triangle: row i depends on up to `maxdep` earlier (or later) rows, some far away
static Tri random_tri(uint32_t n, bool lower, uint32_t maxdep, uint32_t seed)
{
    std::mt19937 g(seed);
    Tri T;
    T.n = n;
    T.rp.push_back(0);
    for (uint32_t r = 0; r < n; ++r)
    {
        std::vector<uint32_t> cols;
        const uint32_t avail = lower ? r : n - 1 - r;
        const uint32_t k = avail ? g() % (std::min(avail, maxdep) + 1) : 0;
        for (uint32_t q = 0; q < k; ++q)
        {
            const uint32_t span = (g() % 4 == 0) ? avail : std::min<uint32_t>(avail, 40);
            const uint32_t off = 1 + g() % span;
            cols.push_back(lower ? r - off : r + off);
        }
        cols.push_back(r);
        std::sort(cols.begin(), cols.end());
        cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
        for (uint32_t c : cols) T.ci.push_back(c);
        T.rp.push_back((uint32_t)T.ci.size());
    }
    return T;
}

static void fill_values(Tri& T, uint32_t bs, uint32_t dv, uint32_t seed)
{
    std::mt19937_64 g(seed);
    std::uniform_real_distribution<double> u(-0.3, 0.3), w(1.0, 2.0), o(-0.2, 0.2);
    const uint32_t bv = bs * bs;
    T.v.resize(T.ci.size() * bv);
    for (double& x : T.v) x = u(g) / bs;
    T.d.resize((size_t)T.n * dv);
    for (uint32_t i = 0; i < T.n; ++i)
        for (uint32_t q = 0; q < dv; ++q)
            T.d[(size_t)i * dv + q] = dv == 1 ? w(g) : (q / bs == q % bs ? 1.0 : o(g));
}

// serial solve in the kernels' arithmetic
template <int BS, typename VT, typename XT, typename RT>
static std::vector<XT> serial_solve(const Tri& T, bool lower, uint32_t dv, const std::vector<RT>& b)
{
    constexpr int BV = BS * BS;
    std::vector<XT> x((size_t)T.n * BS);
    for (uint32_t q = 0; q < T.n; ++q)
    {
        const uint32_t i = lower ? q : T.n - 1 - q;
        XT t[BS];
        for (int c = 0; c < BS; ++c) t[c] = (XT)b[(size_t)i * BS + c];
        for (uint32_t p = T.rp[i]; p < T.rp[i + 1]; ++p)
        {
            const uint32_t j = T.ci[p];
            if (!(lower ? j < i : j > i)) continue;
            if (BS == 1)
                t[0] -= (XT)(VT)T.v[p] * x[j];
            else
                for (int r = 0; r < BS; ++r)
                {
                    XT s = 0;
                    for (int c = 0; c < BS; ++c) s += (XT)(VT)T.v[(size_t)p * BV + r * BS + c] * x[(size_t)j * BS + c];
                    t[r] -= s;
                }
        }
        if (dv == 0)
            for (int c = 0; c < BS; ++c) x[(size_t)i * BS + c] = t[c];
        else if (BS == 1)
            x[i] = t[0] / (XT)(VT)T.d[i];
        else
            for (int r = 0; r < BS; ++r)
            {
                XT s = 0;
                for (int c = 0; c < BS; ++c) s += (XT)(VT)T.d[(size_t)i * BV + r * BS + c] * t[c];
                x[(size_t)i * BS + r] = s;
            }
    }
    return x;
}

// a byte array with per-segment bounds checks
struct Smem
{
    std::vector<uint8_t> b;
    template <typename T>
    T& at(uint32_t seg, uint32_t seg_end, uint32_t idx)
    {
        const uint64_t off = (uint64_t)seg + (uint64_t)idx * sizeof(T);
        CHECK(off + sizeof(T) <= seg_end);
        CHECK(seg_end <= b.size());
        return *reinterpret_cast<T*>(b.data() + off);
    }
};

static uint16_t rd16(const std::vector<uint8_t>& m, uint64_t off)
{
    CHECK(off + 2 <= m.size());
    uint16_t v;
    std::memcpy(&v, m.data() + off, 2);
    return v;
}

template <int BS, typename VT, typename XT, typename RT>
static void run_case(const char* name, Tri T, bool lower, uint32_t dv, uint32_t budget, uint32_t seed, bool verbose)
{
    constexpr uint32_t VS = sizeof(VT), XS = sizeof(XT), RS = sizeof(RT), BV = BS * BS;
    fill_values(T, BS, dv, seed);
    std::vector<RT> b((size_t)T.n * BS);
    std::mt19937_64 g(seed ^ 0x9e37u);
    std::uniform_real_distribution<double> u(-1, 1);
    for (RT& x : b) x = (RT)u(g);
    const std::vector<XT> ref = serial_solve<BS, VT, XT, RT>(T, lower, dv, b);

    // the library plans with (vs, vs, 8); a launch may use a narrower rhs
    const ChunkPlan P = plan_chunks(T.n, T.rp.data(), T.ci.data(), lower, dv, VS, XS, 8, budget, BS);
    if (!P.ok && budget < kChunkSmemBudget) return;  // a block row alone exceeds a toy budget
    CHECK(P.ok);
    CHECK(P.meta.size() % 16 == 0);
    {
        // every row is in exactly one chunk; chunks are contiguous, in processing order
        uint32_t next = lower ? 0 : T.n;
        for (const ChunkDesc& D : P.desc)
        {
            CHECK(D.nr >= 1 && D.nr <= kChunkMaxRows);
            CHECK(D.nd <= kChunkMaxDeps && D.ns <= kChunkMaxSlots);
            if (lower)
            {
                CHECK(D.lo == next);
                next = D.lo + D.nr;
            }
            else
            {
                CHECK(D.lo + D.nr == next);
                next = D.lo;
            }
        }
        CHECK(next == (lower ? T.n : 0u));
    }
    // pack the value blob as k_chunk_pack does
    std::vector<uint8_t> vals(std::max<uint64_t>(VS == 8 ? P.v64_units : P.v32_units, 1) * 16, 0xCD);
    for (const ChunkDesc& D : P.desc)
    {
        const SmemLayout L = smem_layout(D.nr, D.nd, D.nl, D.ns, VS, VS, VS, BS, dv);
        const uint64_t base = (uint64_t)(VS == 8 ? D.v64 : D.v32) * 16;
        CHECK(base + L.vals <= vals.size());
        const uint32_t nv = (L.sd - L.sv) / VS;
        for (uint32_t e = 0; e < nv; ++e)
        {
            VT val = 0;
            if (e < D.nd * BV)
            {
                CHECK(D.dep + e / BV < P.src.size());
                const uint32_t p = P.src[D.dep + e / BV];
                CHECK((size_t)p * BV + e % BV < T.v.size());
                val = (VT)T.v[(size_t)p * BV + e % BV];
            }
            std::memcpy(vals.data() + base + L.sv + (uint64_t)VS * e, &val, VS);
        }
        if (dv)
        {
            const uint32_t nd = (L.vals - L.sd) / VS;
            for (uint32_t e = 0; e < nd; ++e)
            {
                VT val = 0;
                const uint32_t t = e / dv;
                if (t < D.nr)
                {
                    const uint32_t k = rd16(P.meta, (uint64_t)D.meta * 16 + L.m.rec + 8ull * t) & 0x7fffu;
                    CHECK(k < D.nr);
                    val = (VT)T.d[(size_t)(D.lo + k) * dv + e % dv];
                }
                std::memcpy(vals.data() + base + L.sd + (uint64_t)VS * e, &val, VS);
            }
        }
    }
    // replay the kernel
    std::vector<XT> xglob((size_t)T.n * BS, (XT)std::nan(""));
    std::vector<uint8_t> done(T.n, 0), published(T.n, 0);
    uint32_t max_rows = 0, max_levels = 0, max_slots = 0, smem_max = 0;
    for (const ChunkDesc& D : P.desc)
    {
        const SmemLayout L = smem_layout(D.nr, D.nd, D.nl, D.ns, VS, XS, RS, BS, dv);
        CHECK(L.total <= kChunkSmemLimit);
        CHECK(L.total <= budget || D.nr == 1);
        max_rows = std::max(max_rows, D.nr);
        max_levels = std::max(max_levels, D.nl);
        max_slots = std::max(max_slots, D.ns);
        smem_max = std::max(smem_max, L.total);
        Smem S;
        S.b.assign(L.total, 0xAB);
        // 1. stage
        const uint64_t vbase = (uint64_t)(VS == 8 ? D.v64 : D.v32) * 16;
        CHECK(vbase + L.vals <= vals.size());
        std::memcpy(S.b.data() + L.sv, vals.data() + vbase, L.vals);
        CHECK((uint64_t)D.meta * 16 + L.m.bytes <= P.meta.size());
        std::memcpy(S.b.data() + L.meta, P.meta.data() + (uint64_t)D.meta * 16, L.m.bytes);
        for (uint32_t k = 0; k < D.nr * BS; ++k) S.at<RT>(L.sr, L.xv, k) = b[(size_t)D.lo * BS + k];
        for (uint32_t s = 0; s < D.ns; ++s) S.at<uint32_t>(L.xr, L.total, s) = 0;
        // 2a. producer (all slots up front: their rows belong to earlier chunks)
        for (uint32_t s = 0; s < D.ns; ++s)
        {
            CHECK(D.slot + s < P.slot_row.size());
            const uint32_t j = P.slot_row[D.slot + s];
            CHECK(j < T.n && done[j] && published[j]);
            CHECK(j < D.lo || j >= D.lo + D.nr);
            for (int c = 0; c < (int)BS; ++c) S.at<XT>(L.xv, L.xr, s * BS + c) = xglob[(size_t)j * BS + c];
            S.at<uint32_t>(L.xr, L.total, s) = 1;
        }
        // 2b. compute
        const uint32_t mslc = L.meta + L.m.slc, mrec = L.meta + L.m.rec, mslv = L.meta + L.m.slv,
                       mend = L.meta + L.m.bytes;
        std::vector<int32_t> lvl_of_pos(D.nr, -1);
        CHECK(S.at<uint16_t>(mslv, mend, 0) == 0);
        CHECK(S.at<uint16_t>(mslv, mend, D.nl) == D.nr);
        for (uint32_t l = 0; l < D.nl; ++l)
        {
            const uint32_t t0 = S.at<uint16_t>(mslv, mend, l), t1 = S.at<uint16_t>(mslv, mend, l + 1);
            CHECK(t0 < t1 && t1 <= D.nr);
            for (uint32_t t = t0; t < t1; ++t)
            {
                const uint32_t pr = S.at<uint16_t>(mrec, mslv, 4 * t), k = pr & 0x7fffu;
                const uint32_t e0 = S.at<uint16_t>(mrec, mslv, 4 * t + 1), e1 = S.at<uint16_t>(mrec, mslv, 4 * t + 2);
                // the record's slot mask names exactly the row's slot entries (of the first 16)
                uint32_t want_mask = 0;
                for (uint32_t e = e0; e < e1 && e - e0 < 16; ++e)
                    if (S.at<uint16_t>(mslc, mrec, e) & 0x8000u) want_mask |= 1u << (e - e0);
                CHECK(S.at<uint16_t>(mrec, mslv, 4 * t + 3) == want_mask);
                CHECK(k < D.nr);
                // one lane per component (a single lane for scalar rows)
                XT tr[BS];
                for (uint32_t r = 0; r < BS; ++r)
                {
                    tr[r] = (XT)S.at<RT>(L.sr, L.xv, k * BS + r);
                    CHECK(e0 <= e1 && e1 <= D.nd);
                    for (uint32_t e = e0; e < e1; ++e)
                    {
                        const uint32_t m = S.at<uint16_t>(mslc, mrec, e);
                        uint32_t seg, seg_end, base;
                        if (m & 0x8000u)
                        {
                            const uint32_t s = m & 0x7fffu;
                            CHECK(s < D.ns);
                            CHECK(S.at<uint32_t>(L.xr, L.total, s) == 1u);
                            seg = L.xv, seg_end = L.xr, base = s * BS;
                        }
                        else
                        {
                            CHECK(m < D.nr);
                            CHECK(lvl_of_pos[m] >= 0 && (uint32_t)lvl_of_pos[m] < l);
                            seg = L.sx, seg_end = L.sr, base = m * BS;
                        }
                        if (BS == 1)
                            tr[r] -= (XT)S.at<VT>(L.sv, L.sd, e) * S.at<XT>(seg, seg_end, base);
                        else
                        {
                            XT acc = 0;
                            for (uint32_t c = 0; c < BS; ++c)
                                acc += (XT)S.at<VT>(L.sv, L.sd, e * BV + r * BS + c) * S.at<XT>(seg, seg_end, base + c);
                            tr[r] -= acc;
                        }
                    }
                }
                XT xo[BS];
                for (uint32_t r = 0; r < BS; ++r)
                {
                    if (dv == 0)
                        xo[r] = tr[r];
                    else if (BS == 1)
                        xo[r] = tr[r] / (XT)S.at<VT>(L.sd, L.vals, t);
                    else
                    {
                        XT acc = 0;
                        for (uint32_t c = 0; c < BS; ++c) acc += (XT)S.at<VT>(L.sd, L.vals, t * BV + r * BS + c) * tr[c];
                        xo[r] = acc;
                    }
                }
                for (uint32_t r = 0; r < BS; ++r) S.at<XT>(L.sx, L.sr, t * BS + r) = xo[r];
                lvl_of_pos[t] = (int32_t)l;
                const uint32_t row = D.lo + k;
                CHECK(!done[row]);
                for (uint32_t r = 0; r < BS; ++r) xglob[(size_t)row * BS + r] = xo[r];
                done[row] = 1;
                if (pr & 0x8000u) published[row] = 1;
            }
        }
        for (uint32_t t = 0; t < D.nr; ++t) CHECK(lvl_of_pos[t] >= 0);
    }
    for (size_t q = 0; q < xglob.size(); ++q)
    {
        CHECK(done[q / BS]);
        if (std::memcmp(&xglob[q], &ref[q], sizeof(XT)) != 0)
        {
            std::fprintf(stderr, "%s: entry %zu differs: %.17g vs %.17g\n", name, q, (double)xglob[q], (double)ref[q]);
            std::exit(1);
        }
    }
    if (verbose)
        std::printf("%-40s n=%-8u chunks=%-5zu max_rows=%-6u max_levels=%-6u max_slots=%-6u level_rows=%-5u "
                    "smem=%u\n",
                    name, T.n, P.desc.size(), max_rows, max_levels, max_slots, P.max_level_rows, smem_max);
}

// FP64 solve; FP32 forward solve (FP64 rhs); FP32 backward solve (FP32 rhs)
#define RUN3(BS, name, ...)                                                      \
    do                                                                           \
    {                                                                            \
        run_case<BS, double, double, double>(name " [f64]", __VA_ARGS__);        \
        run_case<BS, float, float, double>(name " [f32, f64 rhs]", __VA_ARGS__); \
        run_case<BS, float, float, float>(name " [f32]", __VA_ARGS__);           \
    } while (0)

int main(int argc, char** argv)
{
    const bool big = argc > 1 && std::string(argv[1]) == "big";
    const uint32_t budgets[] = {1024, 4096, 32768, kChunkSmemBudget};
    for (uint32_t bud : budgets)
    {
        // scalar rows: dv 1 = divide by the diagonal, 0 = unit triangle
        RUN3(1, "2d lower+diag", stencil(64, 64, 1, true, true), true, 1, bud, 1, false);
        RUN3(1, "2d upper strict", stencil(64, 64, 1, false, false), false, 1, bud, 2, false);
        RUN3(1, "2d lower unit", stencil(64, 64, 1, true, false), true, 0, bud, 3, false);
        RUN3(1, "3d lower unit", stencil(16, 16, 16, true, false), true, 0, bud, 4, false);
        RUN3(1, "3d upper", stencil(16, 16, 16, false, true), false, 1, bud, 5, false);
        RUN3(1, "random lower", random_tri(5000, true, 12, 6), true, 1, bud, 6, false);
        RUN3(1, "random upper unit", random_tri(5000, false, 12, 7), false, 0, bud, 7, false);
        // block rows: unit lower, upper times the inverse diagonal block
        RUN3(3, "box27 lower bs3", stencil(12, 12, 12, true, false, true), true, 0, bud, 15, false);
        RUN3(3, "box27 upper bs3", stencil(12, 12, 12, false, true, true), false, 9, bud, 16, false);
        RUN3(2, "random lower bs2", random_tri(3000, true, 10, 17), true, 0, bud, 17, false);
        RUN3(4, "random upper bs4", random_tri(3000, false, 10, 18), false, 16, bud, 18, false);
    }
    RUN3(1, "single row", stencil(1, 1, 1, true, true), true, 1, kChunkSmemBudget, 8, false);
    RUN3(1, "dense-ish lower", random_tri(600, true, 200, 9), true, 1, 4096, 9, false);
    RUN3(1, "512^2 lower (C5 IC0 L)", stencil(512, 512, 1, true, true), true, 1, kChunkSmemBudget, 10, true);
    RUN3(1, "512^2 upper (C5 IC0 L^T)", stencil(512, 512, 1, false, false), false, 1, kChunkSmemBudget, 11, true);
    if (big)
    {
        RUN3(1, "128^3 lower unit (C2 ILU L)", stencil(128, 128, 128, true, false), true, 0, kChunkSmemBudget, 12,
             true);
        RUN3(1, "128^3 upper (C2 ILU U)", stencil(128, 128, 128, false, true), false, 1, kChunkSmemBudget, 13, true);
        RUN3(1, "96^3 lower unit (C3 ILU L)", stencil(96, 96, 96, true, false), true, 0, kChunkSmemBudget, 14, true);
        RUN3(3, "65^3 box27 lower bs3 (C4 BILU L)", stencil(65, 65, 65, true, false, true), true, 0,
             kChunkSmemBudget, 19, true);
        RUN3(3, "65^3 box27 upper bs3 (C4 BILU U)", stencil(65, 65, 65, false, true, true), false, 9,
             kChunkSmemBudget, 20, true);
    }
    std::printf("OK\n");
    return 0;
}
