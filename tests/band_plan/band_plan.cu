// Host checks of the planners: the band plan of a lower triangle's strict
// transpose made from the lower pattern (plan_band_transposed, trsv_band.cuh)
// equals plan_band on the transposed pattern, for grid stencils and random
// lower patterns; and the chunk plan (trsv_plan.hpp) is the same with one
// host thread and with sixteen.  Prints OK.
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "../../cpp-fem-solver_b200/csrc/trsv_band.cuh"
#include "../../cpp-fem-solver_b200/csrc/trsv_plan.hpp"

using namespace b2s;

static bool same(const BandPlan& a, const BandPlan& b)
{
    return a.T == b.T && a.B == b.B && a.W == b.W && a.Rmax == b.Rmax && a.smem == b.smem && a.ntiles == b.ntiles;
}

static int check(const char* name, uint32_t n, const std::vector<uint32_t>& rp, const std::vector<uint32_t>& ci)
{
    std::vector<uint32_t> trp, tci;
    strict_transpose(n, rp.data(), ci.data(), true, trp, tci);
    int bad = 0;
    for (int k : {1, 4, 8})
        for (uint32_t S : {1u, 8u})
        {
            const BandPlan a = plan_band_transposed(n, rp.data(), ci.data(), k, 148, S);
            const BandPlan b = plan_band(n, trp.data(), tci.data(), false, k, 148, S);
            if (!same(a, b))
            {
                std::printf("%s k=%d S=%u: T %u/%u B %u/%u W %u/%u ntiles %u/%u\n", name, k, S, a.T, b.T, a.B, b.B, a.W,
                            b.W, a.ntiles, b.ntiles);
                ++bad;
            }
        }
    return bad;
}

int main()
{
    int bad = 0;
    for (uint32_t N : {16u, 100u, 512u})  // 5-point lower (with diagonal), N x N
    {
        const uint32_t n = N * N;
        std::vector<uint32_t> rp{0}, ci;
        for (uint32_t i = 0; i < n; ++i)
        {
            if (i >= N) ci.push_back(i - N);
            if (i % N) ci.push_back(i - 1);
            ci.push_back(i);
            rp.push_back((uint32_t)ci.size());
        }
        bad += check("grid5", n, rp, ci);
    }
    std::mt19937 g(7);
    for (uint32_t n : {50u, 3000u, 20000u})  // random lower patterns of bandwidth <= 700
        for (int w : {1, 3, 6})
        {
            std::vector<uint32_t> rp{0}, ci;
            for (uint32_t i = 0; i < n; ++i)
            {
                std::vector<uint32_t> c{i};
                for (int t = 0; t < w && i > 0; ++t) c.push_back(i - 1 - g() % std::min<uint32_t>(i, 700));
                std::sort(c.begin(), c.end());
                c.erase(std::unique(c.begin(), c.end()), c.end());
                ci.insert(ci.end(), c.begin(), c.end());
                rp.push_back((uint32_t)ci.size());
            }
            bad += check("random", n, rp, ci);
        }
    // the chunk planner's output does not depend on its number of host threads
    for (uint32_t N : {24u, 64u})
    {
        const uint32_t n = N * N * N;
        std::vector<uint32_t> rp{0}, ci;
        for (uint32_t i = 0; i < n; ++i)
        {
            const uint32_t x = i % N, y = (i / N) % N, z = i / (N * N);
            if (z) ci.push_back(i - N * N);
            if (y) ci.push_back(i - N);
            if (x) ci.push_back(i - 1);
            ci.push_back(i);
            rp.push_back((uint32_t)ci.size());
        }
        for (int lower = 0; lower < 2; ++lower)
        {
            std::vector<uint32_t> trp, tci;
            const uint32_t* prp = rp.data();
            const uint32_t* pci = ci.data();
            if (!lower)
            {
                strict_transpose(n, rp.data(), ci.data(), true, trp, tci);
                prp = trp.data();
                pci = tci.data();
            }
            const ChunkPlan a = plan_chunks(n, prp, pci, lower, 1, 8, 8, 8, kChunkSmemBudget, 1, nullptr, 1);
            const ChunkPlan b = plan_chunks(n, prp, pci, lower, 1, 8, 8, 8, kChunkSmemBudget, 1, nullptr, 16);
            const bool eq = a.ok == b.ok && a.desc.size() == b.desc.size() &&
                            std::memcmp(a.desc.data(), b.desc.data(), a.desc.size() * sizeof(ChunkDesc)) == 0 &&
                            a.meta == b.meta && a.slot_row == b.slot_row && a.src == b.src &&
                            a.v64_units == b.v64_units && a.v32_units == b.v32_units &&
                            a.max_level_rows == b.max_level_rows;
            if (!eq)
            {
                std::printf("plan_chunks N=%u lower=%d: 1 and 16 workers differ\n", N, lower);
                ++bad;
            }
        }
    }
    std::printf(bad ? "FAIL\n" : "OK\n");
    return bad ? 1 : 0;
}
