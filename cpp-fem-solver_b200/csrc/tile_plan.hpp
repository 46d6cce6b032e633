// Host planning of the tiled persistent PCG kernel (pcg_tile.cuh).
//
// The rows are cut into one tile per CTA.  A tile owns its rows and keeps,
// for the k Jacobi sweeps of each triangle, the rows its owned rows depend
// on within k steps (its halo): the extended set E of a triangle is found by
// a breadth-first walk over the triangle's strict entries, layer d holding
// the rows first reached after d steps.  Rows are numbered locally: owned
// rows first (ascending), then layer 1, 2, ..., k (each ascending).  Sweep s
// computes the rows of layers 0..k-s -- a prefix of the local order -- so
// every value it reads is the previous sweep's exact value, and the owned
// rows after sweep k equal the global sweep definition bit for bit.
//
// For the SpMV a tile also keeps the columns its owned rows reach (owned
// first, then the others ascending); A's rows are taken from the triangle's
// pattern as [strict lower entries, diagonal, strict upper entries], which is
// A's own pattern when A is structurally symmetric -- the device packing
// checks every column against A and the plan is dropped otherwise.
//
// Tiles: when the triangle's bandwidth B suggests a grid (row i at
// x = i mod B, y = i div B, as natural-order 2-D stencils are), the tiles
// are blocks of that grid, which keeps the halo to a ring of width k around
// the block instead of k B rows; among the block shapes that give at most one
// tile per SM, the one with the smallest estimated extended set is kept
// (one block column is the strip layout of the banded kernel).
//
// Each tile has two blobs with the same segment layout in shared memory:
// the index blob (filled here: global rows, local dependencies, A's local
// columns) and the value blob (filled on the device after factorisation:
// A's values, the triangles' strict entries and reciprocals).
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "trsv_plan.hpp"

namespace b2s {

constexpr int kTileMaxSweeps = 16;
constexpr uint32_t kTileThreads = 768;
constexpr uint32_t kTileMaxQ = 4;  // extended rows per thread
constexpr uint32_t kTileNoDep = 0xFFFFu;
constexpr int kTileMaxTiles = 160;  // the kernel's all-reduce: 5 tiles per lane of one warp

struct TileDesc
{
    uint32_t n_own, n_el, n_eu, n_ae, nnz;
    uint32_t vbytes, ibytes;  // value / index blob bytes (multiples of 16)
    uint32_t pad;
    uint64_t vbase, ibase;    // byte offsets of the tile's blobs
    // value blob: A's values (f64), strict entries (2 x f32 per row), reciprocals (f32)
    uint32_t o_aval, o_lvals, o_uvals, o_ldinv, o_udinv;
    // index blob: owned rows, halos (global rows), dependencies (2 x u16 per row), A's offsets and columns
    uint32_t o_owned, o_lhalo, o_ldeps, o_uhalo, o_udeps, o_ahalo, o_arp, o_acol;
    uint16_t lcnt[kTileMaxSweeps + 1];  // rows of layers 0..d of the lower triangle's set
    uint16_t ucnt[kTileMaxSweeps + 1];
};

struct TilePlan
{
    bool ok = false;
    uint32_t n = 0, ntiles = 0, k = 0, Q = 0;
    uint32_t tiles_x = 0, tiles_y = 0, B = 0;
    uint32_t max_ext = 0, max_own = 0, max_ae = 0;
    uint64_t vbytes = 0, ibytes = 0;
    uint32_t smem = 0;  // dynamic shared memory per CTA: the largest blob pair + work buffers
    uint32_t work = 0;  // offset of the work buffers (bytes)
    std::vector<TileDesc> desc;
    std::vector<uint8_t> idx;  // all index blobs
};

inline uint32_t tile_align16(uint64_t b) { return (uint32_t)((b + 15u) & ~15ull); }

// The strict lower entries (j < i) of a column-sorted CSR pattern.
inline void strict_lower(uint32_t n, const uint32_t* rp, const uint32_t* ci, std::vector<uint32_t>& lrp,
                         std::vector<uint32_t>& lci)
{
    lrp.assign((size_t)n + 1, 0);
    lci.clear();
    lci.reserve(rp[n]);
    for (uint32_t i = 0; i < n; ++i)
    {
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
            if (ci[p] < i) lci.push_back(ci[p]);
        lrp[i + 1] = (uint32_t)lci.size();
    }
}

// work buffers after the blobs: two FP32 sweep vectors, or the staged FP64 p
inline uint32_t tile_work_bytes(uint32_t max_ext, uint32_t max_ae)
{
    return std::max<uint32_t>(2 * tile_align16(4ull * max_ext), tile_align16(8ull * max_ae));
}

struct TileBuild
{
    std::vector<uint32_t> own, el, eu, ae;  // global rows in local order
    std::vector<uint32_t> ldeps, udeps;     // packed 2 x u16 per extended row
    std::vector<uint16_t> lcnt, ucnt;
    std::vector<uint32_t> arp;              // owned rows' entry offsets
    std::vector<uint16_t> acol;             // local columns
};

// Breadth-first extended set of one triangle (layer 0 = own); false when a
// row has more than two strict entries or the set outgrows a CTA.  mark /
// local are per-worker scratch arrays of n entries; stamp is unique per set.
inline bool tile_extend(const std::vector<uint32_t>& own, const uint32_t* rp, const uint32_t* ci, int k, uint32_t stamp,
                        std::vector<uint32_t>& mark, std::vector<uint32_t>& local, std::vector<uint32_t>& ext,
                        std::vector<uint32_t>& deps, std::vector<uint16_t>& cnt)
{
    ext = own;
    for (uint32_t t = 0; t < (uint32_t)own.size(); ++t)
    {
        mark[own[t]] = stamp;
        local[own[t]] = t;
    }
    cnt.assign((size_t)k + 1, 0);
    cnt[0] = (uint16_t)own.size();
    size_t f0 = 0, f1 = own.size();
    std::vector<uint32_t> next;
    for (int d = 1; d <= k; ++d)
    {
        next.clear();
        for (size_t q = f0; q < f1; ++q)
        {
            const uint32_t i = ext[q];
            for (uint32_t e = rp[i]; e < rp[i + 1]; ++e)
            {
                const uint32_t j = ci[e];
                if (mark[j] != stamp)
                {
                    mark[j] = stamp;
                    next.push_back(j);
                }
            }
        }
        std::sort(next.begin(), next.end());
        f0 = ext.size();
        for (uint32_t j : next)
        {
            local[j] = (uint32_t)ext.size();
            ext.push_back(j);
        }
        f1 = ext.size();
        if (ext.size() > (size_t)kTileThreads * kTileMaxQ || ext.size() >= kTileNoDep) return false;
        cnt[d] = (uint16_t)ext.size();
    }
    deps.assign(ext.size(), 0xFFFFFFFFu);
    for (size_t t = 0; t < ext.size(); ++t)
    {
        const uint32_t i = ext[t];
        if (rp[i + 1] - rp[i] > 2) return false;
        uint32_t w = 0xFFFFFFFFu;
        for (uint32_t e = rp[i], s = 0; e < rp[i + 1]; ++e, ++s)
        {
            const uint32_t j = ci[e];
            // outside the set: only layer-k rows reach it, and they are computed at sweep 0 alone
            const uint32_t l = mark[j] == stamp ? local[j] : kTileNoDep;
            w = s == 0 ? ((w & 0xFFFF0000u) | l) : ((w & 0x0000FFFFu) | (l << 16));
        }
        deps[t] = w;
    }
    return true;
}

// The plan.  n rows; the lower triangle's strict entries (lo_rp/lo_ci,
// column order) and the upper's (up_rp/up_ci), at most two per row; k
// sweeps; sm_count CTAs at most; smem_limit bytes of dynamic shared memory
// per CTA; workers host threads.
inline TilePlan plan_tiles_shape(uint32_t n, const uint32_t* lo_rp, const uint32_t* lo_ci, const uint32_t* up_rp,
                                 const uint32_t* up_ci, int k, uint64_t B, uint64_t bx, uint64_t by,
                                 uint32_t smem_limit, unsigned workers);

inline TilePlan plan_tiles(uint32_t n, const uint32_t* lo_rp, const uint32_t* lo_ci, const uint32_t* up_rp,
                           const uint32_t* up_ci, int k, int sm_count, uint32_t smem_limit, unsigned workers)
{
    TilePlan P;
    P.n = n;
    P.k = (uint32_t)k;
    if (!n || k < 1 || k > kTileMaxSweeps || sm_count < 1 || n > 0x7FFFFFFFu) return P;
    sm_count = std::min(sm_count, kTileMaxTiles);
    uint64_t B = 1;
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t e = lo_rp[i]; e < lo_rp[i + 1]; ++e) B = std::max<uint64_t>(B, i - lo_ci[e]);
    if (B > n) B = n;
    const uint64_t ny = (n + B - 1) / B;
    uint64_t best = ~0ull, bx = 1, by = 1;
    for (uint64_t tx = 1; tx <= std::min<uint64_t>(B, (uint64_t)sm_count); ++tx)
    {
        const uint64_t ty = std::min<uint64_t>((uint64_t)sm_count / tx, ny);
        if (!ty) continue;
        const uint64_t w = (B + tx - 1) / tx, h = (ny + ty - 1) / ty;
        const uint64_t est = tx == 1 ? w * h + (uint64_t)k * B : (w + (uint64_t)k) * (h + (uint64_t)k);
        if (est < best)
        {
            best = est;
            bx = tx;
            by = ty;
        }
    }
    P = plan_tiles_shape(n, lo_rp, lo_ci, up_rp, up_ci, k, B, bx, by, smem_limit, workers);
    if (!P.ok && bx != 1)  // the blocks' halos outgrew a CTA (dependencies that cross block columns): strips
    {
        const uint64_t B1 = std::max<uint64_t>(1, (n + (uint64_t)sm_count - 1) / (uint64_t)sm_count);
        P = plan_tiles_shape(n, lo_rp, lo_ci, up_rp, up_ci, k, B1, 1, (n + B1 - 1) / B1, smem_limit, workers);
    }
    return P;
}

// One tile shape: blocks of w = ceil(B / bx) grid columns by h = ceil(ny / by)
// grid rows, row i at (i mod B, i div B).
inline TilePlan plan_tiles_shape(uint32_t n, const uint32_t* lo_rp, const uint32_t* lo_ci, const uint32_t* up_rp,
                                 const uint32_t* up_ci, int k, uint64_t B, uint64_t bx, uint64_t by,
                                 uint32_t smem_limit, unsigned workers)
{
    TilePlan P;
    P.n = n;
    P.k = (uint32_t)k;
    const uint64_t ny = (n + B - 1) / B;
    const uint64_t w = (B + bx - 1) / bx, h = (ny + by - 1) / by;
    const uint32_t tiles_x = (uint32_t)((B + w - 1) / w), tiles_y = (uint32_t)((ny + h - 1) / h);
    const uint32_t ntiles = tiles_x * tiles_y;
    std::vector<TileBuild> tb(ntiles);
    for (uint32_t i = 0; i < n; ++i)
        tb[(uint32_t)(((i / B) / h) * tiles_x + (i % B) / w)].own.push_back(i);
    for (const TileBuild& T : tb)
        if (T.own.empty() || T.own.size() > (size_t)kTileThreads * kTileMaxQ) return P;
    const unsigned nw = std::max(1u, std::min(workers, ntiles));
    std::vector<std::vector<uint32_t>> mark(nw), local(nw);
    std::vector<char> good(ntiles, 0);
    plan_parallel(ntiles, nw, [&](uint32_t t, unsigned wk) {
        std::vector<uint32_t>& mk = mark[wk];
        std::vector<uint32_t>& lc = local[wk];
        if (mk.empty())
        {
            mk.assign(n, 0xFFFFFFFFu);
            lc.assign(n, 0);
        }
        TileBuild& T = tb[t];
        if (!tile_extend(T.own, lo_rp, lo_ci, k, 3 * t, mk, lc, T.el, T.ldeps, T.lcnt)) return;
        if (!tile_extend(T.own, up_rp, up_ci, k, 3 * t + 1, mk, lc, T.eu, T.udeps, T.ucnt)) return;
        // the SpMV's columns: owned rows' [lower strict, diagonal, upper strict]
        const uint32_t stamp = 3 * t + 2;
        T.ae = T.own;
        for (uint32_t q = 0; q < (uint32_t)T.own.size(); ++q)
        {
            mk[T.own[q]] = stamp;
            lc[T.own[q]] = q;
        }
        std::vector<uint32_t> extra;
        auto visit = [&](uint32_t j) {
            if (mk[j] != stamp)
            {
                mk[j] = stamp;
                extra.push_back(j);
            }
        };
        for (uint32_t i : T.own)
        {
            for (uint32_t e = lo_rp[i]; e < lo_rp[i + 1]; ++e) visit(lo_ci[e]);
            for (uint32_t e = up_rp[i]; e < up_rp[i + 1]; ++e) visit(up_ci[e]);
        }
        std::sort(extra.begin(), extra.end());
        for (uint32_t j : extra)
        {
            lc[j] = (uint32_t)T.ae.size();
            T.ae.push_back(j);
        }
        if (T.ae.size() >= kTileNoDep) return;
        T.arp.assign(T.own.size() + 1, 0);
        for (uint32_t q = 0; q < (uint32_t)T.own.size(); ++q)
        {
            const uint32_t i = T.own[q];
            for (uint32_t e = lo_rp[i]; e < lo_rp[i + 1]; ++e) T.acol.push_back((uint16_t)lc[lo_ci[e]]);
            T.acol.push_back((uint16_t)q);
            for (uint32_t e = up_rp[i]; e < up_rp[i + 1]; ++e) T.acol.push_back((uint16_t)lc[up_ci[e]]);
            T.arp[q + 1] = (uint32_t)T.acol.size();
        }
        good[t] = 1;
    });
    for (char g : good)
        if (!g) return P;
    // blob layout
    P.desc.resize(ntiles);
    uint64_t vbase = 0, ibase = 0;
    uint32_t max_pair = 0;
    for (uint32_t t = 0; t < ntiles; ++t)
    {
        const TileBuild& T = tb[t];
        TileDesc& D = P.desc[t];
        std::memset(&D, 0, sizeof(D));
        D.n_own = (uint32_t)T.own.size();
        D.n_el = (uint32_t)T.el.size();
        D.n_eu = (uint32_t)T.eu.size();
        D.n_ae = (uint32_t)T.ae.size();
        D.nnz = (uint32_t)T.acol.size();
        uint32_t o = 0;
        auto seg = [&o](uint64_t bytes) {
            const uint32_t at = o;
            o += tile_align16(bytes);
            return at;
        };
        D.o_aval = seg(8ull * D.nnz);
        D.o_lvals = seg(8ull * D.n_el);
        D.o_uvals = seg(8ull * D.n_eu);
        D.o_ldinv = seg(4ull * D.n_el);
        D.o_udinv = seg(4ull * D.n_eu);
        D.vbytes = o;
        o = 0;
        D.o_owned = seg(4ull * D.n_own);
        D.o_lhalo = seg(4ull * (D.n_el - D.n_own));
        D.o_ldeps = seg(4ull * D.n_el);
        D.o_uhalo = seg(4ull * (D.n_eu - D.n_own));
        D.o_udeps = seg(4ull * D.n_eu);
        D.o_ahalo = seg(4ull * (D.n_ae - D.n_own));
        D.o_arp = seg(4ull * (D.n_own + 1));
        D.o_acol = seg(2ull * D.nnz);
        D.ibytes = o;
        D.vbase = vbase;
        D.ibase = ibase;
        vbase += D.vbytes;
        ibase += D.ibytes;
        for (int d = 0; d <= k; ++d)
        {
            D.lcnt[d] = T.lcnt[d];
            D.ucnt[d] = T.ucnt[d];
        }
        max_pair = std::max(max_pair, D.vbytes + D.ibytes);
        P.max_ext = std::max(P.max_ext, std::max(D.n_el, D.n_eu));
        P.max_own = std::max(P.max_own, D.n_own);
        P.max_ae = std::max(P.max_ae, D.n_ae);
    }
    // the work buffers sit after the largest blob pair, the same offset in every CTA
    P.work = max_pair;
    P.smem = max_pair + tile_work_bytes(P.max_ext, P.max_ae);
    P.Q = (P.max_ext + kTileThreads - 1) / kTileThreads;
    if (P.smem > smem_limit || P.Q > kTileMaxQ) return P;
    P.idx.assign(ibase, 0);
    plan_parallel(ntiles, nw, [&](uint32_t t, unsigned) {
        const TileBuild& T = tb[t];
        const TileDesc& D = P.desc[t];
        uint8_t* b = P.idx.data() + D.ibase;
        auto put = [&](uint32_t off, const void* src, size_t bytes) {
            if (bytes) std::memcpy(b + off, src, bytes);
        };
        put(D.o_owned, T.own.data(), 4 * T.own.size());
        put(D.o_lhalo, T.el.data() + D.n_own, 4 * (size_t)(D.n_el - D.n_own));
        put(D.o_ldeps, T.ldeps.data(), 4 * T.ldeps.size());
        put(D.o_uhalo, T.eu.data() + D.n_own, 4 * (size_t)(D.n_eu - D.n_own));
        put(D.o_udeps, T.udeps.data(), 4 * T.udeps.size());
        put(D.o_ahalo, T.ae.data() + D.n_own, 4 * (size_t)(D.n_ae - D.n_own));
        put(D.o_arp, T.arp.data(), 4 * T.arp.size());
        put(D.o_acol, T.acol.data(), 2 * T.acol.size());
    });
    P.ntiles = ntiles;
    P.tiles_x = tiles_x;
    P.tiles_y = tiles_y;
    P.B = (uint32_t)B;
    P.vbytes = vbase;
    P.ibytes = ibase;
    P.ok = true;
    return P;
}

}  // namespace b2s
