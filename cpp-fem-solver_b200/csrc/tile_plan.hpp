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

#ifdef __CUDACC__
#define B2S_TILE_HD __host__ __device__
#else
#define B2S_TILE_HD
#endif

namespace b2s {

constexpr int kTileMaxSweeps = 16;
constexpr uint32_t kTileThreads = 768;
constexpr uint32_t kTileMaxQ = 4;  // extended rows per thread
constexpr uint32_t kTileNoDep = 0xFFFFu;
constexpr int kTileMaxTiles = 160;  // the kernel's all-reduce: 5 tiles per lane of one warp
// the breadth-first planner runs on the host at set-up; above this many rows it
// would cost more than it saves, and only 5-point grids (closed forms) are tiled
constexpr uint32_t kTilePlanHostMaxRows = 1u << 16;

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
    // rows of layers 0..d of the lower triangle's set; layer 0 is the owned
    // rows, or the whole upper set in a fused plan (rows n_own..lcnt[0]-1 are
    // then the upper halo, and o_lhalo lists the rows past lcnt[0])
    uint16_t lcnt[kTileMaxSweeps + 1];
    uint16_t ucnt[kTileMaxSweeps + 1];
};

struct TilePlan
{
    bool ok = false;
    // fused: the forward (lower) set is grown from the upper set instead of the
    // owned rows, so the backward sweeps find all their right-hand sides in the
    // CTA and one grid-wide exchange per iteration goes away
    bool fused = false;
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
// (each sweep vector holds the set and one spare slot: tile_ystride)
inline uint32_t tile_ystride(uint32_t max_ext) { return tile_align16(4ull * (max_ext + 1)) / 4; }
inline uint32_t tile_work_bytes(uint32_t max_ext, uint32_t max_ae)
{
    return std::max<uint32_t>(8 * tile_ystride(max_ext), tile_align16(8ull * max_ae));
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
                                 uint32_t smem_limit, unsigned workers, bool fused);

// The fused layout is tried first (fused_first), then the separate one, for
// the best 2-D block shape; strips (separate sets) are the last resort.
inline TilePlan plan_tiles(uint32_t n, const uint32_t* lo_rp, const uint32_t* lo_ci, const uint32_t* up_rp,
                           const uint32_t* up_ci, int k, int sm_count, uint32_t smem_limit, unsigned workers,
                           bool fused_first = true)
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
    for (int f = fused_first ? 1 : 0; f >= 0; --f)
    {
        P = plan_tiles_shape(n, lo_rp, lo_ci, up_rp, up_ci, k, B, bx, by, smem_limit, workers, f != 0);
        if (P.ok) return P;
    }
    if (bx != 1)  // the blocks' halos outgrew a CTA (dependencies that cross block columns): strips
    {
        const uint64_t B1 = std::max<uint64_t>(1, (n + (uint64_t)sm_count - 1) / (uint64_t)sm_count);
        P = plan_tiles_shape(n, lo_rp, lo_ci, up_rp, up_ci, k, B1, 1, (n + B1 - 1) / B1, smem_limit, workers, false);
    }
    return P;
}

// One tile shape: blocks of w = ceil(B / bx) grid columns by h = ceil(ny / by)
// grid rows, row i at (i mod B, i div B).
inline TilePlan plan_tiles_shape(uint32_t n, const uint32_t* lo_rp, const uint32_t* lo_ci, const uint32_t* up_rp,
                                 const uint32_t* up_ci, int k, uint64_t B, uint64_t bx, uint64_t by,
                                 uint32_t smem_limit, unsigned workers, bool fused)
{
    TilePlan P;
    P.n = n;
    P.k = (uint32_t)k;
    P.fused = fused;
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
        if (!tile_extend(T.own, up_rp, up_ci, k, 3 * t + 1, mk, lc, T.eu, T.udeps, T.ucnt)) return;
        if (!tile_extend(fused ? T.eu : T.own, lo_rp, lo_ci, k, 3 * t, mk, lc, T.el, T.ldeps, T.lcnt)) return;
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
        D.o_lhalo = seg(4ull * (D.n_el - T.lcnt[0]));  // rows of the lower set past its layer 0
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
        put(D.o_lhalo, T.el.data() + D.lcnt[0], 4 * (size_t)(D.n_el - D.lcnt[0]));
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

// ------------------------------------------------------------------ 5-point grids
//
// A pattern whose strict lower entries are exactly, in column order,
// {i - B if y > 0, i - 1 if x > 0} for x = i mod B, y = i div B, n = B * ny
// (the natural-order 5-point stencil) has closed-form tile sets: for the
// block [x0, x1) x [y0, y1) and k sweeps, the lower set holds the points of
// the box [x0 - k, x1) x [y0 - k, y1) at distance dL = max(0, x0 - x) +
// max(0, y0 - y) <= k, layer dL; the upper set mirrors it; the SpMV's columns
// are the block and its one-wide ring.  plan_tiles_grid5 lays the blobs out
// from these counts alone (no pass over the matrix), and grid5_build_elem /
// grid5_build_dep write a tile's index blob one element at a time -- on the
// device at set-up, and on the CPU in the tests, where it must equal
// plan_tiles' output byte for byte.

struct TileGeom
{
    uint32_t x0, x1, y0, y1;  // the block
};

// the pattern check (rp / ci: L with or without its diagonal last)
inline bool is_grid5(uint32_t n, const uint32_t* rp, const uint32_t* ci, uint32_t B, bool diag_last)
{
    if (B == 0 || n % B) return false;
    for (uint32_t i = 0; i < n; ++i)
    {
        const uint32_t x = i % B, y = i / B;
        uint32_t e = rp[i];
        const uint32_t e1 = rp[i + 1] - (diag_last ? 1u : 0u);
        if (diag_last && (rp[i + 1] == rp[i] || ci[rp[i + 1] - 1] != i)) return false;
        if (y > 0 && (e >= e1 || ci[e++] != i - B)) return false;
        if (x > 0 && (e >= e1 || ci[e++] != i - 1)) return false;
        if (e != e1) return false;
    }
    return true;
}

// points at distance d >= 1 from a block side: rows/columns clipped at ka / kb
B2S_TILE_HD inline uint32_t grid5_layer(uint32_t d, uint32_t w, uint32_t h, uint32_t ka, uint32_t kb)
{
    uint32_t c = (d <= ka ? h : 0) + (d <= kb ? w : 0);
    for (uint32_t a = 1; a <= ka && a < d; ++a)
        if (d - a <= kb) ++c;
    return c;
}

inline TilePlan plan_tiles_grid5_mode(uint32_t n, uint32_t B, int k, int sm_count, uint32_t smem_limit,
                                      std::vector<TileGeom>& geom, bool fused);

// the fused layout first, then the separate one (as plan_tiles)
inline TilePlan plan_tiles_grid5(uint32_t n, uint32_t B, int k, int sm_count, uint32_t smem_limit,
                                 std::vector<TileGeom>& geom, bool fused_first = true)
{
    TilePlan P;
    for (int f = fused_first ? 1 : 0; f >= 0; --f)
    {
        P = plan_tiles_grid5_mode(n, B, k, sm_count, smem_limit, geom, f != 0);
        if (P.ok) return P;
    }
    return P;
}

// the block grown by k up and right (clipped): a fused plan's lower set is
// this block's lower set with the upper set (its staircase) as layer 0
B2S_TILE_HD inline TileGeom grid5_fwd_block(const TileGeom& G, uint32_t B, uint32_t ny, uint32_t K, bool fused)
{
    TileGeom F = G;
    if (fused)
    {
        F.x1 = B < G.x1 + K ? B : G.x1 + K;
        F.y1 = ny < G.y1 + K ? ny : G.y1 + K;
    }
    return F;
}

inline TilePlan plan_tiles_grid5_mode(uint32_t n, uint32_t B, int k, int sm_count, uint32_t smem_limit,
                                      std::vector<TileGeom>& geom, bool fused)
{
    TilePlan P;
    P.n = n;
    P.k = (uint32_t)k;
    P.fused = fused;
    if (!n || !B || n % B || k < 1 || k > kTileMaxSweeps || sm_count < 1) return P;
    sm_count = std::min(sm_count, kTileMaxTiles);
    const uint64_t ny = n / B;
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
    const uint64_t w = (B + bx - 1) / bx, h = (ny + by - 1) / by;
    const uint32_t tiles_x = (uint32_t)((B + w - 1) / w), tiles_y = (uint32_t)((ny + h - 1) / h);
    const uint32_t ntiles = tiles_x * tiles_y;
    P.desc.resize(ntiles);
    geom.resize(ntiles);
    uint64_t vbase = 0, ibase = 0;
    uint32_t max_pair = 0;
    for (uint32_t t = 0; t < ntiles; ++t)
    {
        TileGeom& G = geom[t];
        G.x0 = (uint32_t)((t % tiles_x) * w);
        G.x1 = (uint32_t)std::min<uint64_t>(B, G.x0 + w);
        G.y0 = (uint32_t)((t / tiles_x) * h);
        G.y1 = (uint32_t)std::min<uint64_t>(ny, G.y0 + h);
        const uint32_t tw = G.x1 - G.x0, th = G.y1 - G.y0, K = (uint32_t)k;
        TileDesc& D = P.desc[t];
        std::memset(&D, 0, sizeof(D));
        D.n_own = tw * th;
        // lower set: clipped at the grid's left / bottom edges
        const uint32_t lka = std::min(K, G.x0), lkb = std::min(K, G.y0);
        const uint32_t uka = std::min<uint32_t>(K, B - G.x1), ukb = std::min<uint32_t>(K, (uint32_t)ny - G.y1);
        uint32_t cu = D.n_own;
        D.ucnt[0] = (uint16_t)D.n_own;
        for (uint32_t d = 1; d <= K; ++d)
        {
            cu += grid5_layer(d, tw, th, uka, ukb);
            if (cu >= kTileNoDep) return P;
            D.ucnt[d] = (uint16_t)cu;
        }
        const TileGeom F = grid5_fwd_block(G, B, (uint32_t)ny, K, fused);
        uint32_t cl = fused ? cu : D.n_own;
        D.lcnt[0] = (uint16_t)cl;
        for (uint32_t d = 1; d <= K; ++d)
        {
            cl += grid5_layer(d, F.x1 - F.x0, F.y1 - F.y0, lka, lkb);
            if (cl >= kTileNoDep) return P;
            D.lcnt[d] = (uint16_t)cl;
        }
        D.n_el = cl;
        D.n_eu = cu;
        D.n_ae = D.n_own + (G.x0 > 0 ? th : 0) + (G.x1 < B ? th : 0) + (G.y0 > 0 ? tw : 0) + (G.y1 < ny ? tw : 0);
        D.nnz = D.n_own + th * (tw - (G.x0 == 0)) + th * (tw - (G.x1 == B)) + tw * (th - (G.y0 == 0)) +
                tw * (th - (G.y1 == ny));
        if (D.n_el > kTileThreads * kTileMaxQ || D.n_eu > kTileThreads * kTileMaxQ || D.n_ae >= kTileNoDep) return P;
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
        D.o_lhalo = seg(4ull * (D.n_el - D.lcnt[0]));  // rows of the lower set past its layer 0
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
        max_pair = std::max(max_pair, D.vbytes + D.ibytes);
        P.max_ext = std::max(P.max_ext, std::max(D.n_el, D.n_eu));
        P.max_own = std::max(P.max_own, D.n_own);
        P.max_ae = std::max(P.max_ae, D.n_ae);
    }
    P.work = max_pair;
    P.smem = max_pair + tile_work_bytes(P.max_ext, P.max_ae);
    P.Q = (P.max_ext + kTileThreads - 1) / kTileThreads;
    if (P.smem > smem_limit || P.Q > kTileMaxQ) return P;
    P.ntiles = ntiles;
    P.tiles_x = tiles_x;
    P.tiles_y = tiles_y;
    P.B = B;
    P.vbytes = vbase;
    P.ibytes = ibase;
    P.ok = true;
    return P;
}

// ---- a tile's index blob, one element at a time (the device builds it with
// one thread per element; the tests check it against plan_tiles byte for byte).
//
// A set's box (lower: the block grown by k down and left, upper: up and
// right) is walked in row-major order; an entry at distance d >= 1 from the
// block (d = da + db, the distances along x and y) takes the next local index
// of layer d.  Its rank inside layer d has a closed form: rows of the box
// before it hold, per row, the whole block width when d = db (da = 0) or the
// one entry at da = d - db (when it lies inside the box), and in its own row
// no earlier entry of layer d precedes it unless da = 0.  In a fused plan the
// lower set is that of the block grown up and right (grid5_fwd_block), with
// the upper set as its layer 0.
struct Grid5Box
{
    uint32_t bx0, bx1, by0, by1;
};

B2S_TILE_HD inline Grid5Box grid5_box(const TileGeom& G, uint32_t B, uint32_t ny, uint32_t K, bool lo)
{
    Grid5Box b;
    b.bx0 = lo ? (G.x0 > K ? G.x0 - K : 0) : G.x0;
    b.by0 = lo ? (G.y0 > K ? G.y0 - K : 0) : G.y0;
    b.bx1 = lo ? G.x1 : (B < G.x1 + K ? B : G.x1 + K);
    b.by1 = lo ? G.y1 : (ny < G.y1 + K ? ny : G.y1 + K);
    return b;
}

B2S_TILE_HD inline uint32_t grid5_dx(const TileGeom& G, bool lo, uint32_t x)
{
    return lo ? (x < G.x0 ? G.x0 - x : 0u) : (x >= G.x1 ? x - G.x1 + 1u : 0u);
}

B2S_TILE_HD inline uint32_t grid5_dy(const TileGeom& G, bool lo, uint32_t y)
{
    return lo ? (y < G.y0 ? G.y0 - y : 0u) : (y >= G.y1 ? y - G.y1 + 1u : 0u);
}

// entries of layer d in box row y
B2S_TILE_HD inline uint32_t grid5_row_count(const TileGeom& G, const Grid5Box& b, bool lo, uint32_t y, uint32_t d)
{
    const uint32_t db = grid5_dy(G, lo, y);
    if (d < db) return 0;
    const uint32_t e = d - db;
    if (e == 0) return G.x1 - G.x0;
    return lo ? (G.x0 >= b.bx0 + e ? 1u : 0u) : (G.x1 - 1u + e < b.bx1 ? 1u : 0u);
}

// local index of box point (x, y) at distance d in [1, K] from block G:
// cnt[d-1] plus its rank in layer d, or kTileNoDep past cnt[d]
B2S_TILE_HD inline uint32_t grid5_layer_index(const uint16_t* cnt, const TileGeom& G, const Grid5Box& b, bool lo,
                                              uint32_t x, uint32_t y, uint32_t d)
{
    uint32_t rank = 0;
    // rows of the box before y: those off the block (db >= 1) one by one,
    // those beside the block (db = 0) hold one entry of layer d each
    const uint32_t side0 = lo ? G.y0 : b.by0, side1 = lo ? b.by1 : G.y1;  // rows with db = 0
    const uint32_t per_side = grid5_row_count(G, b, lo, side0 < side1 ? side0 : b.by0, d);
    for (uint32_t yy = b.by0; yy < y; ++yy)
    {
        if (yy >= side0 && yy < side1)
        {
            const uint32_t last = y < side1 ? y : side1;
            rank += (last - yy) * per_side;
            yy = last - 1;
            continue;
        }
        rank += grid5_row_count(G, b, lo, yy, d);
    }
    if (grid5_dx(G, lo, x) == 0) rank += x - G.x0;
    const uint32_t l = cnt[d - 1] + rank;
    return l < cnt[d] ? l : kTileNoDep;
}

// the local index of grid point (x, y) in a tile's lower (lo) or upper set, or
// kTileNoDep when the point is outside it
B2S_TILE_HD inline uint32_t grid5_local(const TileDesc& D, const TileGeom& G, uint32_t B, uint32_t ny, uint32_t K,
                                        bool lo, bool fused, uint32_t x, uint32_t y)
{
    const TileGeom F = lo ? grid5_fwd_block(G, B, ny, K, fused) : G;
    const Grid5Box b = grid5_box(F, B, ny, K, lo);
    if (x < b.bx0 || x >= b.bx1 || y < b.by0 || y >= b.by1) return kTileNoDep;
    const uint32_t d = grid5_dx(F, lo, x) + grid5_dy(F, lo, y);
    if (d == 0)
    {
        if (lo && fused) return grid5_local(D, G, B, ny, K, false, false, x, y);  // the upper set (layer 0)
        return (y - G.y0) * (G.x1 - G.x0) + (x - G.x0);
    }
    if (d > K) return kTileNoDep;
    return grid5_layer_index(lo ? D.lcnt : D.ucnt, F, b, lo, x, y, d);
}

// Elements of a tile's index blob other than the dependencies: the owned
// rows, the two sets' box points, the SpMV ring and the owned rows' entries.
B2S_TILE_HD inline uint32_t grid5_elements(const TileDesc& D, const TileGeom& G, uint32_t B, uint32_t ny, uint32_t K,
                                           bool fused)
{
    const Grid5Box lb = grid5_box(grid5_fwd_block(G, B, ny, K, fused), B, ny, K, true);
    const Grid5Box ub = grid5_box(G, B, ny, K, false);
    return D.n_own + (lb.bx1 - lb.bx0) * (lb.by1 - lb.by0) + (ub.bx1 - ub.bx0) * (ub.by1 - ub.by0) +
           (D.n_ae - D.n_own) + D.n_own;
}

// Writes element e (< grid5_elements) of a tile's index blob; false when an
// index falls outside its segment.  The dependencies follow once the halos
// are in place (grid5_build_dep).
B2S_TILE_HD inline bool grid5_build_elem(const TileDesc& D, const TileGeom& G, uint32_t B, uint32_t ny, uint32_t K,
                                         bool fused, uint32_t e, uint8_t* ib)
{
    const uint32_t tw = G.x1 - G.x0, th = G.y1 - G.y0;
    if (e < D.n_own)
    {
        reinterpret_cast<uint32_t*>(ib + D.o_owned)[e] = (G.y0 + e / tw) * B + G.x0 + e % tw;
        return true;
    }
    e -= D.n_own;
    for (int side = 0; side < 2; ++side)
    {
        const bool lo = side == 0;
        const TileGeom F = lo ? grid5_fwd_block(G, B, ny, K, fused) : G;
        const Grid5Box b = grid5_box(F, B, ny, K, lo);
        const uint32_t bw = b.bx1 - b.bx0, sz = bw * (b.by1 - b.by0);
        if (e < sz)
        {
            const uint32_t x = b.bx0 + e % bw, y = b.by0 + e / bw;
            const uint32_t d = grid5_dx(F, lo, x) + grid5_dy(F, lo, y);
            if (d == 0 || d > K) return true;
            const uint32_t l = grid5_layer_index(lo ? D.lcnt : D.ucnt, F, b, lo, x, y, d);
            const uint32_t base = lo ? D.lcnt[0] : D.n_own;
            if (l == kTileNoDep || l < base) return false;
            reinterpret_cast<uint32_t*>(ib + (lo ? D.o_lhalo : D.o_uhalo))[l - base] = y * B + x;
            return true;
        }
        e -= sz;
    }
    const bool L = G.x0 > 0, R = G.x1 < B, Bo = G.y0 > 0, T = G.y1 < ny;
    const uint32_t nb = Bo ? tw : 0, per_row = (L ? 1u : 0u) + (R ? 1u : 0u);
    if (e < D.n_ae - D.n_own)
    {
        uint32_t g;
        if (e < nb)
            g = (G.y0 - 1) * B + G.x0 + e;
        else if (e - nb < th * per_row)
        {
            const uint32_t r = e - nb, y = G.y0 + r / per_row;
            g = (r % per_row == 0 && L) ? y * B + G.x0 - 1 : y * B + G.x1;
        }
        else
        {
            const uint32_t x = G.x0 + (e - nb - th * per_row);
            if (!T || x >= G.x1) return false;
            g = G.y1 * B + x;
        }
        reinterpret_cast<uint32_t*>(ib + D.o_ahalo)[e] = g;
        return true;
    }
    e -= D.n_ae - D.n_own;
    if (e >= D.n_own) return false;
    // owned row q = e: its CSR offset (the entries of the block's earlier
    // rows and of the row's earlier points) and its columns in local numbering
    const uint32_t q = e, x = G.x0 + q % tw, y = G.y0 + q / tw;
    auto cnt_row = [&](uint32_t yy, uint32_t xa, uint32_t xb) {  // entries of points [xa, xb) of row yy
        const uint32_t w = xb - xa;
        uint32_t c = w * (1u + (yy > 0) + (yy + 1 < ny));
        c += w - (xa == 0 && w ? 1u : 0u);  // left neighbours
        c += w - (xb == B && w ? 1u : 0u);  // right neighbours
        return c;
    };
    uint32_t off = 0;
    for (uint32_t yy = G.y0; yy < y; ++yy) off += cnt_row(yy, G.x0, G.x1);
    off += cnt_row(y, G.x0, x);
    const uint32_t c = 1u + (y > 0) + (x > 0) + (x + 1 < B) + (y + 1 < ny);
    if (off + c > D.nnz) return false;
    uint32_t* arp = reinterpret_cast<uint32_t*>(ib + D.o_arp);
    uint16_t* acol = reinterpret_cast<uint16_t*>(ib + D.o_acol);
    if (q == 0) arp[0] = 0;
    arp[q + 1] = off + c;
    auto col = [&](uint32_t xx, uint32_t yy) -> uint32_t {
        if (xx >= G.x0 && xx < G.x1 && yy >= G.y0 && yy < G.y1) return (yy - G.y0) * tw + (xx - G.x0);
        if (yy + 1 == G.y0) return D.n_own + (xx - G.x0);
        if (yy == G.y1) return D.n_own + nb + th * per_row + (xx - G.x0);
        return D.n_own + nb + (yy - G.y0) * per_row + (xx + 1 == G.x0 ? 0u : (L ? 1u : 0u));
    };
    uint32_t p = off;
    if (y > 0) acol[p++] = (uint16_t)col(x, y - 1);
    if (x > 0) acol[p++] = (uint16_t)col(x - 1, y);
    acol[p++] = (uint16_t)q;
    if (x + 1 < B) acol[p++] = (uint16_t)col(x + 1, y);
    if (y + 1 < ny) acol[p++] = (uint16_t)col(x, y + 1);
    return true;
}

// Dependencies of row t of the lower (lo) or upper set, after the halos are
// written: {first, second} local indices in column order.
B2S_TILE_HD inline void grid5_build_dep(const TileDesc& D, const TileGeom& G, uint32_t B, uint32_t ny, uint32_t K,
                                        bool lo, bool fused, uint32_t t, uint8_t* ib)
{
    const uint32_t tw = G.x1 - G.x0;
    uint32_t x, y;
    if (t < D.n_own)
    {
        x = G.x0 + t % tw;
        y = G.y0 + t / tw;
    }
    else
    {
        const uint32_t base = lo ? D.lcnt[0] : D.n_own;  // (fused lower set: the upper halo before base)
        const uint32_t g = t < base ? reinterpret_cast<const uint32_t*>(ib + D.o_uhalo)[t - D.n_own]
                                    : reinterpret_cast<const uint32_t*>(ib + (lo ? D.o_lhalo : D.o_uhalo))[t - base];
        x = g % B;
        y = g / B;
    }
    uint32_t s[2] = {kTileNoDep, kTileNoDep}, e = 0;
    if (lo)
    {
        if (y > 0) s[e++] = grid5_local(D, G, B, ny, K, true, fused, x, y - 1);
        if (x > 0) s[e++] = grid5_local(D, G, B, ny, K, true, fused, x - 1, y);
    }
    else
    {
        if (x + 1 < B) s[e++] = grid5_local(D, G, B, ny, K, false, false, x + 1, y);
        if (y + 1 < ny) s[e++] = grid5_local(D, G, B, ny, K, false, false, x, y + 1);
    }
    reinterpret_cast<uint32_t*>(ib + (lo ? D.o_ldeps : D.o_udeps))[t] = s[0] | (s[1] << 16);
}

}  // namespace b2s
