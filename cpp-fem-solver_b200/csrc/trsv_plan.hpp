// Host planning of the chunked triangular solve (k_trsv_chunk).
//
// Host-only C++ (no CUDA runtime calls), so that the planner and the index
// arithmetic of the kernel can be exercised on a machine without a GPU.
//
// A triangle's rows, in dependency order (ascending for a lower factor,
// descending for an upper one), are cut into chunks of contiguous rows that
// fit one CTA's shared memory.  Inside a chunk the rows are renumbered into
// "positions" sorted by their global level (the longest dependency chain
// ending at the row in the whole triangle), so that a level is a contiguous
// run of positions.  Global rather than chunk-local levels matter: a chunk's
// first rows often depend on the last rows of the previous chunk, and with
// local levels they would sit in the chunk's first level and hold every
// other row of the chunk until the previous chunk had finished; ordered by
// global level, each chunk follows the wavefront its predecessor produces.  Each row keeps
// only its dependency entries (j < i for lower, j > i for upper), in column
// order; an entry names either the position of an in-chunk row or a "slot":
// a value of an earlier chunk that the CTA's producer warp fetches into shared
// memory.  Slots are numbered in the order the chunk first needs them.
//
// Rows may be blocks (BAIJ, bs x bs): a dependency entry then carries bs*bs
// values, a row bs right-hand-side / solution values, and the divisor of a
// row is either absent (unit triangle), one value (scalar) or a bs x bs
// inverse block ("dv" values per row).
//
// Per chunk the planner writes a metadata blob, copied verbatim into shared
// memory by the kernel:
//     slc  u16[nd]    dependency entries: position, or 0x8000 | slot
//     rec  u16x4[nr]  per position: local row (row - lo) | 0x8000 when rows
//                     of another chunk depend on it (it publishes), then the
//                     position's range [e0, e1) in slc, then 0
//     slv  u16[nl+1]  level boundaries (positions)
// and a value blob per precision (written on the device by k_chunk_pack):
//     sv   VT[nd*bs*bs]  dependency values (blocks row-major), same order as slc
//     sd   VT[nr*dv]     divisors by position (absent for a unit triangle)
// Every segment starts on a 16-byte boundary and every blob is a multiple of
// 16 bytes, so the kernel copies them with 16-byte cp.async.
#pragma once
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <vector>

#ifdef __CUDACC__
#define B2S_HD __host__ __device__ __forceinline__
#else
#define B2S_HD inline
#endif

namespace b2s {

constexpr uint32_t kChunkSmemBudget = 216 * 1024;  // dynamic shared memory a chunk may use
constexpr uint32_t kChunkSmemLimit = 227 * 1024;   // sm_100 per-CTA maximum
constexpr uint32_t kChunkMaxRows = 32767;          // 15-bit position / local row
constexpr uint32_t kChunkMaxDeps = 65535;          // 16-bit offsets into slc
constexpr uint32_t kChunkMaxSlots = 32767;         // 15-bit slot index

B2S_HD uint32_t al16(uint64_t b) { return (uint32_t)((b + 15u) & ~uint64_t(15)); }

struct ChunkDesc
{
    uint32_t lo;    // lowest row of the chunk's contiguous row range
    uint32_t nr;    // rows
    uint32_t nd;    // dependency entries
    uint32_t nl;    // local levels
    uint32_t ns;    // slots (values of earlier chunks)
    uint32_t meta;  // metadata blob offset, 16-byte units
    uint32_t v64;   // FP64 value blob offset, 16-byte units
    uint32_t v32;   // FP32 value blob offset, 16-byte units
    uint32_t slot;  // offset into slot_row
    uint32_t dep;   // offset into src (one per dependency entry)
};

// byte offsets inside the metadata blob (independent of the value type)
struct MetaLayout
{
    uint32_t slc, rec, slv, bytes;
};

B2S_HD MetaLayout meta_layout(uint32_t nr, uint32_t nd, uint32_t nl)
{
    MetaLayout m;
    uint32_t o = 0;
    m.slc = o;
    o += al16((uint64_t)nd * 2);
    m.rec = o;
    o += al16((uint64_t)nr * 8);
    m.slv = o;
    o += al16((uint64_t)(nl + 1) * 2);
    m.bytes = o;
    return m;
}

// fields of a position record (two u32 words: {perm, e0}, {e1, 0})
B2S_HD uint32_t rec_perm(uint32_t w0) { return w0 & 0xffffu; }
B2S_HD uint32_t rec_e0(uint32_t w0) { return w0 >> 16; }
B2S_HD uint32_t rec_e1(uint32_t w1) { return w1 & 0xffffu; }

// byte offsets of the chunk's shared memory: [values][metadata][x][rhs][slot values][slot ready]
struct SmemLayout
{
    uint32_t sv, sd, vals;  // value blob: values, divisors, blob bytes
    uint32_t meta;          // start of the metadata blob
    MetaLayout m;           // offsets relative to `meta`
    uint32_t sx, sr, xv, xr, total;
};

B2S_HD SmemLayout smem_layout(uint32_t nr, uint32_t nd, uint32_t nl, uint32_t ns, uint32_t vs, uint32_t xs,
                              uint32_t rs, uint32_t bs, uint32_t dv)
{
    SmemLayout L;
    uint32_t o = 0;
    L.sv = o;
    o += al16((uint64_t)nd * bs * bs * vs);
    L.sd = o;
    o += al16((uint64_t)nr * dv * vs);
    L.vals = o;
    L.meta = o;
    L.m = meta_layout(nr, nd, nl);
    o += L.m.bytes;
    L.sx = o;
    o += al16((uint64_t)nr * bs * xs);
    L.sr = o;
    o += al16((uint64_t)nr * bs * rs);
    L.xv = o;
    o += al16((uint64_t)ns * bs * xs);
    L.xr = o;
    o += al16((uint64_t)ns * 4);
    L.total = o;
    return L;
}

struct ChunkPlan
{
    uint32_t n = 0;
    bool lower = true;
    uint32_t bs = 1, dv = 1;         // block size; divisor values per row (0: unit)
    std::vector<ChunkDesc> desc;     // in processing order
    std::vector<uint8_t> meta;       // all metadata blobs
    std::vector<uint32_t> slot_row;  // all slots: the row whose value a slot holds
    std::vector<uint32_t> src;       // per dependency entry: index into the factor's values
    uint64_t v64_units = 0, v32_units = 0;
    uint32_t max_level_rows = 0;
    bool ok = false;  // false when some row alone does not fit a chunk

    // largest shared-memory footprint of a chunk for the given element sizes
    uint32_t smem_bytes(uint32_t vs, uint32_t xs, uint32_t rs) const
    {
        uint32_t b = 0;
        for (const ChunkDesc& d : desc) b = std::max(b, smem_layout(d.nr, d.nd, d.nl, d.ns, vs, xs, rs, bs, dv).total);
        return b;
    }
};

// Global level of each row: the longest dependency chain ending at it (0 for
// a row without dependencies).  Dependencies are j < i (lower) or j > i (upper).
inline void compute_levels(uint32_t n, const uint32_t* rp, const uint32_t* ci, bool lower, std::vector<uint32_t>& lev)
{
    lev.assign(n, 0);
    for (uint32_t t = 0; t < n; ++t)
    {
        const uint32_t r = lower ? t : n - 1 - t;
        uint32_t l = 0;
        for (uint32_t p = rp[r]; p < rp[r + 1]; ++p)
        {
            const uint32_t j = ci[p];
            if (lower ? j < r : j > r) l = std::max(l, lev[j] + 1);
        }
        lev[r] = l;
    }
}

// Pattern of the strict transpose of a triangle (j < i entries of rp/ci for
// lower -> rows j with columns i ascending), on the host.
inline void strict_transpose(uint32_t n, const uint32_t* rp, const uint32_t* ci, bool lower,
                             std::vector<uint32_t>& trp, std::vector<uint32_t>& tci)
{
    trp.assign((size_t)n + 1, 0);
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
            if (lower ? ci[p] < i : ci[p] > i) trp[ci[p] + 1]++;
    for (uint32_t i = 0; i < n; ++i) trp[i + 1] += trp[i];
    tci.resize(trp[n] ? trp[n] : 1);
    std::vector<uint32_t> off(trp.begin(), trp.end() - 1);
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t p = rp[i]; p < rp[i + 1]; ++p)
            if (lower ? ci[p] < i : ci[p] > i) tci[off[ci[p]]++] = i;
}

// Plan the chunks of a triangle with (block) CSR pattern rp/ci (dependency
// entries are j < i for lower, j > i for upper; other entries are ignored).
// vs, xs, rs: element sizes of values, solution and right-hand side the chunks
// are sized for; bs: block size; dv: divisor values per row (0 for a unit
// triangle, 1 for a scalar divisor, bs*bs for an inverse block).
// glev: the rows' global levels when the caller has them (compute_levels).
inline ChunkPlan plan_chunks(uint32_t n, const uint32_t* rp, const uint32_t* ci, bool lower, uint32_t dv, uint32_t vs,
                             uint32_t xs, uint32_t rs, uint32_t budget = kChunkSmemBudget, uint32_t bs = 1,
                             const std::vector<uint32_t>* glev_in = nullptr)
{
    ChunkPlan P;
    P.n = n;
    P.lower = lower;
    P.bs = bs;
    P.dv = dv;
    const uint64_t bv = (uint64_t)bs * bs;
    if (!n)
    {
        P.ok = true;
        return P;
    }
    auto is_dep = [&](uint32_t i, uint32_t j) { return lower ? j < i : j > i; };
    std::vector<uint32_t> glev_own;
    if (!glev_in) compute_levels(n, rp, ci, lower, glev_own);
    const std::vector<uint32_t>& glev = glev_in ? *glev_in : glev_own;
    std::vector<uint32_t> stamp(n, 0);     // chunk id + 1 when j already has a slot in the chunk
    std::vector<uint32_t> slot_of(n, 0);   // slot of j in the chunk that stamped it
    std::vector<uint32_t> llev(n, 0);      // local level
    std::vector<uint32_t> pos_of(n, 0);    // position inside its chunk
    std::vector<uint64_t> perm_at(n, 0);   // byte offset of the row's perm entry in P.meta
    std::vector<uint8_t> publish(n, 0);
    std::vector<uint32_t> rows, cnt;
    const uint32_t slack = 16 * 10;
    uint32_t pos = 0, cid = 0;
    while (pos < n)
    {
        // ---- grow the chunk while it fits
        uint64_t bytes = slack;
        uint32_t end = pos, nd = 0, ns = 0;
        const uint32_t first = lower ? pos : n - 1 - pos;  // first row in processing order
        const uint32_t tag = cid + 1;
        while (end < n)
        {
            const uint32_t r = lower ? end : n - 1 - end;
            uint32_t ndep = 0, nnew = 0;
            for (uint32_t p = rp[r]; p < rp[r + 1]; ++p)
            {
                const uint32_t j = ci[p];
                if (!is_dep(r, j)) continue;
                ++ndep;
                const bool inside = lower ? j >= pos : j <= first;
                if (!inside && stamp[j] != tag) ++nnew;
            }
            const uint64_t b = (uint64_t)vs * (ndep * bv + dv) + 2ull * ndep + 10 + (uint64_t)bs * (xs + rs) +
                               (uint64_t)nnew * (bs * xs + 4);
            const bool fits = bytes + b <= budget && end - pos + 1 <= kChunkMaxRows && nd + ndep <= kChunkMaxDeps &&
                              ns + nnew <= kChunkMaxSlots;
            if (!fits)
            {
                if (end == pos) return P;  // a single row does not fit: ok stays false
                break;
            }
            bytes += b;
            nd += ndep;
            ns += nnew;
            for (uint32_t p = rp[r]; p < rp[r + 1]; ++p)
            {
                const uint32_t j = ci[p];
                if (!is_dep(r, j)) continue;
                const bool inside = lower ? j >= pos : j <= first;
                if (!inside) stamp[j] = tag;
            }
            ++end;
        }
        const uint32_t nr = end - pos;
        const uint32_t lo = lower ? pos : n - end;
        // ---- the chunk's levels: its distinct global levels, compressed
        rows.clear();
        uint32_t gmin = ~0u, gmax = 0;
        for (uint32_t t = pos; t < end; ++t)
        {
            const uint32_t r = lower ? t : n - 1 - t;
            gmin = std::min(gmin, glev[r]);
            gmax = std::max(gmax, glev[r]);
            rows.push_back(r);
        }
        cnt.assign(gmax - gmin + 1, 0);
        for (uint32_t r : rows) cnt[glev[r] - gmin] = 1;
        uint32_t nl = 0;
        for (uint32_t& c : cnt) c = c ? nl++ : 0u;  // global level -> chunk level
        for (uint32_t r : rows) llev[r] = cnt[glev[r] - gmin];
        // counting sort by level, stable in processing order
        cnt.assign(nl + 1, 0);
        for (uint32_t r : rows) cnt[llev[r] + 1]++;
        for (uint32_t l = 0; l < nl; ++l) cnt[l + 1] += cnt[l];
        for (uint32_t l = 0; l < nl; ++l) P.max_level_rows = std::max(P.max_level_rows, cnt[l + 1] - cnt[l]);
        std::vector<uint32_t> sorted(nr), off(cnt.begin(), cnt.end() - 1);
        for (uint32_t r : rows) sorted[off[llev[r]]++] = r;
        for (uint32_t t = 0; t < nr; ++t) pos_of[sorted[t]] = t;
        // ---- emit the metadata blob
        const MetaLayout M = meta_layout(nr, nd, nl);
        const uint64_t mbase = P.meta.size();
        P.meta.resize(mbase + M.bytes, 0);
        uint8_t* mb = P.meta.data() + mbase;
        auto put16 = [&](uint32_t off_bytes, uint32_t idx, uint32_t val) {
            const uint16_t v16 = (uint16_t)val;
            std::memcpy(mb + off_bytes + 2ull * idx, &v16, 2);
        };
        ChunkDesc D{};
        D.lo = lo;
        D.nr = nr;
        D.nd = nd;
        D.nl = nl;
        D.meta = (uint32_t)(mbase / 16);
        D.slot = (uint32_t)P.slot_row.size();
        D.dep = (uint32_t)P.src.size();
        uint32_t e = 0, s = 0;
        std::vector<uint32_t>& slot_rows = P.slot_row;
        for (uint32_t t = 0; t < nr; ++t)
        {
            const uint32_t r = sorted[t];
            put16(M.rec, 4 * t, r - lo);
            put16(M.rec, 4 * t + 1, e);
            perm_at[r] = mbase + M.rec + 8ull * t;
            for (uint32_t p = rp[r]; p < rp[r + 1]; ++p)
            {
                const uint32_t j = ci[p];
                if (!is_dep(r, j)) continue;
                uint32_t m;
                if (j >= lo && j < lo + nr)
                    m = pos_of[j];
                else
                {
                    // number the slots in the order of first need
                    if (slot_of[j] == 0)
                    {
                        slot_of[j] = s + 1;
                        slot_rows.push_back(j);
                        publish[j] = 1;
                        ++s;
                    }
                    m = 0x8000u | (slot_of[j] - 1);
                }
                put16(M.slc, e, m);
                P.src.push_back(p);
                ++e;
            }
            put16(M.rec, 4 * t + 2, e);
        }
        for (uint32_t l = 0; l <= nl; ++l) put16(M.slv, l, cnt[l]);
        D.ns = s;
        D.v64 = (uint32_t)P.v64_units;
        D.v32 = (uint32_t)P.v32_units;
        P.v64_units += (al16((uint64_t)nd * bv * 8) + al16((uint64_t)nr * dv * 8)) / 16;
        P.v32_units += (al16((uint64_t)nd * bv * 4) + al16((uint64_t)nr * dv * 4)) / 16;
        P.desc.push_back(D);
        // slot numbering reuses slot_of; clear it for the rows of this chunk's slots
        for (uint32_t q = D.slot; q < D.slot + s; ++q) slot_of[P.slot_row[q]] = 0;
        pos = end;
        ++cid;
    }
    // rows read by another chunk publish a ready flag
    for (uint32_t r = 0; r < n; ++r)
        if (publish[r])
        {
            uint16_t v16;
            std::memcpy(&v16, P.meta.data() + perm_at[r], 2);
            v16 |= 0x8000u;
            std::memcpy(P.meta.data() + perm_at[r], &v16, 2);
        }
    if (P.meta.empty()) P.meta.resize(16, 0);
    P.ok = true;
    return P;
}

}  // namespace b2s
