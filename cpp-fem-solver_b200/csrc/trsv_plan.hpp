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
//                     position's range [e0, e1) in slc, then the mask of its
//                     entries (the first 16) that are slots
//     slv  u16[nl+1]  level boundaries (positions)
// and a value blob per precision (written on the device by k_chunk_pack):
//     sv   VT[nd*bs*bs]  dependency values (blocks row-major), same order as slc
//     sd   VT[nr*dv]     divisors by position (absent for a unit triangle)
// Every segment starts on a 16-byte boundary and every blob is a multiple of
// 16 bytes, so the kernel copies them with 16-byte cp.async.
#pragma once
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <new>
#include <mutex>
#include <stdexcept>
#include <thread>
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
    o += al16(((uint64_t)nr * bs + 1) * xs);  // (+1: a zero the scalar solve reads for absent entries)
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
    uint32_t max_row_deps = 0;  // most dependency entries of one row
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

// Run f(c, worker) for c in [0, count) on up to 16 host threads; chunks are
// handed out one at a time.  The first exception thrown by any call is
// rethrown after every worker has stopped.
template <class F>
inline void plan_parallel(uint32_t count, unsigned max_workers, F&& f)
{
    unsigned hw = std::thread::hardware_concurrency();
    unsigned nt = std::min(std::min(hw ? hw : 1u, max_workers), count ? count : 1u);
    std::atomic<uint32_t> next{0};
    std::atomic<bool> failed{false};
    std::exception_ptr err;
    std::mutex m;
    auto work = [&](unsigned t) {
        try
        {
            for (uint32_t c; !failed.load(std::memory_order_relaxed) && (c = next.fetch_add(1)) < count;) f(c, t);
        }
        catch (...)
        {
            std::lock_guard<std::mutex> g(m);
            if (!err) err = std::current_exception();
            failed = true;
        }
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t)
    {
        try
        {
            th.emplace_back(work, t);
        }
        catch (...)
        {
            break;  // fewer workers when a thread cannot start
        }
    }
    work(0);
    for (std::thread& x : th) x.join();
    if (err) std::rethrow_exception(err);
}

// A chunk's range of positions in processing order and its counts.
struct ChunkSpan
{
    uint32_t pos, end, nd, ns, nl, max_rows;
};

// Pass 1 of plan_chunks: grow each chunk over consecutive rows (in processing
// order) while its shared-memory footprint fits.  A dependency on a row of an
// earlier chunk costs a slot the first time the chunk meets it.  False when a
// single row does not fit.
template <bool LOWER>
inline bool plan_grow(uint32_t n, const uint32_t* rp, const uint32_t* ci, uint32_t dv, uint32_t vs, uint32_t xs,
                      uint32_t rs, uint32_t budget, uint32_t bs, std::vector<ChunkSpan>& span)
{
    const uint64_t bv = (uint64_t)bs * bs;
    const uint64_t row_fixed = (uint64_t)vs * dv + 10 + (uint64_t)bs * (xs + rs);
    const uint64_t per_dep = (uint64_t)vs * bv + 2, per_slot = (uint64_t)bs * xs + 4;
    std::vector<uint32_t> stamp(n, 0);  // chunk id + 1 when j already has a slot in the chunk
    std::vector<uint32_t> fresh;        // rows stamped by the row being tried
    const uint32_t slack = 16 * 10;
    uint32_t pos = 0;
    while (pos < n)
    {
        uint64_t bytes = slack;
        uint32_t end = pos, nd = 0, ns = 0;
        // rows of the chunk so far: [pos, r) for lower, (r, n-1-pos] for upper
        const uint32_t edge = LOWER ? pos : n - 1 - pos;
        const uint32_t tag = (uint32_t)span.size() + 1;
        while (end < n)
        {
            const uint32_t r = LOWER ? end : n - 1 - end;
            uint32_t ndep = 0, nnew = 0;
            fresh.clear();
            for (uint32_t p = rp[r]; p < rp[r + 1]; ++p)
            {
                const uint32_t j = ci[p];
                if (LOWER ? j >= r : j <= r) continue;
                ++ndep;
                const bool inside = LOWER ? j >= edge : j <= edge;
                if (!inside && stamp[j] != tag)
                {
                    stamp[j] = tag;
                    fresh.push_back(j);
                    ++nnew;
                }
            }
            const uint64_t b = row_fixed + per_dep * ndep + per_slot * nnew;
            const bool fits = bytes + b <= budget && end - pos + 1 <= kChunkMaxRows && nd + ndep <= kChunkMaxDeps &&
                              ns + nnew <= kChunkMaxSlots;
            if (!fits)
            {
                for (uint32_t j : fresh) stamp[j] = 0;  // the row starts the next chunk
                if (end == pos) return false;
                break;
            }
            bytes += b;
            nd += ndep;
            ns += nnew;
            ++end;
        }
        span.push_back({pos, end, nd, ns, 0, 0});
        pos = end;
    }
    return true;
}

// Plan the chunks of a triangle with (block) CSR pattern rp/ci (dependency
// entries are j < i for lower, j > i for upper; other entries are ignored).
// vs, xs, rs: element sizes of values, solution and right-hand side the chunks
// are sized for; bs: block size; dv: divisor values per row (0 for a unit
// triangle, 1 for a scalar divisor, bs*bs for an inverse block).
// glev: the rows' global levels when the caller has them (compute_levels).
//
// Three passes: (1) serially, grow each chunk over consecutive rows while its
// shared-memory footprint fits (this fixes the chunk boundaries, dependency
// and slot counts); (2) per chunk in parallel, order the rows by global
// level; (3) after a prefix sum of the blob sizes, per chunk in parallel,
// write the metadata blob, the slot rows and the value sources.  Slots are
// numbered per chunk in the order of first need, so the plan does not depend
// on the number of threads.
inline ChunkPlan plan_chunks(uint32_t n, const uint32_t* rp, const uint32_t* ci, bool lower, uint32_t dv, uint32_t vs,
                             uint32_t xs, uint32_t rs, uint32_t budget = kChunkSmemBudget, uint32_t bs = 1,
                             const std::vector<uint32_t>* glev_in = nullptr, unsigned max_workers = 16)
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
    // ---- pass 1: chunk boundaries, dependency entries and slots
    std::vector<ChunkSpan> span;
    const bool grown = lower ? plan_grow<true>(n, rp, ci, dv, vs, xs, rs, budget, bs, span)
                             : plan_grow<false>(n, rp, ci, dv, vs, xs, rs, budget, bs, span);
    if (!grown) return P;  // a single row does not fit a chunk: ok stays false
    const uint32_t nchunks = (uint32_t)span.size();
    // ---- pass 2: each chunk's rows by global level (order[pos..end): rows by position)
    std::vector<uint32_t> order(n), llev(n), pos_of(n);
    plan_parallel(nchunks, max_workers, [&](uint32_t c, unsigned) {
        ChunkSpan& S = span[c];
        uint32_t gmin = ~0u, gmax = 0;
        for (uint32_t t = S.pos; t < S.end; ++t)
        {
            const uint32_t r = lower ? t : n - 1 - t;
            gmin = std::min(gmin, glev[r]);
            gmax = std::max(gmax, glev[r]);
        }
        // the chunk's distinct global levels, compressed
        std::vector<uint32_t> cnt(gmax - gmin + 1, 0);
        for (uint32_t t = S.pos; t < S.end; ++t) cnt[glev[lower ? t : n - 1 - t] - gmin] = 1;
        uint32_t nl = 0;
        for (uint32_t& x : cnt) x = x ? nl++ : 0u;  // global level -> chunk level
        for (uint32_t t = S.pos; t < S.end; ++t)
        {
            const uint32_t r = lower ? t : n - 1 - t;
            llev[r] = cnt[glev[r] - gmin];
        }
        // counting sort by level, stable in processing order
        std::vector<uint32_t> off(nl + 1, 0);
        for (uint32_t t = S.pos; t < S.end; ++t) off[llev[lower ? t : n - 1 - t] + 1]++;
        uint32_t mx = 0;
        for (uint32_t l = 0; l < nl; ++l)
        {
            mx = std::max(mx, off[l + 1]);
            off[l + 1] += off[l];
        }
        for (uint32_t t = S.pos; t < S.end; ++t)
        {
            const uint32_t r = lower ? t : n - 1 - t;
            const uint32_t q = off[llev[r]]++;
            order[S.pos + q] = r;
            pos_of[r] = q;
        }
        S.nl = nl;
        S.max_rows = mx;
    });
    // ---- blob offsets
    P.desc.resize(nchunks);
    uint64_t meta_bytes = 0, ndeps = 0, nslots = 0;
    for (uint32_t c = 0; c < nchunks; ++c)
    {
        const ChunkSpan& S = span[c];
        const uint32_t nr = S.end - S.pos;
        ChunkDesc& D = P.desc[c];
        D = ChunkDesc{};
        D.lo = lower ? S.pos : n - S.end;
        D.nr = nr;
        D.nd = S.nd;
        D.nl = S.nl;
        D.ns = S.ns;
        D.meta = (uint32_t)(meta_bytes / 16);
        D.slot = (uint32_t)nslots;
        D.dep = (uint32_t)ndeps;
        D.v64 = (uint32_t)P.v64_units;
        D.v32 = (uint32_t)P.v32_units;
        meta_bytes += meta_layout(nr, S.nd, S.nl).bytes;
        ndeps += S.nd;
        nslots += S.ns;
        P.v64_units += (al16((uint64_t)S.nd * bv * 8) + al16((uint64_t)nr * dv * 8)) / 16;
        P.v32_units += (al16((uint64_t)S.nd * bv * 4) + al16((uint64_t)nr * dv * 4)) / 16;
        P.max_level_rows = std::max(P.max_level_rows, S.max_rows);
    }
    P.meta.assign(meta_bytes ? meta_bytes : 16, 0);
    std::vector<uint64_t> rec_at(n);  // byte offset of each row's position record in P.meta
    P.src.resize(ndeps);
    P.slot_row.resize(nslots);
    // ---- pass 3: metadata blobs, slot rows, value sources
    // per worker: slot + 1 of row j in the current chunk, 0 when none.  calloc
    // leaves the pages untouched until a chunk's slot rows reach them.
    struct Scratch
    {
        uint32_t* slot_of = nullptr;
        ~Scratch() { std::free(slot_of); }
    };
    std::vector<Scratch> scratch(std::max(1u, std::min(max_workers, 64u)));
    std::vector<uint32_t> chunk_max_deps(nchunks, 0);
    plan_parallel(nchunks, (unsigned)scratch.size(), [&](uint32_t c, unsigned w) {
        const ChunkSpan& S = span[c];
        const ChunkDesc& D = P.desc[c];
        uint32_t*& slot_of = scratch[w].slot_of;
        if (!slot_of && !(slot_of = (uint32_t*)std::calloc(n, sizeof(uint32_t)))) throw std::bad_alloc();
        const MetaLayout M = meta_layout(D.nr, D.nd, D.nl);
        uint8_t* mb = P.meta.data() + (uint64_t)D.meta * 16;
        auto put16 = [&](uint32_t off_bytes, uint32_t idx, uint32_t val) {
            const uint16_t v16 = (uint16_t)val;
            std::memcpy(mb + off_bytes + 2ull * idx, &v16, 2);
        };
        uint32_t e = 0, s = 0, l = 0;
        for (uint32_t t = 0; t < D.nr; ++t)
        {
            const uint32_t r = order[S.pos + t];
            while (l <= llev[r]) put16(M.slv, l++, t);
            put16(M.rec, 4 * t, r - D.lo);
            put16(M.rec, 4 * t + 1, e);
            rec_at[r] = (uint64_t)D.meta * 16 + M.rec + 8ull * t;
            const uint32_t e_row = e;
            uint32_t smask = 0;  // entries (of the first 16) that are slots
            for (uint32_t p = rp[r]; p < rp[r + 1]; ++p)
            {
                const uint32_t j = ci[p];
                if (!is_dep(r, j)) continue;
                uint32_t m;
                if (j >= D.lo && j < D.lo + D.nr)
                    m = pos_of[j];
                else
                {
                    if (slot_of[j] == 0)
                    {
                        if (s >= D.ns) throw std::logic_error("plan_chunks: slot count");
                        slot_of[j] = s + 1;
                        P.slot_row[D.slot + s] = j;
                        ++s;
                    }
                    m = 0x8000u | (slot_of[j] - 1);
                    if (e - e_row < 16) smask |= 1u << (e - e_row);
                }
                if (e >= D.nd) throw std::logic_error("plan_chunks: dependency count");
                put16(M.slc, e, m);
                P.src[D.dep + e] = p;
                ++e;
            }
            put16(M.rec, 4 * t + 2, e);
            put16(M.rec, 4 * t + 3, smask);
            chunk_max_deps[c] = std::max(chunk_max_deps[c], e - e_row);
        }
        put16(M.slv, D.nl, D.nr);
        for (uint32_t q = 0; q < s; ++q) slot_of[P.slot_row[D.slot + q]] = 0;
        if (e != D.nd || s != D.ns) throw std::logic_error("plan_chunks: chunk counts");
    });
    for (uint32_t c = 0; c < nchunks; ++c) P.max_row_deps = std::max(P.max_row_deps, chunk_max_deps[c]);
    // rows read by another chunk publish a ready flag (bit 15 of the record's local-row field)
    for (uint32_t j : P.slot_row)
    {
        uint16_t v16;
        std::memcpy(&v16, P.meta.data() + rec_at[j], 2);
        v16 |= 0x8000u;
        std::memcpy(P.meta.data() + rec_at[j], &v16, 2);
    }
    P.ok = true;
    return P;
}

}  // namespace b2s
