// Range evaluation over equality-encoded indexes (relic: one bitmap per
// distinct value; bin: one bitmap per value bin) and the AND across columns.
//
// The reference evaluates `lo <op> x <op> hi` as
//   relic::evaluate  (src/irelic.cpp:1827): locate -> sumBins(h0, h1)
//   bin::evaluate    (src/ibin.cpp:6614):   locate -> sumBins over the bins
//                    wholly inside the range, plus the rows of the edge
//                    bins whose values pass the comparison (checkBin /
//                    doScan on the raw values, src/ibin.cpp:2057-2304)
//   index::sumBins   (src/index.cpp:6450): OR of bitmaps [h0, h1), or the
//                    complement OR'ed and flipped when that reads fewer bytes
//   countQuery::doEvaluate (src/countQuery.cpp:953-1036): AND of the terms.
// The hit set is exactly the rows whose value passes the comparison done in
// double (qContinuousRange::inRange, src/qExpr.cpp:1647-1667); the reference's
// OR order (a heap ordered by pointer values) changes only the words of its
// intermediate results, never the bits.
//
// Work item = (query, tile of RT groups), claimed in query-major order
// (row ids by a decoupled look-back in claim order, so each query's ids are
// contiguous and ascending), tile-major order (the queries of a batch share
// each tile's words in L2; counts only, or two passes around a scan of the
// items' hits for row ids).  For each term, warp 0 stages the term and its
// index in shared memory; a span covering whole blocks of the index's
// cumulative rows starts as C(k1) & ~C(k0) read as 16-byte vectors, and the
// remaining bitmaps (the edges of such a span, a short span, or the tile's
// list of bitmaps holding a 1 bit in it) are OR'ed into a shared-memory
// accumulator: a bitmap with a few words over the tile by one lane (32 such
// bitmaps per warp at once), a longer one and each edge bin's row check by a
// whole warp walking its words 128 at a time (positions by ballot / scan).  The
// term result is AND'ed into the query result; a tile whose AND is empty
// skips the query's remaining terms.
#ifndef WAH_RANGE_CUH
#define WAH_RANGE_CUH
#include "wah_dev.cuh"

namespace wah {

constexpr int RT = 4096;             // groups per tile
constexpr int RTHREADS = 256;
constexpr int RWARPS = RTHREADS / 32;
constexpr int RGPT = RT / RTHREADS;  // groups per thread in the epilogue
constexpr uint32_t RDIRECT = 32;     // spans of at most this many bitmaps skip the tile lists
constexpr int RCHK = 2;              // raw values in flight per lane in an edge-bin row check
// the row-id epilogue stages 16 groups' ids (<= 496) in each warp's RT / RWARPS words of S.tmp
static_assert(RGPT * RTHREADS == RT && 16 * 31 <= RT / RWARPS, "row-id staging");

// per-bitmap metadata of an attached index
struct BitmapMeta {
    uint64_t wstart;  // first m_vec word in the index's word pool
    uint32_t n;       // m_vec words
    uint32_t anb;     // active bits
    uint32_t aval;    // active value
    uint32_t groups;  // groups covered by m_vec (set by k_index_tiles)
};

struct DevIndex {
    const uint32_t* words;     // word pool (the bitmaps' serialized arrays)
    const BitmapMeta* bm;      // nobs entries
    const uint32_t* tiles;     // nobs x (ntiles+1) x {word index, first group}
    const uint32_t* tl_off;    // ntiles+1: tile k's bitmaps are tl_bm[tl_off[k], tl_off[k+1])
    const uint32_t* tl_bm;     // bitmaps holding a 1 bit in each tile, ascending
    const uint32_t* cum;       // cum_k dense rows, gx words apart: row k-1 = OR of bitmaps [0, k*cum_stride)
    uint32_t cum_stride, cum_k, gx, pad2;  // gx: groups incl. the active one, rounded up to 4
    const void* values;        // raw column (nrows), or null
    uint32_t nobs;
    uint32_t vtype;            // 0 uint32, 1 float32, 2 int32
    uint32_t ntiles;
    uint32_t pad;
};

// comparison ops (qExpr::COMPARE): 0 none, 1 <, 2 <=
struct DevTerm {
    uint32_t index;       // into the DevIndex table
    uint32_t h0, h1;      // bitmaps wholly inside: [h0, h1)
    uint32_t flip;        // OR the complement [0,h0) u [h1,nobs) and flip
    // with cumulative rows: [h0, h1) = C(c1) & ~C(c0) | OR of [h0, e0) and
    // [e1, h1), C(k) = row k-1 of DevIndex::cum (C(0) empty); c1 == 0: unused
    uint32_t c0, c1, e0, e1;
    uint32_t ncand;       // edge bitmaps to check row by row (0..2)
    uint32_t cand[2];
    uint32_t lop, rop;    // lo lop x rop hi
    double lo, hi;
};

struct DevQuery {
    uint32_t t0, t1;      // terms [t0, t1)
    uint64_t rid_base;    // capped batches: the query's row-id region
    uint64_t rid_lim;     // capped batches: at most this many row ids (the first ones)
};

struct RangeArgs {
    const DevIndex* idx;
    const DevTerm* terms;
    const DevQuery* queries;
    uint32_t nq;
    uint32_t groups;          // whole groups per column (nrows / 31)
    uint32_t anb;             // rows past the last whole group
    uint32_t ntiles;          // tiles per query
    unsigned long long* counts;  // per query (zeroed by the caller)
    uint32_t* rids;           // row ids, all queries back to back (or null)
    uint64_t rid_cap;
    unsigned long long* rid_start;  // per query: offset of its first row id
    uint32_t* dense;          // dense hit words of query 0 (or null)
    TileRec* recs; LaunchSync* sync; uint32_t nitems;
    DevMeta* status;
    uint32_t tile_major;      // 1: items ordered tile by tile (no look-back)
    // two-pass order (tile by tile, row ids placed without a look-back):
    // pass 1 writes each item's hits to item_cnt, the host scans them into
    // item_off, pass 2 writes the row ids; items are indexed q*ntiles + k
    uint32_t pass;            // 0 one pass, 1 counts, 2 row ids
    unsigned long long* item_cnt;
    const unsigned long long* item_off;
    // 1: every query writes at most rid_lim row ids into its own region at
    // rid_base (query-major order: offsets within the query by a segmented
    // look-back; two-pass order: by the items' scan, pass 2 skipping the
    // items whose ids lie past the limit)
    uint32_t capped;
};

// 64-bit sums segmented at the first item of each query: {sum lo, sum hi,
// -, head}; (f1, s1) + (f2, s2) = (f1 | f2, f2 ? s2 : s1 + s2) is
// associative, so the look-back may combine in any grouping.
struct SegSum64Comb {
    __device__ __forceinline__ uint4 operator()(uint4 a, uint4 b) const {
        if (b.w) return b;
        const uint64_t s = ((uint64_t)a.y << 32 | a.x) + ((uint64_t)b.y << 32 | b.x);
        return make_uint4((uint32_t)s, (uint32_t)(s >> 32), 0u, a.w);
    }
};

struct RangeShared {
    uint32_t acc[RT];
    uint32_t tmp[RT];
    uint64_t scan[RWARPS + 1];
    uint32_t hdr[8];
    unsigned long long base;
    DevTerm term;    // the term being evaluated and its index
    DevIndex index;
};
constexpr uint32_t TERM_WORDS = sizeof(DevTerm) / 4, INDEX_WORDS = sizeof(DevIndex) / 4;
static_assert(sizeof(DevTerm) % 4 == 0 && TERM_WORDS <= 32, "a warp stages a term");
static_assert(sizeof(DevIndex) % 4 == 0 && INDEX_WORDS <= 32, "a warp stages an index");

#ifndef WAH_RANGE_TYPES_ONLY
// Shared-memory place of tile group l in the accumulators: bits 2-4 XOR'ed
// with bits 5-7, so groups 32 apart (a sparse bitmap's set bits often are)
// fall in different banks while every aligned quad of groups stays one
// 16-byte vector in order.  rsw4: the same for quad index l (groups 4l..).
__device__ __forceinline__ uint32_t rsw(uint32_t l) { return l ^ (((l >> 5) & 7u) << 2); }
__device__ __forceinline__ uint32_t rsw4(uint32_t l) { return l ^ ((l >> 3) & 7u); }
__device__ __forceinline__ bool pass_cmp(double v, uint32_t lop, double lo, uint32_t rop, double hi) {
    const bool a = lop == 0 ? true : (lop == 1 ? lo < v : lo <= v);
    const bool b = rop == 0 ? true : (rop == 1 ? v < hi : v <= hi);
    return a && b;
}
// a column value from its 4 raw bytes (0 uint32, 1 float32, 2 int32)
__device__ __forceinline__ double raw_value(uint32_t v, uint32_t vtype) {
    if (vtype == 1) return (double)__uint_as_float(v);
    if (vtype == 2) return (double)(int32_t)v;
    return (double)v;
}
__device__ __forceinline__ double col_value(const void* vals, uint32_t vtype, uint32_t row) {
    if (vtype == 1) return (double)__ldg(reinterpret_cast<const float*>(vals) + row);
    if (vtype == 2) return (double)__ldg(reinterpret_cast<const int32_t*>(vals) + row);
    return (double)__ldg(reinterpret_cast<const uint32_t*>(vals) + row);
}

// One warp ORs bitmap b's words for the tile [g0, g1) into S.tmp (the
// virtual group G holds the active bits).
__device__ __forceinline__ void warp_or_bitmap(RangeShared& S, const DevIndex& I, uint32_t b, uint32_t k,
                                               uint32_t g0, uint32_t g1, uint32_t G, uint32_t anb) {
    const uint32_t lane = threadIdx.x & 31u;
    const BitmapMeta m = I.bm[b];
    const uint32_t* tix = I.tiles + ((size_t)b * (I.ntiles + 1) + k) * 2;
    const uint32_t i0 = __ldg(tix), s0 = __ldg(tix + 1);
    const uint32_t in1 = __ldg(tix + 2), sn1 = __ldg(tix + 3);
    const uint32_t i1 = min(sn1 < g1 ? in1 + 1u : in1, m.n);  // words covering [g0, min(g1, G))
    const uint32_t* w = I.words + m.wstart;
    uint32_t carry = s0;
    // four 32-word chunks are loaded before any is placed, so one memory
    // latency covers 128 words
    for (uint32_t base0 = i0; base0 < i1; base0 += 128) {
        uint32_t wv[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t i = base0 + 32u * j + lane;
            wv[j] = i < i1 ? __ldg(w + i) : 0u;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t base = base0 + 32u * j;
            if (base >= i1) break;
            const uint32_t i = base + lane;
            const bool in = i < i1;
            const uint32_t wd = wv[j];
            const uint32_t c = in ? wgroups(wd) : 0u;
            uint32_t p;
            const uint32_t fm = __ballot_sync(0xffffffffu, in && is_fill(wd));
            if (fm == 0) {
                p = carry + lane;
                carry += __popc(__ballot_sync(0xffffffffu, in));
            } else {
                uint32_t x = c;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) { uint32_t t = __shfl_up_sync(0xffffffffu, x, d); if (lane >= (uint32_t)d) x += t; }
                p = carry + x - c;
                carry += __shfl_sync(0xffffffffu, x, 31);
            }
            if (in && wd != 0u && !(is_fill(wd) && wd < HEADER1)) {
                const uint32_t a = max(p, g0), e = min(p + c, g1);
                const uint32_t pat = wpattern(wd);
                for (uint32_t g = a; g < e; ++g) {
                    if (pat == ALLONES) S.tmp[rsw(g - g0)] = ALLONES;
                    else atomicOr(&S.tmp[rsw(g - g0)], pat);
                }
            }
        }
    }
    // the bitmap's active bits form the group after its whole words (the
    // virtual group G when the bitmap covers every row)
    const uint32_t Gb = m.groups;
    if (lane == 0 && m.anb > 0 && Gb >= g0 && Gb < g1) {
        const uint32_t pat = (m.aval & ((1u << m.anb) - 1u)) << (31u - m.anb);
        if (pat) atomicOr(&S.tmp[rsw(Gb - g0)], pat);
    }
}

// An edge bin's row check by one warp: the bin's rows in the tile [g0, g1)
// whose raw values pass the term's comparison are OR'ed into S.tmp.  The
// bin's words are taken 128 at a time; the first set row of every literal
// of the batch has its raw value loaded before any is compared (one memory
// latency per batch for the usual one-row literals of a sparse bin), the
// other rows of a literal and the rows of 1-fills RCHK at a time after.
__device__ __forceinline__ void warp_check_bitmap(RangeShared& S, const DevIndex& I, uint32_t b, uint32_t k,
                                                  uint32_t g0, uint32_t g1, const DevTerm& T) {
    const uint32_t lane = threadIdx.x & 31u;
    const BitmapMeta m = I.bm[b];
    const uint32_t* tix = I.tiles + ((size_t)b * (I.ntiles + 1) + k) * 2;
    const uint32_t i0 = __ldg(tix), s0 = __ldg(tix + 1);
    const uint32_t in1 = __ldg(tix + 2), sn1 = __ldg(tix + 3);
    const uint32_t i1 = min(sn1 < g1 ? in1 + 1u : in1, m.n);
    const uint32_t* w = I.words + m.wstart;
    const uint32_t* raw = reinterpret_cast<const uint32_t*>(I.values);  // every column type is 4 bytes a row
    uint32_t carry = s0;
    for (uint32_t base0 = i0; base0 < i1; base0 += 128) {
        uint32_t wv[4], pv[4], cv[4], v0[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t i = base0 + 32u * j + lane;
            wv[j] = i < i1 ? __ldg(w + i) : 0u;
        }
        // each row's first group per word
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t base = base0 + 32u * j;
            pv[j] = 0; cv[j] = 0;
            if (base < i1) {
                const bool in = base + lane < i1;
                const uint32_t wd = wv[j];
                const uint32_t c = in ? wgroups(wd) : 0u;
                if (__ballot_sync(0xffffffffu, in && is_fill(wd)) == 0u) {
                    pv[j] = carry + lane;
                    carry += __popc(__ballot_sync(0xffffffffu, in));
                } else {
                    uint32_t x = c;
#pragma unroll
                    for (int d = 1; d < 32; d <<= 1) { uint32_t t = __shfl_up_sync(0xffffffffu, x, d); if (lane >= (uint32_t)d) x += t; }
                    pv[j] = carry + x - c;
                    carry += __shfl_sync(0xffffffffu, x, 31);
                }
                cv[j] = c;
            }
        }
        // the first set row of every literal in the tile, all loads in flight
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t wd = wv[j];
            const bool lit = cv[j] == 1u && !is_fill(wd) && wd != 0u && pv[j] >= g0 && pv[j] < g1;
            v0[j] = lit ? __ldg(raw + pv[j] * 31u + (__clz(wd) - 1u)) : 0u;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t wd = wv[j], c = cv[j], p = pv[j];
            if (c == 0u || wd == 0u || (is_fill(wd) && wd < HEADER1)) continue;
            const bool lit = c == 1u && !is_fill(wd);
            const uint32_t a = max(p, g0), e = min(p + c, g1);
            for (uint32_t g = a; g < e; ++g) {
                uint32_t bits = wpattern(wd), set = 0;
                if (lit) {
                    const uint32_t hb = 31u - __clz(bits);
                    if (pass_cmp(raw_value(v0[j], I.vtype), T.lop, T.lo, T.rop, T.hi)) set |= 1u << hb;
                    bits &= ~(1u << hb);
                }
                while (bits) {
                    uint32_t hb[RCHK], v[RCHK];
#pragma unroll
                    for (int q = 0; q < RCHK; ++q) {
                        hb[q] = bits ? 31u - __clz(bits) : 32u;
                        if (bits) bits &= ~(1u << hb[q]);
                    }
#pragma unroll
                    for (int q = 0; q < RCHK; ++q)
                        v[q] = hb[q] < 32u ? __ldg(raw + g * 31u + (30u - hb[q])) : 0u;
#pragma unroll
                    for (int q = 0; q < RCHK; ++q)
                        if (hb[q] < 32u && pass_cmp(raw_value(v[q], I.vtype), T.lop, T.lo, T.rop, T.hi))
                            set |= 1u << hb[q];
                }
                if (set) atomicOr(&S.tmp[rsw(g - g0)], set);
            }
        }
    }
    // the bitmap's active bits form the group after its whole words
    const uint32_t Gb = m.groups;
    if (lane == 0 && m.anb > 0 && Gb >= g0 && Gb < g1) {
        uint32_t bits = (m.aval & ((1u << m.anb) - 1u)) << (31u - m.anb), set = 0;
        while (bits) {
            const uint32_t hb = 31u - __clz(bits);
            const uint32_t row = Gb * 31u + (30u - hb);
            if (pass_cmp(col_value(I.values, I.vtype, row), T.lop, T.lo, T.rop, T.hi)) set |= 1u << hb;
            bits &= ~(1u << hb);
        }
        if (set) atomicOr(&S.tmp[rsw(Gb - g0)], set);
    }
}

// Bitmaps with at most LSHORT words over the tile are OR'ed by one lane
// each; longer ones (or one holding a 1-fill longer than LFILL groups of
// the tile) by the whole warp.
constexpr uint32_t LSHORT = 4, LFILL = 8;

// One lane per bitmap: lane l ORs bitmap b (valid when `have`) into S.tmp
// when its words over the tile are few: its metadata, tile-index entries
// and words are loaded by all lanes at once, so 32 sparse bitmaps cost
// three memory round trips instead of three each.  The bitmaps left over
// are OR'ed by the whole warp, one after the other.
__device__ __forceinline__ void lanes_or_bitmaps(RangeShared& S, const DevIndex& I, bool have, uint32_t b,
                                                 uint32_t k, uint32_t g0, uint32_t g1, uint32_t G, uint32_t anb) {
    uint32_t i0 = 0, i1 = 0, s0 = 0, gb = 0, banb = 0, aval = 0;
    uint64_t wstart = 0;
    if (have) {
        const BitmapMeta* m = I.bm + b;
        const uint32_t* tix = I.tiles + ((size_t)b * (I.ntiles + 1) + k) * 2;
        wstart = __ldg(&m->wstart);
        const uint32_t n = __ldg(&m->n);
        banb = __ldg(&m->anb); aval = __ldg(&m->aval); gb = __ldg(&m->groups);
        i0 = __ldg(tix); s0 = __ldg(tix + 1);
        const uint32_t in1 = __ldg(tix + 2), sn1 = __ldg(tix + 3);
        i1 = min(sn1 < g1 ? in1 + 1u : in1, n);
    }
    bool lng = have && i1 > i0 + LSHORT;
    if (have && !lng) {
        const uint32_t* w = I.words + wstart;
        uint32_t wv[LSHORT];
#pragma unroll
        for (uint32_t j = 0; j < LSHORT; ++j) wv[j] = i0 + j < i1 ? __ldg(w + i0 + j) : 0u;
        uint32_t p = s0;
#pragma unroll
        for (uint32_t j = 0; j < LSHORT; ++j) {
            if (i0 + j >= i1) break;
            const uint32_t wd = wv[j];
            const uint32_t c = wgroups(wd);
            if (!is_fill(wd)) {
                if (wd && p >= g0 && p < g1) atomicOr(&S.tmp[rsw(p - g0)], wd);
            } else if (wd >= HEADER1) {
                const uint32_t a = max(p, g0), e = min(p + c, g1);
                if (e > a + LFILL) lng = true;  // the warp paints it (OR is idempotent)
                else for (uint32_t g = a; g < e; ++g) S.tmp[rsw(g - g0)] = ALLONES;
            }
            p += c;
        }
        // the active bits form the group after the whole words
        if (!lng && banb > 0 && gb >= g0 && gb < g1) {
            const uint32_t pat = (aval & ((1u << banb) - 1u)) << (31u - banb);
            if (pat) atomicOr(&S.tmp[rsw(gb - g0)], pat);
        }
    }
    uint32_t lm = __ballot_sync(0xffffffffu, lng);
    while (lm) {
        const uint32_t src = __ffs(lm) - 1u;
        lm &= lm - 1u;
        warp_or_bitmap(S, I, __shfl_sync(0xffffffffu, b, src), k, g0, g1, G, anb);
    }
}

// Lower bound of v in the ascending list a[0, n) by a group of 16 lanes
// (lanes [gbase, gbase+16) of a full warp; every lane of the warp calls it):
// each round the 16 lanes probe evenly spaced entries of [lo, hi) and the
// count of entries below v narrows the span 16-fold.
__device__ __forceinline__ uint32_t group16_lower_bound(const uint32_t* __restrict__ a, uint32_t n, uint32_t v,
                                                         uint32_t gbase, uint32_t gl) {
    uint32_t lo = 0, hi = n;  // the answer lies in [lo, hi]
    while (__any_sync(0xffffffffu, lo < hi)) {
        uint32_t p = lo;
        bool less = false;
        if (lo < hi) {
            p = lo + (uint32_t)(((uint64_t)(hi - lo) * gl) >> 4);  // < hi
            less = __ldg(a + p) < v;
        }
        const uint32_t c = __popc((__ballot_sync(0xffffffffu, less) >> gbase) & 0xFFFFu);
        const uint32_t plast = __shfl_sync(0xffffffffu, p, gbase + (c ? c - 1u : 0u));
        const uint32_t pnext = __shfl_sync(0xffffffffu, p, gbase + (c < 16u ? c : 0u));
        if (lo < hi) {
            if (c == 0) hi = lo;  // a[lo] >= v
            else { lo = plast + 1u; if (c < 16u) hi = pnext; }
        }
    }
    return lo;
}

// Persistent: every CTA claims items until none is left.
__global__ void __launch_bounds__(RTHREADS, 6) k_range(RangeArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    RangeShared& S = *reinterpret_cast<RangeShared*>(smem_raw);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    if (tid == 0) S.hdr[1] = ld_cg(&A.sync->epoch);
    const uint32_t G = A.groups, anb = A.anb;
    const uint32_t GX = G + (anb > 0 ? 1u : 0u);  // groups incl. the active one
    const uint32_t lastmask = anb > 0 ? (((1u << anb) - 1u) << (31u - anb)) : ALLONES;
    // tile-major items are claimed one item ahead, so the ticket's round
    // trip overlaps the current item (not with the look-back: an item held
    // back behind a long one would stall every later item waiting on it)
    const bool ahead = A.tile_major != 0u;
    uint32_t next = 0;
    if (tid == 0 && ahead) next = claim_tile(A.sync);
    while (true) {
        if (tid == 0) {
            if (ahead) {
                S.hdr[0] = next;
                if (next < A.nitems) next = claim_tile(A.sync);
            } else {
                S.hdr[0] = claim_tile(A.sync);
            }
        }
        __syncthreads();
        const uint32_t item = S.hdr[0], epoch = S.hdr[1];
        if (item >= A.nitems) break;
        // query-major items keep a query's row ids contiguous (look-back in
        // claim order); tile-major items let the queries of one batch share
        // each tile's bitmap words in L2
        const uint32_t q = A.tile_major ? item % A.nq : item / A.ntiles;
        const uint32_t k = A.tile_major ? item / A.nq : item % A.ntiles;
        const uint32_t g0 = k * (uint32_t)RT, g1 = min(g0 + (uint32_t)RT, GX);
        const uint32_t ng = g1 > g0 ? g1 - g0 : 0u;
        const uint32_t qi = q * A.ntiles + k;  // the item's place in query-major order
        const DevQuery Q = A.queries[q];
        if (A.pass == 2u) {
            // row ids of the two-pass order: items without hits are done, and
            // so (capped) are items whose ids all lie past the query's limit
            // (offsets within the query: the scan runs in query-major order)
            if (tid == 0 && k == 0) A.rid_start[q] = A.capped ? Q.rid_base : A.item_off[qi];
            const bool past = A.capped && A.item_off[qi] - A.item_off[q * A.ntiles] >= Q.rid_lim;
            if (A.item_cnt[qi] == 0ull || past) { __syncthreads(); continue; }
        }

        for (uint32_t l = tid; l < RT; l += RTHREADS) S.acc[l] = ALLONES;
        for (uint32_t t = Q.t0; t < Q.t1; ++t) {
            // the term and its index, staged in shared memory by warp 0
            if (warp == 0) {
                const uint32_t v = lane < TERM_WORDS ? __ldg(reinterpret_cast<const uint32_t*>(A.terms + t) + lane) : 0u;
                const uint32_t ix = __shfl_sync(0xffffffffu, v, 0);  // DevTerm::index
                if (lane < TERM_WORDS) reinterpret_cast<uint32_t*>(&S.term)[lane] = v;
                if (lane < INDEX_WORDS)
                    reinterpret_cast<uint32_t*>(&S.index)[lane] = __ldg(reinterpret_cast<const uint32_t*>(A.idx + ix) + lane);
            }
            __syncthreads();
            const DevTerm& T = S.term;
            const DevIndex& I = S.index;
            uint4* t4 = reinterpret_cast<uint4*>(S.tmp);
            if (T.c1) {
                // the wholly-inside span from two cumulative rows
                // (16-byte slices: g0 is a multiple of RT and the rows'
                // padding past the last group is zero)
                const uint4* hi = reinterpret_cast<const uint4*>(I.cum + (size_t)(T.c1 - 1u) * I.gx + g0);
                const uint4* lo = reinterpret_cast<const uint4*>(T.c0 ? I.cum + (size_t)(T.c0 - 1u) * I.gx + g0 : I.cum);
                const uint32_t n4 = (ng + 3u) >> 2;
                const bool two = T.c0 != 0u;
#pragma unroll
                for (uint32_t l = tid; l < RT / 4; l += RTHREADS) {
                    uint4 v = make_uint4(0u, 0u, 0u, 0u);
                    if (l < n4) {
                        const uint4 a = __ldg(hi + l);
                        const uint4 b = two ? __ldg(lo + l) : v;
                        v = make_uint4(a.x & ~b.x, a.y & ~b.y, a.z & ~b.z, a.w & ~b.w);
                    }
                    t4[rsw4(l)] = v;
                }
            } else {
#pragma unroll
                for (uint32_t l = tid; l < RT / 4; l += RTHREADS) t4[l] = make_uint4(0u, 0u, 0u, 0u);
            }
            // the bitmaps to OR, as two ranges: with cumulative rows the
            // edge spans [h0, e0) and [e1, h1), else the span [h0, h1) or
            // the complement [0, h0) and [h1, nobs).  Ranges of at most
            // RDIRECT bitmaps in all are walked directly (one that misses
            // the tile costs its tile-index lookup); wider ones take the
            // entries of the tile's list of bitmaps holding a 1 bit in it
            // that fall in the ranges (lower bounds by 16-lane searches)
            const bool flip = T.flip != 0u;
            uint32_t ra0, ra1, rb0, rb1;  // bitmap ids [ra0, ra1) u [rb0, rb1)
            if (T.c1) { ra0 = T.h0; ra1 = T.e0; rb0 = T.e1; rb1 = T.h1; }
            else if (flip) { ra0 = 0u; ra1 = T.h0; rb0 = T.h1; rb1 = I.nobs; }
            else { ra0 = T.h0; ra1 = T.h1; rb0 = rb1 = T.h1; }
            const bool direct = !flip && (ra1 - ra0) + (rb1 - rb0) <= RDIRECT;
            if (!direct && warp < 2) {
                const uint32_t o0 = __ldg(I.tl_off + k), o1 = __ldg(I.tl_off + k + 1);
                const uint32_t gbase = lane & 16u;
                const uint32_t v = warp == 0 ? (gbase ? ra1 : ra0) : (gbase ? rb1 : rb0);
                const uint32_t r = group16_lower_bound(I.tl_bm + o0, o1 - o0, v, gbase, lane & 15u);
                if ((lane & 15u) == 0) S.hdr[2 + 2 * warp + (gbase >> 4)] = o0 + r;
            }
            __syncthreads();
            // one job list per term: the edge bitmaps' row checks first
            // (the longest jobs), then the bitmaps to OR; a complement is
            // flipped before the checked rows join it
            const uint32_t nc = flip ? 0u : T.ncand;
            uint32_t sa = ra0, sb = rb0, na = ra1 - ra0, nb = rb1 - rb0;  // the two ranges' starts and sizes
            if (!direct) {  // as entries of the tile list
                sa = S.hdr[2]; na = S.hdr[3] - sa;
                sb = S.hdr[4]; nb = S.hdr[5] - sb;
            }
            const uint32_t nsel = na + nb;
            // row checks (the longest jobs) one per warp from warp 0; the
            // bitmaps to OR in batches of up to 32 per warp (one per lane),
            // spread over the warps from the one after the checks, so the
            // warps holding a check get an OR batch last
            for (uint32_t c = warp; c < nc; c += RWARPS) warp_check_bitmap(S, I, T.cand[c], k, g0, g1, T);
            const uint32_t nfree = RWARPS - min(nc, (uint32_t)RWARPS - 1u);  // warps without a check
            const uint32_t per = min(32u, (nsel + nfree - 1) / nfree);
            const uint32_t wr = (warp + RWARPS - nc % RWARPS) % RWARPS;      // the warp's place in the OR order
            for (uint32_t j0 = wr * per; j0 < nsel; j0 += RWARPS * per) {
                const uint32_t jj = j0 + lane;
                const bool have = lane < per && jj < nsel;
                uint32_t b = 0;
                if (have) {
                    const uint32_t e = jj < na ? sa + jj : sb + (jj - na);
                    b = direct ? e : __ldg(I.tl_bm + e);
                }
                lanes_or_bitmaps(S, I, have, b, k, g0, g1, G, anb);
            }
            if (flip) {
                __syncthreads();
                for (uint32_t l = tid; l < ng; l += RTHREADS) {
                    const uint32_t msk = (g0 + l == G && anb > 0) ? lastmask : ALLONES;
                    S.tmp[rsw(l)] ^= msk;
                }
                __syncthreads();
                // edge bitmaps: rows checked against the raw values
                for (uint32_t c = warp; c < T.ncand; c += RWARPS)
                    warp_check_bitmap(S, I, T.cand[c], k, g0, g1, T);
            }
            __syncthreads();
            uint32_t any = 0;
            for (uint32_t l = tid; l < RT; l += RTHREADS) { const uint32_t v = S.acc[l] & S.tmp[l]; S.acc[l] = v; any |= v; }
            // an empty AND ends the query's work on this tile
            if (!__syncthreads_or(any != 0u)) break;
        }
        // ---- counts and row ids
        const uint32_t l0 = tid * RGPT;
        uint32_t cnt = 0;
#pragma unroll
        for (int j = 0; j < RGPT; ++j) {
            const uint32_t l = l0 + j;
            if (l < ng) {
                uint32_t v = S.acc[rsw(l)];
                if (g0 + l == G && anb > 0) v &= lastmask;
                S.acc[rsw(l)] = v;
                cnt += __popc(v);
            } else if (l < RT) {
                S.acc[rsw(l)] = 0u;
            }
        }
        if (A.tile_major && A.pass == 1u) {
            uint64_t total;
            block_exscan64(cnt, S.scan, total);
            if (tid == 0) {
                A.item_cnt[qi] = total;
                if (total) atomicAdd(&A.counts[q], (unsigned long long)total);
            }
            __syncthreads();
            continue;
        }
        if (A.tile_major && A.pass == 0u) {
            cnt = __reduce_add_sync(0xffffffffu, cnt);
            if (lane == 0 && cnt) atomicAdd(&A.counts[q], (unsigned long long)cnt);
            __syncthreads();
            continue;
        }
        uint64_t total;
        const uint64_t ex = block_exscan64(cnt, S.scan, total);
        if (A.pass == 2u) {
            if (tid == 0) S.base = A.capped ? A.item_off[qi] - A.item_off[q * A.ntiles] : A.item_off[qi];
        } else if (warp == 0 && A.capped) {
            // the row ids before this tile within its own query
            const uint4 mine = make_uint4((uint32_t)total, (uint32_t)(total >> 32), 0u, k == 0 ? 1u : 0u);
            uint4 pre = make_uint4(0u, 0u, 0u, 0u);
            bool ok = true;
            if (item == 0) {
                if (lane == 0) publish(&A.recs[0], epoch, REC_INCL, mine);
            } else {
                if (lane == 0) publish(&A.recs[item], epoch, REC_AGG, mine);
                pre = warp_lookback(A.recs, item, epoch, make_uint4(0u, 0u, 0u, 0u), SegSum64Comb(), &ok);
                if (lane == 0) publish(&A.recs[item], epoch, REC_INCL, SegSum64Comb()(pre, mine));
            }
            if (lane == 0) {
                if (!ok) atomicExch(&A.status->status, DEV_ERR_TIMEOUT);
                S.base = k == 0 ? 0ull : ((uint64_t)pre.y << 32 | pre.x);
                if (total) atomicAdd(&A.counts[q], (unsigned long long)total);
                if (k == 0) A.rid_start[q] = Q.rid_base;
            }
        } else if (warp == 0) {
            uint64_t prefix; uint32_t pa, pb;
            const bool ok = lookback64(A.recs, item, epoch, total, 0, 0, prefix, pa, pb);
            if (lane == 0) {
                if (!ok) atomicExch(&A.status->status, DEV_ERR_TIMEOUT);
                S.base = prefix;
                if (total) atomicAdd(&A.counts[q], (unsigned long long)total);
                if (k == 0) A.rid_start[q] = prefix;
            }
        }
        __syncthreads();
        if (A.rids) {
            // capped: offsets are within the query; ids past its limit are
            // dropped and the rest land in its region
            const uint64_t lim = A.capped ? Q.rid_lim : A.rid_cap;
            const uint64_t rbase0 = A.capped ? Q.rid_base : 0ull;
            // each warp owns RGPT * 32 consecutive groups (its threads' in
            // the count above) and writes their ids 16 groups at a time:
            // lanes 0-15 expand a group each into the warp's part of S.tmp
            // (free once the terms are done), then the warp stores the run
            // of ids with consecutive lanes on consecutive slots
            constexpr uint32_t WG = RGPT * 32;      // groups per warp
            uint32_t* st = S.tmp + warp * WG;       // <= 16 * 31 ids per round
            uint64_t off = S.base + __shfl_sync(0xffffffffu, ex, 0);
            for (uint32_t r = 0; r < WG / 16u && off < lim; ++r) {
                const uint32_t l = warp * WG + r * 16u + (lane & 15u);
                uint32_t bits = (lane < 16u && l < ng) ? S.acc[rsw(l)] : 0u;
                const uint32_t c = __popc(bits);
                uint32_t x = c;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const uint32_t u = __shfl_up_sync(0xffffffffu, x, d);
                    if (lane >= (uint32_t)d) x += u;
                }
                const uint32_t rt = __shfl_sync(0xffffffffu, x, 31);
                if (rt == 0u) continue;
                uint32_t p = x - c;
                const uint32_t rbase = (g0 + l) * 31u;
                while (bits) {
                    const uint32_t hb = 31u - __clz(bits);
                    st[p++] = rbase + (30u - hb);
                    bits &= ~(1u << hb);
                }
                __syncwarp();
                for (uint32_t i = lane; i < rt; i += 32u) {
                    const uint64_t o = off + i;
                    if (o < lim && rbase0 + o < A.rid_cap) A.rids[rbase0 + o] = st[i];
                }
                __syncwarp();
                off += rt;
            }
        }
        if (A.dense && q == 0) {
            for (uint32_t l = tid; l < ng; l += RTHREADS) A.dense[g0 + l] = S.acc[rsw(l)];
        }
        __syncthreads();
    }
    if (tid == 0) finish_tile(A.sync, gridDim.x);
}

// Per-bitmap group-tile index of an attached index: one warp per bitmap
// walks its words, records the word covering every multiple of RT, checks
// the words and counts groups and ones.
__global__ void k_index_tiles(const uint32_t* __restrict__ words, BitmapMeta* __restrict__ bm,
                              uint32_t nobs, uint32_t ntiles, uint32_t nrows, uint32_t* __restrict__ tiles,
                              uint32_t* __restrict__ bones, DevMeta* status) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (b >= nobs) return;
    const BitmapMeta m = bm[b];
    const uint32_t* w = words + m.wstart;
    uint32_t* tix = tiles + (size_t)b * (ntiles + 1) * 2;
    uint32_t carry = 0, ones = 0, bad = 0;
    for (uint32_t base = 0; base < m.n; base += 32) {
        const uint32_t i = base + lane;
        const bool in = i < m.n;
        const uint32_t wd = in ? __ldg(w + i) : 0u;
        const uint32_t c = in ? wgroups(wd) : 0u;
        if (in && is_fill(wd) && c == 0) bad = 1;
        if (in) ones += wd > ALLONES ? (wd >= HEADER1 ? c * 31u : 0u) : __popc(wd);
        uint32_t x = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) { uint32_t t = __shfl_up_sync(0xffffffffu, x, d); if (lane >= (uint32_t)d) x += t; }
        const uint32_t p = carry + x - c;  // first group of word i
        // word i covers boundaries t*RT in [p, p+c)
        if (in && c > 0) {
            uint32_t t = (p + RT - 1) / RT;
            for (; (uint64_t)t * RT < (uint64_t)p + c && t <= ntiles; ++t) {
                tix[2 * t] = i;
                tix[2 * t + 1] = p;
            }
        }
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
    // boundaries at or past the end of the words
    for (uint32_t t = lane; t <= ntiles; t += 32) {
        if ((uint64_t)t * RT >= carry) { tix[2 * t] = m.n; tix[2 * t + 1] = carry; }
    }
    ones = __reduce_add_sync(0xffffffffu, ones);
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (lane == 0) {
        bm[b].groups = carry;
        bones[b] = ones + __popc(m.anb ? (m.aval & ((1u << m.anb) - 1u)) : 0u);
        if (bad) atomicExch(&status->status, DEV_ERR_FORMAT);
        else if ((uint64_t)carry * 31u + m.anb > nrows) atomicExch(&status->status, DEV_ERR_RANGE);
    }
}

// Tiles of RT groups in which bitmap b holds a 1 bit, each once and in
// order (one warp per bitmap).  Pass 0 counts them into cnt[b]; pass 1
// writes (tile, bitmap) pairs from pos[b].
__global__ void k_tile_touch(const uint32_t* __restrict__ words, const BitmapMeta* __restrict__ bm,
                             uint32_t nobs, int pass, uint32_t* __restrict__ cnt,
                             const uint32_t* __restrict__ pos, uint32_t* __restrict__ out_tile,
                             uint32_t* __restrict__ out_bm) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (b >= nobs) return;
    const BitmapMeta m = bm[b];
    const uint32_t* w = words + m.wstart;
    uint32_t carry = 0;        // first group of the next word
    int64_t last = -1;         // last tile emitted
    uint32_t n = 0;            // tiles emitted so far
    const uint32_t o = pass ? pos[b] : 0u;
    for (uint32_t base = 0; base < m.n; base += 32) {
        const uint32_t i = base + lane;
        const bool in = i < m.n;
        const uint32_t wd = in ? __ldg(w + i) : 0u;
        const uint32_t c = in ? wgroups(wd) : 0u;
        uint32_t x = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) { uint32_t t = __shfl_up_sync(0xffffffffu, x, d); if (lane >= (uint32_t)d) x += t; }
        const uint32_t p = carry + x - c;
        const bool bits = in && c > 0 && (wd >= HEADER1 || (wd <= ALLONES && wd != 0u));
        // tiles [k0, k1] of this word, minus those an earlier word emitted
        int64_t k0 = bits ? (int64_t)(p / RT) : 0, k1 = bits ? (int64_t)((p + c - 1u) / RT) : -1;
        int64_t prev = bits ? k1 : -1;  // highest tile of lanes up to this one
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int64_t t = __shfl_up_sync(0xffffffffu, prev, d);
            if (lane >= (uint32_t)d) prev = max(prev, t);
        }
        int64_t before = __shfl_up_sync(0xffffffffu, prev, 1);
        if (lane == 0) before = -1;
        before = max(before, last);
        if (bits) k0 = max(k0, before + 1);
        const uint32_t mine = (bits && k1 >= k0) ? (uint32_t)(k1 - k0 + 1) : 0u;
        uint32_t ex = mine;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) { uint32_t t = __shfl_up_sync(0xffffffffu, ex, d); if (lane >= (uint32_t)d) ex += t; }
        if (pass && mine) {
            uint32_t q = o + n + ex - mine;
            for (int64_t k = k0; k <= k1; ++k, ++q) { out_tile[q] = (uint32_t)k; out_bm[q] = b; }
        }
        n += __shfl_sync(0xffffffffu, ex, 31);
        last = max(last, __shfl_sync(0xffffffffu, prev, 31));
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
    // the active bits form the group after the whole words
    if (lane == 0) {
        if (m.anb > 0 && (m.aval & ((1u << m.anb) - 1u)) != 0u) {
            const int64_t k = carry / RT;
            if (k > last) {
                if (pass) { out_tile[o + n] = (uint32_t)k; out_bm[o + n] = b; }
                ++n;
            }
        }
        if (!pass) cnt[b] = n;
    }
}

// CSR offsets of the tile-sorted pairs: off[k] = first pair of tile k.
__global__ void k_tile_offsets(const uint32_t* __restrict__ tile, uint32_t npairs, uint32_t ntiles,
                               uint32_t* __restrict__ off) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e > npairs) return;
    const uint32_t k = e < npairs ? tile[e] : ntiles;
    const uint32_t kp = e > 0 ? tile[e - 1] : 0u;
    const uint32_t from = e > 0 ? kp + 1u : 0u;
    for (uint32_t t = from; t <= k && t <= ntiles; ++t) off[t] = e;  // tiles kp+1 .. k start here
}

// Block ORs for the cumulative rows: bitmap b (< k*stride) is OR'ed into
// row b / stride (one warp per bitmap; fills of more than 32 groups are
// written by the whole warp).
__global__ void k_cum_blocks(const uint32_t* __restrict__ words, const BitmapMeta* __restrict__ bm,
                             uint32_t nb, uint32_t stride, uint32_t gx, uint32_t* __restrict__ rows) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (b >= nb) return;
    const BitmapMeta m = bm[b];
    const uint32_t* w = words + m.wstart;
    uint32_t* row = rows + (size_t)(b / stride) * gx;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < m.n; base += 32) {
        const uint32_t i = base + lane;
        const bool in = i < m.n;
        const uint32_t wd = in ? __ldg(w + i) : 0u;
        const uint32_t c = in ? wgroups(wd) : 0u;
        uint32_t x = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) { uint32_t t = __shfl_up_sync(0xffffffffu, x, d); if (lane >= (uint32_t)d) x += t; }
        const uint32_t p = carry + x - c;
        if (in && wd <= ALLONES && wd != 0u) atomicOr(row + p, wd);
        else if (in && wd >= HEADER1 && c <= 32u) for (uint32_t g = 0; g < c; ++g) row[p + g] = ALLONES;
        uint32_t f = __ballot_sync(0xffffffffu, in && wd >= HEADER1 && c > 32u);
        while (f) {
            const uint32_t src = __ffs(f) - 1u;
            f &= f - 1u;
            const uint32_t fp = __shfl_sync(0xffffffffu, p, src), fc = __shfl_sync(0xffffffffu, c, src);
            for (uint32_t g = lane; g < fc; g += 32u) row[fp + g] = ALLONES;
        }
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0 && m.anb > 0) {
        const uint32_t pat = (m.aval & ((1u << m.anb) - 1u)) << (31u - m.anb);
        if (pat) atomicOr(row + m.groups, pat);
    }
}

// Prefix OR down the rows: row k |= row k-1 for k = 1..nrows-1 (a thread per
// word column; neighbouring threads read neighbouring words of each row).
__global__ void k_cum_prefix(uint32_t* __restrict__ rows, uint32_t nrows, uint32_t gx) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= gx) return;
    uint32_t acc = 0;
    for (uint32_t k = 0; k < nrows; ++k) {
        uint32_t* p = rows + (size_t)k * gx + i;
        acc |= *p;
        *p = acc;
    }
}

#endif  // WAH_RANGE_TYPES_ONLY

}  // namespace wah
#endif
