// Single-pass warp-tile engine for the operators whose result compress()
// leaves canonical (the reference's _d2 / _d1 / _c1 / _c0 paths and the
// all-literal loops, src/bitvector.cpp:2545-2830, 2981-3278, 3354-3619,
// 3748-4079): one launch, operands read once, result words written once.
//
// k_gone<OP>: one warp per tile of GT = 512 groups, warps claiming tiles in
// launch order; no shared-memory staging of words.
//  1. paint: the warp reads each operand's words over its tile as 32-word
//     rows (eight rows of both operands in flight per lane), finds each
//     word's first group (a row of literals by lane number, a row holding
//     fills by a warp scan of the lengths) and writes the word's 31-bit
//     pattern to every group of the tile it covers, in the operand's
//     group-space array in shared memory (a fill of up to GSHORT groups by
//     its own lane, a longer one by the whole warp);
//  2. groups: lane l takes groups 128 j + 4 l .. + 3 of chunk j (one
//     16-byte shared-memory read per operand), R = a OP b, the run heads (a
//     mixed group, a class change, or group 0) and the popcount;
//  3. the tile's {heads, last head, ones} goes to a decoupled look-back over
//     16-byte records, which gives the heads and the last head of all
//     earlier tiles;
//  4. write: per chunk with heads, R is recomputed from shared memory; a
//     lane's first output index is the heads of the lanes before it (three
//     ballots of its 0..4 head count) and the head before its first one is
//     the last head of the nearest lower lane holding one (a ballot and a
//     shuffle).  A mixed head's lane writes its literal; the word of a
//     uniform run (its length is known only at the next head) is written by
//     the lane of the next head, in this tile or a later one (heads packed
//     as (group + 1) << 2 | class, so a later head compares larger); the
//     last tile writes the final run and the metadata.
// No warp waits for another except in the bounded look-back: one that gives
// up sets DEV_ERR_TIMEOUT and writes no words.
#ifndef WAH_GONE_CUH
#define WAH_GONE_CUH
#include "wah_gop.cuh"
#include "wah_fuse.cuh"

namespace wah {

constexpr int GROWS = 8;          // 32-word rows of each operand in flight per lane
constexpr uint32_t GSHORT = 8;    // fills up to this many groups of the tile are painted by their own lane

// per warp: both operands' patterns over its tile (group g0 + i at index i)
struct GoneWarp {
    uint32_t pat[2][GT];
};

// Rows [base, base + 32 GROWS) of an operand's words over the tile (w
// points at the tile's first word, nw words; zeros past them).
__device__ __forceinline__ void gone_load(const uint32_t* __restrict__ w, uint32_t nw, uint32_t base,
                                          uint32_t (&v)[GROWS]) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (int j = 0; j < GROWS; ++j) {
        const uint32_t i = base + 32u * j + lane;
        v[j] = i < nw ? __ldg(w + i) : 0u;
    }
}

// Paints the rows loaded by gone_load: the row's words start at group
// `carry` (advanced past them), each word's pattern goes to every group of
// [g0, g1) it covers.
__device__ __forceinline__ void gone_paint(const uint32_t (&v)[GROWS], uint32_t nw, uint32_t base, uint32_t& carry,
                                           uint32_t g0, uint32_t g1, uint32_t* __restrict__ P) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (int j = 0; j < GROWS; ++j) {
        const uint32_t b = base + 32u * j;
        if (b >= nw) break;
        const bool in = b + lane < nw;
        const uint32_t wd = v[j];
        uint32_t p, c = 1u;
        if (__ballot_sync(0xffffffffu, in && is_fill(wd)) == 0u) {
            p = carry + lane;  // one group per word
            carry += min(32u, nw - b);
        } else {
            c = in ? wgroups(wd) : 0u;
            uint32_t x = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t u = __shfl_up_sync(0xffffffffu, x, d);
                if (lane >= (uint32_t)d) x += u;
            }
            p = carry + x - c;
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
        const uint32_t pt = wpattern(wd);
        const uint32_t a = max(p, g0), e = min(p + c, g1);
        const uint32_t L = (in && e > a) ? e - a : 0u;
        if (L == 1u) {
            P[a - g0] = pt;
        } else if (L <= GSHORT) {
#pragma unroll 1
            for (uint32_t q = a; q < a + L; ++q) P[q - g0] = pt;
        }
        // long fills: the whole warp paints each one
        uint32_t lm = __ballot_sync(0xffffffffu, L > GSHORT);
        while (lm) {
            const uint32_t src = __ffs(lm) - 1u;
            lm &= lm - 1u;
            const uint32_t a0 = __shfl_sync(0xffffffffu, a, src) - g0;
            const uint32_t L0 = __shfl_sync(0xffffffffu, L, src);
            const uint32_t p0 = __shfl_sync(0xffffffffu, pt, src);
            for (uint32_t q = lane; q < L0; q += 32u) P[a0 + q] = p0;
        }
    }
}

template <int OP>
__device__ __forceinline__ uint4 gone_chunk(const GoneWarp& W, int j) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint4 a = reinterpret_cast<const uint4*>(W.pat[0])[32 * j + lane];
    const uint4 b = reinterpret_cast<const uint4*>(W.pat[1])[32 * j + lane];
    return make_uint4(op2<OP>(a.x, b.x), op2<OP>(a.y, b.y), op2<OP>(a.z, b.z), op2<OP>(a.w, b.w));
}

template <int OP>
__global__ void __launch_bounds__(GTHREADS) k_gone(FuseArgs A) {
    extern __shared__ __align__(16) unsigned char gsm[];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    // exactly ntiles warps claim a tile (a launch's tickets must add up to
    // its tile count for the last one out to reset them)
    if (blockIdx.x * GWARPS + warp >= A.ntiles) return;
    GoneWarp& W = reinterpret_cast<GoneWarp*>(gsm)[warp];
    uint32_t t = 0, epoch = 0;
    if (lane == 0) {
        t = claim_tile(A.sync);
        epoch = ld_cg(&A.sync->epoch);
    }
    t = __shfl_sync(0xffffffffu, t, 0);
    epoch = __shfl_sync(0xffffffffu, epoch, 0);
    const uint32_t G = A.groups;
    const uint32_t g0 = t * (uint32_t)GT, g1 = min(g0 + (uint32_t)GT, G);
    const uint32_t ng = g1 - g0;

    // ---- paint both operands over the tile
    uint32_t xi0, xs0, xn, yi0, ys0, yn;
    const bool ok = gop_range(A.xgt, A.nx, g0, g1, xi0, xs0, xn) & gop_range(A.ygt, A.ny, g0, g1, yi0, ys0, yn);
    uint32_t before = 0;  // the result of the group before the current chunk
    if (g0 > 0 && ok) {
        const uint32_t xp = __ldg(A.xw + (xs0 < g0 ? xi0 : xi0 - 1u));
        const uint32_t yp = __ldg(A.yw + (ys0 < g0 ? yi0 : yi0 - 1u));
        before = op2<OP>(wpattern(xp), wpattern(yp));
    }
    {
        uint32_t cx = xs0, cy = ys0;
        const uint32_t nmax = max(xn, yn);
        for (uint32_t base = 0; base < nmax; base += 32u * GROWS) {
            uint32_t wx[GROWS], wy[GROWS];
            gone_load(A.xw + xi0, xn, base, wx);
            gone_load(A.yw + yi0, yn, base, wy);
            gone_paint(wx, xn, base, cx, g0, g1, W.pat[0]);
            gone_paint(wy, yn, base, cy, g0, g1, W.pat[1]);
        }
    }
    __syncwarp();

    // ---- groups: heads and popcount
    uint32_t hm = 0;  // the lane's heads: bit 4 j + e for group 128 j + 4 lane + e
    uint32_t heads = 0, ones = 0, lasth = 0;
#pragma unroll
    for (int j = 0; j < NCH; ++j) {
        const uint4 r = gone_chunk<OP>(W, j);
        uint32_t pb = __shfl_up_sync(0xffffffffu, r.w, 1);
        if (lane == 0) pb = before;
        before = __shfl_sync(0xffffffffu, r.w, 31);
        const uint32_t v[4] = {r.x, r.y, r.z, r.w};
        uint32_t pc = cls_of(pb), m = 0;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const uint32_t pos = 128u * j + 4u * lane + e;
            const uint32_t c = cls_of(v[e]);
            if (pos < ng) {
                if ((g0 + pos == 0u) || c == C_MIXED || c != pc) {
                    m |= 1u << e;
                    lasth = ((g0 + pos + 1u) << 2) | c;
                }
                ones += __popc(v[e]);
            }
            pc = c;
        }
        hm |= m << (4 * j);
        heads += __popc(m);
    }
    // a word range the metadata cannot give: the tile publishes nothing of
    // its own (so no one waits for it in vain) and writes no words
    if (!ok) { heads = 0; ones = 0; lasth = 0; }
    uint4 tot = make_uint4(__reduce_add_sync(0xffffffffu, heads), __reduce_max_sync(0xffffffffu, lasth),
                           __reduce_add_sync(0xffffffffu, ones), 0u);
    const FuseComb comb;
    uint4 pre = make_uint4(0u, 0u, 0u, 0u);
    bool lb_ok = true;
    const bool pub = t != A.withhold;
    if (t == 0) {
        if (lane == 0 && pub) frec_publish(A.recs, 0, epoch, REC_INCL, tot);
    } else {
        if (lane == 0 && pub) frec_publish(A.recs, t, epoch, REC_AGG, tot);
        pre = fuse_lookback(A.recs, t, epoch, &lb_ok);
        if (lane == 0 && pub) frec_publish(A.recs, t, epoch, REC_INCL, comb(pre, tot));
    }
    // a look-back that gave up leaves the prefix unknown; more words than
    // the result holds cannot come from valid operands: write none
    const bool over = pre.x > A.cap || tot.x > A.cap - min(pre.x, A.cap);
    if (lane == 0) {
        if (!ok || over) atomicExch(&A.meta->status, DEV_ERR_FORMAT);
        if (!lb_ok) atomicExch(&A.meta->status, DEV_ERR_TIMEOUT);
    }
    const bool skip = !ok || over || !lb_ok;
    const bool last_tile = t == A.ntiles - 1u;

    bool fill = false;
    if (!skip) {
        uint32_t acc = pre.x;    // words before the chunk
        uint32_t carry = pre.y;  // the last head before the chunk (packed)
        const uint32_t lt = (1u << lane) - 1u;
#pragma unroll 1
        for (int j = 0; j < NCH; ++j) {
            const uint32_t m = (hm >> (4 * j)) & 15u;
            const uint32_t hl = __ballot_sync(0xffffffffu, m != 0u);
            if (hl == 0u) continue;  // a chunk inside a run
            const uint4 r = gone_chunk<OP>(W, j);
            const uint32_t g = g0 + 128u * j + 4u * lane;
            const uint32_t v[4] = {r.x, r.y, r.z, r.w};
            // the lane's last head, packed; 0 without one
            uint32_t mine = 0;
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if ((m >> e) & 1u) mine = ((g + e + 1u) << 2) | cls_of(v[e]);
            // heads of the lanes before this one, from the bits of each
            // lane's count (0..4)
            const uint32_t nh = __popc(m);
            const uint32_t c0 = __ballot_sync(0xffffffffu, nh & 1u);
            const uint32_t c1 = __ballot_sync(0xffffffffu, nh & 2u);
            const uint32_t c2 = __ballot_sync(0xffffffffu, nh & 4u);
            uint32_t o = acc + __popc(c0 & lt) + 2u * __popc(c1 & lt) + 4u * __popc(c2 & lt);
            // the head before this lane's first one: the last head of the
            // nearest lower lane holding one, else the one before the chunk
            const uint32_t below = hl & lt;
            uint32_t prevh = __shfl_sync(0xffffffffu, mine, below ? 31u - __clz(below) : lane);
            if (!below) prevh = carry;
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if ((m >> e) & 1u) {
                    const uint32_t q = g + e;
                    if (prevh && (prevh & 3u) != C_MIXED) {
                        const uint32_t wd = fuse_run(prevh & 3u, q - ((prevh >> 2) - 1u));
                        A.out[o - 1u] = wd;
                        if (o == 1u) A.meta->w0 = wd;
                        fill |= is_fill(wd);
                    }
                    const uint32_t c = cls_of(v[e]);
                    if (c == C_MIXED) {
                        A.out[o] = v[e];
                        if (o == 0u) A.meta->w0 = v[e];
                    }
                    if ((o & 31u) == 0u) A.obp[o >> 5] = q;
                    prevh = ((q + 1u) << 2) | c;
                    ++o;
                }
            acc += __popc(c0) + 2u * __popc(c1) + 4u * __popc(c2);
            carry = __shfl_sync(0xffffffffu, mine, 31u - __clz(hl));
        }
        // the final run of the bitvector, by lane 0 of the last tile
        if (last_tile && lane == 0 && carry && (carry & 3u) != C_MIXED) {
            const uint32_t wd = fuse_run(carry & 3u, G - ((carry >> 2) - 1u));
            A.out[acc - 1u] = wd;
            if (acc == 1u) A.meta->w0 = wd;
            fill |= is_fill(wd);
        }
    }
    if (__any_sync(0xffffffffu, fill) && lane == 0) atomicOr(&A.meta->nfill, 1u);
    if (lane == 0) {
        if (last_tile) {
            const uint4 all = comb(pre, tot);
            const uint32_t n = skip ? 0u : all.x;
            A.obp[(n + 31u) / 32u] = G;
            A.meta->n = n;
            A.meta->groups = G;
            A.meta->nset = all.z;
            A.meta->anb = A.anb;
            A.meta->aval = A.aval;
            if (n == 0) A.meta->w0 = 0;
        }
        finish_tile(A.sync, A.ntiles);
    }
}

}  // namespace wah
#endif
