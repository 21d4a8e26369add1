// Single-pass warp-tile engine for the operators whose result compress()
// leaves canonical (the reference's _d2 / _d1 / _c1 / _c0 paths and the
// all-literal loops, src/bitvector.cpp:2545-2830, 2981-3278, 3354-3619,
// 3748-4079): one launch, operands read once, result words written once.
//
// k_gone<OP>: one warp per tile of GT = 1024 groups, warps claiming tiles in
// launch order.  The warp expands both operands over its tile exactly as the
// two-pass engine's first kernel does (gop_tile) and keeps the eight result
// chunks in registers with their run-head masks (a mixed group, a class
// change, or group 0).  It publishes {heads, last head, ones} for a
// decoupled look-back over 16-byte records, which gives the heads and the
// last head of all earlier tiles, then writes the words from registers:
// a mixed head's lane writes its literal; the word of a uniform run (its
// length is known only at the next head) is written by the lane of the next
// head, in this tile or a later one, which finds the head before it with an
// exclusive max-scan over the lanes (heads packed as (group + 1) << 2 |
// class, so a later head compares larger); the last tile writes the final
// run and the metadata.  No warp waits for another except in the bounded
// look-back: one that gives up sets DEV_ERR_TIMEOUT and writes no words.
#ifndef WAH_GONE_CUH
#define WAH_GONE_CUH
#include "wah_gop.cuh"
#include "wah_fuse.cuh"

namespace wah {

template <int OP>
__global__ void __launch_bounds__(GTHREADS, 5) k_gone(FuseArgs A) {
    extern __shared__ __align__(16) unsigned char gsm[];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    // exactly ntiles warps claim a tile (a launch's tickets must add up to
    // its tile count for the last one out to reset them)
    if (blockIdx.x * GWARPS + warp >= A.ntiles) return;
    GopWarp& W = reinterpret_cast<GopWarp*>(gsm)[warp];
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

    uint4 rv[8];
    uint32_t hm = 0;       // the lane's heads: bit 4 j + e for group 128 j + 4 lane + e
    uint32_t heads = 0, ones = 0, lasth = 0;
    uint32_t before;       // the result of the group before the current chunk
    const bool ok = gop_tile<OP>(A.xw, A.xgt, A.nx, A.yw, A.ygt, A.ny, W, g0, g1, before, [&](int j, uint4 r) {
        rv[j] = r;
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
    });
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
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint32_t m = (hm >> (4 * j)) & 15u;
            const uint32_t g = g0 + 128u * j + 4u * lane;
            const uint32_t v[4] = {rv[j].x, rv[j].y, rv[j].z, rv[j].w};
            // the lane's last head, packed; 0 without one
            uint32_t mine = 0;
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if ((m >> e) & 1u) mine = ((g + e + 1u) << 2) | cls_of(v[e]);
            uint32_t mx = mine, sum = __popc(m);
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t u = __shfl_up_sync(0xffffffffu, mx, d);
                const uint32_t s = __shfl_up_sync(0xffffffffu, sum, d);
                if (lane >= (uint32_t)d) { mx = max(mx, u); sum += s; }
            }
            uint32_t prevh = __shfl_up_sync(0xffffffffu, mx, 1);
            if (lane == 0) prevh = 0;
            prevh = max(prevh, carry);
            uint32_t o = acc + sum - __popc(m);
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
            acc += __shfl_sync(0xffffffffu, sum, 31);
            carry = max(carry, __shfl_sync(0xffffffffu, mx, 31));
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
