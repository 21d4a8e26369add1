// Group-space kernel for the operator paths whose result the reference
// leaves uncompressed or canonical (the _d2 / _d1 / _c1 / _c0 kernels and the
// all-literal loops, src/bitvector.cpp:2545-2830, 2981-3278, 3354-3619,
// 3748-4079): compress() turns their output into canonical runs, so the words
// depend only on the result bits.  The reference takes these paths only when
// the operands hold more words than half their groups (the _d2 rule
// (|a|+|b|)*31 > nbits) or one operand is uncompressed, i.e. for dense data.
//
// Tile t covers groups [t*DT, (t+1)*DT).  Its operands' words come from the
// group-tile index gtile[k] = (index, first group) of the word covering group
// k*DT, so no search is needed.  An operand whose words over the tile are one
// per group ("pure") is read straight from global memory, lane = group;
// otherwise it is first expanded into shared memory (fills longer than 32
// groups are written by the whole CTA).  Each warp then walks 32 groups per
// step: the elementwise result, its class, run heads by ballot, head indices
// by popcount.  A run's word is written by the lane holding the next head
// (its length is only known there) — consecutive indices, so the stores of a
// warp are coalesced.  Head counts and the last run cross warps and tiles
// through a block scan and the decoupled look-back of the merge kernel.
#ifndef WAH_DENSE_CUH
#define WAH_DENSE_CUH
#include "wah_merge.cuh"

namespace wah {

constexpr int DT = 2048;                  // groups per tile
constexpr int DTHREADS = 128;
constexpr int DWARPS = DTHREADS / 32;
constexpr int DGPW = DT / DWARPS;         // 512 groups per warp
constexpr int DSTEPS = DGPW / 32;         // 16 steps of 32 groups
constexpr int DFILL_MAX = DT / 32 + 2;    // long fills per operand and tile

struct DenseShared {
    uint32_t d[2][DT];      // expanded patterns of impure operands
    uint32_t fl_pos[2][DFILL_MAX], fl_len[2][DFILL_MAX], fl_val[2][DFILL_MAX];
    uint32_t fl_n[2];
    uint32_t wsum[2][DWARPS];
    uint32_t warp_agg[DWARPS][4];
    uint32_t tile_prefix[4];
    uint32_t hdr[8];
};

// Group-tile index of a bitvector: gt[2k] = index of the word covering group
// k*DT, gt[2k+1] = that word's first group; k = 0..ceil(groups/DT), the entry
// past the end holding (n, groups).
__global__ void k_gtile(const uint32_t* __restrict__ w, const uint32_t* __restrict__ bpos, uint32_t n,
                        uint32_t groups, uint32_t nt, uint32_t* __restrict__ gt) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > nt) return;
    const uint32_t g = k * (uint32_t)DT;
    if (g >= groups || n == 0) { gt[2 * k] = n; gt[2 * k + 1] = groups; return; }
    const uint32_t nb = (n + 31u) / 32u;
    uint32_t lo = 0, hi = nb;  // bpos[lo] <= g < bpos[hi]
    while (hi - lo > 1) { uint32_t m = (lo + hi) >> 1; if (__ldg(bpos + m) <= g) lo = m; else hi = m; }
    uint32_t p = __ldg(bpos + lo), i = lo * 32u;
    for (; i < n; ++i) {
        const uint32_t c = wgroups(__ldg(w + i));
        if (p + c > g) break;
        p += c;
    }
    gt[2 * k] = i;
    gt[2 * k + 1] = p;
}

struct DenseArgs {
    const uint32_t* xw; const uint32_t* xgt; uint32_t nx;
    const uint32_t* yw; const uint32_t* ygt; uint32_t ny;
    uint32_t groups;
    uint32_t* out; uint32_t* obp; DevMeta* meta;
    TileRec* recs; LaunchSync* sync; uint32_t ntiles;
    uint32_t aval, anb;
};

// Expansion of impure operands in two halves so that the words of both
// operands are requested in one batch: dense_load fetches a warp's chunk of
// words [i0, i1) into registers and sums its groups; dense_place (after one
// block barrier) writes the 31-bit patterns at their positions in S.d[side],
// restricted to the tile [g0, g1).
constexpr int DKMAX = (DT + 2 + DWARPS * 32 - 1) / (DWARPS * 32) + 1;  // words per lane
struct Chunk {
    uint32_t v[DKMAX];
    uint32_t c0, c1;
};
__device__ __forceinline__ void dense_load(DenseShared& S, int side, const uint32_t* __restrict__ w,
                                           uint32_t i0, uint32_t i1, Chunk& ch) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t nw = i1 - i0;
    const uint32_t chunk = ((nw + DWARPS - 1) / DWARPS + 31u) & ~31u;
    ch.c0 = i0 + warp * chunk;
    ch.c1 = min(ch.c0 + chunk, i1);
#pragma unroll
    for (int k = 0; k < DKMAX; ++k) {
        const uint32_t i = ch.c0 + k * 32 + lane;
        ch.v[k] = i < ch.c1 ? __ldg(w + i) : 0u;
    }
}
__device__ __forceinline__ void dense_sum(DenseShared& S, int side, const Chunk& ch) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    // groups = words + (count - 1) summed over fill words
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < DKMAX; ++k) {
        const bool in = ch.c0 + k * 32 + lane < ch.c1;
        sum += in ? 1u : 0u;
        if (in && is_fill(ch.v[k])) sum += wgroups(ch.v[k]) - 1u;
    }
    sum = __reduce_add_sync(0xffffffffu, sum);
    if (lane == 0) S.wsum[side][warp] = sum;
}
__device__ __forceinline__ void dense_place(DenseShared& S, int side, const Chunk& ch, uint32_t s0,
                                            uint32_t g0, uint32_t g1) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t carry = s0;
    for (uint32_t k = 0; k < warp; ++k) carry += S.wsum[side][k];
#pragma unroll
    for (int k = 0; k < DKMAX; ++k) {
        const uint32_t i = ch.c0 + k * 32 + lane;
        if (ch.c0 + k * 32 >= ch.c1) break;  // warp-uniform
        const uint32_t wd = ch.v[k];
        const bool in = i < ch.c1;
        const uint32_t fm = __ballot_sync(0xffffffffu, in && is_fill(wd));
        if (fm == 0 && ch.c0 + k * 32 + 32 <= ch.c1 && carry >= g0 && carry + 32 <= g1) {
            // 32 literals inside the tile: word `lane` is group carry + lane
            S.d[side][carry - g0 + lane] = wd;
            carry += 32;
            continue;
        }
        const uint32_t c = in ? wgroups(wd) : 0u;
        uint32_t p;
        if (fm == 0) {  // literals only: word `lane` starts at carry + lane
            p = carry + lane;
            carry += __popc(__ballot_sync(0xffffffffu, in));
        } else {
            uint32_t x = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) { uint32_t t = __shfl_up_sync(0xffffffffu, x, d); if (lane >= (uint32_t)d) x += t; }
            p = carry + x - c;
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
        if (in) {
            const uint32_t a = max(p, g0), e = min(p + c, g1);
            if (a < e) {
                const uint32_t pat = wpattern(wd);
                if (e - a <= 32u) {
                    for (uint32_t g = a; g < e; ++g) S.d[side][g - g0] = pat;
                } else {
                    const uint32_t slot = atomicAdd(&S.fl_n[side], 1u);
                    S.fl_pos[side][slot] = a - g0; S.fl_len[side][slot] = e - a; S.fl_val[side][slot] = pat;
                }
            }
        }
    }
}

// 31-bit pattern of group g of one operand: straight from the words when the
// operand is pure over the tile, else from the expansion.
__device__ __forceinline__ uint32_t dense_pat(const DenseShared& S, int side, bool pure,
                                              const uint32_t* __restrict__ w, uint32_t wbase, uint32_t l) {
    return pure ? wpattern(__ldg(w + wbase + l)) : S.d[side][l];
}

template <int OP>
__global__ void __launch_bounds__(DTHREADS) k_dense(DenseArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DenseShared& S = *reinterpret_cast<DenseShared*>(smem_raw);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    if (tid == 0) {
        S.hdr[0] = claim_tile(A.sync);
        S.hdr[1] = ld_cg(&A.sync->epoch);
        S.fl_n[0] = 0; S.fl_n[1] = 0;
    }
    __syncthreads();
    const uint32_t t = S.hdr[0], epoch = S.hdr[1];
    const uint32_t G = A.groups;
    const uint32_t g0 = t * (uint32_t)DT, g1 = min(g0 + (uint32_t)DT, G);
    const uint32_t ng = g1 - g0;

    // word ranges; an operand is pure over the tile when its words there are
    // exactly one per group
    const uint32_t xi0 = __ldg(A.xgt + 2 * t), xs0 = __ldg(A.xgt + 2 * t + 1);
    const uint32_t xn0 = __ldg(A.xgt + 2 * t + 2), xns = __ldg(A.xgt + 2 * t + 3);
    const uint32_t yi0 = __ldg(A.ygt + 2 * t), ys0 = __ldg(A.ygt + 2 * t + 1);
    const uint32_t yn0 = __ldg(A.ygt + 2 * t + 2), yns = __ldg(A.ygt + 2 * t + 3);
    const bool xpure = xs0 == g0 && xns == g1 && xn0 - xi0 == ng;
    const bool ypure = ys0 == g0 && yns == g1 && yn0 - yi0 == ng;
    // words covering [g0, g1): [i0, i_end) with i_end past the word covering g1-1
    const uint32_t xi1 = min(xns == g1 ? xn0 : xn0 + 1u, A.nx);
    const uint32_t yi1 = min(yns == g1 ? yn0 : yn0 + 1u, A.ny);
    // one batch of requests: both operands' words and the words before g0
    uint32_t xprev = 0, yprev = 0;
    if (tid == 0 && g0 > 0) {
        xprev = (xs0 < g0) ? __ldg(A.xw + xi0) : __ldg(A.xw + xi0 - 1);
        yprev = (ys0 < g0) ? __ldg(A.yw + yi0) : __ldg(A.yw + yi0 - 1);
    }
    {
        Chunk cx, cy;
        if (!xpure) dense_load(S, 0, A.xw, xi0, xi1, cx);
        if (!ypure) dense_load(S, 1, A.yw, yi0, yi1, cy);
        if (!xpure) dense_sum(S, 0, cx);
        if (!ypure) dense_sum(S, 1, cy);
        if (!xpure || !ypure) __syncthreads();
        if (!xpure) dense_place(S, 0, cx, xs0, g0, g1);
        if (!ypure) dense_place(S, 1, cy, ys0, g0, g1);
    }
    if (tid == 0) S.hdr[2] = (g0 > 0) ? cls_of(apply_op(OP, wpattern(xprev), wpattern(yprev))) : C_NONE;
    if (!xpure || !ypure) {
        __syncthreads();
        for (int side = 0; side < 2; ++side) {
            const uint32_t nf = S.fl_n[side];
            for (uint32_t k = 0; k < nf; ++k) {
                const uint32_t p = S.fl_pos[side][k], len = S.fl_len[side][k], val = S.fl_val[side][k];
                for (uint32_t r = tid; r < len; r += DTHREADS) S.d[side][p + r] = val;
            }
        }
        __syncthreads();
    }

    // ---- pass 1: warp w walks groups [w*DGPW, (w+1)*DGPW) of the tile
    const uint32_t wl0 = warp * DGPW;
    uint32_t r[DSTEPS];
    uint32_t hm[DSTEPS];
    uint32_t popc = 0;
    uint32_t prevc;  // class of the group before this warp's first one
    __syncthreads();  // S.hdr[2] (class before the tile) and the expansion are ready
    {
        uint32_t pc = C_NONE;
        if (lane == 0 && wl0 < ng) {
            if (wl0 > 0) {
                pc = cls_of(apply_op(OP, dense_pat(S, 0, xpure, A.xw, xi0, wl0 - 1),
                                     dense_pat(S, 1, ypure, A.yw, yi0, wl0 - 1)));
            } else {
                pc = S.hdr[2];
            }
        }
        prevc = __shfl_sync(0xffffffffu, pc, 0);
    }
    uint32_t nheads = 0, lastpos = 0, lastcls = 0;
    bool has = false;
    // issue every load of the warp before using any: 2*DSTEPS independent
    // coalesced 128-byte requests in flight per warp
    uint32_t yv[DSTEPS];
#pragma unroll
    for (int s = 0; s < DSTEPS; ++s) {
        const uint32_t l = wl0 + s * 32 + lane;
        r[s] = 0; yv[s] = 0;
        if (l < ng) {
            r[s] = xpure ? __ldg(A.xw + xi0 + l) : S.d[0][l];
            yv[s] = ypure ? __ldg(A.yw + yi0 + l) : S.d[1][l];
        }
    }
#pragma unroll
    for (int s = 0; s < DSTEPS; ++s) {
        const uint32_t l = wl0 + s * 32 + lane;
        const bool in = l < ng;
        uint32_t v = 0, c = C_NONE;
        if (in) {
            v = apply_op(OP, xpure ? wpattern(r[s]) : r[s], ypure ? wpattern(yv[s]) : yv[s]);
            c = cls_of(v);
        }
        uint32_t pcl = __shfl_up_sync(0xffffffffu, c, 1);
        if (lane == 0) pcl = prevc;
        const bool h = in && (c == C_MIXED || c != pcl);
        const uint32_t m = __ballot_sync(0xffffffffu, h);
        prevc = __shfl_sync(0xffffffffu, c, 31);
        r[s] = v;
        hm[s] = m;
        popc += __popc(v);
        if (m) {
            const uint32_t hl = 31u - __clz(m);
            nheads += __popc(m);
            lastpos = g0 + wl0 + s * 32 + hl;
            lastcls = __shfl_sync(0xffffffffu, c, hl);
            has = true;
        }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) popc += __shfl_xor_sync(0xffffffffu, popc, d);
    if (lane == 0) {
        Agg a;
        a.nheads = nheads; a.popc = popc; a.pos = lastpos;
        a.info = mk_info(lastcls, has, 0, FSM_IDENTITY);
        const uint4 v = agg_pack(a);
        S.warp_agg[warp][0] = v.x; S.warp_agg[warp][1] = v.y; S.warp_agg[warp][2] = v.z; S.warp_agg[warp][3] = v.w;
    }
    __syncthreads();
    // ---- block scan of the warp aggregates and look-back (warp 0)
    if (warp == 0) {
        Agg w = agg_identity();
        if (lane < (uint32_t)DWARPS)
            w = agg_unpack(make_uint4(S.warp_agg[lane][0], S.warp_agg[lane][1], S.warp_agg[lane][2], S.warp_agg[lane][3]));
        Agg wi = w;
#pragma unroll
        for (int d = 1; d < DWARPS; d <<= 1) {
            Agg o = agg_shfl_up<false>(wi, d);
            if (lane >= (uint32_t)d) wi = agg_combine<false>(o, wi);
        }
        Agg wx = agg_shfl_up<false>(wi, 1);
        if (lane == 0) wx = agg_identity();
        const Agg tot = agg_unpack(make_uint4(__shfl_sync(0xffffffffu, wi.nheads, DWARPS - 1),
                                              __shfl_sync(0xffffffffu, wi.pos, DWARPS - 1),
                                              __shfl_sync(0xffffffffu, wi.info, DWARPS - 1),
                                              __shfl_sync(0xffffffffu, wi.popc, DWARPS - 1)));
        if (lane < (uint32_t)DWARPS) {
            const uint4 pv = agg_pack(wx);
            S.warp_agg[lane][0] = pv.x; S.warp_agg[lane][1] = pv.y; S.warp_agg[lane][2] = pv.z; S.warp_agg[lane][3] = pv.w;
        }
        Agg prefix = agg_identity();
        if (t == 0) {
            if (lane == 0) publish(&A.recs[0], epoch, REC_INCL, agg_pack(tot));
        } else {
            if (lane == 0) publish(&A.recs[t], epoch, REC_AGG, agg_pack(tot));
            bool ok;
            prefix = agg_unpack(warp_lookback(A.recs, t, epoch, agg_pack(agg_identity()), AggComb<false>(), &ok));
            if (lane == 0) {
                if (!ok) atomicExch(&A.meta->status, DEV_ERR_TIMEOUT);
                publish(&A.recs[t], epoch, REC_INCL, agg_pack(agg_combine<false>(prefix, tot)));
            }
        }
        if (lane == 0) {
            const uint4 pv = agg_pack(prefix);
            S.tile_prefix[0] = pv.x; S.tile_prefix[1] = pv.y; S.tile_prefix[2] = pv.z; S.tile_prefix[3] = pv.w;
            if (t == A.ntiles - 1) {
                const Agg all = agg_combine<false>(prefix, tot);
                const uint32_t n = all.nheads;
                if (agg_has(all.info) && agg_cls(all.info) != C_MIXED) {
                    const uint32_t wd = run_word(agg_cls(all.info), G - all.pos, 0, false);
                    A.out[n - 1] = wd;
                    if (n - 1 == 0) A.meta->w0 = wd;
                    if (is_fill(wd)) atomicOr(&A.meta->nfill, 1u);
                }
                A.obp[(n + 31u) / 32u] = G;
                A.meta->n = n;
                A.meta->groups = G;
                A.meta->nset = all.popc;
                A.meta->anb = A.anb;
                A.meta->aval = A.aval;
                if (n == 0) A.meta->w0 = 0;
            }
        }
    }
    __syncthreads();
    // ---- pass 2: run words.  The lane of each head writes the word of the
    // run before it (a uniform run's length is known only there) and, for a
    // mixed group, its own literal.
    const Agg tp = agg_unpack(make_uint4(S.tile_prefix[0], S.tile_prefix[1], S.tile_prefix[2], S.tile_prefix[3]));
    const Agg wp = agg_unpack(make_uint4(S.warp_agg[warp][0], S.warp_agg[warp][1], S.warp_agg[warp][2], S.warp_agg[warp][3]));
    const Agg pre = agg_combine<false>(tp, wp);
    uint32_t idx = pre.nheads;                 // global index of the warp's next head
    bool lhas = agg_has(pre.info);
    uint32_t lcls = agg_cls(pre.info), lpos = pre.pos;
    uint32_t fill_seen = 0;
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int s = 0; s < DSTEPS; ++s) {
        const uint32_t m = hm[s];
        if (!m) continue;
        const uint32_t v = r[s];
        const uint32_t c = cls_of(v);
        const uint32_t pos = g0 + wl0 + s * 32 + lane;
        if (m == 0xffffffffu && __all_sync(0xffffffffu, c == C_MIXED)) {
            // 32 mixed literals: 32 consecutive words, one coalesced store
            if (lane == 0 && lhas && lcls != C_MIXED) {
                const uint32_t wd = run_word(lcls, pos - lpos, 0, false);
                A.out[idx - 1] = wd;
                if (idx - 1 == 0) A.meta->w0 = wd;
                fill_seen |= is_fill(wd) ? 1u : 0u;
            }
            A.out[idx + lane] = v;
            if (idx + lane == 0) A.meta->w0 = v;
            if (((idx + lane) & 31u) == 0) A.obp[(idx + lane) >> 5] = pos;
            idx += 32;
            lhas = true; lcls = C_MIXED; lpos = pos - lane + 31u;
            continue;
        }
        const bool h = (m >> lane) & 1u;
        const uint32_t before = m & lt;
        const uint32_t my = idx + __popc(before);
        // previous head: the highest head lane below me, else the running one
        const uint32_t pl = before ? 31u - __clz(before) : 0u;
        const uint32_t pcls = __shfl_sync(0xffffffffu, c, pl);
        if (h) {
            const bool phas = before ? true : lhas;
            const uint32_t pc = before ? pcls : lcls;
            const uint32_t pp = before ? (g0 + wl0 + s * 32 + pl) : lpos;
            if (phas && pc != C_MIXED) {
                const uint32_t wd = run_word(pc, pos - pp, 0, false);
                A.out[my - 1] = wd;
                if (my - 1 == 0) A.meta->w0 = wd;
                fill_seen |= is_fill(wd) ? 1u : 0u;
            }
            if (c == C_MIXED) {
                A.out[my] = v;
                if (my == 0) A.meta->w0 = v;
            }
            if ((my & 31u) == 0) A.obp[my >> 5] = pos;
        }
        const uint32_t hl = 31u - __clz(m);
        idx += __popc(m);
        lhas = true;
        lcls = __shfl_sync(0xffffffffu, c, hl);
        lpos = g0 + wl0 + s * 32 + hl;
    }
    if (__any_sync(0xffffffffu, fill_seen) && lane == 0) atomicOr(&A.meta->nfill, 1u);
    __syncthreads();
    if (tid == 0) finish_tile(A.sync, A.ntiles);
}

}  // namespace wah
#endif
