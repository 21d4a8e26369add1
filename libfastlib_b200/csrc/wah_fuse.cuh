// Single-pass group-space engine for the operators whose result compress()
// leaves canonical (the reference's _d2 / _d1 / _c1 / _c0 paths and the
// all-literal loops, src/bitvector.cpp:2545-2830, 2981-3278, 3354-3619,
// 3748-4079): after compress() the result words depend only on the result
// bits — one word per maximal run of equal all-0 / all-1 groups (a fill when
// the run holds two or more groups, else the literal 0 / 0x7FFFFFFF) and
// one literal per mixed group.
//
// k_gfuse<OP, FT>: one CTA per tile of FT groups (2048 by default), one launch, operands
// read once and result words written once (no intermediate array):
//  1. word phase (all the CTA's threads): each thread loads 8 consecutive
//     words of each operand from the 16-byte boundary at or below the
//     tile's first word (two 16-byte loads per operand), measures each
//     word in groups (clipped to the tile), and one block scan of both
//     operands' lengths at once (16-bit halves of one 32-bit sum) gives
//     every word's first group.  Each word then writes its 31-bit pattern
//     into the tile's group-space array of its operand (a fill of up to 8
//     groups by its own thread, a longer one by its whole warp).
//  2. group phase (the first FT / 8 threads, 8 consecutive groups each): the
//     result patterns R = a OP b, their classes, the run heads (a mixed
//     group, a class change, or group 0) and the popcount; one block scan
//     gives each thread its heads' output indices within the tile and the
//     last head before it.  The tile's aggregate {heads, last head, ones}
//     is published for a decoupled look-back, which gives the heads and
//     the last head of all earlier tiles.
//  3. write phase: a mixed head's lane writes its literal; the run word of
//     a uniform head (its length is known only at the next head) is
//     written by the lane of the next head, in this tile or a later one;
//     the last tile writes the final run's word and the metadata.  Words
//     land in shared memory and leave as 16-byte coalesced stores.
// Group arrays are stored transposed (group q at (q % 8) * FT/8 + q / 8) so
// both the painting (words ~ groups per lane) and the group phase (8
// consecutive groups per lane) hit 32 different banks.
//
// Every wait is bounded: a look-back that gives up sets DEV_ERR_TIMEOUT in
// the result's status word and the CTA writes no words.
#ifndef WAH_FUSE_CUH
#define WAH_FUSE_CUH
#include "wah_dense.cuh"

namespace wah {

constexpr int FWPT = 8;                  // word slots per thread and operand
constexpr int FGPT = 8;                  // groups per thread in the group phase
constexpr int FSHORT = 8;                // fills up to this many groups are painted by their own thread

// Tile shape: FT groups per tile (1024, 2048 or 4096: WAHGPU_TUNE_DENSE_TILE),
// enough warps for FT + 3 word slots (the tile's words from the 16-byte
// boundary below its first), FT / 8 threads in the group phase.
template <int FT_>
struct FCfg {
    static constexpr int FT = FT_;
    static constexpr int WARPS = (FT_ + 3 + FWPT * 32 - 1) / (FWPT * 32);
    static constexpr int THREADS = WARPS * 32;
    static constexpr int GTHREADS = FT_ / FGPT;
    static constexpr int ROWS = FT_ / FGPT;   // transposed row length
    static constexpr int MINB = THREADS <= 320 ? 4 : 2;
    static_assert(FT_ % DT == 0 && THREADS * FWPT >= FT_ + 3 && GTHREADS % 32 == 0, "tile shape");
};

struct FuseArgs {
    const uint32_t* xw; const uint32_t* xgt; uint32_t nx;
    const uint32_t* yw; const uint32_t* ygt; uint32_t ny;
    uint32_t groups, ntiles;
    uint32_t* out; uint32_t* obp; DevMeta* meta;
    uint32_t cap;          // words the result can hold (>= nx + ny)
    uint4* recs; LaunchSync* sync;  // one 16-byte look-back record per tile
    uint32_t aval, anb;
    uint32_t withhold;     // test hook: this tile never publishes (UINT32_MAX: none)
};

template <int FT>
struct FuseShared {
    using C = FCfg<FT>;
    uint32_t pat[2][FT];       // group patterns per operand, transposed
    uint32_t out[FT + 4];      // this tile's words, at index o - (obase & ~3)
    uint4 wagg[C::GTHREADS / 32];
    uint32_t wsum[C::WARPS];
    uint4 pre;                 // exclusive prefix of the tile (look-back)
    uint32_t tile, epoch, bad, fill, skip;
};

template <int FT>
__device__ __forceinline__ uint32_t fidx(uint32_t q) { return (q & (FGPT - 1u)) * FCfg<FT>::ROWS + (q / FGPT); }

// Word range of one operand over the tile [g0, g1): words [wi0, wi0 + nw),
// the first starting at group s0 <= g0.  gt: the operand's group-tile index
// (entry k = index and first group of the word covering group DT*k; the
// entry past the end = (n, G)).  False for a range the metadata cannot give.
__device__ __forceinline__ bool fuse_range(const uint32_t* __restrict__ gt, uint32_t n, uint32_t g0, uint32_t g1,
                                           uint32_t FT, uint32_t& wi0, uint32_t& s0, uint32_t& nw) {
    const uint32_t e0 = g0 / DT, e1 = (g1 + DT - 1) / DT;
    wi0 = __ldg(gt + 2 * e0); s0 = __ldg(gt + 2 * e0 + 1);
    const uint32_t wi1 = __ldg(gt + 2 * e1), s1 = __ldg(gt + 2 * e1 + 1);
    // the word covering g1 belongs to the tile when it starts before g1
    const uint32_t wend = (wi1 < n && s1 < g1) ? wi1 + 1u : wi1;
    nw = wend - wi0;
    const bool ok = wi0 < n && wend <= n && wend > wi0 && nw <= (uint32_t)FT && s0 <= g0 &&
                    !(g0 > 0 && s0 == g0 && wi0 == 0);
    if (!ok) { wi0 = 0; s0 = g0; nw = 0; }
    return ok;
}

// 4 words from index k (a multiple of 4) of a 16-byte-aligned array; words
// at or past n (the end of the tile's words) read as 0.
__device__ __forceinline__ uint4 fuse_ld4(const uint32_t* __restrict__ w, uint32_t k, uint32_t n) {
    if (k + 3u < n) return __ldg(reinterpret_cast<const uint4*>(w + k));
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (k < n) v.x = __ldg(w + k);
    if (k + 1u < n) v.y = __ldg(w + k + 1u);
    if (k + 2u < n) v.z = __ldg(w + k + 2u);
    return v;
}

// {heads, last head, ones, -}: sum, max, sum.  A last head is packed as
// (group + 1) << 2 | class, so 0 means "none" and later heads compare larger.
struct FuseComb {
    __device__ __forceinline__ uint4 operator()(uint4 a, uint4 b) const {
        return make_uint4(a.x + b.x, max(a.y, b.y), a.z + b.z, a.w | b.w);
    }
};

// Look-back records: one 16-byte record per tile, {heads, last head, ones,
// epoch * 4 + state}, written and read as one 16-byte access (a record is
// never seen half written; those of earlier launches carry an older epoch).
// A tile publishes its aggregate (REC_AGG) and later, in the same record,
// its inclusive prefix (REC_INCL).
__device__ __forceinline__ void frec_publish(uint4* recs, uint32_t t, uint32_t epoch, uint32_t state, uint4 v) {
    st_cg4(recs + t, make_uint4(v.x, v.y, v.z, epoch * 4u + state));
}
constexpr int FLB = 4;  // predecessors per lane per look-back round: 128 tiles per round trip

// Warp-wide look-back over 16-byte records: each round the lanes read the
// records of the 128 tiles before `hi` (lane l the FLB tiles
// [hi - FLB(l+1), hi - FLB l), all loads in flight together), wait (bounded)
// for any not yet published, and stop at the nearest inclusive record.
// Returns the exclusive prefix of tile t in every lane; *ok turns false in
// every lane when a wait of any lane gave up (warp-uniform, so callers may
// branch on it around warp-wide shuffles).
__device__ __forceinline__ uint4 fuse_lookback(const uint4* recs, uint32_t t, uint32_t epoch, bool* ok) {
    const uint32_t lane = threadIdx.x & 31u;
    const FuseComb comb;
    uint4 acc = make_uint4(0u, 0u, 0u, 0u);  // tiles already visited (later ones)
    int64_t hi = t;
    bool mine_ok = true;
    while (hi > 0) {
        uint4 v[FLB];
        uint32_t st[FLB];
#pragma unroll
        for (int k = 0; k < FLB; ++k) {  // k = 0: the latest tile of the lane
            const int64_t i = hi - 1 - (int64_t)FLB * lane - k;
            v[k] = i >= 0 ? ld_cg4(recs + i) : make_uint4(0u, 0u, 0u, epoch * 4u + REC_INCL);
        }
        uint32_t ns = 8;
        for (uint32_t it = 0;; ++it) {
            bool all = true;
#pragma unroll
            for (int k = 0; k < FLB; ++k) {
                st[k] = (v[k].w >> 2) == (epoch & 0x3FFFFFFFu) ? (v[k].w & 3u) : 0u;
                all &= st[k] != 0u;
            }
            if (all) break;
            if (it >= SPIN_LIMIT) {
                mine_ok = false;
#pragma unroll
                for (int k = 0; k < FLB; ++k)
                    if (!st[k]) { st[k] = REC_INCL; v[k] = make_uint4(0u, 0u, 0u, 0u); }
                break;
            }
            __nanosleep(ns);
            if (ns < 256) ns <<= 1;
#pragma unroll
            for (int k = 0; k < FLB; ++k)
                if (!st[k]) {
                    const int64_t i = hi - 1 - (int64_t)FLB * lane - k;
                    v[k] = ld_cg4(recs + i);
                }
        }
        // the lane's tiles in order, from its latest inclusive record on
        uint4 mine = make_uint4(0u, 0u, 0u, 0u);
        bool incl = false;
#pragma unroll
        for (int k = 0; k < FLB; ++k) {
            if (incl) continue;
            const uint4 x = make_uint4(v[k].x, v[k].y, v[k].z, 0u);
            mine = comb(x, mine);
            incl = st[k] == REC_INCL;
        }
        const uint32_t bal = __ballot_sync(0xffffffffu, incl);
        const uint32_t L = bal ? (uint32_t)(__ffs(bal) - 1) : 31u;  // nearest lane holding an inclusive record
        if (lane > L) mine = make_uint4(0u, 0u, 0u, 0u);
        // ordered tree: lane l ends up with lanes [l, ...] combined, higher
        // lanes being earlier tiles
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint4 o;
            o.x = __shfl_down_sync(0xffffffffu, mine.x, d);
            o.y = __shfl_down_sync(0xffffffffu, mine.y, d);
            o.z = __shfl_down_sync(0xffffffffu, mine.z, d);
            o.w = 0u;
            if (lane + d < 32u) mine = comb(o, mine);
        }
        uint4 win;
        win.x = __shfl_sync(0xffffffffu, mine.x, 0);
        win.y = __shfl_sync(0xffffffffu, mine.y, 0);
        win.z = __shfl_sync(0xffffffffu, mine.z, 0);
        win.w = 0u;
        acc = comb(win, acc);
        if (bal) break;
        hi -= 32 * FLB;
    }
    *ok = __all_sync(0xffffffffu, mine_ok);
    return acc;
}

// The word of a uniform run of class c and len groups.
__device__ __forceinline__ uint32_t fuse_run(uint32_t c, uint32_t len) {
    return len >= 2u ? fill_word(c, len) : (c ? ALLONES : 0u);
}

template <int OP, int FT>
__global__ void __launch_bounds__(FCfg<FT>::THREADS, FCfg<FT>::MINB) k_gfuse(FuseArgs A) {
    using C = FCfg<FT>;
    extern __shared__ __align__(16) unsigned char fsm_raw[];
    FuseShared<FT>& S = *reinterpret_cast<FuseShared<FT>*>(fsm_raw);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    if (tid == 0) {
        S.tile = claim_tile(A.sync);
        S.epoch = ld_cg(&A.sync->epoch);
        S.bad = 0;
        S.fill = 0;
        S.skip = 0;
    }
    __syncthreads();
    const uint32_t t = S.tile, epoch = S.epoch;
    const uint32_t G = A.groups;
    const uint32_t g0 = t * (uint32_t)FT, g1 = min(g0 + (uint32_t)FT, G);
    const uint32_t ng = g1 - g0;

    // ---- word phase
    uint32_t xi0, xs0, xn, yi0, ys0, yn;
    const bool okx = fuse_range(A.xgt, A.nx, g0, g1, FT, xi0, xs0, xn);
    const bool oky = fuse_range(A.ygt, A.ny, g0, g1, FT, yi0, ys0, yn);
    if (!(okx && oky) && tid == 0) {
        S.bad = 1;
        atomicExch(&A.meta->status, DEV_ERR_FORMAT);
    }
    const uint32_t kx = (xi0 & ~3u) + tid * FWPT, ky = (yi0 & ~3u) + tid * FWPT;
    uint32_t wx[FWPT], wy[FWPT];
    {
        const uint4 a0 = fuse_ld4(A.xw, kx, xi0 + xn), a1 = fuse_ld4(A.xw, kx + 4u, xi0 + xn);
        const uint4 b0 = fuse_ld4(A.yw, ky, yi0 + yn), b1 = fuse_ld4(A.yw, ky + 4u, yi0 + yn);
        wx[0] = a0.x; wx[1] = a0.y; wx[2] = a0.z; wx[3] = a0.w; wx[4] = a1.x; wx[5] = a1.y; wx[6] = a1.z; wx[7] = a1.w;
        wy[0] = b0.x; wy[1] = b0.y; wy[2] = b0.z; wy[3] = b0.w; wy[4] = b1.x; wy[5] = b1.y; wy[6] = b1.z; wy[7] = b1.w;
    }
    uint32_t st[FWPT];  // inclusive sums of the packed lengths (x low, y high)
    uint32_t run = 0;
    // slot j holds tile word kx + j - xi0 (valid when in [0, xn)); word 0
    // may start before the tile and is clipped to it
    const uint32_t rx = kx - xi0, ry = ky - yi0;
#pragma unroll
    for (int j = 0; j < FWPT; ++j) {
        uint32_t lx = rx + j < xn ? min(wgroups(wx[j]), (uint32_t)FT) : 0u;
        uint32_t ly = ry + j < yn ? min(wgroups(wy[j]), (uint32_t)FT) : 0u;
        if (rx + j == 0u) lx = min(xs0 + wgroups(wx[j]), g1) - g0;
        if (ry + j == 0u) ly = min(ys0 + wgroups(wy[j]), g1) - g0;
        run += lx | (ly << 16);
        st[j] = run;
    }
    uint32_t inc = run;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= (uint32_t)d) inc += u;
    }
    if (lane == 31) S.wsum[warp] = inc;
    __syncthreads();
    uint32_t base = inc - run;  // exclusive over the warp
    for (uint32_t w = 0; w < warp; ++w) base += S.wsum[w];
    // paint: slot j's word starts where the sums before it end
    bool longx = false, longy = false;
#pragma unroll
    for (int j = 0; j < FWPT; ++j) {
        const uint32_t ex = base + (j ? st[j - 1] : 0u);
        const uint32_t d = st[j] - (j ? st[j - 1] : 0u);
        const uint32_t lx = d & 0xFFFFu, ly = d >> 16;
        const uint32_t qx = ex & 0xFFFFu, qy = ex >> 16;
        // a literal is one store; a short fill a short loop; a long fill
        // goes to the whole warp below
        if (lx && qx < ng) {
            const uint32_t L = min(lx, ng - qx);
            if (L == 1u) {
                S.pat[0][fidx<FT>(qx)] = wpattern(wx[j]);
            } else if (L <= (uint32_t)FSHORT) {
                const uint32_t p = wpattern(wx[j]);
#pragma unroll 1
                for (uint32_t q = qx; q < qx + L; ++q) S.pat[0][fidx<FT>(q)] = p;
            } else {
                longx = true;
            }
        }
        if (ly && qy < ng) {
            const uint32_t L = min(ly, ng - qy);
            if (L == 1u) {
                S.pat[1][fidx<FT>(qy)] = wpattern(wy[j]);
            } else if (L <= (uint32_t)FSHORT) {
                const uint32_t p = wpattern(wy[j]);
#pragma unroll 1
                for (uint32_t q = qy; q < qy + L; ++q) S.pat[1][fidx<FT>(q)] = p;
            } else {
                longy = true;
            }
        }
    }
    // long fills: the whole warp paints each one
    if (__any_sync(0xffffffffu, longx || longy)) {
#pragma unroll
        for (int j = 0; j < FWPT; ++j) {
            const uint32_t ex = base + (j ? st[j - 1] : 0u);
            const uint32_t d = st[j] - (j ? st[j - 1] : 0u);
#pragma unroll
            for (int o = 0; o < 2; ++o) {
                const uint32_t l = o ? (d >> 16) : (d & 0xFFFFu);
                const uint32_t q = o ? (ex >> 16) : (ex & 0xFFFFu);
                const uint32_t L = (l && q < ng) ? min(l, ng - q) : 0u;
                uint32_t m = __ballot_sync(0xffffffffu, L > (uint32_t)FSHORT);
                while (m) {
                    const uint32_t src = __ffs(m) - 1u;
                    m &= m - 1u;
                    const uint32_t q0 = __shfl_sync(0xffffffffu, q, src);
                    const uint32_t L0 = __shfl_sync(0xffffffffu, L, src);
                    const uint32_t p0 = __shfl_sync(0xffffffffu, wpattern(o ? wy[j] : wx[j]), src);
                    for (uint32_t e = lane; e < L0; e += 32u) S.pat[o][fidx<FT>(q0 + e)] = p0;
                }
            }
        }
    }
    __syncthreads();

    // ---- group phase
    uint32_t r[FGPT];
    uint32_t hm = 0, ones = 0, lasth = 0;
    const bool grp = tid < (uint32_t)C::GTHREADS;
    if (grp) {
        const uint32_t q0 = tid * FGPT;
        const bool bad = S.bad != 0;
        uint32_t pr;  // the result of the group before q0
        if (tid > 0) {
            pr = op2<OP>(S.pat[0][fidx<FT>(q0 - 1u)], S.pat[1][fidx<FT>(q0 - 1u)]);
        } else if (g0 > 0 && !bad) {
            const uint32_t xp = __ldg(A.xw + (xs0 < g0 ? xi0 : xi0 - 1u));
            const uint32_t yp = __ldg(A.yw + (ys0 < g0 ? yi0 : yi0 - 1u));
            pr = op2<OP>(wpattern(xp), wpattern(yp));
        } else {
            pr = 0u;
        }
        uint32_t pc = cls_of(pr);
#pragma unroll
        for (int e = 0; e < FGPT; ++e) {
            const uint32_t q = q0 + e;
            const bool in = q < ng;
            const uint32_t a = (in && !bad) ? S.pat[0][fidx<FT>(q)] : 0u;
            const uint32_t b = (in && !bad) ? S.pat[1][fidx<FT>(q)] : 0u;
            r[e] = op2<OP>(a, b);
            const uint32_t c = cls_of(r[e]);
            if (in) {
                if (g0 + q == 0u || c == C_MIXED || c != pc) {
                    hm |= 1u << e;
                    lasth = ((g0 + q + 1u) << 2) | c;
                }
                ones += __popc(r[e]);
            }
            pc = c;
        }
    }
    // block scan of {heads, last head, ones} over the group threads
    const uint4 mine = make_uint4((uint32_t)__popc(hm), lasth, ones, 0u);
    uint4 incl = mine;
    const FuseComb comb;
    if (grp) {
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint4 u;
            u.x = __shfl_up_sync(0xffffffffu, incl.x, d);
            u.y = __shfl_up_sync(0xffffffffu, incl.y, d);
            u.z = __shfl_up_sync(0xffffffffu, incl.z, d);
            u.w = 0u;
            if (lane >= (uint32_t)d) incl = comb(u, incl);
        }
        if (lane == 31) S.wagg[warp] = incl;
    }
    __syncthreads();
    uint4 ex = make_uint4(0u, 0u, 0u, 0u);
    uint4 tot = make_uint4(0u, 0u, 0u, 0u);
    if (grp) {
        uint4 e1;
        e1.x = __shfl_up_sync(0xffffffffu, incl.x, 1);
        e1.y = __shfl_up_sync(0xffffffffu, incl.y, 1);
        e1.z = __shfl_up_sync(0xffffffffu, incl.z, 1);
        e1.w = 0u;
        if (lane == 0) e1 = make_uint4(0u, 0u, 0u, 0u);
        for (uint32_t w = 0; w < warp; ++w) ex = comb(ex, S.wagg[w]);
        ex = comb(ex, e1);
    }
#pragma unroll
    for (int w = 0; w < C::GTHREADS / 32; ++w) tot = comb(tot, S.wagg[w]);
    // look-back for the heads and last head of all earlier tiles
    if (warp == 0) {
        uint4 pre = make_uint4(0u, 0u, 0u, 0u);
        bool ok = true;
        const bool pub = t != A.withhold;
        if (t == 0) {
            if (lane == 0 && pub) frec_publish(A.recs, 0, epoch, REC_INCL, tot);
        } else {
            if (lane == 0 && pub) frec_publish(A.recs, t, epoch, REC_AGG, tot);
            pre = fuse_lookback(A.recs, t, epoch, &ok);
            if (lane == 0 && pub) frec_publish(A.recs, t, epoch, REC_INCL, comb(pre, tot));
        }
        if (lane == 0) {
            // a wait that gave up leaves the prefix unknown: no words are
            // written (the status word reports it)
            if (!ok) { atomicExch(&A.meta->status, DEV_ERR_TIMEOUT); S.skip = 1u; }
            // more words than the result holds cannot come from valid
            // operands; refuse to write them
            if (pre.x > A.cap || tot.x > A.cap - min(pre.x, A.cap)) {
                atomicExch(&A.meta->status, DEV_ERR_FORMAT);
                S.skip = 1u;
            }
            S.pre = pre;
        }
    }
    __syncthreads();
    const uint4 pre = S.pre;
    const uint32_t obase = pre.x, oal = obase & ~3u;
    const bool last_tile = t == A.ntiles - 1u;
    const bool skip = S.skip != 0;

    // ---- write phase
    bool wrote_fill = false;
    if (!skip && grp && (hm || (last_tile && tid == 0 && tot.x == 0u))) {
        uint32_t o = obase + ex.x;
        uint32_t prevh = max(pre.y, ex.y);  // the head before my first one
        // word idx: this tile's words go to shared memory; the last run of
        // an earlier tile straight to its place (word 0 also to w0; tile 0
        // sets w0 from its own words after the flush)
        auto emit = [&](uint32_t idx, uint32_t wd) {
            if (idx >= obase) {
                S.out[idx - oal] = wd;
            } else {
                A.out[idx] = wd;
                if (idx == 0u) A.meta->w0 = wd;
            }
        };
#pragma unroll
        for (int e = 0; e < FGPT; ++e) {
            if ((hm >> e) & 1u) {
                const uint32_t q = g0 + tid * FGPT + e;
                if (prevh && (prevh & 3u) != C_MIXED) {
                    const uint32_t wd = fuse_run(prevh & 3u, q - ((prevh >> 2) - 1u));
                    wrote_fill |= is_fill(wd);
                    emit(o - 1u, wd);
                }
                const uint32_t c = cls_of(r[e]);
                if (c == C_MIXED) S.out[o - oal] = r[e];
                if ((o & 31u) == 0u) A.obp[o >> 5] = q;
                prevh = ((q + 1u) << 2) | c;
                ++o;
            }
        }
        // the final run of the bitvector: by the lane of the last head, or
        // by thread 0 when the last tile has no head
        if (last_tile && ex.x + (uint32_t)__popc(hm) == tot.x && prevh && (prevh & 3u) != C_MIXED) {
            const uint32_t wd = fuse_run(prevh & 3u, G - ((prevh >> 2) - 1u));
            wrote_fill |= is_fill(wd);
            emit(o - 1u, wd);
        }
    }
    if (grp && __any_sync(0xffffffffu, wrote_fill) && lane == 0) S.fill = 1u;
    __syncthreads();
    // flush this tile's words; a uniform last head's word comes from a later tile
    const uint32_t cnt = tot.x - ((!last_tile && tot.x && (tot.y & 3u) != C_MIXED) ? 1u : 0u);
    if (cnt && !skip) {
        const uint32_t end = obase + cnt;
        const uint32_t nv = (end - oal + 3u) / 4u;
        for (uint32_t v = tid; v < nv; v += C::THREADS) {
            const uint32_t gi = oal + 4u * v;
            if (gi >= obase && gi + 3u < end) {
                *reinterpret_cast<uint4*>(A.out + gi) = *reinterpret_cast<const uint4*>(&S.out[4u * v]);
            } else {
#pragma unroll
                for (uint32_t e = 0; e < 4u; ++e)
                    if (gi + e >= obase && gi + e < end) A.out[gi + e] = S.out[4u * v + e];
            }
        }
    }
    if (tid == 0) {
        if (S.fill) atomicOr(&A.meta->nfill, 1u);
        if (obase == 0u && cnt && !skip) A.meta->w0 = S.out[0];
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
