// Group-space kernel for the operator paths whose result the reference
// leaves uncompressed or canonical (the _d2 / _d1 / _c1 / _c0 kernels and the
// all-literal loops, src/bitvector.cpp:2545-2830, 2981-3278, 3354-3619,
// 3748-4079): compress() turns their output into canonical runs, so the words
// depend only on the result bits.  The reference takes these paths only when
// the operands hold more words than half their groups (the _d2 rule
// (|a|+|b|)*31 > nbits) or one operand is uncompressed, i.e. for dense data.
//
// Structure: a persistent, warp-specialised pipeline.  Each CTA runs one
// control warp and NCW compute warps.
//
//  * The control warp claims tiles of TG groups in order (atomic ticket),
//    finds each tile's word ranges in the group-tile index, and prefetches
//    the words of both operands into a ring of NI shared-memory slots with
//    bulk copies (cp.async.bulk) that complete on the slot's mbarrier.  It
//    also runs the decoupled look-back for every claimed tile as soon as the
//    predecessors' records appear, so a tile's prefix is usually known
//    before its words are even consumed.
//  * The compute warps take the slots in order.  For an operand whose words
//    over the tile are one per group ("pure") the patterns are read straight
//    from the slot; otherwise each thread scans a contiguous run of words,
//    a block scan places them, and a marker per word start plus one cover
//    entry per 128-group step let every lane find the word of each of its
//    groups by a warp max-scan — no loop over fill lengths.  Pass 1 gives
//    per group the result, its class and the run heads (4 consecutive
//    groups per lane; a step of 128 mixed results takes a branch-free
//    path), kept in shared memory with the tile's aggregate (heads, last
//    head, popcount), which is published as the tile's look-back record.
//  * Pass 2 of a tile runs one tile later, after pass 1 of the next one, so
//    the control warp's look-back has had a whole tile of time.  The lane of
//    each head writes the word of the run before it (a uniform run's length
//    is only known there) and, for a mixed group, its own literal.
//
// Every wait is bounded (WAIT_LIMIT_NS without progress); a timeout sets the
// result's status word and all warps leave the pipeline.
#ifndef WAH_DENSE_CUH
#define WAH_DENSE_CUH
#include "wah_merge.cuh"

namespace wah {

constexpr int DT = 512;                   // group-tile index stride (k_gtile)
constexpr uint32_t DEND = 0xFFFFFFFFu;    // slot marker: no more tiles
constexpr uint32_t DFAST = 0xFFFFFFFFu;   // step code: 128 mixed literals

template <int TG, int NCW>
struct DCfg {
    static constexpr int NI = 3;                  // prefetch slots
    static constexpr int NP = NI + 2;             // prefix slots (tiles claimed ahead of pass 2)
    static constexpr int CT = NCW * 32;           // compute threads
    static constexpr int GPW = TG / NCW;          // groups per compute warp
    static constexpr int STEPS = GPW / 128;       // steps of 4 groups per lane
    static constexpr int NSTEP = TG / 128;        // steps per tile
    static constexpr int BUFW = TG + 8;           // words per operand slot
    static constexpr int WPT = ((TG + CT - 1) / CT) | 1;  // words per thread when expanding (odd)
    static_assert(TG % DT == 0 && GPW % 128 == 0 && STEPS >= 1, "tile shape");
};

// Tile words as the control warp found them (indices into the slot buffer).
struct DSlot {
    uint32_t t, g0, ng, flags;                    // flags: 1 x pure, 2 y pure
    uint32_t xlo, xhi, xs0, xprev;                // words [xlo, xhi) = [xi0, xi1); xs0 first group of xi0
    uint32_t ylo, yhi, ys0, yprev;                // xprev: the word covering g0-1
};

template <int TG, int NCW>
struct DShared {
    using C = DCfg<TG, NCW>;
    uint4 in[C::NI][2][C::BUFW / 4];              // prefetched words
    uint4 res[2][TG / 4];                         // pass-1 results of the last two tiles
    uint32_t code[2][C::NSTEP * 32];              // head flags | classes per lane and step, or DFAST
    uint16_t mk[2][TG];                           // expansion: buffer index + 1 of the word starting here
    uint32_t cov[2][C::NSTEP];                    // expansion: buffer index of the word covering step q
    uint32_t xsum[2][NCW];
    DSlot slot[C::NI];
    uint4 prefix[C::NP];                          // look-back result per claimed tile
    uint32_t lbt[C::NP];                          // tile of each claim awaiting its look-back (control)
    uint4 wagg[2][NCW];                           // warp aggregates, then warp exclusive prefixes
    uint4 tagg[2];                                // tile aggregate
    uint32_t tinfo[2][4];                         // tile, g0, ng
    uint64_t full[C::NI], empty[C::NI], pre[C::NP];
    uint32_t epoch, abort, ok;
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
    uint4* drecs; LaunchSync* sync; uint32_t ntiles;
    uint32_t aval, anb;
};

// ---- tile aggregates: {popc, nheads | cls << 28 | has << 30, pos, -}.
// The look-back record of tile t is drecs[t] = {popc, nheads|cls|has,
// pos | state << 28, epoch}, written and read as one 16-byte access so that
// a record is never seen half written; records of earlier launches carry an
// older epoch.
__device__ __forceinline__ uint4 dagg_comb(uint4 a, uint4 b) {  // a before b
    const bool hb = (b.y >> 30) & 1u;
    uint4 r;
    r.x = a.x + b.x;
    r.y = ((a.y & 0x0FFFFFFFu) + (b.y & 0x0FFFFFFFu)) | ((hb ? b.y : a.y) & 0x70000000u);
    r.z = hb ? b.z : a.z;
    r.w = 0;
    return r;
}
__device__ __forceinline__ uint4 dagg_make(uint32_t nheads, uint32_t popc, uint32_t pos, uint32_t cls, bool has) {
    return make_uint4(popc, nheads | (cls << 28) | (has ? (1u << 30) : 0u), pos, 0u);
}
__device__ __forceinline__ uint32_t dagg_n(uint4 a) { return a.y & 0x0FFFFFFFu; }
__device__ __forceinline__ uint32_t dagg_cls(uint4 a) { return (a.y >> 28) & 3u; }
__device__ __forceinline__ bool dagg_has(uint4 a) { return (a.y >> 30) & 1u; }
__device__ __forceinline__ void drec_publish(uint4* recs4, uint32_t t, uint32_t epoch, uint32_t state, uint4 a) {
    st_cg4(recs4 + t, make_uint4(a.x, a.y, a.z | (state << 28), epoch));
}

// One step of the warp-wide look-back: reads the records of up to 32 tiles
// before `hi`; if every one of them up to the nearest inclusive record is
// present, folds them into acc and moves hi.  Returns 2 when the prefix is
// complete, 1 when a window was consumed, 0 when a record is not there yet.
__device__ __forceinline__ int dlook_step(const uint4* recs4, uint32_t epoch, uint32_t& hi, uint4& acc) {
    const uint32_t lane = threadIdx.x & 31u;
    if (hi == 0) return 2;
    const int64_t p = (int64_t)hi - 1 - lane;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    bool valid = true, incl = true;
    if (p >= 0) {
        const uint4 r = ld_cg4(recs4 + p);
        const uint32_t st = (r.z >> 28) & 3u;
        valid = r.w == epoch && (st == REC_AGG || st == REC_INCL);
        incl = valid && st == REC_INCL;
        v = make_uint4(r.x, r.y, r.z & 0x0FFFFFFFu, 0u);
    }
    const uint32_t im = __ballot_sync(0xffffffffu, incl);
    const uint32_t vm = __ballot_sync(0xffffffffu, valid);
    const uint32_t L = im ? (uint32_t)(__ffs(im) - 1) : 31u;
    const uint32_t need = L == 31u ? 0xffffffffu : ((2u << L) - 1u);
    if ((vm & need) != need) return 0;
    if (lane > L) v = make_uint4(0u, 0u, 0u, 0u);
    // ordered tree: lane l ends up with lanes [l, 31] combined, higher lanes
    // being earlier tiles
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint4 o;
        o.x = __shfl_down_sync(0xffffffffu, v.x, d);
        o.y = __shfl_down_sync(0xffffffffu, v.y, d);
        o.z = __shfl_down_sync(0xffffffffu, v.z, d);
        o.w = 0;
        if (lane + d < 32u) v = dagg_comb(o, v);
    }
    uint4 win;
    win.x = __shfl_sync(0xffffffffu, v.x, 0);
    win.y = __shfl_sync(0xffffffffu, v.y, 0);
    win.z = __shfl_sync(0xffffffffu, v.z, 0);
    win.w = 0;
    acc = dagg_comb(win, acc);
    if (im) { hi = 0; return 2; }
    hi = hi > 32u ? hi - 32u : 0u;
    return hi == 0 ? 2 : 1;
}

__device__ __forceinline__ void dense_fail(const DenseArgs& A, volatile uint32_t* abort) {
    atomicExch(&A.meta->status, DEV_ERR_TIMEOUT);
    *abort = 1u;
}

// Bounded wait that also gives up when another warp has aborted.
__device__ __forceinline__ bool dwait(uint64_t* b, uint32_t par, volatile uint32_t* abort) {
    if (mbar_test(b, par)) return true;
    const uint64_t t0 = gtimer();
    uint32_t ns = 32;
    while (!mbar_test(b, par)) {
        if (*abort) return false;
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
        if (gtimer() - t0 > WAIT_LIMIT_NS) return false;
    }
    return true;
}

// ------------------------------------------------------------- control warp
template <int TG, int NCW>
__device__ __forceinline__ void dense_control(DShared<TG, NCW>& S, const DenseArgs& A, uint32_t epoch) {
    using C = DCfg<TG, NCW>;
    const uint32_t lane = threadIdx.x & 31u;
    volatile uint32_t* abort = &S.abort;
    const uint4* recs4 = A.drecs;
    const uint32_t G = A.groups;
    const uint32_t nt = (G + DT - 1) / DT;
    uint32_t seq_claim = 0, n_real = 0, seq_lb = 0;
    bool ended = false, lb_active = false;
    uint32_t lb_hi = 0;
    uint4 lb_acc = make_uint4(0u, 0u, 0u, 0u);
    uint64_t last = gtimer();
    uint32_t ns = 32;
    // every branch below is taken by the whole warp: lane 0 decides
    while (true) {
        if (__shfl_sync(0xffffffffu, *abort, 0)) break;
        bool progress = false;
        // 1) claim the next tile and prefetch its words into a free slot
        if (!ended && seq_claim < seq_lb + (uint32_t)C::NP) {
            const uint32_t s = seq_claim % C::NI, u = seq_claim / C::NI;
            const bool free_slot = __shfl_sync(0xffffffffu, (u == 0 || mbar_test(&S.empty[s], (u - 1u) & 1u)) ? 1u : 0u, 0);
            if (free_slot) {
                uint32_t t = 0;
                if (lane == 0) t = atomicAdd(&A.sync->ticket, 1u);
                t = __shfl_sync(0xffffffffu, t, 0);
                if (t >= A.ntiles) {
                    if (lane == 0) { S.slot[s].t = DEND; mbar_arrive(&S.full[s]); }
                    ended = true;
                } else {
                    const uint32_t k0 = t * (uint32_t)(TG / DT), k1 = min(k0 + (uint32_t)(TG / DT), nt);
                    uint2 e = make_uint2(0u, 0u);
                    if (lane < 4) {
                        const uint32_t* gt = (lane < 2) ? A.xgt : A.ygt;
                        e = __ldg(reinterpret_cast<const uint2*>(gt) + ((lane & 1u) ? k1 : k0));
                    }
                    const uint32_t xi0 = __shfl_sync(0xffffffffu, e.x, 0), xs0 = __shfl_sync(0xffffffffu, e.y, 0);
                    const uint32_t xn1 = __shfl_sync(0xffffffffu, e.x, 1), xg1 = __shfl_sync(0xffffffffu, e.y, 1);
                    const uint32_t yi0 = __shfl_sync(0xffffffffu, e.x, 2), ys0 = __shfl_sync(0xffffffffu, e.y, 2);
                    const uint32_t yn1 = __shfl_sync(0xffffffffu, e.x, 3), yg1 = __shfl_sync(0xffffffffu, e.y, 3);
                    if (lane == 0) {
                        const uint32_t g0 = t * (uint32_t)TG, g1 = min(g0 + (uint32_t)TG, G), ng = g1 - g0;
                        const uint32_t xi1 = min(xg1 == g1 ? xn1 : xn1 + 1u, A.nx);
                        const uint32_t yi1 = min(yg1 == g1 ? yn1 : yn1 + 1u, A.ny);
                        // copies start at the word covering g0-1 when that is not
                        // the tile's first word, rounded down to 16 bytes
                        const uint32_t xcs = ((g0 > 0 && xs0 == g0) ? xi0 - 1u : xi0) & ~3u;
                        const uint32_t ycs = ((g0 > 0 && ys0 == g0) ? yi0 - 1u : yi0) & ~3u;
                        const uint32_t xb = ((xi1 - xcs + 3u) & ~3u) * 4u, yb = ((yi1 - ycs + 3u) & ~3u) * 4u;
                        DSlot& m = S.slot[s];
                        m.t = t; m.g0 = g0; m.ng = ng;
                        m.flags = ((xs0 == g0 && xg1 == g1 && xn1 - xi0 == ng) ? 1u : 0u) |
                                  ((ys0 == g0 && yg1 == g1 && yn1 - yi0 == ng) ? 2u : 0u);
                        m.xlo = xi0 - xcs; m.xhi = xi1 - xcs; m.xs0 = xs0;
                        m.xprev = g0 == 0 ? 0u : (xs0 < g0 ? m.xlo : m.xlo - 1u);
                        m.ylo = yi0 - ycs; m.yhi = yi1 - ycs; m.ys0 = ys0;
                        m.yprev = g0 == 0 ? 0u : (ys0 < g0 ? m.ylo : m.ylo - 1u);
                        S.lbt[seq_claim % C::NP] = t;
                        mbar_arrive_tx(&S.full[s], xb + yb);
                        bulk_g2s(S.in[s][0], A.xw + xcs, xb, &S.full[s]);
                        bulk_g2s(S.in[s][1], A.yw + ycs, yb, &S.full[s]);
                    }
                    ++n_real;
                }
                ++seq_claim;
                progress = true;
            }
        }
        // 2) look-back of the oldest claimed tile still without a prefix
        if (seq_lb < n_real) {
            __syncwarp();
            if (!lb_active) {
                lb_active = true;
                lb_hi = S.lbt[seq_lb % C::NP];
                lb_acc = make_uint4(0u, 0u, 0u, 0u);
            }
            int r;
            while ((r = dlook_step(recs4, epoch, lb_hi, lb_acc)) == 1) {}
            if (r == 2) {
                if (lane == 0) {
                    S.prefix[seq_lb % C::NP] = lb_acc;
                    mbar_arrive(&S.pre[seq_lb % C::NP]);
                }
                ++seq_lb;
                lb_active = false;
                progress = true;
            }
        }
        if (ended && seq_lb == n_real) break;
        if (progress) {
            last = gtimer();
            ns = 32;
        } else {
            __nanosleep(ns);
            if (ns < 256) ns <<= 1;
            if (__shfl_sync(0xffffffffu, (gtimer() - last > WAIT_LIMIT_NS) ? 1u : 0u, 0)) {
                if (lane == 0) dense_fail(A, abort);
                break;
            }
        }
    }
    __syncwarp();
    if (lane == 0 && *abort) {
        // leave no bulk copy in flight: wait (bounded) for the last claims
        const uint32_t first = seq_claim > (uint32_t)C::NI ? seq_claim - C::NI : 0u;
        for (uint32_t q = first; q < seq_claim; ++q) {
            if (S.slot[q % C::NI].t == DEND) continue;
            const uint64_t t0 = gtimer();
            while (!mbar_test(&S.full[q % C::NI], (q / C::NI) & 1u) && gtimer() - t0 < WAIT_LIMIT_NS) __nanosleep(256);
        }
    }
}

// ------------------------------------------------------------ compute warps
__device__ __forceinline__ uint4 realign4(const uint4* b4, uint32_t base) {
    // words base .. base+3 of a 16-byte aligned word buffer
    const uint32_t q = base >> 2, a = base & 3u;
    const uint4 A = b4[q];
    if (a == 0) return A;
    const uint4 B = b4[q + 1];
    if (a == 1) return make_uint4(A.y, A.z, A.w, B.x);
    if (a == 2) return make_uint4(A.z, A.w, B.x, B.y);
    return make_uint4(A.w, B.x, B.y, B.z);
}
__device__ __forceinline__ uint4 pattern4(uint4 v) {
    return make_uint4(wpattern(v.x), wpattern(v.y), wpattern(v.z), wpattern(v.w));
}
template <int OP>
__device__ __forceinline__ uint32_t op2(uint32_t a, uint32_t b) {
    if (OP == OP_AND) return a & b;
    if (OP == OP_OR) return a | b;
    if (OP == OP_XOR) return a ^ b;
    return a & ~b;  // patterns have bit 31 clear
}
// 1..ALLONES-1: a group that is neither all-0 nor all-1
__device__ __forceinline__ bool is_mixed(uint32_t v) { return v - 1u < ALLONES - 1u; }
__device__ __forceinline__ uint32_t cls_in(uint32_t v, bool in) { return in ? cls_of(v) : (uint32_t)C_NONE; }

// Expansion of an impure operand: markers at word starts and the word
// covering every step start.  Two calls: phase 0 sums the thread's words
// (returns its exclusive position inside the warp), phase 1 places them.
template <int TG, int NCW>
__device__ __forceinline__ void exp_sum(DShared<TG, NCW>& S, int side, const uint32_t* buf, uint32_t lo, uint32_t hi,
                                        uint32_t (&v)[DCfg<TG, NCW>::WPT], uint32_t& ex) {
    using C = DCfg<TG, NCW>;
    const uint32_t tid = threadIdx.x, lane = tid & 31u;
    const uint32_t j0 = lo + tid * C::WPT;
    uint32_t sum = 0;
#pragma unroll
    for (int j = 0; j < C::WPT; ++j) {
        const bool in = j0 + j < hi;
        v[j] = in ? buf[j0 + j] : 0u;
        if (in) sum += wgroups(v[j]);
    }
    uint32_t x = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= (uint32_t)d) x += t;
    }
    if (lane == 31) S.xsum[side][tid >> 5] = x;
    ex = x - sum;
}
template <int TG, int NCW>
__device__ __forceinline__ void exp_place(DShared<TG, NCW>& S, int side, uint32_t lo, uint32_t hi, uint32_t s0,
                                          const uint32_t (&v)[DCfg<TG, NCW>::WPT], uint32_t ex,
                                          uint32_t g0, uint32_t g1) {
    using C = DCfg<TG, NCW>;
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t j0 = lo + tid * C::WPT;
    uint32_t p = s0 + ex;
    for (uint32_t k = 0; k < warp; ++k) p += S.xsum[side][k];
#pragma unroll
    for (int j = 0; j < C::WPT; ++j) {
        if (j0 + j < hi) {
            const uint32_t c = wgroups(v[j]);
            if (p >= g0 && p < g1) S.mk[side][p - g0] = (uint16_t)(j0 + j + 1u);
            const uint32_t a = max(p, g0), e = min(p + c, g1);
            if (a < e) {
                // step starts q*128 inside [a, e)
                for (uint32_t q = (a - g0 + 127u) >> 7; (q << 7) < e - g0; ++q) S.cov[side][q] = j0 + j;
            }
            p += c;
        }
    }
}
// buffer index of the word covering group 128q-1 of the tile (q >= 1)
template <int TG, int NCW>
__device__ __forceinline__ uint32_t exp_word_before(const DShared<TG, NCW>& S, int side, uint32_t q) {
    return S.mk[side][q << 7] ? S.cov[side][q] - 1u : S.cov[side][q];
}
// the 4 patterns of groups l..l+3 of an impure operand (whole warp)
template <int TG, int NCW>
__device__ __forceinline__ uint4 exp_read4(const DShared<TG, NCW>& S, int side, const uint32_t* buf, uint32_t l,
                                           uint32_t q) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint2 mm = *reinterpret_cast<const uint2*>(&S.mk[side][l]);
    // lane 0 starts from the word covering the step's first group, so every
    // lane's running maximum is at least 1
    uint32_t a0 = max(mm.x & 0xFFFFu, lane == 0 ? S.cov[side][q] + 1u : 0u);
    uint32_t a1 = max(a0, mm.x >> 16);
    uint32_t a2 = max(a1, mm.y & 0xFFFFu);
    uint32_t a3 = max(a2, mm.y >> 16);
    uint32_t inc = a3;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= (uint32_t)d) inc = max(inc, o);
    }
    uint32_t ex = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0) ex = 0u;
    a0 = max(a0, ex); a1 = max(a1, ex); a2 = max(a2, ex); a3 = max(a3, ex);
    return make_uint4(wpattern(buf[a0 - 1u]), wpattern(buf[a1 - 1u]), wpattern(buf[a2 - 1u]), wpattern(buf[a3 - 1u]));
}

// Pass 1 of one tile: results and codes into buffer b, tile aggregate
// published; the slot's words are released.
template <int OP, int TG, int NCW>
__device__ __forceinline__ void dense_pass1(DShared<TG, NCW>& S, const DenseArgs& A, const DSlot& m, uint32_t s,
                                            uint32_t b, uint32_t epoch) {
    using C = DCfg<TG, NCW>;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t* bx = reinterpret_cast<const uint32_t*>(S.in[s][0]);
    const uint32_t* by = reinterpret_cast<const uint32_t*>(S.in[s][1]);
    const uint4* bx4 = S.in[s][0];
    const uint4* by4 = S.in[s][1];
    const bool xpure = m.flags & 1u, ypure = m.flags & 2u;
    const uint32_t g0 = m.g0, ng = m.ng, g1 = g0 + ng;
    if (!xpure || !ypure) {
        uint32_t vx[C::WPT], vy[C::WPT];
        uint32_t ex = 0, ey = 0;
        if (!xpure) for (uint32_t i = tid; i < (uint32_t)TG / 8u; i += C::CT) reinterpret_cast<uint4*>(S.mk[0])[i] = make_uint4(0u, 0u, 0u, 0u);
        if (!ypure) for (uint32_t i = tid; i < (uint32_t)TG / 8u; i += C::CT) reinterpret_cast<uint4*>(S.mk[1])[i] = make_uint4(0u, 0u, 0u, 0u);
        if (!xpure) exp_sum<TG, NCW>(S, 0, bx, m.xlo, m.xhi, vx, ex);
        if (!ypure) exp_sum<TG, NCW>(S, 1, by, m.ylo, m.yhi, vy, ey);
        bar_sync1(C::CT);
        if (!xpure) exp_place<TG, NCW>(S, 0, m.xlo, m.xhi, m.xs0, vx, ex, g0, g1);
        if (!ypure) exp_place<TG, NCW>(S, 1, m.ylo, m.yhi, m.ys0, vy, ey, g0, g1);
        bar_sync1(C::CT);
    }
    // class of the group before the warp's first one
    const uint32_t wl0 = warp * C::GPW;
    uint32_t prevc = C_NONE;
    if (lane == 0 && wl0 < ng) {
        if (wl0 == 0) {
            if (g0 > 0) prevc = cls_of(op2<OP>(wpattern(bx[m.xprev]), wpattern(by[m.yprev])));
        } else {
            const uint32_t q = wl0 >> 7;
            const uint32_t px = xpure ? wpattern(bx[m.xlo + wl0 - 1u]) : wpattern(bx[exp_word_before(S, 0, q)]);
            const uint32_t py = ypure ? wpattern(by[m.ylo + wl0 - 1u]) : wpattern(by[exp_word_before(S, 1, q)]);
            prevc = cls_of(op2<OP>(px, py));
        }
    }
    prevc = __shfl_sync(0xffffffffu, prevc, 0);

    uint32_t nheads = 0, lastpos = 0, lastcls = 0, popc = 0;
    bool has = false;
#pragma unroll
    for (int st = 0; st < C::STEPS; ++st) {
        const uint32_t sb = wl0 + st * 128u;            // step's first group (tile-relative)
        uint32_t* codep = &S.code[b][((warp * C::STEPS + st) << 5) + lane];
        if (sb >= ng) {                                  // past the tile's end
            *codep = 0u;
            S.res[b][(sb >> 2) + lane] = make_uint4(0u, 0u, 0u, 0u);
            continue;
        }
        const uint32_t l = sb + 4u * lane;
        const uint32_t q = sb >> 7;
        uint4 X = xpure ? realign4(bx4, m.xlo + l) : exp_read4(S, 0, bx, l, q);
        uint4 Y = ypure ? realign4(by4, m.ylo + l) : exp_read4(S, 1, by, l, q);
        // pure operands may hold count-1 fill words
        if (__any_sync(0xffffffffu, ((X.x | X.y | X.z | X.w | Y.x | Y.y | Y.z | Y.w) >> 31) != 0u)) {
            X = pattern4(X);
            Y = pattern4(Y);
        }
        uint4 v = make_uint4(op2<OP>(X.x, Y.x), op2<OP>(X.y, Y.y), op2<OP>(X.z, Y.z), op2<OP>(X.w, Y.w));
        const bool full = sb + 128u <= ng;
        const bool allmixed = is_mixed(v.x) & is_mixed(v.y) & is_mixed(v.z) & is_mixed(v.w);
        if (full && __all_sync(0xffffffffu, allmixed)) {
            *codep = DFAST;
            nheads += 128u;
            lastpos = g0 + sb + 127u;
            lastcls = C_MIXED;
            has = true;
            prevc = C_MIXED;
        } else {
            const bool i0 = l < ng, i1 = l + 1u < ng, i2 = l + 2u < ng, i3 = l + 3u < ng;
            if (!i0) v.x = 0u;
            if (!i1) v.y = 0u;
            if (!i2) v.z = 0u;
            if (!i3) v.w = 0u;
            const uint32_t c0 = cls_in(v.x, i0), c1 = cls_in(v.y, i1), c2 = cls_in(v.z, i2), c3 = cls_in(v.w, i3);
            uint32_t pc = __shfl_up_sync(0xffffffffu, c3, 1);
            if (lane == 0) pc = prevc;
            const uint32_t hf = ((i0 && (c0 == C_MIXED || c0 != pc)) ? 1u : 0u) |
                                ((i1 && (c1 == C_MIXED || c1 != c0)) ? 2u : 0u) |
                                ((i2 && (c2 == C_MIXED || c2 != c1)) ? 4u : 0u) |
                                ((i3 && (c3 == C_MIXED || c3 != c2)) ? 8u : 0u);
            const uint32_t cd = hf | (c0 << 4) | (c1 << 6) | (c2 << 8) | (c3 << 10);
            *codep = cd;
            nheads += __reduce_add_sync(0xffffffffu, __popc(hf));
            const uint32_t hm = __ballot_sync(0xffffffffu, hf != 0u);
            if (hm) {
                const uint32_t hl = 31u - __clz(hm);
                const uint32_t hc = __shfl_sync(0xffffffffu, cd, hl);
                const uint32_t j = 31u - __clz(hc & 0xFu);
                lastpos = g0 + sb + 4u * hl + j;
                lastcls = (hc >> (4u + 2u * j)) & 3u;
                has = true;
            }
            prevc = __shfl_sync(0xffffffffu, c3, 31);
        }
        S.res[b][l >> 2] = v;
        popc += __popc(v.x) + __popc(v.y) + __popc(v.z) + __popc(v.w);
    }
    popc = __reduce_add_sync(0xffffffffu, popc);
    if (lane == 0) S.wagg[b][warp] = dagg_make(nheads, popc, lastpos, lastcls, has);
    bar_sync1(C::CT);  // every compute warp is done with the slot's words
    if (tid == 0) mbar_arrive(&S.empty[s]);
    if (warp == 0) {
        uint4 w = make_uint4(0u, 0u, 0u, 0u);
        if (lane < (uint32_t)NCW) w = S.wagg[b][lane];
        uint4 wi = w;
#pragma unroll
        for (int d = 1; d < NCW; d <<= 1) {
            uint4 o;
            o.x = __shfl_up_sync(0xffffffffu, wi.x, d);
            o.y = __shfl_up_sync(0xffffffffu, wi.y, d);
            o.z = __shfl_up_sync(0xffffffffu, wi.z, d);
            o.w = 0;
            if (lane >= (uint32_t)d) wi = dagg_comb(o, wi);
        }
        uint4 wx;
        wx.x = __shfl_up_sync(0xffffffffu, wi.x, 1);
        wx.y = __shfl_up_sync(0xffffffffu, wi.y, 1);
        wx.z = __shfl_up_sync(0xffffffffu, wi.z, 1);
        wx.w = 0;
        if (lane == 0) wx = make_uint4(0u, 0u, 0u, 0u);
        uint4 tot;
        tot.x = __shfl_sync(0xffffffffu, wi.x, NCW - 1);
        tot.y = __shfl_sync(0xffffffffu, wi.y, NCW - 1);
        tot.z = __shfl_sync(0xffffffffu, wi.z, NCW - 1);
        tot.w = 0;
        if (lane < (uint32_t)NCW) S.wagg[b][lane] = wx;
        if (lane == 0) {
            S.tagg[b] = tot;
            S.tinfo[b][0] = m.t; S.tinfo[b][1] = g0; S.tinfo[b][2] = ng;
            drec_publish(A.drecs, m.t, epoch, m.t == 0 ? REC_INCL : REC_AGG, tot);
        }
    }
}

// Pass 2 of the tile whose pass 1 left buffer b, with its prefix in slot p.
template <int TG, int NCW>
__device__ __forceinline__ void dense_pass2(DShared<TG, NCW>& S, const DenseArgs& A, uint32_t b, uint32_t p,
                                            uint32_t epoch) {
    using C = DCfg<TG, NCW>;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint4 prefix = S.prefix[p];
    const uint32_t t = S.tinfo[b][0], g0 = S.tinfo[b][1];
    const uint32_t G = A.groups;
    if (tid == 0) {
        const uint4 all = dagg_comb(prefix, S.tagg[b]);
        if (t > 0) drec_publish(A.drecs, t, epoch, REC_INCL, all);
        if (t == A.ntiles - 1) {
            const uint32_t n = dagg_n(all);
            if (dagg_has(all) && dagg_cls(all) != C_MIXED) {
                const uint32_t wd = run_word(dagg_cls(all), G - all.z, 0, false);
                A.out[n - 1] = wd;
                if (n - 1 == 0) A.meta->w0 = wd;
                if (is_fill(wd)) atomicOr(&A.meta->nfill, 1u);
            }
            A.obp[(n + 31u) / 32u] = G;
            A.meta->n = n;
            A.meta->groups = G;
            A.meta->nset = all.x;
            A.meta->anb = A.anb;
            A.meta->aval = A.aval;
            if (n == 0) A.meta->w0 = 0;
        }
    }
    const uint4 pre = dagg_comb(prefix, S.wagg[b][warp]);
    uint32_t idx = dagg_n(pre);                 // output index of the warp's next head
    bool lhas = dagg_has(pre);                  // the last head before the step
    uint32_t lcls = dagg_cls(pre), lpos = pre.z;
    uint32_t fill_seen = 0;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t wl0 = warp * C::GPW;
#pragma unroll
    for (int st = 0; st < C::STEPS; ++st) {
        const uint32_t sb = wl0 + st * 128u;
        const uint32_t pos0 = g0 + sb;
        const uint32_t gl = pos0 + 4u * lane;
        const uint32_t cd = S.code[b][((warp * C::STEPS + st) << 5) + lane];
        const uint4 v = S.res[b][(sb >> 2) + lane];
        if (cd == DFAST) {                      // warp-uniform: 128 mixed literals
            if (lane == 0 && lhas && lcls != C_MIXED) {
                const uint32_t wd = run_word(lcls, pos0 - lpos, 0, false);
                A.out[idx - 1] = wd;
                if (idx - 1 == 0) A.meta->w0 = wd;
                fill_seen |= is_fill(wd) ? 1u : 0u;
            }
            const uint32_t o = idx + 4u * lane;
            A.out[o] = v.x; A.out[o + 1] = v.y; A.out[o + 2] = v.z; A.out[o + 3] = v.w;
            if (o == 0) A.meta->w0 = v.x;
            const uint32_t rr = (32u - (o & 31u)) & 31u;
            if (rr < 4u) A.obp[(o + rr) >> 5] = gl + rr;
            idx += 128u;
            lhas = true; lcls = C_MIXED; lpos = pos0 + 127u;
            continue;
        }
        const uint32_t hf = cd & 0xFu;
        const uint32_t cnt = __popc(hf);
        const uint32_t b0 = __ballot_sync(0xffffffffu, cnt & 1u);
        const uint32_t b1 = __ballot_sync(0xffffffffu, cnt & 2u);
        const uint32_t b2 = __ballot_sync(0xffffffffu, cnt & 4u);
        const uint32_t ex = __popc(b0 & lt) + 2u * __popc(b1 & lt) + 4u * __popc(b2 & lt);
        const uint32_t tot = __popc(b0) + 2u * __popc(b1) + 4u * __popc(b2);
        const uint32_t hm = __ballot_sync(0xffffffffu, hf != 0u);
        uint32_t mylast = 0;                    // this lane's last head: pos << 2 | class
        if (hf) {
            const uint32_t j = 31u - __clz(hf);
            mylast = ((gl + j) << 2) | ((cd >> (4u + 2u * j)) & 3u);
        }
        const uint32_t before = hm & lt;
        const uint32_t src = before ? 31u - __clz(before) : lane;
        const uint32_t pk = __shfl_sync(0xffffffffu, mylast, src);
        bool phas = before ? true : lhas;
        uint32_t ppos = before ? (pk >> 2) : lpos;
        uint32_t pcls = before ? (pk & 3u) : lcls;
        uint32_t my = idx + ex;
        const uint32_t vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if ((hf >> j) & 1u) {
                const uint32_t pos = gl + j;
                const uint32_t c = (cd >> (4 + 2 * j)) & 3u;
                if (phas && pcls != C_MIXED) {
                    const uint32_t wd = run_word(pcls, pos - ppos, 0, false);
                    A.out[my - 1] = wd;
                    if (my - 1 == 0) A.meta->w0 = wd;
                    fill_seen |= is_fill(wd) ? 1u : 0u;
                }
                if (c == C_MIXED) {
                    A.out[my] = vv[j];
                    if (my == 0) A.meta->w0 = vv[j];
                }
                if ((my & 31u) == 0) A.obp[my >> 5] = pos;
                ++my;
                phas = true; ppos = pos; pcls = c;
            }
        }
        idx += tot;
        if (hm) {
            const uint32_t qk = __shfl_sync(0xffffffffu, mylast, 31u - __clz(hm));
            lhas = true; lpos = qk >> 2; lcls = qk & 3u;
        }
    }
    if (__any_sync(0xffffffffu, fill_seen) && lane == 0) atomicOr(&A.meta->nfill, 1u);
}

template <int OP, int TG, int NCW>
__device__ __forceinline__ void dense_compute(DShared<TG, NCW>& S, const DenseArgs& A, uint32_t epoch) {
    using C = DCfg<TG, NCW>;
    const uint32_t tid = threadIdx.x;
    volatile uint32_t* abort = &S.abort;
    volatile uint32_t* okp = &S.ok;
    uint32_t k = 0;
    bool ok = true;
    while (true) {
        const uint32_t s = k % C::NI;
        // one thread waits for the slot; the barrier hands the outcome to all
        if (tid == 0) {
            const bool w = dwait(&S.full[s], (k / C::NI) & 1u, abort);
            if (!w && !*abort) dense_fail(A, abort);
            *okp = w ? 1u : 0u;
        }
        bar_sync1(C::CT);
        if (!*okp) { ok = false; break; }
        const DSlot m = S.slot[s];
        if (m.t == DEND) break;
        dense_pass1<OP, TG, NCW>(S, A, m, s, k & 1u, epoch);
        if (k > 0) {
            const uint32_t j = k - 1;
            if (tid == 0) {
                const bool w = dwait(&S.pre[j % C::NP], (j / C::NP) & 1u, abort);
                if (!w && !*abort) dense_fail(A, abort);
                *okp = w ? 1u : 0u;
            }
            bar_sync1(C::CT);
            if (!*okp) { ok = false; break; }
            dense_pass2<TG, NCW>(S, A, j & 1u, j % C::NP, epoch);
        }
        ++k;
        bar_sync1(C::CT);  // pass 2 of k-1 done before its buffer is reused
    }
    if (ok && k > 0) {
        const uint32_t j = k - 1;
        if (tid == 0) {
            const bool w = dwait(&S.pre[j % C::NP], (j / C::NP) & 1u, abort);
            if (!w && !*abort) dense_fail(A, abort);
            *okp = w ? 1u : 0u;
        }
        bar_sync1(C::CT);
        if (*okp) dense_pass2<TG, NCW>(S, A, j & 1u, j % C::NP, epoch);
    }
}

template <int OP, int TG, int NCW>
__global__ void __launch_bounds__((NCW + 1) * 32) k_dense(DenseArgs A) {
    using C = DCfg<TG, NCW>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DShared<TG, NCW>& S = *reinterpret_cast<DShared<TG, NCW>*>(smem_raw);
    if (threadIdx.x == 0) {
        for (int i = 0; i < C::NI; ++i) { mbar_init(&S.full[i], 1); mbar_init(&S.empty[i], 1); }
        for (int i = 0; i < C::NP; ++i) mbar_init(&S.pre[i], 1);
        mbar_init_fence();
        S.epoch = ld_cg(&A.sync->epoch);
        S.abort = 0;
        S.ok = 1;
    }
    __syncthreads();
    const uint32_t epoch = S.epoch;
    if (threadIdx.x >= (uint32_t)C::CT) dense_control<TG, NCW>(S, A, epoch);
    else dense_compute<OP, TG, NCW>(S, A, epoch);
    __syncthreads();
    if (threadIdx.x == 0) finish_tile(A.sync, gridDim.x);
}

}  // namespace wah
#endif
