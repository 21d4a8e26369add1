// The merge kernel: one launch computes  x OP y  (or a copy / complemented
// copy of x) over two WAH word streams and writes the words the reference
// holds after compress(), plus the result's block-position index and
// metadata.
//
// Work split.  Every operand carries a block-position index bpos[k] = group
// position where word 32k starts (bpos[nblocks] = total groups).  The CTA for
// tile t takes the t-th run of TILE_BLOCKS entries of the sorted union of the
// two indexes (a merge path over bpos arrays only, found with a 32-way warp
// search), so each CTA gets a group interval [Pa, Pb) holding at most
// 32*(TILE_BLOCKS+2) words of both operands.  Both Pa and Pb are word
// boundaries of one operand, hence segment boundaries.
//
// Segments.  Inside the tile the word ends of x and y are merged again (per
// thread, in shared memory); each gap between consecutive word ends is a
// segment covered by one x word and one y word: its result is either a run
// of equal all-0/all-1 groups or one mixed literal group.
//
// Encoding.  Result words are maximal runs (wah_core.cuh).  A run's word is
// written by the thread that meets the next run head (its length is only
// known then); mixed literals are written at once.  Head counts, the last
// head, popcounts and the step-state transfer function are carried across
// tiles by a single-pass decoupled look-back over TileRec records.
#ifndef WAH_MERGE_CUH
#define WAH_MERGE_CUH
#include "wah_dev.cuh"

namespace wah {

#ifndef WAH_MERGE_THREADS
#define WAH_MERGE_THREADS 256
#endif
constexpr int MERGE_THREADS = WAH_MERGE_THREADS;
// Tile shape: TB bpos entries per tile (16, 32 or 64: WAHGPU_TUNE_MERGE_TILE;
// small tiles give small operands more CTAs and each a shorter chain).
template <int TB>
struct MCfg {
    static constexpr int TILE_BLOCKS = TB;
    static constexpr int TILE_WORDS = 32 * (TB + 2);  // max words held per operand
    // events per thread: a tile holds at most TILE_WORDS words of both operands together
    static constexpr int SEG_PER_THREAD = (TILE_WORDS + MERGE_THREADS - 1) / MERGE_THREADS;
};

struct MergeArgs {
    const uint32_t* xw;   // lhs words
    const uint32_t* xbp;  // lhs block positions (nbx + 1 entries)
    const uint32_t* yw;
    const uint32_t* ybp;
    uint32_t nx, nbx, ny, nby;
    uint32_t groups;
    uint32_t* out;        // result words (capacity nx + ny)
    uint32_t* obp;        // result block positions
    DevMeta* meta;        // result metadata
    TileRec* recs;
    LaunchSync* sync;
    uint32_t ntiles;
    uint32_t aval, anb;   // result active word (already combined)
};

// Look-back aggregate: heads, last head (position, class, count-1 flag for
// each of the 5 possible incoming step states), popcount, transfer function.
struct Agg {
    uint32_t nheads, pos, info, popc;
};
__device__ __forceinline__ uint32_t agg_cls(uint32_t info) { return info & 3u; }
__device__ __forceinline__ bool agg_has(uint32_t info) { return (info >> 2) & 1u; }
__device__ __forceinline__ uint32_t agg_fmask(uint32_t info) { return (info >> 3) & 31u; }
__device__ __forceinline__ uint32_t agg_fsm(uint32_t info) { return (info >> 8) & 0x7FFFu; }
__device__ __forceinline__ uint32_t mk_info(uint32_t cls, bool has, uint32_t fmask, uint32_t fsm) {
    return cls | (has ? 4u : 0u) | (fmask << 3) | (fsm << 8);
}
__device__ __forceinline__ Agg agg_identity() {
    Agg a; a.nheads = 0; a.pos = 0; a.popc = 0; a.info = mk_info(0, false, 0, FSM_IDENTITY);
    return a;
}
// a followed by b
template <bool FSM>
__device__ __forceinline__ Agg agg_combine(const Agg& a, const Agg& b) {
    Agg r;
    r.nheads = a.nheads + b.nheads;
    r.popc = a.popc + b.popc;
    uint32_t fa = agg_fsm(a.info), fb = agg_fsm(b.info);
    uint32_t f = FSM ? fsm_compose(fa, fb) : FSM_IDENTITY;
    if (agg_has(b.info)) {
        r.pos = b.pos;
        // the last head's flags are indexed by the state entering b; seen
        // from the start of a they are re-indexed through a's transfer.
        // Without step states (copy / canonical modes) they do not depend
        // on the state.
        uint32_t bm = agg_fmask(b.info), m = bm;
        if (FSM) {
            m = 0;
#pragma unroll
            for (uint32_t s = 0; s < 5; ++s) m |= ((bm >> fsm_apply(fa, s)) & 1u) << s;
        }
        r.info = mk_info(agg_cls(b.info), true, m, f);
    } else {
        r.pos = a.pos;
        r.info = mk_info(agg_cls(a.info), agg_has(a.info), agg_fmask(a.info), f);
    }
    return r;
}
__device__ __forceinline__ uint4 agg_pack(const Agg& a) { return make_uint4(a.nheads, a.pos, a.info, a.popc); }
__device__ __forceinline__ Agg agg_unpack(uint4 v) { Agg a; a.nheads = v.x; a.pos = v.y; a.info = v.z; a.popc = v.w; return a; }

template <bool FSM>
struct AggComb {
    __device__ __forceinline__ uint4 operator()(uint4 a, uint4 b) const {
        return agg_pack(agg_combine<FSM>(agg_unpack(a), agg_unpack(b)));
    }
};

template <bool FSM>
__device__ __forceinline__ Agg agg_shfl_up(const Agg& a, int d) {
    Agg r;
    r.nheads = __shfl_up_sync(0xffffffffu, a.nheads, d);
    r.pos = __shfl_up_sync(0xffffffffu, a.pos, d);
    r.info = __shfl_up_sync(0xffffffffu, a.info, d);
    r.popc = __shfl_up_sync(0xffffffffu, a.popc, d);
    return r;
}

// Smallest m in [lo, hi] with !(a[m] <= b[d-1-m]) : the number of entries
// of `a` among the first d of merge(a, b) (ties: a first).  Whole warp.
__device__ __forceinline__ uint32_t warp_merge_split(const uint32_t* a, uint32_t na,
                                                     const uint32_t* b, uint32_t nb, uint32_t d) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t lo = d > nb ? d - nb : 0u;
    uint32_t hi = d < na ? d : na;
    while (lo < hi) {
        const uint32_t span = hi - lo;
        const uint32_t step = (span + 31u) / 32u;
        const uint32_t m = lo + lane * step;
        bool p = false;
        if (m < hi) p = __ldg(a + m) <= __ldg(b + (d - 1u - m));
        const uint32_t bal = __ballot_sync(0xffffffffu, p);
        const uint32_t k = __popc(bal);  // predicate is monotone: leading trues
        const uint32_t nlo = k > 0 ? lo + (k - 1u) * step + 1u : lo;
        uint32_t nhi = hi;
        if (k < 32u && lo + k * step < hi) nhi = lo + k * step;
        lo = nlo;
        hi = nhi < lo ? lo : nhi;
        if (step == 1u) break;  // exact in one round
    }
    return lo;
}

template <int TB>
struct TileShared {
    uint32_t wx[MCfg<TB>::TILE_WORDS];
    uint32_t ex[MCfg<TB>::TILE_WORDS];  // end position of each held x word
    uint32_t wy[MCfg<TB>::TILE_WORDS];
    uint32_t ey[MCfg<TB>::TILE_WORDS];
    uint32_t warp_agg[MERGE_THREADS / 32][4];
    uint32_t tile_prefix[4];
    uint32_t hdr[16];  // tile geometry broadcast
    // seg_transfer for every (step, xb, yb, fits_x, fits_y): entry
    // 16 * step + 8 xb + 4 yb + 2 fits_x + fits_y
    uint32_t trans_tab[80];
};

// Starts copying words [g0, g1) of an operand into shared memory (128-bit
// loads: g0 is 32-word aligned, buffers are 256-byte aligned).  The caller
// waits with a block barrier before reading sw.
__device__ __forceinline__ void load_words(const uint32_t* __restrict__ w, uint32_t g0, uint32_t g1, uint32_t* sw) {
    const uint32_t n = g1 - g0;
    const uint32_t n4 = n / 4u;
    const uint4* w4 = reinterpret_cast<const uint4*>(w + g0);
    for (uint32_t i = threadIdx.x; i < n4; i += MERGE_THREADS) {
        uint4 v = __ldg(w4 + i);
        reinterpret_cast<uint4*>(sw)[i] = v;
    }
    for (uint32_t i = n4 * 4u + threadIdx.x; i < n; i += MERGE_THREADS) sw[i] = __ldg(w + g0 + i);
}

// End position of each staged word from the block positions: one warp per
// 32-word block, inclusive scan of the group counts.  bpv[r] holds the
// block position of block warp + r * (MERGE_THREADS / 32), loaded before the
// barrier that made sw readable (so its latency overlaps the word loads).
template <int NR>
__device__ __forceinline__ void word_ends(const uint32_t* sw, uint32_t* se, uint32_t n, const uint32_t (&bpv)[NR]) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t nblk = (n + 31u) / 32u;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const uint32_t b = warp + (uint32_t)r * (MERGE_THREADS / 32);
        if (b >= nblk) break;
        const uint32_t i = b * 32u + lane;
        uint32_t c = i < n ? wgroups(sw[i]) : 0u;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, c, d);
            if (lane >= (uint32_t)d) c += t;
        }
        if (i < n) se[i] = bpv[r] + c;
    }
}
// Block positions for word_ends (lane values; every lane loads the same entry).
template <int NR>
__device__ __forceinline__ void load_bpos(const uint32_t* __restrict__ bp, uint32_t g0, uint32_t n, uint32_t (&bpv)[NR]) {
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t nblk = (n + 31u) / 32u;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const uint32_t b = warp + (uint32_t)r * (MERGE_THREADS / 32);
        bpv[r] = b < nblk ? __ldg(bp + (g0 / 32u) + b) : 0u;
    }
}

// First index in se[0..n) with se[i] > p (se ascending).
__device__ __forceinline__ uint32_t first_end_after(const uint32_t* se, uint32_t n, uint32_t p) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) { uint32_t m = (lo + hi) >> 1; if (se[m] > p) hi = m; else lo = m + 1; }
    return lo;
}

// Segment record kept in registers between the two passes.
struct SegRec {
    uint32_t pos, val, bits;  // bits: trans(20) | cls<<20 | head<<22 | xfill<<23 | yfill<<24
};

template <int OP, bool FSM, bool UNARY, bool FLIP, int TB>
__global__ void __launch_bounds__(MERGE_THREADS, 2) k_merge(MergeArgs A) {
    constexpr int TILE_BLOCKS = TB, SEG_PER_THREAD = MCfg<TB>::SEG_PER_THREAD;
    using TileShared = wah::TileShared<TB>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TileShared& S = *reinterpret_cast<TileShared*>(smem_raw);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;

    // ---- claim a tile and read the launch epoch (two threads, so the two
    // round trips overlap; the epoch only changes after the last CTA of the
    // previous launch on this stream finished)
    if (tid == 0) S.hdr[0] = claim_tile(A.sync);
    if (tid == 32) S.hdr[1] = ld_cg(&A.sync->epoch);
    if (FSM && tid >= 64 && tid < 64 + 80) {
        const uint32_t e = tid - 64;
        S.trans_tab[e] = seg_transfer(e >> 4, (e >> 3) & 1u, (e >> 2) & 1u, (e >> 1) & 1u, e & 1u);
    }
    __syncthreads();
    const uint32_t t = S.hdr[0];
    const uint32_t epoch = S.hdr[1];
    const uint32_t G = A.groups;

    // ---- tile geometry
    if (UNARY) {
        if (tid == 0) {
            uint32_t k0 = t * TILE_BLOCKS, k1 = min(k0 + TILE_BLOCKS, A.nbx);
            k0 = min(k0, A.nbx);
            S.hdr[2] = __ldg(A.xbp + k0);         // Pa
            S.hdr[3] = __ldg(A.xbp + k1);         // Pb
            S.hdr[4] = k0 * 32u;                  // x word range
            S.hdr[5] = min(k1 * 32u, A.nx);
            S.hdr[6] = 0; S.hdr[7] = 0;
        }
    } else if (warp < 2) {
        const uint32_t dtot = A.nbx + A.nby;
        const uint32_t d = min((t + warp) * (uint32_t)TILE_BLOCKS, dtot);
        const uint32_t kx = warp_merge_split(A.xbp, A.nbx, A.ybp, A.nby, d);
        const uint32_t ky = d - kx;
        if (lane == 0) {
            const uint32_t vx = kx < A.nbx ? __ldg(A.xbp + kx) : 0xFFFFFFFFu;
            const uint32_t vy = ky < A.nby ? __ldg(A.ybp + ky) : 0xFFFFFFFFu;
            uint32_t P = min(vx, vy);
            if (P == 0xFFFFFFFFu) P = G;
            if (warp == 0) {
                S.hdr[2] = P;
                // first held block: the one containing P
                S.hdr[8] = (kx < A.nbx && vx == P) ? kx : (kx ? kx - 1 : 0);
                S.hdr[9] = (ky < A.nby && vy == P) ? ky : (ky ? ky - 1 : 0);
            } else {
                S.hdr[3] = P;
                S.hdr[10] = kx;  // blocks before the end
                S.hdr[11] = ky;
            }
        }
    }
    __syncthreads();
    const uint32_t Pa = S.hdr[2], Pb = S.hdr[3];
    uint32_t gx0, gx1, gy0 = 0, gy1 = 0;
    if (UNARY) { gx0 = S.hdr[4]; gx1 = S.hdr[5]; }
    else {
        gx0 = S.hdr[8] * 32u; gx1 = min(max(S.hdr[10], S.hdr[8] + 1u) * 32u, A.nx);
        gy0 = S.hdr[9] * 32u; gy1 = min(max(S.hdr[11], S.hdr[9] + 1u) * 32u, A.ny);
        if (Pa >= Pb) { gx1 = gx0; gy1 = gy0; }
        if (gx0 > A.nx) gx0 = gx1 = A.nx;
        if (gy0 > A.ny) gy0 = gy1 = A.ny;
    }
    const uint32_t hx = gx1 - gx0, hy = gy1 - gy0;
    // both operands' words and block positions in flight together
    constexpr int NR = (TILE_BLOCKS + 2 + MERGE_THREADS / 32 - 1) / (MERGE_THREADS / 32);
    // a tile holds at most TILE_BLOCKS + 1 blocks of an operand (the merge
    // path's TILE_BLOCKS entries and the block holding Pa); NR rows of warps
    // cover them
    static_assert(NR * (MERGE_THREADS / 32) >= TILE_BLOCKS + 2, "block-position registers");
    uint32_t bpx[NR], bpy[NR];
    load_words(A.xw, gx0, gx1, S.wx);
    if (!UNARY) load_words(A.yw, gy0, gy1, S.wy);
    load_bpos(A.xbp, gx0, hx, bpx);
    if (!UNARY) load_bpos(A.ybp, gy0, hy, bpy);
    __syncthreads();
    word_ends(S.wx, S.ex, hx, bpx);
    if (!UNARY) word_ends(S.wy, S.ey, hy, bpy);
    __syncthreads();

    // ---- events of this tile: word ends in (Pa, Pb]; four threads search
    if (tid < 4) {
        uint32_t v = 0;
        if (Pa < Pb) {
            if (tid == 0) v = first_end_after(S.ex, hx, Pa);
            else if (tid == 1) v = first_end_after(S.ex, hx, Pb);
            else if (!UNARY && tid == 2) v = first_end_after(S.ey, hy, Pa);
            else if (!UNARY && tid == 3) v = first_end_after(S.ey, hy, Pb);
        }
        S.hdr[12 + tid] = v;
    }
    __syncthreads();
    const uint32_t ix_lo = S.hdr[12], nxe = S.hdr[13] - S.hdr[12];
    const uint32_t iy_lo = S.hdr[14], nye = S.hdr[15] - S.hdr[14];
    const uint32_t E = nxe + nye;

    // ---- this thread's event range and merge split
    const uint32_t e0 = (uint32_t)(((uint64_t)E * tid) / MERGE_THREADS);
    const uint32_t e1 = (uint32_t)(((uint64_t)E * (tid + 1)) / MERGE_THREADS);
    uint32_t i = e0, j = 0;  // x events before e0, y events before e0
    if (!UNARY) {
        uint32_t lo = e0 > nye ? e0 - nye : 0u, hi = min(e0, nxe);
        while (lo < hi) {
            uint32_t m = (lo + hi) >> 1;
            if (S.ex[ix_lo + m] <= S.ey[iy_lo + e0 - 1u - m]) lo = m + 1; else hi = m;
        }
        i = lo; j = e0 - lo;
    }
    // helpers over held words; k indexes the held range
    auto xstart = [&](uint32_t k) -> uint32_t { return k < hx ? S.ex[k] - wgroups(S.wx[k]) : Pb; };
    auto ystart = [&](uint32_t k) -> uint32_t { return k < hy ? S.ey[k] - wgroups(S.wy[k]) : Pb; };
    auto xendk = [&](uint32_t k) -> uint32_t { return k < hx ? S.ex[k] : 0xFFFFFFFFu; };
    auto yendk = [&](uint32_t k) -> uint32_t { return k < hy ? S.ey[k] : 0xFFFFFFFFu; };

    // ---- pass 1: one record per event, the thread aggregate
    SegRec seg[SEG_PER_THREAD];
    Agg agg = agg_identity();
    uint32_t fsm_run = FSM_IDENTITY;
    bool has_head = false;
    uint32_t h_pre = FSM_IDENTITY, h_bits = 0;  // transfer before the last head, its bits
    {
        uint32_t pos = 0;
        uint32_t prevcls = C_NONE;
        if (e0 < e1) {
            uint32_t kx = ix_lo + i, ky = iy_lo + j;
            pos = UNARY ? xstart(kx) : max(max(xstart(kx), ystart(ky)), Pa);
            if (pos > 0) {
                // words covering pos-1: the current word if it began earlier, else the one before
                uint32_t xp, yp = 0;
                {
                    int64_t k = kx;
                    if (!(k < (int64_t)hx && xstart((uint32_t)k) < pos)) --k;
                    xp = k >= 0 ? S.wx[k] : __ldg(A.xw + gx0 - 1);
                }
                if (!UNARY) {
                    int64_t k = ky;
                    if (!(k < (int64_t)hy && ystart((uint32_t)k) < pos)) --k;
                    yp = k >= 0 ? S.wy[k] : __ldg(A.yw + gy0 - 1);
                }
                const uint32_t pv = UNARY ? (FLIP ? (wpattern(xp) ^ ALLONES) : wpattern(xp))
                                          : apply_op(OP, wpattern(xp), wpattern(yp));
                prevcls = cls_of(pv);
            }
        }
#pragma unroll
        for (int q = 0; q < SEG_PER_THREAD; ++q) {
            seg[q].bits = 0xFFFFFFFFu;  // empty
            if (e0 + q < e1) {
                const uint32_t kx = ix_lo + i, ky = iy_lo + j;
                uint32_t xw_ = kx < hx ? S.wx[kx] : 0u, yw_ = 0, segend, val;
                bool take_x = true;
                if (UNARY) {
                    segend = xendk(kx);
                    val = FLIP ? (wpattern(xw_) ^ ALLONES) : wpattern(xw_);
                } else {
                    yw_ = ky < hy ? S.wy[ky] : 0u;
                    const uint32_t xe = i < nxe ? S.ex[kx] : 0xFFFFFFFFu;
                    const uint32_t ye = j < nye ? S.ey[ky] : 0xFFFFFFFFu;
                    take_x = xe <= ye;
                    segend = take_x ? xe : ye;
                    val = apply_op(OP, wpattern(xw_), wpattern(yw_));
                }
                if (segend > pos) {
                    const uint32_t cls = cls_of(val);
                    const bool head = (cls == C_MIXED) || (cls != prevcls);
                    uint32_t trans = 0;
                    if (FSM) {
                        const uint32_t xe2 = xendk(kx), ye2 = yendk(ky);
                        const bool xb = (pos == xstart(kx)), yb = (pos == ystart(ky));
                        const uint32_t sel = select_step(OP, xw_, xe2 - pos, yw_, ye2 - pos);
                        trans = S.trans_tab[16u * sel + (xb ? 8u : 0u) + (yb ? 4u : 0u) +
                                            (xe2 <= ye2 ? 2u : 0u) + (ye2 <= xe2 ? 1u : 0u)];
                    }
                    const uint32_t len = segend - pos;
                    agg.popc += (cls == C_MIXED) ? __popc(val) : (cls == C_ONE ? len * 31u : 0u);
                    const uint32_t bits = trans | (cls << 20) | ((head ? 1u : 0u) << 22) |
                                          ((is_fill(xw_) ? 1u : 0u) << 23) | ((is_fill(yw_) ? 1u : 0u) << 24);
                    if (head) {
                        ++agg.nheads;
                        agg.pos = pos;
                        has_head = true;
                        h_pre = fsm_run;
                        h_bits = bits;
                    }
                    seg[q].pos = pos;
                    seg[q].val = val;
                    seg[q].bits = bits;
                    if (FSM) fsm_run = fsm_compose(fsm_run, trans);
                    prevcls = cls;
                    pos = segend;
                }
                if (UNARY || take_x) ++i; else ++j;
            }
        }
        // last head: class and count-1 flag for every incoming step state
        uint32_t fmask = 0;
        if (has_head) {
            if (FSM) {
                const uint32_t tr = h_bits & 0xFFFFFu;
#pragma unroll
                for (uint32_t s = 0; s < 5; ++s) {
                    const uint32_t sp = fsm_apply(h_pre, s);
                    const bool st = fsm_started(tr, sp);
                    const uint32_t sn = fsm_apply(tr, sp);
                    const bool f = seg_fill_flag(sn, st, (h_bits >> 23) & 1u ? HEADER0 | 1u : 0u,
                                                 (h_bits >> 24) & 1u ? HEADER0 | 1u : 0u);
                    fmask |= (f ? 1u : 0u) << s;
                }
            } else if (UNARY) {
                fmask = ((h_bits >> 23) & 1u) ? 31u : 0u;
            }
        }
        agg.info = mk_info(has_head ? (h_bits >> 20) & 3u : 0u, has_head, fmask, fsm_run & 0x7FFFu);
    }
    // ---- block-wide exclusive scan of the aggregates
    Agg incl = agg;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        Agg o = agg_shfl_up<FSM>(incl, d);
        if (lane >= (uint32_t)d) incl = agg_combine<FSM>(o, incl);
    }
    if (lane == 31) {
        uint4 v = agg_pack(incl);
        S.warp_agg[warp][0] = v.x; S.warp_agg[warp][1] = v.y; S.warp_agg[warp][2] = v.z; S.warp_agg[warp][3] = v.w;
    }
    Agg excl_in_warp = agg_shfl_up<FSM>(incl, 1);
    if (lane == 0) excl_in_warp = agg_identity();
    __syncthreads();
    if (warp == 0) {
        constexpr int NW = MERGE_THREADS / 32;
        // exclusive scan of the warp totals in warp 0
        Agg w = agg_identity();
        if (lane < (uint32_t)NW)
            w = agg_unpack(make_uint4(S.warp_agg[lane][0], S.warp_agg[lane][1], S.warp_agg[lane][2], S.warp_agg[lane][3]));
        Agg wi = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            Agg o = agg_shfl_up<FSM>(wi, d);
            if (lane >= (uint32_t)d) wi = agg_combine<FSM>(o, wi);
        }
        Agg wx = agg_shfl_up<FSM>(wi, 1);
        if (lane == 0) wx = agg_identity();
        const Agg tot = agg_unpack(make_uint4(__shfl_sync(0xffffffffu, wi.nheads, NW - 1),
                                              __shfl_sync(0xffffffffu, wi.pos, NW - 1),
                                              __shfl_sync(0xffffffffu, wi.info, NW - 1),
                                              __shfl_sync(0xffffffffu, wi.popc, NW - 1)));
        if (lane < (uint32_t)NW) {
            uint4 pv = agg_pack(wx);
            S.warp_agg[lane][0] = pv.x; S.warp_agg[lane][1] = pv.y; S.warp_agg[lane][2] = pv.z; S.warp_agg[lane][3] = pv.w;
        }
        // ---- decoupled look-back over the preceding tiles
        Agg prefix = agg_identity();
        if (t == 0) {
            if (lane == 0) publish(&A.recs[0], epoch, REC_INCL, agg_pack(tot));
        } else {
            if (lane == 0) publish(&A.recs[t], epoch, REC_AGG, agg_pack(tot));
            bool ok;
            prefix = agg_unpack(warp_lookback(A.recs, t, epoch, agg_pack(agg_identity()), AggComb<FSM>(), &ok));
            if (lane == 0) {
                if (!ok) atomicExch(&A.meta->status, DEV_ERR_TIMEOUT);
                publish(&A.recs[t], epoch, REC_INCL, agg_pack(agg_combine<FSM>(prefix, tot)));
            }
        }
        if (lane == 0) {
            uint4 pv = agg_pack(prefix);
            S.tile_prefix[0] = pv.x; S.tile_prefix[1] = pv.y; S.tile_prefix[2] = pv.z; S.tile_prefix[3] = pv.w;
            // the last tile finishes the result
            if (t == A.ntiles - 1) {
                Agg all = agg_combine<FSM>(prefix, tot);
                const uint32_t n = all.nheads;
                if (agg_has(all.info) && agg_cls(all.info) != C_MIXED) {
                    const bool f = (agg_fmask(all.info) & 1u) != 0;
                    const uint32_t w = run_word(agg_cls(all.info), G - all.pos, 0, f);
                    A.out[n - 1] = w;
                    if (n - 1 == 0) A.meta->w0 = w;
                    if (is_fill(w)) atomicOr(&A.meta->nfill, 1u);
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
    // ---- pass 2: emit words
    Agg tp = agg_unpack(make_uint4(S.tile_prefix[0], S.tile_prefix[1], S.tile_prefix[2], S.tile_prefix[3]));
    Agg wp = agg_unpack(make_uint4(S.warp_agg[warp][0], S.warp_agg[warp][1], S.warp_agg[warp][2], S.warp_agg[warp][3]));
    Agg pre = agg_combine<FSM>(agg_combine<FSM>(tp, wp), excl_in_warp);
    uint32_t idx = pre.nheads;
    bool lhas = agg_has(pre.info);
    uint32_t lcls = agg_cls(pre.info), lpos = pre.pos;
    bool lf = (agg_fmask(pre.info) & 1u) != 0;
    uint32_t state = fsm_apply(agg_fsm(pre.info), 0u);
    bool wrote_fill = false;
#pragma unroll
    for (int k = 0; k < SEG_PER_THREAD; ++k) {
        const SegRec& s = seg[k];
        if (s.bits == 0xFFFFFFFFu) continue;
        const uint32_t tr = s.bits & 0xFFFFFu;
        bool f = false;
        if (FSM) {
            const bool st = fsm_started(tr, state);
            state = fsm_apply(tr, state);
            f = seg_fill_flag(state, st, (s.bits >> 23) & 1u ? HEADER0 | 1u : 0u,
                              (s.bits >> 24) & 1u ? HEADER0 | 1u : 0u);
        } else if (UNARY) {
            f = (s.bits >> 23) & 1u;
        }
        if ((s.bits >> 22) & 1u) {  // head
            const uint32_t cls = (s.bits >> 20) & 3u;
            if (lhas && lcls != C_MIXED) {
                const uint32_t w = run_word(lcls, s.pos - lpos, 0, lf);
                A.out[idx - 1] = w;
                if (idx - 1 == 0) A.meta->w0 = w;
                wrote_fill |= is_fill(w);
            }
            if (cls == C_MIXED) {
                A.out[idx] = s.val;
                if (idx == 0) A.meta->w0 = s.val;
            }
            if ((idx & 31u) == 0) A.obp[idx >> 5] = s.pos;
            ++idx;
            lhas = true; lcls = cls; lpos = s.pos; lf = f;
        }
    }
    if (wrote_fill) atomicOr(&A.meta->nfill, 1u);
    __syncthreads();
    if (tid == 0) finish_tile(A.sync, A.ntiles);
}

}  // namespace wah
#endif
