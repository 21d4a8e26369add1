// Two-pass group-space engine for the operators whose result compress()
// leaves canonical (the reference's _d2 / _d1 / _c1 / _c0 paths and the
// all-literal loops, src/bitvector.cpp:2545-2830, 2981-3278, 3354-3619,
// 3748-4079): after compress() the result words depend only on the result
// bits, one word per maximal run of equal all-0 / all-1 groups (a fill when
// the run holds two or more groups) and one literal per mixed group.
//
// Two launches, no look-back and no cross-CTA waits:
//  * k_gop<OP>: one warp per tile of GT = 512 groups (the stride of the
//    operands' group-tile index, which gives each tile's word range).  Both
//    operands' words over the tile are staged in shared memory at once with
//    cp.async and expanded to one 31-bit pattern per group (a word-start
//    marker per word and a warp max-scan find the word of every group, so a
//    fill costs one marker whatever its length; an operand with one word per
//    group is read directly); the result patterns R = a OP b are stored
//    densely (4 bytes per group) and the tile's run heads (a mixed group, or
//    a class change) are counted, with the first head's position and the
//    popcount.  Warps never wait for one another.
//    Each tile's totals are also added into its segment of GSEG tiles.
//  * k_gpack: one warp per tile with heads re-reads R, ranks the heads and
//    writes the words in order: a mixed head's literal, or the run word
//    whose length reaches the next head.
// Lanes own groups in NCH = 4 chunks of four consecutive groups (group
// 128*j + 4*lane + e of the tile), so every global access of R is a
// coalesced 16-byte vector and the chunk-major order is the group order.
#ifndef WAH_GOP_CUH
#define WAH_GOP_CUH
#include "wah_dense.cuh"

namespace wah {

constexpr int GT = DT;                    // groups per tile: one warp's tile (the group-tile index stride)
constexpr int GWARPS = 4;                 // warps (tiles) per CTA
constexpr int GTHREADS = GWARPS * 32;
constexpr int NCH = GT / 128;             // chunks of 128 groups (4 per lane) per tile
constexpr int GWPL = (GT + 4 + 31) / 32;  // staged words per lane
constexpr uint32_t GNONE = 0xFFFFFFFFu;   // no head in the tile
constexpr uint32_t GSEG = 256;            // tiles per segment of the two-level prefix
// staging holds a tile's <= GT words plus up to 3 before them and the
// rest of the last 16-byte chunk
static_assert(GT == NCH * 128 && NCH <= 8 && GWPL * 32 >= GT + 4 && (GWPL * 32 * 4) % 16 == 0, "tile shape");

struct GopArgs {
    const uint32_t* xw; const uint32_t* xgt; uint32_t nx;
    const uint32_t* yw; const uint32_t* ygt; uint32_t ny;
    uint32_t groups, ntiles;
    uint32_t* R;          // ntiles * GT result patterns
    uint4* tiles;         // per tile: {heads, first head (GNONE: none), popcount, -}
    uint4* segs;          // per GSEG tiles (zeroed before k_gop): {heads, GNONE - first head (0: none), popcount, -}
    uint32_t* hmask;      // per tile and lane: the lane's run heads (bit 4 j + e: group 128 j + 4 lane + e)
    uint32_t* out; uint32_t* obp; DevMeta* meta;
    uint32_t aval, anb;
};

// per warp: both operands' words over its tile and the word-start markers
struct GopWarp {
    uint32_t ws[2][GWPL * 32];
    uint16_t mk[GT];
};

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Stages words [wi0, wi0 + nw) of an n-word array w (16-byte aligned) into
// ws with both sides indexed from the 16-byte boundary a0 = wi0 & ~3:
// ws[i] = w[a0 + i], so word wi0 + k lands at ws[k + (wi0 & 3)].  Whole
// 16-byte chunks inside the array go as 16-byte copies (shared and global
// addresses both 16-byte aligned: ws is, and a0 is a multiple of 4 words),
// the at most 3 words of a chunk cut by the array's end as 4-byte ones.
__device__ __forceinline__ void gop_stage(uint32_t* ws, const uint32_t* __restrict__ w, uint32_t wi0, uint32_t nw,
                                          uint32_t n) {
    const uint32_t lane = threadIdx.x & 31u;
    if (nw == 0) return;
    const uint32_t a0 = wi0 & ~3u, end = wi0 + nw;
    const uint32_t nfull = min((end - a0 + 3u) / 4u, (n - a0) / 4u);
    for (uint32_t c = lane; c < nfull; c += 32) cp_async16(ws + 4u * c, w + a0 + 4u * c);
    for (uint32_t i = a0 + 4u * nfull + lane; i < end; i += 32) cp_async4(ws + (i - a0), w + i);
}

// Word range of one operand over the tile [g0, g1): words [wi0, wend), the
// first starting at group s0.  gt: the operand's group-tile index (entry
// past the end = (n, G)).  Returns false for words the metadata scan would
// have rejected (a tile word count that cannot be).
__device__ __forceinline__ bool gop_range(const uint32_t* __restrict__ gt, uint32_t n, uint32_t g0, uint32_t g1,
                                          uint32_t& wi0, uint32_t& s0, uint32_t& nw) {
    const uint32_t e0 = g0 / DT, e1 = (g1 + DT - 1) / DT;
    wi0 = __ldg(gt + 2 * e0); s0 = __ldg(gt + 2 * e0 + 1);
    const uint32_t wi1 = __ldg(gt + 2 * e1), s1 = __ldg(gt + 2 * e1 + 1);
    // the word covering g1 belongs to the tile when it starts before g1
    const uint32_t wend = (wi1 < n && s1 < g1) ? wi1 + 1u : wi1;
    nw = wend - wi0;
    const bool ok = wi0 < n && wend <= n && wend > wi0 && nw <= (uint32_t)GT && !(g0 > 0 && s0 >= g0 && wi0 == 0);
    if (!ok) nw = 0;
    return ok;
}

// Places one operand's staged words: marks, at the first group of the tile
// each word covers, the word's index + 1.  mk must be zero.  The words are
// taken 32 at a time, one per lane; a row of literals needs no scan.
__device__ __forceinline__ void gop_mark(const uint32_t* ws, uint16_t* mk, uint32_t nw, uint32_t s0, uint32_t g0,
                                         uint32_t g1) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t carry = s0;  // first group of the row's first word
    for (uint32_t base = 0; base < nw; base += 32) {
        const uint32_t k = base + lane;
        const bool in = k < nw;
        const uint32_t wd = in ? ws[k] : 0u;
        uint32_t p, c = 1;
        if (__ballot_sync(0xffffffffu, in && is_fill(wd)) == 0u) {
            p = carry + lane;
            carry += min(32u, nw - base);
        } else {
            c = in ? wgroups(wd) : 0u;
            uint32_t x = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, x, d);
                if (lane >= (uint32_t)d) x += t;
            }
            p = carry + x - c;
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
        if (in && p < g1 && p + c > g0) mk[max(p, g0) - g0] = (uint16_t)(k + 1u);
    }
}

// Patterns of chunk j (groups 128*j + 4*lane + e of the tile) of an impure
// operand; carry = the last word index + 1 seen before the chunk (markers,
// word index + 1 at a word's first group, grow with the group).
__device__ __forceinline__ uint4 gop_chunk(const uint32_t* ws, const uint16_t* mk, uint32_t j, uint32_t& carry) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint2 m = reinterpret_cast<const uint2*>(mk)[32 * j + lane];
    const uint32_t r0 = m.x & 0xFFFFu, r1 = max(r0, m.x >> 16), r2 = max(r1, m.y & 0xFFFFu), r3 = max(r2, m.y >> 16);
    // markers grow with the group, so the largest one before this lane is
    // the last one of the nearest lower lane holding any
    const uint32_t nz = __ballot_sync(0xffffffffu, r3 != 0u);
    const uint32_t below = nz & ((1u << lane) - 1u);
    const uint32_t lo = __shfl_sync(0xffffffffu, r3, below ? 31u - __clz(below) : lane);
    const uint32_t hi = __shfl_sync(0xffffffffu, r3, nz ? 31u - __clz(nz) : 0u);
    const uint32_t ex = below ? lo : carry;
    if (nz) carry = hi;
    const uint32_t i0 = max(ex, r0), i1 = max(ex, r1), i2 = max(ex, r2), i3 = max(ex, r3);  // >= 1 inside the tile
    return make_uint4(wpattern(ws[i0 ? i0 - 1u : 0u]), wpattern(ws[i1 ? i1 - 1u : 0u]),
                      wpattern(ws[i2 ? i2 - 1u : 0u]), wpattern(ws[i3 ? i3 - 1u : 0u]));
}

// Staged words 4 q .. 4 q + 3: one 16-byte read when the base is 16-byte
// aligned (al, warp-uniform), else four.
__device__ __forceinline__ uint4 gop_ld4(const uint32_t* ws, uint32_t q, bool al) {
    if (al) return reinterpret_cast<const uint4*>(ws)[q];
    return make_uint4(ws[4u * q], ws[4u * q + 1u], ws[4u * q + 2u], ws[4u * q + 3u]);
}

// Result patterns of one warp's tile [g0, g1) of x OP y: both operands'
// words over the tile are staged in shared memory at once with cp.async and
// expanded to one 31-bit pattern per group (a word-start marker per word
// and a warp max-scan find the word of every group, so a fill costs one
// marker whatever its length; an operand with one word per group is read
// directly).  Calls f(j, r) for the chunks j = 0..7 in order, r holding the
// results of groups 128 j + 4 lane + e of the tile (e = 0..3; groups past
// g1 hold whatever the zero-padded words give and must be ignored).  prev
// is set to the result of group g0 - 1 (0 for g0 = 0).  Returns false for a
// word range the metadata scan would have rejected (the patterns are then
// meaningless).
template <int OP, class F>
__device__ __forceinline__ bool gop_tile(const uint32_t* __restrict__ xw, const uint32_t* __restrict__ xgt,
                                         uint32_t nx, const uint32_t* __restrict__ yw,
                                         const uint32_t* __restrict__ ygt, uint32_t ny, GopWarp& W, uint32_t g0,
                                         uint32_t g1, uint32_t& prev, F&& f) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t ng = g1 - g0;
    uint32_t xi0, xs0, xn, yi0, ys0, yn;
    const bool ok = gop_range(xgt, nx, g0, g1, xi0, xs0, xn) & gop_range(ygt, ny, g0, g1, yi0, ys0, yn);
    // both operands' words in flight at once; word k of the tile at wsx[k]
    gop_stage(W.ws[0], xw, xi0, xn, nx);
    gop_stage(W.ws[1], yw, yi0, yn, ny);
    const uint32_t* wsx = W.ws[0] + (xi0 & 3u);
    const uint32_t* wsy = W.ws[1] + (yi0 & 3u);
    const bool xpure = xs0 == g0 && xn == ng, ypure = ys0 == g0 && yn == ng;
    // the result before the tile (the words covering g0 - 1)
    prev = 0;
    if (g0 > 0 && ok) {
        const uint32_t xp = __ldg(xw + (xs0 < g0 ? xi0 : xi0 - 1u));
        const uint32_t yp = __ldg(yw + (ys0 < g0 ? yi0 : yi0 - 1u));
        prev = op2<OP>(wpattern(xp), wpattern(yp));
    }
    cp_async_wait_all();
    __syncwarp();
    uint32_t xc = 0, yc = 0;
    // an impure operand is placed first (its markers then its patterns);
    // two impure operands share the marker array one after the other, so
    // the second one's patterns are read in a second sweep
    const bool both = !xpure && !ypure;
    uint4 xb[NCH];
    if (!xpure) {
        reinterpret_cast<uint2*>(W.mk)[lane] = make_uint2(0u, 0u);
#pragma unroll
        for (int j = 1; j < NCH; ++j) reinterpret_cast<uint2*>(W.mk)[32 * j + lane] = make_uint2(0u, 0u);
        __syncwarp();
        gop_mark(wsx, W.mk, xn, xs0, g0, g1);
        __syncwarp();
        if (both) {
#pragma unroll
            for (int j = 0; j < NCH; ++j) xb[j] = gop_chunk(wsx, W.mk, j, xc);
            __syncwarp();
#pragma unroll
            for (int j = 0; j < NCH; ++j) reinterpret_cast<uint2*>(W.mk)[32 * j + lane] = make_uint2(0u, 0u);
            __syncwarp();
        }
    }
    if (!ypure) {
        if (xpure) {
#pragma unroll
            for (int j = 0; j < NCH; ++j) reinterpret_cast<uint2*>(W.mk)[32 * j + lane] = make_uint2(0u, 0u);
            __syncwarp();
        }
        if (xpure || both) {
            gop_mark(wsy, W.mk, yn, ys0, g0, g1);
            __syncwarp();
        }
    }
#pragma unroll
    for (int j = 0; j < NCH; ++j) {
        uint4 a, b;
        if (xpure) a = pattern4(gop_ld4(wsx, 32 * j + lane, (xi0 & 3u) == 0u));
        else if (both) a = xb[j];
        else a = gop_chunk(wsx, W.mk, j, xc);
        if (ypure) b = pattern4(gop_ld4(wsy, 32 * j + lane, (yi0 & 3u) == 0u));
        else b = gop_chunk(wsy, W.mk, j, yc);
        f(j, make_uint4(op2<OP>(a.x, b.x), op2<OP>(a.y, b.y), op2<OP>(a.z, b.z), op2<OP>(a.w, b.w)));
    }
    return ok;
}

template <int OP>
__global__ void __launch_bounds__(GTHREADS, 10) k_gop(GopArgs A) {
    extern __shared__ __align__(16) unsigned char gsm[];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t t = blockIdx.x * GWARPS + warp;
    if (t >= A.ntiles) return;
    GopWarp& W = reinterpret_cast<GopWarp*>(gsm)[warp];
    const uint32_t G = A.groups;
    const uint32_t g0 = t * (uint32_t)GT, g1 = min(g0 + (uint32_t)GT, G);
    const uint32_t ng = g1 - g0;
    uint32_t* R = A.R + g0;
    uint32_t heads = 0, first = GNONE, popc = 0, hm = 0;
    uint32_t before;  // the result of the group before the current chunk
    const bool ok = gop_tile<OP>(A.xw, A.xgt, A.nx, A.yw, A.ygt, A.ny, W, g0, g1, before, [&](int j, uint4 r) {
        reinterpret_cast<uint4*>(R)[32 * j + lane] = r;
        uint32_t pb = __shfl_up_sync(0xffffffffu, r.w, 1);
        if (lane == 0) pb = before;
        before = __shfl_sync(0xffffffffu, r.w, 31);
        const uint32_t rv[4] = {r.x, r.y, r.z, r.w};
        uint32_t pc = cls_of(pb);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const uint32_t pos = 128u * j + 4u * lane + e;
            const uint32_t c = cls_of(rv[e]);
            if (pos < ng) {
                if ((g0 + pos == 0u) || c == C_MIXED || c != pc) {
                    ++heads;
                    first = min(first, g0 + pos);
                    hm |= 1u << (4 * j + e);
                }
                popc += __popc(rv[e]);
            }
            pc = c;
        }
    });
    A.hmask[(size_t)t * 32u + lane] = hm;
    if (!ok && lane == 0) atomicExch(&A.meta->status, DEV_ERR_FORMAT);
    heads = __reduce_add_sync(0xffffffffu, heads);
    popc = __reduce_add_sync(0xffffffffu, popc);
    first = __reduce_min_sync(0xffffffffu, first);
    if (lane == 0) {
        A.tiles[t] = make_uint4(heads, first, popc, 0u);
        uint4* sg = A.segs + t / GSEG;
        if (heads) atomicAdd(&sg->x, heads);
        if (first != GNONE) atomicMax(&sg->y, GNONE - first);
        if (popc) atomicAdd(&sg->z, popc);
    }
}

// The words of one tile per warp, in order (tiles without heads have none).
// The tile's first output index is the heads of the segments before its own
// plus those of the tiles before it in its segment; the head after the tile
// is the first head of the later tiles of its segment, else of the first
// later segment holding one.  A head's word needs the next head's position:
// the lanes find it with a suffix minimum over the lanes after them, chunks
// taken last to first.  The warp of the last tile writes the metadata.
__global__ void __launch_bounds__(GTHREADS) k_gpack(GopArgs A) {
    // this tile's words, from the 16-byte boundary at or below its first
    // output index (a tile holds at most GT heads, so GT + 3 slots)
    __shared__ __align__(16) uint32_t sout[GWARPS][GT + 4];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t t = blockIdx.x * GWARPS + warp;
    const uint32_t T = A.ntiles;
    if (t >= T) return;
    const uint32_t G = A.groups;
    // the tile's result patterns and head masks, loaded first so their
    // round trip overlaps the prefix and next-head loads below
    const uint32_t g0 = t * (uint32_t)GT;
    const uint4* R4 = reinterpret_cast<const uint4*>(A.R + g0);
    const uint32_t hm = A.hmask[(size_t)t * 32u + lane];
    uint4 rqs[NCH];
#pragma unroll
    for (int j = 0; j < NCH; ++j) rqs[j] = R4[32 * j + lane];
    const uint32_t sg = t / GSEG, nseg = (T + GSEG - 1) / GSEG;
    uint32_t off = 0;
    for (uint32_t i = lane; i < sg; i += 32) off += A.segs[i].x;
    // the tiles before this one in its segment: at most GSEG / 32 per lane,
    // loaded together
#pragma unroll
    for (uint32_t k = 0; k < GSEG / 32u; ++k) {
        const uint32_t i = sg * GSEG + lane + 32u * k;
        if (i < t) off += A.tiles[i].x;
    }
    off = __reduce_add_sync(0xffffffffu, off);
    const uint32_t cnt = A.tiles[t].x;
    if (t == T - 1) {
        uint32_t ones = 0;
        for (uint32_t i = lane; i < nseg; i += 32) ones += A.segs[i].z;
        ones = __reduce_add_sync(0xffffffffu, ones);
        if (lane == 0) {
            const uint32_t n = off + cnt;
            A.obp[(n + 31u) / 32u] = G;
            A.meta->n = n;
            A.meta->groups = G;
            A.meta->nset = ones;
            A.meta->anb = A.anb;
            A.meta->aval = A.aval;
            if (n == 0) A.meta->w0 = 0;
        }
    }
    if (cnt == 0) return;
    uint32_t nxt = GNONE;
    for (uint32_t i0 = t + 1; i0 < min(T, (sg + 1) * GSEG) && nxt == GNONE; i0 += 32) {
        const uint32_t i = i0 + lane;
        const uint32_t v = i < min(T, (sg + 1) * GSEG) ? A.tiles[i].y : GNONE;
        nxt = __reduce_min_sync(0xffffffffu, v);
    }
    for (uint32_t i0 = sg + 1; i0 < nseg && nxt == GNONE; i0 += 32) {
        const uint32_t i = i0 + lane;
        const uint32_t v = i < nseg ? A.segs[i].y : 0u;
        const uint32_t f = __reduce_max_sync(0xffffffffu, v);
        if (f) nxt = GNONE - f;
    }
    if (nxt == GNONE) nxt = G;
    // hm: the lane's heads as k_gop found them (bit 4 j + e for group 128 j + 4 lane + e)
    uint32_t* so = sout[warp];
    const uint32_t oal = off & ~3u;
    const uint32_t gt = (2u << lane) - 1u;  // lanes up to this one (lane 31: all)
    uint32_t later = nxt;  // the first head after the chunk
    uint32_t rest = cnt;   // heads in the chunks before and at the current one
    bool fill = false;
#pragma unroll
    for (int j = NCH - 1; j >= 0; --j) {
        const uint32_t m = (hm >> (4 * j)) & 15u;
        const uint32_t hl = __ballot_sync(0xffffffffu, m != 0u);
        if (hl == 0u) continue;  // a chunk inside a run
        // heads of the lanes before this one, from the bits of each lane's
        // count (0..4); the chunk's own count
        const uint32_t nh = __popc(m);
        const uint32_t c0 = __ballot_sync(0xffffffffu, nh & 1u);
        const uint32_t c1 = __ballot_sync(0xffffffffu, nh & 2u);
        const uint32_t c2 = __ballot_sync(0xffffffffu, nh & 4u);
        rest -= __popc(c0) + 2u * __popc(c1) + 4u * __popc(c2);
        const uint32_t lt = gt >> 1;  // lanes before this one
        uint32_t o = off + rest + __popc(c0 & lt) + 2u * __popc(c1 & lt) + 4u * __popc(c2 & lt);
        // the head after this lane's last one: the first head of the
        // nearest higher lane holding one, else the first after the chunk
        const uint32_t g = g0 + 128u * j + 4u * lane;
        const uint32_t mine = m ? g + (__ffs(m) - 1u) : GNONE;
        const uint32_t above = hl & ~gt;
        const uint32_t nl = __shfl_sync(0xffffffffu, mine, above ? __ffs(above) - 1u : lane);
        const uint32_t after = above ? nl : later;
        later = __shfl_sync(0xffffffffu, mine, __ffs(hl) - 1u);
        if (m) {
            const uint4 rq = rqs[j];
            const uint32_t r[4] = {rq.x, rq.y, rq.z, rq.w};
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if ((m >> e) & 1u) {
                    const uint32_t more = m >> (e + 1);
                    const uint32_t next = more ? g + e + __ffs(more) : after;
                    const uint32_t wd = run_word(cls_of(r[e]), next - (g + e), r[e], false);
                    so[o - oal] = wd;
                    if ((o & 31u) == 0u) A.obp[o >> 5] = g + e;
                    if (o == 0u) A.meta->w0 = wd;
                    fill |= is_fill(wd);
                    ++o;
                }
        }
    }
    if (__any_sync(0xffffffffu, fill) && lane == 0) atomicOr(&A.meta->nfill, 1u);
    // the tile's words leave as 16-byte stores (the output array is a pool
    // block, 16-byte aligned), the ragged ends word by word
    __syncwarp();
    const uint32_t end = off + cnt;
    for (uint32_t v = lane; 4u * v < end - oal; v += 32u) {
        const uint32_t gi = oal + 4u * v;
        if (gi >= off && gi + 4u <= end) {
            *reinterpret_cast<uint4*>(A.out + gi) = *reinterpret_cast<const uint4*>(so + 4u * v);
        } else {
#pragma unroll
            for (uint32_t e = 0; e < 4u; ++e)
                if (gi + e >= off && gi + e < end) A.out[gi + e] = so[4u * v + e];
        }
    }
}

}  // namespace wah
#endif
