// Per-word scan kernels: the upload scan (validates serialized words and
// builds the block-position index and metadata), row-id extraction, the
// decompress expansion, and the one-thread kernel for results that are a
// single word or none.
#ifndef WAH_KERNELS_CUH
#define WAH_KERNELS_CUH
#include "wah_dev.cuh"

namespace wah {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_WPT = 16;                              // words per thread
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_WPT;        // 4096 words, 128 blocks

// Upload scan: for words w[0..n) writes bpos[k] (k = 0..ceil(n/32)) and
// meta {n, groups, nset, w0, nfill, status}.  A count-0 fill word is a
// format error; more than 2^32-1 bits is a range error (the reference keeps
// the bit count in a 32-bit word).
__global__ void __launch_bounds__(SCAN_THREADS)
k_meta(const uint32_t* __restrict__ w, uint32_t n, uint32_t* __restrict__ bpos, DevMeta* meta,
       uint32_t anb, uint32_t aval, TileRec* recs, LaunchSync* sync, uint32_t ntiles) {
    __shared__ uint64_t sh[SCAN_THREADS / 32 + 1];
    __shared__ uint32_t hdr[2];
    __shared__ uint32_t tile_pre[4];
    if (threadIdx.x == 0) { hdr[0] = claim_tile(sync); hdr[1] = ld_cg(&sync->epoch); }
    __syncthreads();
    const uint32_t t = hdr[0], epoch = hdr[1];
    const uint32_t base = t * SCAN_TILE + threadIdx.x * SCAN_WPT;
    uint64_t groups = 0;
    uint32_t ones = 0, fills = 0, bad = 0;
#pragma unroll
    for (int q = 0; q < SCAN_WPT; q += 4) {
        uint32_t v[4];
        if (base + q + 3 < n) {
            uint4 x = __ldg(reinterpret_cast<const uint4*>(w + base + q));
            v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
        } else {
#pragma unroll
            for (int r = 0; r < 4; ++r) v[r] = (base + q + r < n) ? __ldg(w + base + q + r) : 0u;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            if (base + q + r < n) {
                const uint32_t x = v[r];
                if (x > ALLONES) {
                    const uint32_t c = x & MAXCNT;
                    groups += c;
                    if (x >= HEADER1) ones += c * 31u;
                    fills = 1;
                    if (c == 0) bad = 1;
                } else {
                    groups += 1;
                    ones += __popc(x);
                }
            }
        }
    }
    uint64_t total;
    const uint64_t ex = block_exscan64(groups, sh, total);
    // popcount and flags: block reduction through the same shared buffer
    __syncthreads();
    uint32_t o = ones, f = fills | (bad << 1);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) { o += __shfl_down_sync(0xffffffffu, o, d); f |= __shfl_down_sync(0xffffffffu, f, d); }
    __shared__ uint32_t sh_o[SCAN_THREADS / 32], sh_f[SCAN_THREADS / 32];
    if ((threadIdx.x & 31u) == 0) { sh_o[threadIdx.x >> 5] = o; sh_f[threadIdx.x >> 5] = f; }
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t to = 0, tf = 0;
        for (int k = 0; k < SCAN_THREADS / 32; ++k) { to += sh_o[k]; tf |= sh_f[k]; }
        uint64_t prefix; uint32_t po, pf;
        bool ok = lookback64(recs, t, epoch, total, to, tf, prefix, po, pf);
        if (threadIdx.x != 0) goto meta_done;
        if (!ok) atomicExch(&meta->status, DEV_ERR_TIMEOUT);
        tile_pre[0] = (uint32_t)prefix; tile_pre[1] = (uint32_t)(prefix >> 32);
        if (t == ntiles - 1) {
            const uint64_t g = prefix + total;
            const uint32_t flags = pf | tf;
            meta->n = n;
            meta->groups = (uint32_t)g;
            meta->nset = po + to;
            meta->nfill = flags & 1u;
            meta->anb = anb;
            meta->aval = aval;
            meta->w0 = n ? __ldg(w) : 0u;
            if (flags & 2u) atomicExch(&meta->status, DEV_ERR_FORMAT);
            else if (g * 31u + anb > 0xFFFFFFFFull) atomicExch(&meta->status, DEV_ERR_RANGE);
            bpos[(n + 31u) / 32u] = (uint32_t)g;
        }
    }
meta_done:
    __syncthreads();
    const uint64_t pre = ((uint64_t)tile_pre[1] << 32 | tile_pre[0]) + ex;
    if ((threadIdx.x & 1u) == 0 && base < n) bpos[base / 32u] = (uint32_t)pre;
    __syncthreads();
    if (threadIdx.x == 0) finish_tile(sync, ntiles);
}

// Results that are a single word or none (one-group and zero-group
// operands, and the single 0-fill of `a - b` when b is all ones).
//   mode 0: EMPTY   no words
//   mode 1: RAW1    the one-group loops combine the raw words
//                   (src/bitvector.cpp:1313-1325, 1512-1523, 1640-1652, 1789-1801
//                   and the _c0 kernels)
//   mode 2: ZERO_FILL  append_counter(0, fill_n) on an empty vector
__global__ void k_small(int mode, int op, const uint32_t* xw, const uint32_t* yw, uint32_t fill_n,
                        uint32_t groups, uint32_t* out, uint32_t* obp, DevMeta* meta,
                        uint32_t anb, uint32_t aval) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t n = 0, w = 0;
    if (mode == 1) {
        const uint32_t x = xw[0], y = yw[0];
        switch (op) {
        case OP_AND: w = x & y; break;
        case OP_OR: w = x | y; break;
        case OP_XOR: w = x ^ y; break;
        default: w = x & ~y;
        }
        n = 1;
    } else if (mode == 2) {
        w = HEADER0 | fill_n;
        n = 1;
        groups = fill_n;
    }
    uint32_t g = groups, ones = 0;
    if (n) {
        out[0] = w;
        if (w < HEADER0) { g = 1; ones = __popc(w); }
        else { g = w & MAXCNT; ones = (w >= HEADER1) ? g * 31u : 0u; }
        obp[0] = 0;
        obp[1] = g;
    } else {
        obp[0] = g;
    }
    meta->n = n;
    meta->groups = g;
    meta->nset = ones;
    meta->nfill = (n && w > ALLONES) ? 1u : 0u;
    meta->w0 = n ? w : 0u;
    meta->anb = anb;
    meta->aval = aval;
}

// Row ids of the 1 bits: ascending positions (the reference's indexSet walk,
// src/bitvector.cpp:4524-4590).  Literal bit 30-k of the word at group g is
// row 31g+k; the active word's bits follow, most significant first.
__global__ void __launch_bounds__(SCAN_THREADS)
k_rids(const uint32_t* __restrict__ w, uint32_t n, const uint32_t* __restrict__ bpos,
       uint32_t groups, uint32_t anb, uint32_t aval, uint32_t* __restrict__ out, uint64_t cap,
       unsigned long long* total_out, DevMeta* meta, TileRec* recs, LaunchSync* sync, uint32_t ntiles) {
    __shared__ uint64_t sh[SCAN_THREADS / 32 + 1];
    __shared__ uint32_t hdr[2];
    __shared__ uint64_t tile_pre;
    __shared__ uint32_t fq_n;
    __shared__ uint64_t fq_off[SCAN_TILE / 2];
    __shared__ uint32_t fq_row[SCAN_TILE / 2];
    __shared__ uint32_t fq_len[SCAN_TILE / 2];
    if (threadIdx.x == 0) { hdr[0] = claim_tile(sync); hdr[1] = ld_cg(&sync->epoch); fq_n = 0; }
    __syncthreads();
    const uint32_t t = hdr[0], epoch = hdr[1];
    const uint32_t base = t * SCAN_TILE + threadIdx.x * SCAN_WPT;
    uint32_t v[SCAN_WPT];
    uint64_t cnt = 0;
    uint32_t gpos = 0;
    if (base < n) {
        // group position of this thread's first word: block position + scan within the block
        const uint32_t blk = base / 32u;
        gpos = __ldg(bpos + blk);
        for (uint32_t k = blk * 32u; k < base; ++k) gpos += wgroups(__ldg(w + k));
    }
#pragma unroll
    for (int q = 0; q < SCAN_WPT; ++q) {
        v[q] = (base + q < n) ? __ldg(w + base + q) : 0u;
        const uint32_t x = v[q];
        if (base + q < n) cnt += (x > ALLONES) ? ((x >= HEADER1) ? (uint64_t)(x & MAXCNT) * 31u : 0u) : __popc(x);
    }
    uint64_t total;
    const uint64_t ex = block_exscan64(cnt, sh, total);
    if (threadIdx.x < 32) {
        uint64_t prefix; uint32_t pa, pb;
        bool ok = lookback64(recs, t, epoch, total, 0, 0, prefix, pa, pb);
        if (threadIdx.x == 0 && !ok) atomicExch(&meta->status, DEV_ERR_TIMEOUT);
        if (threadIdx.x == 0) tile_pre = prefix;
        if (threadIdx.x == 0 && t == ntiles - 1) {
            uint64_t off = prefix + total;
            const uint32_t rbase = groups * 31u;
            for (uint32_t b = 0; b < anb; ++b)
                if ((aval >> (anb - 1u - b)) & 1u) { if (off < cap) out[off] = rbase + b; ++off; }
            *total_out = off;
        }
    }
    __syncthreads();
    uint64_t off = tile_pre + ex;
    uint32_t g = gpos;
#pragma unroll
    for (int q = 0; q < SCAN_WPT; ++q) {
        if (base + q < n) {
            const uint32_t x = v[q];
            if (x > ALLONES) {
                const uint32_t c = x & MAXCNT;
                if (x >= HEADER1) {
                    const uint32_t slot = atomicAdd(&fq_n, 1u);
                    if (slot < (uint32_t)(SCAN_TILE / 2)) {
                        fq_off[slot] = off; fq_row[slot] = g * 31u; fq_len[slot] = c * 31u;
                    } else {  // list full: this thread writes the fill
                        for (uint32_t r = 0; r < c * 31u; ++r) if (off + r < cap) out[off + r] = g * 31u + r;
                    }
                    off += (uint64_t)c * 31u;
                }
                g += c;
            } else {
                uint32_t bits = x;
                while (bits) {
                    const uint32_t b = 31u - __clz(bits);  // highest set bit
                    if (off < cap) out[off] = g * 31u + (30u - b);
                    ++off;
                    bits &= ~(1u << b);
                }
                g += 1;
            }
        }
    }
    __syncthreads();
    // the CTA writes every listed 1-fill of the tile cooperatively
    const uint32_t nfq = min(fq_n, (uint32_t)(SCAN_TILE / 2));
    for (uint32_t k = 0; k < nfq; ++k) {
        const uint64_t o = fq_off[k];
        const uint32_t r0 = fq_row[k], len = fq_len[k];
        for (uint32_t r = threadIdx.x; r < len; r += SCAN_THREADS)
            if (o + r < cap) out[o + r] = r0 + r;
    }
    __syncthreads();
    if (threadIdx.x == 0) finish_tile(sync, ntiles);
}

// decompress(): every word expanded to its groups as literal words.
__global__ void __launch_bounds__(SCAN_THREADS)
k_decompress(const uint32_t* __restrict__ w, uint32_t n, const uint32_t* __restrict__ bpos,
             uint32_t* __restrict__ out) {
    __shared__ uint32_t fq_n;
    __shared__ uint32_t fq_pos[SCAN_TILE / 2], fq_len[SCAN_TILE / 2], fq_val[SCAN_TILE / 2];
    if (threadIdx.x == 0) fq_n = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_WPT;
    if (base < n) {
        const uint32_t blk = base / 32u;
        uint32_t g = __ldg(bpos + blk);
        for (uint32_t k = blk * 32u; k < base; ++k) g += wgroups(__ldg(w + k));
        for (int q = 0; q < SCAN_WPT && base + q < n; ++q) {
            const uint32_t x = __ldg(w + base + q);
            if (x > ALLONES) {
                const uint32_t c = x & MAXCNT;
                const uint32_t val = (x >= HEADER1) ? ALLONES : 0u;
                const uint32_t slot = atomicAdd(&fq_n, 1u);
                if (slot < (uint32_t)(SCAN_TILE / 2)) {
                    fq_pos[slot] = g; fq_len[slot] = c; fq_val[slot] = val;
                } else {  // list full: this thread writes the fill
                    for (uint32_t r = 0; r < c; ++r) out[g + r] = val;
                }
                g += c;
            } else {
                out[g] = x;
                g += 1;
            }
        }
    }
    __syncthreads();
    const uint32_t nfq = min(fq_n, (uint32_t)(SCAN_TILE / 2));
    for (uint32_t k = 0; k < nfq; ++k) {
        const uint32_t p = fq_pos[k], len = fq_len[k], val = fq_val[k];
        for (uint32_t r = threadIdx.x; r < len; r += SCAN_THREADS) out[p + r] = val;
    }
}

}  // namespace wah
#endif
