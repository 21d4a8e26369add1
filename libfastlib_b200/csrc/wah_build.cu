// Index construction on the device: equality (relic) and equal-weight
// binned (bin) indexes of a column already in device memory.
//
// The reference builds these on the host one row at a time
// (index::mapValues, src/index.cpp:2552-2611: setBit(row) on the bitmap of
// the row's value; bin::binning, src/ibin.cpp:3350-3449, with equal-weight
// boundaries from scanAndPartition, src/ibin.cpp:2390-2582).  Here:
//   1. (value, row) pairs sorted by value (CUB radix sort, stable, so the
//      rows of one value stay ascending);
//   2. bitmaps = segments of the sorted order: one per distinct value
//      (relic), or runs of whole distinct values of about nrows/nbins rows
//      (bin; every value lies in one bin, so a bin's [min, max] are real
//      values);
//   3. per (bitmap, 31-row group) "unit": its literal, OR-ed from the rows;
//   4. per unit, the WAH words it emits — the zero groups before it as one
//      fill (or a literal 0 for a single group), then its literal, runs of
//      all-1 groups as one fill — counted, scanned and written.
// The words are in compress() form, then heavy bitmaps are decompressed as
// the reference's optionalUnpack does by default (k_unpack_bitmaps), so a
// relic index's words equal relic::construct's; the bits of every bitmap are
// exactly the reference's.
#define WAH_RANGE_TYPES_ONLY
#include "../../include/wahgpu.h"
#include "wah_api_internal.h"
#include "wah_index_internal.h"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_run_length_encode.cuh>
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>
#include <algorithm>
#include <vector>

using namespace wah;

namespace {

constexpr uint32_t BT = 256;

inline uint32_t nblocks(uint64_t n) { return (uint32_t)std::max<uint64_t>(1, (n + BT - 1) / BT); }

// segment heads: 1 at the first sorted position of every bitmap
__global__ void k_mark_segments(const uint32_t* __restrict__ seg_start, uint32_t nseg, uint32_t* __restrict__ flag) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nseg) flag[seg_start[s]] = 1u;
}

// unit heads: the first row of a (bitmap, group) in sorted order
__global__ void k_mark_units(const uint32_t* __restrict__ rows, const uint32_t* __restrict__ seg_of, uint32_t n,
                             uint32_t* __restrict__ flag) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    flag[e] = (e == 0 || seg_of[e] != seg_of[e - 1] || rows[e] / MAXBITS != rows[e - 1] / MAXBITS) ? 1u : 0u;
}

// unit literal: the group's bits (bit 30 - row%31), or for the active group
// the active word's bits (the first row at bit anb-1)
__global__ void k_fill_units(const uint32_t* __restrict__ rows, const uint32_t* __restrict__ seg_of,
                             const uint32_t* __restrict__ unit_of, uint32_t n, uint32_t G, uint32_t anb,
                             uint32_t* __restrict__ u_seg, uint32_t* __restrict__ u_grp, uint32_t* __restrict__ u_lit) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const uint32_t r = rows[e], g = r / MAXBITS, k = r % MAXBITS;
    const uint32_t u = unit_of[e] - 1u;
    if (e == 0 || unit_of[e - 1] != unit_of[e]) { u_seg[u] = seg_of[e] - 1u; u_grp[u] = g; }
    const uint32_t bit = g < G ? (1u << (30u - k)) : (1u << (anb - 1u - k));
    atomicOr(&u_lit[u], bit);
}

__device__ __forceinline__ uint32_t zero_run_words(uint32_t k) { return k >= 2u ? 1u : k; }
__device__ __forceinline__ uint32_t zero_run_word(uint32_t k) { return k >= 2u ? (HEADER0 | k) : 0u; }

// Unit u's neighbours in its bitmap and what it emits.
struct UnitView {
    uint32_t g, lit, gap;   // group, literal, zero groups between it and the previous unit
    bool first, last, cont; // first / last unit of the bitmap; continues an all-1 run
};
__device__ __forceinline__ UnitView unit_view(const uint32_t* u_seg, const uint32_t* u_grp, const uint32_t* u_lit,
                                              uint32_t u, uint32_t nu, uint32_t G) {
    UnitView v;
    v.g = u_grp[u];
    v.lit = u_lit[u];
    v.first = u == 0 || u_seg[u - 1] != u_seg[u];
    v.last = u + 1 == nu || u_seg[u + 1] != u_seg[u];
    const int64_t gp = v.first ? -1 : (int64_t)u_grp[u - 1];
    v.gap = (uint32_t)((int64_t)min(v.g, G) - gp - 1);
    v.cont = !v.first && v.g < G && v.lit == ALLONES && v.gap == 0 && u_lit[u - 1] == ALLONES;
    return v;
}

__global__ void k_count_words(const uint32_t* __restrict__ u_seg, const uint32_t* __restrict__ u_grp,
                              const uint32_t* __restrict__ u_lit, uint32_t nu, uint32_t G, uint32_t* __restrict__ cnt,
                              uint32_t* __restrict__ seg_first) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nu) return;
    const UnitView v = unit_view(u_seg, u_grp, u_lit, u, nu, G);
    if (v.first) seg_first[u_seg[u]] = u;
    uint32_t w = zero_run_words(v.gap);
    if (v.g < G) {
        if (!v.cont) w += 1u;
        if (v.last) w += zero_run_words(G - 1u - v.g);
    }
    cnt[u] = w;
}

__global__ void k_write_words(const uint32_t* __restrict__ u_seg, const uint32_t* __restrict__ u_grp,
                              const uint32_t* __restrict__ u_lit, uint32_t nu, uint32_t G, uint32_t anb,
                              const uint32_t* __restrict__ woff, const uint32_t* __restrict__ seg_first,
                              uint32_t* __restrict__ words, BitmapMeta* __restrict__ bm) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nu) return;
    const UnitView v = unit_view(u_seg, u_grp, u_lit, u, nu, G);
    uint32_t o = woff[u];
    const uint32_t s = u_seg[u];
    if (v.gap) words[o++] = zero_run_word(v.gap);
    if (v.g < G) {
        if (!v.cont) {
            uint32_t wd = v.lit;
            if (v.lit == ALLONES) {  // head of a run of all-1 groups
                uint32_t len = 1;
                while (u + len < nu && u_seg[u + len] == s && u_grp[u + len] == v.g + len &&
                       u_lit[u + len] == ALLONES)
                    ++len;
                if (len >= 2) wd = HEADER1 | len;
            }
            words[o++] = wd;
        }
        if (v.last) {
            const uint32_t k = G - 1u - v.g;
            if (k) words[o++] = zero_run_word(k);
        }
    }
    if (v.last) {
        // the bitmap's words: from its first unit's offset to here (the
        // first unit was recorded by the counting launch)
        const uint32_t w0 = woff[seg_first[s]];
        bm[s].wstart = w0;
        bm[s].n = o - w0;
        bm[s].anb = anb;
        bm[s].aval = v.g >= G ? v.lit : 0u;
        bm[s].groups = 0;
    }
}

// bin of every row: the last bin whose smallest value is <= the row's value
// index::optionalUnpack (src/index.cpp:8730-8856) with no index option and
// no parameter set — what relic::construct and bin::binning do by default:
// a bitmap whose bytes() (m_vec words * 4 + sizeof(ibis::bitvector), 40 on
// LP64) exceed max(nrows / 9, sizeof(ibis::bitvector) + 12) is decompressed,
// every fill becoming its literals.  One warp per bitmap copies its words
// from the old pool to the new one, or expands them (fills of more than 32
// groups by the whole warp).
constexpr uint64_t REF_BITVECTOR_BYTES = 40;
__global__ void k_unpack_bitmaps(const uint32_t* __restrict__ src, const BitmapMeta* __restrict__ old_bm,
                                 const BitmapMeta* __restrict__ new_bm, uint32_t nobs, uint32_t* __restrict__ dst) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (b >= nobs) return;
    const BitmapMeta mo = old_bm[b], mn = new_bm[b];
    const uint32_t* w = src + mo.wstart;
    uint32_t* d = dst + mn.wstart;
    if (mn.n == mo.n) {  // kept as it is
        for (uint32_t i = lane; i < mo.n; i += 32) d[i] = __ldg(w + i);
        return;
    }
    uint32_t carry = 0;
    for (uint32_t base = 0; base < mo.n; base += 32) {
        const uint32_t i = base + lane;
        const bool in = i < mo.n;
        const uint32_t wd = in ? __ldg(w + i) : 0u;
        const uint32_t c = in ? wgroups(wd) : 0u;
        uint32_t x = c;
#pragma unroll
        for (int k = 1; k < 32; k <<= 1) { uint32_t t = __shfl_up_sync(0xffffffffu, x, k); if (lane >= (uint32_t)k) x += t; }
        const uint32_t p = carry + x - c;
        if (in && c <= 32u) for (uint32_t g = 0; g < c; ++g) d[p + g] = wpattern(wd);
        uint32_t f = __ballot_sync(0xffffffffu, in && c > 32u);
        while (f) {
            const uint32_t s = __ffs(f) - 1u;
            f &= f - 1u;
            const uint32_t fp = __shfl_sync(0xffffffffu, p, s), fc = __shfl_sync(0xffffffffu, c, s);
            const uint32_t pat = __shfl_sync(0xffffffffu, wpattern(wd), s);
            for (uint32_t g = lane; g < fc; g += 32u) d[fp + g] = pat;
        }
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
}

template <typename K>
__global__ void k_bin_of(const K* __restrict__ vals, uint32_t n, const K* __restrict__ bmin, uint32_t nb,
                         uint32_t* __restrict__ bin) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const K v = vals[i];
    uint32_t lo = 0, hi = nb;  // bmin[lo] <= v < bmin[hi]
    while (hi - lo > 1) {
        const uint32_t m = (lo + hi) >> 1;
        if (bmin[m] <= v) lo = m; else hi = m;
    }
    bin[i] = lo;
}

__global__ void k_iota(uint32_t* __restrict__ v, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

// Scratch held for the duration of one build, returned to the pool on exit.
struct Scratch {
    wahgpu_ctx* ctx;
    std::vector<void*> p;
    explicit Scratch(wahgpu_ctx* c) : ctx(c) {}
    void* get(size_t bytes) {
        void* q = wg_alloc(ctx, std::max<size_t>(bytes, 16));
        if (q) p.push_back(q);
        return q;
    }
    ~Scratch() {
        cudaStreamSynchronize(ctx->stream);
        for (void* q : p) wg_free(ctx, q);
    }
};

#define BTRY(call)                                                                                 \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return wg_fail(ctx, WAHGPU_ECUDA, "%s failed: %s", #call, cudaGetErrorString(e_));     \
    } while (0)
#define BALLOC(var, type, count)                                                                   \
    type* var = static_cast<type*>(sc.get((size_t)(count) * sizeof(type)));                        \
    if (!var) return wg_fail(ctx, WAHGPU_ENOMEM, "index build: device allocation failed")

template <typename K>
int build_typed(wahgpu_ctx* ctx, int kind, int vtype, const K* dvals, uint32_t n, uint32_t nbins,
                wahgpu_index** out) {
    cudaStream_t st = ctx->stream;
    Scratch sc(ctx);
    const uint32_t G = n / MAXBITS, anb = n % MAXBITS;
    // 1. sort (value, row) by value
    BALLOC(rows_in, uint32_t, n);
    BALLOC(rows, uint32_t, n);
    BALLOC(keys, K, n);
    k_iota<<<nblocks(n), BT, 0, st>>>(rows_in, n);
    size_t tb = 0, tb2 = 0;
    BTRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, dvals, keys, rows_in, rows, n, 0, (int)(sizeof(K) * 8), st));
    // 2. distinct values and their row counts
    BALLOC(uniq, K, n);
    BALLOC(ucnt, uint32_t, n);
    BALLOC(nruns, uint32_t, 1);
    BTRY(cub::DeviceRunLengthEncode::Encode(nullptr, tb2, keys, uniq, ucnt, nruns, n, st));
    tb = std::max(tb, tb2);
    tb2 = 0;
    BTRY(cub::DeviceScan::InclusiveSum(nullptr, tb2, rows_in, rows_in, n + 1, st));
    tb = std::max(tb, tb2);
    BALLOC(temp, unsigned char, tb);
    size_t t = tb;
    BTRY(cub::DeviceRadixSort::SortPairs(temp, t, dvals, keys, rows_in, rows, n, 0, (int)(sizeof(K) * 8), st));
    t = tb;
    BTRY(cub::DeviceRunLengthEncode::Encode(temp, t, keys, uniq, ucnt, nruns, n, st));
    uint32_t nu_val = 0;
    BTRY(cudaMemcpyAsync(&nu_val, nruns, 4, cudaMemcpyDeviceToHost, st));
    BTRY(cudaStreamSynchronize(st));
    std::vector<K> hk(nu_val);
    std::vector<uint32_t> hc(nu_val);
    BTRY(cudaMemcpyAsync(hk.data(), uniq, (size_t)nu_val * sizeof(K), cudaMemcpyDeviceToHost, st));
    BTRY(cudaMemcpyAsync(hc.data(), ucnt, (size_t)nu_val * 4, cudaMemcpyDeviceToHost, st));
    BTRY(cudaStreamSynchronize(st));
    // segments (bitmaps) as [start, end) of the sorted order, with their keys
    std::vector<uint32_t> seg{0};
    std::vector<double> kmin, kmax;
    if (kind == WAHGPU_RELIC) {
        uint64_t pos = 0;
        for (uint32_t i = 0; i < nu_val; ++i) {
            pos += hc[i];
            seg.push_back((uint32_t)pos);
            kmin.push_back((double)hk[i]);
        }
    } else {
        // equal weight: close a bin once it reaches its share of the rows
        // still to be placed; a distinct value never straddles two bins
        uint64_t pos = 0;
        uint32_t i = 0, left_bins = std::max<uint32_t>(nbins, 1);
        while (i < nu_val) {
            const uint64_t target = (n - pos + left_bins - 1) / left_bins;
            const uint32_t b0 = i;
            uint64_t rows_in_bin = 0;
            while (i < nu_val && (rows_in_bin == 0 || rows_in_bin + hc[i] <= target || left_bins == 1)) {
                rows_in_bin += hc[i];
                ++i;
            }
            pos += rows_in_bin;
            seg.push_back((uint32_t)pos);
            kmin.push_back((double)hk[b0]);
            kmax.push_back((double)hk[i - 1]);
            if (left_bins > 1) --left_bins;
        }
    }
    const uint32_t nobs = (uint32_t)seg.size() - 1;
    if (kind == WAHGPU_BIN) {
        // a bin holds several values: order its rows by row id (stable sort
        // of the rows by bin, from row order)
        BALLOC(bmin, K, nobs);
        BALLOC(bin_of, uint32_t, n);
        BALLOC(bin_sorted, uint32_t, n);
        std::vector<K> hmin(nobs);
        for (uint32_t j = 0, i = 0; j < nobs; ++j) { hmin[j] = hk[i]; while (i < nu_val && (double)hk[i] <= kmax[j]) ++i; }
        BTRY(cudaMemcpyAsync(bmin, hmin.data(), (size_t)nobs * sizeof(K), cudaMemcpyHostToDevice, st));
        k_bin_of<K><<<nblocks(n), BT, 0, st>>>(dvals, n, bmin, nobs, bin_of);
        k_iota<<<nblocks(n), BT, 0, st>>>(rows_in, n);
        int bits = 1;
        while (bits < 32 && (1ull << bits) < nobs) ++bits;
        t = tb;
        BTRY(cub::DeviceRadixSort::SortPairs(temp, t, bin_of, bin_sorted, rows_in, rows, n, 0, bits, st));
        ctx->launches += 3;
    }
    // 3. per element: bitmap, unit
    BALLOC(d_seg, uint32_t, nobs + 1);
    BALLOC(seg_of, uint32_t, n);
    BALLOC(unit_of, uint32_t, n);
    BTRY(cudaMemcpyAsync(d_seg, seg.data(), (size_t)(nobs + 1) * 4, cudaMemcpyHostToDevice, st));
    BTRY(cudaMemsetAsync(seg_of, 0, (size_t)n * 4, st));
    k_mark_segments<<<nblocks(nobs), BT, 0, st>>>(d_seg, nobs, seg_of);
    t = tb;
    BTRY(cub::DeviceScan::InclusiveSum(temp, t, seg_of, seg_of, n, st));
    k_mark_units<<<nblocks(n), BT, 0, st>>>(rows, seg_of, n, unit_of);
    t = tb;
    BTRY(cub::DeviceScan::InclusiveSum(temp, t, unit_of, unit_of, n, st));
    uint32_t nu = 0;
    BTRY(cudaMemcpyAsync(&nu, unit_of + (n - 1), 4, cudaMemcpyDeviceToHost, st));
    BTRY(cudaStreamSynchronize(st));
    BALLOC(u_seg, uint32_t, nu);
    BALLOC(u_grp, uint32_t, nu);
    BALLOC(u_lit, uint32_t, nu);
    BALLOC(u_cnt, uint32_t, nu + 1);
    BALLOC(seg_first, uint32_t, nobs);
    BTRY(cudaMemsetAsync(u_lit, 0, (size_t)nu * 4, st));
    k_fill_units<<<nblocks(n), BT, 0, st>>>(rows, seg_of, unit_of, n, G, anb, u_seg, u_grp, u_lit);
    // 4. words: count, scan, write
    k_count_words<<<nblocks(nu), BT, 0, st>>>(u_seg, u_grp, u_lit, nu, G, u_cnt, seg_first);
    BTRY(cudaMemsetAsync(u_cnt + nu, 0, 4, st));
    t = tb;
    BTRY(cub::DeviceScan::ExclusiveSum(temp, t, u_cnt, u_cnt, nu + 1, st));
    uint32_t nwords = 0;
    BTRY(cudaMemcpyAsync(&nwords, u_cnt + nu, 4, cudaMemcpyDeviceToHost, st));
    BTRY(cudaStreamSynchronize(st));

    wahgpu_index* x = new wahgpu_index();
    x->ctx = ctx; x->kind = kind; x->nrows = n; x->groups = G; x->anb = anb; x->nobs = nobs;
    x->keys = kmin;
    if (kind == WAHGPU_BIN) x->keys.insert(x->keys.end(), kmax.begin(), kmax.end());
    x->d_words = static_cast<uint32_t*>(wg_alloc(ctx, std::max<uint64_t>(nwords, 1) * 4));
    x->d_bm = static_cast<BitmapMeta*>(wg_alloc(ctx, std::max<size_t>(nobs, 1) * sizeof(BitmapMeta)));
    if (kind == WAHGPU_BIN) x->d_values = wg_alloc(ctx, (size_t)n * 4);
    if (!x->d_words || !x->d_bm || (kind == WAHGPU_BIN && !x->d_values)) {
        wahgpu_index_free(x);
        return wg_fail(ctx, WAHGPU_ENOMEM, "index build: device allocation failed");
    }
    k_write_words<<<nblocks(nu), BT, 0, st>>>(u_seg, u_grp, u_lit, nu, G, anb, u_cnt, seg_first, x->d_words,
                                             x->d_bm);
    ctx->launches += 9;
    if (kind == WAHGPU_BIN) {
        BTRY(cudaMemcpyAsync(x->d_values, dvals, (size_t)n * 4, cudaMemcpyDeviceToDevice, st));
        x->vtype = (uint32_t)vtype;
    }
    BTRY(cudaGetLastError());
    std::vector<BitmapMeta> hb(nobs);
    BTRY(cudaMemcpyAsync(hb.data(), x->d_bm, (size_t)nobs * sizeof(BitmapMeta), cudaMemcpyDeviceToHost, st));
    BTRY(cudaStreamSynchronize(st));
    // optionalUnpack's default rule: heavy bitmaps decompressed
    {
        const uint64_t bar = std::max<uint64_t>(n / 9, REF_BITVECTOR_BYTES + 12);
        std::vector<BitmapMeta> nb = hb;
        uint64_t pos = 0;
        bool any = false;
        for (uint32_t j = 0; j < nobs; ++j) {
            const bool heavy = (uint64_t)hb[j].n * 4 + REF_BITVECTOR_BYTES > bar && hb[j].n != G;
            nb[j].wstart = pos;
            nb[j].n = heavy ? G : hb[j].n;
            pos += nb[j].n;
            any |= heavy;
        }
        if (any) {
            uint32_t* nw = static_cast<uint32_t*>(wg_alloc(ctx, std::max<uint64_t>(pos, 1) * 4));
            BitmapMeta* nbm = static_cast<BitmapMeta*>(wg_alloc(ctx, std::max<size_t>(nobs, 1) * sizeof(BitmapMeta)));
            if (!nw || !nbm) {
                wg_free(ctx, nw); wg_free(ctx, nbm);
                wahgpu_index_free(x);
                return wg_fail(ctx, WAHGPU_ENOMEM, "index build: device allocation failed (unpacking heavy bitmaps)");
            }
            BTRY(cudaMemcpyAsync(nbm, nb.data(), (size_t)nobs * sizeof(BitmapMeta), cudaMemcpyHostToDevice, st));
            k_unpack_bitmaps<<<nblocks((uint64_t)nobs * 32), BT, 0, st>>>(x->d_words, x->d_bm, nbm, nobs, nw);
            ctx->launches++;
            BTRY(cudaGetLastError());
            BTRY(cudaStreamSynchronize(st));  // nb (host) staged above must outlive the copy
            wg_free(ctx, x->d_words);
            wg_free(ctx, x->d_bm);
            x->d_words = nw;
            x->d_bm = nbm;
            hb = nb;
        }
    }
    x->bwords.resize(nobs);
    for (uint32_t j = 0; j < nobs; ++j) x->bwords[j] = hb[j].n;
    int rc = wg_index_attach(x);
    if (rc) { wahgpu_index_free(x); return rc; }
    *out = x;
    return WAHGPU_OK;
}

}  // namespace

extern "C" int wahgpu_index_build(wahgpu_ctx* ctx, int kind, int vtype, const void* dev_values, uint64_t nrows,
                                  uint32_t nbins, wahgpu_index** out) {
    if (!ctx || !out || !dev_values || nrows == 0 || (kind != WAHGPU_RELIC && kind != WAHGPU_BIN) ||
        (kind == WAHGPU_BIN && nbins == 0))
        return wg_fail(ctx, WAHGPU_EINVAL, "wahgpu_index_build: bad argument");
    if (nrows > 0xFFFFFFFFull) return wg_fail(ctx, WAHGPU_ERANGE, "wahgpu_index_build: more than 2^32-1 rows");
    *out = nullptr;
    const uint32_t n = (uint32_t)nrows;
    switch (vtype) {
    case WAHGPU_U32: return build_typed<uint32_t>(ctx, kind, vtype, static_cast<const uint32_t*>(dev_values), n, nbins, out);
    case WAHGPU_I32: return build_typed<int32_t>(ctx, kind, vtype, static_cast<const int32_t*>(dev_values), n, nbins, out);
    case WAHGPU_F32: return build_typed<float>(ctx, kind, vtype, static_cast<const float*>(dev_values), n, nbins, out);
    default: return wg_fail(ctx, WAHGPU_EINVAL, "wahgpu_index_build: value type %d", vtype);
    }
}

// A copy of bitmap j as a bitvector (index::getBitvector, src/index.h).
extern "C" int wahgpu_index_bitmap(wahgpu_index* x, uint32_t j, wahgpu_bv** out) {
    if (!x || !out || j >= x->nobs) return WAHGPU_EINVAL;
    wahgpu_ctx* ctx = x->ctx;
    BitmapMeta m;
    cudaError_t e = cudaMemcpyAsync(&m, x->d_bm + j, sizeof(BitmapMeta), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return wg_fail(ctx, WAHGPU_ECUDA, "reading bitmap metadata failed");
    // serialized form on the device: m_vec words, then the active word
    uint32_t* d = static_cast<uint32_t*>(wg_alloc(ctx, ((size_t)m.n + 2) * 4));
    if (!d) return wg_fail(ctx, WAHGPU_ENOMEM, "allocation failed");
    if (m.n) e = cudaMemcpyAsync(d, x->d_words + m.wstart, (size_t)m.n * 4, cudaMemcpyDeviceToDevice, ctx->stream);
    const uint32_t tail[2] = {m.aval, m.anb};
    const uint32_t ntail = m.anb ? 2u : 1u;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d + m.n, m.anb ? tail : tail + 1, ntail * 4, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) { wg_free(ctx, d); return wg_fail(ctx, WAHGPU_ECUDA, "copying the bitmap failed"); }
    const int rc = wahgpu_bv_from_device_serial(ctx, d, (uint64_t)m.n + ntail, out);
    wg_free(ctx, d);
    return rc;
}

// The index's keys: relic, the distinct values; bin, the bins' smallest
// values followed by their largest (the layout of the reference's
// (keys, offsets, bitmaps) triple).  Returns the key count.
extern "C" int64_t wahgpu_index_keys(wahgpu_index* x, double* out, uint64_t cap) {
    if (!x || (cap && !out)) return WAHGPU_EINVAL;
    const uint64_t n = x->keys.size();
    if (cap < n) return wg_fail(x->ctx, WAHGPU_ESIZE, "need room for %llu keys", (unsigned long long)n);
    std::copy(x->keys.begin(), x->keys.end(), out);
    return (int64_t)n;
}

// The index as the reference's serialized triple (relic::write(keys, starts,
// bitmaps), src/irelic.cpp:644-667; bin::write, src/ibin.cpp:5836-5859;
// fastbit_iapi_deconstruct_index, src/iapi.cpp:1915): keys (relic: values;
// bin: minval then maxval), nobs + 1 word offsets, and every bitmap's
// serialized words (write(array_t&)) one after the other.
extern "C" int wahgpu_index_deconstruct(wahgpu_index* x, double* keys, uint64_t kcap, uint64_t* nkeys,
                                        int64_t* offsets, uint64_t ocap, uint64_t* noffsets, uint32_t* bitmaps,
                                        uint64_t bcap, uint64_t* nbitmaps) {
    if (!x) return WAHGPU_EINVAL;
    wahgpu_ctx* ctx = x->ctx;
    std::vector<BitmapMeta> bm(x->nobs);
    cudaError_t e = cudaSuccess;
    if (x->nobs) e = cudaMemcpyAsync(bm.data(), x->d_bm, sizeof(BitmapMeta) * x->nobs, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return wg_fail(ctx, WAHGPU_ECUDA, "reading bitmap metadata failed: %s", cudaGetErrorString(e));
    std::vector<int64_t> off(x->nobs + 1ull, 0);
    uint64_t pool = 0;
    for (uint32_t j = 0; j < x->nobs; ++j) {
        off[j + 1] = off[j] + (int64_t)bm[j].n + (bm[j].anb ? 2 : 1);
        pool = std::max<uint64_t>(pool, bm[j].wstart + bm[j].n);
    }
    if (nkeys) *nkeys = x->keys.size();
    if (noffsets) *noffsets = off.size();
    if (nbitmaps) *nbitmaps = (uint64_t)off.back();
    if (!(keys && offsets && bitmaps)) return WAHGPU_OK;
    if (kcap < x->keys.size() || ocap < off.size() || bcap < (uint64_t)off.back())
        return wg_fail(ctx, WAHGPU_ESIZE, "output arrays too small for the triple");
    std::vector<uint32_t> w(pool);
    if (pool) e = cudaMemcpyAsync(w.data(), x->d_words, pool * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return wg_fail(ctx, WAHGPU_ECUDA, "reading the bitmaps failed: %s", cudaGetErrorString(e));
    std::copy(x->keys.begin(), x->keys.end(), keys);
    std::copy(off.begin(), off.end(), offsets);
    for (uint32_t j = 0; j < x->nobs; ++j) {
        uint32_t* d = bitmaps + off[j];
        std::copy(w.begin() + bm[j].wstart, w.begin() + bm[j].wstart + bm[j].n, d);
        d += bm[j].n;
        if (bm[j].anb) *d++ = bm[j].aval;
        *d = bm[j].anb;
    }
    return WAHGPU_OK;
}
