// Index store and range evaluation behind the C ABI (include/wahgpu.h):
// relic / bin indexes attached from the reference's (keys, offsets, bitmaps)
// triple, the host-side locate (which bitmaps a range covers wholly and which
// edge bitmaps need a row check), and batched evaluation through k_range.
#include "../../include/wahgpu.h"
#include "wah_range.cuh"
#include "wah_api_internal.h"
#include "wah_index_internal.h"

#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>

using namespace wah;

#define CUDA_TRY(ctx, call)                                                            \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return wg_fail(ctx, WAHGPU_ECUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// ------------------------------------------------------------------ attach
extern "C" int wahgpu_index_from_triple(wahgpu_ctx* ctx, int kind, uint64_t nrows, const double* keys,
                                        uint64_t nkeys, const int64_t* offsets, uint64_t noffsets,
                                        const uint32_t* bitmaps, uint64_t nbitmaps, wahgpu_index** out) {
    if (!ctx || !out || (kind != WAHGPU_RELIC && kind != WAHGPU_BIN) || noffsets < 1 || !offsets ||
        (nbitmaps && !bitmaps) || nrows > 0xFFFFFFFFull)
        return wg_fail(ctx, WAHGPU_EINVAL, "bad argument");
    *out = nullptr;
    const uint32_t nobs = (uint32_t)(noffsets - 1);
    if ((kind == WAHGPU_RELIC && nkeys != nobs) || (kind == WAHGPU_BIN && nkeys != 2ull * nobs) || (nkeys && !keys))
        return wg_fail(ctx, WAHGPU_EINVAL, "key count %llu does not match %u bitmaps", (unsigned long long)nkeys, nobs);
    if (offsets[0] != 0 || (uint64_t)offsets[nobs] != nbitmaps)
        return wg_fail(ctx, WAHGPU_EFORMAT, "offsets do not span the bitmap array");
    wahgpu_index* x = new wahgpu_index();
    x->ctx = ctx; x->kind = kind; x->nrows = (uint32_t)nrows;
    x->groups = (uint32_t)(nrows / MAXBITS); x->anb = (uint32_t)(nrows % MAXBITS);
    x->nobs = nobs;
    x->ntiles = (x->groups + (x->anb ? 1 : 0) + RT - 1) / RT;
    x->keys.assign(keys, keys + nkeys);
    // per bitmap: the serialized trailer (src/bitvector.cpp:54-105)
    std::vector<BitmapMeta> bm(nobs);
    x->bwords.resize(nobs);
    for (uint32_t j = 0; j < nobs; ++j) {
        const int64_t a = offsets[j], b = offsets[j + 1];
        if (b < a) { delete x; return wg_fail(ctx, WAHGPU_EFORMAT, "offsets decrease at bitmap %u", j); }
        const uint64_t len = (uint64_t)(b - a);
        BitmapMeta& m = bm[j];
        m.wstart = (uint64_t)a; m.n = 0; m.anb = 0; m.aval = 0; m.groups = 0;
        if (len > 1) {
            const uint32_t last = bitmaps[b - 1];
            if (last > 0 && last < MAXBITS) { m.anb = last; m.aval = bitmaps[b - 2]; m.n = (uint32_t)(len - 2); }
            else m.n = (uint32_t)(len - 1);
        }
        x->bwords[j] = m.n;
    }
    x->d_words = static_cast<uint32_t*>(wg_alloc(ctx, std::max<uint64_t>(nbitmaps, 1) * 4));
    x->d_bm = static_cast<BitmapMeta*>(wg_alloc(ctx, std::max<size_t>(nobs, 1) * sizeof(BitmapMeta)));
    if (!x->d_words || !x->d_bm) {
        wahgpu_index_free(x);
        return wg_fail(ctx, WAHGPU_ENOMEM, "index allocation failed");
    }
    CUDA_TRY(ctx, cudaMemcpyAsync(x->d_words, bitmaps, nbitmaps * 4, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(x->d_bm, bm.data(), nobs * sizeof(BitmapMeta), cudaMemcpyHostToDevice, ctx->stream));
    int rc = wg_index_attach(x);
    if (rc) { wahgpu_index_free(x); return rc; }
    *out = x;
    return WAHGPU_OK;
}

// Per tile, the bitmaps holding a 1 bit in it (ascending), so a range term
// visits only bitmaps with data in the tile: pairs (tile, bitmap) emitted in
// bitmap order, stably sorted by tile, cut into CSR offsets.
static int build_tile_lists(wahgpu_index* x) {
    wahgpu_ctx* ctx = x->ctx;
    const uint32_t nobs = x->nobs, nt = x->ntiles;
    x->d_tl_off = static_cast<uint32_t*>(wg_alloc(ctx, ((size_t)nt + 1) * 4));
    if (!x->d_tl_off) return wg_fail(ctx, WAHGPU_ENOMEM, "index allocation failed");
    if (nobs == 0) {
        CUDA_TRY(ctx, cudaMemsetAsync(x->d_tl_off, 0, ((size_t)nt + 1) * 4, ctx->stream));
        x->d_tl_bm = static_cast<uint32_t*>(wg_alloc(ctx, 4));
        return x->d_tl_bm ? WAHGPU_OK : wg_fail(ctx, WAHGPU_ENOMEM, "index allocation failed");
    }
    std::vector<void*> tmp;
    auto get = [&](size_t bytes) { void* p = wg_alloc(ctx, std::max<size_t>(bytes, 16)); if (p) tmp.push_back(p); return p; };
    auto release = [&]() { cudaStreamSynchronize(ctx->stream); for (void* p : tmp) wg_free(ctx, p); };
    uint32_t* cnt = static_cast<uint32_t*>(get(((size_t)nobs + 1) * 4));
    if (!cnt) { release(); return wg_fail(ctx, WAHGPU_ENOMEM, "index allocation failed"); }
    const uint32_t threads = 256, blocks = (nobs * 32 + threads - 1) / threads;
    CUDA_TRY(ctx, cudaMemsetAsync(cnt + nobs, 0, 4, ctx->stream));
    k_tile_touch<<<blocks, threads, 0, ctx->stream>>>(x->d_words, x->d_bm, nobs, 0, cnt, nullptr, nullptr, nullptr);
    size_t tb = 0;
    CUDA_TRY(ctx, cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, cnt, nobs + 1, ctx->stream));
    void* t1 = get(tb);
    if (!t1) { release(); return wg_fail(ctx, WAHGPU_ENOMEM, "index allocation failed"); }
    CUDA_TRY(ctx, cub::DeviceScan::ExclusiveSum(t1, tb, cnt, cnt, nobs + 1, ctx->stream));
    uint32_t npairs = 0;
    CUDA_TRY(ctx, cudaMemcpyAsync(&npairs, cnt + nobs, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    uint32_t* pt = static_cast<uint32_t*>(get((size_t)npairs * 4));
    uint32_t* pb = static_cast<uint32_t*>(get((size_t)npairs * 4));
    uint32_t* st = static_cast<uint32_t*>(get((size_t)npairs * 4));
    x->d_tl_bm = static_cast<uint32_t*>(wg_alloc(ctx, std::max<size_t>((size_t)npairs * 4, 16)));
    if (!pt || !pb || !st || !x->d_tl_bm) { release(); return wg_fail(ctx, WAHGPU_ENOMEM, "index allocation failed"); }
    k_tile_touch<<<blocks, threads, 0, ctx->stream>>>(x->d_words, x->d_bm, nobs, 1, nullptr, cnt, pt, pb);
    int bits = 1;
    while (bits < 32 && (1ull << bits) <= nt) ++bits;
    tb = 0;
    CUDA_TRY(ctx, cub::DeviceRadixSort::SortPairs(nullptr, tb, pt, st, pb, x->d_tl_bm, npairs, 0, bits, ctx->stream));
    void* t2 = get(tb);
    if (!t2) { release(); return wg_fail(ctx, WAHGPU_ENOMEM, "index allocation failed"); }
    CUDA_TRY(ctx, cub::DeviceRadixSort::SortPairs(t2, tb, pt, st, pb, x->d_tl_bm, npairs, 0, bits, ctx->stream));
    k_tile_offsets<<<(npairs + 1 + threads - 1) / threads, threads, 0, ctx->stream>>>(st, npairs, nt, x->d_tl_off);
    ctx->launches += 5;
    CUDA_TRY(ctx, cudaGetLastError());
    release();
    return WAHGPU_OK;
}

// Cumulative rows: for a stride S, dense row k-1 = OR of bitmaps [0, k*S)
// (k = 1..K), so a range's wholly-inside span costs two dense reads per tile
// plus at most 2S edge bitmaps.  S is the smallest stride >= 8 that keeps
// the rows within CUM_BUDGET bytes (or the context's WAHGPU_TUNE_CUM_STRIDE);
// indexes with fewer than two rows' worth of bitmaps keep none.
static constexpr uint64_t CUM_BUDGET = 2ull << 30;
static int build_cumulative(wahgpu_index* x) {
    wahgpu_ctx* ctx = x->ctx;
    const uint32_t nobs = x->nobs;
    // rows are gx words rounded up to 4, so a tile's slice starts 16-byte aligned
    const uint64_t gx = ((uint64_t)x->groups + (x->anb ? 1 : 0) + 3) & ~3ull;
    x->cum_k = 0; x->cum_stride = 0;
    if (ctx->cum_stride == 1 || gx == 0) return WAHGPU_OK;
    const uint64_t stride = ctx->cum_stride ? ctx->cum_stride
                                            : std::max<uint64_t>(8, (nobs * gx * 4 + CUM_BUDGET - 1) / CUM_BUDGET);
    const uint64_t K = nobs / stride;
    if (K < 2) return WAHGPU_OK;
    x->d_cum = static_cast<uint32_t*>(wg_alloc(ctx, K * gx * 4));
    if (!x->d_cum) return WAHGPU_OK;  // no room: ranges use the bitmaps alone
    CUDA_TRY(ctx, cudaMemsetAsync(x->d_cum, 0, K * gx * 4, ctx->stream));
    const uint32_t nb = (uint32_t)(K * stride), threads = 256;
    const uint32_t blocks = (uint32_t)(((uint64_t)nb * 32 + threads - 1) / threads);
    k_cum_blocks<<<blocks, threads, 0, ctx->stream>>>(x->d_words, x->d_bm, nb, (uint32_t)stride, (uint32_t)gx, x->d_cum);
    k_cum_prefix<<<(uint32_t)((gx + 255) / 256), 256, 0, ctx->stream>>>(x->d_cum, (uint32_t)K, (uint32_t)gx);
    ctx->launches += 2;
    CUDA_TRY(ctx, cudaGetLastError());
    x->cum_k = (uint32_t)K;
    x->cum_stride = (uint32_t)stride;
    return WAHGPU_OK;
}

// Second half of building an index, shared by the triple upload and the
// device build: x->d_words / d_bm / bwords / keys are set; computes the
// per-bitmap tile index and 1-bit counts and validates the words.
int wg_index_attach(wahgpu_index* x) {
    wahgpu_ctx* ctx = x->ctx;
    const uint32_t nobs = x->nobs;
    x->ntiles = (x->groups + (x->anb ? 1 : 0) + RT - 1) / RT;
    const size_t tiles_bytes = (size_t)nobs * (x->ntiles + 1) * 8;
    x->d_tiles = static_cast<uint32_t*>(wg_alloc(ctx, std::max<size_t>(tiles_bytes, 8)));
    uint32_t* d_ones = static_cast<uint32_t*>(wg_alloc(ctx, std::max<size_t>(nobs, 1) * 4));
    DevMeta* d_st = static_cast<DevMeta*>(wg_alloc(ctx, sizeof(DevMeta)));
    if (!x->d_tiles || !d_ones || !d_st) {
        wg_free(ctx, d_ones);
        wg_free(ctx, d_st);
        return wg_fail(ctx, WAHGPU_ENOMEM, "index allocation failed");
    }
    int rc = WAHGPU_OK;
    CUDA_TRY(ctx, cudaMemsetAsync(d_st, 0, sizeof(DevMeta), ctx->stream));
    if (nobs) {
        const uint32_t threads = 256, blocks = (nobs * 32 + threads - 1) / threads;
        k_index_tiles<<<blocks, threads, 0, ctx->stream>>>(x->d_words, x->d_bm, nobs, x->ntiles, x->nrows,
                                                           x->d_tiles, d_ones, d_st);
        ctx->launches++;
        CUDA_TRY(ctx, cudaGetLastError());
    }
    DevMeta st{};
    x->bones.resize(nobs);
    CUDA_TRY(ctx, cudaMemcpyAsync(&st, d_st, sizeof(DevMeta), cudaMemcpyDeviceToHost, ctx->stream));
    if (nobs) CUDA_TRY(ctx, cudaMemcpyAsync(x->bones.data(), d_ones, nobs * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    wg_free(ctx, d_ones);
    wg_free(ctx, d_st);
    if (st.status == DEV_ERR_FORMAT) rc = wg_fail(ctx, WAHGPU_EFORMAT, "a bitmap holds a fill word of length 0");
    else if (st.status) rc = wg_fail(ctx, WAHGPU_ERANGE, "a bitmap holds more bits than the index has rows");
    if (rc) return rc;
    rc = build_tile_lists(x);
    if (rc) return rc;
    rc = build_cumulative(x);
    if (rc) return rc;
    x->cum_words.assign(nobs + 1, 0);
    x->cum_ones.assign(nobs + 1, 0);
    for (uint32_t j = 0; j < nobs; ++j) {
        x->cum_words[j + 1] = x->cum_words[j] + x->bwords[j];
        x->cum_ones[j + 1] = x->cum_ones[j] + x->bones[j];
    }
    if (x->kind == WAHGPU_BIN) {
        x->nonempty.clear();
        x->bins_sorted = true;
        for (uint32_t j = 0; j < nobs; ++j) {
            const double mn = x->keys[j], mx = x->keys[nobs + j];
            if (x->bones[j] == 0 || !(mn <= mx)) continue;
            if (!x->nonempty.empty() && !(x->keys[nobs + x->nonempty.back()] < mn)) x->bins_sorted = false;
            x->nonempty.push_back(j);
        }
    }
    x->dev.words = x->d_words; x->dev.bm = x->d_bm; x->dev.tiles = x->d_tiles;
    x->dev.tl_off = x->d_tl_off; x->dev.tl_bm = x->d_tl_bm;
    x->dev.cum = x->d_cum; x->dev.cum_stride = x->cum_stride; x->dev.cum_k = x->cum_k;
    x->dev.gx = (x->groups + (x->anb ? 1u : 0u) + 3u) & ~3u;
    x->dev.values = nullptr; x->dev.nobs = nobs; x->dev.vtype = 0; x->dev.ntiles = x->ntiles;
    if (x->d_values) { x->dev.values = x->d_values; x->dev.vtype = x->vtype; }
    return WAHGPU_OK;
}

extern "C" int wahgpu_index_set_values(wahgpu_index* x, int vtype, const void* values, uint64_t n) {
    if (!x || !values || vtype < 0 || vtype > 2) return WAHGPU_EINVAL;
    wahgpu_ctx* ctx = x->ctx;
    if (n != x->nrows) return wg_fail(ctx, WAHGPU_EINVAL, "%llu values for %u rows", (unsigned long long)n, x->nrows);
    wg_free(ctx, x->d_values);
    x->d_values = wg_alloc(ctx, std::max<uint64_t>(n, 1) * 4);
    if (!x->d_values) return wg_fail(ctx, WAHGPU_ENOMEM, "allocation failed");
    CUDA_TRY(ctx, cudaMemcpyAsync(x->d_values, values, n * 4, cudaMemcpyHostToDevice, ctx->stream));
    x->vtype = (uint32_t)vtype;
    x->dev.values = x->d_values;
    x->dev.vtype = x->vtype;
    return WAHGPU_OK;
}

extern "C" int wahgpu_index_free(wahgpu_index* x) {
    if (!x) return WAHGPU_EINVAL;
    wahgpu_ctx* ctx = x->ctx;
    cudaStreamSynchronize(ctx->stream);
    wg_free(ctx, x->d_words);
    wg_free(ctx, x->d_bm);
    wg_free(ctx, x->d_tiles);
    wg_free(ctx, x->d_tl_off);
    wg_free(ctx, x->d_cum);
    wg_free(ctx, x->d_tl_bm);
    wg_free(ctx, x->d_values);
    delete x;
    return WAHGPU_OK;
}

extern "C" int64_t wahgpu_index_nbitmaps(wahgpu_index* x) { return x ? (int64_t)x->nobs : WAHGPU_EINVAL; }
extern "C" int64_t wahgpu_index_nrows(wahgpu_index* x) { return x ? (int64_t)x->nrows : WAHGPU_EINVAL; }

// estimate(count) of relic / bin (src/irelic.cpp:1843, src/ibin.cpp:6832):
// the 1 bits of all bitmaps.
extern "C" int64_t wahgpu_index_total_ones(wahgpu_index* x) {
    if (!x) return WAHGPU_EINVAL;
    uint64_t s = 0;
    for (uint32_t v : x->bones) s += v;
    return (int64_t)s;
}

// ------------------------------------------------------------------ locate
static bool pass_h(double v, int lop, double lo, int rop, double hi) {
    const bool a = lop == 0 ? true : (lop == 1 ? lo < v : lo <= v);
    const bool b = rop == 0 ? true : (rop == 1 ? v < hi : v <= hi);
    return a && b;
}

// Which bitmaps a range covers: every value of bitmaps [h0, h1) passes, the
// rows of the cand[] bitmaps must be checked, the others hold no passing
// value.  relic (src/irelic.cpp:1416-1809): a bitmap per key; bin
// (src/ibin.cpp:7596-8460): a bin whose [minval, maxval] lies inside the
// range passes whole, one that straddles an end is checked.
// Term modes: the hits (LOC_HITS); the rows certainly hit, i.e. the
// bitmaps wholly inside without the edge bins (LOC_LOWER); the candidate
// rows, the wholly-inside bitmaps and the edge bins OR'ed whole (LOC_UPPER)
// — the lower and upper bounds of bin::estimate(expr, lower, upper),
// src/ibin.cpp:6722-6829.
enum LocMode { LOC_HITS = 0, LOC_LOWER = 1, LOC_UPPER = 2 };

static int locate(wahgpu_ctx* ctx, const wahgpu_index* x, const wahgpu_term* t, DevTerm& out,
                  int mode = LOC_HITS) {
    out = DevTerm{};
    out.lop = (uint32_t)t->lop; out.rop = (uint32_t)t->rop; out.lo = t->lo; out.hi = t->hi;
    uint32_t h0 = 0, h1 = 0, nc = 0;
    if (x->kind == WAHGPU_RELIC) {
        // keys ascending: the passing keys are one interval, found by the
        // same double comparisons (qContinuousRange::inRange) as the scan
        const auto& k = x->keys;
        uint32_t a = 0, b = x->nobs;
        if (t->lop == 1) a = (uint32_t)(std::upper_bound(k.begin(), k.end(), t->lo) - k.begin());
        else if (t->lop == 2) a = (uint32_t)(std::lower_bound(k.begin(), k.end(), t->lo) - k.begin());
        if (t->rop == 1) b = (uint32_t)(std::lower_bound(k.begin(), k.end(), t->hi) - k.begin());
        else if (t->rop == 2) b = (uint32_t)(std::upper_bound(k.begin(), k.end(), t->hi) - k.begin());
        if (b > a) { h0 = a; h1 = b; }
    } else if (x->bins_sorted) {
        // bins ordered and disjoint: every test below is monotone in the bin
        // order, so binary searches over the bins holding rows find the
        // bins wholly inside and the (at most two) straddling ones
        const auto& ne = x->nonempty;
        const uint32_t nb = x->nobs, m = (uint32_t)ne.size();
        auto mn = [&](uint32_t i) { return x->keys[ne[i]]; };
        auto mx = [&](uint32_t i) { return x->keys[nb + ne[i]]; };
        auto low = [&](double v) { return t->lop == 0 || (t->lop == 1 ? t->lo < v : t->lo <= v); };
        auto high = [&](double v) { return t->rop == 0 || (t->rop == 1 ? v < t->hi : v <= t->hi); };
        auto first = [&](auto pred) {  // first i with pred(i), pred monotone false..true
            uint32_t lo = 0, hi = m;
            while (lo < hi) { const uint32_t md = (lo + hi) / 2; if (pred(md)) hi = md; else lo = md + 1; }
            return lo;
        };
        const uint32_t P = first([&](uint32_t i) { return low(mx(i)); });        // some value passes the lower side
        const uint32_t Q = first([&](uint32_t i) { return !high(mn(i)); });      // [P, Q): some value passes both
        const uint32_t I0 = first([&](uint32_t i) { return low(mn(i)); });       // every value passes the lower side
        const uint32_t I1 = first([&](uint32_t i) { return !high(mx(i)); });     // [.., I1): every value passes the upper
        const uint32_t a = std::max(P, I0), b = std::min(Q, I1);
        if (b > a) { h0 = ne[a]; h1 = ne[b - 1] + 1; }
        for (uint32_t i = P; i < Q; ++i) {
            if (i >= a && i < b) { i = b - 1; continue; }
            if (nc >= 2) return wg_fail(ctx, WAHGPU_EINVAL, "more than two bins straddle the range");
            out.cand[nc++] = ne[i];
        }
    } else {
        std::vector<uint8_t> cls(x->nobs);  // 0 none, 1 all, 2 some
        for (uint32_t j = 0; j < x->nobs; ++j) {
            const double mn = x->keys[j], mx = x->keys[x->nobs + j];
            if (x->bones[j] == 0 || !(mn <= mx)) { cls[j] = 0; continue; }
            const bool pmn = pass_h(mn, t->lop, t->lo, t->rop, t->hi), pmx = pass_h(mx, t->lop, t->lo, t->rop, t->hi);
            if (pmn && pmx) cls[j] = 1;
            else {
                // no value in [mn, mx] passes when the range lies wholly on one side
                const bool below = t->rop != 0 && (t->rop == 1 ? !(mn < t->hi) : !(mn <= t->hi));
                const bool above = t->lop != 0 && (t->lop == 1 ? !(t->lo < mx) : !(t->lo <= mx));
                cls[j] = (below || above) ? 0 : 2;
            }
        }
        h0 = x->nobs; h1 = x->nobs;
        for (uint32_t j = 0; j < x->nobs; ++j) {
            if (cls[j] == 1) { if (h0 == x->nobs) h0 = j; h1 = j + 1; }
            else if (cls[j] == 2) {
                if (nc >= 2) return wg_fail(ctx, WAHGPU_EINVAL, "more than two bins straddle the range");
                out.cand[nc++] = j;
            }
        }
        if (h0 == x->nobs) { h0 = 0; h1 = 0; }
        for (uint32_t j = h0; j < h1; ++j)
            if (cls[j] == 0 && x->bones[j] != 0)
                return wg_fail(ctx, WAHGPU_EINVAL, "bitmaps wholly inside the range are not contiguous");
            else if (cls[j] == 2)
                return wg_fail(ctx, WAHGPU_EINVAL, "bitmaps wholly inside the range are not contiguous");
    }
    if (mode == LOC_LOWER) {
        nc = 0;
    } else if (mode == LOC_UPPER && nc > 0) {
        // the edge bins join the span (they are adjacent to it: every bin
        // between two straddling bins lies wholly inside)
        uint32_t a = h1 > h0 ? h0 : out.cand[0], b = h1 > h0 ? h1 : out.cand[0] + 1u;
        for (uint32_t c = 0; c < nc; ++c) { a = std::min(a, out.cand[c]); b = std::max(b, out.cand[c] + 1u); }
        h0 = a; h1 = b; nc = 0;
    }
    if (nc > 0 && !x->d_values)
        return wg_fail(ctx, WAHGPU_EINVAL, "range needs row checks but the index has no raw values attached");
    out.h0 = h0; out.h1 = h1; out.ncand = nc;
    if (x->cum_k && h1 > h0) {
        // C(k1) & ~C(k0) covers [k0*S, k1*S); the rest are edge bitmaps
        const uint32_t S = x->cum_stride;
        const uint32_t k0 = (h0 + S - 1) / S, k1 = std::min(h1 / S, x->cum_k);
        // worth it when the span's words outweigh the dense rows read instead
        const uint64_t span = k1 > k0 ? x->cum_words[k1 * S] - x->cum_words[k0 * S] : 0;
        const uint64_t gx = ((uint64_t)x->groups + (x->anb ? 1 : 0) + 3) & ~3ull;
        if (k1 > k0 && 4 * span >= (k0 ? 2 : 1) * gx) {
            out.c0 = k0; out.c1 = k1; out.e0 = k0 * S; out.e1 = k1 * S;
            out.flip = 0;
            return WAHGPU_OK;
        }
    }
    // sumBins reads the complement when the range holds more than half the
    // index's words (src/index.cpp:6490); the bits are the same either way
    const uint64_t in = x->cum_words[h1] - x->cum_words[h0], all = x->cum_words[x->nobs];
    out.flip = (2 * in > all) ? 1u : 0u;
    return WAHGPU_OK;
}

// Estimated hits of a located term (its bitmaps' 1 bits), for ordering the
// terms of a query: the most selective first, so a tile whose AND is
// already empty skips the rest.
static uint64_t term_estimate(const wahgpu_index* x, const DevTerm& d) {
    uint64_t e = x->cum_ones[d.h1] - x->cum_ones[d.h0];
    for (uint32_t c = 0; c < d.ncand; ++c) e += x->bones[d.cand[c]];
    return e;
}

// ------------------------------------------------------------------ batches
static int batch_create(wahgpu_ctx* ctx, const wahgpu_term* terms, const uint32_t* query_offsets,
                        uint32_t nq, uint64_t rid_cap, int dense_first, int mode, const uint64_t* caps,
                        wahgpu_batch** out);

extern "C" int wahgpu_batch_create(wahgpu_ctx* ctx, const wahgpu_term* terms, const uint32_t* query_offsets,
                                   uint32_t nq, uint64_t rid_cap, int dense_first, wahgpu_batch** out) {
    return batch_create(ctx, terms, query_offsets, nq, rid_cap, dense_first, LOC_HITS, nullptr, out);
}

// Row ids with a limit per query (the first rid_caps[q] of query q, in row
// order, like a LIMIT); every query's ids land in a region of its own.
extern "C" int wahgpu_batch_create_capped(wahgpu_ctx* ctx, const wahgpu_term* terms, const uint32_t* query_offsets,
                                          uint32_t nq, const uint64_t* rid_caps, wahgpu_batch** out) {
    if (!rid_caps) return wg_fail(ctx, WAHGPU_EINVAL, "rid_caps is NULL");
    uint64_t tot = 0;
    for (uint32_t q = 0; q < nq; ++q) tot += rid_caps[q];
    return batch_create(ctx, terms, query_offsets, nq, tot, 0, LOC_HITS, rid_caps, out);
}

static int batch_create(wahgpu_ctx* ctx, const wahgpu_term* terms, const uint32_t* query_offsets,
                        uint32_t nq, uint64_t rid_cap, int dense_first, int mode, const uint64_t* caps,
                        wahgpu_batch** out) {
    if (!ctx || !out || !terms || !query_offsets || nq == 0) return wg_fail(ctx, WAHGPU_EINVAL, "bad argument");
    *out = nullptr;
    const uint32_t nt = query_offsets[nq];
    if (query_offsets[0] != 0 || nt == 0) return wg_fail(ctx, WAHGPU_EINVAL, "bad query offsets");
    const wahgpu_index* x0 = terms[0].idx;
    if (!x0) return wg_fail(ctx, WAHGPU_EINVAL, "term without an index");
    std::vector<const wahgpu_index*> idx;
    std::vector<DevTerm> dt(nt);
    uint64_t bytes = 0, min_bytes = 0;
    for (uint32_t i = 0; i < nt; ++i) {
        const wahgpu_index* x = terms[i].idx;
        if (!x || x->nrows != x0->nrows) return wg_fail(ctx, WAHGPU_EINVAL, "term %u: indexes of one batch must share their row count", i);
        int rc = locate(ctx, x, &terms[i], dt[i], mode);
        if (rc) return rc;
        auto it = std::find(idx.begin(), idx.end(), x);
        dt[i].index = (uint32_t)(it - idx.begin());
        if (it == idx.end()) idx.push_back(x);
        // bytes the term reads: the OR'ed bitmaps' words, the edge bitmaps'
        // words and the raw value of each of their rows
        const uint64_t in = x->cum_words[dt[i].h1] - x->cum_words[dt[i].h0];
        if (dt[i].c1)
            bytes += 4 * ((dt[i].c0 ? 2 : 1) * ((uint64_t)x->groups + (x->anb ? 1 : 0)) +
                          (x->cum_words[dt[i].e0] - x->cum_words[dt[i].h0]) +
                          (x->cum_words[dt[i].h1] - x->cum_words[dt[i].e1]));
        else
            bytes += 4 * (dt[i].flip ? x->cum_words[x->nobs] - in : in);
        for (uint32_t c = 0; c < dt[i].ncand; ++c)
            bytes += 4 * (x->bwords[dt[i].cand[c]] + x->bones[dt[i].cand[c]]);
        // what sumBins itself must read: the covered bitmaps or, when they
        // hold more than half the words, their complement
        // (src/index.cpp:6490), plus the edge bitmaps and their rows
        min_bytes += 4 * std::min(in, x->cum_words[x->nobs] - in);
        for (uint32_t c = 0; c < dt[i].ncand; ++c)
            min_bytes += 4 * (x->bwords[dt[i].cand[c]] + x->bones[dt[i].cand[c]]);
    }
    std::vector<DevQuery> dq(nq);
    for (uint32_t q = 0; q < nq; ++q) {
        if (query_offsets[q + 1] <= query_offsets[q] || query_offsets[q + 1] > nt)
            return wg_fail(ctx, WAHGPU_EINVAL, "query %u has no term", q);
        dq[q].t0 = query_offsets[q]; dq[q].t1 = query_offsets[q + 1];
        dq[q].rid_base = q ? dq[q - 1].rid_base + (caps ? caps[q - 1] : 0) : 0;
        dq[q].rid_lim = caps ? caps[q] : 0;
        std::stable_sort(dt.begin() + dq[q].t0, dt.begin() + dq[q].t1, [&](const DevTerm& a, const DevTerm& b) {
            return term_estimate(idx[a.index], a) < term_estimate(idx[b.index], b);
        });
    }
    std::vector<DevIndex> di;
    for (auto* x : idx) di.push_back(x->dev);
    wahgpu_batch* B = new wahgpu_batch();
    B->ctx = ctx; B->nq = nq; B->nterms = nt; B->nidx = (uint32_t)idx.size();
    B->bytes = bytes + 8ull * nq;
    B->min_bytes = min_bytes + 8ull * nq;
    B->groups = x0->groups; B->anb = x0->anb; B->ntiles = x0->ntiles;
    B->d_idx = static_cast<DevIndex*>(wg_alloc(ctx, di.size() * sizeof(DevIndex)));
    B->d_terms = static_cast<DevTerm*>(wg_alloc(ctx, nt * sizeof(DevTerm)));
    B->d_queries = static_cast<DevQuery*>(wg_alloc(ctx, nq * sizeof(DevQuery)));
    B->d_counts = static_cast<unsigned long long*>(wg_alloc(ctx, nq * 8));
    B->d_start = static_cast<unsigned long long*>(wg_alloc(ctx, nq * 8));
    B->d_status = static_cast<DevMeta*>(wg_alloc(ctx, sizeof(DevMeta)));
    B->rid_cap = rid_cap;
    B->capped = caps != nullptr;
    if (caps) {
        B->h_lim.assign(caps, caps + nq);
        B->h_base.resize(nq);
        for (uint32_t q = 0; q < nq; ++q) B->h_base[q] = dq[q].rid_base;
    }
    if (rid_cap) B->d_rids = static_cast<uint32_t*>(wg_alloc(ctx, rid_cap * 4));
    if (dense_first) B->d_dense = static_cast<uint32_t*>(wg_alloc(ctx, ((size_t)x0->groups + 1) * 4));
    if (!B->d_idx || !B->d_terms || !B->d_queries || !B->d_counts || !B->d_start || !B->d_status ||
        (rid_cap && !B->d_rids) || (dense_first && !B->d_dense)) {
        wahgpu_batch_free(B);
        return wg_fail(ctx, WAHGPU_ENOMEM, "batch allocation failed");
    }
    // the tables leave from pinned staging the batch keeps until it is
    // freed, so the host does not wait for the copies
    const size_t bi = di.size() * sizeof(DevIndex), bt = (size_t)nt * sizeof(DevTerm), bq = (size_t)nq * sizeof(DevQuery);
    B->h_stage = static_cast<unsigned char*>(wg_host_alloc(ctx, bi + bt + bq));
    if (!B->h_stage) {
        wahgpu_batch_free(B);
        return wg_fail(ctx, WAHGPU_ENOMEM, "batch staging allocation failed");
    }
    memcpy(B->h_stage, di.data(), bi);
    memcpy(B->h_stage + bi, dt.data(), bt);
    memcpy(B->h_stage + bi + bt, dq.data(), bq);
    CUDA_TRY(ctx, cudaMemcpyAsync(B->d_idx, B->h_stage, bi, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(B->d_terms, B->h_stage + bi, bt, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(B->d_queries, B->h_stage + bi + bt, bq, cudaMemcpyHostToDevice, ctx->stream));
    *out = B;
    return WAHGPU_OK;
}

extern "C" int wahgpu_batch_run(wahgpu_batch* B) {
    if (!B) return WAHGPU_EINVAL;
    wahgpu_ctx* ctx = B->ctx;
    const uint32_t nitems = B->nq * B->ntiles;
    if (nitems == 0) return WAHGPU_OK;
    TileRec* recs; LaunchSync* sync;
    int rc = wg_scratch(ctx, nitems, &recs, &sync);
    if (rc) return rc;
    CUDA_TRY(ctx, cudaMemsetAsync(B->d_counts, 0, B->nq * 8, ctx->stream));
    CUDA_TRY(ctx, cudaMemsetAsync(B->d_status, 0, sizeof(DevMeta), ctx->stream));
    RangeArgs a;
    a.idx = B->d_idx; a.terms = B->d_terms; a.queries = B->d_queries; a.nq = B->nq;
    a.groups = B->groups; a.anb = B->anb; a.ntiles = B->ntiles;
    a.counts = B->d_counts; a.rids = B->d_rids; a.rid_cap = B->rid_cap; a.rid_start = B->d_start;
    a.dense = B->d_dense;
    a.recs = recs; a.sync = sync; a.nitems = nitems; a.status = B->d_status;
    // tile by tile when only counts are wanted (orders 1 and 2); with row ids
    // order 2 runs two tile-by-tile passes around a scan of the items' hits,
    // order 1 (and a single query) goes query by query with the look-back
    const bool ids = B->d_rids || B->d_dense;
    const bool two_pass = ctx->range_order == 2 && ids && B->nq > 1;
    a.tile_major = ((ctx->range_order != 0 && !ids) || two_pass) ? 1u : 0u;
    a.pass = 0; a.item_cnt = nullptr; a.item_off = nullptr;
    a.capped = B->capped && B->d_rids ? 1u : 0u;
    if (two_pass) {
        if (!B->d_items) {
            B->d_items = static_cast<unsigned long long*>(wg_alloc(ctx, (size_t)nitems * 16));
            cub::DeviceScan::ExclusiveSum(nullptr, B->scan_tmp_bytes, B->d_items, B->d_items + nitems, (int)nitems,
                                          ctx->stream);
            B->d_scan_tmp = wg_alloc(ctx, std::max<size_t>(B->scan_tmp_bytes, 16));
            if (!B->d_items || !B->d_scan_tmp) {
                wg_free(ctx, B->d_items); wg_free(ctx, B->d_scan_tmp);
                B->d_items = nullptr; B->d_scan_tmp = nullptr;
                return wg_fail(ctx, WAHGPU_ENOMEM, "two-pass item arrays: allocation failed");
            }
        }
        if (B->d_dense) CUDA_TRY(ctx, cudaMemsetAsync(B->d_dense, 0, ((size_t)B->groups + 1) * 4, ctx->stream));
    }
    static PerDeviceSetup setup;
    const size_t sm = sizeof(RangeShared);
    const int per_sm = wg_kernel_setup(setup, ctx->device, k_range, RTHREADS, sm);
    const uint32_t ctas = ctx->range_ctas ? std::min<uint32_t>(ctx->range_ctas, (uint32_t)per_sm) : (uint32_t)per_sm;
    const uint32_t grid = std::min<uint32_t>(nitems, ctas * (uint32_t)ctx->sm_count);
    if (two_pass) {
        a.pass = 1; a.item_cnt = B->d_items;
        k_range<<<grid, RTHREADS, sm, ctx->stream>>>(a);
        CUDA_TRY(ctx, cudaGetLastError());
        CUDA_TRY(ctx, cub::DeviceScan::ExclusiveSum(B->d_scan_tmp, B->scan_tmp_bytes, B->d_items, B->d_items + nitems,
                                                    (int)nitems, ctx->stream));
        a.pass = 2; a.item_off = B->d_items + nitems;
        ctx->launches += 2;  // the count pass and the scan
    }
    k_range<<<grid, RTHREADS, sm, ctx->stream>>>(a);
    ctx->launches++;
    CUDA_TRY(ctx, cudaGetLastError());
    B->h_valid = false;
    return WAHGPU_OK;
}

static int batch_fetch(wahgpu_batch* B) {
    if (B->h_valid) return WAHGPU_OK;
    wahgpu_ctx* ctx = B->ctx;
    B->h_counts.resize(B->nq);
    B->h_start.resize(B->nq);
    DevMeta st{};
    CUDA_TRY(ctx, cudaMemcpyAsync(B->h_counts.data(), B->d_counts, B->nq * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(B->h_start.data(), B->d_start, B->nq * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(&st, B->d_status, sizeof(DevMeta), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (st.status == DEV_ERR_TIMEOUT) return wg_fail(ctx, WAHGPU_ETIMEOUT, "a device-side look-back wait gave up");
    B->h_valid = true;
    return WAHGPU_OK;
}

extern "C" int wahgpu_batch_counts(wahgpu_batch* B, uint64_t* counts) {
    if (!B || !counts) return WAHGPU_EINVAL;
    int rc = batch_fetch(B);
    if (rc) return rc;
    for (uint32_t q = 0; q < B->nq; ++q) counts[q] = B->h_counts[q];
    return WAHGPU_OK;
}

extern "C" int64_t wahgpu_batch_rids(wahgpu_batch* B, uint32_t q, uint32_t* out, uint64_t cap) {
    if (!B || q >= B->nq || (cap && !out)) return WAHGPU_EINVAL;
    wahgpu_ctx* ctx = B->ctx;
    int rc = batch_fetch(B);
    if (rc) return rc;
    const uint64_t n = B->capped ? std::min<uint64_t>(B->h_counts[q], B->h_lim[q]) : B->h_counts[q];
    const uint64_t s = B->capped ? B->h_base[q] : B->h_start[q];
    if (!B->d_rids || s + n > B->rid_cap) return wg_fail(ctx, WAHGPU_ESIZE, "row ids exceed the batch's capacity");
    if (cap < n) return wg_fail(ctx, WAHGPU_ESIZE, "need room for %llu row ids", (unsigned long long)n);
    if (n) {
        CUDA_TRY(ctx, cudaMemcpyAsync(out, B->d_rids + s, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return (int64_t)n;
}

extern "C" const uint32_t* wahgpu_batch_device_rids(wahgpu_batch* B) { return B ? B->d_rids : nullptr; }

// Every query's count and the whole row-id buffer (rid_cap words) in one
// round trip, for a caller that answers all the queries of a capped batch
// at once: query q's ids are rids[h_base[q], h_base[q] + min(count, limit)).
int wg_batch_fetch_all(wahgpu_batch* B, uint32_t* rids) {
    wahgpu_ctx* ctx = B->ctx;
    if (B->h_valid) return WAHGPU_OK;
    B->h_counts.resize(B->nq);
    B->h_start.resize(B->nq);
    DevMeta st{};
    CUDA_TRY(ctx, cudaMemcpyAsync(B->h_counts.data(), B->d_counts, B->nq * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(B->h_start.data(), B->d_start, B->nq * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(&st, B->d_status, sizeof(DevMeta), cudaMemcpyDeviceToHost, ctx->stream));
    if (rids && B->d_rids && B->rid_cap)
        CUDA_TRY(ctx, cudaMemcpyAsync(rids, B->d_rids, B->rid_cap * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (st.status == DEV_ERR_TIMEOUT) return wg_fail(ctx, WAHGPU_ETIMEOUT, "a device-side look-back wait gave up");
    B->h_valid = true;
    return WAHGPU_OK;
}

// Algorithmic bytes of one run: per term the words of the bitmaps it ORs
// (or of their complement), of its edge bitmaps and the raw values of the
// edge bitmaps' rows; 8 per query for its count.
extern "C" int64_t wahgpu_batch_bytes(wahgpu_batch* B) { return B ? (int64_t)B->bytes : WAHGPU_EINVAL; }
// Bytes any evaluation of the batch must move, whatever its index layout:
// per term the words of the bitmaps sumBins ORs (the covered set, or its
// complement when that is smaller, src/index.cpp:6490), the edge bitmaps'
// words and one raw value per edge row; 8 bytes per count.
extern "C" int64_t wahgpu_batch_min_bytes(wahgpu_batch* B) { return B ? (int64_t)B->min_bytes : WAHGPU_EINVAL; }

extern "C" int wahgpu_batch_free(wahgpu_batch* B) {
    if (!B) return WAHGPU_EINVAL;
    wahgpu_ctx* ctx = B->ctx;
    cudaStreamSynchronize(ctx->stream);
    wg_free(ctx, B->d_idx); wg_free(ctx, B->d_terms); wg_free(ctx, B->d_queries);
    wg_free(ctx, B->d_counts); wg_free(ctx, B->d_start); wg_free(ctx, B->d_status);
    wg_free(ctx, B->d_rids); wg_free(ctx, B->d_dense);
    wg_free(ctx, B->d_items); wg_free(ctx, B->d_scan_tmp);
    wg_host_free(ctx, B->h_stage);
    delete B;
    return WAHGPU_OK;
}

// One conjunctive query (countQuery::evaluate, src/countQuery.cpp:292):
// returns the hit count; row ids into host memory when out is given; the hit
// bitvector (compress()ed) when hits is given.
static int64_t evaluate_mode(wahgpu_ctx* ctx, const wahgpu_term* terms, uint32_t nterms, uint32_t* rids,
                             uint64_t cap, wahgpu_bv** hits, int mode);

extern "C" int64_t wahgpu_evaluate(wahgpu_ctx* ctx, const wahgpu_term* terms, uint32_t nterms,
                                   uint32_t* rids, uint64_t cap, wahgpu_bv** hits) {
    return evaluate_mode(ctx, terms, nterms, rids, cap, hits, LOC_HITS);
}

// index::estimate(expr, lower, upper) (src/index.h:191; relic,
// src/irelic.h:58-62: lower = the hits, upper empty; bin,
// src/ibin.cpp:6722-6829: lower = the bins wholly inside, upper = lower and
// the edge bins, empty when there is no edge bin).  An empty upper means
// lower is exact, the reference's convention.
extern "C" int wahgpu_estimate(wahgpu_ctx* ctx, const wahgpu_term* term, wahgpu_bv** lower, wahgpu_bv** upper) {
    if (!ctx || !term || !term->idx || !lower || !upper) return wg_fail(ctx, WAHGPU_EINVAL, "bad argument");
    *lower = nullptr;
    *upper = nullptr;
    DevTerm dl, du;  // no edge bin when the two spans agree
    int rc = locate(ctx, term->idx, term, dl, LOC_LOWER);
    if (!rc) rc = locate(ctx, term->idx, term, du, LOC_UPPER);
    if (rc) return rc;
    const bool exact = dl.h0 == du.h0 && dl.h1 == du.h1;
    int64_t n = evaluate_mode(ctx, term, 1, nullptr, 0, lower, LOC_LOWER);
    if (n < 0) return (int)n;
    if (exact) {
        rc = wahgpu_bv_create(ctx, 1, upper);
    } else {
        n = evaluate_mode(ctx, term, 1, nullptr, 0, upper, LOC_UPPER);
        rc = n < 0 ? (int)n : WAHGPU_OK;
    }
    if (rc) { wahgpu_bv_free(*lower); *lower = nullptr; }
    return rc;
}

// index::estimate(expr) (src/index.h:196): an upper bound of the hit count —
// relic: the exact count (src/irelic.cpp:1843-1854); bin: the 1 bits of the
// bins wholly inside and of the edge bins (src/ibin.cpp:6832-6889).  From
// the host-side per-bitmap counts; no device work.
extern "C" int64_t wahgpu_estimate_count(wahgpu_ctx* ctx, const wahgpu_term* term) {
    if (!ctx || !term || !term->idx) return wg_fail(ctx, WAHGPU_EINVAL, "bad argument");
    const wahgpu_index* x = term->idx;
    DevTerm d;
    const int rc = locate(ctx, x, term, d, LOC_UPPER);
    if (rc) return rc;
    return (int64_t)(x->cum_ones[d.h1] - x->cum_ones[d.h0]);
}

static int64_t evaluate_mode(wahgpu_ctx* ctx, const wahgpu_term* terms, uint32_t nterms, uint32_t* rids,
                             uint64_t cap, wahgpu_bv** hits, int mode) {
    if (!ctx || !terms || nterms == 0 || (cap && !rids)) return wg_fail(ctx, WAHGPU_EINVAL, "bad argument");
    const uint32_t qo[2] = {0, nterms};
    wahgpu_batch* B = nullptr;
    int rc = batch_create(ctx, terms, qo, 1, rids ? cap : 0, hits ? 1 : 0, mode, nullptr, &B);
    if (rc) return rc;
    rc = wahgpu_batch_run(B);
    uint64_t cnt = 0;
    if (!rc) rc = wahgpu_batch_counts(B, &cnt);
    if (!rc && rids) {
        int64_t n = wahgpu_batch_rids(B, 0, rids, cap);
        if (n < 0) rc = (int)n;
    }
    if (!rc && hits) {
        // the dense hit words become a bitvector; compress() gives the
        // canonical words the reference holds after compress()
        const wahgpu_index* x = terms[0].idx;
        wahgpu_bv* hv = nullptr;
        rc = wahgpu_bv_create(ctx, (uint64_t)x->groups + 1, &hv);
        if (!rc) {
            wahgpu_bv* b = hv;
            uint32_t aval = 0;
            if (x->anb) {
                uint32_t last = 0;
                cudaMemcpyAsync(&last, B->d_dense + x->groups, 4, cudaMemcpyDeviceToHost, ctx->stream);
                cudaStreamSynchronize(ctx->stream);
                aval = last >> (31u - x->anb);
            }
            cudaMemcpyAsync(b->words, B->d_dense, (size_t)x->groups * 4, cudaMemcpyDeviceToDevice, ctx->stream);
            rc = wg_scan_meta(b, x->groups, x->anb, aval);
            if (!rc) rc = wahgpu_bv_compress(b);
            if (!rc) *hits = hv; else wahgpu_bv_free(hv);
        }
    }
    wahgpu_batch_free(B);
    return rc ? rc : (int64_t)cnt;
}
