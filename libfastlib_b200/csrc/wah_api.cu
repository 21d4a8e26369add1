// C ABI of libwahgpu: contexts, device bitvectors, operators.
// Declarations and the reference interfaces they replace: include/wahgpu.h.
#include "../../include/wahgpu.h"
#include "wah_plan.h"
#include "wah_merge.cuh"
#include "wah_kernels.cuh"
#include "wah_gop.cuh"
#include "wah_fuse.cuh"
#include "wah_gone.cuh"
#include "wah_api_internal.h"

#include <cuda_runtime.h>
#include <algorithm>
#include <cstdio>
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <map>
#include <vector>
#include <string>

using namespace wah;

// ------------------------------------------------------------------ errors
static thread_local std::string g_tls_err;

int wg_fail(wahgpu_ctx* ctx, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (ctx) ctx->err = buf; else g_tls_err = buf;
    return code;
}
#define CUDA_TRY(ctx, call)                                                            \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return wg_fail(ctx, WAHGPU_ECUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// -------------------------------------------------------------- allocator
static size_t size_class(size_t b) {
    if (b < 256) return 256;
    if (b <= (1u << 20)) { size_t c = 256; while (c < b) c <<= 1; return c; }
    return (b + (1u << 20) - 1) & ~(size_t)((1u << 20) - 1);
}
void* wg_alloc(wahgpu_ctx* ctx, size_t bytes) {
    size_t c = size_class(bytes);
    {
        std::lock_guard<std::mutex> g(ctx->mu);
        if (ctx->test_fail_alloc > 0 && --ctx->test_fail_alloc == 0) return nullptr;  // test hook
        auto it = ctx->pool.find(c);
        if (it != ctx->pool.end() && !it->second.empty()) {
            void* p = it->second.back();
            it->second.pop_back();
            return p;
        }
    }
    void* p = nullptr;
    if (cudaMalloc(&p, c) != cudaSuccess) {
        // release cached blocks and retry once
        cudaStreamSynchronize(ctx->stream);
        std::lock_guard<std::mutex> g(ctx->mu);
        for (auto& kv : ctx->pool)
            for (void* q : kv.second) {
                cudaFree(q);
                ctx->sizes.erase(q);
                ctx->bytes_allocated -= kv.first;
            }
        ctx->pool.clear();
        cudaGetLastError();
        if (cudaMalloc(&p, c) != cudaSuccess) { cudaGetLastError(); return nullptr; }
    }
    std::lock_guard<std::mutex> g(ctx->mu);
    ctx->sizes[p] = c;
    ctx->bytes_allocated += c;
    return p;
}
void wg_free(wahgpu_ctx* ctx, void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> g(ctx->mu);
    auto it = ctx->sizes.find(p);
    if (it == ctx->sizes.end()) return;
    ctx->pool[it->second].push_back(p);
}

// Pinned host blocks, pooled by size class like the device blocks: staging
// for copies that must not wait for the host (a block goes back to the pool
// only once the copies reading it are known to be done).
void* wg_host_alloc(wahgpu_ctx* ctx, size_t bytes) {
    const size_t c = size_class(bytes);
    {
        std::lock_guard<std::mutex> g(ctx->mu);
        auto it = ctx->hpool.find(c);
        if (it != ctx->hpool.end() && !it->second.empty()) {
            void* p = it->second.back();
            it->second.pop_back();
            return p;
        }
    }
    void* p = nullptr;
    if (cudaMallocHost(&p, c) != cudaSuccess) { cudaGetLastError(); return nullptr; }
    std::lock_guard<std::mutex> g(ctx->mu);
    ctx->hsizes[p] = c;
    return p;
}
void wg_host_free(wahgpu_ctx* ctx, void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> g(ctx->mu);
    auto it = ctx->hsizes.find(p);
    if (it == ctx->hsizes.end()) return;
    ctx->hpool[it->second].push_back(p);
}

// Scratch for the look-back scans: tile records plus the launch sync words.
int wg_scratch(wahgpu_ctx* ctx, uint32_t ntiles, TileRec** recs, LaunchSync** sync) {
    if (ntiles > ctx->scratch_tiles) {
        uint32_t want = ntiles < 1024 ? 1024 : ntiles + ntiles / 2;
        CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        if (ctx->scratch) cudaFree(ctx->scratch);
        ctx->scratch = nullptr;
        // sync words, TileRec records, then the dense kernel's 16-byte
        // records and the single-pass kernel's (each format in a region of
        // its own, so a stale record of one is never read by the other)
        size_t bytes = sizeof(LaunchSync) * 2 + (size_t)want * (sizeof(TileRec) + 2 * sizeof(uint4));
        if (cudaMalloc(&ctx->scratch, bytes) != cudaSuccess) {
            cudaGetLastError();
            ctx->scratch_tiles = 0;
            return wg_fail(ctx, WAHGPU_ENOMEM, "scratch allocation of %zu bytes failed", bytes);
        }
        CUDA_TRY(ctx, cudaMemsetAsync(ctx->scratch, 0, bytes, ctx->stream));
        ctx->scratch_tiles = want;
    }
    *sync = reinterpret_cast<LaunchSync*>(ctx->scratch);
    *recs = reinterpret_cast<TileRec*>(reinterpret_cast<char*>(ctx->scratch) + 2 * sizeof(LaunchSync));
    return WAHGPU_OK;
}
// The dense kernel's records, after the TileRec array of the scratch block.
static uint4* wg_dense_recs(wahgpu_ctx* ctx, TileRec* recs) {
    return reinterpret_cast<uint4*>(recs + ctx->scratch_tiles);
}
// The single-pass group-space kernel's records, after the dense kernel's.
static uint4* wg_fuse_recs(wahgpu_ctx* ctx, TileRec* recs) {
    return wg_dense_recs(ctx, recs) + ctx->scratch_tiles;
}

// ------------------------------------------------------------------ context
extern "C" int wahgpu_ctx_create(int device, wahgpu_ctx** out) {
    if (!out) return wg_fail(nullptr, WAHGPU_EINVAL, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return wg_fail(nullptr, WAHGPU_ENODEV, "no CUDA device is available");
    }
    if (device < 0 || device >= ndev) return wg_fail(nullptr, WAHGPU_EINVAL, "bad device %d", device);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess)
        return wg_fail(nullptr, WAHGPU_ENODEV, "cannot query device %d", device);
    if (prop.major != 10)
        return wg_fail(nullptr, WAHGPU_ENODEV, "device %d is sm_%d%d; this build runs on sm_100 only",
                       device, prop.major, prop.minor);
    wahgpu_ctx* c = new wahgpu_ctx();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    cudaSetDevice(device);
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return wg_fail(nullptr, WAHGPU_ECUDA, "stream creation failed");
    }
    c->stream = c->own_stream;
    if (cudaMallocHost(&c->h_meta_stage, sizeof(DevMeta) * 4) != cudaSuccess) {
        cudaStreamDestroy(c->own_stream);
        delete c;
        return wg_fail(nullptr, WAHGPU_ENOMEM, "pinned staging allocation failed");
    }
    *out = c;
    return WAHGPU_OK;
}

extern "C" int wahgpu_ctx_destroy(wahgpu_ctx* ctx) {
    if (!ctx) return WAHGPU_EINVAL;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& kv : ctx->sizes) cudaFree(kv.first);
    for (auto& kv : ctx->hsizes) cudaFreeHost(kv.first);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->h_meta_stage) cudaFreeHost(ctx->h_meta_stage);
    cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return WAHGPU_OK;
}

extern "C" int wahgpu_ctx_set_stream(wahgpu_ctx* ctx, void* stream) {
    if (!ctx) return WAHGPU_EINVAL;
    ctx->stream = stream ? reinterpret_cast<cudaStream_t>(stream) : ctx->own_stream;
    return WAHGPU_OK;
}
extern "C" int wahgpu_ctx_set_tuning(wahgpu_ctx* ctx, int key, int64_t value) {
    if (!ctx) return WAHGPU_EINVAL;
    switch (key) {
    case WAHGPU_TUNE_DENSE_TILE:
        if (value != 1024 && value != 2048 && value != 4096)
            return wg_fail(ctx, WAHGPU_EINVAL, "dense tile must be 1024, 2048 or 4096 groups, not %lld", (long long)value);
        ctx->dense_tile = (uint32_t)value;
        return WAHGPU_OK;
    case WAHGPU_TUNE_DENSE_ENGINE:
        if (value < 0 || value > 5) return wg_fail(ctx, WAHGPU_EINVAL, "dense engine must be 0 .. 5");
        ctx->dense_engine = (uint32_t)value;
        return WAHGPU_OK;
    case WAHGPU_TUNE_RANGE_ORDER:
        if (value < 0 || value > 2) return wg_fail(ctx, WAHGPU_EINVAL, "range order must be 0, 1 or 2");
        ctx->range_order = (uint32_t)value;
        return WAHGPU_OK;
    case WAHGPU_TUNE_RANGE_CTAS:
        if (value < 0 || value > 32) return wg_fail(ctx, WAHGPU_EINVAL, "range CTAs per SM must be 0..32");
        ctx->range_ctas = (uint32_t)value;
        return WAHGPU_OK;
    case WAHGPU_TEST_WITHHOLD_TILE:
        ctx->test_withhold = value < 0 ? 0xFFFFFFFFu : (uint32_t)value;
        return WAHGPU_OK;
    case WAHGPU_TEST_FAIL_ALLOC:
        if (value < 0) return wg_fail(ctx, WAHGPU_EINVAL, "allocation count must be >= 0");
        ctx->test_fail_alloc = value;
        return WAHGPU_OK;
    case WAHGPU_TUNE_MERGE_TILE:
        if (value != 0 && value != 16 && value != 32 && value != 64)
            return wg_fail(ctx, WAHGPU_EINVAL, "merge tile must be 0 (auto), 16, 32 or 64 entries, not %lld", (long long)value);
        ctx->merge_tile = (uint32_t)value;
        return WAHGPU_OK;
    case WAHGPU_TUNE_CUM_STRIDE:
        if (value < 0 || value > (1 << 30)) return wg_fail(ctx, WAHGPU_EINVAL, "cumulative stride must be 0 (auto), 1 (none) or a stride");
        ctx->cum_stride = (uint32_t)value;
        return WAHGPU_OK;
    default:
        return wg_fail(ctx, WAHGPU_EINVAL, "unknown tuning key %d", key);
    }
}
extern "C" int64_t wahgpu_ctx_get_tuning(wahgpu_ctx* ctx, int key) {
    if (!ctx) return WAHGPU_EINVAL;
    switch (key) {
    case WAHGPU_TUNE_DENSE_TILE: return ctx->dense_tile;
    case WAHGPU_TUNE_DENSE_ENGINE: return ctx->dense_engine;
    case WAHGPU_TUNE_RANGE_ORDER: return ctx->range_order;
    case WAHGPU_TUNE_RANGE_CTAS: return ctx->range_ctas;
    case WAHGPU_TUNE_CUM_STRIDE: return ctx->cum_stride;
    case WAHGPU_TUNE_MERGE_TILE: return ctx->merge_tile;
    default: return wg_fail(ctx, WAHGPU_EINVAL, "unknown tuning key %d", key);
    }
}
extern "C" void* wahgpu_ctx_stream(wahgpu_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }
extern "C" int wahgpu_ctx_sync(wahgpu_ctx* ctx) {
    if (!ctx) return WAHGPU_EINVAL;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return WAHGPU_OK;
}
extern "C" const char* wahgpu_last_error(wahgpu_ctx* ctx) {
    return ctx ? ctx->err.c_str() : g_tls_err.c_str();
}
extern "C" int64_t wahgpu_ctx_launches(wahgpu_ctx* ctx) { return ctx ? (int64_t)ctx->launches : -1; }

// --------------------------------------------------------------- bitvectors
static int bv_reserve(wahgpu_bv* b, uint64_t cap) {
    wahgpu_ctx* ctx = b->ctx;
    if (cap < 1) cap = 1;
    if (cap > 0xFFFFFFFFull) return wg_fail(ctx, WAHGPU_ERANGE, "capacity %llu words too large", (unsigned long long)cap);
    if (b->words && b->cap >= cap) return WAHGPU_OK;
    wg_free(ctx, b->words);
    wg_free(ctx, b->bpos);
    b->words = static_cast<uint32_t*>(wg_alloc(ctx, cap * 4));
    b->bpos = static_cast<uint32_t*>(wg_alloc(ctx, ((cap + 31) / 32 + 2) * 4));
    if (!b->words || !b->bpos) return wg_fail(ctx, WAHGPU_ENOMEM, "device allocation of %llu words failed", (unsigned long long)cap);
    b->cap = (uint32_t)cap;
    b->gt_valid = false;
    return WAHGPU_OK;
}

wahgpu_bv* wg_bv_new(wahgpu_ctx* ctx) {
    wahgpu_bv* b = new wahgpu_bv();
    b->ctx = ctx;
    b->meta = static_cast<DevMeta*>(wg_alloc(ctx, sizeof(DevMeta)));
    if (!b->meta) { delete b; return nullptr; }
    return b;
}

// Waits for the producer of b and copies its metadata to the host.
int wg_bv_meta(wahgpu_bv* b) {
    if (b->h_valid) return WAHGPU_OK;
    wahgpu_ctx* ctx = b->ctx;
    DevMeta* st = reinterpret_cast<DevMeta*>(ctx->h_meta_stage);
    CUDA_TRY(ctx, cudaMemcpyAsync(st, b->meta, sizeof(DevMeta), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    b->h = *st;
    b->h_valid = true;
    switch (b->h.status) {
    case 0: return WAHGPU_OK;
    case DEV_ERR_TIMEOUT: return wg_fail(ctx, WAHGPU_ETIMEOUT, "a device-side look-back wait gave up");
    case DEV_ERR_FORMAT: return wg_fail(ctx, WAHGPU_EFORMAT, "serialized bitvector holds a fill word of length 0");
    case DEV_ERR_RANGE: return wg_fail(ctx, WAHGPU_ERANGE, "bitvector holds more than 2^32-1 bits");
    default: return wg_fail(ctx, WAHGPU_ECUDA, "device status %u", b->h.status);
    }
}

// Launches the upload scan over b->words[0..n) (device data already there).
int wg_scan_meta(wahgpu_bv* b, uint32_t n, uint32_t anb, uint32_t aval) {
    wahgpu_ctx* ctx = b->ctx;
    CUDA_TRY(ctx, cudaMemsetAsync(b->meta, 0, sizeof(DevMeta), ctx->stream));
    if (n == 0) {
        k_small<<<1, 32, 0, ctx->stream>>>(0, 0, nullptr, nullptr, 0, 0, b->words, b->bpos, b->meta, anb, aval);
    } else {
        uint32_t ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
        TileRec* recs; LaunchSync* sync;
        int rc = wg_scratch(ctx, ntiles, &recs, &sync);
        if (rc) return rc;
        k_meta<<<ntiles, SCAN_THREADS, 0, ctx->stream>>>(b->words, n, b->bpos, b->meta, anb, aval, recs, sync, ntiles);
    }
    ctx->launches++;
    CUDA_TRY(ctx, cudaGetLastError());
    b->h_valid = false;
    return WAHGPU_OK;
}

static void parse_trailer(const uint32_t* tail2, uint64_t nwords, uint32_t& n, uint32_t& anb, uint32_t& aval) {
    // src/bitvector.cpp:54-105: the last word is the active bit count when it
    // is in 1..30 (then the word before is the active value); any other last
    // word is dropped and the active word is empty
    n = 0; anb = 0; aval = 0;
    if (nwords <= 1) return;
    const uint32_t last = tail2[1];
    if (last > 0 && last < MAXBITS) { anb = last; aval = tail2[0]; n = (uint32_t)(nwords - 2); }
    else n = (uint32_t)(nwords - 1);
}

extern "C" int wahgpu_bv_from_serial(wahgpu_ctx* ctx, const uint32_t* words, uint64_t nwords, wahgpu_bv** out) {
    if (!ctx || !out || (nwords && !words)) return wg_fail(ctx, WAHGPU_EINVAL, "bad argument");
    if (nwords > 0xFFFFFFFFull) return wg_fail(ctx, WAHGPU_ERANGE, "too many words");
    *out = nullptr;
    uint32_t n, anb, aval;
    uint32_t tail[2] = {0, 0};
    if (nwords >= 2) { tail[0] = words[nwords - 2]; tail[1] = words[nwords - 1]; }
    parse_trailer(tail, nwords, n, anb, aval);
    wahgpu_bv* b = wg_bv_new(ctx);
    if (!b) return wg_fail(ctx, WAHGPU_ENOMEM, "allocation failed");
    int rc = bv_reserve(b, n);
    if (rc) { wahgpu_bv_free(b); return rc; }
    if (n) {
        cudaError_t e = cudaMemcpyAsync(b->words, words, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) { wahgpu_bv_free(b); return wg_fail(ctx, WAHGPU_ECUDA, "upload failed: %s", cudaGetErrorString(e)); }
    }
    rc = wg_scan_meta(b, n, anb, aval);
    if (rc) { wahgpu_bv_free(b); return rc; }
    b->compressed_form = false;
    *out = b;
    return WAHGPU_OK;
}

extern "C" int wahgpu_bv_from_device_serial(wahgpu_ctx* ctx, const uint32_t* dev_words, uint64_t nwords,
                                            wahgpu_bv** out) {
    if (!ctx || !out || (nwords && !dev_words)) return wg_fail(ctx, WAHGPU_EINVAL, "bad argument");
    if (nwords > 0xFFFFFFFFull) return wg_fail(ctx, WAHGPU_ERANGE, "too many words");
    *out = nullptr;
    uint32_t tail[2] = {0, 0};
    if (nwords >= 2) {
        CUDA_TRY(ctx, cudaMemcpyAsync(tail, dev_words + nwords - 2, 8, cudaMemcpyDeviceToHost, ctx->stream));
        CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    }
    uint32_t n, anb, aval;
    parse_trailer(tail, nwords, n, anb, aval);
    wahgpu_bv* b = wg_bv_new(ctx);
    if (!b) return wg_fail(ctx, WAHGPU_ENOMEM, "allocation failed");
    int rc = bv_reserve(b, n);
    if (rc) { wahgpu_bv_free(b); return rc; }
    if (n) {
        const cudaError_t e = cudaMemcpyAsync(b->words, dev_words, (size_t)n * 4, cudaMemcpyDeviceToDevice, ctx->stream);
        if (e != cudaSuccess) {
            wahgpu_bv_free(b);
            return wg_fail(ctx, WAHGPU_ECUDA, "device copy failed: %s", cudaGetErrorString(e));
        }
    }
    rc = wg_scan_meta(b, n, anb, aval);
    if (rc) { wahgpu_bv_free(b); return rc; }
    b->compressed_form = false;
    *out = b;
    return WAHGPU_OK;
}

extern "C" int wahgpu_bv_create(wahgpu_ctx* ctx, uint64_t cap_words, wahgpu_bv** out) {
    if (!ctx || !out) return wg_fail(ctx, WAHGPU_EINVAL, "bad argument");
    wahgpu_bv* b = wg_bv_new(ctx);
    if (!b) return wg_fail(ctx, WAHGPU_ENOMEM, "allocation failed");
    int rc = bv_reserve(b, cap_words);
    if (rc) { wahgpu_bv_free(b); return rc; }
    rc = wg_scan_meta(b, 0, 0, 0);
    if (rc) { wahgpu_bv_free(b); return rc; }
    *out = b;
    return WAHGPU_OK;
}

extern "C" int wahgpu_bv_free(wahgpu_bv* b) {
    if (!b) return WAHGPU_EINVAL;
    wahgpu_ctx* ctx = b->ctx;
    // buffers go back to the context's pool; the pool never hands a block
    // to later work before earlier work on the same stream has used it
    wg_free(ctx, b->words);
    wg_free(ctx, b->bpos);
    wg_free(ctx, b->meta);
    wg_free(ctx, b->gt);
    delete b;
    return WAHGPU_OK;
}

extern "C" int wahgpu_bv_info_get(wahgpu_bv* b, wahgpu_bv_info* info) {
    if (!b || !info) return WAHGPU_EINVAL;
    int rc = wg_bv_meta(b);
    if (rc) return rc;
    info->nwords = b->h.n;
    info->nbits = (uint64_t)b->h.groups * MAXBITS + b->h.anb;
    info->cnt = (uint64_t)b->h.nset + __builtin_popcount(b->h.aval);
    info->anb = b->h.anb;
    info->aval = b->h.aval;
    info->compressed_form = b->compressed_form ? 1u : 0u;
    return WAHGPU_OK;
}
extern "C" int64_t wahgpu_bv_size(wahgpu_bv* b) {
    wahgpu_bv_info i; int rc = wahgpu_bv_info_get(b, &i); return rc ? rc : (int64_t)i.nbits;
}
extern "C" int64_t wahgpu_bv_cnt(wahgpu_bv* b) {
    wahgpu_bv_info i; int rc = wahgpu_bv_info_get(b, &i); return rc ? rc : (int64_t)i.cnt;
}
extern "C" int64_t wahgpu_bv_serial_size(wahgpu_bv* b) {
    wahgpu_bv_info i; int rc = wahgpu_bv_info_get(b, &i);
    return rc ? rc : (int64_t)(i.nwords + 1 + (i.anb > 0));
}
extern "C" int64_t wahgpu_bv_write(wahgpu_bv* b, uint32_t* out, uint64_t cap) {
    if (!b || (cap && !out)) return WAHGPU_EINVAL;
    int rc = wg_bv_meta(b);
    if (rc) return rc;
    wahgpu_ctx* ctx = b->ctx;
    const uint64_t len = (uint64_t)b->h.n + 1 + (b->h.anb > 0);
    if (cap < len) return wg_fail(ctx, WAHGPU_ESIZE, "need %llu words", (unsigned long long)len);
    if (b->h.n) {
        CUDA_TRY(ctx, cudaMemcpyAsync(out, b->words, (size_t)b->h.n * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    }
    uint64_t k = b->h.n;
    if (b->h.anb > 0) out[k++] = b->h.aval;
    out[k] = b->h.anb;
    return (int64_t)len;
}
extern "C" const uint32_t* wahgpu_bv_device_words(wahgpu_bv* b) { return b ? b->words : nullptr; }

// ---------------------------------------------------------------- operators
static uint32_t combine_active(int op, uint32_t a, uint32_t b) {
    switch (op) {
    case OP_AND: return a & b;
    case OP_OR: return a | b;
    case OP_XOR: return a ^ b;
    default: return a & ~b;
    }
}

// Launches one instantiation of the merge kernel (its shared-memory
// attribute set once per device).
template <int OP, bool FSM, bool UNARY, bool FLIP, int TB>
static void launch_k(const wahgpu_ctx* ctx, dim3 g, cudaStream_t s, const MergeArgs& a) {
    static PerDeviceSetup setup;
    const size_t sm = sizeof(TileShared<TB>);
    wg_kernel_setup(setup, ctx->device, k_merge<OP, FSM, UNARY, FLIP, TB>, MERGE_THREADS, sm);
    k_merge<OP, FSM, UNARY, FLIP, TB><<<g, MERGE_THREADS, sm, s>>>(a);
}
template <int TB>
static void launch_merge_tb(const wahgpu_ctx* ctx, int op, bool fsm, bool unary, bool flip, dim3 g, cudaStream_t s,
                            const MergeArgs& a) {
    if (unary) {
        if (flip) launch_k<0, false, true, true, TB>(ctx, g, s, a);
        else launch_k<0, false, true, false, TB>(ctx, g, s, a);
        return;
    }
#define WG_MERGE_OP(O)                                                          \
    if (fsm) launch_k<O, true, false, false, TB>(ctx, g, s, a);                 \
    else launch_k<O, false, false, false, TB>(ctx, g, s, a);
    switch (op) {
    case OP_AND: WG_MERGE_OP(OP_AND) break;
    case OP_OR: WG_MERGE_OP(OP_OR) break;
    case OP_XOR: WG_MERGE_OP(OP_XOR) break;
    default: WG_MERGE_OP(OP_MINUS) break;
    }
#undef WG_MERGE_OP
}
// Block-index entries per merge tile: the context's setting, else by the
// operands' size: the largest of 64 / 32 / 16 that still gives about two
// tiles per SM, so small operands spread over the GPU in short tiles.
static uint32_t merge_tile_blocks(const wahgpu_ctx* ctx, uint32_t nblocks) {
    if (ctx->merge_tile) return ctx->merge_tile;
    const uint64_t want = 2ull * (uint64_t)ctx->sm_count;
    if ((uint64_t)nblocks >= want * 64u) return 64;
    if ((uint64_t)nblocks >= want * 32u) return 32;
    return 16;
}

// Merge launch: x OP y, or a (complemented) copy of x when y == nullptr.
int wg_launch_merge(wahgpu_ctx* ctx, int op, bool fsm, bool unary, bool flip,
                    const wahgpu_bv* x, const wahgpu_bv* y, uint32_t groups,
                    uint32_t anb, uint32_t aval, wahgpu_bv* res) {
    const uint32_t nx = x->h.n, ny = y ? y->h.n : 0;
    const uint32_t nbx = (nx + 31) / 32, nby = (ny + 31) / 32;
    const uint32_t need = nx + ny;
    int rc = bv_reserve(res, need);
    if (rc) return rc;
    const uint32_t nblk = unary ? nbx : nbx + nby;
    const uint32_t tb = merge_tile_blocks(ctx, nblk);
    uint32_t ntiles = (nblk + tb - 1) / tb;
    if (ntiles == 0) ntiles = 1;
    TileRec* recs; LaunchSync* sync;
    rc = wg_scratch(ctx, ntiles, &recs, &sync);
    if (rc) return rc;
    MergeArgs a;
    a.xw = x->words; a.xbp = x->bpos; a.nx = nx; a.nbx = nbx;
    a.yw = y ? y->words : x->words; a.ybp = y ? y->bpos : x->bpos; a.ny = ny; a.nby = nby;
    a.groups = groups;
    a.out = res->words; a.obp = res->bpos; a.meta = res->meta;
    a.recs = recs; a.sync = sync; a.ntiles = ntiles;
    a.aval = aval; a.anb = anb;
    CUDA_TRY(ctx, cudaMemsetAsync(res->meta, 0, sizeof(DevMeta), ctx->stream));
    dim3 g(ntiles);
    if (tb == 16) launch_merge_tb<16>(ctx, op, fsm, unary, flip, g, ctx->stream, a);
    else if (tb == 32) launch_merge_tb<32>(ctx, op, fsm, unary, flip, g, ctx->stream, a);
    else launch_merge_tb<64>(ctx, op, fsm, unary, flip, g, ctx->stream, a);
    ctx->launches++;
    CUDA_TRY(ctx, cudaGetLastError());
    res->h_valid = false;
    res->gt_valid = false;
    res->compressed_form = true;
    return WAHGPU_OK;
}

// Group-tile index of b (host metadata must be valid); built once.
static int wg_gtile(wahgpu_bv* b) {
    if (b->gt_valid) return WAHGPU_OK;
    wahgpu_ctx* ctx = b->ctx;
    const uint32_t nt = (b->h.groups + DT - 1) / DT;
    if (!b->gt) {
        b->gt = static_cast<uint32_t*>(wg_alloc(ctx, ((size_t)nt + 2) * 8));
        if (!b->gt) return wg_fail(ctx, WAHGPU_ENOMEM, "allocation failed");
    } else {
        // reallocate when the current block may be too small
        wg_free(ctx, b->gt);
        b->gt = static_cast<uint32_t*>(wg_alloc(ctx, ((size_t)nt + 2) * 8));
        if (!b->gt) return wg_fail(ctx, WAHGPU_ENOMEM, "allocation failed");
    }
    const uint32_t threads = 128, blocks = (nt + 1 + threads - 1) / threads;
    k_gtile<<<blocks, threads, 0, ctx->stream>>>(b->words, b->bpos, b->h.n, b->h.groups, nt, b->gt);
    ctx->launches++;
    CUDA_TRY(ctx, cudaGetLastError());
    b->gt_valid = true;
    return WAHGPU_OK;
}

template <int OP, int TG, int NCW>
static void launch_dense_op(const wahgpu_ctx* ctx, uint32_t ntiles, cudaStream_t s, const DenseArgs& a) {
    static PerDeviceSetup setup;
    const size_t sm = sizeof(DShared<TG, NCW>);
    const int per_sm = wg_kernel_setup(setup, ctx->device, k_dense<OP, TG, NCW>, (NCW + 1) * 32, sm);
    // persistent: at most one wave of resident CTAs
    const uint32_t grid = std::min<uint32_t>(ntiles, (uint32_t)(per_sm * ctx->sm_count));
    k_dense<OP, TG, NCW><<<grid, (NCW + 1) * 32, sm, s>>>(a);
}
template <int OP>
static void launch_dense_tg(const wahgpu_ctx* ctx, uint32_t tg, uint32_t ntiles, cudaStream_t s, const DenseArgs& a) {
    if (tg == 1024) launch_dense_op<OP, 1024, 4>(ctx, ntiles, s, a);
    else if (tg == 4096) launch_dense_op<OP, 4096, 8>(ctx, ntiles, s, a);
    else launch_dense_op<OP, 2048, 8>(ctx, ntiles, s, a);
}

int wg_launch_dense(wahgpu_ctx* ctx, int op, wahgpu_bv* x, wahgpu_bv* y, uint32_t groups,
                    uint32_t anb, uint32_t aval, wahgpu_bv* res) {
    int rc = bv_reserve(res, (uint64_t)x->h.n + y->h.n);
    if (rc) return rc;
    rc = wg_gtile(x);
    if (rc) return rc;
    rc = wg_gtile(y);
    if (rc) return rc;
    const uint32_t tg = ctx->dense_tile;
    const uint32_t ntiles = (groups + tg - 1) / tg;
    TileRec* recs; LaunchSync* sync;
    rc = wg_scratch(ctx, ntiles, &recs, &sync);
    if (rc) return rc;
    DenseArgs a;
    a.xw = x->words; a.xgt = x->gt; a.nx = x->h.n;
    a.yw = y->words; a.ygt = y->gt; a.ny = y->h.n;
    a.groups = groups;
    a.out = res->words; a.obp = res->bpos; a.meta = res->meta;
    a.drecs = wg_dense_recs(ctx, recs); a.sync = sync; a.ntiles = ntiles;
    a.aval = aval; a.anb = anb;
    CUDA_TRY(ctx, cudaMemsetAsync(res->meta, 0, sizeof(DevMeta), ctx->stream));
    switch (op) {
    case OP_AND: launch_dense_tg<OP_AND>(ctx, tg, ntiles, ctx->stream, a); break;
    case OP_OR: launch_dense_tg<OP_OR>(ctx, tg, ntiles, ctx->stream, a); break;
    case OP_XOR: launch_dense_tg<OP_XOR>(ctx, tg, ntiles, ctx->stream, a); break;
    default: launch_dense_tg<OP_MINUS>(ctx, tg, ntiles, ctx->stream, a); break;
    }
    ctx->launches++;
    CUDA_TRY(ctx, cudaGetLastError());
    res->h_valid = false;
    res->gt_valid = false;
    res->compressed_form = true;
    return WAHGPU_OK;
}

// Two-pass group-space engine (wah_gop.cuh): expand + operate into dense
// result patterns with per-tile head counts, then pack the words.
int wg_launch_gop(wahgpu_ctx* ctx, int op, wahgpu_bv* x, wahgpu_bv* y, uint32_t groups,
                  uint32_t anb, uint32_t aval, wahgpu_bv* res) {
    int rc = bv_reserve(res, (uint64_t)x->h.n + y->h.n);
    if (rc) return rc;
    // the staging copies 16-byte chunks of the operands' word arrays (pool
    // blocks, 256-byte aligned)
    if ((reinterpret_cast<uintptr_t>(x->words) | reinterpret_cast<uintptr_t>(y->words)) & 15u)
        return wg_fail(ctx, WAHGPU_EINVAL, "operand word arrays must be 16-byte aligned");
    rc = wg_gtile(x);
    if (rc) return rc;
    rc = wg_gtile(y);
    if (rc) return rc;
    const uint32_t ntiles = (groups + GT - 1) / GT;
    uint32_t* R = static_cast<uint32_t*>(wg_alloc(ctx, (size_t)ntiles * GT * 4));
    const uint32_t nseg = (ntiles + GSEG - 1) / GSEG;
    uint4* tiles = static_cast<uint4*>(wg_alloc(ctx, ((size_t)ntiles + nseg) * 16));
    uint32_t* hmask = static_cast<uint32_t*>(wg_alloc(ctx, (size_t)ntiles * 32 * 4));
    if (!R || !tiles || !hmask) {
        wg_free(ctx, R); wg_free(ctx, tiles); wg_free(ctx, hmask);
        return wg_fail(ctx, WAHGPU_ENOMEM, "allocation of %u tiles of result patterns failed", ntiles);
    }
    GopArgs a;
    a.xw = x->words; a.xgt = x->gt; a.nx = x->h.n;
    a.yw = y->words; a.ygt = y->gt; a.ny = y->h.n;
    a.groups = groups; a.ntiles = ntiles;
    a.R = R; a.tiles = tiles; a.segs = tiles + ntiles; a.hmask = hmask;
    a.out = res->words; a.obp = res->bpos; a.meta = res->meta;
    a.aval = aval; a.anb = anb;
    cudaStream_t s = ctx->stream;
    rc = WAHGPU_OK;
    if (cudaMemsetAsync(res->meta, 0, sizeof(DevMeta), s) != cudaSuccess ||
        cudaMemsetAsync(a.segs, 0, (size_t)nseg * 16, s) != cudaSuccess)
        rc = wg_fail(ctx, WAHGPU_ECUDA, "memset failed");
    if (!rc) {
        const uint32_t grid = (ntiles + GWARPS - 1) / GWARPS;
        const size_t sm_op = GWARPS * sizeof(GopWarp);
        static PerDeviceSetup setup[4];
        wg_kernel_setup(setup[0], ctx->device, k_gop<OP_AND>, GTHREADS, sm_op);
        wg_kernel_setup(setup[1], ctx->device, k_gop<OP_OR>, GTHREADS, sm_op);
        wg_kernel_setup(setup[2], ctx->device, k_gop<OP_XOR>, GTHREADS, sm_op);
        wg_kernel_setup(setup[3], ctx->device, k_gop<OP_MINUS>, GTHREADS, sm_op);
        switch (op) {
        case OP_AND: k_gop<OP_AND><<<grid, GTHREADS, sm_op, s>>>(a); break;
        case OP_OR: k_gop<OP_OR><<<grid, GTHREADS, sm_op, s>>>(a); break;
        case OP_XOR: k_gop<OP_XOR><<<grid, GTHREADS, sm_op, s>>>(a); break;
        default: k_gop<OP_MINUS><<<grid, GTHREADS, sm_op, s>>>(a); break;
        }
        k_gpack<<<grid, GTHREADS, 0, s>>>(a);
        ctx->launches += 2;
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = wg_fail(ctx, WAHGPU_ECUDA, "launch failed: %s", cudaGetErrorString(e));
    }
    // stream-ordered: the next user of these blocks on this context's
    // stream runs after the launches above
    wg_free(ctx, R);
    wg_free(ctx, tiles);
    wg_free(ctx, hmask);
    if (rc) return rc;
    res->h_valid = false;
    res->gt_valid = false;
    res->compressed_form = true;
    return WAHGPU_OK;
}

// Single-pass group-space engine (wah_fuse.cuh): one launch per call,
// operands read once, words written once.  Needs 16-byte-aligned word arrays
// (every block of the allocator is); the two-pass engine runs otherwise.
static bool fuse_applies(const wahgpu_bv* x, const wahgpu_bv* y, const wahgpu_bv* res, uint32_t groups) {
    auto al = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    return groups > 0 && al(x->words) && al(y->words) && al(res->words);
}
template <int OP, int FT>
static void launch_fuse_op(const wahgpu_ctx* ctx, uint32_t ntiles, cudaStream_t s, const FuseArgs& a) {
    static PerDeviceSetup setup;
    const size_t sm = sizeof(FuseShared<FT>);
    wg_kernel_setup(setup, ctx->device, k_gfuse<OP, FT>, FCfg<FT>::THREADS, sm);
    k_gfuse<OP, FT><<<ntiles, FCfg<FT>::THREADS, sm, s>>>(a);
}
template <int OP>
static void launch_fuse_tile(const wahgpu_ctx* ctx, uint32_t ft, uint32_t ntiles, cudaStream_t s, const FuseArgs& a) {
    if (ft == 1024) launch_fuse_op<OP, 1024>(ctx, ntiles, s, a);
    else if (ft == 4096) launch_fuse_op<OP, 4096>(ctx, ntiles, s, a);
    else launch_fuse_op<OP, 2048>(ctx, ntiles, s, a);
}
int wg_launch_fuse(wahgpu_ctx* ctx, int op, wahgpu_bv* x, wahgpu_bv* y, uint32_t groups,
                   uint32_t anb, uint32_t aval, wahgpu_bv* res) {
    int rc = bv_reserve(res, (uint64_t)x->h.n + y->h.n);
    if (rc) return rc;
    if (!fuse_applies(x, y, res, groups)) return wg_launch_gop(ctx, op, x, y, groups, anb, aval, res);
    rc = wg_gtile(x);
    if (rc) return rc;
    rc = wg_gtile(y);
    if (rc) return rc;
    const uint32_t ft = ctx->dense_tile;  // WAHGPU_TUNE_DENSE_TILE: 1024, 2048 (default) or 4096 groups
    const uint32_t ntiles = (groups + ft - 1) / ft;
    TileRec* recs; LaunchSync* sync;
    rc = wg_scratch(ctx, ntiles, &recs, &sync);
    if (rc) return rc;
    FuseArgs a;
    a.xw = x->words; a.xgt = x->gt; a.nx = x->h.n;
    a.yw = y->words; a.ygt = y->gt; a.ny = y->h.n;
    a.groups = groups; a.ntiles = ntiles;
    a.out = res->words; a.obp = res->bpos; a.meta = res->meta; a.cap = res->cap;
    a.recs = wg_fuse_recs(ctx, recs); a.sync = sync;
    a.aval = aval; a.anb = anb;
    a.withhold = ctx->test_withhold;
    ctx->test_withhold = 0xFFFFFFFFu;
    CUDA_TRY(ctx, cudaMemsetAsync(res->meta, 0, sizeof(DevMeta), ctx->stream));
    switch (op) {
    case OP_AND: launch_fuse_tile<OP_AND>(ctx, ft, ntiles, ctx->stream, a); break;
    case OP_OR: launch_fuse_tile<OP_OR>(ctx, ft, ntiles, ctx->stream, a); break;
    case OP_XOR: launch_fuse_tile<OP_XOR>(ctx, ft, ntiles, ctx->stream, a); break;
    default: launch_fuse_tile<OP_MINUS>(ctx, ft, ntiles, ctx->stream, a); break;
    }
    ctx->launches++;
    CUDA_TRY(ctx, cudaGetLastError());
    res->h_valid = false;
    res->gt_valid = false;
    res->compressed_form = true;
    return WAHGPU_OK;
}

// Single-pass warp-tile engine (wah_gone.cuh): one launch per call, one
// warp per 1024-group tile, operands read once, words written once.
int wg_launch_gone(wahgpu_ctx* ctx, int op, wahgpu_bv* x, wahgpu_bv* y, uint32_t groups,
                   uint32_t anb, uint32_t aval, wahgpu_bv* res) {
    int rc = bv_reserve(res, (uint64_t)x->h.n + y->h.n);
    if (rc) return rc;
    if (groups == 0) return wg_launch_gop(ctx, op, x, y, groups, anb, aval, res);
    rc = wg_gtile(x);
    if (rc) return rc;
    rc = wg_gtile(y);
    if (rc) return rc;
    const uint32_t ntiles = (groups + GT - 1) / GT;
    TileRec* recs; LaunchSync* sync;
    rc = wg_scratch(ctx, ntiles, &recs, &sync);
    if (rc) return rc;
    FuseArgs a;
    a.xw = x->words; a.xgt = x->gt; a.nx = x->h.n;
    a.yw = y->words; a.ygt = y->gt; a.ny = y->h.n;
    a.groups = groups; a.ntiles = ntiles;
    a.out = res->words; a.obp = res->bpos; a.meta = res->meta; a.cap = res->cap;
    a.recs = wg_fuse_recs(ctx, recs); a.sync = sync;
    a.aval = aval; a.anb = anb;
    a.withhold = ctx->test_withhold;
    ctx->test_withhold = 0xFFFFFFFFu;
    CUDA_TRY(ctx, cudaMemsetAsync(res->meta, 0, sizeof(DevMeta), ctx->stream));
    const uint32_t grid = (ntiles + GWARPS - 1) / GWARPS;
    const size_t sm = GWARPS * sizeof(GoneWarp);
    static PerDeviceSetup setup[4];
    cudaStream_t s = ctx->stream;
    switch (op) {
    case OP_AND:
        wg_kernel_setup(setup[0], ctx->device, k_gone<OP_AND>, GTHREADS, sm);
        k_gone<OP_AND><<<grid, GTHREADS, sm, s>>>(a);
        break;
    case OP_OR:
        wg_kernel_setup(setup[1], ctx->device, k_gone<OP_OR>, GTHREADS, sm);
        k_gone<OP_OR><<<grid, GTHREADS, sm, s>>>(a);
        break;
    case OP_XOR:
        wg_kernel_setup(setup[2], ctx->device, k_gone<OP_XOR>, GTHREADS, sm);
        k_gone<OP_XOR><<<grid, GTHREADS, sm, s>>>(a);
        break;
    default:
        wg_kernel_setup(setup[3], ctx->device, k_gone<OP_MINUS>, GTHREADS, sm);
        k_gone<OP_MINUS><<<grid, GTHREADS, sm, s>>>(a);
        break;
    }
    ctx->launches++;
    CUDA_TRY(ctx, cudaGetLastError());
    res->h_valid = false;
    res->gt_valid = false;
    res->compressed_form = true;
    return WAHGPU_OK;
}

// A one-word device bitvector holding the collapsed form of an all-zero
// operand (do_cnt(), src/bitvector.cpp:601-604).
static int collapsed_copy(wahgpu_ctx* ctx, const wahgpu_bv* src, wahgpu_bv** out) {
    wahgpu_bv* b = wg_bv_new(ctx);
    if (!b) return wg_fail(ctx, WAHGPU_ENOMEM, "allocation failed");
    int rc = bv_reserve(b, 1);
    if (rc) { wahgpu_bv_free(b); return rc; }
    uint32_t* st = reinterpret_cast<uint32_t*>(ctx->h_meta_stage) + 16;
    st[0] = HEADER0 | src->h.groups;
    st[1] = 0;
    st[2] = src->h.groups;
    CUDA_TRY(ctx, cudaMemcpyAsync(b->words, st, 4, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(b->bpos, st + 1, 8, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    b->h = src->h;
    b->h.n = 1;
    b->h.w0 = st[0];
    b->h.nfill = 1;
    b->h_valid = true;
    // device meta mirrors the host copy
    CUDA_TRY(ctx, cudaMemcpyAsync(b->meta, &b->h, sizeof(DevMeta), cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    *out = b;
    return WAHGPU_OK;
}

static OperandMeta opmeta(const wahgpu_bv* b) {
    OperandMeta m;
    m.n = b->h.n; m.groups = b->h.groups; m.anb = b->h.anb; m.aval = b->h.aval;
    m.nset = b->h.nset; m.w0 = b->h.w0;
    return m;
}

// Engine for a canonical-result operator (WAHGPU_TUNE_DENSE_ENGINE): 1 the
// pipelined group-space kernel, 2 the word-space merge, 3 the two-pass
// group-space kernels, 4 the single-pass group-space kernel; 0 (default)
// the single-pass kernel.
static bool dense_in_word_space(const wahgpu_ctx* ctx, const wahgpu_bv*, const wahgpu_bv*, uint32_t) {
    return ctx->dense_engine == 2;
}
static bool dense_two_pass(const wahgpu_ctx* ctx) {
    return ctx->dense_engine == 0 || ctx->dense_engine == 3;
}
static bool dense_fused(const wahgpu_ctx* ctx) {
    return ctx->dense_engine == 4;
}
static bool dense_warp_tiles(const wahgpu_ctx* ctx) {
    return ctx->dense_engine == 5;
}

// adjustSize(0, nt) of a copy of b (src/bitvector.cpp:4086-4108): the copy
// grows by appendFill(0, nt - size()) (src/bitvector.h:800-831), whose
// append_active / append_counter (699-760) may merge into b's last word, so
// the copy keeps b's words up to the last one and the rest is rebuilt here.
static int padded_copy(wahgpu_ctx* ctx, wahgpu_bv* b, uint64_t nt, wahgpu_bv** out) {
    *out = nullptr;
    const uint32_t n = b->h.n;
    std::vector<uint32_t> t;  // b's last word, then the appended words
    if (n) {
        uint32_t last = 0;
        CUDA_TRY(ctx, cudaMemcpyAsync(&last, b->words + n - 1, 4, cudaMemcpyDeviceToHost, ctx->stream));
        CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        t.push_back(last);
    }
    // append_active of a literal (bitvector.h:699-737)
    auto push_active = [&](uint32_t v) {
        if (t.empty()) { t.push_back(v); return; }
        uint32_t& bk = t.back();
        if (v == 0) {
            if (bk == 0) bk = HEADER0 + 2;
            else if (bk >= HEADER0 && bk < HEADER1) ++bk;
            else t.push_back(v);
        } else if (v == ALLONES) {
            if (bk == ALLONES) bk = HEADER1 | 2;
            else if (bk >= HEADER1) ++bk;
            else t.push_back(v);
        } else {
            t.push_back(v);
        }
    };
    // append_counter(0, cnt) (bitvector.h:741-760)
    auto push_zeros = [&](uint32_t cnt) {
        const uint32_t w = HEADER0 + cnt;
        if (t.empty()) { t.push_back(w); return; }
        uint32_t& bk = t.back();
        if ((bk >> 30) == 2u) bk += cnt;
        else if (bk == 0) bk = w + 1;
        else t.push_back(w);
    };
    uint32_t anb = b->h.anb, aval = b->h.aval;
    uint64_t need = nt - ((uint64_t)b->h.groups * MAXBITS + anb);
    if (anb > 0) {
        const uint32_t k = (uint32_t)std::min<uint64_t>(MAXBITS - anb, need);
        anb += k;
        aval <<= k;
        need -= k;
        if (anb >= MAXBITS) { push_active(aval); anb = 0; aval = 0; }
    }
    if (need >= MAXBITS) {
        const uint64_t cnt = need / MAXBITS;
        if (cnt > MAXCNT) return wg_fail(ctx, WAHGPU_ERANGE, "padding of %llu groups", (unsigned long long)cnt);
        if (cnt > 1) push_zeros((uint32_t)cnt);
        else push_active(0);
        need -= cnt * MAXBITS;
    }
    if (need > 0) { anb = (uint32_t)need; aval = 0; }
    const uint32_t keep = n ? n - 1 : 0;
    const uint64_t m = (uint64_t)keep + t.size();
    wahgpu_bv* p = wg_bv_new(ctx);
    if (!p) return wg_fail(ctx, WAHGPU_ENOMEM, "allocation failed");
    int rc = bv_reserve(p, m);
    if (!rc && keep && cudaMemcpyAsync(p->words, b->words, (size_t)keep * 4, cudaMemcpyDeviceToDevice, ctx->stream))
        rc = wg_fail(ctx, WAHGPU_ECUDA, "copy failed");
    if (!rc && !t.empty() && (cudaMemcpyAsync(p->words + keep, t.data(), t.size() * 4, cudaMemcpyHostToDevice,
                                              ctx->stream) || cudaStreamSynchronize(ctx->stream)))
        rc = wg_fail(ctx, WAHGPU_ECUDA, "copy failed");
    if (!rc) rc = wg_scan_meta(p, (uint32_t)m, anb, aval);
    if (!rc) rc = wg_bv_meta(p);
    if (rc) { wahgpu_bv_free(p); return rc; }
    *out = p;
    return WAHGPU_OK;
}

// Operands of different sizes (src/bitvector.cpp:1194-1838): the shorter
// one is padded with 0 bits and the operator runs in its OP= form — for
// a OP b with a longer a: res = b padded, res OP= a (& | ^) or res = a,
// res -= b padded (-); with a shorter a: res = a padded, res OP= b; for
// a OP= b: a OP= (b padded), or (a padded) OP= b.
static int binop_unequal(wahgpu_ctx* ctx, int op, bool inplace, wahgpu_bv* a, wahgpu_bv* b, wahgpu_bv* res) {
    const uint64_t sa = (uint64_t)a->h.groups * MAXBITS + a->h.anb;
    const uint64_t sb = (uint64_t)b->h.groups * MAXBITS + b->h.anb;
    wahgpu_bv* pad = nullptr;
    int rc = padded_copy(ctx, sa > sb ? b : a, sa > sb ? sa : sb, &pad);
    if (rc) return rc;
    if (sa < sb) rc = wahgpu_bv_binop_into(ctx, op, 1, pad, b, res);
    else if (inplace || op == OP_MINUS) rc = wahgpu_bv_binop_into(ctx, op, 1, a, pad, res);
    else rc = wahgpu_bv_binop_into(ctx, op, 1, pad, a, res);
    cudaStreamSynchronize(ctx->stream);
    wahgpu_bv_free(pad);
    return rc;
}

extern "C" int wahgpu_bv_binop_into(wahgpu_ctx* ctx, int op, int inplace, wahgpu_bv* a, wahgpu_bv* b,
                                    wahgpu_bv* res) {
    if (!ctx || !a || !b || !res || op < 0 || op > 3) return wg_fail(ctx, WAHGPU_EINVAL, "bad argument");
    if (res == a || res == b) return wg_fail(ctx, WAHGPU_EINVAL, "result must differ from the operands");
    int rc = wg_bv_meta(a);
    if (rc) return rc;
    rc = wg_bv_meta(b);
    if (rc) return rc;
    OperandMeta ma = effective(opmeta(a)), mb = effective(opmeta(b));
    Plan p = plan_binop(op, inplace != 0, ma, mb);
    if (p.kind == PK_UNEQUAL) {
        // pad the operands the reference would hold (an all-0 one collapsed
        // by do_cnt, src/bitvector.cpp:601-604)
        wahgpu_bv* ea = a;
        wahgpu_bv* eb = b;
        wahgpu_bv* ta = nullptr;
        wahgpu_bv* tb = nullptr;
        if (ma.n != a->h.n) { rc = collapsed_copy(ctx, a, &ta); if (rc) return rc; ea = ta; }
        if (mb.n != b->h.n) { rc = collapsed_copy(ctx, b, &tb); if (rc) { if (ta) wahgpu_bv_free(ta); return rc; } eb = tb; }
        rc = binop_unequal(ctx, op, inplace != 0, ea, eb, res);
        if (ta || tb) {
            cudaStreamSynchronize(ctx->stream);
            if (ta) wahgpu_bv_free(ta);
            if (tb) wahgpu_bv_free(tb);
        }
        return rc;
    }
    const uint32_t G = ma.groups;
    if (G >= 2 && ((ma.n == G && a->h.nfill && ma.n == a->h.n) || (mb.n == G && b->h.nfill && mb.n == b->h.n)))
        return wg_fail(ctx, WAHGPU_EDEGENERATE,
                       "an operand has one word per group and count-1 fill words; the reference "
                       "combines such fill headers as literal bits");
    const uint32_t aval = combine_active(op, a->h.aval, b->h.aval);
    const uint32_t anb = a->h.anb;
    wahgpu_bv* ca = a;
    wahgpu_bv* cb = b;
    wahgpu_bv* tmpa = nullptr;
    wahgpu_bv* tmpb = nullptr;
    if (ma.n != a->h.n) { rc = collapsed_copy(ctx, a, &tmpa); if (rc) return rc; ca = tmpa; }
    if (mb.n != b->h.n) { rc = collapsed_copy(ctx, b, &tmpb); if (rc) { if (tmpa) wahgpu_bv_free(tmpa); return rc; } cb = tmpb; }
    switch (p.kind) {
    case PK_MERGE_FSM:
        rc = wg_launch_merge(ctx, op, true, false, false, ca, cb, G, anb, aval, res);
        break;
    case PK_MERGE_CANON:
        // canonical result: the group-space kernel, or the word-space merge
        // (no step states) when the tuning asks for it
        if (dense_in_word_space(ctx, ca, cb, G))
            rc = wg_launch_merge(ctx, op, false, false, false, ca, cb, G, anb, aval, res);
        else if (dense_warp_tiles(ctx))
            rc = wg_launch_gone(ctx, op, ca, cb, G, anb, aval, res);
        else if (dense_fused(ctx))
            rc = wg_launch_fuse(ctx, op, ca, cb, G, anb, aval, res);
        else if (dense_two_pass(ctx))
            rc = wg_launch_gop(ctx, op, ca, cb, G, anb, aval, res);
        else
            rc = wg_launch_dense(ctx, op, ca, cb, G, anb, aval, res);
        break;
    case PK_COPY:
    case PK_COPY_FLIP:
        rc = wg_launch_merge(ctx, 0, false, true, p.kind == PK_COPY_FLIP, p.src ? cb : ca, nullptr, G, anb, aval, res);
        break;
    default: {
        rc = bv_reserve(res, 1);
        if (rc) break;
        int mode = p.kind == PK_EMPTY ? 0 : (p.kind == PK_RAW1 ? 1 : 2);
        cudaError_t e = cudaMemsetAsync(res->meta, 0, sizeof(DevMeta), ctx->stream);
        if (e != cudaSuccess) { rc = wg_fail(ctx, WAHGPU_ECUDA, "memset failed"); break; }
        k_small<<<1, 32, 0, ctx->stream>>>(mode, op, ca->words, cb->words, p.fill_n, G, res->words, res->bpos,
                                           res->meta, anb, aval);
        ctx->launches++;
        e = cudaGetLastError();
        if (e != cudaSuccess) { rc = wg_fail(ctx, WAHGPU_ECUDA, "launch failed: %s", cudaGetErrorString(e)); break; }
        res->h_valid = false;
        res->gt_valid = false;
        res->compressed_form = true;
    }
    }
    if (tmpa || tmpb) {
        cudaStreamSynchronize(ctx->stream);
        if (tmpa) wahgpu_bv_free(tmpa);
        if (tmpb) wahgpu_bv_free(tmpb);
    }
    return rc;
}

extern "C" int wahgpu_bv_binop(wahgpu_ctx* ctx, int op, int inplace, wahgpu_bv* a, wahgpu_bv* b,
                               wahgpu_bv** res) {
    if (!res) return wg_fail(ctx, WAHGPU_EINVAL, "res is NULL");
    *res = nullptr;
    wahgpu_bv* r = wg_bv_new(ctx);
    if (!r) return wg_fail(ctx, WAHGPU_ENOMEM, "allocation failed");
    int rc = wahgpu_bv_binop_into(ctx, op, inplace, a, b, r);
    if (rc) { wahgpu_bv_free(r); return rc; }
    *res = r;
    return WAHGPU_OK;
}

// Replaces b's storage with that of tmp (both on the same context).
static void bv_take(wahgpu_bv* b, wahgpu_bv* tmp) {
    std::swap(b->words, tmp->words);
    std::swap(b->bpos, tmp->bpos);
    std::swap(b->meta, tmp->meta);
    std::swap(b->cap, tmp->cap);
    std::swap(b->h, tmp->h);
    std::swap(b->h_valid, tmp->h_valid);
    std::swap(b->gt, tmp->gt);
    std::swap(b->gt_valid, tmp->gt_valid);
    b->compressed_form = tmp->compressed_form;
}

static int unary_op(wahgpu_bv* b, bool flip) {
    wahgpu_ctx* ctx = b->ctx;
    int rc = wg_bv_meta(b);
    if (rc) return rc;
    wahgpu_bv* r = wg_bv_new(ctx);
    if (!r) return wg_fail(ctx, WAHGPU_ENOMEM, "allocation failed");
    const uint32_t aval = flip && b->h.anb ? (b->h.aval ^ ((1u << b->h.anb) - 1)) : b->h.aval;
    if (b->h.n == 0) {
        rc = bv_reserve(r, 1);
        if (!rc) rc = wg_scan_meta(r, 0, b->h.anb, aval);
    } else {
        rc = wg_launch_merge(ctx, 0, false, true, flip, b, nullptr, b->h.groups, b->h.anb, aval, r);
    }
    if (rc) { wahgpu_bv_free(r); return rc; }
    cudaStreamSynchronize(ctx->stream);
    bv_take(b, r);
    wahgpu_bv_free(r);
    return WAHGPU_OK;
}
extern "C" int wahgpu_bv_compress(wahgpu_bv* b) {
    if (!b) return WAHGPU_EINVAL;
    if (b->compressed_form) return WAHGPU_OK;
    return unary_op(b, false);
}
extern "C" int wahgpu_bv_flip(wahgpu_bv* b) {
    if (!b) return WAHGPU_EINVAL;
    return unary_op(b, true);
}
extern "C" int wahgpu_bv_decompress(wahgpu_bv* b) {
    if (!b) return WAHGPU_EINVAL;
    wahgpu_ctx* ctx = b->ctx;
    int rc = wg_bv_meta(b);
    if (rc) return rc;
    const uint32_t G = b->h.groups;
    if (b->h.n == G) return WAHGPU_OK;  // already uncompressed
    wahgpu_bv* r = wg_bv_new(ctx);
    if (!r) return wg_fail(ctx, WAHGPU_ENOMEM, "allocation failed");
    rc = bv_reserve(r, G);
    if (!rc && b->h.n) {
        uint32_t nt = (b->h.n + SCAN_TILE - 1) / SCAN_TILE;
        k_decompress<<<nt, SCAN_THREADS, 0, ctx->stream>>>(b->words, b->h.n, b->bpos, r->words);
        ctx->launches++;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = wg_fail(ctx, WAHGPU_ECUDA, "launch failed: %s", cudaGetErrorString(e));
    }
    if (!rc) rc = wg_scan_meta(r, G, b->h.anb, b->h.aval);
    if (rc) { wahgpu_bv_free(r); return rc; }
    cudaStreamSynchronize(ctx->stream);
    bv_take(b, r);
    b->compressed_form = false;
    wahgpu_bv_free(r);
    return WAHGPU_OK;
}

int64_t wg_rids_device(wahgpu_bv* b, uint32_t* dev_out, uint64_t cap, uint64_t* total) {
    wahgpu_ctx* ctx = b->ctx;
    int rc = wg_bv_meta(b);
    if (rc) return rc;
    const uint64_t cnt = (uint64_t)b->h.nset + __builtin_popcount(b->h.anb ? b->h.aval & ((1u << b->h.anb) - 1) : 0u);
    *total = cnt;
    if (cap < cnt) return wg_fail(ctx, WAHGPU_ESIZE, "need room for %llu row ids", (unsigned long long)cnt);
    const uint32_t n = b->h.n;
    const uint32_t ntiles = n ? (n + SCAN_TILE - 1) / SCAN_TILE : 1;
    TileRec* recs; LaunchSync* sync;
    rc = wg_scratch(ctx, ntiles, &recs, &sync);
    if (rc) return rc;
    unsigned long long* dtot = reinterpret_cast<unsigned long long*>(wg_alloc(ctx, 8));
    if (!dtot) return wg_fail(ctx, WAHGPU_ENOMEM, "allocation failed");
    k_rids<<<ntiles, SCAN_THREADS, 0, ctx->stream>>>(b->words, n, b->bpos, b->h.groups, b->h.anb, b->h.aval,
                                                      dev_out, cap, dtot, b->meta, recs, sync, ntiles);
    ctx->launches++;
    CUDA_TRY(ctx, cudaGetLastError());
    wg_free(ctx, dtot);
    return (int64_t)cnt;
}

extern "C" int64_t wahgpu_bv_rids_device(wahgpu_bv* b, uint32_t* dev_out, uint64_t cap) {
    if (!b || (cap && !dev_out)) return WAHGPU_EINVAL;
    uint64_t total = 0;
    return wg_rids_device(b, dev_out, cap, &total);
}

extern "C" int64_t wahgpu_bv_rids(wahgpu_bv* b, uint32_t* out, uint64_t cap) {
    if (!b || (cap && !out)) return WAHGPU_EINVAL;
    wahgpu_ctx* ctx = b->ctx;
    int rc = wg_bv_meta(b);
    if (rc) return rc;
    const uint64_t cnt = (uint64_t)b->h.nset + __builtin_popcount(b->h.anb ? b->h.aval & ((1u << b->h.anb) - 1) : 0u);
    if (cap < cnt) return wg_fail(ctx, WAHGPU_ESIZE, "need room for %llu row ids", (unsigned long long)cnt);
    if (cnt == 0) return 0;
    uint32_t* d = static_cast<uint32_t*>(wg_alloc(ctx, cnt * 4));
    if (!d) return wg_fail(ctx, WAHGPU_ENOMEM, "allocation failed");
    uint64_t total = 0;
    int64_t r = wg_rids_device(b, d, cnt, &total);
    if (r < 0) { wg_free(ctx, d); return r; }
    cudaError_t e = cudaMemcpyAsync(out, d, cnt * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    wg_free(ctx, d);
    if (e != cudaSuccess) return wg_fail(ctx, WAHGPU_ECUDA, "row-id copy failed: %s", cudaGetErrorString(e));
    rc = wg_bv_meta(b);
    return rc ? rc : (int64_t)cnt;
}
