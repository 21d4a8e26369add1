// Internal state behind the opaque handles of include/wahgpu.h.
#ifndef WAH_API_INTERNAL_H
#define WAH_API_INTERNAL_H
#include <cuda_runtime.h>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <vector>
#include "wah_dev.cuh"

struct wahgpu_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;      // where work is queued
    cudaStream_t own_stream = nullptr;  // the context's own stream
    std::string err;
    std::mutex mu;
    // caching device allocator: size class -> free blocks; block -> class
    std::map<size_t, std::vector<void*>> pool;
    std::map<void*, size_t> sizes;
    std::map<size_t, std::vector<void*>> hpool;  // pinned host blocks by size class
    std::map<void*, size_t> hsizes;
    size_t bytes_allocated = 0;
    // look-back scratch: two LaunchSync words then TileRec records
    void* scratch = nullptr;
    uint32_t scratch_tiles = 0;
    void* h_meta_stage = nullptr;  // pinned staging for metadata reads
    uint64_t launches = 0;
    uint32_t dense_tile = 2048;         // WAHGPU_TUNE_DENSE_TILE
    uint32_t dense_engine = 0;          // WAHGPU_TUNE_DENSE_ENGINE
    uint32_t range_order = 1;           // WAHGPU_TUNE_RANGE_ORDER
    uint32_t range_ctas = 0;            // WAHGPU_TUNE_RANGE_CTAS (0: as many as fit)
    uint32_t merge_tile = 0;            // WAHGPU_TUNE_MERGE_TILE (0: by operand size)
    uint32_t cum_stride = 0;            // WAHGPU_TUNE_CUM_STRIDE (0 auto, 1 none)
    // failure-path test hooks (WAHGPU_TEST_*): the tile of the next
    // single-pass operator launch that never publishes its look-back record
    // (UINT32_MAX: none), and the allocations left before one fails (0: off)
    uint32_t test_withhold = 0xFFFFFFFFu;
    int64_t test_fail_alloc = 0;
};

struct wahgpu_bv {
    wahgpu_ctx* ctx = nullptr;
    uint32_t* words = nullptr;  // m_vec
    uint32_t* bpos = nullptr;   // block positions: group where word 32k starts
    wah::DevMeta* meta = nullptr;
    uint32_t cap = 0;           // capacity in words
    wah::DevMeta h{};           // host copy of *meta
    bool h_valid = false;
    uint32_t* gt = nullptr;     // group-tile index (k_gtile), built on first use
    bool gt_valid = false;
    bool compressed_form = false;  // words are as compress() leaves them
};

// A kernel's launch setup on each device (the dynamic shared-memory limit is
// a per-device setting): resident CTAs per SM once set up, 0 before.
struct PerDeviceSetup {
    std::atomic<int> per_sm[64];
};
// Sets the kernel's dynamic shared-memory limit on the current device the
// first time it launches there; returns its resident CTAs per SM.
template <class Kernel>
int wg_kernel_setup(PerDeviceSetup& s, int device, Kernel k, int threads, size_t smem) {
    const int d = device >= 0 && device < 64 ? device : 0;
    int v = s.per_sm[d].load(std::memory_order_relaxed);
    if (v) return v;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k, threads, smem);
    if (v < 1) v = 1;
    s.per_sm[d].store(v, std::memory_order_relaxed);
    return v;
}
int wg_fail(wahgpu_ctx* ctx, int code, const char* fmt, ...);
void* wg_alloc(wahgpu_ctx* ctx, size_t bytes);
void wg_free(wahgpu_ctx* ctx, void* p);
void* wg_host_alloc(wahgpu_ctx* ctx, size_t bytes);
void wg_host_free(wahgpu_ctx* ctx, void* p);
int wg_scratch(wahgpu_ctx* ctx, uint32_t ntiles, wah::TileRec** recs, wah::LaunchSync** sync);
int wg_bv_meta(wahgpu_bv* b);
wahgpu_bv* wg_bv_new(wahgpu_ctx* ctx);
int wg_scan_meta(wahgpu_bv* b, uint32_t n, uint32_t anb, uint32_t aval);
int wg_launch_merge(wahgpu_ctx* ctx, int op, bool fsm, bool unary, bool flip,
                    const wahgpu_bv* x, const wahgpu_bv* y, uint32_t groups,
                    uint32_t anb, uint32_t aval, wahgpu_bv* res);
#endif
