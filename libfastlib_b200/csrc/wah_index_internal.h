// Internal state behind the opaque index and batch handles of
// include/wahgpu.h, shared by the index store (wah_index.cu) and the device
// index builder (wah_build.cu).
#ifndef WAH_INDEX_INTERNAL_H
#define WAH_INDEX_INTERNAL_H
#include <vector>
#include "wah_range.cuh"
#include "wah_api_internal.h"

struct wahgpu_index {
    wahgpu_ctx* ctx = nullptr;
    int kind = 0;                 // WAHGPU_RELIC / WAHGPU_BIN
    uint32_t nrows = 0, groups = 0, anb = 0, nobs = 0, ntiles = 0;
    std::vector<double> keys;     // relic: distinct values; bin: minval then maxval
    std::vector<uint64_t> bwords; // m_vec words per bitmap (for the complement choice)
    std::vector<uint32_t> bones;  // 1 bits per bitmap
    std::vector<uint64_t> cum_words, cum_ones;  // prefix sums of bwords / bones
    // bin: the bins holding rows, in bitmap order, and whether their
    // [minval, maxval] are ordered and disjoint (then locate searches them)
    std::vector<uint32_t> nonempty;
    bool bins_sorted = false;
    uint32_t* d_words = nullptr;
    wah::BitmapMeta* d_bm = nullptr;
    uint32_t* d_tiles = nullptr;
    uint32_t* d_tl_off = nullptr;     // per tile: bitmaps with a 1 bit there (CSR)
    uint32_t* d_tl_bm = nullptr;
    uint32_t* d_cum = nullptr;        // cumulative dense rows (range spans in two reads)
    uint32_t cum_stride = 0, cum_k = 0;
    void* d_values = nullptr;
    uint32_t vtype = 0;
    wah::DevIndex dev{};
};

struct wahgpu_batch {
    wahgpu_ctx* ctx = nullptr;
    uint32_t nq = 0, nterms = 0, nidx = 0;
    uint32_t groups = 0, anb = 0, ntiles = 0;
    wah::DevIndex* d_idx = nullptr;
    wah::DevTerm* d_terms = nullptr;
    wah::DevQuery* d_queries = nullptr;
    unsigned long long* d_counts = nullptr;
    unsigned long long* d_start = nullptr;
    uint32_t* d_rids = nullptr;
    uint64_t rid_cap = 0;
    uint32_t* d_dense = nullptr;
    wah::DevMeta* d_status = nullptr;
    // two-pass order: per-item hits and first row-id slots (2 x nq*ntiles)
    // and the scan's temporary storage, allocated at the first such run
    unsigned long long* d_items = nullptr;
    void* d_scan_tmp = nullptr;
    size_t scan_tmp_bytes = 0;
    std::vector<unsigned long long> h_counts, h_start;
    uint64_t bytes = 0;               // algorithmic bytes one run reads
    uint64_t min_bytes = 0;           // the bytes sumBins itself must read (covered set or complement)
    bool capped = false;              // row ids limited per query, each query in a region of its own
    std::vector<uint64_t> h_lim, h_base;
    bool h_valid = false;
    unsigned char* h_stage = nullptr;  // pinned staging of the uploaded tables
};

int wg_index_attach(wahgpu_index* x);
int wg_batch_fetch_all(wahgpu_batch* B, uint32_t* rids);
#endif
