/*
 * libwahgpu — B200 (sm_100a) implementation of FastBit's WAH bitvector
 * operators and relic/bin range evaluation, behind a C ABI.
 *
 * Every entry point returns an int (or int64_t) status: >= 0 on success,
 * a negative WAHGPU_E* code on failure (the convention of the reference's
 * in-memory C API, src/iapi.cpp:1383-1429).  The text of the last error of a
 * context is available from wahgpu_last_error().  No C++ exception crosses
 * this boundary and no call falls back to a CPU computation: without a
 * usable sm_100 device every call fails with WAHGPU_ENODEV.
 *
 * Bitvectors use the reference's serialized layout (src/bitvector.cpp:
 * 2283-2313, write(array_t<word_t>&)): the whole 32-bit WAH words of m_vec,
 * then the active word's value if it holds any bits, then the active word's
 * bit count.  Row ids are uint32 positions, ascending.
 *
 * A context belongs to one device (wahgpu_ctx_create makes it current);
 * like the CUDA runtime's own libraries, its calls run on the calling
 * thread's current device, so a process that drives several GPUs makes the
 * context's device current (cudaSetDevice) before calling into it.
 */
#ifndef WAHGPU_H
#define WAHGPU_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WAHGPU_OK 0
#define WAHGPU_EINVAL (-1)     /* bad argument */
#define WAHGPU_ENODEV (-2)     /* no usable CUDA device */
#define WAHGPU_ECUDA (-3)      /* a CUDA call failed */
#define WAHGPU_ENOMEM (-4)     /* device or host allocation failed */
#define WAHGPU_EFORMAT (-5)    /* malformed serialized bitvector */
#define WAHGPU_ERANGE (-6)     /* more bits than a 32-bit count holds */
#define WAHGPU_ETIMEOUT (-7)   /* a bounded device-side wait gave up */
#define WAHGPU_ESIZE (-8)      /* output buffer too small */
#define WAHGPU_EDEGENERATE (-9) /* operand the reference would corrupt, see below */
#define WAHGPU_EBUSY (-10)     /* admission refused: scratch budget exhausted */

/* Operators, numbered as the oracle and the reference's operator order. */
#define WAHGPU_AND 0   /* operator&  / &=  (src/bitvector.cpp:1194, 1292) */
#define WAHGPU_OR 1    /* operator|  / |=  (src/bitvector.cpp:1413, 1488) */
#define WAHGPU_XOR 2   /* operator^  / ^=  (src/bitvector.cpp:1557, 1624) */
#define WAHGPU_MINUS 3 /* operator-  / -=  (src/bitvector.cpp:1685, 1768) */

typedef struct wahgpu_ctx wahgpu_ctx; /* a device, a stream, scratch, a pool */
typedef struct wahgpu_bv wahgpu_bv;   /* a device-resident ibis::bitvector */

typedef struct {
    uint64_t nwords;  /* m_vec.size() */
    uint64_t nbits;   /* size(): bits in m_vec plus active bits */
    uint64_t cnt;     /* cnt(): number of 1 bits */
    uint32_t anb;     /* active.nbits */
    uint32_t aval;    /* active.val */
    uint32_t compressed_form; /* 1: words are as compress() leaves them */
} wahgpu_bv_info;

/* ---- context ---------------------------------------------------------- */
/* Creates a context on CUDA device `device` with its own stream. */
int wahgpu_ctx_create(int device, wahgpu_ctx** out);
int wahgpu_ctx_destroy(wahgpu_ctx* ctx);
/* Runs the context's work on `stream` (a cudaStream_t); NULL restores the
 * context's own stream. */
int wahgpu_ctx_set_stream(wahgpu_ctx* ctx, void* stream);
void* wahgpu_ctx_stream(wahgpu_ctx* ctx);
/* Waits for all work queued on the context's stream. */
int wahgpu_ctx_sync(wahgpu_ctx* ctx);
const char* wahgpu_last_error(wahgpu_ctx* ctx);
/* Number of kernels this context has launched (diagnostics). */
int64_t wahgpu_ctx_launches(wahgpu_ctx* ctx);

/* Launch-shape knobs, set by an autotuner (no counterpart in the reference;
 * results never depend on them).  Values outside the listed set are
 * rejected with WAHGPU_EINVAL. */
#define WAHGPU_TUNE_DENSE_TILE 1  /* groups per tile of the dense-path kernel: 1024 | 2048 | 4096 */
#define WAHGPU_TUNE_DENSE_ENGINE 4 /* canonical-result operators: 0 auto (= 3), 1 pipelined group-space kernel, \
                                      2 word-space merge, 3 two-pass group-space kernels, \
                                      4 single-pass group-space kernel over CTA tiles, \
                                      5 single-pass group-space kernel over warp tiles */
#define WAHGPU_TUNE_RANGE_ORDER 2 /* batch work order: 0 query by query; 1 (default) tile by tile for count-only \
                                     batches, else query by query; 2 tile by tile, row ids of several queries \
                                     placed by a count pass and a scan (capped batches: the id pass revisits \
                                     only the tiles holding ids under each query's limit) */
#define WAHGPU_TUNE_RANGE_CTAS 3  /* resident CTAs per SM of the persistent range launch: 0 (all that fit) .. 32 */
#define WAHGPU_TUNE_CUM_STRIDE 5  /* bitmaps per cumulative row of indexes built or attached later: 0 auto, 1 none, >= 2 that stride */
#define WAHGPU_TUNE_MERGE_TILE 6  /* block-index entries per tile of the word-space merge: 0 auto (by operand size), 16 | 32 | 64 */
/* Failure-path test hooks (no counterpart in the reference; never needed in
 * normal use).  WAHGPU_TEST_WITHHOLD_TILE = t: in the next operator call on
 * the single-pass group-space engine, tile t never publishes its look-back
 * record, so the tile after it waits until its bounded wait gives up and
 * the call reports WAHGPU_ETIMEOUT (the hook then clears itself).
 * WAHGPU_TEST_FAIL_ALLOC = n: the n-th device allocation from now fails as
 * if the device were out of memory (WAHGPU_ENOMEM), once. */
#define WAHGPU_TEST_WITHHOLD_TILE 100
#define WAHGPU_TEST_FAIL_ALLOC 101
int wahgpu_ctx_set_tuning(wahgpu_ctx* ctx, int key, int64_t value);
int64_t wahgpu_ctx_get_tuning(wahgpu_ctx* ctx, int key);

/* ---- bitvectors ------------------------------------------------------- */
/* Builds a device bitvector from a serialized host array, like the
 * reference's constructor from array_t<word_t> (src/bitvector.cpp:54-105):
 * the words are copied as given (not compressed). */
int wahgpu_bv_from_serial(wahgpu_ctx* ctx, const uint32_t* words, uint64_t nwords,
                          wahgpu_bv** out);
/* Same from a serialized array already in device memory (read on the
 * device; the trailer words are read back to the host).  The words are read
 * in order on the context's stream, which waits for no other stream: work
 * still writing them on another stream must be ordered before the call
 * (an event recorded there and waited on by wahgpu_ctx_stream's stream). */
int wahgpu_bv_from_device_serial(wahgpu_ctx* ctx, const uint32_t* dev_words, uint64_t nwords,
                                 wahgpu_bv** out);
/* An empty bitvector with room for `cap_words` whole words, for use as the
 * destination of wahgpu_bv_binop_into. */
int wahgpu_bv_create(wahgpu_ctx* ctx, uint64_t cap_words, wahgpu_bv** out);
int wahgpu_bv_free(wahgpu_bv* bv);
/* Metadata; waits for the kernel that produced the bitvector. */
int wahgpu_bv_info_get(wahgpu_bv* bv, wahgpu_bv_info* info);
/* size() (src/bitvector.h:647) and cnt() (src/bitvector.h:652). */
int64_t wahgpu_bv_size(wahgpu_bv* bv);
int64_t wahgpu_bv_cnt(wahgpu_bv* bv);
/* Serialized length in words (getSerialSize()/4, src/bitvector.h:150). */
int64_t wahgpu_bv_serial_size(wahgpu_bv* bv);
/* write(array_t<word_t>&) (src/bitvector.cpp:2283): copies the serialized
 * form to host memory; returns its length in words, WAHGPU_ESIZE if cap is
 * too small. */
int64_t wahgpu_bv_write(wahgpu_bv* bv, uint32_t* out, uint64_t cap);
/* Device pointer to the whole words (m_vec) of a bitvector. */
const uint32_t* wahgpu_bv_device_words(wahgpu_bv* bv);

/* ---- operators --------------------------------------------------------- */
/* *res = a OP b, or a OP= b when inplace != 0, followed by compress():
 * the words equal the reference's operator output after compress()
 * (src/bitvector.cpp:1194-1838, kernels 2419-4079, compress 378-469).
 * For inplace the result is also returned in *res (a is not modified: the
 * device keeps operands immutable).  Operands of different sizes are handled
 * as the reference does: the shorter one is padded with 0 bits (adjustSize,
 * src/bitvector.cpp:4086) and the operator runs in its OP= form.
 *
 * Operands whose every word covers one 31-bit group while some word is a
 * fill (a count-1 fill word) make the reference take its uncompressed loops
 * with the fill header combined as literal bits; such calls return
 * WAHGPU_EDEGENERATE. */
int wahgpu_bv_binop(wahgpu_ctx* ctx, int op, int inplace, wahgpu_bv* a, wahgpu_bv* b,
                    wahgpu_bv** res);
/* Same into an existing bitvector (its capacity must be at least
 * nwords(a) + nwords(b)); allocation free when the capacity suffices. */
int wahgpu_bv_binop_into(wahgpu_ctx* ctx, int op, int inplace, wahgpu_bv* a, wahgpu_bv* b,
                         wahgpu_bv* res);
/* compress() (src/bitvector.cpp:378): in place on the device. */
int wahgpu_bv_compress(wahgpu_bv* bv);
/* decompress() (src/bitvector.cpp:474): in place on the device. */
int wahgpu_bv_decompress(wahgpu_bv* bv);
/* flip() (src/bitvector.cpp:1128) followed by compress(). */
int wahgpu_bv_flip(wahgpu_bv* bv);
/* Row ids of the 1 bits in ascending order (firstIndexSet()/indexSet walk,
 * src/bitvector.cpp:4524), into host memory; returns the count (cnt()),
 * WAHGPU_ESIZE if cap is too small. */
int64_t wahgpu_bv_rids(wahgpu_bv* bv, uint32_t* out, uint64_t cap);
/* Same into device memory (dev_out holds cap uint32). */
int64_t wahgpu_bv_rids_device(wahgpu_bv* bv, uint32_t* dev_out, uint64_t cap);

/* ---- indexes and range evaluation ------------------------------------- */
#define WAHGPU_RELIC 1  /* ibis::relic: one bitmap per distinct value */
#define WAHGPU_BIN 2    /* ibis::bin: one bitmap per value bin */
/* comparison of a range term (qExpr::COMPARE subset) */
#define WAHGPU_CMP_NONE 0
#define WAHGPU_CMP_LT 1
#define WAHGPU_CMP_LE 2
/* value types of a raw column */
#define WAHGPU_U32 0
#define WAHGPU_F32 1
#define WAHGPU_I32 2

typedef struct wahgpu_index wahgpu_index; /* a device-resident relic / bin index */
typedef struct wahgpu_batch wahgpu_batch; /* a prepared set of queries */

/* One range term  `lo lop x rop hi`  on the column of `idx`
 * (ibis::qContinuousRange, src/qExpr.h:259-280; CMP_NONE drops a side). */
typedef struct {
    wahgpu_index* idx;
    int lop;
    double lo;
    int rop;
    double hi;
} wahgpu_term;

/* Attaches an index given as the reference's serialized triple — keys
 * (relic: the distinct values; bin: minval[nobs] then maxval[nobs]), word
 * offsets of the nobs+1 bitmap boundaries, and the concatenated serialized
 * bitmaps — as produced by relic::write / bin::write (src/irelic.cpp:644,
 * src/ibin.cpp:5836) and fastbit_iapi_deconstruct_index (src/iapi.cpp:1915);
 * the constructors from such a triple are relic(col, nb, keys, offs, bms)
 * (src/irelic.h:30-34) and bin(col, nb, keys, offs) (src/ibin.cpp:432).
 * The arrays are copied to the device; nrows is the column's row count. */
int wahgpu_index_from_triple(wahgpu_ctx* ctx, int kind, uint64_t nrows, const double* keys,
                             uint64_t nkeys, const int64_t* offsets, uint64_t noffsets,
                             const uint32_t* bitmaps, uint64_t nbitmaps, wahgpu_index** out);
/* The raw column (nrows values of type vtype) for the rows of edge bins that
 * the reference checks value by value (bin::checkBin / part::doScan,
 * src/ibin.cpp:2057-2304, src/part.cpp:4273). */
int wahgpu_index_set_values(wahgpu_index* idx, int vtype, const void* values, uint64_t n);
/* Builds an index of a column held in device memory, on the device
 * (replaces relic::construct, src/irelic.cpp:879-925, with mapValues,
 * src/index.cpp:2552-2611; and bin construction with
 * <binning nbins=N equal_weight/>, src/ibin.cpp:2390-2582, 3350-3449).
 * kind WAHGPU_RELIC: one bitmap per distinct value, keys ascending.
 * kind WAHGPU_BIN: nbins bins of about equal row counts; a distinct value is
 * never split between bins, and each bin's keys are the smallest and
 * largest value it holds; the raw values are kept for edge-bin row checks.
 * Every bitmap holds exactly the rows the reference's would; its words are
 * in compress() form.  `dev_values` is read on the context's stream, as for
 * wahgpu_bv_from_device_serial: order its producers before the call. */
int wahgpu_index_build(wahgpu_ctx* ctx, int kind, int vtype, const void* dev_values, uint64_t nrows,
                       uint32_t nbins, wahgpu_index** out);
/* Index files.  wahgpu_index_read replaces relic::read(const char*) and
 * bin::read(const char*) (src/irelic.cpp:690-786, src/ibin.cpp:468-540) for
 * the .idx files relic::write / bin::write produce (src/irelic.cpp:354-642,
 * src/ibin.cpp:5530-5834; index types RELIC and BINNING, 4- or 8-byte
 * bitmap offsets): the file is read on the host and attached like a
 * triple.  The raw column for bin edge checks still comes from
 * wahgpu_index_set_values.  Errors: WAHGPU_EINVAL (cannot open or read),
 * WAHGPU_EFORMAT (not such a file, or its offsets are inconsistent). */
int wahgpu_index_read(wahgpu_ctx* ctx, const char* path, wahgpu_index** out);
/* The same from a file image already in host memory (a mapped file). */
int wahgpu_index_from_file_image(wahgpu_ctx* ctx, const void* data, uint64_t bytes, wahgpu_index** out);
/* Host only, no device: the triple an index file image holds, in the layout
 * wahgpu_index_from_triple takes (kind, nrows, keys, word offsets, bitmaps;
 * a bitmap the writer left out stays zero words long).
 * Sizes are always reported; the arrays are filled when all three are given
 * (WAHGPU_ESIZE when a capacity is short).  Errors: wahgpu_last_error(NULL). */
int wahgpu_idxfile_parse(const void* data, uint64_t bytes, int* kind, uint64_t* nrows, double* keys,
                         uint64_t kcap, uint64_t* nkeys, int64_t* offsets, uint64_t ocap, uint64_t* noffsets,
                         uint32_t* bitmaps, uint64_t bcap, uint64_t* nbitmaps);
/* A copy of bitmap j as a bitvector (index::getBitvector, src/index.h). */
int wahgpu_index_bitmap(wahgpu_index* idx, uint32_t j, wahgpu_bv** out);
/* The index's keys in the triple's layout (relic: values; bin: minval then
 * maxval); returns their count, WAHGPU_ESIZE if cap is too small. */
int64_t wahgpu_index_keys(wahgpu_index* idx, double* out, uint64_t cap);

/* The index as the reference's serialized triple, the layout
 * wahgpu_index_from_triple takes and relic::write(keys, starts, bitmaps) /
 * bin::write(keys, starts, bitmaps) produce (src/irelic.cpp:644-667,
 * src/ibin.cpp:5836-5859; fastbit_iapi_deconstruct_index,
 * src/iapi.cpp:1915): keys (relic: values; bin: minval then maxval), the
 * nobs + 1 word offsets, the bitmaps' serialized words.  Sizes are always
 * reported; the arrays are filled when all three are given (WAHGPU_ESIZE
 * when a capacity is short).  A triple from here attaches to the reference
 * with fastbit_iapi_attach_full_index (src/iapi.cpp:2018). */
int wahgpu_index_deconstruct(wahgpu_index* idx, double* keys, uint64_t kcap, uint64_t* nkeys,
                             int64_t* offsets, uint64_t ocap, uint64_t* noffsets, uint32_t* bitmaps,
                             uint64_t bcap, uint64_t* nbitmaps);

int wahgpu_index_free(wahgpu_index* idx);
int64_t wahgpu_index_nbitmaps(wahgpu_index* idx);
int64_t wahgpu_index_nrows(wahgpu_index* idx);
/* estimate(count) without a range: all 1 bits (src/irelic.cpp:1843). */
int64_t wahgpu_index_total_ones(wahgpu_index* idx);

/* index::estimate(expr, lower, upper) (src/index.h:191) for one term:
 * *lower = the rows certainly hit, *upper = a superset of the hits, both as
 * new bitvectors (compress() form).  relic (src/irelic.h:58-62): lower =
 * the hits, upper empty.  bin (src/ibin.cpp:6722-6829): lower = the bins
 * wholly inside the range, upper = those and the edge bins, empty when no
 * bin straddles an end.  An empty upper means lower is exact (the
 * reference's convention).  Needs no raw values. */
int wahgpu_estimate(wahgpu_ctx* ctx, const wahgpu_term* term, wahgpu_bv** lower, wahgpu_bv** upper);
/* index::estimate(expr) (src/index.h:196): an upper bound of one term's hit
 * count — relic: exact (src/irelic.cpp:1843-1854); bin: the 1 bits of the
 * bins wholly inside and of the edge bins (src/ibin.cpp:6832-6889).
 * Computed on the host from per-bitmap counts. */
int64_t wahgpu_estimate_count(wahgpu_ctx* ctx, const wahgpu_term* term);

/* Evaluates the AND of nterms range terms (countQuery::evaluate,
 * src/countQuery.cpp:292-332, whose terms go through relic::evaluate /
 * bin::evaluate, src/irelic.cpp:1827, src/ibin.cpp:6614).  Returns the hit
 * count (getNumHits, src/countQuery.cpp:376); writes the ascending row ids
 * (getHitRows, src/countQuery.cpp:387) to rids when it is non-NULL, and the
 * hit bitvector after compress() to *hits when hits is non-NULL. */
int64_t wahgpu_evaluate(wahgpu_ctx* ctx, const wahgpu_term* terms, uint32_t nterms,
                        uint32_t* rids, uint64_t cap, wahgpu_bv** hits);

/* Batches: nq conjunctive queries, query q being terms
 * [query_offsets[q], query_offsets[q+1]); all indexes of a batch share one
 * row count.  The whole batch runs as one kernel launch (wahgpu_batch_run,
 * capturable in a CUDA graph); rid_cap > 0 keeps the row ids of all queries
 * back to back in device memory, rid_cap == 0 counts only. */
int wahgpu_batch_create(wahgpu_ctx* ctx, const wahgpu_term* terms, const uint32_t* query_offsets,
                        uint32_t nq, uint64_t rid_cap, int dense_first, wahgpu_batch** out);
/* Like wahgpu_batch_create with row ids, but each query keeps at most
 * rid_caps[q] of its row ids (the first ones, ascending — a LIMIT), in a
 * region of its own, so one query with many hits cannot crowd out the
 * others (no counterpart in the reference, whose getHitRows returns all
 * rows, src/countQuery.cpp:387-410).  Counts are always complete;
 * wahgpu_batch_rids returns min(count, rid_caps[q]) ids.  Runs query by
 * query. */
int wahgpu_batch_create_capped(wahgpu_ctx* ctx, const wahgpu_term* terms, const uint32_t* query_offsets,
                               uint32_t nq, const uint64_t* rid_caps, wahgpu_batch** out);
int wahgpu_batch_run(wahgpu_batch* batch);
int wahgpu_batch_counts(wahgpu_batch* batch, uint64_t* counts);
int64_t wahgpu_batch_rids(wahgpu_batch* batch, uint32_t q, uint32_t* out, uint64_t cap);
const uint32_t* wahgpu_batch_device_rids(wahgpu_batch* batch);
/* Algorithmic bytes one run reads: per term the words of the bitmaps it
 * ORs (or their complement), of its edge bitmaps and the raw values of the
 * edge bitmaps' rows; 8 per query for the count. */
int64_t wahgpu_batch_bytes(wahgpu_batch* batch);
/* Bytes any evaluation of the batch must move, whatever the index layout:
 * per term the words of the bitmaps sumBins ORs — the covered set, or its
 * complement when that is smaller (src/index.cpp:6450-6520) — plus the edge
 * bitmaps' words and one raw value per edge row (bin::checkBin,
 * src/ibin.cpp:2220); 8 bytes per count.  (Row ids add 4 bytes each.) */
int64_t wahgpu_batch_min_bytes(wahgpu_batch* batch);
int wahgpu_batch_free(wahgpu_batch* batch);


/* ---- serving ----------------------------------------------------------- */
/* Continuous batching of conjunctive range queries over resident indexes
 * (no counterpart in the reference, which evaluates one query per caller
 * under a global lock, src/iapi.cpp:33).  A worker thread keeps `nslots`
 * execution slots (each its own stream and scratch); an idle slot takes the
 * waiting queries in arrival order, as many as fit `max_batch` and the
 * scratch budget (device bytes for their evaluation), and runs them as one
 * batch while later arrivals queue for the next idle slot.  Results are
 * those of wahgpu_evaluate for each query alone. */
typedef struct wahgpu_server wahgpu_server;
int wahgpu_server_create(wahgpu_ctx* ctx, uint32_t nslots, uint32_t max_batch, uint64_t scratch_budget,
                         wahgpu_server** out);
/* Queues one query (its terms are copied); returns a request id > 0, or
 * WAHGPU_EBUSY when the query's scratch alone exceeds the budget.  rid_cap
 * > 0 asks for its first rid_cap row ids (ascending, like a LIMIT); its
 * count is always complete. */
int64_t wahgpu_server_submit(wahgpu_server* s, const wahgpu_term* terms, uint32_t nterms, uint64_t rid_cap);
/* Waits for a request: hit count, row ids (if asked for), latency in
 * seconds from submit to answer; returns the number of row ids written. */
int64_t wahgpu_server_wait(wahgpu_server* s, int64_t id, uint64_t* count, uint32_t* rids, uint64_t cap,
                           double* latency_s);
/* Open-loop replay: query q = terms[qoff[q], qoff[q+1]) arrives arrival_s[q]
 * seconds after the call starts; waits for all; counts and latencies
 * (scheduled arrival to answer) per query; with rid_cap > 0 every query also
 * returns its first rid_cap row ids, written to rids + q * rid_cap (when
 * rids is non-NULL) with their number in nrids[q].  Returns the wall time
 * in microseconds. */
int64_t wahgpu_server_replay(wahgpu_server* s, const wahgpu_term* terms, const uint32_t* qoff, uint32_t nq,
                             const double* arrival_s, uint64_t rid_cap, uint64_t* counts, double* latency_s,
                             uint32_t* rids, uint64_t* nrids);
int wahgpu_server_stats(wahgpu_server* s, uint64_t* batches, uint64_t* served);
int wahgpu_server_free(wahgpu_server* s);

/* ---- allocation-free row ids -------------------------------------------
 * No counterpart in the reference: an addition for callers that cannot
 * allocate device memory while they run — pipelines driven from host
 * callbacks (which may not call CUDA API functions such as cudaMalloc),
 * runtimes that own all device memory through their own pool and do not let
 * a library allocate behind their back, and latency-bound paths that cannot
 * afford the device-wide synchronisation an allocation may cause.  Computes
 * the ascending row ids of the serialized bitvector at dev_serial (nwords
 * words in device memory, the write(array_t&) layout) into dev_rids (room
 * for cap ids; ids past cap are dropped, the count is still the full count)
 * and its count into *dev_count (device memory), on `stream`, without
 * allocating anything: its scratch is a fixed area of about 197 KiB compiled
 * into the library, held by every device that loads it until the process
 * exits.  *dev_count reads UINT64_MAX when a device-side wait gave up or the
 * bitvector holds more bits than 32-bit row ids can number (the reference's
 * nbits limit).  Limit: at most 16,777,216 whole words (WAHGPU_ESIZE
 * beyond).  The first call on a device looks up the scratch area's device
 * address (cudaGetSymbolAddress) — make it before any stream capture.  All
 * calls share the scratch area and it keeps the last call's contents (each
 * call clears what must start at zero): calls whose kernels overlap on the
 * GPU race, so order them (one stream).  Errors: wahgpu_last_error(NULL). */
int wahgpu_rids_noalloc(const uint32_t* dev_serial, uint64_t nwords, uint32_t* dev_rids,
                        uint64_t cap, unsigned long long* dev_count, void* stream);

#ifdef __cplusplus
}
#endif
#endif
