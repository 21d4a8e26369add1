// Row ids of a serialized WAH bitvector in device memory, with no memory
// allocation anywhere on the call path.
//
// Who needs it: callers that must not allocate device memory while they
// work — GPU pipelines driven from host callbacks (a callback may not call
// cudaMalloc), embedding runtimes that own every device byte through their
// own memory pool and forbid a library from calling cudaMalloc behind their
// back, and latency-bound paths that cannot take the device-wide
// synchronisation an allocation may bring.  They pass device pointers for
// the input words and for the output, and this entry point computes into
// them using only a fixed scratch area compiled into the library.
//
// The scratch is one file-scope static __device__ array of NOALLOC_SCRATCH
// bytes; every device that loads the library holds it until the process
// exits.  All calls share it and it keeps the last call's contents (each
// call clears the words that must start at zero), so calls whose kernels
// overlap on the GPU race with each other: issue them on one stream, or
// order them.
#include "../../include/wahgpu.h"
#include "wah_dev.cuh"
#include "wah_api_internal.h"

#include <cuda_runtime.h>
#include <cstdio>
#include <mutex>
#include <string>

using namespace wah;

namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_WPT = 16;                            // words per thread
constexpr int NA_TILE = NA_THREADS * NA_WPT;          // 4096 words per tile
constexpr uint64_t NA_MAX_WORDS = 1ull << 24;         // 16,777,216 words (64 MiB)
constexpr uint32_t NA_MAX_TILES = (uint32_t)(NA_MAX_WORDS / NA_TILE) + 1;

struct NoAllocScratch {
    LaunchSync sync;          // ticket / done start at zero; epoch persists
    DevMeta status;           // cleared by every call
    TileRec recs[NA_MAX_TILES];
};
constexpr size_t NOALLOC_SCRATCH = sizeof(NoAllocScratch);  // about 197 KiB

// The scratch area.  Host code must not use this name as a device address:
// on the host it is a stand-in symbol; its device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH];

// Row ids are 32-bit (the reference's nbits is a 32-bit count), so a
// bitvector may cover at most 0xFFFFFFFF / 31 = 138,547,332 whole groups.
// Group counts saturate here in the look-back: above that limit, below the
// point where the sum of two could wrap.
constexpr uint32_t NA_GROUP_SAT = 0x7FFFFFFFu;

// 64-bit ones count + group count saturating at NA_GROUP_SAT (saturating
// addition is associative, so the look-back may combine in any grouping)
struct PosComb {
    __device__ __forceinline__ uint4 operator()(uint4 a, uint4 b) const {
        const uint64_t s = ((uint64_t)a.y << 32 | a.x) + ((uint64_t)b.y << 32 | b.x);
        return make_uint4((uint32_t)s, (uint32_t)(s >> 32), min(a.z + b.z, NA_GROUP_SAT), a.w | b.w);
    }
};

// One pass over serialized words: group positions and output offsets of
// every word come from a single decoupled look-back carrying both sums, so
// no block-position index (and no allocation for one) is needed.  Row ids:
// literal bit 30-k of the word at group g is row 31g+k; then the active
// word's bits, most significant first.
__global__ void __launch_bounds__(NA_THREADS)
k_rids_serial(const uint32_t* __restrict__ ser, uint64_t nser, uint32_t* __restrict__ out, uint64_t cap,
              unsigned long long* count, NoAllocScratch* S0, uint32_t ntiles) {
    __shared__ uint64_t sh_ones[NA_THREADS / 32 + 1];
    __shared__ uint64_t sh_grp[NA_THREADS / 32 + 1];
    __shared__ uint32_t hdr[2];
    __shared__ uint64_t tile_ones;
    __shared__ uint32_t tile_grp;
    __shared__ uint32_t fq_n;
    __shared__ uint64_t fq_off[NA_TILE / 2];
    __shared__ uint32_t fq_row[NA_TILE / 2];
    __shared__ uint64_t fq_len[NA_TILE / 2];
    if (threadIdx.x == 0) {
        hdr[0] = claim_tile(&S0->sync);
        hdr[1] = ld_cg(&S0->sync.epoch);
        fq_n = 0;
    }
    __syncthreads();
    const uint32_t t = hdr[0], epoch = hdr[1];
    // serialized trailer (src/bitvector.cpp:54-105)
    uint32_t n = 0, anb = 0, aval = 0;
    if (nser > 1) {
        const uint32_t last = __ldg(ser + nser - 1);
        if (last > 0 && last < MAXBITS) { anb = last; aval = __ldg(ser + nser - 2); n = (uint32_t)(nser - 2); }
        else n = (uint32_t)(nser - 1);
    }
    const uint32_t base = t * NA_TILE + threadIdx.x * NA_WPT;
    uint32_t v[NA_WPT];
    uint64_t ones = 0;
    uint64_t grp = 0;
#pragma unroll
    for (int q = 0; q < NA_WPT; ++q) {
        const bool in = base + q < n;
        v[q] = in ? __ldg(ser + base + q) : 0u;
        if (in) {
            const uint32_t x = v[q];
            if (x > ALLONES) {
                const uint32_t c = x & MAXCNT;
                grp += c;
                if (x >= HEADER1) ones += (uint64_t)c * 31u;
            } else {
                grp += 1;
                ones += __popc(x);
            }
        }
    }
    uint64_t ones_tot, grp_tot;
    const uint64_t ones_ex = block_exscan64(ones, sh_ones, ones_tot);
    const uint64_t grp_ex = block_exscan64(grp, sh_grp, grp_tot);
    if (threadIdx.x < 32) {
        const uint4 mine = make_uint4((uint32_t)ones_tot, (uint32_t)(ones_tot >> 32),
                                      (uint32_t)min(grp_tot, (uint64_t)NA_GROUP_SAT), 0u);
        uint4 pre = make_uint4(0, 0, 0, 0);
        bool ok = true;
        if (t == 0) {
            if (threadIdx.x == 0) publish(&S0->recs[0], epoch, REC_INCL, mine);
        } else {
            if (threadIdx.x == 0) publish(&S0->recs[t], epoch, REC_AGG, mine);
            pre = warp_lookback(S0->recs, t, epoch, make_uint4(0, 0, 0, 0), PosComb(), &ok);
            if (threadIdx.x == 0) publish(&S0->recs[t], epoch, REC_INCL, PosComb()(pre, mine));
        }
        if (threadIdx.x == 0) {
            if (!ok) {
                // a wait gave up: the count reads UINT64_MAX
                atomicExch(&S0->status.status, DEV_ERR_TIMEOUT);
                atomicMax(count, ~0ull);
            }
            tile_ones = (uint64_t)pre.y << 32 | pre.x;
            tile_grp = pre.z;
            if (t == ntiles - 1) {
                const uint64_t groups = (uint64_t)tile_grp + grp_tot;
                if (groups * 31u + anb > 0xFFFFFFFFull) {
                    // more bits than 32-bit row ids can number: the count
                    // reads UINT64_MAX, as for a wait that gave up
                    atomicExch(&S0->status.status, DEV_ERR_RANGE);
                    atomicMax(count, ~0ull);
                } else {
                    // the active word's rows follow the last whole group
                    uint64_t off = tile_ones + ones_tot;
                    const uint32_t rbase = (uint32_t)groups * 31u;
                    for (uint32_t b = 0; b < anb; ++b)
                        if ((aval >> (anb - 1u - b)) & 1u) { if (off < cap) out[off] = rbase + b; ++off; }
                    atomicMax(count, (unsigned long long)off);
                }
            }
        }
    }
    __syncthreads();
    uint64_t off = tile_ones + ones_ex;
    uint32_t g = tile_grp + (uint32_t)grp_ex;
#pragma unroll
    for (int q = 0; q < NA_WPT; ++q) {
        if (base + q < n) {
            const uint32_t x = v[q];
            if (x > ALLONES) {
                const uint32_t c = x & MAXCNT;
                if (x >= HEADER1) {
                    // only the ids that fit below cap are written; the
                    // count comes from the look-back, not from these loops
                    const uint64_t len = off < cap ? min((uint64_t)c * 31u, cap - off) : 0ull;
                    if (len) {
                        const uint32_t slot = atomicAdd(&fq_n, 1u);
                        if (slot < (uint32_t)(NA_TILE / 2)) {
                            fq_off[slot] = off; fq_row[slot] = g * 31u; fq_len[slot] = len;
                        } else {  // list full: this thread writes the fill
                            for (uint64_t r = 0; r < len; ++r) out[off + r] = g * 31u + (uint32_t)r;
                        }
                    }
                    off += (uint64_t)c * 31u;
                }
                g += c;
            } else {
                uint32_t bits = x;
                while (bits) {
                    const uint32_t b = 31u - __clz(bits);
                    if (off < cap) out[off] = g * 31u + (30u - b);
                    ++off;
                    bits &= ~(1u << b);
                }
                g += 1;
            }
        }
    }
    __syncthreads();
    const uint32_t nfq = min(fq_n, (uint32_t)(NA_TILE / 2));
    for (uint32_t k = 0; k < nfq; ++k) {
        const uint64_t o = fq_off[k], len = fq_len[k];  // o + len <= cap
        const uint32_t r0 = fq_row[k];
        for (uint64_t r = threadIdx.x; r < len; r += NA_THREADS) out[o + r] = r0 + (uint32_t)r;
    }
    __syncthreads();
    if (threadIdx.x == 0) finish_tile(&S0->sync, ntiles);
}

// Per-device address of the scratch area, looked up once per device.
std::mutex g_mu;
void* g_addr[64] = {};

int na_fail(int code, const char* msg) { return wg_fail(nullptr, code, "%s", msg); }

}  // namespace

extern "C" int wahgpu_rids_noalloc(const uint32_t* dev_serial, uint64_t nwords, uint32_t* dev_rids,
                                   uint64_t cap, unsigned long long* dev_count, void* stream) {
    if ((nwords && !dev_serial) || !dev_count || (cap && !dev_rids))
        return na_fail(WAHGPU_EINVAL, "wahgpu_rids_noalloc: a pointer argument is NULL");
    if (nwords > NA_MAX_WORDS + 2)
        return na_fail(WAHGPU_ESIZE, "wahgpu_rids_noalloc: the bitvector holds more than 16,777,216 words, "
                                     "the limit of the fixed scratch area; use wahgpu_bv_rids_device");
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return na_fail(WAHGPU_ENODEV, "wahgpu_rids_noalloc: no current CUDA device");
    }
    void* addr = nullptr;
    {
        std::lock_guard<std::mutex> g(g_mu);
        if (!g_addr[dev]) {
            // once per device, with that device current: the device address
            // of the scratch array (its host-side name is not one)
            cudaError_t e = cudaGetSymbolAddress(&g_addr[dev], g_noalloc_scratch);
            if (e != cudaSuccess) {
                g_addr[dev] = nullptr;
                cudaGetLastError();
                return na_fail(WAHGPU_ECUDA, "wahgpu_rids_noalloc: cudaGetSymbolAddress failed");
            }
        }
        addr = g_addr[dev];
    }
    NoAllocScratch* S0 = static_cast<NoAllocScratch*>(addr);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // ticket and done must be zero when a launch starts (a finished launch
    // leaves them zero); the status word is per call; the epoch is kept so
    // records of earlier calls never pass for current ones
    if (cudaMemsetAsync(&S0->sync, 0, 2 * sizeof(uint32_t), s) != cudaSuccess ||
        cudaMemsetAsync(&S0->status, 0, sizeof(DevMeta), s) != cudaSuccess ||
        cudaMemsetAsync(dev_count, 0, sizeof(unsigned long long), s) != cudaSuccess) {
        cudaGetLastError();
        return na_fail(WAHGPU_ECUDA, "wahgpu_rids_noalloc: clearing the scratch area failed");
    }
    const uint64_t n = nwords > 1 ? nwords - 1 : 0;  // at most this many whole words
    const uint32_t ntiles = n ? (uint32_t)((n + NA_TILE - 1) / NA_TILE) : 1u;
    k_rids_serial<<<ntiles, NA_THREADS, 0, s>>>(dev_serial, nwords, dev_rids, cap, dev_count, S0, ntiles);
    if (cudaGetLastError() != cudaSuccess) return na_fail(WAHGPU_ECUDA, "wahgpu_rids_noalloc: launch failed");
    return WAHGPU_OK;
}
