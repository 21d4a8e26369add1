// Device-side plumbing shared by the kernels: result metadata, tile records
// for single-pass decoupled look-back scans, bounded waits, and warp helpers.
#ifndef WAH_DEV_CUH
#define WAH_DEV_CUH
#include <stdint.h>
#include <cuda/atomic>
#include "wah_core.cuh"

namespace wah {

// Metadata of a device-resident bitvector, written by the kernel that
// produced it (or by the upload scan).  Mirrors the reference's members:
// m_vec.size() = n, nbits = 31*groups, nset, active.{nbits,val}.
struct DevMeta {
    uint32_t n;       // words in m_vec
    uint32_t groups;  // 31-bit groups covered by m_vec
    uint32_t nset;    // 1 bits in m_vec
    uint32_t anb;     // active bits
    uint32_t aval;    // active value
    uint32_t w0;      // first word (0 when n == 0)
    uint32_t nfill;   // nonzero when m_vec holds at least one fill word
    uint32_t status;  // 0 ok, else a WAH_E* code raised on the device
};

// error codes raised on the device (mirrored in include/wahgpu.h)
constexpr uint32_t DEV_ERR_TIMEOUT = 1;  // a look-back wait gave up
constexpr uint32_t DEV_ERR_FORMAT = 2;   // malformed words (count-0 fill)
constexpr uint32_t DEV_ERR_RANGE = 3;    // more groups than fit in 32 bits

// Per-launch synchronisation words in scratch memory.  A launch claims tile
// numbers from `ticket`; the last CTA to finish resets `ticket` and `done`
// and advances `epoch`, so tile records from earlier launches (including
// earlier replays of a captured graph) are never mistaken for current ones.
struct LaunchSync {
    uint32_t ticket;
    uint32_t done;
    uint32_t epoch;
    uint32_t pad;
};

constexpr uint32_t REC_AGG = 1, REC_INCL = 2;
constexpr uint32_t SPIN_LIMIT = 1u << 22;  // ~1 s worst case with backoff

struct TileRec {
    uint32_t flag;  // epoch*4 + state
    uint32_t pad[3];
    uint4 agg;      // this tile alone
    uint4 incl;     // this tile and all before it
};

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> r(*const_cast<uint32_t*>(p));
    return r.load(cuda::memory_order_acquire);
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> r(*p);
    r.store(v, cuda::memory_order_release);
}
// Look-back records are read and written at L2 only (.cg): polling them with
// acquire loads would invalidate the L1 of the polling SM on every poll and
// stall the other CTAs resident there.
__device__ __forceinline__ uint32_t ld_cg(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint4 ld_cg4(const uint4* p) {
    uint4 v;
    asm volatile("ld.global.cg.v4.u32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_cg4(uint4* p, uint4 v) {
    asm volatile("st.global.cg.v4.u32 [%0], {%1,%2,%3,%4};"
                 :: "l"(p), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w) : "memory");
}
__device__ __forceinline__ void st_cg(uint32_t* p, uint32_t v) {
    asm volatile("st.global.cg.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

// Payload first, a fence, then the flag.
__device__ __forceinline__ void publish(TileRec* r, uint32_t epoch, uint32_t state, uint4 v) {
    st_cg4(state == REC_AGG ? &r->agg : &r->incl, v);
    __threadfence();
    st_cg(&r->flag, epoch * 4u + state);
}

// Claims a tile number for this CTA (thread 0 writes it to *slot).
__device__ __forceinline__ uint32_t claim_tile(LaunchSync* s) {
    return atomicAdd(&s->ticket, 1u);
}
// Called once per CTA at exit by thread 0; the last CTA of the launch resets
// the ticket and advances the epoch.
__device__ __forceinline__ void finish_tile(LaunchSync* s, uint32_t ntiles) {
    __threadfence();
    uint32_t d = atomicAdd(&s->done, 1u);
    if (d == ntiles - 1) {
        s->ticket = 0;
        s->done = 0;
        __threadfence();
        atomicAdd(&s->epoch, 1u);
    }
}

template <typename T>
__device__ __forceinline__ T shfl_up(T v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }

// Bounded wait for tile `t`'s record of the current epoch.  Returns the
// state (REC_AGG / REC_INCL) and the payload, or 0 after SPIN_LIMIT polls.
__device__ __forceinline__ uint32_t wait_record(const TileRec* recs, uint32_t t, uint32_t epoch,
                                                uint4& out) {
    uint32_t ns = 8;
    for (uint32_t it = 0; it < SPIN_LIMIT; ++it) {
        const uint32_t f = ld_cg(&recs[t].flag);
        if ((f >> 2) == (epoch & 0x3FFFFFFFu) && (f & 3u)) {
            const uint32_t st = f & 3u;
            out = ld_cg4(st == REC_INCL ? &recs[t].incl : &recs[t].agg);
            return st;
        }
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
    }
    return 0;
}

// Warp-wide decoupled look-back (whole warp, any lane order of calls).
// Reads the records of up to 32 predecessors of tile t per round trip, stops
// at the nearest one holding an inclusive prefix, and combines the window in
// tile order with `comb(earlier, later)`.  Returns the exclusive prefix of
// tile t in every lane; *ok turns false in every lane when any wait gave up.
template <class Comb>
__device__ __forceinline__ uint4 warp_lookback(const TileRec* recs, uint32_t t, uint32_t epoch,
                                               uint4 identity, Comb comb, bool* ok) {
    const uint32_t lane = threadIdx.x & 31u;
    uint4 acc = identity;  // combination of the tiles already visited (later ones)
    int64_t hi = t;        // tiles [0, hi) not yet visited
    bool mine_ok = true;
    while (hi > 0) {
        const int64_t p = hi - 1 - lane;
        uint4 v = identity;
        uint32_t st = REC_INCL;  // lanes past tile 0 act as an inclusive identity
        if (p >= 0) {
            st = wait_record(recs, (uint32_t)p, epoch, v);
            if (st == 0) { mine_ok = false; st = REC_INCL; v = identity; }
        }
        const uint32_t incl = __ballot_sync(0xffffffffu, st == REC_INCL);
        const uint32_t L = __ffs(incl) - 1u;  // nearest inclusive record in the window
        if (lane > L) v = identity;
        // ordered tree: lane l ends up with lanes [l, ...] combined, higher
        // lanes being earlier tiles
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint4 o;
            o.x = __shfl_down_sync(0xffffffffu, v.x, d);
            o.y = __shfl_down_sync(0xffffffffu, v.y, d);
            o.z = __shfl_down_sync(0xffffffffu, v.z, d);
            o.w = __shfl_down_sync(0xffffffffu, v.w, d);
            if (lane + d < 32u) v = comb(o, v);
        }
        uint4 win;
        win.x = __shfl_sync(0xffffffffu, v.x, 0);
        win.y = __shfl_sync(0xffffffffu, v.y, 0);
        win.z = __shfl_sync(0xffffffffu, v.z, 0);
        win.w = __shfl_sync(0xffffffffu, v.w, 0);
        acc = comb(win, acc);
        if (incl) break;
        hi -= 32;
    }
    // warp-uniform: false in every lane when any lane's wait gave up
    *ok = __all_sync(0xffffffffu, mine_ok);
    return acc;
}

// Block-wide exclusive scan of 64-bit values; returns the block total.
// (blockDim.x threads, a multiple of 32; sh holds blockDim.x/32 + 1 values)
__device__ __forceinline__ uint64_t block_exscan64(uint64_t v, uint64_t* sh, uint64_t& total) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint64_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint64_t t = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= (uint32_t)d) x += t;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t s = 0;
        const uint32_t nw = blockDim.x / 32;
        for (uint32_t w = 0; w < nw; ++w) { uint64_t t = sh[w]; sh[w] = s; s += t; }
        sh[nw] = s;
    }
    __syncthreads();
    total = sh[blockDim.x / 32];
    return sh[warp] + x - v;
}

// 64-bit sums packed in uint4 {lo, hi, sum32, or32}
struct Sum64Comb {
    __device__ __forceinline__ uint4 operator()(uint4 a, uint4 b) const {
        const uint64_t s = ((uint64_t)a.y << 32 | a.x) + ((uint64_t)b.y << 32 | b.x);
        return make_uint4((uint32_t)s, (uint32_t)(s >> 32), a.z + b.z, a.w | b.w);
    }
};

// Warp 0 only: publishes this tile's totals, looks back, publishes the
// inclusive prefix; returns the exclusive prefix.
__device__ __forceinline__ bool lookback64(TileRec* recs, uint32_t t, uint32_t epoch,
                                           uint64_t tot, uint32_t aux, uint32_t aux2,
                                           uint64_t& prefix, uint32_t& paux, uint32_t& paux2) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint4 mine = make_uint4((uint32_t)tot, (uint32_t)(tot >> 32), aux, aux2);
    uint4 pre = make_uint4(0, 0, 0, 0);
    bool ok = true;
    if (t == 0) {
        if (lane == 0) publish(&recs[0], epoch, REC_INCL, mine);
    } else {
        if (lane == 0) publish(&recs[t], epoch, REC_AGG, mine);
        pre = warp_lookback(recs, t, epoch, make_uint4(0, 0, 0, 0), Sum64Comb(), &ok);
        if (lane == 0) publish(&recs[t], epoch, REC_INCL, Sum64Comb()(pre, mine));
    }
    prefix = (uint64_t)pre.y << 32 | pre.x;
    paux = pre.z;
    paux2 = pre.w;
    return ok;
}

// ---- mbarriers and bulk copies (sm_90+ PTX), shared memory addressed by
// its 32-bit shared-window offset
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(b)), "r"(count) : "memory");
}
// makes barrier initialisation visible to the bulk-copy (async) proxy
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(b)), "r"(bytes) : "memory");
}
// non-blocking: has the phase of parity `par` completed?
__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t par) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_u32(b)), "r"(par) : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
constexpr uint64_t WAIT_LIMIT_NS = 2000000000ull;  // 2 s without progress: give up
// Bounded wait for phase `par` of barrier b; false after WAIT_LIMIT_NS.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t par) {
    if (mbar_test(b, par)) return true;
    const uint64_t t0 = gtimer();
    uint32_t ns = 32;
    while (!mbar_test(b, par)) {
        __nanosleep(ns);
        if (ns < 512) ns <<= 1;
        if (gtimer() - t0 > WAIT_LIMIT_NS) return false;
    }
    return true;
}
// Bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned)
// from global memory into this CTA's shared memory, completing on barrier b.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* b) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(b)) : "memory");
}
// Named barrier over the first `nthreads` threads of the CTA (id 1).
__device__ __forceinline__ void bar_sync1(uint32_t nthreads) {
    asm volatile("bar.sync 1, %0;" :: "r"(nthreads) : "memory");
}

}  // namespace wah
#endif
