// Oracle driver — TEST INFRASTRUCTURE ONLY.
//
// Runs the reference FastBit library (built from source by
// oracle/Makefile.ref into oracle/_ref/) on requests read from a binary file
// and writes the reference's answers to another binary file.  It is used to
// make the golden fixtures under tests/golden/ and to pin the C restatement
// in oracle/wah_oracle.c against the reference itself.
//
// Request stream (all little-endian uint32 unless stated):
//   1 op inplace compress na a[na] nb b[nb]   -> ibis::bitvector a OP b
//        (operator& | ^ - , bitvector.cpp:1292-1838, or the OP= forms),
//        operands built with the array_t constructor (bitvector.cpp:54);
//        reply: status cnt len words[len]   (serialized result, write(array_t&))
//   2 na a[na]                                -> compress(); reply like 1
//   3 na a[na]                                -> firstIndexSet walk (rids);
//        reply: status n rids[n]
//   4 nruns(u64) runs[nruns](u64)             -> appendFill-built bitvector
//        (alternating 0/1 runs, 0 first); reply like 1
//   5 nrows vals[nrows] nq (lo hi)(f64 x2)[nq] -> ibis::relic over the uint32
//        column (construct(array_t), irelic.cpp:879) + evaluate of
//        qContinuousRange(lo <= x < hi) (irelic.cpp:1827) for each query;
//        reply: nkeys keys(f64)[nkeys] noffs offs(i64)[noffs] nbms bms[nbms]
//               then per query: status count nrids rids[nrids]
//   6 na a[na] -> decompress(); reply like 1
//   7 na a[na] -> flip(); reply like 1
//   9 nrows vals(f32)[nrows] nbins nq (lo hi)(f64 x2)[nq] -> ibis::bin index
//        through the in-memory C API: fastbit_iapi_register_array +
//        fastbit_iapi_build_index("<binning nbins=N equal_weight/>") +
//        fastbit_iapi_deconstruct_index (src/iapi.cpp:1644, 1893, 1915), then
//        per query osr(x >= lo) AND osr(x < hi), evaluate and
//        get_coordinates (src/iapi.cpp:2062, 1285, 1383, 1517);
//        reply: the triple like 5, then per query: status count nrids rids
//  10 kind plen path[plen] nrows vals[nrows] nbins -> writes the index file
//        the reference's own writer produces: kind 1 ibis::relic over the
//        uint32 column (construct(array_t), irelic.cpp:879; write(".idx"),
//        irelic.cpp:354-642), kind 2 ibis::bin over the column as float32
//        through fastbit_iapi_build_index("<binning nbins=N equal_weight/>")
//        and its triple (bin ctor, ibin.cpp:358; write, ibin.cpp:5530-5834);
//        reply: status (0 ok)
//  11 nruns_a(u64) runs_a[nruns_a](u64) nruns_b(u64) runs_b[nruns_b](u64)
//        -> two appendFill-built bitvectors (alternating 0/1 runs, 0 first,
//        bitvector.h:800) and, for op & | ^ - in both forms (a OP b, then
//        a OP= b on a private copy of a), the compress()ed result;
//        reply: len a[len], len b[len], then 8 x (status cnt len words[len])
//  12 nthreads reps flags ncols, per column: vtype(1 uint32, 2 int32,
//        3 float32) nrows vals[nrows](4 B) nkeys(u64) keys(f64) noffs(u64)
//        offs(i64) nbms(u64) bms(u32); then nq, per query: nterms, per term:
//        col lo(f64) hi(f64) for lo <= x < hi
//        -> the in-memory C API on indexes given as triples: every column
//        registered (fastbit_iapi_register_array, src/iapi.cpp:1644) with
//        its triple attached (fastbit_iapi_attach_full_index, 2018); a query
//        is osr(x >= lo) AND osr(x < hi) per term, AND across terms
//        (fastbit_selection_osr / combine, 2062, 1285), evaluated
//        (fastbit_selection_evaluate, 1383) and, with flags bit 0, its row
//        ids read (fastbit_selection_get_coordinates, 1517); each selection
//        is freed after use, so no cached answer is reused.  One untimed
//        pass on one thread gives the answers; then `reps` timed passes on
//        nthreads threads (queries round robin).
//        reply: status seconds(f64, timed passes, max over threads), then
//        per query: count(u64) seconds(f64, the untimed one-thread pass)
//        [nrids rids[nrids] with row ids]
//  13 nthreads reps nrows vals[nrows] nq (lo hi)(f64 x2)[nq] -> times
//        ibis::relic over the uint32 column (construct(array_t),
//        irelic.cpp:879): per query evaluate(qContinuousRange(lo <= x < hi),
//        hits) (irelic.cpp:1827) and the firstIndexSet row-id walk
//        (bitvector.h:421-542).  One untimed pass on one thread warms the
//        lazily counted members; then `reps` timed passes on nthreads threads
//        (queries round robin, each thread its own hit vectors).
//        reply: seconds(f64, max over threads), then per query count(u64)
//   8 nthreads reps nops (op na a[na] nb b[nb])[nops] -> times the reference's
//        operators: each of nthreads threads builds its own operand copies,
//        then runs its share of the ops (round robin) reps times, each as
//        r = a OP b; r->compress(); r->cnt().  reply: seconds(f64) for the
//        timed part (max over threads, after a barrier), then per op the
//        serialized result length in words
#include "ibis.h"
#include "irelic.h"
#include "iapi.h"
#include "ibin.h"
#include "bitvector.h"
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <stdint.h>
#include <pthread.h>
#include <time.h>

static FILE *fin, *fout;

// ibis::bin rebuilt from a triple; the index keeps its row count in a
// protected member, which the ctor from a triple leaves 0 without a column
struct BinFromTriple : public ibis::bin {
    BinFromTriple(uint32_t nb, double* keys, int64_t* offs, uint32_t* bms, uint32_t rows)
        : ibis::bin(0, nb, keys, offs, bms) { nrows = rows; }
};
static uint32_t rd32() { uint32_t v; if (fread(&v, 4, 1, fin) != 1) exit(3); return v; }
static uint64_t rd64() { uint64_t v; if (fread(&v, 8, 1, fin) != 1) exit(3); return v; }
static double rdf64() { double v; if (fread(&v, 8, 1, fin) != 1) exit(3); return v; }
static void wr32(uint32_t v) { fwrite(&v, 4, 1, fout); }
static void wrv(const std::vector<uint32_t>& v) { wr32((uint32_t)v.size()); if (!v.empty()) fwrite(&v[0], 4, v.size(), fout); }
static std::vector<uint32_t> rdvec() {
    uint32_t n = rd32(); std::vector<uint32_t> v(n);
    if (n && fread(&v[0], 4, n, fin) != n) exit(3);
    return v;
}
static ibis::bitvector* from_serial(const std::vector<uint32_t>& w) {
    ibis::array_t<uint32_t> arr(w.size());
    for (size_t i = 0; i < w.size(); ++i) arr[i] = w[i];
    return new ibis::bitvector(arr);
}
static void reply_bv(int status, ibis::bitvector* r) {
    wr32((uint32_t)status);
    if (status != 0 || r == 0) { wr32(0); wr32(0); return; }
    // serialize first: cnt() may collapse an all-zero m_vec (do_cnt)
    ibis::array_t<uint32_t> out;
    r->write(out);
    uint32_t cnt = r->cnt();
    wr32(cnt);
    std::vector<uint32_t> v(out.begin(), out.end());
    wrv(v);
}
static void rids_of(const ibis::bitvector& bv, std::vector<uint32_t>& rids) {
    for (ibis::bitvector::indexSet is = bv.firstIndexSet(); is.nIndices() > 0; ++is) {
        const ibis::bitvector::word_t* ii = is.indices();
        if (is.isRange()) { for (uint32_t j = ii[0]; j < ii[1]; ++j) rids.push_back(j); }
        else { for (uint32_t j = 0; j < is.nIndices(); ++j) rids.push_back(ii[j]); }
    }
}

struct TimeJob {
    std::vector<int> ops;
    std::vector<ibis::bitvector*> a, b;
    int reps;
    pthread_barrier_t* bar;
    double secs;
    std::vector<uint32_t> lens;
};
static double now_s() { struct timespec t; clock_gettime(CLOCK_MONOTONIC, &t); return t.tv_sec + 1e-9 * t.tv_nsec; }
static void* time_thread(void* p) {
    TimeJob* j = (TimeJob*)p;
    j->lens.assign(j->ops.size(), 0);
    // warm the lazily counted members of the operands once, outside the timing
    for (size_t k = 0; k < j->ops.size(); ++k) { j->a[k]->size(); j->b[k]->size(); j->a[k]->cnt(); j->b[k]->cnt(); }
    pthread_barrier_wait(j->bar);
    double t0 = now_s();
    for (int r = 0; r < j->reps; ++r) {
        for (size_t k = 0; k < j->ops.size(); ++k) {
            ibis::bitvector* R;
            switch (j->ops[k]) { case 0: R = *j->a[k] & *j->b[k]; break; case 1: R = *j->a[k] | *j->b[k]; break;
                                 case 2: R = *j->a[k] ^ *j->b[k]; break; default: R = *j->a[k] - *j->b[k]; }
            R->compress();
            (void)R->cnt();
            j->lens[k] = (uint32_t)(R->getSerialSize() / 4);
            delete R;
        }
    }
    j->secs = now_s() - t0;
    return 0;
}

// request 12: one query of the in-memory C API on the registered columns
struct Term12 { uint32_t col; double lo, hi; };
struct Job12 {
    const std::vector<std::vector<Term12> >* qs;
    uint32_t tid, nth, reps, rids;
    pthread_barrier_t* bar;
    double secs;
};
static int64_t eval12(const std::vector<Term12>& q, uint32_t rids, std::vector<uint32_t>* out) {
    FastBitSelectionHandle h = 0;
    for (size_t k = 0; k < q.size(); ++k) {
        char nm[16];
        snprintf(nm, sizeof nm, "c%u", q[k].col);
        FastBitSelectionHandle a = fastbit_selection_osr(nm, FastBitCompareGreaterEqual, q[k].lo);
        FastBitSelectionHandle b = fastbit_selection_osr(nm, FastBitCompareLess, q[k].hi);
        FastBitSelectionHandle t = fastbit_selection_combine(a, FastBitCombineAnd, b);
        h = h ? fastbit_selection_combine(h, FastBitCombineAnd, t) : t;
    }
    int64_t cnt = fastbit_selection_evaluate(h);
    if (cnt > 0 && rids) {
        std::vector<uint64_t> co(cnt);
        const int64_t got = fastbit_selection_get_coordinates(h, &co[0], cnt, 0);
        if (out) for (int64_t i = 0; i < got; ++i) out->push_back((uint32_t)co[i]);
    }
    fastbit_selection_free(h);
    return cnt;
}
static void* job12(void* p) {
    Job12* j = (Job12*)p;
    pthread_barrier_wait(j->bar);
    const double t0 = now_s();
    for (uint32_t r = 0; r < j->reps; ++r)
        for (size_t q = j->tid; q < j->qs->size(); q += j->nth) eval12((*j->qs)[q], j->rids, 0);
    j->secs = now_s() - t0;
    return 0;
}

// request 13: relic::evaluate and the row-id walk per query
struct Job13 {
    const ibis::relic* rel;
    const std::vector<double>* lo;
    const std::vector<double>* hi;
    uint32_t tid, nth, reps;
    pthread_barrier_t* bar;
    double secs;
    uint64_t sink;
};
static uint64_t eval13(const ibis::relic& rel, double lo, double hi, std::vector<uint32_t>& rids) {
    ibis::qContinuousRange expr(lo, ibis::qExpr::OP_LE, "x", ibis::qExpr::OP_LT, hi);
    ibis::bitvector hits;
    const long c = rel.evaluate(expr, hits);
    rids.clear();
    rids_of(hits, rids);
    return c < 0 ? 0 : (uint64_t)c;
}
static void* job13(void* p) {
    Job13* j = (Job13*)p;
    std::vector<uint32_t> rids;
    pthread_barrier_wait(j->bar);
    const double t0 = now_s();
    for (uint32_t r = 0; r < j->reps; ++r)
        for (size_t q = j->tid; q < j->lo->size(); q += j->nth) j->sink += eval13(*j->rel, (*j->lo)[q], (*j->hi)[q], rids);
    j->secs = now_s() - t0;
    return 0;
}

int main(int argc, char** argv) {
    if (argc != 3) { fprintf(stderr, "usage: refdrv in out\n"); return 2; }
    ibis::init();
    fin = fopen(argv[1], "rb"); fout = fopen(argv[2], "wb");
    if (!fin || !fout) return 2;
    uint32_t kind;
    while (fread(&kind, 4, 1, fin) == 1) {
        if (kind == 1) {
            uint32_t op = rd32(), inplace = rd32(), comp = rd32();
            std::vector<uint32_t> a = rdvec(), b = rdvec();
            ibis::bitvector *A = from_serial(a), *B = from_serial(b), *R = 0;
            int st = 0;
            try {
                if (inplace) {
                    switch (op) { case 0: *A &= *B; break; case 1: *A |= *B; break;
                                  case 2: *A ^= *B; break; default: *A -= *B; }
                    R = A; A = 0;
                } else {
                    switch (op) { case 0: R = *A & *B; break; case 1: R = *A | *B; break;
                                  case 2: R = *A ^ *B; break; default: R = *A - *B; }
                }
                if (comp) R->compress();
            } catch (...) { st = 1; }
            reply_bv(st, R);
            delete A; delete B; delete R;
        } else if (kind == 2 || kind == 6 || kind == 7) {
            std::vector<uint32_t> a = rdvec();
            ibis::bitvector* A = from_serial(a);
            if (kind == 2) A->compress(); else if (kind == 6) A->decompress(); else A->flip();
            reply_bv(0, A);
            delete A;
        } else if (kind == 3) {
            std::vector<uint32_t> a = rdvec();
            ibis::bitvector* A = from_serial(a);
            std::vector<uint32_t> rids;
            rids_of(*A, rids);
            wr32(0); wrv(rids);
            delete A;
        } else if (kind == 4) {
            uint64_t n = rd64();
            ibis::bitvector A;
            for (uint64_t i = 0; i < n; ++i) A.appendFill((int)(i & 1), (uint32_t)rd64());
            reply_bv(0, &A);
        } else if (kind == 5) {
            uint32_t nrows = rd32();
            ibis::array_t<uint32_t> vals(nrows);
            for (uint32_t i = 0; i < nrows; ++i) vals[i] = rd32();
            ibis::relic rel(0);
            rel.construct(vals);
            ibis::array_t<double> keys; ibis::array_t<int64_t> offs; ibis::array_t<uint32_t> bms;
            rel.write(keys, offs, bms);
            wr32((uint32_t)keys.size()); fwrite(keys.begin(), 8, keys.size(), fout);
            wr32((uint32_t)offs.size()); fwrite(offs.begin(), 8, offs.size(), fout);
            wr32((uint32_t)bms.size()); fwrite(bms.begin(), 4, bms.size(), fout);
            uint32_t nq = rd32();
            for (uint32_t q = 0; q < nq; ++q) {
                double lo = rdf64(), hi = rdf64();
                ibis::qContinuousRange expr(lo, ibis::qExpr::OP_LE, "x", ibis::qExpr::OP_LT, hi);
                ibis::bitvector hits;
                long c = rel.evaluate(expr, hits);
                hits.compress();
                std::vector<uint32_t> rids;
                rids_of(hits, rids);
                wr32(c < 0 ? 1u : 0u); wr32((uint32_t)c); wrv(rids);
            }
        } else if (kind == 8) {
            uint32_t nth = rd32(), reps = rd32(), nops = rd32();
            std::vector<uint32_t> ops(nops);
            std::vector<std::vector<uint32_t> > A(nops), B(nops);
            for (uint32_t k = 0; k < nops; ++k) { ops[k] = rd32(); A[k] = rdvec(); B[k] = rdvec(); }
            std::vector<TimeJob> jobs(nth);
            std::vector<pthread_t> th(nth);
            pthread_barrier_t bar;
            pthread_barrier_init(&bar, 0, nth);
            std::vector<uint32_t> lens(nops, 0);
            for (uint32_t t = 0; t < nth; ++t) {
                jobs[t].reps = reps; jobs[t].bar = &bar;
                for (uint32_t k = t; k < nops; k += nth) {
                    jobs[t].ops.push_back((int)ops[k]);
                    jobs[t].a.push_back(from_serial(A[k]));
                    jobs[t].b.push_back(from_serial(B[k]));
                }
            }
            for (uint32_t t = 0; t < nth; ++t) pthread_create(&th[t], 0, time_thread, &jobs[t]);
            double mx = 0;
            for (uint32_t t = 0; t < nth; ++t) { pthread_join(th[t], 0); if (jobs[t].secs > mx) mx = jobs[t].secs; }
            for (uint32_t t = 0; t < nth; ++t) {
                for (size_t q = 0; q < jobs[t].ops.size(); ++q) {
                    lens[t + q * nth] = jobs[t].lens[q];
                    delete jobs[t].a[q]; delete jobs[t].b[q];
                }
            }
            pthread_barrier_destroy(&bar);
            fwrite(&mx, 8, 1, fout);
            for (uint32_t k = 0; k < nops; ++k) wr32(lens[k]);
        } else if (kind == 9) {
            uint32_t nrows = rd32();
            std::vector<float> vals(nrows);
            if (nrows && fread(&vals[0], 4, nrows, fin) != nrows) exit(3);
            uint32_t nbins = rd32();
            fastbit_iapi_register_array("x", FastBitDataTypeFloat, &vals[0], nrows);
            char spec[128];
            snprintf(spec, sizeof spec, "<binning nbins=%u equal_weight/>", nbins);
            int ierr = fastbit_iapi_build_index("x", spec);
            double* keys = 0; int64_t* offs = 0; uint32_t* bms = 0;
            uint64_t nk = 0, no = 0, nb = 0;
            if (ierr >= 0) ierr = fastbit_iapi_deconstruct_index("x", &keys, &nk, &offs, &no, &bms, &nb);
            if (ierr < 0) { nk = no = nb = 0; }
            wr32((uint32_t)nk); if (nk) fwrite(keys, 8, nk, fout);
            wr32((uint32_t)no); if (no) fwrite(offs, 8, no, fout);
            wr32((uint32_t)nb); if (nb) fwrite(bms, 4, nb, fout);
            uint32_t nq = rd32();
            for (uint32_t q = 0; q < nq; ++q) {
                double lo = rdf64(), hi = rdf64();
                FastBitSelectionHandle a = fastbit_selection_osr("x", FastBitCompareGreaterEqual, lo);
                FastBitSelectionHandle b = fastbit_selection_osr("x", FastBitCompareLess, hi);
                FastBitSelectionHandle c = fastbit_selection_combine(a, FastBitCombineAnd, b);
                int64_t cnt = fastbit_selection_evaluate(c);
                std::vector<uint32_t> rids;
                if (cnt > 0) {
                    std::vector<uint64_t> co(cnt);
                    int64_t got = fastbit_selection_get_coordinates(c, &co[0], cnt, 0);
                    for (int64_t i = 0; i < got; ++i) rids.push_back((uint32_t)co[i]);
                }
                wr32(cnt < 0 ? 1u : 0u); wr32((uint32_t)(cnt < 0 ? 0 : cnt)); wrv(rids);
                fastbit_selection_free(c);
            }
            delete [] keys; delete [] offs; delete [] bms;
            fastbit_iapi_free_all();
        } else if (kind == 11) {
            ibis::bitvector A, B;
            for (int k = 0; k < 2; ++k) {
                ibis::bitvector& X = k ? B : A;
                const uint64_t n = rd64();
                for (uint64_t i = 0; i < n; ++i) X.appendFill((int)(i & 1), (uint32_t)rd64());
            }
            std::vector<uint32_t> wa, wb;
            for (int k = 0; k < 2; ++k) {
                ibis::array_t<uint32_t> w;
                (k ? B : A).write(w);
                std::vector<uint32_t>& v = k ? wb : wa;
                v.assign(w.begin(), w.end());
                wrv(v);
            }
            for (int op = 0; op < 4; ++op) {
                for (int inplace = 0; inplace < 2; ++inplace) {
                    ibis::bitvector* R = 0;
                    int st = 0;
                    try {
                        if (inplace) {
                            // a private copy of a (its own storage), then a OP= b
                            R = from_serial(wa);
                            switch (op) { case 0: *R &= B; break; case 1: *R |= B; break;
                                          case 2: *R ^= B; break; default: *R -= B; }
                        } else {
                            switch (op) { case 0: R = A & B; break; case 1: R = A | B; break;
                                          case 2: R = A ^ B; break; default: R = A - B; }
                        }
                        R->compress();
                    } catch (...) { st = 1; }
                    reply_bv(st, R);
                    delete R;
                }
            }
        } else if (kind == 12) {
            const uint32_t nth = rd32(), reps = rd32(), flags = rd32(), ncols = rd32();
            std::vector<std::vector<char> > vals(ncols);
            std::vector<std::vector<double> > keys(ncols);
            std::vector<std::vector<int64_t> > offs(ncols);
            std::vector<std::vector<uint32_t> > bms(ncols);
            int st = 0;
            for (uint32_t c = 0; c < ncols; ++c) {
                const uint32_t vt = rd32(), nrows = rd32();
                vals[c].resize((size_t)nrows * 4 + 4);
                if (nrows && fread(&vals[c][0], 4, nrows, fin) != nrows) exit(3);
                const uint64_t nk = rd64();
                keys[c].resize(nk ? nk : 1);
                if (nk && fread(&keys[c][0], 8, nk, fin) != nk) exit(3);
                const uint64_t no = rd64();
                offs[c].resize(no ? no : 1);
                if (no && fread(&offs[c][0], 8, no, fin) != no) exit(3);
                const uint64_t nb = rd64();
                bms[c].resize(nb ? nb : 1);
                if (nb && fread(&bms[c][0], 4, nb, fin) != nb) exit(3);
                char nm[16];
                snprintf(nm, sizeof nm, "c%u", c);
                const FastBitDataType dt = vt == 1 ? FastBitDataTypeUInt : vt == 2 ? FastBitDataTypeInt : FastBitDataTypeFloat;
                if (fastbit_iapi_register_array(nm, dt, &vals[c][0], nrows) < 0) st = 1;
                else if (fastbit_iapi_attach_full_index(nm, &keys[c][0], nk, &offs[c][0], no, &bms[c][0], nb) < 0) st = 2;
            }
            const uint32_t nq = rd32();
            std::vector<std::vector<Term12> > qs(nq);
            for (uint32_t q = 0; q < nq; ++q) {
                const uint32_t nt = rd32();
                for (uint32_t k = 0; k < nt; ++k) {
                    Term12 t;
                    t.col = rd32(); t.lo = rdf64(); t.hi = rdf64();
                    qs[q].push_back(t);
                }
            }
            const uint32_t rids = flags & 1u;
            std::vector<uint64_t> counts(nq, 0);
            std::vector<double> lat(nq, 0.0);
            std::vector<std::vector<uint32_t> > ids(nq);
            for (uint32_t q = 0; q < nq && st == 0; ++q) {
                const double t0 = now_s();
                const int64_t c = eval12(qs[q], rids, &ids[q]);
                lat[q] = now_s() - t0;
                if (c < 0) st = 3;
                counts[q] = c < 0 ? 0 : (uint64_t)c;
            }
            double mx = 0;
            if (st == 0 && reps > 0 && nth > 0) {
                std::vector<Job12> jobs(nth);
                std::vector<pthread_t> th(nth);
                pthread_barrier_t bar;
                pthread_barrier_init(&bar, 0, nth);
                for (uint32_t t = 0; t < nth; ++t) {
                    jobs[t].qs = &qs; jobs[t].tid = t; jobs[t].nth = nth; jobs[t].reps = reps;
                    jobs[t].rids = rids; jobs[t].bar = &bar; jobs[t].secs = 0;
                    pthread_create(&th[t], 0, job12, &jobs[t]);
                }
                for (uint32_t t = 0; t < nth; ++t) { pthread_join(th[t], 0); if (jobs[t].secs > mx) mx = jobs[t].secs; }
                pthread_barrier_destroy(&bar);
            }
            wr32((uint32_t)st);
            fwrite(&mx, 8, 1, fout);
            for (uint32_t q = 0; q < nq; ++q) {
                fwrite(&counts[q], 8, 1, fout);
                fwrite(&lat[q], 8, 1, fout);
                if (rids) wrv(ids[q]);
            }
            fastbit_iapi_free_all();
        } else if (kind == 13) {
            const uint32_t nth = rd32(), reps = rd32(), nrows = rd32();
            ibis::array_t<uint32_t> vals(nrows);
            for (uint32_t i = 0; i < nrows; ++i) vals[i] = rd32();
            const uint32_t nq = rd32();
            std::vector<double> lo(nq), hi(nq);
            for (uint32_t q = 0; q < nq; ++q) { lo[q] = rdf64(); hi[q] = rdf64(); }
            ibis::relic rel(0);
            rel.construct(vals);
            std::vector<uint64_t> counts(nq);
            std::vector<uint32_t> rids;
            for (uint32_t q = 0; q < nq; ++q) counts[q] = eval13(rel, lo[q], hi[q], rids);
            double mx = 0;
            if (nth > 0 && reps > 0) {
                std::vector<Job13> jobs(nth);
                std::vector<pthread_t> th(nth);
                pthread_barrier_t bar;
                pthread_barrier_init(&bar, 0, nth);
                for (uint32_t t = 0; t < nth; ++t) {
                    jobs[t].rel = &rel; jobs[t].lo = &lo; jobs[t].hi = &hi; jobs[t].tid = t; jobs[t].nth = nth;
                    jobs[t].reps = reps; jobs[t].bar = &bar; jobs[t].secs = 0; jobs[t].sink = 0;
                    pthread_create(&th[t], 0, job13, &jobs[t]);
                }
                for (uint32_t t = 0; t < nth; ++t) { pthread_join(th[t], 0); if (jobs[t].secs > mx) mx = jobs[t].secs; }
                pthread_barrier_destroy(&bar);
            }
            fwrite(&mx, 8, 1, fout);
            for (uint32_t q = 0; q < nq; ++q) fwrite(&counts[q], 8, 1, fout);
        } else if (kind == 10) {
            const uint32_t ik = rd32(), plen = rd32();
            std::vector<char> path(plen + 1, 0);
            if (plen && fread(&path[0], 1, plen, fin) != plen) exit(3);
            const uint32_t nrows = rd32();
            std::vector<uint32_t> raw(nrows);
            for (uint32_t i = 0; i < nrows; ++i) raw[i] = rd32();
            const uint32_t nbins = rd32();
            int ierr = -1;
            if (ik == 1) {
                ibis::array_t<uint32_t> vals(nrows);
                for (uint32_t i = 0; i < nrows; ++i) vals[i] = raw[i];
                ibis::relic rel(0);
                rel.construct(vals);
                ierr = rel.write(&path[0]);
            } else if (ik == 2) {
                std::vector<float> vals(nrows);
                for (uint32_t i = 0; i < nrows; ++i) memcpy(&vals[i], &raw[i], 4);
                fastbit_iapi_register_array("x", FastBitDataTypeFloat, &vals[0], nrows);
                char spec[128];
                snprintf(spec, sizeof spec, "<binning nbins=%u equal_weight/>", nbins);
                ierr = fastbit_iapi_build_index("x", spec);
                double* keys = 0; int64_t* offs = 0; uint32_t* bms = 0;
                uint64_t nk = 0, no = 0, nb = 0;
                if (ierr >= 0) ierr = fastbit_iapi_deconstruct_index("x", &keys, &nk, &offs, &no, &bms, &nb);
                if (ierr >= 0) {
                    BinFromTriple b((uint32_t)(no - 1), keys, offs, bms, nrows);
                    ierr = b.write(&path[0]);
                }
                delete [] keys; delete [] offs; delete [] bms;
                fastbit_iapi_free_all();
            }
            wr32(ierr < 0 ? 1u : 0u);
        } else if (kind == 14) {
            // relic::construct over uint32 values, then per query
            // relic::evaluate of  lo lop x rop hi  (0: no bound, 1: <, 2: <=)
            // (src/irelic.cpp:879, 1827; qContinuousRange src/qExpr.h:259-280):
            // the count and the row ids
            const uint32_t nrows = rd32();
            ibis::array_t<uint32_t> vals(nrows);
            for (uint32_t i = 0; i < nrows; ++i) vals[i] = rd32();
            ibis::relic rel(0);
            rel.construct(vals);
            const ibis::qExpr::COMPARE cmp[3] = {ibis::qExpr::OP_UNDEFINED, ibis::qExpr::OP_LT, ibis::qExpr::OP_LE};
            const uint32_t nq = rd32();
            for (uint32_t q = 0; q < nq; ++q) {
                const double lo = rdf64(), hi = rdf64();
                const uint32_t lop = rd32(), rop = rd32();
                if (lop > 2 || rop > 2) exit(3);
                ibis::qContinuousRange expr(lo, cmp[lop], "x", cmp[rop], hi);
                ibis::bitvector hits;
                const long c = rel.evaluate(expr, hits);
                std::vector<uint32_t> rids;
                if (c > 0) rids_of(hits, rids);
                wr32(c < 0 ? 1u : 0u); wr32(c < 0 ? 0u : (uint32_t)c); wrv(rids);
            }
        } else {
            fprintf(stderr, "refdrv: unknown request %u\n", kind);
            return 4;
        }
    }
    fclose(fout);
    return 0;
}
