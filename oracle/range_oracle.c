/*
 * CPU oracle for range evaluation — TEST INFRASTRUCTURE ONLY.
 *
 * The reference evaluates `lo <= x < hi` on a column through its relic / bin
 * index (src/irelic.cpp:1827 relic::evaluate, src/ibin.cpp:6614
 * bin::evaluate, then column::evaluateRange src/column.cpp:6029 and
 * part::doScan for the candidate rows); the hit set it returns is exactly the
 * rows whose value satisfies the comparison carried out in double
 * (qContinuousRange::inRange, src/qExpr.cpp:1647-1667).  The scans below
 * restate that hit set directly; tests compare the GPU's hit counts and row
 * ids with them, and with the reference's own answers in tests/golden/.
 */
#include <stdint.h>
#include <stddef.h>

/* rows i with lo <= (double)x[i] < hi; returns the count, writes up to cap ids */
long ro_range_u32(const uint32_t *x, uint64_t n, double lo, double hi, uint32_t *out, uint64_t cap) {
    uint64_t k = 0;
    for (uint64_t i = 0; i < n; ++i) {
        double v = (double)x[i];
        if (lo <= v && v < hi) { if (k < cap) out[k] = (uint32_t)i; ++k; }
    }
    return (long)k;
}

long ro_range_f32(const float *x, uint64_t n, double lo, double hi, uint32_t *out, uint64_t cap) {
    uint64_t k = 0;
    for (uint64_t i = 0; i < n; ++i) {
        double v = (double)x[i];
        if (lo <= v && v < hi) { if (k < cap) out[k] = (uint32_t)i; ++k; }
    }
    return (long)k;
}

/* Conjunction of up to 8 range terms over columns given as pointers with a
 * type tag each (0 = uint32, 1 = float32): count and row ids. */
long ro_conj(int nterms, const void *const *cols, const int *types, const double *lo,
             const double *hi, uint64_t n, uint32_t *out, uint64_t cap) {
    uint64_t k = 0;
    for (uint64_t i = 0; i < n; ++i) {
        int ok = 1;
        for (int t = 0; t < nterms && ok; ++t) {
            double v = types[t] ? (double)((const float *)cols[t])[i] : (double)((const uint32_t *)cols[t])[i];
            ok = (lo[t] <= v && v < hi[t]);
        }
        if (ok) { if (k < cap) out[k] = (uint32_t)i; ++k; }
    }
    return (long)k;
}

/* Counts only, many queries at once over one uint32 column, parallel over
 * queries (the CPU baseline's throughput leg). */
void ro_count_many_u32(const uint32_t *x, uint64_t n, const double *lo, const double *hi,
                       long nq, uint64_t *counts) {
#pragma omp parallel for schedule(dynamic, 1)
    for (long q = 0; q < nq; ++q) {
        uint64_t k = 0;
        const double a = lo[q], b = hi[q];
        for (uint64_t i = 0; i < n; ++i) { double v = (double)x[i]; k += (a <= v && v < b); }
        counts[q] = k;
    }
}
