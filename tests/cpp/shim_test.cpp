// Drives include/wahgpu.hpp the way FastBit code would use ibis::bitvector,
// relic/bin and countQuery.  Reads cases from argv[1], writes results to
// argv[2] (binary, little endian); tests/test_gpu_cpp_shim.py checks them.
#include <cuda_runtime.h>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>
#include "wahgpu.hpp"

using namespace wahgpu_ibis;

static uint32_t rd(std::ifstream& f) { uint32_t v; f.read(reinterpret_cast<char*>(&v), 4); return v; }
static std::vector<uint32_t> rdv(std::ifstream& f) {
    std::vector<uint32_t> v(rd(f));
    if (!v.empty()) f.read(reinterpret_cast<char*>(v.data()), v.size() * 4);
    return v;
}
static void wr(std::ofstream& f, uint64_t v) { f.write(reinterpret_cast<const char*>(&v), 8); }
static void wrv(std::ofstream& f, const std::vector<uint32_t>& v) {
    wr(f, v.size());
    f.write(reinterpret_cast<const char*>(v.data()), v.size() * 4);
}

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    std::ifstream in(argv[1], std::ios::binary);
    std::ofstream out(argv[2], std::ios::binary);
    context& ctx = context::standard();
    // 1. operators: a OP b and a OP= b, words and cnt()
    const uint32_t nbin = rd(in);
    for (uint32_t i = 0; i < nbin; ++i) {
        const uint32_t op = rd(in), inplace = rd(in);
        bitvector a(rdv(in)), b(rdv(in));
        std::vector<uint32_t> w;
        uint64_t c;
        if (inplace) {
            bitvector r(a);
            if (op == 0) r &= b; else if (op == 1) r |= b; else if (op == 2) r ^= b; else r -= b;
            r.write(w);
            c = r.cnt();
        } else {
            bitvector* r = op == 0 ? (a & b) : op == 1 ? (a | b) : op == 2 ? (a ^ b) : (a - b);
            r->write(w);
            c = r->cnt();
            delete r;
        }
        wrv(out, w);
        wr(out, c);
    }
    // 2. construction: setBit in row order, then appendFill to the size
    const uint32_t nset = rd(in);
    for (uint32_t i = 0; i < nset; ++i) {
        const uint32_t nbits = rd(in);
        std::vector<uint32_t> rows = rdv(in);
        bitvector b;
        b.set(0, 0);
        for (uint32_t r : rows) b.setBit(r, 1);
        if (b.size() < nbits) b.appendFill(0, (uint32_t)(nbits - b.size()));
        std::vector<uint32_t> w;
        b.write(w);
        wrv(out, w);
        wrv(out, b.rows());
        // adjustSize: 45 more 0 bits; count(mask) of the vector with itself
        b.adjustSize(0, nbits + 45);
        b.write(w);
        wrv(out, w);
        wr(out, b.count(b));
    }
    // 3. countQuery over two device-built indexes
    const uint32_t n = rd(in);
    std::vector<uint32_t> ca = rdv(in), cb = rdv(in);  // column b holds float32 bits
    void *da = nullptr, *db = nullptr;
    cudaMalloc(&da, (size_t)n * 4);
    cudaMalloc(&db, (size_t)n * 4);
    cudaMemcpy(da, ca.data(), (size_t)n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(db, cb.data(), (size_t)n * 4, cudaMemcpyHostToDevice);
    {
        relic ra(WAHGPU_U32, da, n);
        bin rb(WAHGPU_F32, db, n, 64);
        countQuery q;
        q.addColumn("a", ra);
        q.addColumn("b", rb);
        const uint32_t nq = rd(in);
        for (uint32_t i = 0; i < nq; ++i) {
            std::vector<uint32_t> txt = rdv(in);
            std::string clause(txt.begin(), txt.end());
            const int rc = q.setWhereClause(clause.c_str());
            wr(out, (uint64_t)(int64_t)rc);
            if (rc == 0) {
                q.evaluate();
                std::vector<uint32_t> rows;
                q.getHitRows(rows);
                wr(out, (uint64_t)q.getNumHits());
                wrv(out, rows);
            }
        }
        // relic::evaluate / estimate with a qContinuousRange
        bitvector hits;
        const long c = ra.evaluate(qContinuousRange(10, qContinuousRange::OP_LE, 20, qContinuousRange::OP_LT), hits);
        wr(out, (uint64_t)c);
        wr(out, ra.estimate(qContinuousRange(10, qContinuousRange::OP_LE, 20, qContinuousRange::OP_LT)));
        wrv(out, hits.rows());
        // bin::estimate(expr, lower, upper) and estimate(expr)
        const qContinuousRange eb(-0.5, qContinuousRange::OP_LE, 0.25, qContinuousRange::OP_LT);
        bitvector lower, upper;
        rb.estimate(eb, lower, upper);
        wrv(out, lower.rows());
        wr(out, upper.size());
        wrv(out, upper.rows());
        wr(out, rb.estimate(eb));
    }
    cudaFree(da);
    cudaFree(db);
    // 4. a relic read from its .idx file (argv[3]), and a bin file (argv[4])
    //    refused as a relic
    if (argc > 4) {
        relic rf(argv[3]);
        bitvector hits;
        const long c = rf.evaluate(qContinuousRange(10, qContinuousRange::OP_LE, 30, qContinuousRange::OP_LT), hits);
        wr(out, (uint64_t)c);
        wrv(out, hits.rows());
        int refused = 0;
        try {
            relic wrong(argv[4]);
        } catch (const error& e) {
            refused = e.code() == WAHGPU_EFORMAT ? 1 : 2;
        }
        wr(out, (uint64_t)refused);
    }
    // 5. a bitvector from an array-like of serialized words, setBit inside
    //    the vector (set then clear), a shrinking adjustSize, and the
    //    indexSet walk of the result
    {
        struct words {  // shaped like FastBit's array_t<uint32_t>
            std::vector<uint32_t> v;
            const uint32_t* begin() const { return v.data(); }
            size_t size() const { return v.size(); }
        } arr{rdv(in)};
        const uint32_t set_at = rd(in), clear_at = rd(in), keep = rd(in);
        bitvector b(arr);
        b.setBit(set_at, 1);
        b.setBit(clear_at, 0);
        wrv(out, b.rows());
        b.adjustSize(0, keep);
        wr(out, b.size());
        std::vector<uint32_t> pos;
        for (bitvector::indexSet is = b.firstIndexSet(); is.nIndices() > 0; ++is) {
            const uint32_t* ii = is.indices();
            if (is.isRange()) for (uint32_t j = ii[0]; j < ii[1]; ++j) pos.push_back(j);
            else for (uint32_t j = 0; j < is.nIndices(); ++j) pos.push_back(ii[j]);
        }
        wrv(out, pos);
    }
    return 0;
}
