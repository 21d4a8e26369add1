/*
 * wahgpu.hpp — C++ classes over the C ABI of libwahgpu (include/wahgpu.h),
 * shaped like the reference's interfaces so that code written against them
 * changes little:
 *
 *   wahgpu_ibis::bitvector    ibis::bitvector   (src/bitvector.h:62-318)
 *   wahgpu_ibis::qContinuousRange                (src/qExpr.h:259-280)
 *   wahgpu_ibis::relic / bin  ibis::relic / ibis::bin evaluate / estimate
 *                             (src/irelic.h, src/ibin.h; index.h:168-196)
 *   wahgpu_ibis::countQuery   ibis::countQuery (src/countQuery.h:25+):
 *                             setWhereClause, evaluate, getNumHits,
 *                             getHitRows
 *
 * Defining WAHGPU_AS_IBIS before including this header makes `ibis` an
 * alias of wahgpu_ibis (for code that does not also include FastBit).
 * Errors are thrown as wahgpu_ibis::error (code + text); the C ABI below
 * never throws.  Everything runs on the GPU; bitvectors live in device
 * memory and operands are never modified by binary operators.
 */
#ifndef WAHGPU_HPP
#define WAHGPU_HPP
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "wahgpu.h"

namespace wahgpu_ibis {

class error : public std::runtime_error {
public:
    error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

/* The device and stream everything below runs on (one per process by
 * default; several contexts may be used from different threads). */
class context {
public:
    explicit context(int device = 0) {
        if (int rc = wahgpu_ctx_create(device, &h_)) throw error(rc, wahgpu_last_error(nullptr));
    }
    ~context() { if (h_) wahgpu_ctx_destroy(h_); }
    context(const context&) = delete;
    context& operator=(const context&) = delete;
    wahgpu_ctx* get() const { return h_; }
    int64_t check(int64_t rc) const {
        if (rc < 0) throw error((int)rc, wahgpu_last_error(h_));
        return rc;
    }
    static context& standard() {
        static context c(0);
        return c;
    }

private:
    wahgpu_ctx* h_ = nullptr;
};

/* ibis::bitvector: 32-bit WAH words, 31 bits per group, active word. */
class bitvector {
public:
    typedef uint32_t word_t;
    class indexSet;

    explicit bitvector(context& c = context::standard()) : ctx_(&c) { set(0, 0); }
    /* bitvector(const array_t<word_t>&): a serialized array (words, then the
     * active value if it holds bits, then the active bit count). */
    bitvector(const std::vector<word_t>& serialized, context& c = context::standard()) : ctx_(&c) {
        upload(serialized.data(), serialized.size());
    }
    bitvector(const word_t* serialized, size_t n, context& c = context::standard()) : ctx_(&c) { upload(serialized, n); }
    /* bitvector(const array_t<word_t>&) (src/bitvector.cpp:54): any
     * contiguous array of serialized words with begin() and size() (FastBit's
     * array_t, ...).  The reference shares the array's storage
     * (array_t.h:104-107); here the words are copied to the device once, so
     * the array may be released or changed afterwards. */
    template <class Array, class = decltype(static_cast<const word_t*>(&*std::declval<const Array&>().begin())),
              class = decltype(std::declval<const Array&>().size()),
              class = typename std::enable_if<!std::is_same<Array, std::vector<word_t>>::value>::type>
    explicit bitvector(const Array& arr, context& c = context::standard()) : ctx_(&c) {
        upload(arr.size() ? &*arr.begin() : nullptr, arr.size());
    }
    bitvector(const bitvector& o) : ctx_(o.ctx_) {
        std::vector<word_t> w;
        o.write(w);
        upload(w.data(), w.size());
    }
    bitvector& operator=(const bitvector& o) {
        if (this != &o) {
            std::vector<word_t> w;
            o.write(w);
            release();
            ctx_ = o.ctx_;
            upload(w.data(), w.size());
        }
        return *this;
    }
    bitvector(bitvector&& o) noexcept : ctx_(o.ctx_), h_(o.h_) { o.h_ = nullptr; }
    bitvector& operator=(bitvector&& o) noexcept {
        std::swap(ctx_, o.ctx_);
        std::swap(h_, o.h_);
        return *this;
    }
    ~bitvector() { release(); }

    /* set(val, n): n bits all equal to val (src/bitvector.h:256). */
    void set(int val, uint32_t n) {
        std::vector<word_t> w;
        const uint32_t G = n / 31, anb = n % 31;
        if (G >= 2) w.push_back((val ? 0xC0000000u : 0x80000000u) | G);
        else if (G == 1) w.push_back(val ? 0x7FFFFFFFu : 0u);
        if (anb) w.push_back(val ? ((1u << anb) - 1u) : 0u);
        w.push_back(anb);
        release();
        upload(w.data(), w.size());
    }
    /* appendFill(val, n) (src/bitvector.h:800) and setBit(i, val) for i at
     * or past the end (src/bitvector.cpp:621, append case): the bits are
     * appended on the host and the vector is uploaded again, so these are
     * construction-time operations. */
    void appendFill(int val, uint32_t n) {
        std::vector<word_t> w;
        write(w);
        host_append(w, val, n);
        release();
        upload(w.data(), w.size());
    }
    /* adjustSize(nv, nt) (src/bitvector.cpp:4086-4108): growing, bits up to
     * position nv become 1 and the rest up to nt 0, through appendFill as in
     * the reference; shrinking keeps the first nt bits (erase(nt, size()),
     * src/bitvector.cpp:1012-1036: the whole words before bit nt, then the
     * covering word's leading part appended).  Construction-time, on the
     * host. */
    void adjustSize(uint32_t nv, uint32_t nt) {
        const uint64_t sz = size();
        if (nt == sz) return;
        if (nt < sz) {
            std::vector<word_t> w;
            write(w);
            truncate(w, nt);
            release();
            upload(w.data(), w.size());
            return;
        }
        if (nv > nt) nv = nt;
        if (nv > sz) {
            appendFill(1, (uint32_t)(nv - sz));
            if (nt > nv) appendFill(0, nt - nv);
        } else {
            appendFill(0, (uint32_t)(nt - sz));
        }
    }
    /* count(mask) (src/bitvector.h:1089-1124): the 1 bits of *this & mask. */
    uint64_t count(const bitvector& mask) const {
        std::unique_ptr<bitvector> r(*this & mask);
        return r->cnt();
    }
    /* setBit(i, val) (src/bitvector.cpp:621).  Past the end the bits are
     * appended on the host; inside the vector the bit is OR'ed in (val 1)
     * or cleared with - (val 0) on the device, with a one-bit operand of the
     * same size.  The bits equal the reference's; the words are in
     * compress() form. */
    void setBit(uint32_t i, int val) {
        const uint64_t n = size();
        if (i < n) {
            std::vector<word_t> w{0u};
            host_append(w, 0, i);
            host_append(w, 1, 1);
            host_append(w, 0, (uint32_t)(n - i - 1));
            bitvector one(w, *ctx_);
            if (val) *this |= one; else *this -= one;
            return;
        }
        std::vector<word_t> w;
        write(w);
        host_append(w, 0, (uint32_t)(i - n));
        host_append(w, val, 1);
        release();
        upload(w.data(), w.size());
    }

    uint64_t size() const { return (uint64_t)ctx_->check(wahgpu_bv_size(h_)); }
    uint64_t cnt() const { return (uint64_t)ctx_->check(wahgpu_bv_cnt(h_)); }
    void compress() { ctx_->check(wahgpu_bv_compress(h_)); }
    void decompress() { ctx_->check(wahgpu_bv_decompress(h_)); }
    void flip() { ctx_->check(wahgpu_bv_flip(h_)); }
    /* write(array_t<word_t>&): the serialized words (src/bitvector.cpp:2283). */
    void write(std::vector<word_t>& out) const {
        out.resize((size_t)ctx_->check(wahgpu_bv_serial_size(h_)));
        ctx_->check(wahgpu_bv_write(h_, out.data(), out.size()));
    }
    /* The rows of the 1 bits, ascending (what an indexSet walk yields). */
    std::vector<uint32_t> rows() const {
        std::vector<uint32_t> r((size_t)cnt());
        ctx_->check(wahgpu_bv_rids(h_, r.data(), r.size()));
        return r;
    }

    bitvector& operator&=(const bitvector& b) { return inplace(WAHGPU_AND, b); }
    bitvector& operator|=(const bitvector& b) { return inplace(WAHGPU_OR, b); }
    bitvector& operator^=(const bitvector& b) { return inplace(WAHGPU_XOR, b); }
    bitvector& operator-=(const bitvector& b) { return inplace(WAHGPU_MINUS, b); }
    /* Like the reference, the binary operators return a new bitvector the
     * caller deletes (src/bitvector.cpp:1289). */
    bitvector* operator&(const bitvector& b) const { return binary(WAHGPU_AND, b); }
    bitvector* operator|(const bitvector& b) const { return binary(WAHGPU_OR, b); }
    bitvector* operator^(const bitvector& b) const { return binary(WAHGPU_XOR, b); }
    bitvector* operator-(const bitvector& b) const { return binary(WAHGPU_MINUS, b); }

    /* firstIndexSet() (src/bitvector.h:1253): the first set of 1-bit
     * positions, walking a host copy of the words (see indexSet). */
    inline indexSet firstIndexSet() const;

    wahgpu_bv* handle() const { return h_; }
    static bitvector adopt(wahgpu_bv* h, context& c) {
        bitvector b(c, h);
        return b;
    }
    /* The first nt bits of serialized words w (the leading part of
     * erase(nt, size()), src/bitvector.cpp:1012-1036). */
    static void truncate(std::vector<word_t>& w, uint32_t nt) {
        uint32_t anb = w.back(), aval = 0;
        w.pop_back();
        if (anb) { aval = w.back(); w.pop_back(); }
        std::vector<word_t> r{0u};
        uint64_t pos = 0;
        for (size_t k = 0; k < w.size() && pos < nt; ++k) {
            const word_t x = w[k];
            const uint64_t g = x > 0x7FFFFFFFu ? (x & 0x3FFFFFFFu) : 1u;
            if (pos + 31 * g <= nt) {          // a whole word, kept verbatim
                r.back() = x;
                r.push_back(0u);
                pos += 31 * g;
            } else if (x > 0x7FFFFFFFu) {      // the covering fill's leading part
                host_append(r, x >= 0xC0000000u ? 1 : 0, (uint32_t)(nt - pos));
                pos = nt;
            } else {                           // the covering literal's leading bits
                const uint32_t k2 = (uint32_t)(nt - pos);
                for (uint32_t b = 0; b < k2; ++b) host_append(r, (x >> (30u - b)) & 1u, 1);
                pos = nt;
            }
        }
        for (uint32_t b = 0; pos < nt && b < anb; ++b, ++pos) host_append(r, (aval >> (anb - 1u - b)) & 1u, 1);
        w.swap(r);
    }

private:
    bitvector(context& c, wahgpu_bv* h) : ctx_(&c), h_(h) {}
    void upload(const word_t* w, size_t n) { ctx_->check(wahgpu_bv_from_serial(ctx_->get(), w, n, &h_)); }
    void release() {
        if (h_) wahgpu_bv_free(h_);
        h_ = nullptr;
    }
    bitvector& inplace(int op, const bitvector& b) {
        wahgpu_bv* r = nullptr;
        ctx_->check(wahgpu_bv_binop(ctx_->get(), op, 1, h_, b.h_, &r));
        release();
        h_ = r;
        return *this;
    }
    bitvector* binary(int op, const bitvector& b) const {
        wahgpu_bv* r = nullptr;
        ctx_->check(wahgpu_bv_binop(ctx_->get(), op, 0, h_, b.h_, &r));
        return new bitvector(*ctx_, r);
    }
    /* Appends n bits of value v to serialized words w (compress() form:
     * maximal all-0/all-1 runs of 2+ groups as fills). */
    static void push_groups(std::vector<word_t>& w, uint32_t g, uint32_t k) {
        if (k == 0) return;
        const uint32_t fillv = g ? 0xC0000000u : 0x80000000u;
        if (!w.empty()) {
            uint32_t& last = w.back();
            if (last > 0x7FFFFFFFu && (last & 0xC0000000u) == fillv) { last += k; return; }
            if (last == g) { last = fillv | (k + 1u); return; }
        }
        w.push_back(k == 1 ? g : (fillv | k));
    }
    static void push_group(std::vector<word_t>& w, uint32_t g) {
        if (g == 0u || g == 0x7FFFFFFFu) push_groups(w, g, 1);
        else w.push_back(g);
    }
    static void host_append(std::vector<word_t>& w, int v, uint32_t n) {
        uint32_t anb = w.back(), aval = 0;
        w.pop_back();
        if (anb) { aval = w.back(); w.pop_back(); }
        const uint32_t bit = v ? 1u : 0u;
        while (n > 0 && anb > 0) {          // complete the active word
            aval = (aval << 1) | bit; ++anb; --n;
            if (anb == 31) { push_group(w, aval); aval = 0; anb = 0; }
        }
        if (n >= 31) {                       // whole groups
            push_groups(w, v ? 0x7FFFFFFFu : 0u, n / 31);
            n %= 31;
        }
        while (n > 0) { aval = (aval << 1) | bit; ++anb; --n; }
        if (anb) w.push_back(aval);
        w.push_back(anb);
    }

    context* ctx_;
    wahgpu_bv* h_ = nullptr;
};

/* ibis::bitvector::indexSet (src/bitvector.h:421-522; operator++,
 * src/bitvector.cpp:4524-4590): the 1-bit positions one WAH word at a time.
 * For a 1-fill (or an all-ones literal) isRange() is true and indices()
 * holds [first, past-the-end); otherwise indices() holds the nIndices()
 * positions of the word's 1 bits; 0-fills and zero literals are skipped and
 * the active word comes last.  nIndices() == 0 marks the end.  The walk runs
 * over a host copy of the serialized words taken by firstIndexSet();
 * bitvector::rows() gives all positions at once from the GPU. */
class bitvector::indexSet {
public:
    indexSet() {}
    /* Over serialized words w (the write(array_t&) layout). */
    explicit indexSet(std::shared_ptr<const std::vector<word_t>> w) : w_(std::move(w)) {
        const std::vector<word_t>& v = *w_;
        anb_ = v.empty() ? 0u : v.back();
        if (anb_ >= 31u) anb_ = 0u;
        aval_ = anb_ && v.size() >= 2 ? v[v.size() - 2] : 0u;
        end_ = v.empty() ? 0u : v.size() - (anb_ ? 2u : 1u);
        it_ = -1;
        ind_[0] = 0xFFFFFFFFu;
        nind_ = 0;
        ++*this;
    }
    bool isRange() const { return nind_ >= 31u; }
    const word_t* indices() const { return ind_; }
    word_t nIndices() const { return nind_; }
    indexSet& operator++() {
        const int64_t end = (int64_t)end_;
        if (it_ > end) { nind_ = 0; return *this; }
        word_t index0 = ((ind_[0] + (nind_ > 31u ? nind_ : 31u)) / 31u) * 31u;
        ++it_;
        nind_ = 0;
        const std::vector<word_t>& v = *w_;
        while (it_ < end) {
            const word_t x = v[(size_t)it_];
            if (x >= 0xC0000000u) {               // 1-fill
                nind_ = (x & 0x3FFFFFFFu) * 31u;
                ind_[1] = index0 + nind_;
                ind_[0] = index0;
                return *this;
            } else if (x >= 0x80000000u) {        // 0-fill
                index0 += (x & 0x3FFFFFFFu) * 31u;
                ++it_;
            } else if (x > 0) {                   // non-zero literal
                if (x < 0x7FFFFFFFu) {
                    word_t i = 0, j = x << 1;
                    for (; j > 0; ++i, j <<= 1)
                        if (j > 0x7FFFFFFFu) ind_[nind_++] = index0 + i;
                } else {
                    nind_ = 31u;
                    ind_[0] = index0;
                    ind_[1] = index0 + 31u;
                }
                return *this;
            } else {                              // zero literal
                index0 += 31u;
                ++it_;
            }
        }
        if (anb_ > 0 && aval_ > 0) {
            word_t i = 0, j = aval_ << (32u - anb_);
            for (; j > 0; ++i, j <<= 1)
                if (j > 0x7FFFFFFFu) ind_[nind_++] = index0 + i;
        }
        it_ = end + 1;
        return *this;
    }

private:
    std::shared_ptr<const std::vector<word_t>> w_;
    int64_t it_ = 0;
    size_t end_ = 0;
    word_t anb_ = 0, aval_ = 0;
    word_t nind_ = 0;
    word_t ind_[32] = {0};
};

inline bitvector::indexSet bitvector::firstIndexSet() const {
    auto w = std::make_shared<std::vector<word_t>>();
    write(*w);
    return indexSet(w);
}

/* ibis::qContinuousRange: lower lop x rop upper, compared in double. */
struct qContinuousRange {
    enum COMPARE { OP_UNDEFINED = 0, OP_LT = 1, OP_LE = 2 };
    double lower = 0, upper = 0;
    int lop = OP_UNDEFINED, rop = OP_UNDEFINED;
    qContinuousRange() {}
    qContinuousRange(double lo, COMPARE lo_op, double hi, COMPARE hi_op) : lower(lo), upper(hi), lop(lo_op), rop(hi_op) {}
};

/* The index classes: attached from the (keys, offsets, bitmaps) triple the
 * reference writes, or built on the device from a column in device memory. */
class index {
public:
    index(const index&) = delete;
    index& operator=(const index&) = delete;
    virtual ~index() { if (h_) wahgpu_index_free(h_); }
    wahgpu_index* handle() const { return h_; }
    uint32_t nrows() const { return (uint32_t)ctx_->check(wahgpu_index_nrows(h_)); }
    /* Raw values for the edge-bin row checks (host array of n values). */
    void setValues(int vtype, const void* values, uint64_t n) { ctx_->check(wahgpu_index_set_values(h_, vtype, values, n)); }
    /* evaluate(expr, hits) (src/index.h:168): the hit count, the hits in
     * compress() form. */
    long evaluate(const qContinuousRange& e, bitvector& hits) const {
        wahgpu_term t = term(e);
        wahgpu_bv* h = nullptr;
        const int64_t n = ctx_->check(wahgpu_evaluate(ctx_->get(), &t, 1, nullptr, 0, &h));
        hits = bitvector::adopt(h, *ctx_);
        return (long)n;
    }
    /* estimate(expr) (src/index.h:196): an upper bound of the hit count —
     * relic: exact; bin: the 1 bits of the bins wholly inside and of the
     * edge bins (src/ibin.cpp:6832-6889). */
    uint32_t estimate(const qContinuousRange& e) const {
        wahgpu_term t = term(e);
        return (uint32_t)ctx_->check(wahgpu_estimate_count(ctx_->get(), &t));
    }
    /* estimate(expr, lower, upper) (src/index.h:191): lower = rows certainly
     * hit, upper = a superset of the hits, empty when lower is exact (relic,
     * src/irelic.h:58-62; bin, src/ibin.cpp:6722-6829). */
    void estimate(const qContinuousRange& e, bitvector& lower, bitvector& upper) const {
        wahgpu_term t = term(e);
        wahgpu_bv* lo = nullptr;
        wahgpu_bv* up = nullptr;
        ctx_->check(wahgpu_estimate(ctx_->get(), &t, &lo, &up));
        lower = bitvector::adopt(lo, *ctx_);
        upper = bitvector::adopt(up, *ctx_);
    }
    wahgpu_term term(const qContinuousRange& e) const {
        wahgpu_term t;
        t.idx = h_; t.lop = e.lop; t.lo = e.lower; t.rop = e.rop; t.hi = e.upper;
        return t;
    }

protected:
    index(context& c, int kind, uint32_t nrows, const std::vector<double>& keys, const std::vector<int64_t>& offsets,
          const std::vector<uint32_t>& bms) : ctx_(&c) {
        ctx_->check(wahgpu_index_from_triple(ctx_->get(), kind, nrows, keys.data(), keys.size(), offsets.data(),
                                             offsets.size(), bms.data(), bms.size(), &h_));
    }
    index(context& c, int kind, int vtype, const void* dev_values, uint64_t nrows, uint32_t nbins) : ctx_(&c) {
        ctx_->check(wahgpu_index_build(ctx_->get(), kind, vtype, dev_values, nrows, nbins, &h_));
    }
    /* From a .idx file whose index type byte (header[5]) must be `type`. */
    index(context& c, const char* f, int type) : ctx_(&c) {
        char header[8] = {0};
        std::FILE* fp = f ? std::fopen(f, "rb") : nullptr;
        const bool ok = fp && std::fread(header, 1, 8, fp) == 8;
        if (fp) std::fclose(fp);
        if (!ok) throw error(WAHGPU_EINVAL, std::string("cannot read index file ") + (f ? f : "(null)"));
        if (header[5] != type) throw error(WAHGPU_EFORMAT, std::string("index file of another type: ") + f);
        ctx_->check(wahgpu_index_read(ctx_->get(), f, &h_));
    }
    context* ctx_;
    wahgpu_index* h_ = nullptr;
};

class relic : public index {
public:
    /* relic(nbits, keys, offsets, bms) from relic::write's triple. */
    relic(uint32_t nrows, const std::vector<double>& keys, const std::vector<int64_t>& offsets,
          const std::vector<uint32_t>& bms, context& c = context::standard())
        : index(c, WAHGPU_RELIC, nrows, keys, offsets, bms) {}
    /* relic::construct over a column in device memory. */
    relic(int vtype, const void* dev_values, uint64_t nrows, context& c = context::standard())
        : index(c, WAHGPU_RELIC, vtype, dev_values, nrows, 0) {}
    /* relic(col, f): the index file f written by relic::write
     * (src/irelic.cpp:354, read 690). */
    explicit relic(const char* f, context& c = context::standard()) : index(c, f, 7) {}
};

class bin : public index {
public:
    bin(uint32_t nrows, const std::vector<double>& keys, const std::vector<int64_t>& offsets,
        const std::vector<uint32_t>& bms, context& c = context::standard())
        : index(c, WAHGPU_BIN, nrows, keys, offsets, bms) {}
    /* <binning nbins=N equal_weight/> over a column in device memory. */
    bin(int vtype, const void* dev_values, uint64_t nrows, uint32_t nbins, context& c = context::standard())
        : index(c, WAHGPU_BIN, vtype, dev_values, nrows, nbins) {}
    /* bin(col, f): the index file f written by bin::write (src/ibin.cpp:5530,
     * read 468); the raw column for edge checks comes from setValues. */
    explicit bin(const char* f, context& c = context::standard()) : index(c, f, 0) {}
};

/* ibis::countQuery over named columns.  A WHERE clause combines range
 * conditions — "a >= 3", "2.5 <= b < 7", "c between 1 and 4", "d = 5",
 * "d != 5", "e in (1, 4, 9)" or "e in (1 4 9)" (a qDiscreteRange, as an OR of equalities) —
 * with AND, OR, NOT (also &&, ||, !) and parentheses, as
 * countQuery::doEvaluate does with its LOGICAL_AND / OR / NOT nodes over
 * qContinuousRange leaves (src/countQuery.cpp:929-1036): an AND of ranges
 * is one fused evaluation; other nodes combine the hit bitvectors of their
 * children with the bitvector operators (OR |=, NOT flip()), on the device. */
class countQuery {
public:
    explicit countQuery(context& c = context::standard()) : ctx_(&c) {}
    void addColumn(const std::string& name, const index& idx) { cols_[lower(name)] = &idx; }
    /* setWhereClause(const char*) (src/countQuery.cpp:81); 0 on success, a
     * negative code when the clause does not parse or names an unknown
     * column. */
    int setWhereClause(const char* clause) {
        nodes_.clear();
        terms_.clear();
        root_ = -1;
        hits_ = -1;
        rows_.clear();
        try {
            Lexer L{clause ? clause : "", std::string(), false, 0.0};
            while (L.next()) { toks_.push_back(L.tok); vals_.push_back(L.val); nums_.push_back(L.num); }
            pos_ = 0;
            root_ = parse_or();
            if (pos_ != toks_.size()) throw error(WAHGPU_EINVAL, "unexpected '" + toks_[pos_] + "'");
        } catch (const error& e) {
            nodes_.clear();
            root_ = -1;
            toks_.clear(); vals_.clear(); nums_.clear();
            return e.code();
        }
        toks_.clear(); vals_.clear(); nums_.clear();
        // a plain AND of ranges keeps the fused single-launch path
        if (!leaves_of_and(root_, terms_)) terms_.clear();
        return 0;
    }
    /* evaluate() (src/countQuery.cpp:292); getNumHits (376); getHitRows
     * (387-410). */
    int evaluate() {
        if (root_ < 0) return WAHGPU_EINVAL;
        if (!terms_.empty()) {
            // the count first, then the row ids into a buffer of that size
            const int64_t n = ctx_->check(wahgpu_evaluate(ctx_->get(), terms_.data(), (uint32_t)terms_.size(),
                                                          nullptr, 0, nullptr));
            rows_.resize((size_t)n);
            if (n) ctx_->check(wahgpu_evaluate(ctx_->get(), terms_.data(), (uint32_t)terms_.size(), rows_.data(),
                                               rows_.size(), nullptr));
            hits_ = n;
            return 0;
        }
        bitvector h = eval(root_);
        hits_ = (int64_t)h.cnt();
        rows_ = h.rows();
        return 0;
    }
    long getNumHits() const { return (long)hits_; }
    long getHitRows(std::vector<uint32_t>& rids) const {
        rids = rows_;
        return (long)rids.size();
    }
    /* The range terms of a clause that is an AND of ranges (else empty). */
    const std::vector<wahgpu_term>& terms() const { return terms_; }

private:
    enum Kind { LEAF, AND, OR, NOT };
    struct Node {
        Kind kind;
        wahgpu_term term;          // LEAF
        std::vector<int> kids;     // AND, OR: two or more; NOT: one
    };
    static std::string lower(std::string s) {
        for (char& ch : s) ch = (char)std::tolower((unsigned char)ch);
        return s;
    }
    struct Lexer {
        const char* p;
        std::string tok;
        bool num = false;
        double val = 0;
        bool next() {
            while (*p && std::isspace((unsigned char)*p)) ++p;
            tok.clear();
            num = false;
            if (!*p) return false;
            const char c = *p;
            if (std::isdigit((unsigned char)c) || c == '.' || ((c == '-' || c == '+') && (std::isdigit((unsigned char)p[1]) || p[1] == '.'))) {
                char* end = nullptr;
                val = std::strtod(p, &end);
                tok.assign(p, (size_t)(end - p));
                p = end;
                num = true;
            } else if (std::isalpha((unsigned char)c) || c == '_') {
                const char* s = p;
                while (*p && (std::isalnum((unsigned char)*p) || *p == '_' || *p == '.')) ++p;
                tok.assign(s, (size_t)(p - s));
            } else if (((c == '<' || c == '>' || c == '=' || c == '!') && p[1] == '=') ||
                       (c == '&' && p[1] == '&') || (c == '|' && p[1] == '|')) {
                tok.assign(p, 2);
                p += 2;
            } else {
                tok.assign(p, 1);
                ++p;
            }
            return true;
        }
    };
    const index* column(const std::string& name) const {
        auto it = cols_.find(lower(name));
        if (it == cols_.end()) throw error(WAHGPU_EINVAL, "unknown column " + name);
        return it->second;
    }
    int leaf(const index* idx, int lop, double lo, int rop, double hi) {
        Node n{LEAF, wahgpu_term(), {}};
        n.term.idx = idx->handle(); n.term.lop = lop; n.term.lo = lo; n.term.rop = rop; n.term.hi = hi;
        nodes_.push_back(n);
        return (int)nodes_.size() - 1;
    }
    int inner(Kind k, std::vector<int> kids) {
        nodes_.push_back(Node{k, wahgpu_term(), std::move(kids)});
        return (int)nodes_.size() - 1;
    }
    bool at(const char* w) const { return pos_ < toks_.size() && lower(toks_[pos_]) == w; }
    bool is_cmp(size_t k) const {
        return k < toks_.size() && (toks_[k] == "<" || toks_[k] == "<=" || toks_[k] == ">" || toks_[k] == ">=" ||
                                    toks_[k] == "=" || toks_[k] == "==" || toks_[k] == "!=");
    }
    int parse_or() {
        std::vector<int> kids{parse_and()};
        while (at("or") || at("||")) { ++pos_; kids.push_back(parse_and()); }
        return kids.size() == 1 ? kids[0] : inner(OR, kids);
    }
    int parse_and() {
        std::vector<int> kids{parse_unary()};
        while (at("and") || at("&&")) { ++pos_; kids.push_back(parse_unary()); }
        return kids.size() == 1 ? kids[0] : inner(AND, kids);
    }
    int parse_unary() {
        if (at("not") || at("!")) { ++pos_; return inner(NOT, {parse_unary()}); }
        if (at("(")) {
            ++pos_;
            const int e = parse_or();
            if (!at(")")) throw error(WAHGPU_EINVAL, "missing ')'");
            ++pos_;
            return e;
        }
        return parse_condition();
    }
    // name op num | num op name [op num] | name between a and b
    int parse_condition() {
        const size_t i = pos_;
        const auto& T = toks_;
        if (i >= T.size()) throw error(WAHGPU_EINVAL, "missing condition");
        if (!nums_[i] && i + 2 < T.size() && lower(T[i + 1]) == "in" && T[i + 2] == "(") {
            // x in (v1, v2, ...) or x in (v1 v2 ...): qDiscreteRange as an
            // OR of equalities
            const index* c = column(T[i]);
            std::vector<int> kids;
            size_t k = i + 3;
            while (true) {
                if (k >= T.size() || !nums_[k]) throw error(WAHGPU_EINVAL, "bad IN list");
                kids.push_back(leaf(c, WAHGPU_CMP_LE, vals_[k], WAHGPU_CMP_LE, vals_[k]));
                if (k + 1 < T.size() && T[k + 1] == ",") { k += 2; continue; }
                if (k + 1 < T.size() && nums_[k + 1]) { k += 1; continue; }
                if (k + 1 < T.size() && T[k + 1] == ")") break;
                throw error(WAHGPU_EINVAL, "bad IN list");
            }
            pos_ = k + 2;
            return kids.size() == 1 ? kids[0] : inner(OR, kids);
        }
        if (!nums_[i] && i + 1 < T.size() && lower(T[i + 1]) == "between") {
            if (i + 4 >= T.size() || !nums_[i + 2] || lower(T[i + 3]) != "and" || !nums_[i + 4])
                throw error(WAHGPU_EINVAL, "bad BETWEEN");
            pos_ = i + 5;
            return leaf(column(T[i]), WAHGPU_CMP_LE, vals_[i + 2], WAHGPU_CMP_LE, vals_[i + 4]);
        }
        if (!nums_[i] && is_cmp(i + 1) && i + 2 < T.size() && nums_[i + 2]) {
            const std::string& op = T[i + 1];
            const double v = vals_[i + 2];
            const index* c = column(T[i]);
            pos_ = i + 3;
            if (op == "<") return leaf(c, WAHGPU_CMP_NONE, 0, WAHGPU_CMP_LT, v);
            if (op == "<=") return leaf(c, WAHGPU_CMP_NONE, 0, WAHGPU_CMP_LE, v);
            if (op == ">") return leaf(c, WAHGPU_CMP_LT, v, WAHGPU_CMP_NONE, 0);
            if (op == ">=") return leaf(c, WAHGPU_CMP_LE, v, WAHGPU_CMP_NONE, 0);
            const int eq = leaf(c, WAHGPU_CMP_LE, v, WAHGPU_CMP_LE, v);
            return op == "!=" ? inner(NOT, {eq}) : eq;
        }
        if (nums_[i] && is_cmp(i + 1) && T[i + 1] != "!=" && i + 2 < T.size() && !nums_[i + 2]) {
            const std::string& op = T[i + 1];
            const double v = vals_[i];
            const index* c = column(T[i + 2]);
            int lop = WAHGPU_CMP_LE, rop = WAHGPU_CMP_NONE;
            double hi = 0;
            if (op == "<") lop = WAHGPU_CMP_LT;
            else if (op == "<=") lop = WAHGPU_CMP_LE;
            else if (op == ">") { lop = WAHGPU_CMP_NONE; rop = WAHGPU_CMP_LT; hi = v; }
            else if (op == ">=") { lop = WAHGPU_CMP_NONE; rop = WAHGPU_CMP_LE; hi = v; }
            else { rop = WAHGPU_CMP_LE; hi = v; }
            pos_ = i + 3;
            if ((op == "<" || op == "<=") && pos_ + 1 < T.size() && nums_[pos_ + 1] &&
                (T[pos_] == "<" || T[pos_] == "<=")) {
                rop = T[pos_] == "<" ? WAHGPU_CMP_LT : WAHGPU_CMP_LE;
                hi = vals_[pos_ + 1];
                pos_ += 2;
            }
            return leaf(c, lop, lop == WAHGPU_CMP_NONE ? 0 : v, rop, hi);
        }
        throw error(WAHGPU_EINVAL, "not a range condition near '" + T[i] + "'");
    }
    // the terms of a node that is a leaf or an AND of leaves
    bool leaves_of_and(int n, std::vector<wahgpu_term>& out) const {
        const Node& x = nodes_[(size_t)n];
        if (x.kind == LEAF) { out.push_back(x.term); return true; }
        if (x.kind != AND) return false;
        for (int k : x.kids)
            if (nodes_[(size_t)k].kind != LEAF) { out.clear(); return false; }
        for (int k : x.kids) out.push_back(nodes_[(size_t)k].term);
        return true;
    }
    bitvector eval_terms(const std::vector<wahgpu_term>& t) {
        wahgpu_bv* h = nullptr;
        ctx_->check(wahgpu_evaluate(ctx_->get(), t.data(), (uint32_t)t.size(), nullptr, 0, &h));
        return bitvector::adopt(h, *ctx_);
    }
    bitvector eval(int n) {
        const Node& x = nodes_[(size_t)n];
        if (x.kind == LEAF) return eval_terms({x.term});
        if (x.kind == NOT) {
            bitvector h = eval(x.kids[0]);
            h.flip();
            return h;
        }
        if (x.kind == AND) {
            // the range leaves of the AND in one fused evaluation
            std::vector<wahgpu_term> t;
            for (int k : x.kids)
                if (nodes_[(size_t)k].kind == LEAF) t.push_back(nodes_[(size_t)k].term);
            std::vector<bitvector> parts;
            if (!t.empty()) parts.push_back(eval_terms(t));
            for (int k : x.kids)
                if (nodes_[(size_t)k].kind != LEAF) parts.push_back(eval(k));
            bitvector acc = std::move(parts[0]);
            for (size_t k = 1; k < parts.size(); ++k) acc &= parts[k];
            return acc;
        }
        bitvector acc = eval(x.kids[0]);
        for (size_t k = 1; k < x.kids.size(); ++k) acc |= eval(x.kids[k]);
        return acc;
    }

    context* ctx_;
    std::map<std::string, const index*> cols_;
    std::vector<Node> nodes_;
    int root_ = -1;
    std::vector<std::string> toks_;
    std::vector<double> vals_;
    std::vector<bool> nums_;
    size_t pos_ = 0;
    std::vector<wahgpu_term> terms_;
    std::vector<uint32_t> rows_;
    int64_t hits_ = -1;
};

}  // namespace wahgpu_ibis

#ifdef WAHGPU_AS_IBIS
namespace ibis = wahgpu_ibis;
#endif
#endif
