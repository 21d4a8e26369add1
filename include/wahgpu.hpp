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

    explicit bitvector(context& c = context::standard()) : ctx_(&c) { set(0, 0); }
    /* bitvector(const array_t<word_t>&): a serialized array (words, then the
     * active value if it holds bits, then the active bit count). */
    bitvector(const std::vector<word_t>& serialized, context& c = context::standard()) : ctx_(&c) {
        upload(serialized.data(), serialized.size());
    }
    bitvector(const word_t* serialized, size_t n, context& c = context::standard()) : ctx_(&c) { upload(serialized, n); }
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
    void setBit(uint32_t i, int val) {
        const uint64_t n = size();
        if (i < n) throw error(WAHGPU_EINVAL, "setBit inside the vector is not supported; append in row order");
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

    wahgpu_bv* handle() const { return h_; }
    static bitvector adopt(wahgpu_bv* h, context& c) {
        bitvector b(c, h);
        return b;
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
    /* estimate(expr) (src/index.h:196) — here exact. */
    uint32_t estimate(const qContinuousRange& e) const {
        wahgpu_term t = term(e);
        return (uint32_t)ctx_->check(wahgpu_evaluate(ctx_->get(), &t, 1, nullptr, 0, nullptr));
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

/* ibis::countQuery over named columns: a WHERE clause that is an AND of
 * range conditions — "a >= 3 and a < 10", "2.5 <= b < 7", "c between 1
 * and 4", "d = 5" — (the qContinuousRange leaves of countQuery::evaluate,
 * src/countQuery.cpp:953-1036). */
class countQuery {
public:
    explicit countQuery(context& c = context::standard()) : ctx_(&c) {}
    void addColumn(const std::string& name, const index& idx) { cols_[lower(name)] = &idx; }
    /* setWhereClause(const char*) (src/countQuery.cpp:81); 0 on success, a
     * negative code when the clause is not an AND of ranges on known
     * columns. */
    int setWhereClause(const char* clause) {
        terms_.clear();
        hits_ = -1;
        rows_.clear();
        try {
            parse(clause ? clause : "");
        } catch (const error& e) {
            terms_.clear();
            return e.code();
        }
        return terms_.empty() ? WAHGPU_EINVAL : 0;
    }
    /* evaluate() (src/countQuery.cpp:292); getNumHits (376); getHitRows
     * (387-410). */
    int evaluate() {
        if (terms_.empty()) return WAHGPU_EINVAL;
        // the count first, then the row ids into a buffer of that size
        const int64_t n = ctx_->check(wahgpu_evaluate(ctx_->get(), terms_.data(), (uint32_t)terms_.size(),
                                                      nullptr, 0, nullptr));
        rows_.resize((size_t)n);
        if (n) ctx_->check(wahgpu_evaluate(ctx_->get(), terms_.data(), (uint32_t)terms_.size(), rows_.data(),
                                           rows_.size(), nullptr));
        hits_ = n;
        return 0;
    }
    long getNumHits() const { return (long)hits_; }
    long getHitRows(std::vector<uint32_t>& rids) const {
        rids = rows_;
        return (long)rids.size();
    }
    const std::vector<wahgpu_term>& terms() const { return terms_; }

private:
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
            } else if ((c == '<' || c == '>' || c == '=' || c == '!') && p[1] == '=') {
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
    void add(const index* idx, int lop, double lo, int rop, double hi) {
        wahgpu_term t;
        t.idx = idx->handle(); t.lop = lop; t.lo = lo; t.rop = rop; t.hi = hi;
        terms_.push_back(t);
    }
    // one condition: name op num | num op name [op num] | name between a and b
    void parse(const char* s) {
        Lexer L{s, std::string(), false, 0.0};
        std::vector<std::string> toks;
        std::vector<double> vals;
        std::vector<bool> nums;
        while (L.next()) { toks.push_back(L.tok); vals.push_back(L.val); nums.push_back(L.num); }
        size_t i = 0;
        auto is_cmp = [&](size_t k) {
            return k < toks.size() && (toks[k] == "<" || toks[k] == "<=" || toks[k] == ">" || toks[k] == ">=" ||
                                       toks[k] == "=" || toks[k] == "==");
        };
        while (i < toks.size()) {
            if (!nums[i] && i + 1 < toks.size() && lower(toks[i + 1]) == "between") {
                if (i + 4 >= toks.size() || !nums[i + 2] || lower(toks[i + 3]) != "and" || !nums[i + 4])
                    throw error(WAHGPU_EINVAL, "bad BETWEEN");
                add(column(toks[i]), WAHGPU_CMP_LE, vals[i + 2], WAHGPU_CMP_LE, vals[i + 4]);
                i += 5;
            } else if (!nums[i] && is_cmp(i + 1) && i + 2 < toks.size() && nums[i + 2]) {
                const std::string& op = toks[i + 1];
                const double v = vals[i + 2];
                const index* c = column(toks[i]);
                if (op == "<") add(c, WAHGPU_CMP_NONE, 0, WAHGPU_CMP_LT, v);
                else if (op == "<=") add(c, WAHGPU_CMP_NONE, 0, WAHGPU_CMP_LE, v);
                else if (op == ">") add(c, WAHGPU_CMP_LT, v, WAHGPU_CMP_NONE, 0);
                else if (op == ">=") add(c, WAHGPU_CMP_LE, v, WAHGPU_CMP_NONE, 0);
                else add(c, WAHGPU_CMP_LE, v, WAHGPU_CMP_LE, v);
                i += 3;
            } else if (nums[i] && is_cmp(i + 1) && i + 2 < toks.size() && !nums[i + 2]) {
                const std::string& op = toks[i + 1];
                const double v = vals[i];
                const index* c = column(toks[i + 2]);
                int lop = WAHGPU_CMP_LE, rop = WAHGPU_CMP_NONE;
                double hi = 0;
                if (op == "<") lop = WAHGPU_CMP_LT;
                else if (op == "<=") lop = WAHGPU_CMP_LE;
                else if (op == ">") { lop = WAHGPU_CMP_NONE; rop = WAHGPU_CMP_LT; hi = v; }
                else if (op == ">=") { lop = WAHGPU_CMP_NONE; rop = WAHGPU_CMP_LE; hi = v; }
                else { rop = WAHGPU_CMP_LE; hi = v; }
                i += 3;
                if ((op == "<" || op == "<=") && is_cmp(i) && i + 1 < toks.size() && nums[i + 1] &&
                    (toks[i] == "<" || toks[i] == "<=")) {
                    rop = toks[i] == "<" ? WAHGPU_CMP_LT : WAHGPU_CMP_LE;
                    hi = vals[i + 1];
                    i += 2;
                }
                add(c, lop, lop == WAHGPU_CMP_NONE ? 0 : v, rop, hi);
            } else {
                throw error(WAHGPU_EINVAL, "not a range condition near '" + toks[i] + "'");
            }
            if (i < toks.size()) {
                if (lower(toks[i]) != "and") throw error(WAHGPU_EINVAL, "only AND of ranges is supported");
                ++i;
            }
        }
    }

    context* ctx_;
    std::map<std::string, const index*> cols_;
    std::vector<wahgpu_term> terms_;
    std::vector<uint32_t> rows_;
    int64_t hits_ = -1;
};

}  // namespace wahgpu_ibis

#ifdef WAHGPU_AS_IBIS
namespace ibis = wahgpu_ibis;
#endif
#endif
