// FastBit index files (.idx) read into device-resident indexes, host side.
//
// The file layouts are the ones the reference's writers produce and its
// readers accept:
//   header (8 bytes): "#IBIS", index type (ibis::index::INDEX_TYPE, src/
//   index.h:86: BINNING = 0, RELIC = 7), offset size 4 or 8, then 0
//   (relic::write src/irelic.cpp:354-457, bin::write src/ibin.cpp:5530-5654).
//   relic (relic::write32/64 src/irelic.cpp:459-642, read 690-786):
//     u32 nrows, u32 nobs, u32 card; at 8*ceil((8+12)/8) = 24 the card
//     keys (double); then nobs+1 bitmap offsets (int32 or int64, absolute
//     byte positions); then the bitmaps.
//   bin (bin::write32/64 src/ibin.cpp:5656-5834, read 468-540):
//     u32 nrows, u32 nobs; at 16 the nobs+1 offsets; at the next multiple
//     of 8 bounds, maxval and minval (nobs doubles each); then the bitmaps.
// A bitmap is the serialized bitvector (m_vec, then active.val when
// active.nbits > 0, then active.nbits; bitvector::write(int) src/
// bitvector.cpp:2179-2225); a bitmap the writer skipped (no bitvector) has
// zero bytes and holds no row; it stays zero words long in the triple.
//
// The triple handed to wahgpu_index_from_triple: relic keys = the values;
// bin keys = minval then maxval (the layout of the bin constructor from a
// triple, src/ibin.cpp:358-373); offsets in words from the first bitmap.
#include "../../include/wahgpu.h"
#include "wah_api_internal.h"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {

constexpr int IDX_BINNING = 0;
constexpr int IDX_RELIC = 7;

struct Triple {
    int kind = 0;
    uint64_t nrows = 0;
    std::vector<double> keys;
    std::vector<int64_t> offsets;
    std::vector<uint32_t> bitmaps;
};

template <class T>
bool get(const unsigned char* p, uint64_t bytes, uint64_t pos, T& v) {
    if (pos > bytes || bytes - pos < sizeof(T)) return false;
    std::memcpy(&v, p + pos, sizeof(T));
    return true;
}

// Fills t from a file image; returns 0 or a message describing the defect.
const char* parse(const void* data, uint64_t bytes, Triple& t) {
    const unsigned char* p = static_cast<const unsigned char*>(data);
    if (!p || bytes < 16) return "shorter than an index header";
    if (std::memcmp(p, "#IBIS", 5) != 0 || p[7] != 0 || (p[6] != 4 && p[6] != 8))
        return "not a FastBit index file (bad header)";
    const int type = p[5];
    const uint64_t osz = p[6];
    uint32_t nrows = 0, nobs = 0;
    get(p, bytes, 8, nrows);
    get(p, bytes, 12, nobs);
    uint64_t offpos, first;
    std::vector<double> a, b;  // relic: values; bin: minval, maxval
    if (type == IDX_RELIC) {
        uint32_t card = 0;
        if (!get(p, bytes, 16, card)) return "truncated relic header";
        if (card != nobs) return "relic file with a key count unlike its bitmap count";
        const uint64_t valpos = 24;
        offpos = valpos + 8ull * nobs;
        first = offpos + osz * (nobs + 1ull);
        if (first > bytes) return "truncated relic keys or offsets";
        a.resize(nobs);
        if (nobs) std::memcpy(a.data(), p + valpos, 8ull * nobs);
        t.kind = WAHGPU_RELIC;
    } else if (type == IDX_BINNING) {
        offpos = 16;
        const uint64_t dblpos = 8 * ((offpos + osz * (nobs + 1ull) + 7) / 8);
        first = dblpos + 24ull * nobs;
        if (first > bytes) return "truncated bin offsets or bounds";
        a.resize(nobs);
        b.resize(nobs);
        // bounds at dblpos, maxval at dblpos + 8*nobs, minval after it
        if (nobs) {
            std::memcpy(b.data(), p + dblpos + 8ull * nobs, 8ull * nobs);
            std::memcpy(a.data(), p + dblpos + 16ull * nobs, 8ull * nobs);
        }
        t.kind = WAHGPU_BIN;
    } else {
        return "index type is neither relic (7) nor bin (0)";
    }
    if (nobs == 0) return "index without bitmaps";
    std::vector<uint64_t> off(nobs + 1ull);
    for (uint64_t i = 0; i <= nobs; ++i) {
        if (osz == 4) {
            int32_t v = 0;
            if (!get(p, bytes, offpos + 4 * i, v)) return "truncated bitmap offsets";
            if (v < 0) return "negative bitmap offset";
            off[i] = (uint64_t)v;
        } else {
            int64_t v = 0;
            if (!get(p, bytes, offpos + 8 * i, v)) return "truncated bitmap offsets";
            if (v < 0) return "negative bitmap offset";
            off[i] = (uint64_t)v;
        }
    }
    if (off[0] != first) return "first bitmap offset does not follow the keys";
    if (off[nobs] > bytes) return "bitmaps run past the end of the file";
    // the whole table before any copy: every offset inside the file and
    // none smaller than the one before it
    for (uint64_t i = 0; i < nobs; ++i) {
        if (off[i + 1] < off[i]) return "bitmap offsets decrease";
        if (off[i + 1] > bytes) return "bitmaps run past the end of the file";
    }
    t.nrows = nrows;
    t.keys = a;
    t.keys.insert(t.keys.end(), b.begin(), b.end());
    t.offsets.assign(nobs + 1ull, 0);
    t.bitmaps.clear();
    t.bitmaps.reserve((off[nobs] - off[0]) / 4 + nobs);
    for (uint64_t i = 0; i < nobs; ++i) {
        if (off[i + 1] < off[i]) return "bitmap offsets decrease";
        const uint64_t len = off[i + 1] - off[i];
        if (len % 4) return "a bitmap's byte count is not a multiple of 4";
        // a bitmap the writer left out stays empty, as in the triple
        // fastbit_iapi_deconstruct_index gives for it
        const size_t w0 = t.bitmaps.size();
        t.bitmaps.resize(w0 + len / 4);
        if (len) std::memcpy(t.bitmaps.data() + w0, p + off[i], len);
        t.offsets[i + 1] = (int64_t)t.bitmaps.size();
    }
    return nullptr;
}

}  // namespace

// Host-only: the triple of an index file image (see wahgpu.h).
extern "C" int wahgpu_idxfile_parse(const void* data, uint64_t bytes, int* kind, uint64_t* nrows,
                                    double* keys, uint64_t kcap, uint64_t* nkeys, int64_t* offsets,
                                    uint64_t ocap, uint64_t* noffsets, uint32_t* bitmaps, uint64_t bcap,
                                    uint64_t* nbitmaps) {
    Triple t;
    const char* err = parse(data, bytes, t);
    if (err) return wg_fail(nullptr, WAHGPU_EFORMAT, "index file: %s", err);
    if (kind) *kind = t.kind;
    if (nrows) *nrows = t.nrows;
    if (nkeys) *nkeys = t.keys.size();
    if (noffsets) *noffsets = t.offsets.size();
    if (nbitmaps) *nbitmaps = t.bitmaps.size();
    if (keys && offsets && bitmaps) {
        if (kcap < t.keys.size() || ocap < t.offsets.size() || bcap < t.bitmaps.size())
            return wg_fail(nullptr, WAHGPU_ESIZE, "index file: output arrays too small");
        std::memcpy(keys, t.keys.data(), t.keys.size() * 8);
        std::memcpy(offsets, t.offsets.data(), t.offsets.size() * 8);
        std::memcpy(bitmaps, t.bitmaps.data(), t.bitmaps.size() * 4);
    }
    return WAHGPU_OK;
}

// relic::read / bin::read (src/irelic.cpp:690, src/ibin.cpp:468) from a
// file image already in host memory (e.g. a FastBit fileManager mapping).
extern "C" int wahgpu_index_from_file_image(wahgpu_ctx* ctx, const void* data, uint64_t bytes,
                                            wahgpu_index** out) {
    if (!ctx || !out) return wg_fail(ctx, WAHGPU_EINVAL, "bad argument");
    *out = nullptr;
    Triple t;
    const char* err = parse(data, bytes, t);
    if (err) return wg_fail(ctx, WAHGPU_EFORMAT, "index file: %s", err);
    return wahgpu_index_from_triple(ctx, t.kind, t.nrows, t.keys.data(), t.keys.size(), t.offsets.data(),
                                    t.offsets.size(), t.bitmaps.data(), t.bitmaps.size(), out);
}

// relic::read(const char*) / bin::read(const char*): the named .idx file.
extern "C" int wahgpu_index_read(wahgpu_ctx* ctx, const char* path, wahgpu_index** out) {
    if (!ctx || !path || !out) return wg_fail(ctx, WAHGPU_EINVAL, "bad argument");
    *out = nullptr;
    FILE* f = std::fopen(path, "rb");
    if (!f) return wg_fail(ctx, WAHGPU_EINVAL, "cannot open index file %s", path);
    std::vector<unsigned char> buf;
    unsigned char chunk[1 << 16];
    size_t n;
    while ((n = std::fread(chunk, 1, sizeof chunk, f)) > 0) buf.insert(buf.end(), chunk, chunk + n);
    const bool bad = std::ferror(f) != 0;
    std::fclose(f);
    if (bad) return wg_fail(ctx, WAHGPU_EINVAL, "cannot read index file %s", path);
    return wahgpu_index_from_file_image(ctx, buf.data(), buf.size(), out);
}
