// Host-only parts of include/wahgpu.hpp, no device: the indexSet walk over
// serialized words and the truncation used by a shrinking adjustSize.
// Reads bitvectors from argv[1] (count, then per vector: bits to keep,
// word count, words), writes per vector the positions the indexSet walk
// yields and the truncated serialized words to argv[2].
#include <cstdio>
#include <fstream>
#include <memory>
#include <vector>
#include "wahgpu.hpp"

using wahgpu_ibis::bitvector;

static uint32_t rd(std::ifstream& f) { uint32_t v = 0; f.read(reinterpret_cast<char*>(&v), 4); return v; }
static void wr(std::ofstream& f, uint32_t v) { f.write(reinterpret_cast<const char*>(&v), 4); }
static void wrv(std::ofstream& f, const std::vector<uint32_t>& v) {
    wr(f, (uint32_t)v.size());
    if (!v.empty()) f.write(reinterpret_cast<const char*>(v.data()), v.size() * 4);
}

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    std::ifstream in(argv[1], std::ios::binary);
    std::ofstream out(argv[2], std::ios::binary);
    const uint32_t n = rd(in);
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t keep = rd(in), nw = rd(in);
        auto w = std::make_shared<std::vector<uint32_t>>(nw);
        if (nw) in.read(reinterpret_cast<char*>(w->data()), nw * 4);
        std::vector<uint32_t> pos;
        for (bitvector::indexSet is(w); is.nIndices() > 0; ++is) {
            const uint32_t* ii = is.indices();
            if (is.isRange()) for (uint32_t j = ii[0]; j < ii[1]; ++j) pos.push_back(j);
            else for (uint32_t j = 0; j < is.nIndices(); ++j) pos.push_back(ii[j]);
        }
        wrv(out, pos);
        std::vector<uint32_t> t(*w);
        bitvector::truncate(t, keep);
        wrv(out, t);
    }
    return 0;
}
