// Word-level arithmetic of 32-bit WAH bitvectors, shared by the CUDA kernels
// and by the host-side dispatcher.
//
// Layout (reference src/bitvector.h:35-58, constants src/bitvector.cpp:18-31):
//   literal word: MSB 0, 31 payload bits, the first row of the group is bit 30
//   fill word   : MSB 1, bit 30 = fill value, bits 0..29 = number of 31-bit
//                 groups the fill covers
// A bitvector is m_vec (whole groups) plus an "active" word of < 31 bits whose
// newest bit is the LSB.
//
// Emission model.  The reference's two-operand kernels (and_c2, or_c2, xor_c2,
// minus_c2 in src/bitvector.cpp:2419-3745) walk both word streams with two
// cursors and emit through append_active / append_counter / copy_runs
// (src/bitvector.h:699-910); compress() (src/bitvector.cpp:378-469) later
// merges equal neighbours.  The words left after compress() are therefore
//   * one word per maximal run of equal all-0 / all-1 groups, and one literal
//     per mixed group;
//   * a run of >= 2 groups is a fill word;
//   * a run of exactly one group is a count-1 fill word iff the walk emitted
//     that group through append_counter or by copying a count-1 fill word
//     verbatim, else the literal 0 / 0x7FFFFFFF.
// The walk is sequential, but its step structure is a finite-state function
// of local information at every boundary between the two streams' words:
// each step lies inside one word of its "driver" operand, and whether a step
// continues across a boundary depends only on the step type and the words
// meeting there.  So the step state at every segment follows from a parallel
// prefix over per-segment transfer functions (5 states, composed as tables).
#ifndef WAH_CORE_CUH
#define WAH_CORE_CUH
#include <stdint.h>

#if defined(__CUDACC__)
#define WAH_HD __host__ __device__ __forceinline__
#else
#define WAH_HD inline
#endif

namespace wah {

constexpr uint32_t MAXBITS = 31u;
constexpr uint32_t ALLONES = 0x7FFFFFFFu;
constexpr uint32_t MAXCNT = 0x3FFFFFFFu;
constexpr uint32_t FILLBIT = 0x40000000u;
constexpr uint32_t HEADER0 = 0x80000000u;
constexpr uint32_t HEADER1 = 0xC0000000u;

enum Op : int { OP_AND = 0, OP_OR = 1, OP_XOR = 2, OP_MINUS = 3 };

// step types of the reference walk
enum Step : uint32_t {
    S_CNT_Y = 0,  // one append_counter spanning to the end of the rhs word
    S_CNT_X = 1,  // one append_counter spanning to the end of the lhs word
    S_CPY_X = 2,  // copy_runs(n) of lhs words, budget = rest of the rhs fill
    S_CPY_Y = 3,  // copy_runs(n) of rhs words, budget = rest of the lhs fill
    S_LIT = 4     // literal & literal through append_active
};

// group classes of a result segment
enum Cls : uint32_t { C_ZERO = 0, C_ONE = 1, C_MIXED = 2, C_NONE = 3 };

WAH_HD bool is_fill(uint32_t w) { return w > ALLONES; }
WAH_HD uint32_t wgroups(uint32_t w) { return w > ALLONES ? (w & MAXCNT) : 1u; }
// fill value as decoded by the reference's run::decode (w > HEADER1)
WAH_HD uint32_t fill_bit(uint32_t w) { return w > HEADER1 ? 1u : 0u; }
// 31-bit pattern of one group covered by word w
WAH_HD uint32_t wpattern(uint32_t w) {
    return w > ALLONES ? (w >= HEADER1 ? ALLONES : 0u) : w;
}
WAH_HD uint32_t apply_op(int op, uint32_t a, uint32_t b) {
    switch (op) {
    case OP_AND: return a & b;
    case OP_OR: return a | b;
    case OP_XOR: return a ^ b;
    default: return a & ~b & ALLONES;
    }
}
WAH_HD uint32_t cls_of(uint32_t v) {
    return v == 0 ? C_ZERO : (v == ALLONES ? C_ONE : C_MIXED);
}
WAH_HD uint32_t fill_word(uint32_t bit, uint32_t n) {
    return (bit ? HEADER1 : HEADER0) | n;
}

// Step chosen by the reference walk when a new step starts at a boundary
// where the lhs word x (remaining rx groups) meets the rhs word y (ry).
//   and_c2 src/bitvector.cpp:2481-2516, or_c2 2874-2924,
//   xor_c2 3287-3320, minus_c2 3681-3720
WAH_HD uint32_t select_step(int op, uint32_t x, uint32_t rx, uint32_t y, uint32_t ry) {
    const bool xf = is_fill(x), yf = is_fill(y);
    const uint32_t xb = fill_bit(x), yb = fill_bit(y);
    switch (op) {
    case OP_AND:
        if (xf) {
            if (yf) return yb == 0 ? S_CNT_Y : (ry >= rx ? S_CPY_X : S_CNT_Y);
            return xb == 0 ? S_CNT_X : S_CPY_Y;
        }
        if (yf) return yb == 0 ? S_CNT_Y : S_CPY_X;
        return S_LIT;
    case OP_OR:
        if (xf) {
            if (yf) return yb != 0 ? S_CNT_Y : (ry < rx ? S_CNT_Y : S_CPY_X);
            return xb != 0 ? S_CNT_X : S_CPY_Y;
        }
        if (yf) return yb != 0 ? S_CNT_Y : S_CPY_X;
        return S_LIT;
    case OP_XOR:
        if (xf) {
            if (yf && ry >= rx) return S_CPY_X;
            return S_CPY_Y;
        }
        if (yf) return S_CPY_X;
        return S_LIT;
    default:  // OP_MINUS
        if (xf) {
            if (yf && ry >= rx) return yb == 0 ? S_CPY_X : S_CNT_Y;
            return xb == 0 ? S_CNT_X : S_CPY_Y;
        }
        if (yf) return yb == 0 ? S_CPY_X : S_CNT_Y;
        return S_LIT;
    }
}

// Does a step of type s in progress continue across a boundary where the lhs
// has a word boundary (xb), the rhs has one (yb), and, for a copy step, the
// word starting there fits in the copy budget (fits_x: lhs word ends no later
// than the rhs driver word; fits_y symmetric)?
WAH_HD bool step_continues(uint32_t s, bool xb, bool yb, bool fits_x, bool fits_y) {
    if (xb && yb) return false;
    if (xb) return s == S_CNT_Y || (s == S_CPY_X && fits_x);
    return s == S_CNT_X || (s == S_CPY_Y && fits_y);
}

// Transfer function of one segment on the 5 step states, packed as 5 x 3-bit
// next-state entries; bit 15+s set when input state s starts a new step.
WAH_HD uint32_t seg_transfer(uint32_t sel, bool xb, bool yb, bool fits_x, bool fits_y) {
    uint32_t f = 0;
#pragma unroll
    for (uint32_t s = 0; s < 5; ++s) {
        const bool c = step_continues(s, xb, yb, fits_x, fits_y);
        f |= (c ? s : sel) << (3 * s);
        f |= (c ? 0u : 1u) << (15 + s);
    }
    return f;
}
constexpr uint32_t FSM_IDENTITY = (0u) | (1u << 3) | (2u << 6) | (3u << 9) | (4u << 12);
WAH_HD uint32_t fsm_apply(uint32_t f, uint32_t s) { return (f >> (3 * s)) & 7u; }
WAH_HD bool fsm_started(uint32_t f, uint32_t s) { return (f >> (15 + s)) & 1u; }
// (g after f): state mapping only; "started" bits are not composed
WAH_HD uint32_t fsm_compose(uint32_t f, uint32_t g) {
    uint32_t h = 0;
#pragma unroll
    for (uint32_t s = 0; s < 5; ++s) h |= fsm_apply(g, fsm_apply(f, s)) << (3 * s);
    return h;
}

// Would the reference emit a one-group uniform segment as a count-1 fill
// word?  Counters always are; inside a copy step the first word goes through
// append_active (a literal) and later whole words are pushed verbatim.
WAH_HD bool seg_fill_flag(uint32_t step, bool started, uint32_t xw, uint32_t yw) {
    switch (step) {
    case S_CNT_Y:
    case S_CNT_X: return true;
    case S_CPY_X: return !started && is_fill(xw);
    case S_CPY_Y: return !started && is_fill(yw);
    default: return false;
    }
}

// The word that represents a maximal run of class c with length len groups
// starting at a segment whose literal value is v and count-1 flag is fflag.
WAH_HD uint32_t run_word(uint32_t c, uint32_t len, uint32_t v, bool fflag) {
    if (c == C_MIXED) return v;
    if (len >= 2) return fill_word(c, len);
    return fflag ? fill_word(c, 1) : (c ? ALLONES : 0u);
}

}  // namespace wah
#endif
