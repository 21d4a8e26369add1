// Host-side choice of the device operation that reproduces one reference
// bitvector operator.  The reference picks its kernel from the operands'
// word counts and shapes (src/bitvector.cpp:1194-1838); the words it leaves
// after compress() depend on that choice, so the same choice is made here
// from the operands' metadata, and one of a handful of device operations
// produces the identical words:
//   MERGE_FSM    the _c2 kernels: merge with the walk's count-1-fill rule
//   MERGE_CANON  the _d2/_d1/_c1/_c0 kernels and the all-literal loops:
//                their output is uncompressed (or compressed without
//                count-1 fills), so compress() makes it canonical
//   COPY         a copy of one operand's words, then compress()
//   COPY_FLIP    a complemented copy (flip()), then compress()
//   ZERO_FILL    a single 0-fill word written by append_counter
//   RAW1         one-group operands: the all-literal loops combine the raw
//                words (a count-1 fill word is combined as raw bits)
//   EMPTY        no whole words; only the active words combine
// The result's active word is always op(lhs.active, rhs.active).
#ifndef WAH_PLAN_H
#define WAH_PLAN_H
#include <stdint.h>
#include "wah_core.cuh"

namespace wah {

// Operand as the reference sees it after size() has run: operands built
// from serialized arrays count their bits lazily, and do_cnt()
// (src/bitvector.cpp:583-608) collapses an m_vec with no 1 bits and more
// than one word into a single 0-fill.
struct OperandMeta {
    uint32_t n;       // words in m_vec
    uint32_t groups;  // nbits / 31
    uint32_t anb;     // active bits
    uint32_t aval;    // active value
    uint32_t nset;    // 1 bits in m_vec
    uint32_t w0;      // first word (valid when n >= 1)
};

inline OperandMeta effective(OperandMeta m) {
    if (m.nset == 0 && m.n > 1) { m.n = 1; m.w0 = HEADER0 | m.groups; }
    return m;
}
inline bool all0s(const OperandMeta& m) {  // src/bitvector.h all0s()
    return m.n == 0 || (m.n == 1 && (m.w0 == 0 || (m.w0 >= HEADER0 && m.w0 < HEADER1)));
}
inline bool all1s(const OperandMeta& m) {  // src/bitvector.h all1s()
    return m.n == 1 && (m.w0 == ALLONES || m.w0 > HEADER1);
}

enum PlanKind : int {
    PK_MERGE_FSM = 0,
    PK_MERGE_CANON = 1,
    PK_COPY = 2,
    PK_COPY_FLIP = 3,
    PK_ZERO_FILL = 4,
    PK_RAW1 = 5,
    PK_EMPTY = 6,
    PK_UNEQUAL = 7  // sizes differ: the shorter operand is padded first
};

struct Plan {
    int kind;
    int src;          // COPY / COPY_FLIP: 0 = lhs, 1 = rhs
    uint32_t fill_n;  // ZERO_FILL count
};

// op: OP_AND..OP_MINUS; inplace: the OP= form.  a = lhs ("this"), r = rhs,
// both already passed through effective().
inline Plan plan_binop(int op, bool inplace, const OperandMeta& a, const OperandMeta& r) {
    Plan p{PK_MERGE_CANON, 0, 0};
    const uint64_t sa = (uint64_t)a.groups * MAXBITS + a.anb;
    const uint64_t sr = (uint64_t)r.groups * MAXBITS + r.anb;
    if (sa != sr) { p.kind = PK_UNEQUAL; return p; }
    const uint32_t G = a.groups;
    if (G == 0) {
        // operator- tests n*31==nbits without nbits>0 (src/bitvector.cpp:1788):
        // both "uncompressed", active words only; the others reach all0s()
        p.kind = PK_EMPTY;
        return p;
    }
    if (G == 1) { p.kind = PK_RAW1; return p; }
    const bool ca = (a.n == G), cb = (r.n == G);
    const uint64_t nsum = (uint64_t)a.n + r.n;
    if (!inplace) {
        if (ca || cb) return p;  // all-literal loop or _c1/_c1x: canonical
        switch (op) {
        case OP_AND:
            if (all0s(a) || all1s(r)) { p.kind = PK_COPY; p.src = 0; return p; }
            if (all1s(a) || all0s(r)) { p.kind = PK_COPY; p.src = 1; return p; }
            break;
        case OP_OR:
            if (all1s(a) || all0s(r)) { p.kind = PK_COPY; p.src = 0; return p; }
            if (all0s(a) || all1s(r)) { p.kind = PK_COPY; p.src = 1; return p; }
            break;
        case OP_XOR: break;
        default:
            if (all0s(a) || all0s(r)) { p.kind = PK_COPY; p.src = 0; return p; }
            if (all1s(r)) { p.kind = PK_ZERO_FILL; p.fill_n = r.w0 & MAXCNT; return p; }
            if (all1s(a)) { p.kind = PK_COPY_FLIP; p.src = 1; return p; }
        }
        p.kind = (nsum > G) ? PK_MERGE_CANON : PK_MERGE_FSM;
        return p;
    }
    // OP= forms
    if (ca || cb) return p;  // _c0 / _d1 / swapped _d1 / _c1: canonical
    switch (op) {
    case OP_AND:
        if (all0s(a) || all1s(r)) { p.kind = PK_COPY; p.src = 0; return p; }
        if (all0s(r) || all1s(a)) { p.kind = PK_COPY; p.src = 1; return p; }
        break;
    case OP_OR:
        if (all1s(a) || all0s(r)) { p.kind = PK_COPY; p.src = 0; return p; }
        if (all0s(a) || all1s(r)) { p.kind = PK_COPY; p.src = 1; return p; }
        break;
    case OP_XOR: break;
    default:
        if (all0s(a) || all0s(r)) { p.kind = PK_COPY; p.src = 0; return p; }
        if (all1s(r)) { p.kind = PK_ZERO_FILL; p.fill_n = r.w0 & MAXCNT; return p; }
        if (all1s(a)) { p.kind = PK_COPY_FLIP; p.src = 1; return p; }
    }
    p.kind = (nsum >= G) ? PK_MERGE_CANON : PK_MERGE_FSM;
    return p;
}

}  // namespace wah
#endif
