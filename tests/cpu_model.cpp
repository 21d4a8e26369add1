// CPU model of the device operations — test code.
//
// Runs the host-side plan (wah_plan.h) and the segment / step-state rules
// (wah_core.cuh) that the CUDA kernels apply, sequentially on the CPU, with
// the step-state transfer functions composed over random tile splits as the
// look-back composes them across CTAs.  tests/test_host_model.py compares it
// with the reference's golden outputs, so the host logic and the emission
// rules are checked without a GPU.
#include "../libfastlib_b200/csrc/wah_plan.h"
#include <vector>
#include <cstdio>
#include <cstring>
#include <cstdlib>
using namespace wah;
typedef std::vector<uint32_t> V;

struct Bv { V w; uint32_t anb = 0, aval = 0; };
static Bv parse(const uint32_t* s, uint32_t ns) {
    Bv b;
    if (ns > 1) {
        b.w.assign(s, s + ns);
        if (b.w.back() > 0 && b.w.back() < 31) { b.anb = b.w.back(); b.w.pop_back(); b.aval = b.w.back(); }
        b.w.pop_back();
    }
    return b;
}
static OperandMeta meta(const Bv& b) {
    OperandMeta m{(uint32_t)b.w.size(), 0, b.anb, b.aval, 0, b.w.empty() ? 0u : b.w[0]};
    for (uint32_t w : b.w) {
        if (w < HEADER0) { m.groups += 1; m.nset += __builtin_popcount(w); }
        else { uint32_t c = w & MAXCNT; m.groups += c; if (w >= HEADER1) m.nset += c * 31; }
    }
    return m;
}
struct Seg { uint32_t pos, len, val, cls; bool fflag; };
static void encode(const std::vector<Seg>& segs, uint32_t G, V& out) {
    // maximal runs
    size_t i = 0;
    while (i < segs.size()) {
        const Seg& h = segs[i];
        if (h.cls == C_MIXED) { out.push_back(h.val); ++i; continue; }
        size_t j = i + 1;
        while (j < segs.size() && segs[j].cls == h.cls) ++j;
        uint32_t end = (j < segs.size()) ? segs[j].pos : G;
        out.push_back(run_word(h.cls, end - h.pos, h.val, h.fflag));
        i = j;
    }
}
static void merge(int op, bool fsm, const V& X, const V& Y, uint32_t G, V& out, unsigned seed) {
    std::vector<Seg> segs;
    std::vector<uint32_t> trans, sel_unused;
    std::vector<uint32_t> xw, yw;
    size_t i = 0, j = 0;
    uint32_t pos = 0, xs = 0, ys = 0;  // start positions of current words
    uint32_t xe = X.empty() ? 0 : wgroups(X[0]), ye = Y.empty() ? 0 : wgroups(Y[0]);
    while (i < X.size() && j < Y.size()) {
        uint32_t e = xe <= ye ? xe : ye;
        uint32_t xwd = X[i], ywd = Y[j];
        if (e > pos) {
            Seg s; s.pos = pos; s.len = e - pos;
            s.val = apply_op(op, wpattern(xwd), wpattern(ywd));
            s.cls = cls_of(s.val);
            if (s.len > 1 && s.cls == C_MIXED) { fprintf(stderr, "mixed multi\n"); exit(1); }
            bool xb = (pos == xs), yb = (pos == ys);
            uint32_t sel = select_step(op, xwd, xe - pos, ywd, ye - pos);
            trans.push_back(seg_transfer(sel, xb, yb, xe <= ye, ye <= xe));
            xw.push_back(xwd); yw.push_back(ywd);
            s.fflag = false;
            segs.push_back(s);
            pos = e;
        }
        if (xe <= ye) { ++i; xs = xe; if (i < X.size()) xe += wgroups(X[i]); }
        else { ++j; ys = ye; if (j < Y.size()) ye += wgroups(Y[j]); }
    }
    if (fsm) {
        // tile the segments randomly, compose per tile, then resolve
        srand(seed);
        std::vector<size_t> cuts{0};
        for (size_t k = 1; k < segs.size(); ++k) if (rand() % 3 == 0) cuts.push_back(k);
        cuts.push_back(segs.size());
        uint32_t state = S_LIT;  // arbitrary: first segment always starts a step
        for (size_t t = 0; t + 1 < cuts.size(); ++t) {
            uint32_t agg = FSM_IDENTITY;
            for (size_t k = cuts[t]; k < cuts[t + 1]; ++k) agg = fsm_compose(agg, trans[k]);
            uint32_t s = state;
            for (size_t k = cuts[t]; k < cuts[t + 1]; ++k) {
                bool st = fsm_started(trans[k], s);
                s = fsm_apply(trans[k], s);
                segs[k].fflag = seg_fill_flag(s, st, xw[k], yw[k]);
            }
            uint32_t s2 = fsm_apply(agg, state);
            if (s2 != s) { fprintf(stderr, "compose mismatch\n"); exit(1); }
            state = s;
        }
    }
    encode(segs, G, out);
}
static void copyc(const V& X, bool flip, uint32_t G, V& out) {
    std::vector<Seg> segs;
    uint32_t pos = 0;
    for (uint32_t w : X) {
        Seg s; s.pos = pos; s.len = wgroups(w);
        uint32_t p = wpattern(w);
        if (flip) p ^= ALLONES;
        s.val = p; s.cls = cls_of(p); s.fflag = is_fill(w);
        segs.push_back(s); pos += s.len;
    }
    encode(segs, G, out);
}
static uint32_t wcnt(uint32_t w) {
    if (w < HEADER0) return __builtin_popcount(w);
    return (w >= HEADER1) ? (w & MAXCNT) * 31 : 0;
}
extern "C" long model_binop(int op, int inplace, const uint32_t* sa, uint32_t na,
                            const uint32_t* sb, uint32_t nb, uint32_t* out, uint32_t cap,
                            uint32_t* cnt, int* kind) {
    Bv A = parse(sa, na), B = parse(sb, nb);
    OperandMeta ma = effective(meta(A)), mb = effective(meta(B));
    if (ma.n == 1 && A.w.size() > 1) A.w.assign(1, ma.w0);
    if (mb.n == 1 && B.w.size() > 1) B.w.assign(1, mb.w0);
    Plan p = plan_binop(op, inplace, ma, mb);
    *kind = p.kind;
    V res;
    switch (p.kind) {
    case PK_UNEQUAL: return -2;
    case PK_EMPTY: break;
    case PK_RAW1: {
        uint32_t x = A.w[0], y = B.w[0], r;
        switch (op) { case OP_AND: r = x & y; break; case OP_OR: r = x | y; break;
                      case OP_XOR: r = x ^ y; break; default: r = x & ~y; }
        res.push_back(r); break; }
    case PK_ZERO_FILL: res.push_back(HEADER0 | p.fill_n); break;
    case PK_COPY: copyc(p.src ? B.w : A.w, false, ma.groups, res); break;
    case PK_COPY_FLIP: copyc(p.src ? B.w : A.w, true, ma.groups, res); break;
    case PK_MERGE_CANON: merge(op, false, A.w, B.w, ma.groups, res, 0); break;
    case PK_MERGE_FSM: merge(op, true, A.w, B.w, ma.groups, res, na * 7 + nb); break;
    }
    uint32_t aval = apply_op(op, A.aval, B.aval);
    if (op == OP_MINUS) aval = A.aval & ~B.aval;
    uint32_t anb = A.anb;
    if (anb) aval &= (1u << anb) - 1; else aval = 0;
    uint32_t c = 0;
    for (uint32_t w : res) c += wcnt(w);
    *cnt = c + __builtin_popcount(aval);
    V ser = res;
    if (anb) ser.push_back(aval);
    ser.push_back(anb);
    if (ser.size() <= cap) memcpy(out, ser.data(), ser.size() * 4);
    return (long)ser.size();
}
