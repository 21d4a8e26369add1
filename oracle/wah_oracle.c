/*
 * CPU oracle for the WAH bitvector hot path — TEST INFRASTRUCTURE ONLY.
 * See wah_oracle.h.  Every function below restates the reference function
 * named in its comment (paths relative to the reference's src/), including
 * the reference's emission rules, its lazy counters and its quirks on
 * one-word operands, because word-for-word parity depends on them.
 */
#include "wah_oracle.h"
#include <stdlib.h>
#include <string.h>

#define MAXBITS   31u
#define SECONDBIT 30u
#define ALLONES   0x7FFFFFFFu
#define MAXCNT    0x3FFFFFFFu
#define FILLBIT   0x40000000u
#define HEADER0   0x80000000u
#define HEADER1   0xC0000000u

/* ---------------------------------------------------------------- vector */
static void vreserve(wo_bv *b, uint32_t n) {
    if (n <= b->cap) return;
    uint32_t c = b->cap ? b->cap : 16;
    while (c < n) c = (c > 0x7FFFFFFFu) ? n : 2 * c;
    b->v = (uint32_t *)realloc(b->v, (size_t)c * 4);
    b->cap = c;
}
static void vpush(wo_bv *b, uint32_t w) {
    if (b->n == b->cap) vreserve(b, b->n + 1);
    b->v[b->n++] = w;
}
static void vresize(wo_bv *b, uint32_t n) {
    vreserve(b, n);
    if (n > b->n) memset(b->v + b->n, 0, (size_t)(n - b->n) * 4);
    b->n = n;
}
static uint32_t cnt_ones(uint32_t w) { return (uint32_t)__builtin_popcount(w); }

void wo_init(wo_bv *b) { memset(b, 0, sizeof(*b)); }
void wo_free(wo_bv *b) { free(b->v); wo_init(b); }
/* clear() bitvector.cpp:304 */
static void bv_clear(wo_bv *b) { b->nset = 0; b->nbits = 0; b->n = 0; b->aval = 0; b->anb = 0; }
/* copy() bitvector.h: deep copy of every member */
void wo_copy(wo_bv *d, const wo_bv *s) {
    if (d == s) return;
    vreserve(d, s->n);
    if (s->n) memcpy(d->v, s->v, (size_t)s->n * 4);
    d->n = s->n; d->nbits = s->nbits; d->nset = s->nset;
    d->aval = s->aval; d->anb = s->anb;
}
static void vcopy_words(wo_bv *d, const wo_bv *s) { /* m_vec.deepCopy */
    vreserve(d, s->n);
    if (s->n) memcpy(d->v, s->v, (size_t)s->n * 4);
    d->n = s->n;
}
static void bv_swap(wo_bv *a, wo_bv *b) { wo_bv t = *a; *a = *b; *b = t; }

/* do_cnt() bitvector.cpp:583-608, including its collapse of an all-zero
 * m_vec into one 0-fill */
static uint32_t do_cnt(wo_bv *b) {
    uint32_t ns = 0, nb = 0;
    if (b->n > 0) {
        for (uint32_t i = 0; i < b->n; ++i) {
            uint32_t w = b->v[i];
            if (w < HEADER0) { nb += MAXBITS; ns += cnt_ones(w); }
            else { uint32_t t = (w & MAXCNT) * MAXBITS; nb += t; ns += t * (w >= HEADER1); }
        }
        if (ns == 0 && b->n > 1) { b->v[0] = HEADER0 + (nb / MAXBITS); b->n = 1; }
    }
    b->nset = ns;
    return nb;
}
/* size() bitvector.h:647 */
uint32_t wo_size(wo_bv *b) { return (b->nbits ? b->nbits : (b->nbits = do_cnt(b))) + b->anb; }
/* cnt() bitvector.h:652 */
uint32_t wo_cnt(wo_bv *b) {
    if (b->nset == 0 && b->n > 0) b->nbits = do_cnt(b);
    return b->nset + cnt_ones(b->aval);
}
static int all0s(const wo_bv *b) { /* bitvector.h all0s() */
    if (b->n == 0) return 1;
    if (b->n == 1) return b->v[0] == 0 || (b->v[0] >= HEADER0 && b->v[0] < HEADER1);
    return 0;
}
static int all1s(const wo_bv *b) { /* bitvector.h all1s() */
    if (b->n == 1) return b->v[0] == ALLONES || b->v[0] > HEADER1;
    return 0;
}

/* ------------------------------------------------------ emission helpers */
/* append_active() bitvector.h:699-737 */
static void append_active(wo_bv *b) {
    if (b->n == 0) vpush(b, b->aval);
    else if (b->aval == 0) {
        uint32_t *bk = &b->v[b->n - 1];
        if (*bk == 0) *bk = HEADER0 + 2;
        else if (*bk >= HEADER0 && *bk < HEADER1) ++*bk;
        else vpush(b, b->aval);
    } else if (b->aval == ALLONES) {
        uint32_t *bk = &b->v[b->n - 1];
        if (*bk == ALLONES) *bk = HEADER1 | 2;
        else if (*bk >= HEADER1) ++*bk;
        else vpush(b, b->aval);
    } else vpush(b, b->aval);
    b->nbits += MAXBITS;
    b->aval = 0; b->anb = 0;
    b->nset = 0;
}
/* append_counter() bitvector.h:741-760 */
static void append_counter(wo_bv *b, int val, uint32_t cnt) {
    uint32_t head = 2 + (uint32_t)val;
    uint32_t w = (head << SECONDBIT) + cnt;
    b->nbits += cnt * MAXBITS;
    if (b->n == 0) vpush(b, w);
    else {
        uint32_t *bk = &b->v[b->n - 1];
        if ((*bk >> SECONDBIT) == head) *bk += cnt;
        else if (*bk == ALLONES && head == 3) *bk = w + 1;
        else if (*bk == 0 && head == 2) *bk = w + 1;
        else vpush(b, w);
    }
}

/* run struct bitvector.h:225-261, over a word array */
typedef struct { int isFill, fillBit; uint32_t nWords; uint32_t it; const uint32_t *a; } run_t;
static void rdecode(run_t *r) {
    uint32_t w = r->a[r->it];
    r->fillBit = (w > HEADER1);
    if (w > ALLONES) { r->nWords = w & MAXCNT; r->isFill = 1; }
    else { r->nWords = 1; r->isFill = 0; }
}
static void rsub(run_t *r, uint32_t len) { /* run::operator-= */
    while (len > 0) {
        if (r->nWords == 0) rdecode(r);
        if (r->isFill) {
            if (r->nWords > len) { r->nWords -= len; len = 0; }
            else if (r->nWords == len) { r->nWords = 0; len = 0; ++r->it; }
            else { len -= r->nWords; ++r->it; r->nWords = 0; }
        } else { --len; ++r->it; r->nWords = 0; }
    }
}

/* copy_runs(run&, word_t&) bitvector.h:838-875 */
static void copy_runs(wo_bv *b, run_t *it, uint32_t *nw) {
    if (it->isFill == 0) { b->aval = it->a[it->it]; append_active(b); --*nw; }
    else if (it->nWords > 1) { append_counter(b, it->fillBit, it->nWords); *nw -= it->nWords; }
    else if (it->nWords == 1) { b->aval = it->fillBit ? ALLONES : 0; append_active(b); --*nw; }
    ++it->it;
    b->nset = 0;
    it->nWords = 0;
    b->nbits += MAXBITS * *nw;
    while (*nw > 0) {
        rdecode(it);
        if (*nw >= it->nWords) {
            vpush(b, it->a[it->it]);
            *nw -= it->nWords; it->nWords = 0; ++it->it;
        } else break;
    }
    b->nbits -= MAXBITS * *nw;
}
/* copy_runsn(run&, word_t&) bitvector.h:879-910 */
static void copy_runsn(wo_bv *b, run_t *it, uint32_t *nw) {
    if (it->isFill == 0) { b->aval = ALLONES ^ it->a[it->it]; append_active(b); --*nw; }
    else if (it->nWords > 1) { append_counter(b, !it->fillBit, it->nWords); *nw -= it->nWords; }
    else if (it->nWords == 1) { b->aval = it->fillBit ? 0 : ALLONES; append_active(b); --*nw; }
    ++it->it;
    b->nset = 0;
    it->nWords = 0;
    b->nbits += MAXBITS * *nw;
    while (*nw > 0) {
        rdecode(it);
        if (*nw >= it->nWords) {
            vpush(b, (it->isFill ? FILLBIT : ALLONES) ^ it->a[it->it]);
            *nw -= it->nWords; it->nWords = 0; ++it->it;
        } else break;
    }
    b->nbits -= MAXBITS * *nw;
}
/* copy_fill(iterator&, run&) bitvector.h:915-957 */
static void copy_fill_d(uint32_t **jt, run_t *it) {
    uint32_t v = it->fillBit ? ALLONES : 0;
    for (uint32_t k = 0; k < it->nWords; ++k) *(*jt)++ = v;
    it->nWords = 0;
    ++it->it;
}
/* copy_runs(iterator&, run&, word_t&) bitvector.h:963-997 */
static void copy_runs_d(uint32_t **jt, run_t *it, uint32_t *nw) {
    while (*nw >= it->nWords && *nw > 0) {
        if (it->isFill) {
            uint32_t v = it->fillBit ? ALLONES : 0;
            for (uint32_t k = 0; k < it->nWords; ++k) *(*jt)++ = v;
            *nw -= it->nWords;
        } else { *(*jt)++ = it->a[it->it]; --*nw; }
        ++it->it;
        if (*nw > 0) rdecode(it);
        else { it->nWords = 0; return; }
    }
}
/* copy_runsn(iterator&, run&, word_t&) bitvector.h:1001-1033 */
static void copy_runsn_d(uint32_t **jt, run_t *it, uint32_t *nw) {
    while (*nw >= it->nWords) {
        if (it->isFill) {
            uint32_t v = it->fillBit ? 0 : ALLONES;
            for (uint32_t k = 0; k < it->nWords; ++k) *(*jt)++ = v;
            *nw -= it->nWords;
        } else { *(*jt)++ = it->a[it->it] ^ ALLONES; --*nw; }
        ++it->it;
        if (*nw > 0) rdecode(it);
        else { it->nWords = 0; return; }
    }
}

/* ------------------------------------------------------- whole-vector ops */
/* decompress(array_t&) const bitvector.cpp:515-540 */
static void decompress_to(wo_bv *b, wo_bv *tmp) {
    uint32_t nb = (b->nbits == 0 && b->n > 0) ? do_cnt(b) : b->nbits;
    vresize(tmp, nb / MAXBITS);
    uint32_t k = 0;
    for (uint32_t i = 0; i < b->n; ++i) {
        uint32_t w = b->v[i];
        if (w > ALLONES) {
            uint32_t c = w & MAXCNT, val = (w >= HEADER1) ? ALLONES : 0;
            for (uint32_t j = 0; j < c; ++j) tmp->v[k++] = val;
        } else tmp->v[k++] = w;
    }
}
/* copy_comp(array_t&) const bitvector.cpp:544-567 */
static void copy_comp(wo_bv *b, wo_bv *tmp) {
    uint32_t c0 = (b->nbits == 0 && b->n > 0 ? do_cnt(b) : b->nbits) / MAXBITS;
    vresize(tmp, c0);
    uint32_t k = 0;
    for (uint32_t i = 0; i < b->n; ++i) {
        uint32_t w = b->v[i];
        if (w > ALLONES) {
            uint32_t c = w & MAXCNT, val = (w >= HEADER1) ? 0 : ALLONES;
            for (uint32_t j = 0; j < c; ++j) tmp->v[k++] = val;
        } else tmp->v[k++] = ALLONES ^ w;
    }
}
/* decompress() bitvector.cpp:474-512 */
void wo_decompress(wo_bv *b) {
    if (b->nbits == 0 && b->n > 0) b->nbits = do_cnt(b);
    if ((uint64_t)b->n * MAXBITS == b->nbits) return;
    wo_bv tmp; wo_init(&tmp);
    vresize(&tmp, b->nbits / MAXBITS);
    uint32_t k = 0;
    for (uint32_t i = 0; i < b->n; ++i) {
        uint32_t w = b->v[i];
        if (w > ALLONES) {
            uint32_t c = w & MAXCNT, val = (w >= HEADER1) ? ALLONES : 0;
            for (uint32_t j = 0; j < c; ++j) tmp.v[k++] = val;
        } else tmp.v[k++] = w;
    }
    free(b->v); b->v = tmp.v; b->n = tmp.n; b->cap = tmp.cap;
}
/* compress() bitvector.cpp:378-469 */
void wo_compress(wo_bv *b) {
    if (b->n < 2) return;
    uint32_t *v = b->v;
    uint32_t last = 0;
    int lastFill = v[0] > ALLONES, lastBit = v[0] > HEADER1;
    for (uint32_t cur = 1; cur < b->n; ++cur) {
        uint32_t w = v[cur];
        int cFill = w > ALLONES, cBit = w > HEADER1;
        uint32_t cN = w & MAXCNT;
        if (lastFill) {
            if (cFill) {
                if (cBit == lastBit) v[last] += cN;
                else { ++last; v[last] = w; lastBit = cBit; }
            } else if ((lastBit == 0 && w == 0) || (lastBit != 0 && w == ALLONES)) {
                ++v[last];
            } else { ++last; lastFill = 0; v[last] = w; }
        } else if (cFill) {
            if ((cBit == 0 && v[last] == 0) || (cBit != 0 && v[last] == ALLONES)) {
                v[last] = w + 1; lastBit = cBit; lastFill = 1;
            } else { ++last; lastFill = 1; v[last] = w; lastBit = cBit; }
        } else if (v[last] == w) {
            if (w == 0) { v[last] = HEADER0 | 2; lastFill = 1; lastBit = 0; }
            else if (w == ALLONES) { v[last] = HEADER1 | 2; lastFill = 1; lastBit = 1; }
            else { ++last; v[last] = w; }
        } else { ++last; v[last] = w; }
    }
    ++last;
    if (last < b->n) b->n = last;
}
/* flip() bitvector.cpp:1128-1174 */
void wo_flip(wo_bv *b) {
    if (b->nbits > 0) {
        for (uint32_t i = 0; i < b->n; ++i) b->v[i] ^= (b->v[i] > ALLONES) ? FILLBIT : ALLONES;
    } else {
        b->nbits = 0;
        for (uint32_t i = 0; i < b->n; ++i) {
            if (b->v[i] > ALLONES) { b->v[i] ^= FILLBIT; b->nbits += MAXBITS * (b->v[i] & MAXCNT); }
            else { b->v[i] ^= ALLONES; b->nbits += MAXBITS; }
        }
    }
    if (b->nset > 0) b->nset = b->nbits - b->nset;
    if (b->anb > 0) b->aval ^= ((1u << b->anb) - 1);
}
/* set(val, n) bitvector.cpp:316-340 */
void wo_set(wo_bv *b, int val, uint32_t n) {
    bv_clear(b);
    uint32_t k = n / MAXBITS;
    if (k > 1) append_counter(b, val, k);
    else if (k == 1) { b->aval = val ? ALLONES : 0; append_active(b); }
    b->anb = n - k * MAXBITS;
    if (val) { b->aval = (1u << b->anb) - 1; b->nset = k * MAXBITS; }
}
/* appendFill(val, n) bitvector.h:800-834 */
void wo_append_fill(wo_bv *b, int val, uint32_t n) {
    if (n == 0) return;
    if (b->anb > 0) {
        uint32_t tmp = MAXBITS - b->anb;
        if (tmp > n) tmp = n;
        b->anb += tmp;
        b->aval <<= tmp;
        n -= tmp;
        if (val) b->aval |= (1u << tmp) - 1;
        if (b->anb >= MAXBITS) append_active(b);
    }
    if (n >= MAXBITS) {
        uint32_t cnt = n / MAXBITS;
        if (cnt > 1) append_counter(b, val, cnt);
        else if (val) { b->aval = ALLONES; append_active(b); }
        else { b->aval = 0; append_active(b); }
        n -= cnt * MAXBITS;
    }
    if (n > 0) { b->anb = n; b->aval = (uint32_t)val * ((1u << n) - 1); }
}
/* adjustSize(nv, nt) bitvector.cpp:4086-4108; only the growing branch is
 * reachable from the logical operators */
void wo_adjust_size(wo_bv *b, uint32_t nv, uint32_t nt) {
    if (b->nbits == 0 || (uint64_t)b->nbits < (uint64_t)b->n * MAXBITS) b->nbits = do_cnt(b);
    uint32_t sz = b->nbits + b->anb;
    if (sz == nt) return;
    if (nt > sz) {
        if (nv > nt) nv = nt;
        if (nv > sz) { wo_append_fill(b, 1, nv - sz); if (nt > nv) wo_append_fill(b, 0, nt - nv); }
        else wo_append_fill(b, 0, nt - sz);
    }
}
/* setBit(ind, 1) for ind >= size(): the appending case of
 * bitvector.cpp:621-660, used to build bitmaps row by row */
void wo_set_bit(wo_bv *b, uint32_t ind, int val) {
    uint32_t sz = wo_size(b);
    if (ind >= sz) {
        if (ind > sz) wo_append_fill(b, 0, ind - sz);
        b->aval = (b->aval << 1) | (val != 0); ++b->anb;
        if (b->anb >= MAXBITS) append_active(b);
        b->nset = 0;
    }
}

/* ------------------------------------------------------------ AND kernels */
/* and_c2 bitvector.cpp:2419-2542 */
static void and_c2(wo_bv *x_, wo_bv *y_, wo_bv *res) {
    bv_clear(res);
    if (x_->n == 1) {
        uint32_t w = x_->v[0];
        if (w > HEADER1) { vcopy_words(res, y_); res->nbits = y_->nbits; res->nset = y_->nset; }
        else if (w > ALLONES) { vcopy_words(res, x_); res->nbits = x_->nbits; res->nset = 0; }
        else { vpush(res, w & y_->v[0]); res->nbits = x_->nbits; }
    } else if (y_->n == 1) {
        uint32_t w = y_->v[0];
        if (w > HEADER1) { vcopy_words(res, x_); res->nbits = x_->nbits; res->nset = x_->nset; }
        else if (w > ALLONES) { vcopy_words(res, y_); res->nbits = y_->nbits; res->nset = 0; }
        else { vpush(res, w & x_->v[0]); res->nbits = x_->nbits; }
    } else if (x_->n > 1) {
        run_t x = {0, 0, 0, 0, x_->v}, y = {0, 0, 0, 0, y_->v};
        while (x.it < x_->n) {
            if (x.nWords == 0) rdecode(&x);
            if (y.nWords == 0) rdecode(&y);
            if (x.isFill) {
                if (y.isFill) {
                    if (y.fillBit == 0) { append_counter(res, 0, y.nWords); rsub(&x, y.nWords); y.nWords = 0; ++y.it; }
                    else if (y.nWords >= x.nWords) { copy_runs(res, &x, &y.nWords); y.it += (y.nWords == 0); }
                    else { append_counter(res, x.fillBit, y.nWords); x.nWords -= y.nWords; y.nWords = 0; ++y.it; }
                } else if (x.fillBit == 0) { append_counter(res, 0, x.nWords); rsub(&y, x.nWords); x.nWords = 0; ++x.it; }
                else { copy_runs(res, &y, &x.nWords); x.it += (x.nWords == 0); }
            } else if (y.isFill) {
                if (y.fillBit == 0) { append_counter(res, 0, y.nWords); rsub(&x, y.nWords); y.nWords = 0; ++y.it; }
                else { copy_runs(res, &x, &y.nWords); y.it += (y.nWords == 0); }
            } else {
                res->aval = x_->v[x.it] & y_->v[y.it]; append_active(res);
                x.nWords = 0; y.nWords = 0; ++x.it; ++y.it;
            }
        }
    }
    if (x_->anb) { res->aval = x_->aval & y_->aval; res->anb = x_->anb; }
}
/* and_c1 bitvector.cpp:2545-2610 (rhs uncompressed) */
static void and_c1(wo_bv *x_, wo_bv *y_, wo_bv *res) {
    bv_clear(res);
    if (x_->n == 1) {
        uint32_t w = x_->v[0];
        if (w > HEADER1) { vcopy_words(res, y_); res->nbits = y_->nbits; res->nset = y_->nset; }
        else if (w > ALLONES) { vcopy_words(res, x_); res->nbits = x_->nbits; res->nset = 0; }
        else { vpush(res, w & y_->v[0]); res->nbits = x_->nbits; }
    } else if (x_->n > 1) {
        uint32_t i1 = 0;
        for (uint32_t i0 = 0; i0 < x_->n; ++i0) {
            uint32_t w = x_->v[i0];
            if (w > ALLONES) {
                uint32_t s0 = w & MAXCNT;
                if (w < HEADER1) { if (s0 > 1) append_counter(res, 0, s0); else append_active(res); i1 += s0; }
                else { for (uint32_t k = 0; k < s0; ++k) vpush(res, y_->v[i1++]); res->nbits += s0 * MAXBITS; }
            } else { res->aval = w & y_->v[i1]; append_active(res); i1++; }
        }
    }
    res->aval = x_->aval & y_->aval; res->anb = x_->anb;
}
static uint32_t d2_nbits(wo_bv *x, wo_bv *y) { /* res.nbits expression of the _d2 kernels */
    return (x->nbits == 0 && x->n > 0) ?
        ((y->nbits == 0 && y->n > 0) ? (x->n <= y->n ? do_cnt(x) : do_cnt(y)) : y->nbits) : x->nbits;
}
/* and_d2 bitvector.cpp:2613-2749 */
static void and_d2(wo_bv *x_, wo_bv *y_, wo_bv *res) {
    res->nbits = d2_nbits(x_, y_);
    vresize(res, res->nbits / MAXBITS);
    if (x_->n == 1) {
        uint32_t w = x_->v[0];
        if (w > HEADER1) { decompress_to(y_, res); res->nset = y_->nset; }
        else if (w > ALLONES) { decompress_to(x_, res); res->nset = 0; }
        else { res->v[0] = w & y_->v[0]; res->nset = cnt_ones(res->v[0]); }
    } else if (y_->n == 1) {
        uint32_t w = y_->v[0];
        if (w > HEADER1) { decompress_to(x_, res); res->nset = x_->nset; }
        else if (w > ALLONES) { decompress_to(y_, res); res->nset = 0; }
        else { res->v[0] = w & x_->v[0]; res->nset = cnt_ones(res->v[0]); }
    } else if (x_->n > 1) {
        run_t x = {0, 0, 0, 0, x_->v}, y = {0, 0, 0, 0, y_->v};
        res->nset = 0;
        uint32_t *ir = res->v;
        while (x.it < x_->n) {
            if (x.nWords == 0) rdecode(&x);
            if (y.nWords == 0) rdecode(&y);
            if (x.isFill) {
                if (y.isFill) {
                    if (y.fillBit == 0) { rsub(&x, y.nWords); copy_fill_d(&ir, &y); }
                    else if (y.nWords < x.nWords) { x.nWords -= y.nWords; y.fillBit = x.fillBit; copy_fill_d(&ir, &y); }
                    else { copy_runs_d(&ir, &x, &y.nWords); y.it += (y.nWords == 0); }
                } else if (x.fillBit == 0) { rsub(&y, x.nWords); copy_fill_d(&ir, &x); }
                else { copy_runs_d(&ir, &y, &x.nWords); x.it += (x.nWords == 0); }
            } else if (y.isFill) {
                if (y.fillBit == 0) { rsub(&x, y.nWords); copy_fill_d(&ir, &y); }
                else { copy_runs_d(&ir, &x, &y.nWords); y.it += (y.nWords == 0); }
            } else { *ir++ = x_->v[x.it] & y_->v[y.it]; x.nWords = 0; y.nWords = 0; ++x.it; ++y.it; }
        }
    }
    res->aval = x_->aval & y_->aval; res->anb = x_->anb;
}
/* and_d1 bitvector.cpp:2753-2805 (this uncompressed, rhs compressed) */
static void and_d1(wo_bv *b, wo_bv *r) {
    if (r->n == 1) {
        uint32_t w = r->v[0];
        if (w < HEADER1) {
            if (w > ALLONES) { memset(b->v, 0, (size_t)b->n * 4); b->nset = 0; }
            else { b->v[0] = w & r->v[0]; b->nset = cnt_ones(b->v[0]); }
        }
    } else if (r->n > 1) {
        uint32_t i0 = 0;
        b->nset = 0;
        for (uint32_t i1 = 0; i1 < r->n; ++i1) {
            uint32_t w = r->v[i1];
            if (w > ALLONES) {
                uint32_t s0 = w & MAXCNT;
                if (w < HEADER1) memset(b->v + i0, 0, (size_t)s0 * 4);
                i0 += s0;
            } else { b->v[i0] &= w; ++i0; }
        }
    }
    b->aval &= r->aval;
}
/* and_c0 bitvector.cpp:2808-2830 */
static void and_c0(wo_bv *b, wo_bv *r) {
    b->nset = 0;
    for (uint32_t i = 0; i < b->n; ++i) b->v[i] &= r->v[i];
    b->aval &= r->aval;
}

/* ------------------------------------------------------------- OR kernels */
/* or_c2 bitvector.cpp:2833-2978 */
static void or_c2(wo_bv *x_, wo_bv *y_, wo_bv *res) {
    bv_clear(res);
    if (x_->n == 1) {
        uint32_t w = x_->v[0];
        if (w > HEADER1) { vcopy_words(res, x_); res->nbits = x_->nbits; res->nset = x_->nbits; }
        else if (w > ALLONES) { vcopy_words(res, y_); res->nbits = y_->nbits; res->nset = y_->nset; }
        else { vpush(res, w | y_->v[0]); res->nbits = x_->nbits; }
    } else if (y_->n == 1) {
        uint32_t w = y_->v[0];
        if (w > HEADER1) { vcopy_words(res, y_); res->nbits = y_->nbits; res->nset = y_->nbits; }
        else if (w > ALLONES) { vcopy_words(res, x_); res->nbits = x_->nbits; res->nset = x_->nset; }
        else { vpush(res, w | x_->v[0]); res->nbits = x_->nbits; }
    } else if (x_->n > 1) {
        run_t x = {0, 0, 0, 0, x_->v}, y = {0, 0, 0, 0, y_->v};
        while (x.it < x_->n) {
            if (x.nWords == 0) rdecode(&x);
            if (y.nWords == 0) rdecode(&y);
            if (x.isFill) {
                if (y.isFill) {
                    if (y.fillBit != 0) { append_counter(res, y.fillBit, y.nWords); rsub(&x, y.nWords); y.nWords = 0; ++y.it; }
                    else if (y.nWords < x.nWords) { append_counter(res, x.fillBit, y.nWords); x.nWords -= y.nWords; y.nWords = 0; ++y.it; }
                    else { copy_runs(res, &x, &y.nWords); y.it += (y.nWords == 0); }
                } else if (x.fillBit) { append_counter(res, x.fillBit, x.nWords); rsub(&y, x.nWords); x.nWords = 0; ++x.it; }
                else { copy_runs(res, &y, &x.nWords); x.it += (x.nWords == 0); }
            } else if (y.isFill) {
                if (y.fillBit) { append_counter(res, y.fillBit, y.nWords); rsub(&x, y.nWords); y.nWords = 0; ++y.it; }
                else { copy_runs(res, &x, &y.nWords); y.it += (y.nWords == 0); }
            } else {
                res->aval = x_->v[x.it] | y_->v[y.it]; append_active(res);
                x.nWords = 0; y.nWords = 0; ++x.it; ++y.it;
            }
        }
    }
    res->aval = x_->aval | y_->aval; res->anb = x_->anb;
}
/* or_c1 bitvector.cpp:2981-3050 */
static void or_c1(wo_bv *x_, wo_bv *y_, wo_bv *res) {
    bv_clear(res);
    if (x_->n == 1) {
        uint32_t w = x_->v[0];
        if (w > HEADER1) { vcopy_words(res, x_); res->nbits = x_->nbits; res->nset = x_->nbits; }
        else if (w > ALLONES) { vcopy_words(res, y_); res->nbits = y_->nbits; res->nset = y_->nset; }
        else { vpush(res, w | y_->v[0]); res->nbits = x_->nbits; }
    } else if (x_->n > 1) {
        uint32_t i1 = 0;
        for (uint32_t i0 = 0; i0 < x_->n; ++i0) {
            uint32_t w = x_->v[i0];
            if (w > ALLONES) {
                uint32_t s0 = w & MAXCNT;
                if (w >= HEADER1) {
                    if (s0 > 1) append_counter(res, 1, s0);
                    else { res->aval = ALLONES; append_active(res); }
                    i1 += s0;
                } else { for (uint32_t k = 0; k < s0; ++k) vpush(res, y_->v[i1++]); res->nbits += s0 * MAXBITS; }
            } else { res->aval = w | y_->v[i1]; append_active(res); i1++; }
        }
    }
    res->aval = x_->aval | y_->aval; res->anb = x_->anb;
}
/* or_d2 bitvector.cpp:3053-3181 */
static void or_d2(wo_bv *x_, wo_bv *y_, wo_bv *res) {
    res->nbits = d2_nbits(x_, y_);
    vresize(res, res->nbits / MAXBITS);
    if (x_->n == 1) {
        uint32_t w = x_->v[0];
        if (w > HEADER1) { decompress_to(x_, res); res->nset = x_->nbits; }
        else if (w > ALLONES) { decompress_to(y_, res); res->nset = y_->nset; }
        else { res->v[0] = w | y_->v[0]; res->nset = cnt_ones(res->v[0]); }
    } else if (y_->n == 1) {
        uint32_t w = y_->v[0];
        if (w > HEADER1) { decompress_to(y_, res); res->nset = y_->nbits; }
        else if (w > ALLONES) { decompress_to(x_, res); res->nset = x_->nset; }
        else { res->v[0] = w | x_->v[0]; res->nset = cnt_ones(res->v[0]); }
    } else if (x_->n > 1) {
        run_t x = {0, 0, 0, 0, x_->v}, y = {0, 0, 0, 0, y_->v};
        res->nset = 0;
        uint32_t *ir = res->v;
        while (x.it < x_->n) {
            if (x.nWords == 0) rdecode(&x);
            if (y.nWords == 0) rdecode(&y);
            if (x.isFill) {
                if (y.isFill && y.nWords >= x.nWords) {
                    if (y.fillBit == 0) { copy_runs_d(&ir, &x, &y.nWords); y.it += (y.nWords == 0); }
                    else { rsub(&x, y.nWords); copy_fill_d(&ir, &y); }
                } else if (x.fillBit == 0) { copy_runs_d(&ir, &y, &x.nWords); x.it += (x.nWords == 0); }
                else { rsub(&y, x.nWords); copy_fill_d(&ir, &x); }
            } else if (y.isFill) {
                if (y.fillBit == 0) { copy_runs_d(&ir, &x, &y.nWords); y.it += (y.nWords == 0); }
                else { rsub(&x, y.nWords); copy_fill_d(&ir, &y); }
            } else { *ir++ = x_->v[x.it] | y_->v[y.it]; x.nWords = 0; y.nWords = 0; ++x.it; ++y.it; }
        }
    }
    res->aval = x_->aval | y_->aval; res->anb = x_->anb;
}
/* or_d1 bitvector.cpp:3185-3240 */
static void or_d1(wo_bv *b, wo_bv *r) {
    if (r->n == 1) {
        uint32_t w = r->v[0];
        if (w > HEADER1) { decompress_to(r, b); b->nset = b->nbits; }
        else if (w <= ALLONES) { b->v[0] = w | r->v[0]; b->nset = cnt_ones(b->v[0]); }
    } else if (r->n > 1) {
        uint32_t i0 = 0;
        b->nset = 0;
        for (uint32_t i1 = 0; i1 < r->n; ++i1) {
            uint32_t w = r->v[i1];
            if (w > ALLONES) {
                uint32_t s0 = w & MAXCNT;
                if (w >= HEADER1) { for (uint32_t k = 0; k < s0; ++k) b->v[i0 + k] = ALLONES; }
                i0 += s0;
            } else { b->v[i0] |= w; ++i0; }
        }
    }
    b->aval |= r->aval;
}
/* or_c0 bitvector.cpp:3243-3278 */
static void or_c0(wo_bv *b, wo_bv *r) {
    b->nset = 0;
    for (uint32_t i = 0; i < b->n; ++i) b->v[i] |= r->v[i];
    b->aval |= r->aval;
}

/* ------------------------------------------------------------ XOR kernels */
/* xor_c2 bitvector.cpp:3281-3351 */
static void xor_c2(wo_bv *x_, wo_bv *y_, wo_bv *res) {
    run_t x = {0, 0, 0, 0, x_->v}, y = {0, 0, 0, 0, y_->v};
    bv_clear(res);
    while (x.it < x_->n) {
        if (x.nWords == 0) rdecode(&x);
        if (y.nWords == 0) rdecode(&y);
        if (x.isFill) {
            if (y.isFill && y.nWords >= x.nWords) {
                if (y.fillBit == 0) copy_runs(res, &x, &y.nWords); else copy_runsn(res, &x, &y.nWords);
                y.it += (y.nWords == 0);
            } else if (x.fillBit == 0) { copy_runs(res, &y, &x.nWords); x.it += (x.nWords == 0); }
            else { copy_runsn(res, &y, &x.nWords); x.it += (x.nWords == 0); }
        } else if (y.isFill) {
            if (y.fillBit == 0) copy_runs(res, &x, &y.nWords); else copy_runsn(res, &x, &y.nWords);
            y.it += (y.nWords == 0);
        } else {
            res->aval = x_->v[x.it] ^ y_->v[y.it]; append_active(res);
            x.nWords = 0; y.nWords = 0; ++x.it; ++y.it;
        }
    }
    res->aval = x_->aval ^ y_->aval; res->anb = x_->anb;
}
/* xor_c1 bitvector.cpp:3354-3398 */
static void xor_c1(wo_bv *x_, wo_bv *y_, wo_bv *res) {
    uint32_t i1 = 0;
    bv_clear(res);
    for (uint32_t i0 = 0; i0 < x_->n; ++i0) {
        uint32_t w = x_->v[i0];
        if (w > ALLONES) {
            uint32_t s0 = w & MAXCNT;
            res->nbits += s0 * MAXBITS;
            if (w >= HEADER1) { for (uint32_t k = 0; k < s0; ++k) vpush(res, y_->v[i1++] ^ ALLONES); }
            else { for (uint32_t k = 0; k < s0; ++k) vpush(res, y_->v[i1++]); }
        } else { res->aval = w ^ y_->v[i1]; append_active(res); i1++; }
    }
    res->aval = x_->aval ^ y_->aval; res->anb = x_->anb;
}
/* xor_d2 bitvector.cpp:3401-3523 */
static void xor_d2(wo_bv *x_, wo_bv *y_, wo_bv *res) {
    res->nbits = d2_nbits(x_, y_);
    vresize(res, res->nbits / MAXBITS);
    if (x_->n == 1) {
        uint32_t w = x_->v[0];
        if (w > HEADER1) { copy_comp(y_, res); if (y_->nset > 0) res->nset = x_->nbits - y_->nset; }
        else if (w > ALLONES) { decompress_to(y_, res); res->nset = y_->nset; }
        else { res->v[0] = w ^ y_->v[0]; res->nset = cnt_ones(res->v[0]); }
    } else if (y_->n == 1) {
        uint32_t w = y_->v[0];
        if (w > HEADER1) { copy_comp(x_, res); if (x_->nset > 0) res->nset = x_->nbits - x_->nset; }
        else if (w > ALLONES) { decompress_to(x_, res); res->nset = x_->nset; }
        else { res->v[0] = w ^ x_->v[0]; res->nset = cnt_ones(res->v[0]); }
    } else if (x_->n > 1) {
        run_t x = {0, 0, 0, 0, x_->v}, y = {0, 0, 0, 0, y_->v};
        res->nset = 0;
        uint32_t *ir = res->v;
        while (x.it < x_->n) {
            if (x.nWords == 0) rdecode(&x);
            if (y.nWords == 0) rdecode(&y);
            if (x.isFill) {
                if (y.isFill && y.nWords >= x.nWords) {
                    if (y.fillBit == 0) copy_runs_d(&ir, &x, &y.nWords); else copy_runsn_d(&ir, &x, &y.nWords);
                    y.it += (y.nWords == 0);
                } else {
                    if (x.fillBit == 0) copy_runs_d(&ir, &y, &x.nWords); else copy_runsn_d(&ir, &y, &x.nWords);
                    x.it += (x.nWords == 0);
                }
            } else if (y.isFill) {
                if (y.fillBit == 0) copy_runs_d(&ir, &x, &y.nWords); else copy_runsn_d(&ir, &x, &y.nWords);
                y.it += (y.nWords == 0);
            } else { *ir++ = x_->v[x.it] ^ y_->v[y.it]; x.nWords = 0; y.nWords = 0; ++x.it; ++y.it; }
        }
    }
    res->aval = x_->aval ^ y_->aval; res->anb = x_->anb;
}
/* xor_d1 bitvector.cpp:3527-3584 */
static void xor_d1(wo_bv *b, wo_bv *r) {
    if (r->n == 1) {
        uint32_t w = r->v[0];
        if (w > HEADER1) {
            for (uint32_t i = 0; i < b->n; ++i) b->v[i] ^= (b->v[i] > ALLONES) ? FILLBIT : ALLONES;
            if (b->nset > 0) b->nset = b->nbits - b->nset;
        } else if (w <= ALLONES) { b->v[0] = w ^ r->v[0]; b->nset = cnt_ones(b->v[0]); }
    } else if (r->n > 1) {
        b->nset = 0;
        uint32_t i0 = 0;
        for (uint32_t i1 = 0; i1 < r->n; ++i1) {
            uint32_t w = r->v[i1];
            if (w > ALLONES) {
                uint32_t s0 = w & MAXCNT;
                if (w >= HEADER1) { for (uint32_t k = 0; k < s0; ++k) b->v[i0 + k] ^= ALLONES; }
                i0 += s0;
            } else { b->v[i0] ^= w; ++i0; }
        }
    }
    b->aval ^= r->aval;
}
/* xor_c0 bitvector.cpp:3587-3619 */
static void xor_c0(wo_bv *b, wo_bv *r) {
    b->nset = 0;
    for (uint32_t i = 0; i < b->n; ++i) b->v[i] ^= r->v[i];
    b->aval ^= r->aval;
}

/* ---------------------------------------------------------- MINUS kernels */
/* minus_c2 bitvector.cpp:3622-3745 */
static void minus_c2(wo_bv *x_, wo_bv *y_, wo_bv *res) {
    bv_clear(res);
    if (x_->n == 1) {
        uint32_t w = x_->v[0];
        if (w > HEADER1) {
            vresize(res, y_->n);
            for (uint32_t i = 0; i < y_->n; ++i) res->v[i] = y_->v[i] ^ ((y_->v[i] > ALLONES) ? FILLBIT : ALLONES);
            res->nbits = y_->nbits;
            if (y_->nset > 0) res->nset = y_->nbits - y_->nset;
        } else if (w > ALLONES) { vcopy_words(res, x_); res->nbits = x_->nbits; res->nset = 0; }
        else { vpush(res, w & ~y_->v[0]); res->nbits = x_->nbits; }
    } else if (y_->n == 1) {
        uint32_t w = y_->v[0];
        if (w > HEADER1) wo_append_fill(res, 0, y_->nbits);
        else if (w > ALLONES) { vcopy_words(res, x_); res->nbits = x_->nbits; res->nset = x_->nset; }
        else { vpush(res, w & x_->v[0]); res->nbits = x_->nbits; }
    } else if (x_->n > 1) {
        run_t x = {0, 0, 0, 0, x_->v}, y = {0, 0, 0, 0, y_->v};
        while (x.it < x_->n) {
            if (x.nWords == 0) rdecode(&x);
            if (y.nWords == 0) rdecode(&y);
            if (x.isFill) {
                if (y.isFill && y.nWords >= x.nWords) {
                    if (y.fillBit == 0) { copy_runs(res, &x, &y.nWords); y.it += (y.nWords == 0); }
                    else { append_counter(res, 0, y.nWords); rsub(&x, y.nWords); y.nWords = 0; ++y.it; }
                } else if (x.fillBit == 0) { append_counter(res, 0, x.nWords); rsub(&y, x.nWords); x.nWords = 0; ++x.it; }
                else { copy_runsn(res, &y, &x.nWords); x.it += (x.nWords == 0); }
            } else if (y.isFill) {
                if (y.fillBit == 0) { copy_runs(res, &x, &y.nWords); y.it += (y.nWords == 0); }
                else { append_counter(res, 0, y.nWords); rsub(&x, y.nWords); y.nWords = 0; ++y.it; }
            } else {
                res->aval = x_->v[x.it] & ~y_->v[y.it]; append_active(res);
                x.nWords = 0; y.nWords = 0; ++x.it; ++y.it;
            }
        }
    }
    res->aval = x_->aval & ~y_->aval; res->anb = x_->anb;
}
/* minus_c1 bitvector.cpp:3748-3818 (rhs uncompressed) */
static void minus_c1(wo_bv *x_, wo_bv *y_, wo_bv *res) {
    bv_clear(res);
    if (x_->n == 1) {
        uint32_t w = x_->v[0];
        if (w > HEADER1) {
            vresize(res, y_->n);
            for (uint32_t i = 0; i < y_->n; ++i) res->v[i] = y_->v[i] ^ ALLONES;
            res->nbits = y_->nbits;
            if (y_->nset > 0) res->nset = y_->nbits - y_->nset;
        } else if (w > ALLONES) { vcopy_words(res, x_); res->nbits = x_->nbits; res->nset = 0; }
        else { vpush(res, w & ~y_->v[0]); res->nbits = x_->nbits; }
    } else if (x_->n > 1) {
        uint32_t i1 = 0;
        bv_clear(res);
        for (uint32_t i0 = 0; i0 < x_->n; ++i0) {
            uint32_t w = x_->v[i0];
            if (w > ALLONES) {
                uint32_t s0 = w & MAXCNT;
                if (w >= HEADER1) { for (uint32_t k = 0; k < s0; ++k) vpush(res, y_->v[i1++] ^ ALLONES); res->nbits += s0 * MAXBITS; }
                else { i1 += s0; if (s0 > 1) append_counter(res, 0, s0); else append_active(res); }
            } else { res->aval = w & ~y_->v[i1]; append_active(res); i1++; }
        }
    }
    res->aval = x_->aval & ~y_->aval; res->anb = x_->anb;
}
/* minus_c1x bitvector.cpp:3821-3869 (this uncompressed) */
static void minus_c1x(wo_bv *x_, wo_bv *y_, wo_bv *res) {
    uint32_t i0 = 0;
    bv_clear(res);
    for (uint32_t i1 = 0; i1 < y_->n; ++i1) {
        uint32_t w = y_->v[i1];
        if (w > ALLONES) {
            uint32_t s0 = w & MAXCNT;
            if (w >= HEADER1) { i0 += s0; if (s0 > 1) append_counter(res, 0, s0); else append_active(res); }
            else { for (uint32_t k = 0; k < s0; ++k) vpush(res, x_->v[i0++]); res->nbits += s0 * MAXBITS; }
        } else { res->aval = x_->v[i0] & ~w; append_active(res); i0++; }
    }
    res->aval = x_->aval & ~y_->aval; res->anb = x_->anb;
}
/* minus_d2 bitvector.cpp:3872-3998 */
static void minus_d2(wo_bv *x_, wo_bv *y_, wo_bv *res) {
    res->nbits = d2_nbits(x_, y_);
    vresize(res, res->nbits / MAXBITS);
    if (x_->n == 1) {
        uint32_t w = x_->v[0];
        if (w > HEADER1) { copy_comp(y_, res); if (y_->nset > 0) res->nset = x_->nbits - y_->nset; }
        else if (w > ALLONES) { decompress_to(x_, res); res->nset = 0; }
        else { res->v[0] = w & ~y_->v[0]; res->nset = cnt_ones(res->v[0]); }
    } else if (y_->n == 1) {
        uint32_t w = y_->v[0];
        if (w > HEADER1) { memset(res->v, 0, (size_t)res->n * 4); res->nset = 0; }
        else if (w > ALLONES) { vcopy_words(res, x_); res->nset = x_->nset; }
        else { res->v[0] = w & ~x_->v[0]; res->nset = cnt_ones(res->v[0]); }
    } else if (x_->n > 1) {
        run_t x = {0, 0, 0, 0, x_->v}, y = {0, 0, 0, 0, y_->v};
        res->nset = 0;
        uint32_t *ir = res->v;
        while (x.it < x_->n) {
            if (x.nWords == 0) rdecode(&x);
            if (y.nWords == 0) rdecode(&y);
            if (x.isFill) {
                if (y.isFill && y.nWords >= x.nWords) {
                    if (y.fillBit == 0) { copy_runs_d(&ir, &x, &y.nWords); y.it += (y.nWords == 0); }
                    else { rsub(&x, y.nWords); y.fillBit = 0; copy_fill_d(&ir, &y); }
                } else if (x.fillBit == 0) { rsub(&y, x.nWords); copy_fill_d(&ir, &x); }
                else { copy_runsn_d(&ir, &y, &x.nWords); x.it += (x.nWords == 0); }
            } else if (y.isFill) {
                if (y.fillBit == 0) { copy_runs_d(&ir, &x, &y.nWords); y.it += (y.nWords == 0); }
                else { rsub(&x, y.nWords); y.fillBit = 0; copy_fill_d(&ir, &y); }
            } else { *ir++ = x_->v[x.it] & ~y_->v[y.it]; x.nWords = 0; y.nWords = 0; ++x.it; ++y.it; }
        }
    }
    res->aval = x_->aval & ~y_->aval; res->anb = x_->anb;
}
/* minus_d1 bitvector.cpp:4002-4050 */
static void minus_d1(wo_bv *b, wo_bv *r) {
    if (r->n == 1) {
        uint32_t w = r->v[0];
        if (w > HEADER1) { memset(b->v, 0, (size_t)b->n * 4); b->nset = 0; }
        else if (w <= ALLONES) { b->v[0] = w & ~r->v[0]; b->nset = cnt_ones(b->v[0]); }
    } else if (r->n > 1) {
        b->nset = 0;
        uint32_t i0 = 0;
        for (uint32_t i1 = 0; i1 < r->n; ++i1) {
            uint32_t w = r->v[i1];
            if (w > ALLONES) {
                uint32_t s0 = w & MAXCNT;
                if (w >= HEADER1) memset(b->v + i0, 0, (size_t)s0 * 4);
                i0 += s0;
            } else { b->v[i0] &= ~w; ++i0; }
        }
    }
    b->aval &= ~r->aval;
}
/* minus_c0 bitvector.cpp:4053-4079 */
static void minus_c0(wo_bv *b, wo_bv *r) {
    b->nset = 0;
    for (uint32_t i = 0; i < b->n; ++i) b->v[i] &= ~r->v[i];
    b->aval &= ~r->aval;
}

/* ------------------------------------------------------------ dispatchers */
static int uncomp(const wo_bv *b) { return (uint64_t)b->n * MAXBITS == b->nbits && b->nbits > 0; }
static void active_and(wo_bv *a, const wo_bv *r) { /* shared tail of &= */
    if (a->anb == r->anb) a->aval &= r->aval;
    else if (a->anb > r->anb) a->aval &= (r->aval << (a->anb - r->anb));
    else { a->aval = (a->aval << (r->anb - a->anb)) & r->aval; a->anb = r->anb; }
}

/* operator&= bitvector.cpp:1194-1284 */
static void op_and_eq(wo_bv *a, wo_bv *r) {
    if (wo_size(a) > wo_size(r)) {
        wo_bv tmp; wo_init(&tmp); wo_copy(&tmp, r);
        wo_adjust_size(&tmp, 0, wo_size(a));
        op_and_eq(a, &tmp); wo_free(&tmp); return;
    } else if (wo_size(a) < wo_size(r)) wo_adjust_size(a, 0, wo_size(r));
    int ca = uncomp(a), cb = uncomp(r);
    if (ca) { if (cb) and_c0(a, r); else and_d1(a, r); }
    else if (cb) { wo_bv tmp; wo_init(&tmp); wo_copy(&tmp, r); bv_swap(a, &tmp); and_d1(a, &tmp); wo_free(&tmp); }
    else if (all0s(a) || all1s(r)) active_and(a, r);
    else if (all0s(r) || all1s(a)) { a->nset = r->nset; vcopy_words(a, r); active_and(a, r); }
    else if ((uint64_t)(a->n + (uint64_t)r->n) * MAXBITS >= r->nbits) { wo_bv res; wo_init(&res); and_d2(a, r, &res); bv_swap(a, &res); wo_free(&res); }
    else { wo_bv res; wo_init(&res); and_c2(a, r, &res); bv_swap(a, &res); wo_free(&res); }
}
/* operator& bitvector.cpp:1292-1407 */
static void op_and(wo_bv *a, wo_bv *r, wo_bv *res) {
    bv_clear(res);
    if (wo_size(a) > wo_size(r)) { wo_copy(res, r); wo_adjust_size(res, 0, wo_size(a)); op_and_eq(res, a); return; }
    else if (wo_size(a) < wo_size(r)) { wo_copy(res, a); wo_adjust_size(res, 0, wo_size(r)); op_and_eq(res, r); return; }
    int ca = uncomp(a), cb = uncomp(r);
    if (ca && cb) {
        uint32_t nw = a->n >= r->n ? a->n : r->n;
        vresize(res, nw);
        if (a->n == r->n) {
            for (uint32_t i = 0; i < nw; ++i) res->v[i] = a->v[i] & r->v[i];
            res->nbits = a->nbits;
            if (a->anb == r->anb) { res->aval = a->aval & r->aval; res->anb = a->anb; }
            else if (a->anb > r->anb) { res->aval = a->aval & (r->aval << (a->anb - r->anb)); res->anb = a->anb; }
            else { res->aval = r->aval & (a->aval << (r->anb - a->anb)); res->anb = r->anb; }
        } else if (a->n > r->n) {
            uint32_t j = 0;
            for (; j < r->n; ++j) res->v[j] = a->v[j] & r->v[j];
            if (r->anb > 0) { res->v[j] = a->v[j] & (r->aval << (MAXBITS - r->anb)); ++j; }
            for (; j < nw; ++j) res->v[j] = 0;
            res->anb = a->anb; res->aval = 0;
        } else {
            uint32_t j = 0;
            for (; j < a->n; ++j) res->v[j] = a->v[j] & r->v[j];
            if (a->anb > 0) { res->v[j] = (a->aval << (MAXBITS - a->anb)) & r->v[j]; ++j; }
            for (; j < nw; ++j) res->v[j] = 0;
            res->anb = r->anb; res->aval = 0;
        }
    }
    else if (ca) and_c1(r, a, res);
    else if (cb) and_c1(a, r, res);
    else if (all0s(a) || all1s(r)) { wo_copy(res, a); res->aval &= r->aval; }
    else if (all1s(a) || all0s(r)) { wo_copy(res, r); res->aval &= a->aval; }
    else if ((uint64_t)(a->n + (uint64_t)r->n) * MAXBITS > a->nbits) and_d2(a, r, res);
    else and_c2(a, r, res);
}
/* operator|= bitvector.cpp:1413-1483 */
static void op_or_eq(wo_bv *a, wo_bv *r) {
    if (wo_size(a) > wo_size(r)) {
        wo_bv tmp; wo_init(&tmp); wo_copy(&tmp, r);
        wo_adjust_size(&tmp, 0, wo_size(a));
        op_or_eq(a, &tmp); wo_free(&tmp); return;
    } else if (wo_size(a) < wo_size(r)) wo_adjust_size(a, 0, wo_size(r));
    int ca = uncomp(a), cb = uncomp(r);
    if (ca) { if (cb) or_c0(a, r); else or_d1(a, r); }
    else if (cb) { wo_bv tmp; wo_init(&tmp); wo_copy(&tmp, r); bv_swap(a, &tmp); or_d1(a, &tmp); wo_free(&tmp); }
    else if (all1s(a) || all0s(r)) a->aval |= r->aval;
    else if (all0s(a) || all1s(r)) { a->nset = r->nset; vcopy_words(a, r); a->aval |= r->aval; }
    else if ((uint64_t)(a->n + (uint64_t)r->n) * MAXBITS >= r->nbits) { wo_bv res; wo_init(&res); or_d2(a, r, &res); bv_swap(a, &res); wo_free(&res); }
    else { wo_bv res; wo_init(&res); or_c2(a, r, &res); bv_swap(a, &res); wo_free(&res); }
}
/* operator| bitvector.cpp:1488-1551 */
static void op_or(wo_bv *a, wo_bv *r, wo_bv *res) {
    bv_clear(res);
    if (wo_size(a) > wo_size(r)) { wo_copy(res, r); wo_adjust_size(res, 0, wo_size(a)); op_or_eq(res, a); return; }
    else if (wo_size(a) < wo_size(r)) { wo_copy(res, a); wo_adjust_size(res, 0, wo_size(r)); op_or_eq(res, r); return; }
    int ca = uncomp(a), cb = uncomp(r);
    if (ca && cb) {
        vresize(res, a->n);
        for (uint32_t i = 0; i < a->n; ++i) res->v[i] = a->v[i] | r->v[i];
        res->aval = a->aval | r->aval; res->anb = a->anb; res->nbits = a->nbits;
    }
    else if (ca) or_c1(r, a, res);
    else if (cb) or_c1(a, r, res);
    else if (all1s(a) || all0s(r)) { wo_copy(res, a); res->aval |= r->aval; }
    else if (all0s(a) || all1s(r)) { wo_copy(res, r); res->aval |= a->aval; }
    else if ((uint64_t)(a->n + (uint64_t)r->n) * MAXBITS > a->nbits) or_d2(a, r, res);
    else or_c2(a, r, res);
}
/* operator^= bitvector.cpp:1557-1619 */
static void op_xor_eq(wo_bv *a, wo_bv *r) {
    if (wo_size(a) > wo_size(r)) {
        wo_bv tmp; wo_init(&tmp); wo_copy(&tmp, r);
        wo_adjust_size(&tmp, 0, wo_size(a));
        op_xor_eq(a, &tmp); wo_free(&tmp); return;
    } else if (wo_size(a) < wo_size(r)) wo_adjust_size(a, 0, wo_size(r));
    int ca = uncomp(a), cb = uncomp(r);
    if (ca) { if (cb) xor_c0(a, r); else xor_d1(a, r); }
    else if (cb) { wo_bv res; wo_init(&res); xor_c1(a, r, &res); bv_swap(a, &res); wo_free(&res); }
    else if ((uint64_t)(a->n + (uint64_t)r->n) * MAXBITS >= r->nbits) { wo_bv res; wo_init(&res); xor_d2(a, r, &res); bv_swap(a, &res); wo_free(&res); }
    else { wo_bv res; wo_init(&res); xor_c2(a, r, &res); bv_swap(a, &res); wo_free(&res); }
}
/* operator^ bitvector.cpp:1624-1679 */
static void op_xor(wo_bv *a, wo_bv *r, wo_bv *res) {
    bv_clear(res);
    if (wo_size(a) > wo_size(r)) { wo_copy(res, r); wo_adjust_size(res, 0, wo_size(a)); op_xor_eq(res, a); return; }
    else if (wo_size(a) < wo_size(r)) { wo_copy(res, a); wo_adjust_size(res, 0, wo_size(r)); op_xor_eq(res, r); return; }
    int ca = uncomp(a), cb = uncomp(r);
    if (ca && cb) {
        vresize(res, a->n);
        for (uint32_t i = 0; i < a->n; ++i) res->v[i] = a->v[i] ^ r->v[i];
        res->aval = a->aval ^ r->aval; res->anb = a->anb; res->nbits = a->nbits;
    }
    else if (ca) xor_c1(r, a, res);
    else if (cb) xor_c1(a, r, res);
    else if ((uint64_t)(a->n + (uint64_t)r->n) * MAXBITS > a->nbits) xor_d2(a, r, res);
    else xor_c2(a, r, res);
}
/* operator-= bitvector.cpp:1685-1763 */
static void op_minus_eq(wo_bv *a, wo_bv *r) {
    if (wo_size(a) > wo_size(r)) {
        wo_bv tmp; wo_init(&tmp); wo_copy(&tmp, r);
        wo_adjust_size(&tmp, 0, wo_size(a));
        op_minus_eq(a, &tmp); wo_free(&tmp); return;
    } else if (wo_size(a) < wo_size(r)) wo_adjust_size(a, 0, wo_size(r));
    int ca = uncomp(a), cb = uncomp(r);
    if (ca) { if (cb) minus_c0(a, r); else minus_d1(a, r); }
    else if (cb) { wo_bv res; wo_init(&res); minus_c1(a, r, &res); bv_swap(a, &res); wo_free(&res); }
    else if (all0s(a) || all0s(r)) a->aval &= ~r->aval;
    else if (all1s(r)) {
        a->nset = 0; a->nbits = 0; a->n = 0;
        a->aval &= ~r->aval;
        append_counter(a, 0, r->v[0] & MAXCNT);
    }
    else if (all1s(a)) { uint32_t t = a->aval; wo_copy(a, r); wo_flip(a); a->aval &= t; }
    else if ((uint64_t)(a->n + (uint64_t)r->n) * MAXBITS >= r->nbits) { wo_bv res; wo_init(&res); minus_d2(a, r, &res); bv_swap(a, &res); wo_free(&res); }
    else { wo_bv res; wo_init(&res); minus_c2(a, r, &res); bv_swap(a, &res); wo_free(&res); }
}
/* operator- bitvector.cpp:1768-1838 */
static void op_minus(wo_bv *a, wo_bv *r, wo_bv *res) {
    bv_clear(res);
    if (wo_size(a) > wo_size(r)) {
        wo_bv tmp; wo_init(&tmp); wo_copy(&tmp, r); wo_adjust_size(&tmp, 0, wo_size(a));
        wo_copy(res, a); op_minus_eq(res, &tmp); wo_free(&tmp); return;
    } else if (wo_size(a) < wo_size(r)) { wo_copy(res, a); wo_adjust_size(res, 0, wo_size(r)); op_minus_eq(res, r); return; }
    int ca = ((uint64_t)a->n * MAXBITS == a->nbits), cb = ((uint64_t)r->n * MAXBITS == r->nbits);
    if (ca && cb) {
        vresize(res, a->n);
        for (uint32_t i = 0; i < a->n; ++i) res->v[i] = a->v[i] & ~r->v[i];
        res->aval = a->aval & ~r->aval; res->anb = a->anb; res->nbits = a->nbits;
    }
    else if (ca) minus_c1x(a, r, res);
    else if (cb) minus_c1(a, r, res);
    else if (all0s(a) || all0s(r)) { wo_copy(res, a); res->aval &= ~r->aval; }
    else if (all1s(r)) { append_counter(res, 0, r->v[0] & MAXCNT); res->anb = a->anb; res->aval = a->aval & ~r->aval; }
    else if (all1s(a)) { wo_copy(res, r); wo_flip(res); res->aval &= a->aval; }
    else if ((uint64_t)(a->n + (uint64_t)r->n) * MAXBITS > a->nbits) minus_d2(a, r, res);
    else minus_c2(a, r, res);
}

int wo_binop(int op, wo_bv *a, wo_bv *b, wo_bv *res) {
    switch (op) {
    case WO_AND: op_and(a, b, res); return 0;
    case WO_OR: op_or(a, b, res); return 0;
    case WO_XOR: op_xor(a, b, res); return 0;
    case WO_MINUS: op_minus(a, b, res); return 0;
    }
    return -1;
}
int wo_binop_inplace(int op, wo_bv *a, wo_bv *b) {
    switch (op) {
    case WO_AND: op_and_eq(a, b); return 0;
    case WO_OR: op_or_eq(a, b); return 0;
    case WO_XOR: op_xor_eq(a, b); return 0;
    case WO_MINUS: op_minus_eq(a, b); return 0;
    }
    return -1;
}

/* ---------------------------------------------------------- serialization */
int wo_from_serial(wo_bv *b, const uint32_t *w, uint32_t nw) {
    wo_init(b);
    if (nw > 1) {
        vreserve(b, nw);
        memcpy(b->v, w, (size_t)nw * 4);
        b->n = nw;
        if (b->v[b->n - 1] > 0) {
            if (b->v[b->n - 1] < MAXBITS) {
                b->anb = b->v[b->n - 1];
                b->n--;
                b->aval = b->v[b->n - 1];
            }
        } else { b->aval = 0; b->anb = 0; }
        b->n--;
    }
    return 0;
}
uint32_t wo_serial_size(const wo_bv *b) { return b->n + 1 + (b->anb > 0); }
uint32_t wo_serialize(const wo_bv *b, uint32_t *out, uint32_t cap) {
    uint32_t len = wo_serial_size(b);
    if (len <= cap) {
        if (b->n) memcpy(out, b->v, (size_t)b->n * 4);
        uint32_t k = b->n;
        if (b->anb > 0) out[k++] = b->aval;
        out[k] = b->anb;
    }
    return len;
}

uint64_t wo_rids(const wo_bv *b, uint32_t *out, uint64_t cap) {
    uint64_t k = 0, base = 0;
    for (uint32_t i = 0; i < b->n; ++i) {
        uint32_t w = b->v[i];
        if (w >= HEADER1) {
            uint64_t c = (uint64_t)(w & MAXCNT) * MAXBITS;
            for (uint64_t j = 0; j < c; ++j, ++k) if (k < cap) out[k] = (uint32_t)(base + j);
            base += c;
        } else if (w >= HEADER0) base += (uint64_t)(w & MAXCNT) * MAXBITS;
        else {
            for (int j = 0; j < 31; ++j)
                if (w & (1u << (30 - j))) { if (k < cap) out[k] = (uint32_t)(base + j); ++k; }
            base += MAXBITS;
        }
    }
    for (uint32_t j = 0; j < b->anb; ++j)
        if (b->aval & (1u << (b->anb - 1 - j))) { if (k < cap) out[k] = (uint32_t)(base + j); ++k; }
    return k;
}

/* ----------------------------------------------------- ctypes wrappers */
long wo_ser_binop(int op, int inplace, int do_compress,
                  const uint32_t *a, uint32_t na, const uint32_t *b, uint32_t nb,
                  uint32_t *out, uint32_t cap, uint32_t *cnt) {
    wo_bv A, B, R;
    wo_from_serial(&A, a, na); wo_from_serial(&B, b, nb); wo_init(&R);
    wo_bv *res;
    if (inplace) { if (wo_binop_inplace(op, &A, &B)) return -1; res = &A; }
    else { if (wo_binop(op, &A, &B, &R)) return -1; res = &R; }
    if (do_compress) wo_compress(res);
    long len = (long)wo_serialize(res, out, cap);
    if (cnt) *cnt = wo_cnt(res);
    wo_free(&A); wo_free(&B); wo_free(&R);
    return len;
}
long wo_ser_compress(const uint32_t *a, uint32_t na, uint32_t *out, uint32_t cap, uint32_t *cnt) {
    wo_bv A; wo_from_serial(&A, a, na);
    wo_compress(&A);
    long len = (long)wo_serialize(&A, out, cap);
    if (cnt) *cnt = wo_cnt(&A);
    wo_free(&A);
    return len;
}
long wo_ser_decompress(const uint32_t *a, uint32_t na, uint32_t *out, uint32_t cap) {
    wo_bv A; wo_from_serial(&A, a, na);
    wo_decompress(&A);
    long len = (long)wo_serialize(&A, out, cap);
    wo_free(&A);
    return len;
}
long wo_ser_rids(const uint32_t *a, uint32_t na, uint32_t *out, uint64_t cap) {
    wo_bv A; wo_from_serial(&A, a, na);
    long n = (long)wo_rids(&A, out, cap);
    wo_free(&A);
    return n;
}
long wo_ser_flip(const uint32_t *a, uint32_t na, uint32_t *out, uint32_t cap) {
    wo_bv A; wo_from_serial(&A, a, na);
    wo_flip(&A);
    long len = (long)wo_serialize(&A, out, cap);
    wo_free(&A);
    return len;
}
long wo_build_runs(const uint64_t *runs, uint64_t nruns, uint32_t *out, uint32_t cap) {
    wo_bv A; wo_init(&A);
    for (uint64_t i = 0; i < nruns; ++i) wo_append_fill(&A, (int)(i & 1), (uint32_t)runs[i]);
    long len = (long)wo_serialize(&A, out, cap);
    wo_free(&A);
    return len;
}
