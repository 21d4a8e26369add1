/*
 * CPU oracle for the WAH bitvector hot path — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's 32-bit Word-Aligned-Hybrid
 * ibis::bitvector (src/bitvector.{h,cpp}) and of the range evaluation that
 * feeds it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it, and only as the checker or the timed CPU
 * baseline.  The product (libwahgpu) never links or calls it.
 *
 * Parity of this restatement is pinned against the reference library itself
 * (compiled from source by oracle/Makefile.ref) through the golden fixtures
 * in tests/golden/, made by tests/golden/make_golden.py.
 */
#ifndef WAH_ORACLE_H
#define WAH_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One bitvector: the reference's members nbits, nset, active, m_vec
 * (bitvector.h:266-269). nbits==0 means "not yet counted" exactly as in the
 * reference, whose size() computes it lazily (bitvector.h:647). */
typedef struct {
    uint32_t *v;
    uint32_t n, cap;
    uint32_t nbits;
    uint32_t nset;
    uint32_t aval, anb;
} wo_bv;

enum { WO_AND = 0, WO_OR = 1, WO_XOR = 2, WO_MINUS = 3 };

/* life cycle */
void wo_init(wo_bv *b);
void wo_free(wo_bv *b);
void wo_copy(wo_bv *dst, const wo_bv *src);
/* ctor from a serialized array (bitvector.cpp:54-105); returns 0 */
int  wo_from_serial(wo_bv *b, const uint32_t *w, uint32_t nw);
/* write(array_t&) (bitvector.cpp:2283-2313): returns serialized length,
 * writes min(len, cap) words into out */
uint32_t wo_serial_size(const wo_bv *b);
uint32_t wo_serialize(const wo_bv *b, uint32_t *out, uint32_t cap);

/* bitvector API */
uint32_t wo_size(wo_bv *b);                  /* size()  */
uint32_t wo_cnt(wo_bv *b);                   /* cnt()   */
void wo_compress(wo_bv *b);                  /* compress() */
void wo_decompress(wo_bv *b);                /* decompress() */
void wo_flip(wo_bv *b);                      /* flip() */
void wo_set(wo_bv *b, int val, uint32_t n);  /* set(val, n) */
void wo_append_fill(wo_bv *b, int val, uint32_t n); /* appendFill */
void wo_adjust_size(wo_bv *b, uint32_t nv, uint32_t nt);
void wo_set_bit(wo_bv *b, uint32_t ind, int val); /* setBit (append case) */

/* r = a OP b (operator& | ^ -, returns new bitvector) */
int  wo_binop(int op, wo_bv *a, wo_bv *b, wo_bv *res);
/* a OP= b */
int  wo_binop_inplace(int op, wo_bv *a, wo_bv *b);

/* ascending row ids of the 1 bits (indexSet walk, bitvector.cpp:4524) ;
 * returns the number of ids, writes at most cap */
uint64_t wo_rids(const wo_bv *b, uint32_t *out, uint64_t cap);

/* Convenience wrappers over serialized arrays, used through ctypes.
 * They return the serialized length of the result (or a negative error) and
 * write up to cap words; *cnt receives cnt() of the result. */
long wo_ser_binop(int op, int inplace, int do_compress,
                  const uint32_t *a, uint32_t na,
                  const uint32_t *b, uint32_t nb,
                  uint32_t *out, uint32_t cap, uint32_t *cnt);
long wo_ser_compress(const uint32_t *a, uint32_t na, uint32_t *out,
                     uint32_t cap, uint32_t *cnt);
long wo_ser_decompress(const uint32_t *a, uint32_t na, uint32_t *out,
                       uint32_t cap);
long wo_ser_rids(const uint32_t *a, uint32_t na, uint32_t *out, uint64_t cap);
long wo_ser_flip(const uint32_t *a, uint32_t na, uint32_t *out, uint32_t cap);

/* Builds a bitvector of nbits bits from alternating 0/1 runs (first run is
 * 0s) with appendFill, run lengths given in runs[0..nruns).  Serializes it. */
long wo_build_runs(const uint64_t *runs, uint64_t nruns, uint32_t *out,
                   uint32_t cap);

#ifdef __cplusplus
}
#endif
#endif
