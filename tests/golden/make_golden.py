"""Generates the golden fixtures in tests/golden/ by running the REFERENCE
library itself (FastBit built from source by oracle/Makefile.ref, driven by
oracle/refdrv.cpp).  Run it where the reference sources are available:

    python tests/golden/make_golden.py

Outputs (all seeded, compressed .npz):
  binop_random.npz  1500 random operand pairs of every word form the
                    reference can hold, the four operators in both the
                    OP and OP= forms, each followed by compress():
                    reference words and cnt()
  binop_geom.npz    appendFill-built 2^20-bit operands with alternating
                    geometric 0/1 runs at densities 1e-4..0.5 (the raw-WAH
                    workload at reduced length), all ops, both forms
  binop_unequal.npz 400 operand pairs of DIFFERENT sizes (the shorter one is
                    padded by adjustSize inside the reference's operators),
                    some ending in a literal 0, a 0-fill or a 1-fill, the
                    four operators in both forms: reference words and cnt()
  unary.npz         compress(), decompress(), flip() and the indexSet row
                    ids of random bitvectors
  relic_small.npz   relic index over 20000 uint32 values in [0,100) and 40
                    ranges lo <= x < hi: the index triple (keys, offsets,
                    bitmaps) from relic::write and hit counts + row ids from
                    relic::evaluate
  bin_small.npz     bin index (<binning nbins=100 equal_weight/>) over
                    200000 float32 values (70% normal(0,1), 30% Zipf(1.2)
                    ranks) built through the in-memory C API, its triple from
                    fastbit_iapi_deconstruct_index, and 30 ranges
                    lo <= x < hi evaluated by the reference (counts and row
                    ids from get_coordinates)
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import wahgen as G  # noqa: E402


def pack(arrs):
    offs = np.zeros(len(arrs) + 1, dtype=np.int64)
    for i, a in enumerate(arrs):
        offs[i + 1] = offs[i] + len(a)
    flat = np.concatenate([np.asarray(a, dtype=np.uint32) for a in arrs]) if arrs else np.zeros(0, np.uint32)
    return flat, offs


def unpack(flat, offs, i):
    return flat[offs[i]:offs[i + 1]]


def unequal(td):
    """Pairs of different sizes, every operator in both forms."""
    rng = np.random.default_rng(404)
    styles = ["mixed", "short", "sparse", "canon", "dense"]
    A, B, ops, inpl = [], [], [], []
    while len(A) < 400:
        k = len(A)
        wa = G.random_words(rng, int(rng.integers(1, 3000)), styles[k % 5])
        wb = G.random_words(rng, int(rng.integers(1, 3000)), styles[(k + 2) % 5])
        if k % 6 == 1:
            wa = list(wa[:-1]) + [0]
        if k % 6 == 2:
            wb = list(wb) + [G.fill(0, 5)]
        if k % 6 == 3:
            wa = list(wa) + [G.fill(1, 3)]
        a = G.serialize(wa, int(rng.integers(0, 31)), int(rng.integers(0, 1 << 31)))
        b = G.serialize(wb, int(rng.integers(0, 31)), int(rng.integers(0, 1 << 31)))
        if G.groups_of(wa) == G.groups_of(wb) or oracle.is_degenerate(a) or oracle.is_degenerate(b):
            continue
        A.append(a); B.append(b)
        ops.append(int(rng.integers(0, 4))); inpl.append(int(rng.integers(0, 2)))
    R = G.run_refdrv(oracle.REFDRV, [G.req_binop(o, i, 1, a, b) for o, i, a, b in zip(ops, inpl, A, B)], td)
    res, cnt, st = [], [], []
    for _ in A:
        s, c, w = R.bv()
        st.append(s); cnt.append(c); res.append(w)
    fa, oa = pack(A); fb, ob = pack(B); fr, orr = pack(res)
    np.savez_compressed(os.path.join(HERE, "binop_unequal.npz"), a=fa, a_off=oa, b=fb, b_off=ob,
                        res=fr, res_off=orr, cnt=np.array(cnt, np.uint64), status=np.array(st, np.uint32),
                        op=np.array(ops, np.int32), inplace=np.array(inpl, np.int32))


def main():
    if not oracle.build_reference():
        sys.exit("the reference library could not be built (needs the reference sources)")
    td = tempfile.mkdtemp()
    unequal(td)

    # ---- random operand pairs
    rng = np.random.default_rng(20241203)
    A, B, ops, inpl = [], [], [], []
    for _ in range(1500):
        a, b = G.random_pair(rng, equal=True)
        A.append(a); B.append(b)
        ops.append(int(rng.integers(0, 4))); inpl.append(int(rng.integers(0, 2)))
    R = G.run_refdrv(oracle.REFDRV, [G.req_binop(o, i, 1, a, b) for o, i, a, b in zip(ops, inpl, A, B)], td)
    res, cnt, st = [], [], []
    for _ in A:
        s, c, w = R.bv()
        st.append(s); cnt.append(c); res.append(w)
    fa, oa = pack(A); fb, ob = pack(B); fr, orr = pack(res)
    np.savez_compressed(os.path.join(HERE, "binop_random.npz"), a=fa, a_off=oa, b=fb, b_off=ob,
                        res=fr, res_off=orr, cnt=np.array(cnt, np.uint64), status=np.array(st, np.uint32),
                        op=np.array(ops, np.int32), inplace=np.array(inpl, np.int32))

    # ---- geometric-run operands (appendFill, reference-built)
    dens = [1e-4, 1e-3, 1e-2, 0.1, 0.5]
    nbits = 1 << 20
    reqs = []
    runs = []
    for di, d in enumerate(dens):
        for s in (1, 2):
            r = G.geometric_runs(1000 * di + s, nbits, d)
            runs.append(r)
            reqs.append(G.req_runs(r))
    R = G.run_refdrv(oracle.REFDRV, reqs, td)
    operands = [R.bv()[2] for _ in reqs]
    cases = []
    reqs = []
    for di in range(len(dens)):
        a, b = operands[2 * di], operands[2 * di + 1]
        for op in range(4):
            for ip in (0, 1):
                cases.append((di, op, ip))
                reqs.append(G.req_binop(op, ip, 1, a, b))
    R = G.run_refdrv(oracle.REFDRV, reqs, td)
    gres, gcnt = [], []
    for _ in cases:
        s, c, w = R.bv()
        assert s == 0
        gres.append(w); gcnt.append(c)
    fo, oo = pack(operands); fr, orr = pack(gres)
    np.savez_compressed(os.path.join(HERE, "binop_geom.npz"), operands=fo, operands_off=oo,
                        res=fr, res_off=orr, cnt=np.array(gcnt, np.uint64),
                        case=np.array(cases, np.int32), density=np.array(dens), nbits=nbits,
                        runs=np.concatenate(runs), runs_off=pack([np.zeros(len(r)) for r in runs])[1])

    # ---- unary operations
    rng = np.random.default_rng(7)
    U = []
    for _ in range(400):
        a, _b = G.random_pair(rng, equal=True)
        U.append(a)
    reqs = []
    for a in U:
        reqs += [G.req_unary(2, a), G.req_unary(6, a), G.req_unary(7, a), G.req_unary(3, a)]
    R = G.run_refdrv(oracle.REFDRV, reqs, td)
    comp, decomp, flp, rid, ccnt = [], [], [], [], []
    for _ in U:
        s, c, w = R.bv(); comp.append(w); ccnt.append(c)
        s, c, w = R.bv(); decomp.append(w)
        s, c, w = R.bv(); flp.append(w)
        s = R.u32(); rid.append(R.vec())
    arrs = {}
    for name, lst in (("src", U), ("compress", comp), ("decompress", decomp), ("flip", flp), ("rids", rid)):
        f, o = pack(lst)
        arrs[name] = f
        arrs[name + "_off"] = o
    np.savez_compressed(os.path.join(HERE, "unary.npz"), compress_cnt=np.array(ccnt, np.uint64), **arrs)

    # ---- relic, small
    rng = np.random.default_rng(42)
    vals = rng.integers(0, 100, size=20000).astype(np.uint32)
    qs = []
    while len(qs) < 40:
        lo, hi = sorted(int(v) for v in rng.integers(0, 101, size=2))
        if lo < hi:
            qs.append((float(lo), float(hi)))
    R = G.run_refdrv(oracle.REFDRV, [G.req_relic(vals, qs)], td)
    nk = R.u32(); keys = np.frombuffer(R.d, np.float64, nk, R.p).copy(); R.p += 8 * nk
    no = R.u32(); offs = np.frombuffer(R.d, np.int64, no, R.p).copy(); R.p += 8 * no
    bms = R.vec()
    qc, qr = [], []
    for _ in qs:
        s = R.u32(); c = R.u32(); r = R.vec()
        assert s == 0
        qc.append(c); qr.append(r)
    fr, orr = pack(qr)
    np.savez_compressed(os.path.join(HERE, "relic_small.npz"), vals=vals, queries=np.array(qs),
                        keys=keys, offsets=offs, bitmaps=bms, counts=np.array(qc, np.uint64),
                        rids=fr, rids_off=orr)
    # ---- bin, small
    import struct
    rng = np.random.default_rng(43)
    n = 200000
    z = rng.zipf(1.2, size=n) % 100000
    vals = np.where(rng.random(n) < 0.7, rng.normal(size=n), z).astype(np.float32)
    qv = np.sort(rng.choice(vals, size=60).astype(np.float64)).reshape(30, 2)
    qv[:5, 0] -= 0.25  # a few ranges starting between values
    req = (struct.pack("<II", 9, n) + vals.tobytes() + struct.pack("<II", 100, len(qv)) + qv.tobytes())
    R = G.run_refdrv(oracle.REFDRV, [req], td)
    nk = R.u32(); keys = np.frombuffer(R.d, np.float64, nk, R.p).copy(); R.p += 8 * nk
    no = R.u32(); offs = np.frombuffer(R.d, np.int64, no, R.p).copy(); R.p += 8 * no
    bms = R.vec()
    qc, qr = [], []
    for _ in range(len(qv)):
        s_ = R.u32(); c = R.u32(); r = R.vec()
        assert s_ == 0
        qc.append(c); qr.append(r)
    fr, orr = pack(qr)
    np.savez_compressed(os.path.join(HERE, "bin_small.npz"), vals=vals, queries=qv, keys=keys, offsets=offs,
                        bitmaps=bms, counts=np.array(qc, np.uint64), rids=fr, rids_off=orr)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
