"""Generates the FastBit index files under tests/golden/ with the REFERENCE
library's own writers (FastBit built from source by oracle/Makefile.ref,
driven by oracle/refdrv.cpp request 10).  Run it where the reference sources
are available:

    python tests/golden/make_idx_files.py

Outputs:
  relic_3001.idx      relic::write of an ibis::relic over 3001 uint32 values
                      (seeded, 47 distinct values in [0, 60)); 4-byte offsets
  bin_5000.idx        bin::write of the <binning nbins=40 equal_weight/> index
                      of 5000 float32 values (70 % normal(0,1), 30 % Zipf(1.2)
                      ranks) built through the in-memory C API; 4-byte offsets
  relic_3001_o64.idx  the same two files with 8-byte bitmap offsets, the
  bin_5000_o64.idx    layout relic::write64 / bin::write64 use for indexes
                      past 2 GB (irelic.cpp:552-642, ibin.cpp:5746-5834);
                      converted by this script, since the reference writes
                      small indexes with 4-byte offsets
  idxfile_inputs.npz  the two columns and the reference's own triples for
                      them (relic::write(keys, offs, bms), irelic.cpp:644;
                      fastbit_iapi_deconstruct_index, iapi.cpp:1915)
"""
import os
import struct
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import wahgen as G  # noqa: E402


def write_req(kind, path, vals_u32, nbins):
    p = path.encode()
    return (struct.pack("<III", 10, kind, len(p)) + p + struct.pack("<I", len(vals_u32))
            + np.ascontiguousarray(vals_u32, np.uint32).tobytes() + struct.pack("<I", nbins))


def triple_relic(vals, td):
    req = struct.pack("<II", 5, len(vals)) + np.ascontiguousarray(vals, np.uint32).tobytes() + struct.pack("<I", 0)
    R = G.run_refdrv(oracle.REFDRV, [req], td)
    nk = R.u32(); keys = np.frombuffer(R.d, np.float64, nk, R.p).copy(); R.p += 8 * nk
    no = R.u32(); offs = np.frombuffer(R.d, np.int64, no, R.p).copy(); R.p += 8 * no
    return keys, offs, np.asarray(R.vec(), np.uint32)


def triple_bin(vals, nbins, td):
    req = (struct.pack("<II", 9, len(vals)) + np.ascontiguousarray(vals, np.float32).tobytes()
           + struct.pack("<II", nbins, 0))
    R = G.run_refdrv(oracle.REFDRV, [req], td)
    nk = R.u32(); keys = np.frombuffer(R.d, np.float64, nk, R.p).copy(); R.p += 8 * nk
    no = R.u32(); offs = np.frombuffer(R.d, np.int64, no, R.p).copy(); R.p += 8 * no
    return keys, offs, np.asarray(R.vec(), np.uint32)


def to_offsets64(img):
    """Rewrites a 4-byte-offset relic or bin file with 8-byte offsets, moving
    the keys and bitmaps to where relic::write64 / bin::write64 put them."""
    typ = img[5]
    nrows, nobs = struct.unpack_from("<II", img, 8)
    if typ == 7:  # relic: header, nrows nobs card, keys at 24, offsets, bitmaps
        keys = img[24:24 + 8 * nobs]
        off32 = np.frombuffer(img, np.int32, nobs + 1, 24 + 8 * nobs).astype(np.int64)
        first = 24 + 8 * nobs + 8 * (nobs + 1)
        off64 = off32 - off32[0] + first
        out = (img[:5] + bytes([7, 8, 0]) + img[8:20] + b"\0" * 4 + keys + off64.tobytes()
               + img[off32[0]:off32[-1]])
    else:  # bin: header, nrows nobs, offsets at 16, bounds/maxval/minval, bitmaps
        off32 = np.frombuffer(img, np.int32, nobs + 1, 16).astype(np.int64)
        dbl32 = 8 * ((16 + 4 * (nobs + 1) + 7) // 8)
        dbl = img[dbl32:dbl32 + 24 * nobs]
        dbl64 = 8 * ((16 + 8 * (nobs + 1) + 7) // 8)
        first = dbl64 + 24 * nobs
        off64 = off32 - off32[0] + first
        pad = b"\0" * (dbl64 - 16 - 8 * (nobs + 1))
        out = (img[:5] + bytes([0, 8, 0]) + img[8:16] + off64.tobytes() + pad + dbl
               + img[off32[0]:off32[-1]])
    return out


def main():
    if not oracle.build_reference():
        sys.exit("the reference library could not be built (needs the reference sources)")
    rng = np.random.default_rng(2024)
    relic_vals = rng.choice(np.setdiff1d(np.arange(60), rng.choice(60, 13, replace=False)), 3001).astype(np.uint32)
    n = 5000
    z = rng.zipf(1.2, size=n) % 100000
    bin_vals = np.where(rng.random(n) < 0.7, rng.normal(size=n), z).astype(np.float32)
    with tempfile.TemporaryDirectory() as td:
        rp, bp = os.path.join(HERE, "relic_3001.idx"), os.path.join(HERE, "bin_5000.idx")
        for p in (rp, bp):
            if os.path.exists(p):
                os.remove(p)
        R = G.run_refdrv(oracle.REFDRV, [write_req(1, rp, relic_vals, 0),
                                         write_req(2, bp, bin_vals.view(np.uint32), 40)], td)
        assert R.u32() == 0 and R.u32() == 0, "the reference failed to write an index file"
        rk, ro, rb = triple_relic(relic_vals, td)
        bk, bo, bb = triple_bin(bin_vals, 40, td)
    for src in (rp, bp):
        img = open(src, "rb").read()
        open(src[:-4] + "_o64.idx", "wb").write(to_offsets64(img))
    np.savez_compressed(os.path.join(HERE, "idxfile_inputs.npz"), relic_vals=relic_vals, bin_vals=bin_vals,
                        relic_keys=rk, relic_offsets=ro, relic_bitmaps=rb,
                        bin_keys=bk, bin_offsets=bo, bin_bitmaps=bb)
    print("wrote", rp, bp, "and their _o64 forms, idxfile_inputs.npz")


if __name__ == "__main__":
    main()
