"""Requests to the reference library itself — TEST INFRASTRUCTURE ONLY.

oracle/_ref/refdrv is a small driver of this repository linked against the
reference FastBit library compiled from its sources (oracle/Makefile.ref).
These helpers write a request file, run the driver and parse its reply.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs use them: to pin the GPU's answers on the reference's own,
and to time the reference's own code on the host cores.
"""
from __future__ import annotations

import os
import shutil
import struct
import subprocess
import tempfile

import numpy as np

from . import REFDRV

VT_U32, VT_I32, VT_F32 = 1, 2, 3
_LAST = {"latency": []}


def available() -> bool:
    return os.path.exists(REFDRV)


def _run(req: bytes) -> bytes:
    d = None  # the default temporary directory, unless /dev/shm has room for request and reply
    try:
        if os.access("/dev/shm", os.W_OK) and shutil.disk_usage("/dev/shm").free > 3 * len(req) + (1 << 30):
            d = "/dev/shm"
    except OSError:
        d = None
    with tempfile.TemporaryDirectory(dir=d) as td:
        fi, fo = os.path.join(td, "req.bin"), os.path.join(td, "rep.bin")
        with open(fi, "wb") as f:
            f.write(req)
        subprocess.run([REFDRV, fi, fo], check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        with open(fo, "rb") as f:
            return f.read()


def vtype_of(values: np.ndarray) -> int:
    return {np.dtype(np.uint32): VT_U32, np.dtype(np.int32): VT_I32, np.dtype(np.float32): VT_F32}[values.dtype]


def iapi_queries(columns, queries, nthreads: int = 1, reps: int = 0, rids: bool = False):
    """Request 12: the in-memory C API (fastbit_iapi_register_array +
    fastbit_iapi_attach_full_index, then per query fastbit_selection_osr /
    combine / evaluate / get_coordinates) on columns given as
    (values, (keys, offsets, bitmaps)) with the index triple attached.
    queries: [[(column, lo, hi), ...], ...] for lo <= x < hi, AND'ed.
    Returns (seconds of `reps` timed passes on `nthreads` threads, counts,
    row ids per query or None); latencies() then gives each query's seconds
    in the first, one-thread pass."""
    out = [struct.pack("<IIIII", 12, max(1, nthreads), reps, 1 if rids else 0, len(columns))]
    for values, (keys, offs, bms) in columns:
        v = np.ascontiguousarray(values)
        out.append(struct.pack("<II", vtype_of(v), len(v)))
        out.append(v.tobytes())
        k = np.ascontiguousarray(keys, np.float64)
        o = np.ascontiguousarray(offs, np.int64)
        b = np.ascontiguousarray(bms, np.uint32)
        out.append(struct.pack("<Q", len(k)) + k.tobytes() + struct.pack("<Q", len(o)) + o.tobytes()
                   + struct.pack("<Q", len(b)) + b.tobytes())
    out.append(struct.pack("<I", len(queries)))
    for q in queries:
        out.append(struct.pack("<I", len(q)) + b"".join(struct.pack("<Idd", int(c), float(lo), float(hi))
                                                         for c, lo, hi in q))
    d = _run(b"".join(out))
    st, secs = struct.unpack_from("<Id", d, 0)
    if st != 0:
        raise RuntimeError(f"reference request 12 failed with status {st}")
    p = 12
    counts, ids, lat = [], ([] if rids else None), []
    for _ in queries:
        counts.append(struct.unpack_from("<Q", d, p)[0])
        lat.append(struct.unpack_from("<d", d, p + 8)[0])
        p += 16
        if rids:
            n = struct.unpack_from("<I", d, p)[0]
            ids.append(np.frombuffer(d, np.uint32, n, p + 4).copy())
            p += 4 + 4 * n
    _LAST["latency"] = lat
    return secs, counts, ids


def latencies():
    """Per-query seconds of the first (one-thread) pass of the last
    iapi_queries call."""
    return list(_LAST["latency"])


def relic_timed(values, queries, nthreads: int = 1, reps: int = 1):
    """Request 13: ibis::relic::construct, then per query relic::evaluate
    and the firstIndexSet row-id walk, `reps` timed passes on `nthreads`
    threads.  Returns (seconds, counts)."""
    v = np.ascontiguousarray(values, np.uint32)
    q = np.asarray(queries, np.float64).reshape(-1, 2)
    req = (struct.pack("<IIII", 13, max(1, nthreads), reps, len(v)) + v.tobytes()
           + struct.pack("<I", len(q)) + q.tobytes())
    d = _run(req)
    secs = struct.unpack_from("<d", d, 0)[0]
    return secs, [int(c) for c in np.frombuffer(d, np.uint64, len(q), 8)]


def _triple(d, p):
    nk = struct.unpack_from("<I", d, p)[0]; p += 4
    keys = np.frombuffer(d, np.float64, nk, p).copy(); p += 8 * nk
    no = struct.unpack_from("<I", d, p)[0]; p += 4
    offs = np.frombuffer(d, np.int64, no, p).copy(); p += 8 * no
    nb = struct.unpack_from("<I", d, p)[0]; p += 4
    bms = np.frombuffer(d, np.uint32, nb, p).copy(); p += 4 * nb
    return (keys, offs, bms), p


def relic_triple(values):
    """Request 5 without queries: relic::construct + write(keys, offs, bms)."""
    v = np.ascontiguousarray(values, np.uint32)
    d = _run(struct.pack("<II", 5, len(v)) + v.tobytes() + struct.pack("<I", 0))
    return _triple(d, 0)[0]


def relic_compare(values, queries):
    """Request 14: relic::construct over uint32 values, then per query
    (lo, lop, hi, rop) -- lo lop x rop hi with 0 = no bound, 1 = <, 2 = <= --
    relic::evaluate's count and row ids.  Returns [(count, rids), ...]."""
    v = np.ascontiguousarray(values, np.uint32)
    req = [struct.pack("<II", 14, len(v)), v.tobytes(), struct.pack("<I", len(queries))]
    for lo, lop, hi, rop in queries:
        req.append(struct.pack("<ddII", float(lo), float(hi), int(lop), int(rop)))
    d = _run(b"".join(req))
    res, p = [], 0
    for _ in range(len(queries)):
        st, c, n = struct.unpack_from("<III", d, p)
        p += 12
        if st:
            raise RuntimeError("relic::evaluate failed")
        res.append((c, np.frombuffer(d, np.uint32, n, p).copy()))
        p += 4 * n
    return res


def bin_index(values, nbins: int, queries=()):
    """Request 9: the reference's own bin index
    (fastbit_iapi_build_index "<binning nbins=N equal_weight/>" then
    fastbit_iapi_deconstruct_index) and, per query lo <= x < hi, its count
    and row ids.  Returns ((keys, offs, bms), [(count, rids), ...])."""
    v = np.ascontiguousarray(values, np.float32)
    q = np.asarray(list(queries), np.float64).reshape(-1, 2)
    d = _run(struct.pack("<II", 9, len(v)) + v.tobytes() + struct.pack("<II", nbins, len(q)) + q.tobytes())
    tri, p = _triple(d, 0)
    res = []
    for _ in range(len(q)):
        st, c, n = struct.unpack_from("<III", d, p)
        p += 12
        res.append((c, np.frombuffer(d, np.uint32, n, p).copy()))
        p += 4 * n
    return tri, res


def runs_pair_all_ops(runs_a, runs_b):
    """Request 11: both operands built by appendFill, then a OP b and
    a OP= b for & | ^ - with compress().  Returns (a, b, [(status, cnt,
    words)] * 8 in the order (op, form))."""
    out = [struct.pack("<I", 11)]
    for r in (runs_a, runs_b):
        r = np.ascontiguousarray(r, dtype=np.uint64)
        out.append(struct.pack("<Q", len(r)) + r.tobytes())
    d = _run(b"".join(out))
    p = 0
    vecs = []
    for _ in range(2):
        n = struct.unpack_from("<I", d, p)[0]
        vecs.append(np.frombuffer(d, np.uint32, n, p + 4).copy())
        p += 4 + 4 * n
    res = []
    for _ in range(8):
        st, cnt, n = struct.unpack_from("<III", d, p)
        res.append((st, cnt, np.frombuffer(d, np.uint32, n, p + 12).copy()))
        p += 12 + 4 * n
    return vecs[0], vecs[1], res
