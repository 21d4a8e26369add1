"""CPU oracle — TEST INFRASTRUCTURE ONLY.

ctypes wrappers over oracle/wah_oracle.c (a C restatement of the reference's
ibis::bitvector and range evaluation).  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg use this package, as the checker or as the
timed CPU baseline; the product (libfastlib_b200 / libwahgpu.so) never
imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REFDRV = os.path.join(REF_DIR, "refdrv")

_lib = None
_U32P = ctypes.POINTER(ctypes.c_uint32)


def build(force: bool = False) -> str:
    src = [os.path.join(HERE, "wah_oracle.c"), os.path.join(HERE, "range_oracle.c")]
    if force or not os.path.exists(LIB) or any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in src):
        subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-o", LIB, *src], check=True)
    return LIB


def build_reference(ref_root: str = None, jobs: int = 8) -> bool:
    """Compiles the reference library and the oracle driver into oracle/_ref
    (only where the reference sources exist: `ref_root`, else the directory
    named by the FASTBIT_REFERENCE environment variable, else ../reference
    beside this repository).  Returns True when refdrv is available
    afterwards."""
    if ref_root is None:
        ref_root = os.environ.get("FASTBIT_REFERENCE") or os.path.join(os.path.dirname(os.path.dirname(HERE)),
                                                                        "reference")
    if os.path.isdir(os.path.join(ref_root, "src")):
        subprocess.run(["make", "-s", "-f", os.path.join(HERE, "Makefile.ref"), f"REF={ref_root}",
                        f"-j{jobs}", "all"], check=True, cwd=os.path.dirname(HERE),
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    return os.path.exists(REFDRV)


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        for name in ("wo_ser_binop", "wo_ser_compress", "wo_ser_decompress", "wo_ser_rids",
                     "wo_ser_flip", "wo_build_runs"):
            getattr(L, name).restype = ctypes.c_long
        _lib = L
    return _lib


def _arr(x):
    return np.ascontiguousarray(x, dtype=np.uint32)


def _groups(serial):
    w = np.asarray(serial, dtype=np.uint32)
    if len(w) <= 1:
        return 0
    body = w[:-1]
    if 0 < w[-1] < 31:
        body = w[:-2]
    f = body >= 0x80000000
    return int(np.sum(np.where(f, body & 0x3FFFFFFF, 1).astype(np.int64)))


def binop(op: int, a, b, inplace: bool = False, compress: bool = True):
    """Reference a OP b (or a OP= b), then compress(); returns (serial, cnt)."""
    A, B = _arr(a), _arr(b)
    cap = len(A) + len(B) + 8 + 2 * (_groups(A) + _groups(B))
    out = np.empty(cap, dtype=np.uint32)
    cnt = ctypes.c_uint32()
    n = lib().wo_ser_binop(op, int(inplace), int(compress), A.ctypes.data_as(_U32P), len(A),
                           B.ctypes.data_as(_U32P), len(B), out.ctypes.data_as(_U32P), cap,
                           ctypes.byref(cnt))
    if n < 0:
        raise RuntimeError("oracle binop failed")
    return out[:n].copy(), int(cnt.value)


def compress(a):
    A = _arr(a)
    out = np.empty(len(A) + 2, dtype=np.uint32)
    cnt = ctypes.c_uint32()
    n = lib().wo_ser_compress(A.ctypes.data_as(_U32P), len(A), out.ctypes.data_as(_U32P), len(out), ctypes.byref(cnt))
    return out[:n].copy(), int(cnt.value)


def decompress(a):
    A = _arr(a)
    cap = _groups(A) + 3
    out = np.empty(cap, dtype=np.uint32)
    n = lib().wo_ser_decompress(A.ctypes.data_as(_U32P), len(A), out.ctypes.data_as(_U32P), cap)
    return out[:n].copy()


def flip(a):
    A = _arr(a)
    out = np.empty(len(A) + 2, dtype=np.uint32)
    n = lib().wo_ser_flip(A.ctypes.data_as(_U32P), len(A), out.ctypes.data_as(_U32P), len(out))
    return out[:n].copy()


def rids(a):
    A = _arr(a)
    cap = _groups(A) * 31 + 31
    out = np.empty(max(cap, 1), dtype=np.uint32)
    n = lib().wo_ser_rids(A.ctypes.data_as(_U32P), len(A), out.ctypes.data_as(_U32P), cap)
    return out[:n].copy()


def build_runs(runs):
    """appendFill-built bitvector (alternating 0/1 runs, 0 first), serialized."""
    r = np.ascontiguousarray(runs, dtype=np.uint64)
    nbits = int(r.sum())
    cap = nbits // 31 + 4
    out = np.empty(cap, dtype=np.uint32)
    n = lib().wo_build_runs(r.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), len(r),
                            out.ctypes.data_as(_U32P), cap)
    return out[:n].copy()


def is_degenerate(serial) -> bool:
    """One word per 31-bit group with some fill word, as the reference sees the
    operand after size() (an all-zero m_vec of several words collapses into
    one 0-fill first).  The reference's uncompressed loops then combine the
    fill header as literal bits."""
    w = np.asarray(serial, dtype=np.uint32)
    if len(w) <= 1:
        return False
    body = w[:-2] if 0 < w[-1] < 31 else w[:-1]
    if len(body) < 2:
        return False
    fill = body >= 0x80000000
    ones = np.where(fill, np.where(body >= 0xC0000000, (body & 0x3FFFFFFF).astype(np.int64) * 31, 0),
                    np.array([bin(int(x)).count("1") for x in body]) if len(body) < 4096 else
                    np.unpackbits(body.view(np.uint8)).reshape(-1, 32).sum(1))
    if int(np.sum(ones)) == 0:
        return False
    return _groups(w) == len(body) and bool(fill.any())
