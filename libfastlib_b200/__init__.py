"""libfastlib_b200 — B200-native WAH bitvector operators and relic/bin range
evaluation with FastBit's interface.

The compute runs in ``libwahgpu.so`` (CUDA, sm_100a), reached through its C
ABI (``include/wahgpu.h``).  This module mirrors the reference's
``ibis::bitvector`` surface (src/bitvector.h:62-318): the logical operators
``& | ^ -`` return new bitvectors, the ``&= |= ^= -=`` forms rebind the left
operand, and ``cnt()``, ``size()``, ``compress()``, ``decompress()``,
``flip()``, ``write()`` and row-id extraction behave as there.  There is no
CPU path: without the library or an sm_100 device every call raises.
"""
from __future__ import annotations

import ctypes
import os
import weakref
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libwahgpu.so")

AND, OR, XOR, MINUS = 0, 1, 2, 3

_ERRORS = {
    -1: "EINVAL", -2: "ENODEV", -3: "ECUDA", -4: "ENOMEM", -5: "EFORMAT",
    -6: "ERANGE", -7: "ETIMEOUT", -8: "ESIZE", -9: "EDEGENERATE", -10: "EBUSY",
}


class WahError(RuntimeError):
    """A negative status from libwahgpu."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERRORS.get(code, code)}: {msg}")
        self.code = code


class _Info(ctypes.Structure):
    _fields_ = [("nwords", ctypes.c_uint64), ("nbits", ctypes.c_uint64), ("cnt", ctypes.c_uint64),
                ("anb", ctypes.c_uint32), ("aval", ctypes.c_uint32),
                ("compressed_form", ctypes.c_uint32)]


class _Term(ctypes.Structure):
    _fields_ = [("idx", ctypes.c_void_p), ("lop", ctypes.c_int), ("lo", ctypes.c_double),
                ("rop", ctypes.c_int), ("hi", ctypes.c_double)]


RELIC, BIN = 1, 2
TUNE_DENSE_TILE = 1
TUNE_RANGE_ORDER = 2
TUNE_RANGE_CTAS = 3
TUNE_DENSE_ENGINE = 4  # 0 auto (= 3), 1 pipelined group space, 2 word space, 3 two-pass group space, 4 / 5 single pass (CTA / warp tiles)
TUNE_CUM_STRIDE = 5
TUNE_MERGE_TILE = 6   # 0 auto, 16, 32 or 64 block-index entries per tile of the word-space merge
TEST_WITHHOLD_TILE = 100  # failure-path test hook: a tile that never publishes its look-back record
TEST_FAIL_ALLOC = 101     # failure-path test hook: the n-th device allocation from now fails
DENSE_TILES = (1024, 2048, 4096)
CMP_NONE, CMP_LT, CMP_LE = 0, 1, 2
U32, F32, I32 = 0, 1, 2

_lib = None


def load_library(path: Optional[str] = None) -> ctypes.CDLL:
    """Loads libwahgpu.so (built by ``libfastlib_b200.build``).  Raises if
    it is missing: there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"{p} is missing: build it with `python -m libfastlib_b200.build`")
    lib = ctypes.CDLL(p)
    P = ctypes.c_void_p
    U32P = ctypes.POINTER(ctypes.c_uint32)
    sig = {
        "wahgpu_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(P)]),
        "wahgpu_ctx_destroy": (ctypes.c_int, [P]),
        "wahgpu_ctx_set_stream": (ctypes.c_int, [P, P]),
        "wahgpu_ctx_stream": (P, [P]),
        "wahgpu_ctx_sync": (ctypes.c_int, [P]),
        "wahgpu_last_error": (ctypes.c_char_p, [P]),
        "wahgpu_ctx_launches": (ctypes.c_int64, [P]),
        "wahgpu_ctx_set_tuning": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int64]),
        "wahgpu_ctx_get_tuning": (ctypes.c_int64, [P, ctypes.c_int]),
        "wahgpu_bv_from_serial": (ctypes.c_int, [P, U32P, ctypes.c_uint64, ctypes.POINTER(P)]),
        "wahgpu_bv_from_device_serial": (ctypes.c_int, [P, P, ctypes.c_uint64, ctypes.POINTER(P)]),
        "wahgpu_bv_create": (ctypes.c_int, [P, ctypes.c_uint64, ctypes.POINTER(P)]),
        "wahgpu_bv_free": (ctypes.c_int, [P]),
        "wahgpu_bv_info_get": (ctypes.c_int, [P, ctypes.POINTER(_Info)]),
        "wahgpu_bv_size": (ctypes.c_int64, [P]),
        "wahgpu_bv_cnt": (ctypes.c_int64, [P]),
        "wahgpu_bv_serial_size": (ctypes.c_int64, [P]),
        "wahgpu_bv_write": (ctypes.c_int64, [P, U32P, ctypes.c_uint64]),
        "wahgpu_bv_device_words": (P, [P]),
        "wahgpu_bv_binop": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, P, P, ctypes.POINTER(P)]),
        "wahgpu_bv_binop_into": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, P, P, P]),
        "wahgpu_bv_compress": (ctypes.c_int, [P]),
        "wahgpu_bv_decompress": (ctypes.c_int, [P]),
        "wahgpu_bv_flip": (ctypes.c_int, [P]),
        "wahgpu_bv_rids": (ctypes.c_int64, [P, U32P, ctypes.c_uint64]),
        "wahgpu_bv_rids_device": (ctypes.c_int64, [P, P, ctypes.c_uint64]),
        "wahgpu_index_from_triple": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double),
                                                    ctypes.c_uint64, ctypes.POINTER(ctypes.c_int64), ctypes.c_uint64,
                                                    U32P, ctypes.c_uint64, ctypes.POINTER(P)]),
        "wahgpu_index_set_values": (ctypes.c_int, [P, ctypes.c_int, P, ctypes.c_uint64]),
        "wahgpu_index_read": (ctypes.c_int, [P, ctypes.c_char_p, ctypes.POINTER(P)]),
        "wahgpu_index_from_file_image": (ctypes.c_int, [P, P, ctypes.c_uint64, ctypes.POINTER(P)]),
        "wahgpu_idxfile_parse": (ctypes.c_int, [P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int),
                                                ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_double),
                                                ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64),
                                                ctypes.POINTER(ctypes.c_int64), ctypes.c_uint64,
                                                ctypes.POINTER(ctypes.c_uint64), U32P, ctypes.c_uint64,
                                                ctypes.POINTER(ctypes.c_uint64)]),
        "wahgpu_index_free": (ctypes.c_int, [P]),
        "wahgpu_index_build": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, P, ctypes.c_uint64, ctypes.c_uint32,
                                              ctypes.POINTER(P)]),
        "wahgpu_index_bitmap": (ctypes.c_int, [P, ctypes.c_uint32, ctypes.POINTER(P)]),
        "wahgpu_index_keys": (ctypes.c_int64, [P, ctypes.POINTER(ctypes.c_double), ctypes.c_uint64]),
        "wahgpu_index_deconstruct": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_double), ctypes.c_uint64,
                                                    ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int64),
                                                    ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64), U32P,
                                                    ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
        "wahgpu_index_nbitmaps": (ctypes.c_int64, [P]),
        "wahgpu_index_nrows": (ctypes.c_int64, [P]),
        "wahgpu_index_total_ones": (ctypes.c_int64, [P]),
        "wahgpu_evaluate": (ctypes.c_int64, [P, ctypes.POINTER(_Term), ctypes.c_uint32, U32P, ctypes.c_uint64,
                                             ctypes.POINTER(P)]),
        "wahgpu_estimate": (ctypes.c_int, [P, ctypes.POINTER(_Term), ctypes.POINTER(P), ctypes.POINTER(P)]),
        "wahgpu_estimate_count": (ctypes.c_int64, [P, ctypes.POINTER(_Term)]),
        "wahgpu_batch_create": (ctypes.c_int, [P, ctypes.POINTER(_Term), U32P, ctypes.c_uint32, ctypes.c_uint64,
                                               ctypes.c_int, ctypes.POINTER(P)]),
        "wahgpu_batch_run": (ctypes.c_int, [P]),
        "wahgpu_batch_counts": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_uint64)]),
        "wahgpu_batch_rids": (ctypes.c_int64, [P, ctypes.c_uint32, U32P, ctypes.c_uint64]),
        "wahgpu_batch_device_rids": (P, [P]),
        "wahgpu_batch_free": (ctypes.c_int, [P]),
        "wahgpu_batch_bytes": (ctypes.c_int64, [P]),
        "wahgpu_batch_create_capped": (ctypes.c_int, [P, ctypes.POINTER(_Term), ctypes.POINTER(ctypes.c_uint32),
                                                      ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64),
                                                      ctypes.POINTER(P)]),
        "wahgpu_batch_min_bytes": (ctypes.c_int64, [P]),
        "wahgpu_server_create": (ctypes.c_int, [P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(P)]),
        "wahgpu_server_submit": (ctypes.c_int64, [P, ctypes.POINTER(_Term), ctypes.c_uint32, ctypes.c_uint64]),
        "wahgpu_server_wait": (ctypes.c_int64, [P, ctypes.c_int64, ctypes.POINTER(ctypes.c_uint64), U32P,
                                                 ctypes.c_uint64, ctypes.POINTER(ctypes.c_double)]),
        "wahgpu_server_replay": (ctypes.c_int64, [P, ctypes.POINTER(_Term), U32P, ctypes.c_uint32,
                                                   ctypes.POINTER(ctypes.c_double), ctypes.c_uint64,
                                                   ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_double),
                                                   U32P, ctypes.POINTER(ctypes.c_uint64)]),
        "wahgpu_server_stats": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
        "wahgpu_server_free": (ctypes.c_int, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class Context:
    """A device, a stream and the scratch/pool memory of libwahgpu."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.wahgpu_ctx_create(device, ctypes.byref(h))
        if rc != 0:
            raise WahError(rc, self.lib.wahgpu_last_error(None).decode())
        self.h = h
        self.device = device
        self._live = weakref.WeakSet()

    def check(self, rc: int) -> int:
        if rc < 0:
            raise WahError(rc, self.lib.wahgpu_last_error(self.h).decode())
        return rc

    def set_stream(self, stream_ptr: Optional[int]) -> None:
        self.check(self.lib.wahgpu_ctx_set_stream(self.h, ctypes.c_void_p(stream_ptr or 0)))

    def sync(self) -> None:
        self.check(self.lib.wahgpu_ctx_sync(self.h))

    def after_torch(self, t) -> None:
        """Orders the context's stream after the work torch has queued on
        its current stream, so a CUDA tensor handed to the library is read
        only once the kernels producing it are done (the context's own
        stream is non-blocking: it does not wait for torch's by itself)."""
        import torch
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(t.device))
        torch.cuda.ExternalStream(int(self.lib.wahgpu_ctx_stream(self.h) or 0), device=t.device).wait_event(ev)

    @property
    def launches(self) -> int:
        return int(self.lib.wahgpu_ctx_launches(self.h))

    def set_tuning(self, key: int, value: int) -> None:
        """Launch-shape knob (TUNE_DENSE_TILE); results never depend on it."""
        self.check(self.lib.wahgpu_ctx_set_tuning(self.h, key, value))

    def get_tuning(self, key: int) -> int:
        return self.check(int(self.lib.wahgpu_ctx_get_tuning(self.h, key)))

    def close(self) -> None:
        """Frees every bitvector still alive on this context, then the
        context itself."""
        if getattr(self, "h", None):
            for bv in list(self._live):
                bv._release()
            self.lib.wahgpu_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # constructors
    def bitvector(self, serial) -> "Bitvector":
        """ibis::bitvector(const array_t<word_t>&) from a serialized array
        (host array, or a CUDA tensor of 32-bit words read on the device)."""
        if getattr(serial, "is_cuda", False):
            t = serial.contiguous()
            self.after_torch(t)
            h = ctypes.c_void_p()
            self.check(self.lib.wahgpu_bv_from_device_serial(self.h, ctypes.c_void_p(t.data_ptr()), t.numel(),
                                                            ctypes.byref(h)))
            return Bitvector(self, h)
        a = np.ascontiguousarray(serial, dtype=np.uint32)
        h = ctypes.c_void_p()
        self.check(self.lib.wahgpu_bv_from_serial(
            self.h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), len(a), ctypes.byref(h)))
        return Bitvector(self, h)

    def empty(self, cap_words: int) -> "Bitvector":
        h = ctypes.c_void_p()
        self.check(self.lib.wahgpu_bv_create(self.h, cap_words, ctypes.byref(h)))
        return Bitvector(self, h)


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class Bitvector:
    """A device-resident ``ibis::bitvector``."""

    def __init__(self, ctx: Context, h: ctypes.c_void_p):
        self.ctx = ctx
        self.h = h
        ctx._live.add(self)

    def _release(self) -> None:
        if self.h:
            self.ctx.lib.wahgpu_bv_free(self.h)
            self.h = None

    @classmethod
    def from_serial(cls, serial, ctx: Optional[Context] = None) -> "Bitvector":
        return (ctx or default_context()).bitvector(serial)

    def __del__(self):
        try:
            if self.h and self.ctx.h:
                self._release()
        except Exception:
            pass

    def _info(self) -> _Info:
        i = _Info()
        self.ctx.check(self.ctx.lib.wahgpu_bv_info_get(self.h, ctypes.byref(i)))
        return i

    def size(self) -> int:
        return int(self._info().nbits)

    def cnt(self) -> int:
        return int(self._info().cnt)

    count = cnt

    def nwords(self) -> int:
        return int(self._info().nwords)

    def write(self) -> np.ndarray:
        """Serialized words (write(array_t<word_t>&))."""
        n = self.ctx.check(self.ctx.lib.wahgpu_bv_serial_size(self.h))
        out = np.empty(n, dtype=np.uint32)
        self.ctx.check(self.ctx.lib.wahgpu_bv_write(
            self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), n))
        return out

    def rids(self) -> np.ndarray:
        """Ascending row ids of the 1 bits (indexSet walk)."""
        i = self._info()
        cap = int(i.cnt)
        out = np.empty(max(cap, 1), dtype=np.uint32)
        n = self.ctx.check(self.ctx.lib.wahgpu_bv_rids(
            self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), cap))
        return out[:n]

    def compress(self) -> "Bitvector":
        self.ctx.check(self.ctx.lib.wahgpu_bv_compress(self.h))
        return self

    def decompress(self) -> "Bitvector":
        self.ctx.check(self.ctx.lib.wahgpu_bv_decompress(self.h))
        return self

    def flip(self) -> "Bitvector":
        self.ctx.check(self.ctx.lib.wahgpu_bv_flip(self.h))
        return self

    def _binop(self, op: int, other: "Bitvector", inplace: bool) -> "Bitvector":
        h = ctypes.c_void_p()
        self.ctx.check(self.ctx.lib.wahgpu_bv_binop(self.ctx.h, op, 1 if inplace else 0,
                                                    self.h, other.h, ctypes.byref(h)))
        return Bitvector(self.ctx, h)

    def binop_into(self, op: int, other: "Bitvector", res: "Bitvector", inplace: bool = False) -> "Bitvector":
        self.ctx.check(self.ctx.lib.wahgpu_bv_binop_into(self.ctx.h, op, 1 if inplace else 0,
                                                         self.h, other.h, res.h))
        return res

    def __and__(self, o): return self._binop(AND, o, False)
    def __or__(self, o): return self._binop(OR, o, False)
    def __xor__(self, o): return self._binop(XOR, o, False)
    def __sub__(self, o): return self._binop(MINUS, o, False)
    def __iand__(self, o): return self._binop(AND, o, True)
    def __ior__(self, o): return self._binop(OR, o, True)
    def __ixor__(self, o): return self._binop(XOR, o, True)
    def __isub__(self, o): return self._binop(MINUS, o, True)


class Index:
    """A device-resident ``ibis::relic`` / ``ibis::bin`` index attached from
    the reference's (keys, offsets, bitmaps) triple."""

    def __init__(self, ctx: Context, kind: int, nrows: int, keys, offsets, bitmaps, values=None):
        self.ctx = ctx
        k = np.ascontiguousarray(keys, dtype=np.float64)
        o = np.ascontiguousarray(offsets, dtype=np.int64)
        b = np.ascontiguousarray(bitmaps, dtype=np.uint32)
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.wahgpu_index_from_triple(
            ctx.h, kind, nrows, k.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(k),
            o.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), len(o),
            b.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), len(b), ctypes.byref(h)))
        self.h = h
        self.nrows = nrows
        ctx._live.add(self)
        if values is not None:
            self.set_values(values)

    @classmethod
    def build(cls, ctx: Context, kind: int, values, nbins: int = 0) -> "Index":
        """Builds the index on the device from a column (a CUDA tensor or a
        numpy array of uint32 / int32 / float32): RELIC, one bitmap per
        distinct value; BIN, `nbins` equal-weight bins."""
        import torch
        t = values if isinstance(values, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(values))
        vt = {torch.int32: I32, torch.float32: F32, torch.uint32: U32}[t.dtype]
        if not t.is_cuda:
            t = t.to(f"cuda:{ctx.device}")
        t = t.contiguous()
        ctx.after_torch(t)
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.wahgpu_index_build(ctx.h, kind, vt, ctypes.c_void_p(t.data_ptr()), t.numel(), nbins,
                                             ctypes.byref(h)))
        self = cls.__new__(cls)
        self.ctx, self.h, self.nrows = ctx, h, t.numel()
        ctx._live.add(self)
        return self

    @classmethod
    def read(cls, ctx: Context, path: str, values=None) -> "Index":
        """A FastBit .idx file written by relic::write / bin::write."""
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.wahgpu_index_read(ctx.h, os.fsencode(path), ctypes.byref(h)))
        return cls._adopt(ctx, h, values)

    @classmethod
    def from_file_image(cls, ctx: Context, data: bytes, values=None) -> "Index":
        """The same from the bytes of such a file already in host memory."""
        buf = np.frombuffer(data, dtype=np.uint8)
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.wahgpu_index_from_file_image(ctx.h, buf.ctypes.data_as(ctypes.c_void_p), len(buf),
                                                       ctypes.byref(h)))
        return cls._adopt(ctx, h, values)

    @classmethod
    def _adopt(cls, ctx, h, values):
        self = cls.__new__(cls)
        self.ctx, self.h = ctx, h
        self.nrows = int(ctx.lib.wahgpu_index_nrows(h))
        ctx._live.add(self)
        if values is not None:
            self.set_values(values)
        return self

    def nbitmaps(self) -> int:
        return self.ctx.check(int(self.ctx.lib.wahgpu_index_nbitmaps(self.h)))

    def keys(self) -> np.ndarray:
        cap = 2 * self.nbitmaps() + 2
        out = np.empty(cap, dtype=np.float64)
        n = self.ctx.check(int(self.ctx.lib.wahgpu_index_keys(
            self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cap)))
        return out[:n]

    def deconstruct(self):
        """The reference's (keys, offsets, bitmaps) triple of this index
        (relic::write / bin::write to arrays, fastbit_iapi_deconstruct_index)."""
        lib, h = self.ctx.lib, self.h
        nk, no, nb = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self.ctx.check(lib.wahgpu_index_deconstruct(h, None, 0, ctypes.byref(nk), None, 0, ctypes.byref(no),
                                                    None, 0, ctypes.byref(nb)))
        keys = np.empty(nk.value, np.float64)
        offs = np.empty(no.value, np.int64)
        bms = np.empty(max(nb.value, 1), np.uint32)
        self.ctx.check(lib.wahgpu_index_deconstruct(
            h, keys.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(keys), ctypes.byref(nk),
            offs.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), len(offs), ctypes.byref(no),
            bms.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), len(bms), ctypes.byref(nb)))
        return keys, offs, bms[:nb.value]

    def bitmap(self, j: int) -> "Bitvector":
        h = ctypes.c_void_p()
        self.ctx.check(self.ctx.lib.wahgpu_index_bitmap(self.h, j, ctypes.byref(h)))
        return Bitvector(self.ctx, h)

    def _release(self):
        self.close()

    def set_values(self, values):
        v = np.ascontiguousarray(values)
        vt = {np.dtype(np.uint32): U32, np.dtype(np.float32): F32, np.dtype(np.int32): I32}[v.dtype]
        self.ctx.check(self.ctx.lib.wahgpu_index_set_values(self.h, vt, v.ctypes.data_as(ctypes.c_void_p), len(v)))
        self._values = v

    def term(self, lo=None, hi=None, lop=CMP_LE, rop=CMP_LT) -> _Term:
        """lo lop x rop hi; a missing bound drops that side."""
        return _Term(self.h, CMP_NONE if lo is None else lop, 0.0 if lo is None else float(lo),
                     CMP_NONE if hi is None else rop, 0.0 if hi is None else float(hi))

    def close(self):
        if getattr(self, "h", None) and self.ctx.h:
            self.ctx.lib.wahgpu_index_free(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def parse_index_file(data: bytes):
    """Host only (no device): the (kind, nrows, keys, word offsets, bitmaps)
    triple that a FastBit .idx file image holds, as the library reads it."""
    lib = load_library()
    buf = np.frombuffer(data, dtype=np.uint8)
    kind, nrows = ctypes.c_int(), ctypes.c_uint64()
    nk, no, nb = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    ptr = buf.ctypes.data_as(ctypes.c_void_p)
    rc = lib.wahgpu_idxfile_parse(ptr, len(buf), ctypes.byref(kind), ctypes.byref(nrows), None, 0, ctypes.byref(nk),
                                  None, 0, ctypes.byref(no), None, 0, ctypes.byref(nb))
    if rc < 0:
        raise WahError(rc, (lib.wahgpu_last_error(None) or b"").decode())
    keys = np.empty(nk.value, np.float64)
    offs = np.empty(no.value, np.int64)
    bms = np.empty(nb.value, np.uint32)
    rc = lib.wahgpu_idxfile_parse(ptr, len(buf), None, None, keys.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                  len(keys), None, offs.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), len(offs),
                                  None, bms.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), len(bms), None)
    if rc < 0:
        raise WahError(rc, (lib.wahgpu_last_error(None) or b"").decode())
    return kind.value, nrows.value, keys, offs, bms


def evaluate(ctx: Context, terms, want_rids: bool = True, want_hits: bool = False):
    """AND of the terms: (count, row ids or None, hit Bitvector or None)."""
    arr = (_Term * len(terms))(*terms)
    nrows = None
    cap = 0
    rids = None
    if want_rids:
        # an upper bound without evaluating twice: the row count
        nrows = int(ctx.lib.wahgpu_index_nrows(terms[0].idx))
        cap = nrows
        rids = np.empty(max(cap, 1), dtype=np.uint32)
    hp = ctypes.c_void_p()
    n = ctx.check(ctx.lib.wahgpu_evaluate(ctx.h, arr, len(terms),
                                          rids.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)) if want_rids else None,
                                          cap, ctypes.byref(hp) if want_hits else None))
    hits = Bitvector(ctx, hp) if want_hits else None
    return n, (rids[:n].copy() if want_rids else None), hits


def estimate(ctx: Context, term):
    """index::estimate(expr, lower, upper): (lower, upper) Bitvectors — the
    rows certainly hit and a superset of the hits (upper is empty when
    lower is exact)."""
    lo, up = ctypes.c_void_p(), ctypes.c_void_p()
    t = _Term(term.idx, term.lop, term.lo, term.rop, term.hi)
    ctx.check(ctx.lib.wahgpu_estimate(ctx.h, ctypes.byref(t), ctypes.byref(lo), ctypes.byref(up)))
    return Bitvector(ctx, lo), Bitvector(ctx, up)


def estimate_count(ctx: Context, term) -> int:
    """index::estimate(expr): an upper bound of the hit count (relic:
    exact; bin: the bins wholly inside and the edge bins)."""
    t = _Term(term.idx, term.lop, term.lo, term.rop, term.hi)
    return ctx.check(int(ctx.lib.wahgpu_estimate_count(ctx.h, ctypes.byref(t))))


class Batch:
    """Queries prepared once and run as one kernel launch (capturable in a
    CUDA graph).  queries: list of lists of terms."""

    def __init__(self, ctx: Context, queries, rid_cap: int = 0, caps=None):
        """rid_cap: room for the row ids of all queries, back to back; caps:
        instead, at most caps[q] row ids of query q (the first ones), each
        query in a region of its own."""
        self.ctx = ctx
        flat = [t for q in queries for t in q]
        offs = np.zeros(len(queries) + 1, dtype=np.uint32)
        offs[1:] = np.cumsum([len(q) for q in queries])
        self._terms = (_Term * len(flat))(*flat)
        self._offs = offs
        h = ctypes.c_void_p()
        op = offs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        if caps is not None:
            c = np.ascontiguousarray(caps, dtype=np.uint64)
            ctx.check(ctx.lib.wahgpu_batch_create_capped(ctx.h, self._terms, op, len(queries),
                                                         c.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                                         ctypes.byref(h)))
        else:
            ctx.check(ctx.lib.wahgpu_batch_create(ctx.h, self._terms, op, len(queries), rid_cap, 0, ctypes.byref(h)))
        self.h = h
        self.nq = len(queries)

    def run(self):
        self.ctx.check(self.ctx.lib.wahgpu_batch_run(self.h))

    def nbytes(self) -> int:
        """Algorithmic bytes of one run (bitmap words read, edge-row values)."""
        return self.ctx.check(int(self.ctx.lib.wahgpu_batch_bytes(self.h)))

    def min_bytes(self) -> int:
        """Bytes any evaluation must move: the bitmaps sumBins ORs (covered
        set or complement), edge bitmaps and edge rows, 8 per count."""
        return self.ctx.check(int(self.ctx.lib.wahgpu_batch_min_bytes(self.h)))

    def counts(self) -> np.ndarray:
        out = np.zeros(self.nq, dtype=np.uint64)
        self.ctx.check(self.ctx.lib.wahgpu_batch_counts(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        return out

    def rids(self, q: int, count: int) -> np.ndarray:
        out = np.empty(max(count, 1), dtype=np.uint32)
        n = self.ctx.check(self.ctx.lib.wahgpu_batch_rids(self.h, q, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), count))
        return out[:n]

    def close(self):
        if getattr(self, "h", None) and self.ctx.h:
            self.ctx.lib.wahgpu_batch_free(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous batching of conjunctive queries over resident indexes
    (wahgpu_server_*): `nslots` batches in flight, batches of up to
    `max_batch` queries admitted by a device scratch budget."""

    def __init__(self, ctx: Context, nslots: int = 2, max_batch: int = 1024, scratch_budget: int = 256 << 20):
        self.ctx = ctx
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.wahgpu_server_create(ctx.h, nslots, max_batch, scratch_budget, ctypes.byref(h)))
        self.h = h

    def submit(self, terms, rid_cap: int = 0) -> int:
        arr = (_Term * len(terms))(*terms)
        return self.ctx.check(int(self.ctx.lib.wahgpu_server_submit(self.h, arr, len(terms), rid_cap)))

    def wait(self, rid: int, rid_cap: int = 0):
        """(count, row ids or None, latency seconds)."""
        c = ctypes.c_uint64()
        lat = ctypes.c_double()
        out = np.empty(max(rid_cap, 1), dtype=np.uint32)
        n = self.ctx.check(int(self.ctx.lib.wahgpu_server_wait(
            self.h, rid, ctypes.byref(c), out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)) if rid_cap else None,
            rid_cap, ctypes.byref(lat))))
        return int(c.value), (out[:n].copy() if rid_cap else None), float(lat.value)

    def replay(self, queries, arrival_s, rid_cap: int = 0):
        """Open-loop replay; returns (counts, latencies seconds, wall seconds,
        row ids per query or None) — with rid_cap > 0 each query's first
        rid_cap row ids."""
        flat = [t for q in queries for t in q]
        offs = np.zeros(len(queries) + 1, dtype=np.uint32)
        offs[1:] = np.cumsum([len(q) for q in queries])
        arr = (_Term * len(flat))(*flat)
        arrival = np.ascontiguousarray(arrival_s, dtype=np.float64)
        counts = np.zeros(len(queries), dtype=np.uint64)
        lat = np.zeros(len(queries), dtype=np.float64)
        rids = np.zeros(max(len(queries) * rid_cap, 1), dtype=np.uint32)
        nrids = np.zeros(len(queries), dtype=np.uint64)
        U64P = ctypes.POINTER(ctypes.c_uint64)
        us = self.ctx.check(int(self.ctx.lib.wahgpu_server_replay(
            self.h, arr, offs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), len(queries),
            arrival.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), rid_cap,
            counts.ctypes.data_as(U64P), lat.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            rids.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)) if rid_cap else None,
            nrids.ctypes.data_as(U64P))))
        ids = [rids[q * rid_cap: q * rid_cap + int(nrids[q])] for q in range(len(queries))] if rid_cap else None
        return counts, lat, us / 1e6, ids

    def stats(self):
        b, s = ctypes.c_uint64(), ctypes.c_uint64()
        self.ctx.check(self.ctx.lib.wahgpu_server_stats(self.h, ctypes.byref(b), ctypes.byref(s)))
        return int(b.value), int(s.value)

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.wahgpu_server_free(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
