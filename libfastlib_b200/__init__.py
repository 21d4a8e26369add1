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
        self._live = weakref.WeakSet()

    def check(self, rc: int) -> int:
        if rc < 0:
            raise WahError(rc, self.lib.wahgpu_last_error(self.h).decode())
        return rc

    def set_stream(self, stream_ptr: Optional[int]) -> None:
        self.check(self.lib.wahgpu_ctx_set_stream(self.h, ctypes.c_void_p(stream_ptr or 0)))

    def sync(self) -> None:
        self.check(self.lib.wahgpu_ctx_sync(self.h))

    @property
    def launches(self) -> int:
        return int(self.lib.wahgpu_ctx_launches(self.h))

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
        """ibis::bitvector(const array_t<word_t>&) from a serialized array."""
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
