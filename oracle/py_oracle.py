"""ctypes binding to the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the
benchmark's CPU-baseline leg, as the checker.  The product library does not
import this module.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

TYPE_CODE = {np.dtype(np.int32): 1, np.dtype(np.int64): 2, np.dtype(np.float32): 3, np.dtype(np.float64): 4}
ROUNDING = {"never": 0, "first": 1, "last": 2}


class OrcField(C.Structure):
    _fields_ = [("type", C.c_int), ("nx", C.c_size_t), ("ny", C.c_size_t), ("nz", C.c_size_t),
                ("nw", C.c_size_t), ("sx", C.c_ssize_t), ("sy", C.c_ssize_t), ("sz", C.c_ssize_t),
                ("sw", C.c_ssize_t), ("data", C.c_void_p)]


class OrcConfig(C.Structure):
    _fields_ = [("minbits", C.c_uint32), ("maxbits", C.c_uint32), ("maxprec", C.c_uint32),
                ("minexp", C.c_int32), ("rounding", C.c_int), ("tight", C.c_int)]


def build() -> Path:
    """Compile the oracle if its library is missing or stale."""
    src = [HERE / "zfp_oracle.cpp", HERE / "zfp_oracle.h", HERE / "Makefile"]
    if not LIB_PATH.exists() or any(p.stat().st_mtime > LIB_PATH.stat().st_mtime for p in src):
        subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB_PATH))
        vp, u64, u32, sz = C.c_void_p, C.c_uint64, C.c_uint32, C.c_size_t
        L.orc_stream_open.restype = vp
        L.orc_stream_open.argtypes = [vp, sz]
        L.orc_stream_close.argtypes = [vp]
        L.orc_stream_rewind.argtypes = [vp]
        for n in ("orc_stream_wtell", "orc_stream_rtell"):
            getattr(L, n).restype = u64
            getattr(L, n).argtypes = [vp]
        L.orc_stream_rseek.argtypes = [vp, u64]
        L.orc_stream_wseek.argtypes = [vp, u64]
        L.orc_stream_write_bits.restype = u64
        L.orc_stream_write_bits.argtypes = [vp, u64, u32]
        L.orc_stream_read_bits.restype = u64
        L.orc_stream_read_bits.argtypes = [vp, u32]
        L.orc_stream_flush.restype = u32
        L.orc_stream_flush.argtypes = [vp]
        L.orc_stream_align.restype = u32
        L.orc_stream_align.argtypes = [vp]
        L.orc_stream_size.restype = sz
        L.orc_stream_size.argtypes = [vp]
        L.orc_compress.restype = C.c_longlong
        L.orc_compress.argtypes = [vp, C.POINTER(OrcField), C.POINTER(OrcConfig), C.c_int]
        L.orc_decompress.restype = C.c_longlong
        L.orc_decompress.argtypes = [vp, C.POINTER(OrcField), C.POINTER(OrcConfig), C.c_int]
        L.orc_write_header.restype = sz
        L.orc_write_header.argtypes = [vp, C.POINTER(OrcField), C.POINTER(OrcConfig), C.c_uint]
        L.orc_read_header.restype = sz
        L.orc_read_header.argtypes = [vp, C.POINTER(OrcField), C.POINTER(OrcConfig), C.c_uint]
        L.orc_encode_block.restype = sz
        L.orc_encode_block.argtypes = [vp, C.c_int, C.c_int, vp, C.POINTER(C.c_ssize_t),
                                       C.POINTER(C.c_size_t), C.POINTER(OrcConfig)]
        L.orc_decode_block.restype = sz
        L.orc_decode_block.argtypes = [vp, C.c_int, C.c_int, vp, C.POINTER(C.c_ssize_t),
                                       C.POINTER(C.c_size_t), C.POINTER(OrcConfig)]
        L.orc_block_bits.restype = u32
        L.orc_block_bits.argtypes = [C.POINTER(OrcConfig), C.c_int, C.c_int]
        L.orc_maximum_size.restype = sz
        L.orc_maximum_size.argtypes = [C.POINTER(OrcConfig), C.POINTER(OrcField)]
        L.orc_mode.restype = C.c_int
        L.orc_mode.argtypes = [C.POINTER(OrcConfig)]
        L.orc_mode_bits.restype = u64
        L.orc_mode_bits.argtypes = [C.POINTER(OrcConfig)]
        _lib = L
    return _lib


def config(minbits, maxbits, maxprec, minexp, rounding="never", tight=False) -> OrcConfig:
    return OrcConfig(minbits, maxbits, maxprec, minexp, ROUNDING[rounding], int(bool(tight)))


def field_of(arr: np.ndarray, dims=None, strides=None, data_ptr=None) -> OrcField:
    """zfp field over a C-order array: zfp nx is the last (fastest) numpy axis."""
    if dims is None:
        dims = tuple(reversed(arr.shape))
    n = list(dims) + [0] * (4 - len(dims))
    s = list(strides or ()) + [0] * (4 - len(strides or ()))
    ptr = data_ptr if data_ptr is not None else arr.ctypes.data
    return OrcField(TYPE_CODE[arr.dtype], n[0], n[1], n[2], n[3], s[0], s[1], s[2], s[3], ptr)


class Stream:
    """A stream over a caller-owned word buffer (numpy uint64)."""

    def __init__(self, words: np.ndarray):
        assert words.dtype == np.uint64
        self.words = words
        self.h = lib().orc_stream_open(words.ctypes.data, words.size)

    def close(self):
        if self.h:
            lib().orc_stream_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rewind(self):
        lib().orc_stream_rewind(self.h)

    def wtell(self):
        return lib().orc_stream_wtell(self.h)

    def rtell(self):
        return lib().orc_stream_rtell(self.h)

    def flush(self):
        return lib().orc_stream_flush(self.h)

    def size(self):
        return lib().orc_stream_size(self.h)

    def bytes(self) -> bytes:
        return self.words.view(np.uint8)[: self.size()].tobytes()


def compress(arr: np.ndarray, cfg: OrcConfig, *, threads=1, dims=None, strides=None, data_ptr=None,
             capacity_words=None, header_mask=0):
    """Compress `arr` (optionally after a header); returns (stream bytes, size) or (None, -1)."""
    f = field_of(arr, dims, strides, data_ptr)
    if capacity_words is None:
        capacity_words = lib().orc_maximum_size(C.byref(cfg), C.byref(f)) // 8 + 4
    words = np.zeros(capacity_words, dtype=np.uint64)
    s = Stream(words)
    if header_mask:
        if lib().orc_write_header(s.h, C.byref(f), C.byref(cfg), header_mask) == 0:
            return None, -1
    n = lib().orc_compress(s.h, C.byref(f), C.byref(cfg), threads)
    if n < 0:
        return None, -1
    return words.view(np.uint8)[:n].tobytes(), n


def decompress(stream_bytes: bytes, out: np.ndarray, cfg: OrcConfig, *, threads=1, dims=None,
               strides=None, data_ptr=None, skip_bits=0):
    """Decompress into `out` (pre-allocated); returns bytes consumed or -1 (truncated)."""
    nwords = len(stream_bytes) // 8
    words = np.frombuffer(stream_bytes[: nwords * 8], dtype=np.uint64).copy()
    s = Stream(words)
    if skip_bits:
        lib().orc_stream_rseek(s.h, skip_bits)
    f = field_of(out, dims, strides, data_ptr)
    return lib().orc_decompress(s.h, C.byref(f), C.byref(cfg), threads)
