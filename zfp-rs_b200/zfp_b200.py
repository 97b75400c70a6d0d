"""Python binding of libzfp_b200.so, shaped like zfp-rs's public API.

`ZfpConfig` mirrors zfp-rs src/config.rs (fixed_rate, fixed_precision,
fixed_accuracy, reversible, expert, with_rounding); `compress` and
`decompress` mirror `ZfpBitStream::compress` / `decompress` through the
library's zfp.h C ABI (zfp_stream_open, zfp_write_header, zfp_compress, ...),
which runs the codec on the GPU.  `compress_device` / `decompress_device`
take torch CUDA tensors and keep everything in device memory.

Errors follow the reference: a call that fails raises ZfpError carrying the
library's status (buffer too small, truncated stream, ...).
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, replace
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libzfp_b200.so"

ZFP_MIN_BITS, ZFP_MAX_BITS, ZFP_MAX_PREC, ZFP_MIN_EXP = 1, 16658, 64, -1074
HEADER_MAGIC, HEADER_META, HEADER_MODE, HEADER_FULL = 1, 2, 4, 7
TYPE_CODE = {np.dtype(np.int32): 1, np.dtype(np.int64): 2, np.dtype(np.float32): 3, np.dtype(np.float64): 4}
CODE_TYPE = {v: k for k, v in TYPE_CODE.items()}
ROUND_NEVER, ROUND_FIRST, ROUND_LAST = 0, -1, 1
ERRORS = {1: "buffer too small", 2: "stream is truncated", 3: "CUDA error", 4: "invalid arguments",
          6: "field too large for the no-allocation scratch"}


class ZfpError(RuntimeError):
    def __init__(self, what: str, code: int):
        super().__init__(f"{what}: {ERRORS.get(code, 'failed')}")
        self.code = code


class ZfpField(C.Structure):
    _fields_ = [("type", C.c_int), ("nx", C.c_size_t), ("ny", C.c_size_t), ("nz", C.c_size_t),
                ("nw", C.c_size_t), ("sx", C.c_ssize_t), ("sy", C.c_ssize_t), ("sz", C.c_ssize_t),
                ("sw", C.c_ssize_t), ("data", C.c_void_p)]


class ZfpExecution(C.Structure):
    _fields_ = [("policy", C.c_int), ("params", C.c_void_p)]


class ZfpStream(C.Structure):
    _fields_ = [("minbits", C.c_uint), ("maxbits", C.c_uint), ("maxprec", C.c_uint), ("minexp", C.c_int32),
                ("stream", C.c_void_p), ("exec", ZfpExecution)]


class _ZfpExpert(C.Structure):
    _fields_ = [("minbits", C.c_uint), ("maxbits", C.c_uint), ("maxprec", C.c_uint), ("minexp", C.c_int32)]


class _ZfpConfigArg(C.Union):
    _fields_ = [("rate", C.c_double), ("precision", C.c_uint), ("tolerance", C.c_double), ("expert", _ZfpExpert)]


class ZfpConfigC(C.Structure):
    """zfp_config (include/zfp.h)."""

    _fields_ = [("mode", C.c_int), ("arg", _ZfpConfigArg)]


class ZfpDesc(C.Structure):
    _fields_ = [("type", C.c_int), ("nx", C.c_size_t), ("ny", C.c_size_t), ("nz", C.c_size_t),
                ("nw", C.c_size_t), ("sx", C.c_ssize_t), ("sy", C.c_ssize_t), ("sz", C.c_ssize_t),
                ("sw", C.c_ssize_t), ("minbits", C.c_uint), ("maxbits", C.c_uint), ("maxprec", C.c_uint),
                ("minexp", C.c_int32), ("rounding", C.c_int), ("tight_error", C.c_int32)]


class ZfpBatchItem(C.Structure):
    """zfpb_batch_item (include/zfp_b200.h)."""

    _fields_ = [("desc", ZfpDesc), ("d_field", C.c_void_p), ("d_stream", C.c_void_p), ("stream_bytes", C.c_size_t),
                ("d_block_offsets", C.c_void_p), ("header_mask", C.c_uint), ("result", C.c_size_t),
                ("status", C.c_int)]


class ZfpRequestDone(C.Structure):
    """zfpb_request_done (include/zfp_b200.h)."""

    _fields_ = [("tag", C.c_uint64), ("result", C.c_size_t), ("status", C.c_int), ("queue_ms", C.c_double),
                ("latency_ms", C.c_double)]


# (name, restype, argtypes) of every function include/zfp.h and include/zfp_b200.h declare.
_vp, _sz, _u, _u64, _i32, _b = C.c_void_p, C.c_size_t, C.c_uint, C.c_uint64, C.c_int32, C.c_int32
_F = C.POINTER(ZfpField)
_S = C.POINTER(ZfpStream)
SIGNATURES = [
    ("stream_open", _vp, [_vp, _sz]), ("stream_close", None, [_vp]), ("stream_clone", _vp, [_vp]),
    ("stream_alignment", _sz, []), ("stream_data", _vp, [_vp]), ("stream_size", _sz, [_vp]),
    ("stream_capacity", _sz, [_vp]), ("stream_stride_block", _sz, [_vp]),
    ("stream_stride_delta", C.c_ssize_t, [_vp]), ("stream_read_bit", _u, [_vp]),
    ("stream_write_bit", _u, [_vp, _u]), ("stream_read_bits", _u64, [_vp, _sz]),
    ("stream_write_bits", _u64, [_vp, _u64, _sz]), ("stream_rtell", _u64, [_vp]),
    ("stream_wtell", _u64, [_vp]), ("stream_rewind", None, [_vp]), ("stream_rseek", None, [_vp, _u64]),
    ("stream_wseek", None, [_vp, _u64]), ("stream_skip", None, [_vp, _u64]), ("stream_pad", None, [_vp, _u64]),
    ("stream_align", _sz, [_vp]), ("stream_flush", _sz, [_vp]), ("stream_copy", None, [_vp, _vp, _u64]),
    ("zfp_field_alloc", _F, []), ("zfp_field_1d", _F, [_vp, C.c_int, _sz]),
    ("zfp_field_2d", _F, [_vp, C.c_int, _sz, _sz]), ("zfp_field_3d", _F, [_vp, C.c_int, _sz, _sz, _sz]),
    ("zfp_field_4d", _F, [_vp, C.c_int, _sz, _sz, _sz, _sz]), ("zfp_field_free", None, [_F]),
    ("zfp_field_pointer", _vp, [_F]), ("zfp_field_begin", _vp, [_F]), ("zfp_field_type", C.c_int, [_F]),
    ("zfp_field_precision", _u, [_F]), ("zfp_field_dimensionality", _u, [_F]),
    ("zfp_field_size", _sz, [_F, C.POINTER(C.c_size_t)]), ("zfp_field_size_bytes", _sz, [_F]),
    ("zfp_field_blocks", _sz, [_F]), ("zfp_field_stride", _b, [_F, C.POINTER(C.c_ssize_t)]),
    ("zfp_field_is_contiguous", _b, [_F]), ("zfp_field_metadata", _u64, [_F]),
    ("zfp_field_set_pointer", None, [_F, _vp]), ("zfp_field_set_type", C.c_int, [_F, C.c_int]),
    ("zfp_field_set_size_1d", None, [_F, _sz]), ("zfp_field_set_size_2d", None, [_F, _sz, _sz]),
    ("zfp_field_set_size_3d", None, [_F, _sz, _sz, _sz]), ("zfp_field_set_size_4d", None, [_F, _sz, _sz, _sz, _sz]),
    ("zfp_field_set_stride_1d", None, [_F, C.c_ssize_t]),
    ("zfp_field_set_stride_2d", None, [_F, C.c_ssize_t, C.c_ssize_t]),
    ("zfp_field_set_stride_3d", None, [_F, C.c_ssize_t, C.c_ssize_t, C.c_ssize_t]),
    ("zfp_field_set_stride_4d", None, [_F, C.c_ssize_t, C.c_ssize_t, C.c_ssize_t, C.c_ssize_t]),
    ("zfp_field_set_metadata", _b, [_F, _u64]),
    ("zfp_config_none", ZfpConfigC, []), ("zfp_config_rate", ZfpConfigC, [C.c_double, _b]),
    ("zfp_config_precision", ZfpConfigC, [C.c_uint32]), ("zfp_config_accuracy", ZfpConfigC, [C.c_double]),
    ("zfp_config_reversible", ZfpConfigC, []),
    ("zfp_config_expert", ZfpConfigC, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_int32]),
    ("zfp_type_size", _sz, [C.c_int]), ("zfp_stream_open", _S, [_vp]), ("zfp_stream_close", None, [_S]),
    ("zfp_stream_bit_stream", _vp, [_S]), ("zfp_stream_compression_mode", C.c_int, [_S]),
    ("zfp_stream_rate", C.c_double, [_S, _u]), ("zfp_stream_precision", _u, [_S]),
    ("zfp_stream_accuracy", C.c_double, [_S]), ("zfp_stream_mode", _u64, [_S]),
    ("zfp_stream_params", None, [_S, C.POINTER(_u), C.POINTER(_u), C.POINTER(_u), C.POINTER(_i32)]),
    ("zfp_stream_compressed_size", _sz, [_S]), ("zfp_block_maximum_size", _sz, [C.c_int, _u, _b]),
    ("zfp_stream_maximum_size", _sz, [_S, _F]), ("zfp_write_header", _sz, [_S, _F, _u]),
    ("zfp_read_header", _sz, [_S, _F, _u]), ("zfp_compress", _sz, [_S, _F]), ("zfp_decompress", _sz, [_S, _F]),
    ("zfp_stream_rewind", None, [_S]), ("zfp_stream_set_bit_stream", None, [_S, _vp]),
    ("zfp_stream_set_reversible", None, [_S]),
    ("zfp_stream_set_rate", C.c_double, [_S, C.c_double, C.c_int, _u, _b]),
    ("zfp_stream_set_precision", _u, [_S, _u]), ("zfp_stream_set_accuracy", C.c_double, [_S, C.c_double]),
    ("zfp_stream_set_mode", C.c_int, [_S, _u64]), ("zfp_stream_set_params", _b, [_S, _u, _u, _u, _i32]),
    ("zfp_stream_execution", C.c_int, [_S]), ("zfp_stream_omp_threads", _u, [_S]),
    ("zfp_stream_omp_chunk_size", _u, [_S]), ("zfp_stream_set_execution", _b, [_S, C.c_int]),
    ("zfp_stream_set_omp_threads", _b, [_S, _u]), ("zfp_stream_set_omp_chunk_size", _b, [_S, _u]),
    ("zfp_stream_flush", _sz, [_S]), ("zfp_stream_align", _sz, [_S]),
    ("zfp_stream_set_rounding", _b, [_S, C.c_int, _b]), ("zfp_stream_rounding", C.c_int, [_S, C.POINTER(_b)]),
    ("zfpb_last_error", C.c_int, []), ("zfpb_timing_enable", None, [C.c_int]),
    ("zfpb_timing_read", C.c_int, [C.POINTER(C.c_double), C.POINTER(C.c_ulonglong), C.c_int]),
    ("zfpb_compress_device", _sz, [C.POINTER(ZfpDesc), _vp, _vp, _sz, _vp, _vp]),
    ("zfpb_decompress_device", _sz, [C.POINTER(ZfpDesc), _vp, _sz, _vp, _vp, _vp]),
    ("zfpb_compress_device_noalloc", _sz, [C.POINTER(ZfpDesc), _vp, _vp, _sz, _vp]),
    ("zfpb_compress_batch", _sz, [C.POINTER(ZfpBatchItem), _sz, _vp]),
    ("zfpb_decompress_batch", _sz, [C.POINTER(ZfpBatchItem), _sz, _vp]),
    ("zfpb_server_create", _vp, [_sz, C.c_int, _sz, _sz]),
    ("zfpb_server_submit", C.c_int, [_vp, C.POINTER(ZfpBatchItem), C.c_int, C.c_uint64]),
    ("zfpb_server_poll", _sz, [_vp, C.POINTER(ZfpRequestDone), _sz, C.c_int]),
    ("zfpb_server_outstanding", _sz, [_vp]),
    ("zfpb_server_destroy", None, [_vp]),
]
BLOCK_TYPES = ("int32", "int64", "float", "double")


def _block_signatures():
    """include/zfp_block.h (block-level calls, promotion) and the batched
    block calls of include/zfp_b200.h."""
    out = []
    ss = C.c_ssize_t
    for name in BLOCK_TYPES:
        for d in (1, 2, 3, 4):
            out += [(f"zfp_encode_block_{name}_{d}", _sz, [_S, _vp]),
                    (f"zfp_decode_block_{name}_{d}", _sz, [_S, _vp]),
                    (f"zfp_encode_block_strided_{name}_{d}", _sz, [_S, _vp] + [ss] * d),
                    (f"zfp_decode_block_strided_{name}_{d}", _sz, [_S, _vp] + [ss] * d),
                    (f"zfp_encode_partial_block_strided_{name}_{d}", _sz, [_S, _vp] + [_sz] * d + [ss] * d),
                    (f"zfp_decode_partial_block_strided_{name}_{d}", _sz, [_S, _vp] + [_sz] * d + [ss] * d)]
    for name in ("int8", "uint8", "int16", "uint16"):
        out += [(f"zfp_promote_{name}_to_int32", None, [_vp, _vp, _u]),
                (f"zfp_demote_int32_to_{name}", None, [_vp, _vp, _u])]
    out += [("zfpb_encode_blocks", _sz, [C.POINTER(ZfpDesc), _u, _sz, _vp, _vp, _sz, _vp, _vp]),
            ("zfpb_decode_blocks", _sz, [C.POINTER(ZfpDesc), _u, _sz, _vp, _sz, _vp, _vp, _vp])]
    return out


SIGNATURES += _block_signatures()
DATA_SYMBOLS = ["stream_word_bits", "zfp_codec_version", "zfp_library_version"]

_lib = None


def lib():
    """Load libzfp_b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise OSError(f"{LIB_PATH} is missing: build it with `make -C {HERE}`")
        L = C.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _type_header_bits(code: int) -> int:
    return 9 if code == 3 else 12 if code == 4 else 0


@dataclass(frozen=True)
class ZfpConfig:
    """Expert parameters plus rounding (zfp-rs src/config.rs:163-174)."""

    min_bits: int
    max_bits: int
    max_prec: int
    min_exp: int
    rounding: str = "never"  # "never", "first", "last"
    tight_error: bool = False

    @staticmethod
    def fixed_rate(rate: float, dtype, dims: int, word_aligned: bool = False) -> "ZfpConfig":
        """config.rs:266-280: rate bits per value, rounded, raised to the float header."""
        if rate < 0 or dims not in (1, 2, 3, 4):
            raise ValueError("invalid ZFP fixed rate")
        rounded = math.floor((4 ** dims) * rate + 0.5)
        if not 0 <= rounded <= 0xFFFFFFFF:
            raise ValueError("invalid ZFP fixed rate")
        bits = max(rounded, _type_header_bits(TYPE_CODE[np.dtype(dtype)]))
        if word_aligned:
            bits = (bits + 63) // 64 * 64
        if not 1 <= bits <= ZFP_MAX_BITS:
            raise ValueError("invalid ZFP fixed rate")
        return ZfpConfig(bits, bits, ZFP_MAX_PREC, ZFP_MIN_EXP)

    @staticmethod
    def fixed_precision(precision: int) -> "ZfpConfig":
        """config.rs:308-315"""
        p = min(precision, ZFP_MAX_PREC) if precision > 0 else ZFP_MAX_PREC
        return ZfpConfig(ZFP_MIN_BITS, ZFP_MAX_BITS, p, ZFP_MIN_EXP)

    @staticmethod
    def fixed_accuracy(tolerance: float) -> "ZfpConfig":
        """config.rs:324-333: min_exp = frexp(tolerance).exponent - 1."""
        emin = math.frexp(tolerance)[1] - 1 if tolerance > 0 else ZFP_MIN_EXP
        return ZfpConfig(ZFP_MIN_BITS, ZFP_MAX_BITS, ZFP_MAX_PREC, emin)

    @staticmethod
    def reversible() -> "ZfpConfig":
        """config.rs:337-339"""
        return ZfpConfig(ZFP_MIN_BITS, ZFP_MAX_BITS, ZFP_MAX_PREC, ZFP_MIN_EXP - 1)

    @staticmethod
    def expert(min_bits: int, max_bits: int, max_prec: int, min_exp: int) -> "ZfpConfig":
        """config.rs:354-365"""
        if not (min_bits <= max_bits and 0 < max_prec <= 64):
            raise ValueError("invalid ZFP compression parameters")
        return ZfpConfig(min_bits, max_bits, max_prec, min_exp)

    def with_rounding(self, rounding: str, tight_error: bool = False) -> "ZfpConfig":
        if rounding not in ("never", "first", "last"):
            raise ValueError(rounding)
        return replace(self, rounding=rounding, tight_error=bool(tight_error) and rounding != "never")

    @property
    def rounding_code(self) -> int:
        return {"never": ROUND_NEVER, "first": ROUND_FIRST, "last": ROUND_LAST}[self.rounding]


def field_of(arr: np.ndarray, dims=None, strides=None, data_ptr=None) -> ZfpField:
    """A zfp field over a C-order array: zfp's x is the last (fastest) axis."""
    if dims is None:
        dims = tuple(reversed(arr.shape))
    n = list(dims) + [0] * (4 - len(dims))
    s = list(strides or ()) + [0] * (4 - len(strides or ()))
    ptr = data_ptr if data_ptr is not None else arr.ctypes.data
    return ZfpField(TYPE_CODE[np.dtype(arr.dtype)], n[0], n[1], n[2], n[3], s[0], s[1], s[2], s[3], ptr)


class Stream:
    """A zfp_stream over a bitstream on `buffer` (numpy uint64 or a device pointer)."""

    def __init__(self, config: ZfpConfig, buffer=None, nbytes=None, device_ptr=None):
        L = lib()
        if device_ptr is not None:
            self.bs = L.stream_open(device_ptr, nbytes)
        else:
            self.buffer = buffer
            self.bs = L.stream_open(buffer.ctypes.data, buffer.nbytes)
        self.zfp = L.zfp_stream_open(self.bs)
        self.set_config(config)

    def set_config(self, c: ZfpConfig):
        L = lib()
        if not L.zfp_stream_set_params(self.zfp, c.min_bits, c.max_bits, c.max_prec, c.min_exp):
            # Unvalidated parameters, as a C caller may write the struct directly.
            z = self.zfp.contents
            z.minbits, z.maxbits, z.maxprec, z.minexp = c.min_bits, c.max_bits, c.max_prec, c.min_exp
        L.zfp_stream_set_rounding(self.zfp, c.rounding_code, int(c.tight_error))

    def close(self):
        if getattr(self, "zfp", None):
            lib().zfp_stream_close(self.zfp)
            lib().stream_close(self.bs)
            self.zfp = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def maximum_size(arr_or_shape, dtype, config: ZfpConfig) -> int:
    """config.rs:642-658, header included."""
    shape = arr_or_shape.shape if hasattr(arr_or_shape, "shape") else tuple(arr_or_shape)
    f = ZfpField(TYPE_CODE[np.dtype(dtype)], *(list(reversed(shape)) + [0] * (4 - len(shape))), 0, 0, 0, 0, None)
    s = Stream(config, np.zeros(1, dtype=np.uint64))
    try:
        return lib().zfp_stream_maximum_size(s.zfp, C.byref(f))
    finally:
        s.close()


def compress(arr: np.ndarray, config: ZfpConfig, *, header: bool = False, dims=None, strides=None,
             data_ptr=None, capacity=None) -> bytes:
    """Compress a host array through zfp_compress; returns the stream bytes."""
    L = lib()
    f = field_of(arr, dims, strides, data_ptr)
    if capacity is None:
        s0 = Stream(config, np.zeros(1, dtype=np.uint64))
        capacity = L.zfp_stream_maximum_size(s0.zfp, C.byref(f))
        s0.close()
    words = np.zeros(max(capacity // 8 + 1, 1), dtype=np.uint64)
    s = Stream(config, words)
    try:
        if header and L.zfp_write_header(s.zfp, C.byref(f), HEADER_FULL) == 0:
            raise ZfpError("write_header", 4)
        n = L.zfp_compress(s.zfp, C.byref(f))
        if n == 0:
            raise ZfpError("compress", L.zfpb_last_error())
        return words.view(np.uint8)[:n].tobytes()
    finally:
        s.close()


def decompress(stream: bytes, out: np.ndarray, config: ZfpConfig | None = None, *, header: bool = False,
               dims=None, strides=None, data_ptr=None) -> int:
    """Decompress into `out` through zfp_decompress; returns bytes consumed."""
    L = lib()
    words = np.zeros((len(stream) + 7) // 8, dtype=np.uint64)
    words.view(np.uint8)[: len(stream)] = np.frombuffer(stream, dtype=np.uint8)
    s = Stream(config or ZfpConfig.fixed_precision(64), words)
    s.buffer = words
    try:
        f = field_of(out, dims, strides, data_ptr)
        if header and L.zfp_read_header(s.zfp, C.byref(f), HEADER_FULL) == 0:
            raise ZfpError("read_header", 4)
        n = L.zfp_decompress(s.zfp, C.byref(f))
        if n == 0:
            raise ZfpError("decompress", L.zfpb_last_error())
        return n
    finally:
        s.close()


def desc_of(shape, dtype, config: ZfpConfig, strides=None) -> ZfpDesc:
    n = list(reversed(tuple(shape))) + [0] * (4 - len(shape))
    s = list(strides or ()) + [0] * (4 - len(strides or ()))
    return ZfpDesc(TYPE_CODE[np.dtype(dtype)], n[0], n[1], n[2], n[3], s[0], s[1], s[2], s[3], config.min_bits,
                   config.max_bits, config.max_prec, config.min_exp, config.rounding_code, int(config.tight_error))


KERNEL_KINDS = ["encode_fixed", "encode_var", "scan", "pack", "decode_fixed", "decode_var", "walk", "claim",
                "offsets", "parse", "finish"]


def timing_enable(on: bool = True):
    lib().zfpb_timing_enable(int(on))


def timing_read() -> dict:
    """Per kernel kind: (total ms, launches) since timing_enable."""
    n = len(KERNEL_KINDS)
    ms = (C.c_double * n)()
    cnt = (C.c_ulonglong * n)()
    lib().zfpb_timing_read(ms, cnt, n)
    return {k: (ms[i], cnt[i]) for i, k in enumerate(KERNEL_KINDS)}


def _np_dtype(t):
    import torch

    return {torch.float32: np.float32, torch.float64: np.float64, torch.int32: np.int32,
            torch.int64: np.int64}[t]


def compress_device(x, config: ZfpConfig, out=None, offsets=None, stream=None) -> int:
    """Compress a contiguous torch CUDA tensor into the uint8/uint64 CUDA tensor `out`.

    Returns the stream size in bytes.  `offsets` (int64 CUDA tensor of
    nblocks + 1 entries), if given, receives the block bit offsets.
    """
    import torch

    d = desc_of(x.shape, _np_dtype(x.dtype), config)
    cs = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    n = lib().zfpb_compress_device(C.byref(d), x.data_ptr(), out.data_ptr(), out.numel() * out.element_size(),
                                   offsets.data_ptr() if offsets is not None else None, cs)
    if n == 0:
        raise ZfpError("compress_device", lib().zfpb_last_error())
    return n


def decompress_device(stream_t, nbytes: int, out, config: ZfpConfig, offsets=None, stream=None) -> int:
    """Decompress `nbytes` of the CUDA tensor `stream_t` into the CUDA tensor `out`."""
    import torch

    d = desc_of(out.shape, _np_dtype(out.dtype), config)
    cs = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    n = lib().zfpb_decompress_device(C.byref(d), stream_t.data_ptr(), nbytes, out.data_ptr(),
                                     offsets.data_ptr() if offsets is not None else None, cs)
    if n == 0:
        raise ZfpError("decompress_device", lib().zfpb_last_error())
    return n


def batch_items(fields, configs, streams, nbytes=None, offsets=None, header_mask=0):
    """A ctypes array of zfpb_batch_item for torch CUDA tensors.

    fields[i] is a contiguous CUDA tensor (the input of a compress, the output
    of a decompress), streams[i] a CUDA tensor holding its stream, nbytes[i]
    the stream size for a decompress (default: the stream tensor's size),
    offsets[i] an optional int64 CUDA tensor of nblocks + 1 block offsets, and
    header_mask the ZFP_HEADER_* bits of the header each stream carries (an
    int for all items, or one per item; 0 = none).
    """
    n = len(fields)
    items = (ZfpBatchItem * n)()
    for i in range(n):
        f, st = fields[i], streams[i]
        items[i].desc = desc_of(f.shape, _np_dtype(f.dtype), configs[i])
        items[i].d_field = f.data_ptr()
        items[i].d_stream = st.data_ptr()
        items[i].stream_bytes = nbytes[i] if nbytes is not None else st.numel() * st.element_size()
        o = offsets[i] if offsets is not None else None
        items[i].d_block_offsets = o.data_ptr() if o is not None else None
        items[i].header_mask = header_mask[i] if isinstance(header_mask, (list, tuple)) else header_mask
    return items


def compress_batch(items, stream=None):
    """zfpb_compress_batch over `items` (from batch_items); returns each item's stream bytes."""
    import torch

    cs = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    ok = lib().zfpb_compress_batch(items, len(items), cs)
    if ok != len(items):
        raise ZfpError("compress_batch", lib().zfpb_last_error())
    return [it.result for it in items]


def decompress_batch(items, stream=None):
    """zfpb_decompress_batch over `items`; returns the bytes each item consumed."""
    import torch

    cs = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    ok = lib().zfpb_decompress_batch(items, len(items), cs)
    if ok != len(items):
        raise ZfpError("decompress_batch", lib().zfpb_last_error())
    return [it.result for it in items]


class Server:
    """The serving loop (zfpb_server_*): submit requests, poll results."""

    def __init__(self, budget_bytes: int, lanes: int = 0, max_batch: int = 0, batch_bytes: int = 0):
        self.h = lib().zfpb_server_create(budget_bytes, lanes, max_batch, batch_bytes)
        if not self.h:
            raise ZfpError("server_create", lib().zfpb_last_error())
        self._keep = {}

    def submit(self, item: "ZfpBatchItem", decompress: bool, tag: int) -> bool:
        ok = lib().zfpb_server_submit(self.h, C.byref(item), int(decompress), tag)
        if ok:
            self._keep[tag] = item
        return bool(ok)

    def poll(self, max_n: int = 256, wait_ms: int = 0):
        out = (ZfpRequestDone * max_n)()
        n = lib().zfpb_server_poll(self.h, out, max_n, wait_ms)
        res = [(d.tag, d.result, d.status, d.queue_ms, d.latency_ms) for d in out[:n]]
        for r in res:
            self._keep.pop(r[0], None)
        return res

    def outstanding(self) -> int:
        return lib().zfpb_server_outstanding(self.h)

    def close(self):
        if self.h:
            lib().zfpb_server_destroy(self.h)
            self.h = None
