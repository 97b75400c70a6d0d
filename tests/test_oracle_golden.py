"""Pin the CPU oracle against the reference's golden checksum tables.

Follows zfp-rs tests/c/encode_block.rs, decode_block.rs,
encode_block_strided.rs and decode_block_strided.rs: 16 (dims, type) pairs,
fixed-rate blocks with maxbits = 19 * 4^dims, partial strided blocks, and the
ten IEEE special-value blocks in reversible mode.
"""

import ctypes as C

import numpy as np
import pytest

from oracle import py_oracle as orc
from tests import zfp_checks as zc

PAIRS = [(d, t) for d in (1, 2, 3, 4) for t in ("int32", "int64", "float", "double")]


def fixed_rate_cfg(dims):
    mb = (4 ** dims) * zc.RATE_PARAM_BITS
    return orc.config(mb, mb, 64, -1074)


def encode_block(arr, tname, dims, strides, lengths, cfg):
    words = np.zeros(4096, dtype=np.uint64)
    s = orc.Stream(words)
    st = (C.c_ssize_t * 4)(*(list(strides) + [0] * (4 - len(strides))))
    ln = None if lengths is None else (C.c_size_t * 4)(*(list(lengths) + [0] * (4 - len(lengths))))
    code = {"int32": 1, "int64": 2, "float": 3, "double": 4}[tname]
    bits = orc.lib().orc_encode_block(s.h, code, dims, arr.ctypes.data, st, ln, C.byref(cfg))
    assert bits == s.wtell()
    s.flush()
    return s, words, bits


def decode_block(words, tname, dims, out, strides, lengths, cfg):
    s = orc.Stream(words)
    st = (C.c_ssize_t * 4)(*(list(strides) + [0] * (4 - len(strides))))
    ln = None if lengths is None else (C.c_size_t * 4)(*(list(lengths) + [0] * (4 - len(lengths))))
    code = {"int32": 1, "int64": 2, "float": 3, "double": 4}[tname]
    bits = orc.lib().orc_decode_block(s.h, code, dims, out.ctypes.data, st, ln, C.byref(cfg))
    assert bits == s.rtell()
    return bits


def nlen(dims):
    return [4] * dims + [0] * (4 - dims)


@pytest.mark.parametrize("dims,tname", PAIRS)
def test_seeded_input_matches_golden(dims, tname):
    blk = zc.random_block(tname, dims)
    k1, k2 = zc.compute_key(zc.BLOCK_FULL, zc.ORIGINAL, nlen(dims), zc.MODE_NULL, 0)
    assert zc.hash_array(blk) == zc.golden(dims, tname, k1, k2)


@pytest.mark.parametrize("dims,tname", PAIRS)
def test_full_block_stream_and_decode_match_golden(dims, tname):
    blk = zc.random_block(tname, dims)
    cfg = fixed_rate_cfg(dims)
    s, words, bits = encode_block(blk, tname, dims, [1, 4, 16, 64][:dims], None, cfg)
    assert bits == (4 ** dims) * zc.RATE_PARAM_BITS
    k1, k2 = zc.compute_key(zc.BLOCK_FULL, zc.COMPRESSED, nlen(dims), zc.MODE_FIXED_RATE, 0)
    assert hex(zc.hash_bitstream(s.bytes())) == hex(zc.golden(dims, tname, k1, k2))
    out = np.zeros_like(blk)
    decode_block(words, tname, dims, out, [1, 4, 16, 64][:dims], None, cfg)
    k1, k2 = zc.compute_key(zc.BLOCK_FULL, zc.DECOMPRESSED, nlen(dims), zc.MODE_FIXED_RATE, 0)
    assert hex(zc.hash_array(out)) == hex(zc.golden(dims, tname, k1, k2))


@pytest.mark.parametrize("dims,tname", PAIRS)
def test_strided_full_block_equals_contiguous(dims, tname):
    data = zc.strided_array(tname, dims)
    k1, k2 = zc.compute_key(zc.BLOCK_FULL, zc.ORIGINAL, nlen(dims), zc.MODE_NULL, 0)
    assert zc.hash_strided(data, nlen(dims), list(zc.STRIDES[:dims]) + [0] * (4 - dims)) == zc.golden(
        dims, tname, k1, k2)
    cfg = fixed_rate_cfg(dims)
    s, _, _ = encode_block(data, tname, dims, zc.STRIDES[:dims], None, cfg)
    k1, k2 = zc.compute_key(zc.BLOCK_FULL, zc.COMPRESSED, nlen(dims), zc.MODE_FIXED_RATE, 0)
    assert zc.hash_bitstream(s.bytes()) == zc.golden(dims, tname, k1, k2)


@pytest.mark.parametrize("dims,tname", PAIRS)
def test_partial_strided_block_matches_golden(dims, tname):
    data = zc.strided_array(tname, dims)
    cfg = fixed_rate_cfg(dims)
    lengths = zc.PARTIAL[:dims]
    s, words, _ = encode_block(data, tname, dims, zc.STRIDES[:dims], lengths, cfg)
    k1, k2 = zc.compute_key(zc.BLOCK_PARTIAL, zc.COMPRESSED, nlen(dims), zc.MODE_FIXED_RATE, 0)
    assert hex(zc.hash_bitstream(s.bytes())) == hex(zc.golden(dims, tname, k1, k2))
    out = np.zeros_like(data)
    decode_block(words, tname, dims, out, zc.STRIDES[:dims], lengths, cfg)
    k1, k2 = zc.compute_key(zc.BLOCK_PARTIAL, zc.DECOMPRESSED, nlen(dims), zc.MODE_FIXED_RATE, 0)
    st = list(zc.STRIDES[:dims]) + [0] * (4 - dims)
    assert hex(zc.hash_strided(out, nlen(dims), st)) == hex(zc.golden(dims, tname, k1, k2))
    # Only entries inside the partial block are written.
    mask = np.zeros(out.size, dtype=bool)
    for idx in np.ndindex(*reversed(lengths)):
        rev = list(reversed(idx))
        mask[sum(rev[d] * zc.STRIDES[d] for d in range(dims))] = True
    assert np.all(out[~mask] == 0)


@pytest.mark.parametrize("dims,tname", [(d, t) for d in (1, 2, 3, 4) for t in ("float", "double")])
def test_special_value_blocks_reversible_match_golden(dims, tname):
    cfg = orc.config(1, 16658, 64, -1075)  # ZfpConfig::reversible (config.rs:337-339)
    for i in range(10):
        blk = zc.special_block(tname, dims, i)
        s, words, _ = encode_block(blk, tname, dims, [1, 4, 16, 64][:dims], None, cfg)
        k1, k2 = zc.compute_key(zc.BLOCK_FULL, zc.COMPRESSED, nlen(dims), zc.MODE_REVERSIBLE, i + 1)
        assert hex(zc.hash_bitstream(s.bytes())) == hex(zc.golden(dims, tname, k1, k2)), i
        out = np.zeros_like(blk)
        decode_block(words, tname, dims, out, [1, 4, 16, 64][:dims], None, cfg)
        assert out.view(np.uint8).tobytes() == blk.view(np.uint8).tobytes()
