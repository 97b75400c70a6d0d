"""Block-level C ABI (include/zfp_block.h) and the batched block calls.

The reference exports zfp_encode_block_*, zfp_decode_block_*, their strided
and partial variants (zfp-rs-ffi/src/block.rs:34-776) and zfp_promote_* /
zfp_demote_* (zfp-rs-ffi/src/promote.rs).  The GPU tests reproduce the
reference's golden block checksums through these symbols, as its own tests
do through the same calls (tests/c/encode_block.rs, decode_block.rs,
encode_block_strided.rs, decode_block_strided.rs): full fixed-rate blocks
(key 0xa0 / 0x120), partial strided blocks (0x2a0 / 0x320) and the
special-value blocks in reversible mode.  Variable-rate block sequences and
zfpb_encode_blocks / zfpb_decode_blocks are compared with the oracle's
block coder.  Promotion and demotion are host maps, tested on the CPU.
"""

import ctypes as C

import numpy as np
import pytest

from oracle import py_oracle as orc
from tests import zfp_checks as zc
from tests import zfpb

Z = zfpb.load()
PAIRS = [(d, t) for d in (1, 2, 3, 4) for t in ("int32", "int64", "float", "double")]
CONTIG = (1, 4, 16, 64)


def nlen(dims):
    return [4] * dims + [0] * (4 - dims)


class HostStream:
    """A zfp_stream over a host word buffer, with expert parameters."""

    def __init__(self, params, words=None, rounding=("never", False)):
        L = Z.lib()
        self.words = np.zeros(8192, dtype=np.uint64) if words is None else words
        self.bs = L.stream_open(self.words.ctypes.data, self.words.nbytes)
        self.zs = L.zfp_stream_open(self.bs)
        z = self.zs.contents
        z.minbits, z.maxbits, z.maxprec, z.minexp = params
        L.zfp_stream_set_rounding(self.zs, Z.ZfpConfig(*params, *rounding).rounding_code, int(rounding[1]))

    def bytes(self):
        return self.words.view(np.uint8)[: Z.lib().stream_size(self.bs)].tobytes()

    def close(self):
        Z.lib().zfp_stream_close(self.zs)
        Z.lib().stream_close(self.bs)


def call(kind, tname, dims, zs, arr, strides=None, lengths=None):
    fn = getattr(Z.lib(), {"enc": "zfp_encode_block", "dec": "zfp_decode_block",
                           "enc_s": "zfp_encode_block_strided", "dec_s": "zfp_decode_block_strided",
                           "enc_p": "zfp_encode_partial_block_strided",
                           "dec_p": "zfp_decode_partial_block_strided"}[kind] + f"_{tname}_{dims}")
    args = [zs, arr.ctypes.data]
    if lengths is not None:
        args += list(lengths[:dims])
    if strides is not None:
        args += list(strides[:dims])
    return fn(*args)


def rate_params(dims):
    mb = (4 ** dims) * zc.RATE_PARAM_BITS
    return (mb, mb, 64, -1074)


@pytest.mark.gpu
@pytest.mark.parametrize("dims,tname", PAIRS)
def test_full_blocks_reproduce_the_golden_checksums(dims, tname):
    blk = zc.random_block(tname, dims)
    s = HostStream(rate_params(dims))
    bits = call("enc", tname, dims, s.zs, blk)
    assert bits == (4 ** dims) * zc.RATE_PARAM_BITS
    assert Z.lib().stream_flush(s.bs) >= 0
    k1, k2 = zc.compute_key(zc.BLOCK_FULL, zc.COMPRESSED, nlen(dims), zc.MODE_FIXED_RATE, 0)
    assert hex(zc.hash_bitstream(s.bytes())) == hex(zc.golden(dims, tname, k1, k2))
    Z.lib().zfp_stream_rewind(s.zs)
    out = np.zeros_like(blk)
    assert call("dec", tname, dims, s.zs, out) == bits
    k1, k2 = zc.compute_key(zc.BLOCK_FULL, zc.DECOMPRESSED, nlen(dims), zc.MODE_FIXED_RATE, 0)
    assert hex(zc.hash_array(out)) == hex(zc.golden(dims, tname, k1, k2))
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("dims,tname", PAIRS)
def test_strided_and_partial_blocks_reproduce_the_golden_checksums(dims, tname):
    data = zc.strided_array(tname, dims)
    st = zc.STRIDES
    s = HostStream(rate_params(dims))
    call("enc_s", tname, dims, s.zs, data, strides=st)
    Z.lib().stream_flush(s.bs)
    k1, k2 = zc.compute_key(zc.BLOCK_FULL, zc.COMPRESSED, nlen(dims), zc.MODE_FIXED_RATE, 0)
    assert zc.hash_bitstream(s.bytes()) == zc.golden(dims, tname, k1, k2)
    s.close()
    # Partial block: encode, then decode into a zeroed array of the same layout.
    s = HostStream(rate_params(dims))
    call("enc_p", tname, dims, s.zs, data, strides=st, lengths=zc.PARTIAL)
    Z.lib().stream_flush(s.bs)
    k1, k2 = zc.compute_key(zc.BLOCK_PARTIAL, zc.COMPRESSED, nlen(dims), zc.MODE_FIXED_RATE, 0)
    assert hex(zc.hash_bitstream(s.bytes())) == hex(zc.golden(dims, tname, k1, k2))
    Z.lib().zfp_stream_rewind(s.zs)
    out = np.zeros_like(data)
    call("dec_p", tname, dims, s.zs, out, strides=st, lengths=zc.PARTIAL)
    k1, k2 = zc.compute_key(zc.BLOCK_PARTIAL, zc.DECOMPRESSED, nlen(dims), zc.MODE_FIXED_RATE, 0)
    stv = list(st[:dims]) + [0] * (4 - dims)
    assert hex(zc.hash_strided(out, nlen(dims), stv)) == hex(zc.golden(dims, tname, k1, k2))
    mask = np.zeros(out.size, dtype=bool)
    for idx in np.ndindex(*reversed(zc.PARTIAL[:dims])):
        rev = list(reversed(idx))
        mask[sum(rev[d] * st[d] for d in range(dims))] = True
    assert np.all(out[~mask] == 0), "a partial decode wrote outside the block"
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("dims,tname", [(d, t) for d in (1, 2, 3, 4) for t in ("float", "double")])
def test_special_value_blocks_reversible(dims, tname):
    for i in range(10):
        blk = zc.special_block(tname, dims, i)
        s = HostStream((1, 16658, 64, -1075))
        call("enc", tname, dims, s.zs, blk)
        Z.lib().stream_flush(s.bs)
        k1, k2 = zc.compute_key(zc.BLOCK_FULL, zc.COMPRESSED, nlen(dims), zc.MODE_REVERSIBLE, i + 1)
        assert hex(zc.hash_bitstream(s.bytes())) == hex(zc.golden(dims, tname, k1, k2)), i
        Z.lib().zfp_stream_rewind(s.zs)
        out = np.zeros_like(blk)
        call("dec", tname, dims, s.zs, out)
        assert out.view(np.uint8).tobytes() == blk.view(np.uint8).tobytes()
        s.close()


def smooth_blocks(tname, dims, count, seed):
    rng = np.random.default_rng(seed)
    n = 4 ** dims
    v = np.sin(0.3 * np.arange(n * count)) * 100 + rng.normal(0, 1e-2, n * count)
    if tname in ("int32", "int64"):
        v = v * (2 ** 16 if tname == "int32" else 2 ** 36)
    return v.astype(zc.ZFP_TYPES[tname])


VAR_PARAMS = [(1, 16658, 20, -1074), (1, 16658, 64, -20), (1, 16658, 64, -1075), (30, 900, 40, -60)]


@pytest.mark.gpu
@pytest.mark.parametrize("dims,tname", PAIRS)
@pytest.mark.parametrize("params", VAR_PARAMS)
def test_block_sequences_match_the_oracle(dims, tname, params):
    """Five variable-size blocks appended to one stream, then read back one by
    one: bits per call and stream bytes as the oracle's block coder; then the
    same blocks in one zfpb_encode_blocks / zfpb_decode_blocks call."""
    import torch

    n, count = 4 ** dims, 5
    vals = smooth_blocks(tname, dims, count, dims)
    code = {"int32": 1, "int64": 2, "float": 3, "double": 4}[tname]
    ocfg = orc.config(*params, "first", False)
    ow = np.zeros(8192, dtype=np.uint64)
    os_ = orc.Stream(ow)
    s = HostStream(params, rounding=("first", False))
    st = (C.c_ssize_t * 4)(*CONTIG)
    for b in range(count):
        blk = np.ascontiguousarray(vals[b * n:(b + 1) * n])
        want = orc.lib().orc_encode_block(os_.h, code, dims, blk.ctypes.data, st, None, C.byref(ocfg))
        assert call("enc", tname, dims, s.zs, blk) == want
    os_.flush()
    Z.lib().stream_flush(s.bs)
    assert s.bytes() == os_.bytes()
    Z.lib().zfp_stream_rewind(s.zs)
    os_.rewind()
    for b in range(count):
        got = np.zeros(n, dtype=vals.dtype)
        ref = np.zeros(n, dtype=vals.dtype)
        want = orc.lib().orc_decode_block(os_.h, code, dims, ref.ctypes.data, st, None, C.byref(ocfg))
        assert call("dec", tname, dims, s.zs, got) == want
        assert got.tobytes() == ref.tobytes()
    s.close()
    # Batched: the same blocks, one device call each way.
    cfg = Z.ZfpConfig(*params, "first", False)
    desc = Z.desc_of((count * n,), vals.dtype, cfg)
    d_vals = torch.from_numpy(vals).cuda()
    cap = 8 * 8192
    d_stream = torch.zeros(cap // 8, dtype=torch.int64, device="cuda")
    cs = torch.cuda.current_stream().cuda_stream
    nb = Z.lib().zfpb_encode_blocks(C.byref(desc), dims, count, d_vals.data_ptr(), d_stream.data_ptr(), cap, None, cs)
    assert nb == len(os_.bytes())
    assert d_stream.view(torch.uint8)[:nb].cpu().numpy().tobytes() == os_.bytes()
    back = torch.zeros_like(d_vals)
    assert Z.lib().zfpb_decode_blocks(C.byref(desc), dims, count, d_stream.data_ptr(), nb, back.data_ptr(), None,
                                      cs) == nb
    ref = np.zeros_like(vals)
    os_.rewind()
    for b in range(count):
        orc.lib().orc_decode_block(os_.h, code, dims, ref[b * n:].ctypes.data, st, None, C.byref(ocfg))
    assert back.cpu().numpy().tobytes() == ref.tobytes()
    os_.close()


def test_block_calls_reject_null_and_bad_lengths():
    L = Z.lib()
    blk = np.zeros(64, dtype=np.float32)
    assert L.zfp_encode_block_float_3(None, blk.ctypes.data) == 0
    s = HostStream((1, 16658, 64, -1074))
    assert L.zfp_encode_block_float_3(s.zs, None) == 0
    assert L.zfp_encode_partial_block_strided_float_3(s.zs, blk.ctypes.data, 5, 1, 1, 1, 4, 16) == 0
    assert L.zfp_decode_partial_block_strided_float_2(s.zs, blk.ctypes.data, 0, 2, 1, 4) == 0
    s.close()


@pytest.mark.parametrize("dims", [1, 2, 3, 4])
def test_promote_and_demote_match_the_reference_maps(dims):
    """promote.rs: i8 << 23, (u8 - 0x80) << 23, i16 << 15, (u16 - 0x8000) << 15;
    demotion shifts back and clamps."""
    L = Z.lib()
    n = 4 ** dims
    rng = np.random.default_rng(dims)
    for src_t, shift, off, name in ((np.int8, 23, 0, "int8"), (np.uint8, 23, 0x80, "uint8"),
                                    (np.int16, 15, 0, "int16"), (np.uint16, 15, 0x8000, "uint16")):
        info = np.iinfo(src_t)
        src = rng.integers(info.min, info.max + 1, size=n).astype(src_t)
        out = np.full(n + 1, 7, dtype=np.int32)
        getattr(L, f"zfp_promote_{name}_to_int32")(out.ctypes.data, src.ctypes.data, dims)
        want = ((src.astype(np.int64) - off) << shift).astype(np.int32)
        assert np.array_equal(out[:n], want) and out[n] == 7
        wide = rng.integers(-2 ** 31, 2 ** 31, size=n).astype(np.int32)
        wide[:4] = [0x7FFFFFFF, -0x80000000, 0, -1]
        back = np.zeros(n, dtype=src_t)
        getattr(L, f"zfp_demote_int32_to_{name}")(back.ctypes.data, wide.ctypes.data, dims)
        want = np.clip((wide.astype(np.int64) >> shift) + off, info.min, info.max).astype(src_t)
        assert np.array_equal(back, want)
        getattr(L, f"zfp_demote_int32_to_{name}")(back.ctypes.data, want.ctypes.data, 5)  # invalid dims: no-op
        assert np.array_equal(back, want)
