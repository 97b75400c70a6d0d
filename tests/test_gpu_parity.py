"""GPU parity: streams byte-identical and decoded arrays bit-identical to the oracle.

Every case compresses the same seeded input with the oracle (the CPU
restatement of zfp-rs) and through libzfp_b200.so's zfp_compress, then
decompresses each stream with both.  Cases follow the reference's test
matrix (tests/c/endtoend.rs:180-191 mode parameters, tests/proptest/*):
all four scalar types and 1-4 dimensions, partial blocks, strides, headers,
every mode and rounding.
"""

import ctypes as C

import numpy as np
import pytest

from oracle import py_oracle as orc
from tests import zfp_checks as zc
from tests import zfpb

pytestmark = pytest.mark.gpu
Z = zfpb.load()

DTYPES = [np.int32, np.int64, np.float32, np.float64]
SHAPES = {1: [(37,), (64,)], 2: [(13, 10), (16, 16)], 3: [(9, 7, 6), (8, 8, 12)], 4: [(5, 4, 6, 3)]}


def smooth(shape, dtype, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    grids = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in shape], indexing="ij")
    v = np.ones(shape)
    for i, g in enumerate(grids):
        v = v * np.sin(0.1 * (i + 1) * g + 0.3 * i)
    v = v + rng.normal(0, 1e-3, size=shape)
    if np.dtype(dtype).kind == "i":
        big = 2 ** 20 if dtype == np.int32 else 2 ** 40
        return (v * big).astype(dtype)
    return (v * scale).astype(dtype)


def oracle_cfg(c):
    return orc.config(c.min_bits, c.max_bits, c.max_prec, c.min_exp, c.rounding, c.tight_error)


def configs_for(dtype, dims):
    out = []
    for rate in (1.5, 4, 8, 19, 32):
        try:
            out.append(Z.ZfpConfig.fixed_rate(rate, dtype, dims))
        except ValueError:
            pass
    out.append(Z.ZfpConfig.fixed_rate(8, dtype, dims, word_aligned=True))
    out += [Z.ZfpConfig.fixed_precision(p) for p in (4, 16, 32, 64)]
    if np.dtype(dtype).kind == "f":
        out += [Z.ZfpConfig.fixed_accuracy(t) for t in (1e-2, 1e-6, 2.0 ** -30)]
    out.append(Z.ZfpConfig.reversible())
    out.append(Z.ZfpConfig.expert(20, 300, 24, -40))
    return out


ROUNDINGS = [("never", False), ("first", False), ("first", True), ("last", False), ("last", True)]


def check(arr, cfg, **kw):
    ocfg = oracle_cfg(cfg)
    want, n = orc.compress(arr, ocfg, header_mask=7 if kw.get("header") else 0,
                           dims=kw.get("dims"), strides=kw.get("strides"), data_ptr=kw.get("data_ptr"))
    assert n > 0
    got = Z.compress(arr, cfg, **kw)
    assert got == want, f"stream differs for {cfg}"
    out_o = np.zeros_like(arr)
    out_g = np.zeros_like(arr)
    skip = 0
    if kw.get("header"):
        words = np.frombuffer(want[:16].ljust(16, b"\0"), dtype=np.uint64)
        skip = 96 if (int(words[1]) >> 20) & 0xFFF <= 4094 else 148
    optr = kw.get("data_ptr")
    k2 = dict(kw)
    if optr is not None:
        k2["data_ptr"] = out_g.ctypes.data + (optr - arr.ctypes.data)
    oo = dict(dims=kw.get("dims"), strides=kw.get("strides"))
    if optr is not None:
        oo["data_ptr"] = out_o.ctypes.data + (optr - arr.ctypes.data)
    used_o = orc.decompress(want, out_o, ocfg, skip_bits=skip, **oo)
    used_g = Z.decompress(got, out_g, cfg, **{k: v for k, v in k2.items()})
    assert used_o == used_g == n
    assert out_g.tobytes() == out_o.tobytes()
    return got


@pytest.mark.parametrize("dtype", DTYPES, ids=lambda d: np.dtype(d).name)
@pytest.mark.parametrize("dims", [1, 2, 3, 4])
def test_every_mode_matches_oracle(dtype, dims):
    for si, shape in enumerate(SHAPES[dims]):
        arr = smooth(shape, dtype, seed=dims * 10 + si, scale=1e3)
        for cfg in configs_for(dtype, dims):
            check(arr, cfg)


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.int32], ids=lambda d: np.dtype(d).name)
@pytest.mark.parametrize("rounding,tight", ROUNDINGS)
def test_rounding_modes_match_oracle(dtype, rounding, tight):
    arr = smooth((10, 9, 11), dtype, seed=5, scale=7.0)
    for cfg in [Z.ZfpConfig.fixed_rate(6, dtype, 3), Z.ZfpConfig.fixed_precision(20),
                Z.ZfpConfig.fixed_accuracy(1e-4), Z.ZfpConfig.reversible()]:
        check(arr, cfg.with_rounding(rounding, tight))


@pytest.mark.parametrize("dtype", DTYPES, ids=lambda d: np.dtype(d).name)
def test_header_offsets_match_oracle(dtype):
    arr = smooth((12, 11, 10), dtype, seed=3)
    for cfg in [Z.ZfpConfig.fixed_rate(8, dtype, 3), Z.ZfpConfig.fixed_rate(3, dtype, 3),
                Z.ZfpConfig.fixed_precision(12), Z.ZfpConfig.expert(1, 4000, 30, -1000)]:
        check(arr, cfg, header=True)


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.int64], ids=lambda d: np.dtype(d).name)
@pytest.mark.parametrize("nx", [6, 7], ids=["disjoint", "aliasing"])
def test_strided_and_negative_strides_match_oracle(dtype, nx):
    """Every other x, reversed y, a sub-volume of a larger array.

    With nx = 7 the x range (13 elements) overlaps the next row (stride 12):
    two blocks hold the same element, and, as in the reference's serial
    decode (decompress.rs:153-186), the later block's value is kept.
    """
    base = smooth((14, 13, 12), dtype, seed=9)
    nz, ny = 5, 6
    sx, sy, sz = 2, -base.shape[2], base.shape[1] * base.shape[2]
    origin = base.ctypes.data + ((ny - 1) * base.shape[2]) * base.itemsize
    for cfg in [Z.ZfpConfig.fixed_rate(10, dtype, 3), Z.ZfpConfig.fixed_precision(18), Z.ZfpConfig.reversible()]:
        check(base, cfg, dims=(nx, ny, nz), strides=(sx, sy, sz), data_ptr=origin)


def test_special_values_and_tiny_blocks_match_oracle():
    rng = np.random.default_rng(1)
    for dtype, bits in [(np.float32, zc.SPECIAL_FLOAT_BITS), (np.float64, zc.SPECIAL_DOUBLE_BITS)]:
        arr = smooth((8, 8, 8), dtype, seed=2)
        flat = arr.reshape(-1).view(np.uint32 if dtype == np.float32 else np.uint64)
        idx = rng.choice(flat.size, size=40, replace=False)
        flat[idx] = rng.choice(np.array(bits, dtype=flat.dtype), size=40)
        for cfg in [Z.ZfpConfig.fixed_rate(12, dtype, 3), Z.ZfpConfig.fixed_precision(30), Z.ZfpConfig.reversible()]:
            check(arr, cfg)
        tiny = (smooth((8, 8, 8), dtype, seed=4) * (1e-33 if dtype == np.float32 else 1e-300)).astype(dtype)
        for cfg in [Z.ZfpConfig.fixed_rate(8, dtype, 3), Z.ZfpConfig.fixed_precision(16), Z.ZfpConfig.reversible()]:
            check(tiny, cfg)


def test_golden_blocks_through_the_gpu():
    """A one-block field reproduces the reference's block checksums (0xa0, 0x2a0)."""
    for dims in (1, 2, 3, 4):
        for tname, dtype in zc.ZFP_TYPES.items():
            mb = (4 ** dims) * zc.RATE_PARAM_BITS
            cfg = Z.ZfpConfig.expert(mb, mb, 64, -1074)
            blk = zc.random_block(tname, dims)
            got = Z.compress(blk, cfg, dims=(4,) * dims)
            k1, k2 = zc.compute_key(zc.BLOCK_FULL, zc.COMPRESSED, [4] * dims + [0] * (4 - dims), zc.MODE_FIXED_RATE, 0)
            assert zc.hash_bitstream(got) == zc.golden(dims, tname, k1, k2)
            data = zc.strided_array(tname, dims)
            got = Z.compress(data, cfg, dims=zc.PARTIAL[:dims], strides=zc.STRIDES[:dims])
            k1, k2 = zc.compute_key(zc.BLOCK_PARTIAL, zc.COMPRESSED, [4] * dims + [0] * (4 - dims),
                                    zc.MODE_FIXED_RATE, 0)
            assert zc.hash_bitstream(got) == zc.golden(dims, tname, k1, k2)


def test_foreign_variable_rate_stream_decodes_without_an_index():
    """A stream this library did not write is walked for block offsets."""
    for dtype in DTYPES:
        arr = smooth((11, 10, 9), dtype, seed=8)
        for cfg in [Z.ZfpConfig.fixed_precision(22), Z.ZfpConfig.reversible()]:
            stream, n = orc.compress(arr, oracle_cfg(cfg))
            out = np.zeros_like(arr)
            assert Z.decompress(stream, out, cfg) == n
            ref = np.zeros_like(arr)
            orc.decompress(stream, ref, oracle_cfg(cfg))
            assert out.tobytes() == ref.tobytes()


def test_truncated_stream_and_small_buffer_fail_like_the_reference():
    arr = smooth((16, 16, 16), np.float32, seed=6)
    for cfg in [Z.ZfpConfig.fixed_rate(8, np.float32, 3), Z.ZfpConfig.fixed_precision(20)]:
        stream = Z.compress(arr, cfg)
        cut = stream[: len(stream) // 2]
        out = np.zeros_like(arr)
        assert orc.decompress(cut, np.zeros_like(arr), oracle_cfg(cfg)) == -1
        with pytest.raises(Z.ZfpError) as e:
            Z.decompress(cut, out, cfg)
        assert e.value.code == 2
        with pytest.raises(Z.ZfpError) as e:
            Z.compress(arr, cfg, capacity=len(stream) // 2)
        assert e.value.code == 1


def test_device_api_round_trip_and_index():
    import torch

    dev = torch.device("cuda:0")
    for dtype, tdt in [(np.float32, torch.float32), (np.float64, torch.float64)]:
        arr = smooth((24, 20, 28), dtype, seed=12)
        x = torch.from_numpy(arr).to(dev)
        for cfg in [Z.ZfpConfig.fixed_rate(8, dtype, 3), Z.ZfpConfig.fixed_accuracy(1e-5)]:
            cap = Z.maximum_size(arr, dtype, cfg)
            out = torch.zeros((cap + 7) // 8, dtype=torch.int64, device=dev)
            nb = (24 // 4) * (20 // 4) * (28 // 4)
            off = torch.zeros(nb + 1, dtype=torch.int64, device=dev)
            n = Z.compress_device(x, cfg, out=out, offsets=off)
            want, wn = orc.compress(arr, oracle_cfg(cfg))
            assert n == wn and out.cpu().numpy().view(np.uint8)[:n].tobytes() == want
            y = torch.zeros_like(x)
            assert Z.decompress_device(out, n, y, cfg, offsets=off) == n
            ref = np.zeros_like(arr)
            orc.decompress(want, ref, oracle_cfg(cfg))
            assert y.cpu().numpy().tobytes() == ref.tobytes()
            # A wrong index is detected and the offsets recomputed.
            if cfg.min_bits != cfg.max_bits:
                bad = off.clone()
                bad[5] += 3
                y.zero_()
                assert Z.decompress_device(out, n, y, cfg, offsets=bad) == n
                assert y.cpu().numpy().tobytes() == ref.tobytes()


def test_device_resident_zfp_field_and_stream():
    """zfp_compress/zfp_decompress with field and stream in device memory."""
    import torch

    L = Z.lib()
    arr = smooth((16, 12, 20), np.float32, seed=21)
    cfg = Z.ZfpConfig.fixed_precision(18)
    x = torch.from_numpy(arr).cuda()
    buf = torch.zeros(200000, dtype=torch.int64, device="cuda")
    bs = L.stream_open(buf.data_ptr(), buf.numel() * 8)
    zs = L.zfp_stream_open(bs)
    L.zfp_stream_set_params(zs, cfg.min_bits, cfg.max_bits, cfg.max_prec, cfg.min_exp)
    f = L.zfp_field_3d(x.data_ptr(), 3, 20, 12, 16)
    assert L.zfp_write_header(zs, f, 7) == 96
    n = L.zfp_compress(zs, f)
    want, wn = orc.compress(arr, oracle_cfg(cfg), header_mask=7)
    assert n == wn and buf.cpu().numpy().view(np.uint8)[:n].tobytes() == want
    L.zfp_stream_rewind(zs)
    y = torch.zeros_like(x)
    g = L.zfp_field_alloc()
    assert L.zfp_read_header(zs, g, 7) == 96
    L.zfp_field_set_pointer(g, y.data_ptr())
    assert L.zfp_decompress(zs, g) == n
    ref = np.zeros_like(arr)
    orc.decompress(want, ref, oracle_cfg(cfg), skip_bits=96)
    assert y.cpu().numpy().tobytes() == ref.tobytes()
    for p in (f, g):
        L.zfp_field_free(p)
    L.zfp_stream_close(zs)
    L.stream_close(bs)


def spiky(n, dtype, seed):
    """A bench-like field: smooth x1e3 + noise, 10% zero blocks, 1% spikes."""
    rng = np.random.default_rng(seed)
    x = np.arange(n, dtype=np.float64)
    f = np.sin(0.10 * x)[None, None, :] * np.cos(0.13 * x)[None, :, None] * np.sin(0.07 * x)[:, None, None]
    f = (f + rng.normal(0, 1e-3, size=(n, n, n))) * 1e3
    nb = n // 4
    zero = rng.random((nb, nb, nb)) < 0.10
    f.reshape(nb, 4, nb, 4, nb, 4)[zero[:, None, :, None, :, None].repeat(4, 1).repeat(4, 3).repeat(4, 5)] = 0.0
    spikes = rng.random(f.shape) < 0.01
    k = int(spikes.sum())
    f[spikes] = rng.choice([-1.0, 1.0], size=k) * 10.0 ** rng.uniform(-30, 30, size=k)
    return f.astype(dtype)


@pytest.mark.parametrize("dtype", [np.float32, np.float64], ids=lambda d: np.dtype(d).name)
def test_spiky_field_many_blocks_matches_oracle(dtype):
    arr = spiky(48, dtype, seed=4)
    for cfg in [Z.ZfpConfig.fixed_accuracy(1e-6), Z.ZfpConfig.fixed_precision(32).with_rounding("last", True),
                Z.ZfpConfig.fixed_rate(8, dtype, 3), Z.ZfpConfig.fixed_rate(21, dtype, 3).with_rounding("last"),
                Z.ZfpConfig.reversible()]:
        check(arr, cfg)


@pytest.mark.parametrize("dtype", DTYPES, ids=lambda d: np.dtype(d).name)
def test_one_kernel_decoder_matches_two_kernel_decoder(dtype, monkeypatch):
    """3D fields decode with k_parse + k_finish; ZFPB_ONE_KERNEL_DECODE=1
    selects the one-kernel decoder (used for other dimensions and when the
    plane scratch cannot be allocated).  Both must give the oracle's values."""
    arr = spiky(24, dtype, seed=8) if np.dtype(dtype).kind == "f" else smooth((24, 20, 16), dtype, seed=8)
    cfgs = [Z.ZfpConfig.fixed_rate(7, dtype, 3), Z.ZfpConfig.fixed_precision(24).with_rounding("last"),
            Z.ZfpConfig.reversible(), Z.ZfpConfig.expert(30, 900, 40, -60)]
    if np.dtype(dtype).kind == "f":
        cfgs.append(Z.ZfpConfig.fixed_accuracy(1e-5).with_rounding("first", True))
    for cfg in cfgs:
        monkeypatch.setenv("ZFPB_ONE_KERNEL_DECODE", "1")
        a = check(arr, cfg)
        monkeypatch.delenv("ZFPB_ONE_KERNEL_DECODE")
        assert check(arr, cfg) == a
