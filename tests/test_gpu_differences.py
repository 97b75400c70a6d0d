"""The documented differences from C zfp, through the GPU path.

zfp-rs departs from C zfp in a few corner cases and pins its own behaviour
with known answers (tests/proptest/differences.rs:43-227,
docs/differences-from-c.md:101-168): blocks whose max_bits is below the block
header, reversible all-zero blocks padded to min_bits, maximum_size for such
configs, tiny blocks, and 4-D fields.  These tests run the same cases through
libzfp_b200.so's zfp_compress / zfp_decompress (the GPU) and compare with the
known answers and with the oracle.
"""

import ctypes as C

import numpy as np
import pytest

from oracle import py_oracle as orc
from tests import zfpb

pytestmark = pytest.mark.gpu
Z = zfpb.load()


def values():
    return np.array([np.sin(0.37 * i) * 100.0 for i in range(16)], dtype=np.float64)


def both(data, params):
    cfg = Z.ZfpConfig(*params)
    want, n = orc.compress(data, orc.config(*params))
    got = Z.compress(data, cfg)
    assert got == want
    out_g = np.zeros_like(data)
    out_o = np.zeros_like(data)
    assert Z.decompress(got, out_g, cfg) == n
    assert orc.decompress(want, out_o, orc.config(*params)) == n
    assert out_g.tobytes() == out_o.tobytes()
    return got, out_g


@pytest.mark.parametrize("params,nbytes", [((1, 11, 64, -1074), 8), ((12, 12, 64, -1074), 8),
                                           ((1, 18, 64, -1075), 16), ((19, 19, 64, -1075), 16)])
def test_max_bits_below_the_header(params, nbytes):
    got, _ = both(values(), params)
    assert len(got) == nbytes


def test_reversible_zero_blocks_are_padded():
    data = values()
    data[:4] = 0
    for min_bits in [2, 3, 17, 64, 100, 127, 128, 1000, 16658]:
        got, out = both(data, (min_bits, 16658, 64, -1075))
        assert out.tobytes() == data.tobytes()
        if min_bits == 100:
            assert len(got) == 104
    got, out = both(data, (1, 16658, 64, -1075))
    assert len(got) == 96 and out.tobytes() == data.tobytes()


def test_maximum_size_holds_blocks_longer_than_max_bits():
    cfg = Z.ZfpConfig(1, 11, 64, -1074)
    assert Z.maximum_size((16,), np.float64, cfg) == 32
    got, _ = both(values(), (1, 11, 64, -1074))
    assert len(got) <= 32


def fmt_err(a, b):
    return f"{float(np.max(np.abs(a.astype(np.float64) - b.astype(np.float64)))):.1e}"


def test_tiny_blocks_keep_their_values():
    tiny32 = np.array([(np.float32(i) - np.float32(7.5)) * np.float32(1.0e-31) for i in range(16)],
                      dtype=np.float32)
    tiny64 = values() * 1.0e-300
    for data, params, nbytes, err in [(tiny32, (1, 16658, 16, -1074), 32, "3.1e-35"),
                                      (tiny32, (32, 32, 64, -1074), 16, "6.1e-33"),
                                      (tiny64, (1, 16658, 16, -1074), 40, "1.1e-302")]:
        got, out = both(data, params)
        assert (len(got), fmt_err(data, out)) == (nbytes, err)


@pytest.mark.parametrize("dtype", [np.int32, np.int64, np.float32, np.float64])
@pytest.mark.parametrize("params", [(1, 16658, 64, -1075), (30, 900, 40, -60), (1, 16658, 24, -1074)])
def test_4d_fields_without_an_index(dtype, params):
    """A 4-D stream decoded on the GPU without its block offsets (the walk)."""
    import torch

    rng = np.random.default_rng(4)
    shape = (7, 9, 6, 11)
    v = np.sin(0.2 * np.arange(np.prod(shape))).reshape(shape) + rng.normal(0, 1e-3, shape)
    arr = (v * (2 ** 20 if np.dtype(dtype).kind == "i" else 100)).astype(dtype)
    want, n = orc.compress(arr, orc.config(*params))
    ref = np.zeros_like(arr)
    assert orc.decompress(want, ref, orc.config(*params)) == n
    words = np.zeros((n + 7) // 8, dtype=np.uint64)
    words.view(np.uint8)[:n] = np.frombuffer(want, dtype=np.uint8)
    s = torch.from_numpy(words.view(np.int64)).cuda()
    y = torch.zeros(shape, dtype=getattr(torch, np.dtype(dtype).name), device="cuda")
    assert Z.decompress_device(s, n, y, Z.ZfpConfig(*params)) == n
    assert y.cpu().numpy().tobytes() == ref.tobytes()
