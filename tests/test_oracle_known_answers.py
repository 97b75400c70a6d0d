"""Known answers for whole-field streams from the reference's own tests.

zfp-rs tests/proptest/differences.rs:43-227 (also docs/differences-from-c.md)
gives stream sizes, and the largest decode error of zfp-rs's streams, for 16
values as a 1-D field.  These pin the oracle's variable-rate paths
(expert, reversible, fixed precision) where no checksum table exists.
"""

import numpy as np
import pytest

from oracle import py_oracle as orc


def values():
    return np.array([np.sin(0.37 * i) * 100.0 for i in range(16)], dtype=np.float64)


def roundtrip(data, cfg):
    stream, n = orc.compress(data, cfg)
    out = np.zeros_like(data)
    assert orc.decompress(stream, out, cfg) == n
    return stream, out


@pytest.mark.parametrize("params,nbytes", [((1, 11, 64, -1074), 8), ((12, 12, 64, -1074), 8),
                                           ((1, 18, 64, -1075), 16), ((19, 19, 64, -1075), 16)])
def test_max_bits_below_the_header(params, nbytes):
    stream, n = orc.compress(values(), orc.config(*params))
    assert n == nbytes


def test_reversible_zero_blocks_are_padded():
    data = values()
    data[:4] = 0
    for min_bits in list(range(2, 129)) + [1000, 16658]:
        cfg = orc.config(min_bits, 16658, 64, -1075)
        stream, out = roundtrip(data, cfg)
        assert out.tobytes() == data.tobytes()
        if min_bits == 100:
            assert len(stream) == 104
    stream, out = roundtrip(data, orc.config(1, 16658, 64, -1075))
    assert len(stream) == 96 and out.tobytes() == data.tobytes()


def fmt_err(a, b):
    return f"{float(np.max(np.abs(a.astype(np.float64) - b.astype(np.float64)))):.1e}"


def test_tiny_blocks_keep_their_values():
    tiny32 = np.array([(np.float32(i) - np.float32(7.5)) * np.float32(1.0e-31) for i in range(16)],
                      dtype=np.float32)
    tiny64 = values() * 1.0e-300
    rate8 = (32, 32, 64, -1074)  # fixed_rate(8.0, f32, 1-D): floor(4 * 8 + 0.5) bits
    prec16 = (1, 16658, 16, -1074)  # fixed_precision(16)
    for data, params, nbytes, err in [(tiny32, prec16, 32, "3.1e-35"), (tiny32, rate8, 16, "6.1e-33"),
                                      (tiny64, prec16, 40, "1.1e-302")]:
        stream, out = roundtrip(data, orc.config(*params))
        assert (len(stream), fmt_err(data, out)) == (nbytes, err)


def test_maximum_size_holds_blocks_longer_than_max_bits():
    cfg = orc.config(1, 11, 64, -1074)
    f = orc.field_of(values())
    assert orc.lib().orc_maximum_size(orc.C.byref(cfg), orc.C.byref(f)) == 32
