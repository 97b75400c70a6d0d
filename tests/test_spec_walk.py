"""Decoding variable-rate streams that come without a block index.

The block offsets then come from the speculative parallel walk (segments
walked from guessed starts, fixed up from the previous segment's exit); on
fields large enough to give it several segments (1-D to 4-D), the decoded values must be
bit-identical to a decode with the compressor's index and to one whose
offsets come from the serial one-thread walk (ZFPB_SERIAL_WALK=1), and a
stream cut short must be reported as truncated either way.
"""

import os

import numpy as np
import pytest

from tests import zfpb

pytestmark = pytest.mark.gpu
Z = zfpb.load()


def field(shape, dtype, seed):
    import torch

    g = torch.Generator(device="cuda").manual_seed(seed)
    f = torch.ones(shape, dtype=torch.float64, device="cuda")
    for i, n in enumerate(shape):
        c = torch.arange(n, dtype=torch.float64, device="cuda")
        view = [1] * len(shape)
        view[i] = -1
        f = f * torch.sin((0.1 + 0.03 * i) * c + 0.2 * i).view(view)
    f = f + 1e-3 * torch.randn(shape, dtype=torch.float64, device="cuda", generator=g)
    if dtype in (torch.int32, torch.int64):
        return torch.round(f * 2 ** 20).to(dtype)
    return (f * 100).to(dtype)


CASES = [
    ((1 << 20,), "float32", lambda: Z.ZfpConfig.fixed_accuracy(1e-6)),
    ((300_001,), "float64", lambda: Z.ZfpConfig.fixed_precision(30).with_rounding("first", True)),
    ((200_003,), "int32", lambda: Z.ZfpConfig.reversible()),
    ((400, 515), "float32", lambda: Z.ZfpConfig.fixed_accuracy(1e-4).with_rounding("last")),
    ((310, 270), "float64", lambda: Z.ZfpConfig.expert(8, 900, 40, -30)),
    ((70, 66, 63), "float64", lambda: Z.ZfpConfig.fixed_accuracy(1e-6)),
    ((64, 64, 70), "float32", lambda: Z.ZfpConfig.fixed_precision(20)),
    ((50, 50, 50), "int64", lambda: Z.ZfpConfig.fixed_precision(40)),
    ((24, 28, 32, 36), "float64", lambda: Z.ZfpConfig.fixed_accuracy(1e-6)),
    ((36, 32, 28, 24), "float32", lambda: Z.ZfpConfig.fixed_precision(20).with_rounding("last")),
    ((20, 24, 28, 40), "int32", lambda: Z.ZfpConfig.reversible()),
]


@pytest.mark.parametrize("shape,dtype,cfg", CASES)
def test_decode_without_index_matches(shape, dtype, cfg):
    import torch

    dt = getattr(torch, dtype)
    x = field(shape, dt, seed=len(shape) * 7 + len(dtype))
    c = cfg()
    nb = int(np.prod([(n + 3) // 4 for n in shape]))
    cap = Z.maximum_size(x.shape, Z._np_dtype(x.dtype), c)
    st = torch.zeros((cap + 7) // 8, dtype=torch.int64, device="cuda")
    off = torch.zeros(nb + 1, dtype=torch.int64, device="cuda")
    n = Z.compress_device(x, c, out=st, offsets=off)
    want = torch.zeros_like(x)
    assert Z.decompress_device(st, n, want, c, offsets=off) == n
    got = torch.full_like(x, 3)
    assert Z.decompress_device(st, n, got, c) == n
    assert torch.equal(got.view(torch.uint8), want.view(torch.uint8))
    os.environ["ZFPB_SERIAL_WALK"] = "1"
    try:
        serial = torch.full_like(x, 5)
        assert Z.decompress_device(st, n, serial, c) == n
    finally:
        del os.environ["ZFPB_SERIAL_WALK"]
    assert torch.equal(serial.view(torch.uint8), want.view(torch.uint8))


def test_truncated_stream_without_index():
    import torch

    x = field((1 << 19,), torch.float32, seed=3)
    c = Z.ZfpConfig.fixed_accuracy(1e-6)
    cap = Z.maximum_size(x.shape, np.float32, c)
    st = torch.zeros((cap + 7) // 8, dtype=torch.int64, device="cuda")
    n = Z.compress_device(x, c, out=st)
    short = (n // 2) // 8 * 8
    errs = []
    for serial in (False, True):
        if serial:
            os.environ["ZFPB_SERIAL_WALK"] = "1"
        try:
            with pytest.raises(Z.ZfpError) as e:
                Z.decompress_device(st, short, torch.zeros_like(x), c)
            errs.append(e.value.code)
        finally:
            os.environ.pop("ZFPB_SERIAL_WALK", None)
    assert errs == [2, 2]


def test_batch_without_index_decodes_large_and_small_streams():
    """A batch of streams without an index: large ones (decoded alone, by the
    speculative walk) and small ones (walked in the batch) give what a decode
    with the compressor's index gives; so do their headers."""
    import torch

    specs = [((1 << 18,), torch.float32, Z.ZfpConfig.fixed_accuracy(1e-5)),
             ((3000,), torch.float64, Z.ZfpConfig.fixed_precision(24)),
             ((260, 300), torch.float32, Z.ZfpConfig.fixed_precision(18)),
             ((40, 30), torch.float64, Z.ZfpConfig.fixed_accuracy(1e-7)),
             ((90, 100, 80), torch.float64, Z.ZfpConfig.fixed_accuracy(1e-6).with_rounding("first")),
             ((9, 10, 11), torch.float32, Z.ZfpConfig.reversible())]
    fields, cfgs, streams = [], [], []
    for k, (shape, dt, c) in enumerate(specs):
        x = field(shape, dt, seed=50 + k)
        cap = Z.maximum_size(x.shape, Z._np_dtype(x.dtype), c)
        st = torch.zeros((cap + 7) // 8, dtype=torch.int64, device="cuda")
        fields.append(x)
        cfgs.append(c)
        streams.append(st)
    items = Z.batch_items(fields, cfgs, streams, header_mask=7)
    sizes = Z.compress_batch(items)
    outs = [torch.full_like(x, 9) for x in fields]
    used = Z.decompress_batch(Z.batch_items(outs, cfgs, streams, nbytes=sizes, header_mask=7))
    assert used == sizes
    for k, x in enumerate(fields):
        nb = int(np.prod([(n + 3) // 4 for n in x.shape]))
        off = torch.zeros(nb + 1, dtype=torch.int64, device="cuda")
        st = torch.zeros_like(streams[k])
        n = Z.compress_device(x, cfgs[k], out=st, offsets=off)
        ref = torch.zeros_like(x)
        Z.decompress_device(st, n, ref, cfgs[k], offsets=off)
        assert torch.equal(outs[k].view(torch.uint8), ref.view(torch.uint8)), k
