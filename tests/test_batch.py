"""Batched compress/decompress (zfpb_compress_batch / zfpb_decompress_batch).

Many arrays of mixed type, dimensionality, size and mode go through one
batched call; every array's stream must be byte-identical, and every decoded
array bit-identical, to what the single-array device calls give for that
array alone (which the parity tests pin to the oracle), on the first call
(planned, tuned, run directly) and on a repeat (replayed CUDA graph).
"""

import ctypes as C

import numpy as np
import pytest

from oracle import py_oracle as orc
from tests import zfpb

pytestmark = pytest.mark.gpu
Z = zfpb.load()


def smooth_t(shape, dtype, seed):
    import torch

    rng = np.random.default_rng(seed)
    grids = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in shape], indexing="ij")
    v = np.ones(shape)
    for i, g in enumerate(grids):
        v = v * np.sin(0.1 * (i + 1) * g + 0.3 * i)
    v = v + rng.normal(0, 1e-3, size=shape)
    if np.dtype(dtype).kind == "i":
        v = v * (2 ** 20 if dtype == np.int32 else 2 ** 40)
    else:
        v = v * 100.0
    return torch.from_numpy(np.ascontiguousarray(v.astype(dtype))).cuda()


def mixed_jobs(seed, n=40):
    """A mix like the batched workload: types, 1-4 D, partial blocks, every mode."""
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(n):
        dtype = [np.float32, np.float64, np.int32, np.int64][rng.integers(0, 4)]
        dims = int(rng.integers(1, 5))
        side = {1: (5, 3000), 2: (3, 90), 3: (2, 30), 4: (2, 9)}[dims]
        shape = tuple(int(x) for x in rng.integers(side[0], side[1], size=dims))
        kind = rng.integers(0, 5)
        if kind == 0:
            cfg = Z.ZfpConfig.fixed_rate(float(rng.integers(2, 33)), dtype, dims)
        elif kind == 1:
            cfg = Z.ZfpConfig.fixed_precision(int(rng.integers(8, 49)))
        elif kind == 2 and np.dtype(dtype).kind == "f":
            cfg = Z.ZfpConfig.fixed_accuracy(float(10.0 ** -rng.integers(2, 10)))
        elif kind == 3:
            cfg = Z.ZfpConfig.reversible()
        else:
            cfg = Z.ZfpConfig.expert(int(rng.integers(1, 40)), int(rng.integers(400, 3000)), int(rng.integers(10, 64)),
                                     -int(rng.integers(20, 200)))
        if kind != 3:
            cfg = cfg.with_rounding(["never", "first", "last"][rng.integers(0, 3)], bool(rng.integers(0, 2)))
        jobs.append((smooth_t(shape, dtype, seed * 1000 + i), cfg))
    return jobs


def single(jobs):
    import torch

    out = []
    for x, cfg in jobs:
        cap = Z.maximum_size(x.shape, Z._np_dtype(x.dtype), cfg)
        buf = torch.zeros((cap + 7) // 8, dtype=torch.int64, device="cuda")
        n = Z.compress_device(x, cfg, out=buf)
        y = torch.zeros_like(x)
        Z.decompress_device(buf, n, y, cfg)
        out.append((buf[: n // 8].clone(), y))
    return out


def batch_buffers(jobs):
    import torch

    streams, offsets = [], []
    for x, cfg in jobs:
        cap = Z.maximum_size(x.shape, Z._np_dtype(x.dtype), cfg)
        streams.append(torch.zeros((cap + 7) // 8, dtype=torch.int64, device="cuda"))
        nb = int(np.prod([(n + 3) // 4 for n in x.shape]))
        offsets.append(torch.zeros(nb + 1, dtype=torch.int64, device="cuda"))
    return streams, offsets


def test_batch_matches_single_calls_and_replays():
    import torch

    jobs = mixed_jobs(1)
    ref = single(jobs)
    streams, offsets = batch_buffers(jobs)
    fields = [x for x, _ in jobs]
    cfgs = [c for _, c in jobs]
    items = Z.batch_items(fields, cfgs, streams, offsets=offsets)
    for rep in range(2):  # planned and run directly, then the replayed graph
        for s in streams:
            s.zero_()
        sizes = Z.compress_batch(items)
        torch.cuda.synchronize()
        for i, (buf, _) in enumerate(ref):
            assert sizes[i] == buf.numel() * 8, (rep, i)
            assert torch.equal(streams[i][: sizes[i] // 8], buf), (rep, i, cfgs[i])
    # decode with the batch's index, then with no index (walker), twice each
    for use_index in (True, False):
        outs = [torch.full_like(x, 7) for x in fields]
        ditems = Z.batch_items(outs, cfgs, streams, nbytes=sizes, offsets=offsets if use_index else None)
        for rep in range(2):
            for o in outs:
                o.fill_(7)
            used = Z.decompress_batch(ditems)
            torch.cuda.synchronize()
            for i, (_, y) in enumerate(ref):
                assert used[i] == sizes[i]
                assert torch.equal(outs[i].view(torch.uint8), y.view(torch.uint8)), (use_index, rep, i, cfgs[i])


def test_batch_streams_match_oracle():
    import torch

    jobs = mixed_jobs(2, n=12)
    streams, _ = batch_buffers(jobs)
    items = Z.batch_items([x for x, _ in jobs], [c for _, c in jobs], streams)
    sizes = Z.compress_batch(items)
    for i, (x, cfg) in enumerate(jobs):
        want, n = orc.compress(x.cpu().numpy(), orc.config(cfg.min_bits, cfg.max_bits, cfg.max_prec, cfg.min_exp,
                                                          cfg.rounding, cfg.tight_error))
        assert sizes[i] == n
        assert streams[i][: n // 8].cpu().numpy().tobytes() == want


def test_batch_headers_match_oracle_and_are_checked():
    """Items whose streams carry a zfp header (full, mode only, magic + meta,
    magic only, none): each stream is the oracle's header-then-blocks stream,
    decompress reads the blocks after the header (with the index, and by
    walking without it), and a stream whose header does not match its
    description fails with status 7 while the other items decode."""
    import torch

    jobs = mixed_jobs(4, n=15)
    ref = single(jobs)
    streams, offsets = batch_buffers(jobs)
    fields = [x for x, _ in jobs]
    cfgs = [c for _, c in jobs]
    masks = [[7, 0, 4, 3, 1][i % 5] for i in range(len(jobs))]
    items = Z.batch_items(fields, cfgs, streams, offsets=offsets, header_mask=masks)
    sizes = Z.compress_batch(items)
    for i, (x, cfg) in enumerate(jobs):
        want, n = orc.compress(x.cpu().numpy(), orc.config(cfg.min_bits, cfg.max_bits, cfg.max_prec, cfg.min_exp,
                                                          cfg.rounding, cfg.tight_error), header_mask=masks[i])
        assert sizes[i] == n, (i, masks[i])
        assert streams[i][: n // 8].cpu().numpy().tobytes() == want, (i, masks[i], cfg)
    for use_index in (True, False):
        outs = [torch.full_like(x, 7) for x in fields]
        used = Z.decompress_batch(Z.batch_items(outs, cfgs, streams, nbytes=sizes,
                                                offsets=offsets if use_index else None, header_mask=masks))
        for i, (_, y) in enumerate(ref):
            assert used[i] == sizes[i]
            assert torch.equal(outs[i].view(torch.uint8), y.view(torch.uint8)), (use_index, i, masks[i])
    bad = masks.index(7)
    streams[bad][0] ^= 1  # the magic's first byte
    outs = [torch.full_like(x, 7) for x in fields]
    ditems = Z.batch_items(outs, cfgs, streams, nbytes=sizes, offsets=offsets, header_mask=masks)
    ok = Z.lib().zfpb_decompress_batch(ditems, len(ditems), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert ok == len(ditems) - 1
    assert ditems[bad].status == 7 and ditems[bad].result == 0
    for i, (_, y) in enumerate(ref):
        if i != bad:
            assert ditems[i].status == 0 and ditems[i].result == sizes[i]
            assert torch.equal(outs[i].view(torch.uint8), y.view(torch.uint8)), i


def test_batch_reports_overflow_and_bad_index_per_item():
    import torch

    jobs = mixed_jobs(3, n=6)
    ref = single(jobs)
    streams, offsets = batch_buffers(jobs)
    fields = [x for x, _ in jobs]
    cfgs = [c for _, c in jobs]
    items = Z.batch_items(fields, cfgs, streams, offsets=offsets)
    items[2].stream_bytes = 8  # too small for item 2
    ok = Z.lib().zfpb_compress_batch(items, len(items), torch.cuda.current_stream().cuda_stream)
    assert ok == len(items) - 1
    assert items[2].result == 0 and items[2].status == 1
    for i in (0, 1, 3, 4, 5):
        assert items[i].status == 0 and items[i].result == ref[i][0].numel() * 8
    # a wrong index for one variable-rate item: detected, decoded by walking
    items[2].stream_bytes = streams[2].numel() * 8
    sizes = Z.compress_batch(items)
    var = [i for i, c in enumerate(cfgs) if c.min_bits != c.max_bits]
    if var:
        offsets[var[0]][1] += 1
    outs = [torch.zeros_like(x) for x in fields]
    Z.decompress_batch(Z.batch_items(outs, cfgs, streams, nbytes=sizes, offsets=offsets))
    for i, (_, y) in enumerate(ref):
        assert torch.equal(outs[i].view(torch.uint8), y.view(torch.uint8)), i


def test_batch_decodes_aliasing_strides_like_a_serial_decode():
    """An item whose strides make two blocks share elements is decoded apart
    from the batch kernels, keeping the later block's value as a serial
    decode does (decompress.rs:153-186)."""
    import torch

    base = smooth_t((6, 7, 12), np.float32, 5)
    cfg = Z.ZfpConfig.fixed_precision(18)
    nx, ny, nz = 7, 6, 5
    strides = (2, 12, 84)
    d = Z.desc_of((nz, ny, nx), np.float32, cfg, strides=strides)
    cap = Z.maximum_size((nz, ny, nx), np.float32, cfg)
    buf = torch.zeros((cap + 7) // 8, dtype=torch.int64, device="cuda")
    L = Z.lib()
    cs = torch.cuda.current_stream().cuda_stream
    n = L.zfpb_compress_device(C.byref(d), base.data_ptr(), buf.data_ptr(), cap, None, cs)
    assert n > 0
    want = torch.zeros_like(base)
    assert L.zfpb_decompress_device(C.byref(d), buf.data_ptr(), n, want.data_ptr(), None, cs) == n
    got = torch.zeros_like(base)
    other = smooth_t((9, 9), np.float64, 6)
    other_cfg = Z.ZfpConfig.fixed_rate(12, np.float64, 2)
    cap2 = Z.maximum_size(other.shape, np.float64, other_cfg)
    buf2 = torch.zeros((cap2 + 7) // 8, dtype=torch.int64, device="cuda")
    n2 = Z.compress_device(other, other_cfg, out=buf2)
    out2 = torch.zeros_like(other)
    items = (Z.ZfpBatchItem * 2)()
    items[0].desc = d
    items[0].d_field = got.data_ptr()
    items[0].d_stream = buf.data_ptr()
    items[0].stream_bytes = n
    items[1].desc = Z.desc_of(other.shape, np.float64, other_cfg)
    items[1].d_field = out2.data_ptr()
    items[1].d_stream = buf2.data_ptr()
    items[1].stream_bytes = n2
    assert L.zfpb_decompress_batch(items, 2, cs) == 2
    torch.cuda.synchronize()
    assert torch.equal(got.view(torch.uint8), want.view(torch.uint8))
    ref2 = torch.zeros_like(other)
    Z.decompress_device(buf2, n2, ref2, other_cfg)
    assert torch.equal(out2.view(torch.uint8), ref2.view(torch.uint8))
