"""GPU parity with the oracle at the full sizes of the benchmark workloads.

The small-field tests in test_gpu_parity.py cover every mode and layout; the
paths that only appear at scale (multi-tile length scans, long pack runs,
host-buffer chunking, speculative-walk segments and fixes, batch rounds) are
pinned here: each case compresses the same seeded array with the GPU path and
with the oracle (the CPU restatement of zfp-rs, on all host cores) and
compares the streams byte for byte, then decodes the stream with both and
compares the arrays bit for bit.  Reference semantics: zfp-rs
src/compress.rs:22-116 and src/decompress.rs:27-147 (identical output under
any execution policy, docs/differences-from-c.md:70-77).

Workloads (tests/workloads.py): the 512^3 float64 field with zero blocks and
spikes under fixed-accuracy 1e-6 and fixed-precision 32 with every rounding;
the 8192^2 float32 Gaussian random field at fixed rates 4, 12 and 24; the
2^28-value int32 random walk and the 256^3 uniform int64 field in
fixed-precision and reversible mode (reversible also round trips exactly);
the oracle's own 512^3 stream decoded without a block index; and 100 arrays
of the 2,000-array batch.
"""

import os

import numpy as np
import pytest

from oracle import py_oracle as orc
from tests import workloads as W
from tests import zfpb

pytestmark = pytest.mark.gpu
Z = zfpb.load()
THREADS = os.cpu_count() or 1


def ocfg(c):
    return orc.config(c.min_bits, c.max_bits, c.max_prec, c.min_exp, c.rounding, c.tight_error)


def same_bits(a, b):
    return a.nbytes == b.nbytes and np.array_equal(a.reshape(-1).view(np.uint8), b.reshape(-1).view(np.uint8))


def nblocks(shape):
    return int(np.prod([(n + 3) // 4 for n in shape]))


def gpu_compress(x, cfg):
    import torch

    cap = Z.maximum_size(x.shape, Z._np_dtype(x.dtype), cfg)
    out = torch.empty((cap + 7) // 8, dtype=torch.int64, device="cuda")
    offs = torch.empty(nblocks(x.shape) + 1, dtype=torch.int64, device="cuda")
    n = Z.compress_device(x, cfg, out=out, offsets=offs)
    return out, n, offs


def check(arr, cfg, *, lossless=False, oracle_stream=None):
    """GPU stream == oracle stream, GPU decode == oracle decode; returns the oracle stream."""
    import torch

    x = torch.from_numpy(arr).cuda()
    if oracle_stream is None:
        want, n = orc.compress(arr, ocfg(cfg), threads=THREADS)
        assert n > 0
    else:
        want, n = oracle_stream
    out, got_n, offs = gpu_compress(x, cfg)
    assert got_n == n, (got_n, n)
    got = out.view(torch.uint8)[:n].cpu().numpy()
    assert same_bits(got, np.frombuffer(want, dtype=np.uint8)), "stream differs from the oracle"
    ref = np.empty_like(arr)
    assert orc.decompress(want, ref, ocfg(cfg), threads=THREADS) == n
    y = torch.empty_like(x)
    assert Z.decompress_device(out, n, y, cfg, offsets=offs) == n
    assert same_bits(y.cpu().numpy(), ref), "decode differs from the oracle"
    if lossless:
        assert same_bits(ref, arr)
    return want, n, ref


@pytest.fixture(scope="module")
def spiky():
    return W.spiky_f64(512)


SPIKY_CASES = [(mode, rnd, tight) for mode in ("accuracy_1e-6", "precision_32")
               for rnd in ("first", "last") for tight in (False, True)]


@pytest.mark.parametrize("mode,rounding,tight", SPIKY_CASES)
def test_spiky_f64_512_matches_oracle(spiky, mode, rounding, tight):
    base = Z.ZfpConfig.fixed_accuracy(1e-6) if mode == "accuracy_1e-6" else Z.ZfpConfig.fixed_precision(32)
    check(spiky, base.with_rounding(rounding, tight))


def test_oracle_stream_without_index_decodes_like_the_oracle(spiky):
    """The oracle's 512^3 stream (2,097,152 blocks) handed to the GPU without
    block offsets: the speculative parallel walk finds them."""
    import torch

    cfg = Z.ZfpConfig.fixed_accuracy(1e-6).with_rounding("first")
    want, n = orc.compress(spiky, ocfg(cfg), threads=THREADS)
    ref = np.empty_like(spiky)
    assert orc.decompress(want, ref, ocfg(cfg), threads=THREADS) == n
    words = np.zeros((n + 7) // 8, dtype=np.uint64)
    words.view(np.uint8)[:n] = np.frombuffer(want, dtype=np.uint8)
    s = torch.from_numpy(words.view(np.int64)).cuda()
    y = torch.empty(spiky.shape, dtype=torch.float64, device="cuda")
    assert Z.decompress_device(s, n, y, cfg) == n
    assert same_bits(y.cpu().numpy(), ref)


@pytest.mark.parametrize("rate", [4, 12, 24])
def test_grf_f32_8192_fixed_rate_matches_oracle(rate):
    arr = W.grf_f32(8192)
    check(arr, Z.ZfpConfig.fixed_rate(rate, np.float32, 2))


@pytest.mark.parametrize("mode", ["precision_20", "reversible"])
def test_random_walk_i32_2p28_matches_oracle(mode):
    arr = W.random_walk_i32(1 << 28)
    cfg = Z.ZfpConfig.reversible() if mode == "reversible" else Z.ZfpConfig.fixed_precision(20)
    check(arr, cfg, lossless=mode == "reversible")


@pytest.mark.parametrize("mode", ["precision_32", "reversible"])
def test_uniform_i64_256_matches_oracle(mode):
    arr = W.uniform_i64((256, 256, 256))
    cfg = Z.ZfpConfig.reversible() if mode == "reversible" else Z.ZfpConfig.fixed_precision(32)
    check(arr, cfg, lossless=mode == "reversible")


def test_batched_workload_subset_matches_oracle():
    """The 2,000-array batch compressed and decompressed in one call each; 100
    arrays drawn at random compared with the oracle (stream and decode)."""
    import torch

    specs = W.batched_specs(Z, 2000, 16_777_216)
    fields = [W.batched_array(s, i, "cuda") for i, s in enumerate(specs)]
    cfgs = [c for _, _, c in specs]
    caps = [Z.maximum_size(s[0], s[1], s[2]) for s in specs]
    streams = [torch.empty((cap + 7) // 8, dtype=torch.int64, device="cuda") for cap in caps]
    outs = [torch.empty_like(x) for x in fields]
    sizes = Z.compress_batch(Z.batch_items(fields, cfgs, streams))
    Z.decompress_batch(Z.batch_items(outs, cfgs, streams, nbytes=sizes))
    pick = np.random.default_rng(11).choice(len(specs), size=100, replace=False)
    for i in pick.tolist():
        arr = fields[i].cpu().numpy()
        want, n = orc.compress(arr, ocfg(cfgs[i]), threads=THREADS)
        assert sizes[i] == n, (i, sizes[i], n)
        got = streams[i].view(torch.uint8)[:n].cpu().numpy()
        assert same_bits(got, np.frombuffer(want, dtype=np.uint8)), f"array {i}: stream differs"
        ref = np.empty_like(arr)
        assert orc.decompress(want, ref, ocfg(cfgs[i]), threads=THREADS) == n
        assert same_bits(outs[i].cpu().numpy(), ref), f"array {i}: decode differs"
