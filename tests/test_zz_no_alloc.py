"""zfpb_compress_device_noalloc: compression that allocates no device memory.

Some callers cannot let a library call cudaMalloc: an application that has
reserved all device memory for its own pool, or a latency-critical loop that
cannot take cudaMalloc's device-wide synchronization.  This entry point gives
them the same stream as zfpb_compress_device, with its scratch taken from a
fixed device array inside the library.  The tests call it through the C ABI:
first before any other entry point, checking that a call after the warm-up
one leaves the device's free memory unchanged; then twice in a row per mode,
checking each stream byte for byte against the existing entry point.  The
file runs last (file name) and also passes alone in a fresh process.
"""

import ctypes as C

import numpy as np
import pytest

from tests import zfpb

pytestmark = pytest.mark.gpu
Z = zfpb.load()


def field(shape, seed, dtype):
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    z, y, x = [torch.arange(n, device="cuda", dtype=torch.float64) for n in shape]
    f = torch.sin(0.1 * x)[None, None, :] * torch.cos(0.13 * y)[None, :, None] * torch.sin(0.07 * z)[:, None, None]
    f = f + 1e-3 * torch.randn(shape, generator=g, device="cuda", dtype=torch.float64)
    return (f * 100).to(dtype)


def compress_both(x, cfg):
    import torch

    L = Z.lib()
    np_dt = {torch.float32: np.float32, torch.float64: np.float64}[x.dtype]
    desc = Z.desc_of(x.shape, np_dt, cfg)
    cap = Z.maximum_size(x.shape, np_dt, cfg)
    a = torch.zeros((cap + 7) // 8, dtype=torch.int64, device="cuda")
    b = torch.zeros_like(a)
    cs = torch.cuda.current_stream().cuda_stream
    na = L.zfpb_compress_device(C.byref(desc), x.data_ptr(), a.data_ptr(), cap, None, cs)
    nb = L.zfpb_compress_device_noalloc(C.byref(desc), x.data_ptr(), b.data_ptr(), cap, cs)
    assert na > 0 and nb == na, (na, nb, L.zfpb_last_error())
    assert torch.equal(a[: (na + 7) // 8], b[: (nb + 7) // 8])
    return na


def test_noalloc_allocates_no_device_memory():
    """The first library call of this file is the no-allocation entry point.

    Its first call on a device loads the library's kernels (and with them
    the module holding the fixed scratch array), which takes device memory
    once.  After that warm-up call a second call must leave the device's
    free memory unchanged; only then does the existing, allocating entry
    point run, for the byte comparison."""
    import torch

    L = Z.lib()
    x = field((24, 20, 28), 3, torch.float64)
    cfg = Z.ZfpConfig.fixed_accuracy(1e-5)
    desc = Z.desc_of(x.shape, np.float64, cfg)
    cap = Z.maximum_size(x.shape, np.float64, cfg)
    first = torch.zeros((cap + 7) // 8, dtype=torch.int64, device="cuda")
    second = torch.zeros_like(first)
    ref = torch.zeros_like(first)
    cs = torch.cuda.current_stream().cuda_stream
    n1 = L.zfpb_compress_device_noalloc(C.byref(desc), x.data_ptr(), first.data_ptr(), cap, cs)
    assert n1 > 0, L.zfpb_last_error()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    n2 = L.zfpb_compress_device_noalloc(C.byref(desc), x.data_ptr(), second.data_ptr(), cap, cs)
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert n2 == n1 and free_after == free_before, (n1, n2, free_before, free_after)
    nref = L.zfpb_compress_device(C.byref(desc), x.data_ptr(), ref.data_ptr(), cap, None, cs)
    assert nref == n1
    assert torch.equal(first, ref) and torch.equal(second, ref)


@pytest.mark.parametrize("dtype_name", ["float32", "float64"])
def test_noalloc_matches_existing_entry_point_twice_in_a_row(dtype_name):
    import torch

    dt = getattr(torch, dtype_name)
    cfgs = [Z.ZfpConfig.fixed_accuracy(1e-5), Z.ZfpConfig.fixed_precision(20).with_rounding("first", True),
            Z.ZfpConfig.reversible(), Z.ZfpConfig.fixed_rate(8, np.dtype(dtype_name), 3)]
    for cfg in cfgs:
        # Two calls in a row on different fields: the shared scratch keeps the
        # first call's contents, which must not leak into the second stream.
        compress_both(field((20, 24, 28), 1, dt), cfg)
        compress_both(field((13, 9, 30), 2, dt), cfg)


def test_noalloc_rejects_fields_beyond_its_scratch():
    import torch

    L = Z.lib()
    x = torch.zeros((256, 256, 256), dtype=torch.float64, device="cuda")
    cfg = Z.ZfpConfig.fixed_accuracy(1e-6)
    desc = Z.desc_of(x.shape, np.float64, cfg)
    out = torch.zeros(1024, dtype=torch.int64, device="cuda")
    n = L.zfpb_compress_device_noalloc(C.byref(desc), x.data_ptr(), out.data_ptr(), 8192,
                                       torch.cuda.current_stream().cuda_stream)
    assert n == 0 and L.zfpb_last_error() == 6
