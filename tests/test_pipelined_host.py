"""zfp_compress / zfp_decompress on large host buffers.

Host fields of 32 MB and more with natural strides go through the pipelined
path (the field, the stream and the output are copied in chunks of block
layers while other chunks are coded).  Its streams and decoded arrays must be
identical to those of the one-pass device calls.
"""

import numpy as np
import pytest

from tests import zfpb
from tests.test_gpu_parity import smooth

pytestmark = pytest.mark.gpu
Z = zfpb.load()


def device_reference(arr, cfg):
    import torch

    x = torch.from_numpy(arr).cuda()
    cap = Z.maximum_size(arr.shape, arr.dtype, cfg)
    buf = torch.zeros((cap + 7) // 8, dtype=torch.int64, device="cuda")
    n = Z.compress_device(x, cfg, out=buf)
    y = torch.zeros_like(x)
    Z.decompress_device(buf, n, y, cfg)
    return buf[: n // 8].cpu().numpy().tobytes(), y.cpu().numpy()


@pytest.mark.parametrize("shape,dtype", [((150, 256, 256), np.float32), ((67, 256, 256), np.float64),
                                         ((4099, 2053), np.float32), ((9_000_001,), np.float32)],
                         ids=["3d-f32", "3d-f64", "2d-f32", "1d-f32"])
def test_large_host_fields_match_the_device_path(shape, dtype):
    arr = smooth(shape, dtype, seed=11, scale=1e3)
    assert arr.nbytes >= 32 << 20
    cfgs = [Z.ZfpConfig.fixed_accuracy(1e-4), Z.ZfpConfig.fixed_rate(8, dtype, len(shape)),
            Z.ZfpConfig.fixed_precision(20).with_rounding("last", True)]
    for cfg in cfgs:
        want_stream, want_out = device_reference(arr, cfg)
        got = Z.compress(arr, cfg)  # zfp_compress, host buffers
        assert got == want_stream, cfg
        out = np.full_like(arr, 7)
        assert Z.decompress(got, out, cfg) == len(got)  # a fresh stream handle: no index
        assert out.tobytes() == want_out.tobytes(), cfg


def test_index_kept_with_the_stream_decodes_in_chunks():
    """Compress and decompress through one stream handle: the second call uses
    the block index kept from the first, so variable-rate data also decodes in
    overlapped chunks."""
    import ctypes as C

    arr = smooth((140, 256, 256), np.float32, seed=12, scale=50.0)
    cfg = Z.ZfpConfig.fixed_accuracy(1e-5).with_rounding("first", True)
    want_stream, want_out = device_reference(arr, cfg)
    L = Z.lib()
    cap = Z.maximum_size(arr.shape, arr.dtype, cfg)
    buf = np.zeros((cap + 7) // 8, dtype=np.uint64)
    s = Z.Stream(cfg, buf)
    try:
        f = Z.field_of(arr)
        n = L.zfp_compress(s.zfp, C.byref(f))
        assert n == len(want_stream) and buf.tobytes()[:n] == want_stream
        L.zfp_stream_rewind(s.zfp)
        out = np.zeros_like(arr)
        fo = Z.field_of(out)
        assert L.zfp_decompress(s.zfp, C.byref(fo)) == n
        assert out.tobytes() == want_out.tobytes()
        # The stream is changed behind the handle's back: the kept index no
        # longer matches, which is detected, and the stream is walked instead.
        buf[5] ^= np.uint64(1 << 17)
        L.zfp_stream_rewind(s.zfp)
        out2 = np.zeros_like(arr)
        fo2 = Z.field_of(out2)
        L.zfp_decompress(s.zfp, C.byref(fo2))
        ref = np.zeros_like(arr)
        import torch

        bt = torch.from_numpy(buf.view(np.int64)).cuda()
        yt = torch.zeros(arr.shape, dtype=torch.float32, device="cuda")
        Z.decompress_device(bt, n, yt, cfg)
        assert out2.tobytes() == yt.cpu().numpy().tobytes()
    finally:
        s.close()
