"""The oracle's reader/worker decode pipeline against its serial decoder.

zfp-rs decodes variable-rate streams of 2-4 dimensions with a plane-reader /
reconstruction pipeline (src/decompress/pipeline.rs:193-229) and promises the
same output as its serial decoder under any execution policy
(docs/differences-from-c.md:70-77).  The oracle restates that pipeline; these
CPU tests check it against the oracle's serial decode for every scalar type,
2-4 dimensions, partial blocks and each mode family, including truncation.
"""

import numpy as np
import pytest

from oracle import py_oracle as orc

SHAPES = {2: (70, 53), 3: (21, 18, 26), 4: (9, 7, 11, 6)}
DTYPES = [np.int32, np.int64, np.float32, np.float64]
CONFIGS = [
    ("precision", orc.config(1, 16658, 20, -1074, "first", True)),
    ("accuracy", orc.config(1, 16658, 64, -20, "last", False)),
    ("reversible", orc.config(1, 16658, 64, -1075)),
    ("expert", orc.config(30, 900, 40, -60, "last", True)),
]


def field(shape, dtype, seed):
    rng = np.random.default_rng(seed)
    grids = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in shape], indexing="ij")
    v = np.ones(shape)
    for i, g in enumerate(grids):
        v = v * np.sin(0.11 * (i + 1) * g + 0.2 * i)
    v = v + rng.normal(0, 1e-3, size=shape)
    if np.dtype(dtype).kind == "i":
        return (v * (2 ** 20 if dtype == np.int32 else 2 ** 40)).astype(dtype)
    return (v * 1e3).astype(dtype)


@pytest.mark.parametrize("dims", [2, 3, 4])
@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("name,cfg", CONFIGS, ids=[c[0] for c in CONFIGS])
def test_pipeline_decode_matches_serial(dims, dtype, name, cfg):
    arr = field(SHAPES[dims], dtype, dims)
    stream, n = orc.compress(arr, cfg, threads=4)
    assert n > 0
    serial = np.zeros_like(arr)
    piped = np.zeros_like(arr)
    assert orc.decompress(stream, serial, cfg, threads=1) == n
    assert orc.decompress(stream, piped, cfg, threads=6) == n
    assert piped.tobytes() == serial.tobytes()


def test_pipeline_reports_truncation_like_serial():
    arr = field(SHAPES[3], np.float64, 7)
    cfg = CONFIGS[1][1]
    stream, n = orc.compress(arr, cfg)
    cut = stream[: (n // 2) // 8 * 8]
    a, b = np.zeros_like(arr), np.zeros_like(arr)
    assert orc.decompress(cut, a, cfg, threads=1) == -1
    assert orc.decompress(cut, b, cfg, threads=6) == -1
    assert a.tobytes() == b.tobytes()
