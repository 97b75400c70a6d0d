"""The C-ABI boundary without a GPU: symbols, bit streams, fields, configs.

Host-side behaviour follows zfp-rs-ffi (bitstream.rs, field.rs, stream.rs,
header.rs) and zfp-rs src/config.rs; the known answers come from the
reference's own unit tests (config.rs:769-810, stream.rs:173-205).
"""

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import py_oracle as orc
from tests import zfpb

Z = zfpb.load()
ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = []
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"\b([a-z_][a-z0-9_]*)\s*\([^;{]*\)\s*;", text)
    return sorted(set(n for n in names if n not in ("sizeof",)))


def test_library_exports_every_declared_symbol():
    L = Z.lib()
    decl = declared_functions()
    assert len(decl) >= 90
    bound = {name for name, _, _ in Z.SIGNATURES}
    for name in decl:
        assert hasattr(L, name), name
        assert name in bound, f"{name} has no ctypes signature"
    for name in Z.DATA_SYMBOLS:
        C.c_size_t.in_dll(L, name)


def test_version_constants():
    L = Z.lib()
    assert C.c_size_t.in_dll(L, "stream_word_bits").value == 64
    assert C.c_uint32.in_dll(L, "zfp_codec_version").value == 5
    assert C.c_uint32.in_dll(L, "zfp_library_version").value == (1 << 12) + (0 << 8) + (1 << 4)


def test_bit_stream_ops_match_the_oracle():
    """Random write/read/seek/pad/flush sequences give the same words and cursors."""
    L = Z.lib()
    rng = np.random.default_rng(7)
    for trial in range(40):
        nwords = int(rng.integers(1, 12))
        a = np.zeros(nwords, dtype=np.uint64)
        b = np.zeros(nwords, dtype=np.uint64)
        s = L.stream_open(a.ctypes.data, a.nbytes)
        o = orc.Stream(b)
        for _ in range(60):
            op = int(rng.integers(0, 7))
            if op == 0:
                n = int(rng.integers(0, 65))
                v = int(rng.integers(0, 2 ** 63)) & ((1 << n) - 1 if n < 64 else (1 << 64) - 1)
                assert L.stream_write_bits(s, v, n) == orc.lib().orc_stream_write_bits(o.h, v, n)
            elif op == 1:
                n = int(rng.integers(0, 65))
                assert L.stream_read_bits(s, n) == orc.lib().orc_stream_read_bits(o.h, n)
            elif op == 2:
                off = int(rng.integers(0, 64 * nwords + 70))
                L.stream_rseek(s, off)
                orc.lib().orc_stream_rseek(o.h, off)
            elif op == 3:
                off = int(rng.integers(0, 64 * nwords + 70))
                L.stream_wseek(s, off)
                orc.lib().orc_stream_wseek(o.h, off)
            elif op == 4:
                assert L.stream_flush(s) == orc.lib().orc_stream_flush(o.h)
            elif op == 5:
                assert L.stream_align(s) == orc.lib().orc_stream_align(o.h)
            else:
                L.stream_rewind(s)
                o.rewind()
            assert L.stream_wtell(s) == o.wtell()
            assert L.stream_rtell(s) == o.rtell()
        assert np.array_equal(a, b), trial
        L.stream_close(s)


def test_stream_open_copies_misaligned_buffers_and_reports_capacity():
    L = Z.lib()
    raw = np.zeros(33, dtype=np.uint8)
    s = L.stream_open(raw.ctypes.data + 1, 20)
    assert L.stream_capacity(s) == 24
    assert L.stream_data(s) != raw.ctypes.data + 1
    L.stream_close(s)
    words = np.zeros(4, dtype=np.uint64)
    s = L.stream_open(words.ctypes.data, 30)
    assert L.stream_capacity(s) == 24 and L.stream_data(s) == words.ctypes.data
    assert L.stream_stride_block(s) == 8 and L.stream_stride_delta(s) == -8 and L.stream_alignment() == 8
    L.stream_close(s)


def test_field_functions():
    L = Z.lib()
    a = np.zeros((5, 6, 7), dtype=np.float32)
    f = L.zfp_field_3d(a.ctypes.data, 3, 7, 6, 5)
    assert L.zfp_field_dimensionality(f) == 3 and L.zfp_field_precision(f) == 32
    dims = (C.c_size_t * 4)()
    assert L.zfp_field_size(f, dims) == 210 and list(dims) == [7, 6, 5, 0]
    assert L.zfp_field_blocks(f) == 2 * 2 * 2
    assert L.zfp_field_is_contiguous(f) == 1
    assert L.zfp_field_size_bytes(f) == 210 * 4
    meta = L.zfp_field_metadata(f)
    g = L.zfp_field_alloc()
    assert L.zfp_field_set_metadata(g, meta) == 1
    assert (g.contents.type, g.contents.nx, g.contents.ny, g.contents.nz, g.contents.nw) == (3, 7, 6, 5, 0)
    L.zfp_field_set_stride_3d(f, -1, 7, 42)
    assert L.zfp_field_is_contiguous(f) == 0
    assert L.zfp_field_begin(f) == a.ctypes.data - 6 * 4
    assert L.zfp_field_set_type(f, 9) == 0 and L.zfp_field_type(f) == 3
    bad = L.zfp_field_2d(None, 4, 0, 3)
    assert L.zfp_field_metadata(bad) == 2 ** 64 - 1
    for p in (f, g, bad):
        L.zfp_field_free(p)


def open_stream():
    L = Z.lib()
    buf = np.zeros(64, dtype=np.uint64)
    bs = L.stream_open(buf.ctypes.data, buf.nbytes)
    return L, buf, bs, L.zfp_stream_open(bs)


@pytest.mark.parametrize("tname,dims,rate,bits", [
    ("double", 3, 8.0, 512),  # config.rs:769-787: f64 3-D rate 8 -> 512 bits
    ("double", 3, 5.0, 320),
    ("float", 1, 0.1, 9),     # config.rs:790-810: raised to the f32 header
    ("double", 1, 0.1, 12),
    ("int32", 2, 1.5, 24),
])
def test_set_rate_budgets(tname, dims, rate, bits):
    L, buf, bs, zs = open_stream()
    code = {"int32": 1, "int64": 2, "float": 3, "double": 4}[tname]
    got = L.zfp_stream_set_rate(zs, rate, code, dims, 0)
    assert zs.contents.maxbits == bits and zs.contents.minbits == bits
    assert got == bits / 4 ** dims
    assert L.zfp_stream_compression_mode(zs) == 2
    aligned = L.zfp_stream_set_rate(zs, 5.0, 4, 1, 1)
    assert zs.contents.maxbits == 64 and aligned == 16.0
    assert L.zfp_stream_set_rate(zs, float("nan"), 3, 3, 0) == 0.0
    L.zfp_stream_close(zs)
    L.stream_close(bs)


def test_modes_and_mode_words_match_the_oracle():
    L, buf, bs, zs = open_stream()
    assert L.zfp_stream_set_precision(zs, 0) == 64
    assert L.zfp_stream_compression_mode(zs) == 1  # the defaults are expert mode
    assert L.zfp_stream_set_precision(zs, 16) == 16 and L.zfp_stream_precision(zs) == 16
    assert L.zfp_stream_compression_mode(zs) == 3
    assert L.zfp_stream_set_accuracy(zs, 1e-6) == 2.0 ** -20 and zs.contents.minexp == -20
    assert L.zfp_stream_compression_mode(zs) == 4 and L.zfp_stream_accuracy(zs) == 2.0 ** -20
    L.zfp_stream_set_reversible(zs)
    assert L.zfp_stream_compression_mode(zs) == 5 and L.zfp_stream_mode(zs) == 2048 + 128
    rng = np.random.default_rng(3)
    for _ in range(300):
        minb = int(rng.integers(0, 20000))
        maxb = int(rng.integers(minb, 40000))
        maxp = int(rng.integers(1, 65))
        mine = int(rng.integers(-1100, 900))
        assert L.zfp_stream_set_params(zs, minb, maxb, maxp, mine) == 1
        cfg = orc.config(minb, maxb, maxp, mine)
        assert L.zfp_stream_compression_mode(zs) == orc.lib().orc_mode(C.byref(cfg))
        mode = L.zfp_stream_mode(zs)
        assert mode == orc.lib().orc_mode_bits(C.byref(cfg))
    assert L.zfp_stream_set_params(zs, 5, 4, 10, 0) == 0
    assert L.zfp_stream_set_mode(zs, 2047) == 2 and zs.contents.maxbits == 2048
    L.zfp_stream_close(zs)
    L.stream_close(bs)


def test_block_maximum_size_table():
    """zfp-rs-ffi/src/stream.rs:173-205."""
    L = Z.lib()
    want = {
        0: [[131, 527, 2111, 8447], [259, 1039, 4159, 16639], [140, 536, 2120, 8456], [271, 1051, 4171, 16651]],
        1: [[136, 532, 2116, 8452], [265, 1045, 4165, 16645], [146, 542, 2126, 8462], [278, 1058, 4178, 16658]],
    }
    for rev, rows in want.items():
        for t, row in enumerate(rows):
            for d, v in enumerate(row):
                assert L.zfp_block_maximum_size(t + 1, d + 1, rev) == v
    assert L.zfp_block_maximum_size(0, 1, 0) == 0 and L.zfp_block_maximum_size(1, 5, 0) == 0


def test_header_round_trip_matches_the_oracle():
    L = Z.lib()
    rng = np.random.default_rng(11)
    for _ in range(50):
        t = int(rng.integers(1, 5))
        d = int(rng.integers(1, 5))
        n = [int(x) for x in rng.integers(1, 300, size=d)] + [0] * (4 - d)
        params = (int(rng.integers(1, 100)), int(rng.integers(100, 20000)), int(rng.integers(1, 65)),
                  int(rng.integers(-1075, 500)))
        buf = np.zeros(8, dtype=np.uint64)
        bs = L.stream_open(buf.ctypes.data, buf.nbytes)
        zs = L.zfp_stream_open(bs)
        L.zfp_stream_set_params(zs, *params)
        f = L.zfp_field_alloc()
        f.contents.type, f.contents.nx, f.contents.ny, f.contents.nz, f.contents.nw = t, *n
        bits = L.zfp_write_header(zs, f, 7)
        L.stream_flush(bs)
        ob = np.zeros(8, dtype=np.uint64)
        os_ = orc.Stream(ob)
        of = orc.OrcField(t, *n, 0, 0, 0, 0, None)
        oc = orc.config(*params)
        assert bits == orc.lib().orc_write_header(os_.h, C.byref(of), C.byref(oc), 7)
        os_.flush()
        assert np.array_equal(buf, ob)
        L.stream_rewind(bs)
        g = L.zfp_field_alloc()
        zs2 = L.zfp_stream_open(bs)
        assert L.zfp_read_header(zs2, g, 7) == bits
        assert (g.contents.type, g.contents.nx, g.contents.ny, g.contents.nz, g.contents.nw) == (t, *n)
        assert L.zfp_stream_mode(zs2) == L.zfp_stream_mode(zs)
        for p in (f, g):
            L.zfp_field_free(p)
        L.zfp_stream_close(zs)
        L.zfp_stream_close(zs2)
        L.stream_close(bs)


def test_rounding_and_execution_settings():
    L, buf, bs, zs = open_stream()
    tight = C.c_int32()
    assert L.zfp_stream_rounding(zs, C.byref(tight)) == 0 and tight.value == 0
    assert L.zfp_stream_set_rounding(zs, -1, 1) == 1
    assert L.zfp_stream_rounding(zs, C.byref(tight)) == -1 and tight.value == 1
    assert L.zfp_stream_set_rounding(zs, 7, 0) == 0
    assert L.zfp_stream_set_execution(zs, 2) == 1 and L.zfp_stream_execution(zs) == 2
    assert L.zfp_stream_set_omp_threads(zs, 4) == 1 and L.zfp_stream_omp_threads(zs) == 4
    assert L.zfp_stream_set_omp_chunk_size(zs, 9) == 1 and L.zfp_stream_omp_chunk_size(zs) == 9
    assert L.zfp_stream_set_execution(zs, 0) == 1 and L.zfp_stream_omp_threads(zs) == 0
    L.zfp_stream_close(zs)
    L.stream_close(bs)


def test_python_config_mirrors_the_reference():
    cfg = Z.ZfpConfig.fixed_rate(8, np.float64, 3)
    assert (cfg.min_bits, cfg.max_bits, cfg.max_prec, cfg.min_exp) == (512, 512, 64, -1074)
    assert Z.ZfpConfig.fixed_accuracy(1e-6).min_exp == -20
    assert Z.ZfpConfig.fixed_precision(100).max_prec == 64
    assert Z.ZfpConfig.reversible().min_exp == -1075
    with pytest.raises(ValueError):
        Z.ZfpConfig.expert(5, 4, 10, 0)
    with pytest.raises(ValueError):
        Z.ZfpConfig.fixed_rate(-1, np.float32, 2)


def test_config_constructors():
    """zfp-rs-ffi/src/header.rs:60-140: a negative rate means not word aligned."""
    L = Z.lib()
    c = L.zfp_config_rate(8.0, 0)
    assert c.mode == 2 and c.arg.rate == -8.0
    assert L.zfp_config_rate(8.0, 1).arg.rate == 8.0
    assert L.zfp_config_precision(16).arg.precision == 16 and L.zfp_config_precision(16).mode == 3
    assert L.zfp_config_accuracy(1e-3).arg.tolerance == 1e-3
    assert L.zfp_config_reversible().mode == 5 and L.zfp_config_none().mode == 0
    e = L.zfp_config_expert(1, 2, 3, -4).arg.expert
    assert (e.minbits, e.maxbits, e.maxprec, e.minexp) == (1, 2, 3, -4)
    assert L.zfp_type_size(1) == 4 and L.zfp_type_size(4) == 8 and L.zfp_type_size(0) == 0
