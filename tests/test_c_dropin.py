"""A C caller of the drop-in boundary: tests/c/dropin.c built against
include/zfp.h only and linked with libzfp_b200.so.

The CPU test compiles and links it (its _Static_asserts pin the zfp_stream,
zfp_field, zfp_config and zfp_execution layouts of zfp-rs-ffi
src/abi.rs:122-233); the GPU test also runs it: three round trips through
zfp_compress / zfp_decompress, as the reference's own C drop-in smoke test
does (zfp-rs-ffi/tests/c-dropin/compress.c).
"""

import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
LIBDIR = ROOT / "zfp-rs_b200"
SRC = ROOT / "tests" / "c" / "dropin.c"


def build(tmp_path):
    exe = tmp_path / "dropin"
    cmd = ["gcc", "-std=c11", "-O2", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}", str(SRC),
           f"-L{LIBDIR}", "-lzfp_b200", f"-Wl,-rpath,{LIBDIR}", "-lm", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_dropin_compiles_and_links(tmp_path):
    assert (LIBDIR / "libzfp_b200.so").exists(), "build the library first"
    build(tmp_path)


@pytest.mark.gpu
def test_dropin_round_trips_on_the_gpu(tmp_path):
    exe = build(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "dropin ok" in r.stdout
