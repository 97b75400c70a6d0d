"""Test helpers: the checksum machinery and seeded inputs of zfp's own test suite.

Restates zfp-rs tests/c/checksums.rs:13-247 (Jenkins one-at-a-time hashes and
the test keys) and the LCG generators and special IEEE blocks of
tests/c/encode_block.rs:35-146, so that the golden tables in
tests/golden/checksums.json can be checked against.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = json.loads((Path(__file__).parent / "golden" / "checksums.json").read_text())["entries"]

ZFP_TYPES = {"int32": np.int32, "int64": np.int64, "float": np.float32, "double": np.float64}
RATE_PARAM_BITS = 19  # tests/c/encode_block.rs:26
M32 = 0xFFFFFFFF


def _hash_value(val: int, h: int) -> int:
    h = (h + val) & M32
    h = (h + (h << 10)) & M32
    h ^= h >> 6
    return h


def _hash_finish(h: int) -> int:
    h = (h + (h << 3)) & M32
    h ^= h >> 11
    h = (h + (h << 15)) & M32
    return h


def hash_bitstream(buf: bytes) -> int:
    """checksums.rs:31-44 (committed words, little-endian)."""
    h1 = h2 = 0
    w = np.frombuffer(buf[: len(buf) // 8 * 8], dtype="<u8")
    for word in w.tolist():
        h1 = _hash_value(word & M32, h1)
        h2 = _hash_value((word >> 32) & M32, h2)
    return _hash_finish(h1) + (_hash_finish(h2) << 32)


def hash_array(arr: np.ndarray) -> int:
    """hashArray32/64 (checksums.rs:48-77) over the flat array."""
    a = np.ascontiguousarray(arr).reshape(-1)
    if a.dtype.itemsize == 4:
        h = 0
        for v in a.view(np.uint32).tolist():
            h = _hash_value(v, h)
        return _hash_finish(h)
    h1 = h2 = 0
    for v in a.view(np.uint64).tolist():
        h1 = _hash_value(v & M32, h1)
        h2 = _hash_value((v >> 32) & M32, h2)
    return _hash_finish(h1) + (_hash_finish(h2) << 32)


def hash_strided(arr: np.ndarray, n, s) -> int:
    """hashStridedArray32/64 (checksums.rs:82-153): n dims, s element strides."""
    flat = arr.reshape(-1)
    dims = [max(n[0], 1)] + [x if x > 0 else 1 for x in n[1:4]]
    idx = []
    for l in range(dims[3]):
        for k in range(dims[2]):
            for j in range(dims[1]):
                for i in range(dims[0]):
                    idx.append(i * s[0] + j * s[1] + k * s[2] + l * s[3])
    return hash_array(flat[np.array(idx)])


# checksums.rs:158-247
BLOCK_FULL, BLOCK_PARTIAL, ARRAY = 0, 1, 2
ORIGINAL, COMPRESSED, DECOMPRESSED = 0, 1, 2
MODE_NULL, MODE_FIXED_RATE, MODE_REVERSIBLE = 0, 2, 5


def compute_key(tt, subject, n, mode, misc):
    r = tt
    r = (r << 2) + subject
    r = (r << 3) + mode
    r = (r << 4) + misc
    dims = 4 if n[3] else 3 if n[2] else 2 if n[1] else 1
    if dims == 1:
        k2 = n[0] - 1
    elif dims == 2:
        k2 = ((n[0] - 1) << 24) + n[1] - 1
    elif dims == 3:
        k2 = ((((n[0] - 1) << 16) + n[1] - 1) << 16) + n[2] - 1
    else:
        k2 = ((((((n[0] - 1) << 12) + n[1] - 1) << 12) + n[2] - 1) << 12) + n[3] - 1
    return r, k2


def golden(dims, tname, key1, key2):
    for e in GOLDEN:
        if e["dims"] == dims and e["type"] == tname and e["key1"] == key1 and e["key2"] == key2:
            return e["checksum"]
    raise KeyError((dims, tname, hex(key1), hex(key2)))


class Rand32:
    """encode_block.rs:35-62: LCG x = (0x5deece66d x + 0xb) mod 2^48, seed 5."""

    def __init__(self):
        self.x = 5

    def next_unsigned(self):
        self.x = (0x5DEECE66D * self.x + 0xB) % (1 << 48)
        return (self.x >> 16) & 0x7FFFFFFF

    def next_int(self):
        return self.next_unsigned() - 0x40000000

    def next_float(self):
        u = (self.next_unsigned() >> 7) & 0x00FFFFFF
        return np.float32(np.ldexp(np.float32(u - 0x00800000), -12))


class Rand64:
    """encode_block.rs:64-88: x = 2862933555777941757 x + 3037000493 mod 2^64, seed 5."""

    def __init__(self):
        self.x = 5

    def next_unsigned(self):
        self.x = (2862933555777941757 * self.x + 3037000493) % (1 << 64)
        return self.x & 0x7FFFFFFFFFFFFFFF

    def next_int(self):
        return self.next_unsigned() - (1 << 62)

    def next_float(self):
        u = (self.next_unsigned() >> 11) & 0x001FFFFFFFFFFFFF
        return np.float64(np.ldexp(np.float64(u - 0x0010000000000000), -26))


def rng_for(tname):
    r = Rand64() if tname in ("int64", "double") else Rand32()
    return r, (r.next_float if tname in ("float", "double") else r.next_int)


def random_block(tname, dims):
    """encode_block.rs make_block: 4^dims values from the type's LCG."""
    _, nxt = rng_for(tname)
    return np.array([nxt() for _ in range(4 ** dims)], dtype=ZFP_TYPES[tname])


SPECIAL_FLOAT_BITS = [0x00000000, 0x80000000, 0x00000001, 0x80000001, 0x7F7FFFFF, 0xFF7FFFFF,
                      0x7F800000, 0xFF800000, 0x7FC00000, 0x7FA00000]
SPECIAL_DOUBLE_BITS = [0x0, 0x8000000000000000, 0x1, 0x8000000000000001, 0x7FEFFFFFFFFFFFFF,
                       0xFFEFFFFFFFFFFFFF, 0x7FF0000000000000, 0xFFF0000000000000, 0x7FF8000000000000,
                       0x7FF4000000000000]


def special_block(tname, dims, i):
    """encode_block.rs:117-139: special value at every 4th position, zeros elsewhere."""
    if tname == "float":
        b = np.zeros(4 ** dims, dtype=np.uint32)
        b[::4] = SPECIAL_FLOAT_BITS[i]
        return b.view(np.float32)
    b = np.zeros(4 ** dims, dtype=np.uint64)
    b[::4] = SPECIAL_DOUBLE_BITS[i]
    return b.view(np.float64)


# encode_block_strided.rs: SX = 2, SY = 3*4*SX, SZ = 2*4*SY, SW = 3*4*SZ;
# partial lengths PX=1, PY=2, PZ=3, PW=4; dummy 99 elsewhere.
STRIDES = (2, 24, 192, 2304)
PARTIAL = (1, 2, 3, 4)


def strided_array(tname, dims):
    """The strided test array (random values at strided positions, 99 elsewhere)."""
    st = STRIDES[:dims]
    counts = [4 * st[0]] + [st[d] // st[d - 1] for d in range(1, dims)]
    total = int(np.prod(counts))
    data = np.full(total, 99, dtype=ZFP_TYPES[tname])
    _, nxt = rng_for(tname)
    # Random values fill the strided positions in array order.
    it = np.ndindex(*reversed(counts))
    for idx in it:
        rev = list(reversed(idx))
        if all(rev[d] % (counts[d] // 4) == 0 for d in range(dims)):
            lin = 0
            mul = 1
            for d in range(dims):
                lin += rev[d] * mul
                mul *= counts[d]
            data[lin] = nxt()
    return data
