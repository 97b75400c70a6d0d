"""Generate tests/golden/checksums.json from the reference's own golden tables.

Reads zfp-rs's tests/c/checksums.rs (a port of C zfp's
tests/constants/checksums/*.h) and writes every (dims, type, key1, key2,
checksum) entry as JSON.  Run once, in a checkout that has the reference:

    python tests/golden/make_golden.py /path/to/zfp-rs

The JSON is committed; the tests never read the reference itself.
"""

import json
import re
import sys
from pathlib import Path

TABLE = re.compile(r"static CHECKSUMS_(\d)D_(INT32|INT64|FLOAT|DOUBLE): &\[\(u64, u64, u64\)\] = &\[(.*?)\];", re.S)
ENTRY = re.compile(r"\(\s*(0x[0-9a-fA-F]+|\d+)\s*,\s*(0x[0-9a-fA-F]+|\d+)\s*,\s*(0x[0-9a-fA-F]+|\d+)\s*\)")
TYPES = {"INT32": "int32", "INT64": "int64", "FLOAT": "float", "DOUBLE": "double"}


def main(root: str) -> None:
    src = (Path(root) / "tests" / "c" / "checksums.rs").read_text()
    out = []
    for dims, ty, body in TABLE.findall(src):
        for k1, k2, cs in ENTRY.findall(body):
            out.append({"dims": int(dims), "type": TYPES[ty], "key1": int(k1, 0), "key2": int(k2, 0),
                        "checksum": int(cs, 0)})
    dest = Path(__file__).with_name("checksums.json")
    dest.write_text(json.dumps({"source": "zfp-rs 1.0.1 tests/c/checksums.rs:268-757", "entries": out}, indent=0))
    print(f"wrote {len(out)} entries to {dest}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <zfp-rs checkout>")
    main(sys.argv[1])
