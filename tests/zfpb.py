"""Import helper: the package directory `zfp-rs_b200` is not a Python identifier."""

import importlib.util
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "zfp-rs_b200"


def load():
    if "zfp_b200" in sys.modules:
        return sys.modules["zfp_b200"]
    spec = importlib.util.spec_from_file_location("zfp_b200", PKG / "zfp_b200.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["zfp_b200"] = mod
    spec.loader.exec_module(mod)
    return mod
