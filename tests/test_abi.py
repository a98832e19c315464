"""The C-ABI library loads without a GPU and exports every entry point include/multem_b200.h declares."""
import re
from pathlib import Path

from multem_b200 import capi

HDR = Path(__file__).resolve().parents[1] / "include" / "multem_b200.h"


def declared():
    src = HDR.read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mt_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    lib = capi.load()
    names = declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_the_header():
    assert set(declared()) <= set(capi.SIGNATURES)


def test_abi_version_and_error_string():
    lib = capi.load()
    assert lib.mt_abi_version() == 1
    assert isinstance(lib.mt_last_error(), bytes)
