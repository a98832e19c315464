"""The C-ABI library loads without a GPU and exports every entry point include/*.h declares."""
import re
from pathlib import Path

import numpy as np
import pytest

from multem_b200 import capi

HDRS = sorted((Path(__file__).resolve().parents[1] / "include").glob("*.h"))


def declared():
    src = "\n".join(h.read_text() for h in HDRS)
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


def test_propagate_host_checks_and_zero_distance_without_gpu():
    """mt_propagate validates its input on the host, and at z = 0 in real space returns the wave
    itself (isZero in Propagator::operator()) without touching a GPU."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).parent / "golden"))
    from cases import prop_case
    from multem_b200 import api, capi
    p = prop_case()
    out = api.propagate(None, p, 0.0, 1)
    np.testing.assert_array_equal(out, np.asarray(p.iw_psi).astype(np.complex64))
    p.iw_type = 4
    with pytest.raises(capi.MtError) as e:
        api.propagate(None, p, 10.0, 1)
    assert e.value.status == 1
    q = prop_case()
    with pytest.raises(capi.MtError):
        api.propagate(None, q, 10.0, 3)


def test_batch_reports_per_input_status():
    """A batch with an unsupported input reports it by index and fills every status entry."""
    import ctypes as C
    from multem_b200 import specimens
    lib = capi.load()
    good = specimens.hrtem_si001(nx=128, ny=128, na=2, nb=2, nc=2)
    bad = specimens.hrtem_si001(nx=128, ny=128, na=2, nb=2, nc=2)
    bad.nx = 100
    ins = (capi.MtInputMultislice * 2)()
    keep = []
    for i, p in enumerate((good, bad)):
        s, k = p.to_c()
        keep.append((s, k))
        ins[i] = s
    outs = (capi.MtOutputMultislice * 2)()
    status = (C.c_int * 2)(-1, -1)
    rc = lib.mt_multislice_run_batch(None, 2, ins, outs, status)
    assert rc != 0
    assert all(v != -1 for v in status)
    assert status[1] != 0
    assert b"input" in lib.mt_last_error()
    assert lib.mt_multislice_run_batch(None, -1, ins, outs, None) == 1
