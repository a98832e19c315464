"""The allocation-free spline-table entry point (mt_spline_tables_noalloc).

It is for callers that cannot call cudaMalloc: code whose GPU memory belongs to a framework's pool
allocator (an allocation outside the pool escapes its budget, or fails once the pool holds the
device's memory), and loops that must not allocate while they run. They pass their own device
output buffer; the library's only scratch is a fixed device array inside the library. This test
calls it (and mt_spline_tables_noalloc_ex for other parameterisations) through the C ABI several
times in a row, on different element lists, checks each result against the allocating entry with
the tolerance the table-parity test uses, and checks that the calls make no device allocation
(the library's allocation counter does not move). The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from multem_b200 import api, capi

pytestmark = pytest.mark.gpu

RTOL = 2e-6


def _noalloc(lib, Z, dR, nR, torch, pt=6):
    z = np.ascontiguousarray(np.asarray(Z, dtype=np.int32))
    d_tab = torch.full((z.size * 5 * nR,), float("nan"), dtype=torch.float32, device="cuda")
    heads = np.zeros((z.size, 4))
    stream = torch.cuda.current_stream()
    args = (z.ctypes.data_as(capi.P_int), z.size, float(dR), 0.015, nR, heads.ctypes.data_as(capi.P_double),
            C.c_void_p(d_tab.data_ptr()), C.c_void_p(stream.cuda_stream))
    if pt == 6:
        rc = lib.mt_spline_tables_noalloc(*args)
    else:  # (potential_type, Z, charge = NULL for neutral atoms, n, ...)
        rc = lib.mt_spline_tables_noalloc_ex(pt, args[0], None, *args[1:])
    capi.check(rc)
    stream.synchronize()
    return heads, d_tab.cpu().numpy().reshape(z.size, 5, nR)


def _alloc_count(lib):
    n = C.c_longlong(-1)
    capi.check(lib.mt_device_alloc_count(C.byref(n)))
    return n.value


def test_noalloc_tables_match_allocating_entry_on_two_calls():
    torch = pytest.importorskip("torch")
    lib = capi.load()
    dR = np.float32(np.float32(15.62) / np.float32(128))
    for Z, pt in (([8, 22, 38], 6), ([14, 79, 6, 1, 78], 6), ([14, 79, 6, 1, 78], 4), ([8, 22, 38], 3)):
        heads_ref, tab_ref = api.spline_tables(Z, float(dR), potential_type=pt)
        n0 = _alloc_count(lib)
        heads, tab = _noalloc(lib, Z, dR, 128, torch, pt)
        assert _alloc_count(lib) == n0, "the allocation-free entry point allocated device memory"
        np.testing.assert_array_equal(heads, heads_ref)
        assert np.all(np.isfinite(tab))
        for i in range(len(Z)):
            for k in range(5):
                ref = tab_ref[i, k]
                np.testing.assert_allclose(tab[i, k], ref, rtol=RTOL, atol=1e-7 * np.abs(ref).max())


def test_noalloc_rejects_requests_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    lib = capi.load()
    z = np.full(129, 6, dtype=np.int32)
    d_tab = torch.zeros(129 * 5 * 128, dtype=torch.float32, device="cuda")
    rc = lib.mt_spline_tables_noalloc(z.ctypes.data_as(capi.P_int), 129, 0.06, 0.015, 128, None,
                                      C.c_void_p(d_tab.data_ptr()), None)
    assert rc == 1  # MT_ERR_INVALID_ARG
    assert b"128" in lib.mt_last_error()
