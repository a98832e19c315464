"""mt_multislice_run_batch: several different simulations in one call give exactly the outputs of
one mt_multislice_run call each (engines are deterministic; running them as the branches of one
CUDA graph, the default, or on concurrent host workers and CUDA streams must not change a bit)."""
import numpy as np
import pytest

from multem_b200 import api, specimens

pytestmark = pytest.mark.gpu


def _cases():
    from cases import ew_384x256, stem_384
    return [specimens.stem_srtio3(nx=128, ny=128, na=4, nb=4, nc=4, ns=4, nconf=2, seed=7),
            specimens.hrtem_si001(nx=128, ny=128, na=2, nb=2, nc=2),
            ew_384x256(), stem_384(),
            specimens.stem_srtio3(nx=256, ny=256, na=4, nb=4, nc=3, ns=3, nconf=1, seed=2)]


def _same(a, b):
    assert a.keys() == b.keys()
    for k in ("x", "y", "thick"):
        np.testing.assert_array_equal(a[k], b[k])
    assert a["dx"] == b["dx"] and a["dy"] == b["dy"]
    for da, db in zip(a["data"], b["data"]):
        for k in da:
            np.testing.assert_array_equal(np.asarray(da[k]), np.asarray(db[k]))


@pytest.mark.parametrize("mode", ["graph", "threads"])
@pytest.mark.parametrize("workers", ["1", "4"])
def test_batch_equals_single_runs(mode, workers, monkeypatch):
    monkeypatch.setenv("MTB_BATCH_WORKERS", workers)
    monkeypatch.setenv("MTB_BATCH_MODE", mode)
    ps = _cases()
    got = api.ilc_multem_batch(None, ps)
    for p, g in zip(ps, got):
        _same(g, api.ilc_multem(None, p))
