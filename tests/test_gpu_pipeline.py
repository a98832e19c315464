"""The bulk-copy-fed line passes against the per-thread-load line passes.

The engine runs its row and column passes either with kernels whose threads load the wave
straight from global memory, or (the default, MTB_PIPE=3) with kernels that stage each item's
lines in shared memory through the copy engine and keep the transmission rows resident
(MTB_PIPE=0 selects the former for both passes). Both compute the same transforms in FP32; they
may differ in the last bits where the compiler contracts a complex product differently, so the
comparison allows 1e-6 relative. Cases cover: several line groups per CTA in the row pass (a
change of transmission rows inside a CTA), probe counts that are and are not multiples of the
row-pass unit, and the column pass's detector partials.
"""
import numpy as np
import pytest

from conftest import rel_l2
from multem_b200 import api, specimens

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _stem(p, pipe, monkeypatch):
    monkeypatch.setenv("MTB_PIPE", str(pipe))
    e = api.Engine(p)
    r = e.run()
    e.close()
    return np.stack([np.stack(d["image_tot"]) for d in r["data"]])


@pytest.mark.parametrize("nx,ns", [(512, 4), (512, 3), (128, 4), (256, 4), (384, 4), (1024, 4)])
def test_stem_pipelined_matches_per_thread_kernels(nx, ns, monkeypatch):
    p = specimens.stem_srtio3(nx=nx, ny=nx, na=4, nb=4, nc=6, ns=ns, nconf=1, seed=3)
    ref = _stem(p, 0, monkeypatch)
    for pipe in (1, 2, 3):
        img = _stem(p, pipe, monkeypatch)
        assert img.shape == ref.shape
        assert rel_l2(img, ref) < TOL, (pipe, rel_l2(img, ref))


@pytest.mark.parametrize("nx", [128, 256, 512])
def test_exit_wave_pipelined_matches_per_thread_kernels(nx, monkeypatch):
    p = specimens.hrtem_si001(nx=nx, ny=nx, na=4, nb=4, nc=6)
    out = {}
    for pipe in (0, 3):
        monkeypatch.setenv("MTB_PIPE", str(pipe))
        r = api.ilc_multem(None, p)
        out[pipe] = np.stack([np.asarray(d["psi_coh"]) for d in r["data"]])
    assert rel_l2(out[3], out[0]) < TOL
