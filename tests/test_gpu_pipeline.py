"""The bulk-copy-fed line passes against the per-thread-load line passes.

The engine runs its row and column passes either with kernels whose threads load the wave
straight from global memory, or with kernels that stage each item's lines in shared memory through
the copy engine and keep the transmission rows resident; MTB_PIPE pins the choice (bit 0 rows,
bit 1 columns), otherwise the engine's autotuner picks the faster per shape. All variants compute
the same transforms with the same rounding, so the waves are bit-identical; the FP64 detector sums
are too where both variants use tiles of the same width, and agree to FP64 rounding (1e-13
relative) where they do not (1024: 8-column tiles in the bulk-copy-fed pass, 16 in the other; the
per-tile partials are then added in a different order). Cases cover:
several line groups per CTA in the row pass (a change of transmission rows inside a CTA), probe
counts that are and are not multiples of the row-pass unit, and the column pass's detector
partials.
"""
import numpy as np
import pytest

from multem_b200 import api, specimens

pytestmark = pytest.mark.gpu



def _stem(p, pipe, monkeypatch):
    monkeypatch.setenv("MTB_PIPE", str(pipe))
    e = api.Engine(p)
    r = e.run()
    e.close()
    return np.stack([np.stack(d["image_tot"]) for d in r["data"]])


@pytest.mark.parametrize("nx,ns", [(512, 4), (512, 3), (64, 4), (128, 4), (256, 4), (384, 4), (1024, 4), (2048, 4)])
def test_stem_pipelined_matches_per_thread_kernels(nx, ns, monkeypatch):
    p = specimens.stem_srtio3(nx=nx, ny=nx, na=4, nb=4, nc=6, ns=ns, nconf=1, seed=3)
    ref = _stem(p, 0, monkeypatch)
    exact = nx < 1024
    for pipe in (1, 2, 3):
        img = _stem(p, pipe, monkeypatch)
        assert img.shape == ref.shape
        if exact:
            np.testing.assert_array_equal(img, ref, err_msg=f"MTB_PIPE={pipe}")
        else:
            np.testing.assert_allclose(img, ref, rtol=1e-13, atol=0, err_msg=f"MTB_PIPE={pipe}")
    monkeypatch.delenv("MTB_PIPE")
    e = api.Engine(p)
    r = e.run()
    e.close()
    np.testing.assert_allclose(np.stack([np.stack(d["image_tot"]) for d in r["data"]]), ref, rtol=0 if exact else 1e-13,
                               atol=0)


@pytest.mark.parametrize("nx", [128, 256, 384, 512, 1024])
def test_exit_wave_pipelined_matches_per_thread_kernels(nx, monkeypatch):
    p = specimens.hrtem_si001(nx=nx, ny=nx, na=4, nb=4, nc=6)
    out = {}
    for pipe in (0, 3):
        monkeypatch.setenv("MTB_PIPE", str(pipe))
        r = api.ilc_multem(None, p)
        out[pipe] = np.stack([np.asarray(d["psi_coh"]) for d in r["data"]])
    np.testing.assert_array_equal(out[3], out[0])


@pytest.mark.parametrize("shape", [1, 2])
@pytest.mark.parametrize("nx", [64, 128, 256, 384, 512, 1024, 2048])
def test_alternative_pipeline_shapes_match(nx, shape, monkeypatch):
    """The autotuner's alternative pipeline shapes of the slice step (shape 1: one-warp row groups,
    4 x 128 column groups; shape 2: early issue with full exchange buffers) give the waves of the
    per-thread-load kernels bit for bit."""
    p = specimens.stem_srtio3(nx=nx, ny=nx, na=4, nb=4, nc=6 if nx < 2048 else 2, ns=4, nconf=1, seed=3)
    ref = _stem(p, 0, monkeypatch)
    monkeypatch.setenv("MTB_SHAPE", str(shape | (shape << 2)))
    img = _stem(p, 3, monkeypatch)
    monkeypatch.delenv("MTB_SHAPE")
    if nx == 1024:
        np.testing.assert_allclose(img, ref, rtol=1e-13, atol=0)
    else:
        np.testing.assert_array_equal(img, ref)


def test_autotuner_reports_its_choice():
    p = specimens.stem_srtio3(nx=512, ny=512, na=8, nb=8, nc=3, ns=16, nconf=1, seed=3)
    e = api.Engine(p)
    e.run()
    t = e.tuning()
    e.close()
    assert t["rows"] in (0, 1, 2, 3) and t["cols"] in (0, 1, 2, 3)
    assert t["probes_per_launch"] in (128, 256)
