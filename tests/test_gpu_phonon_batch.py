"""Frozen-phonon configurations of exit-wave simulations advancing together.

With several configurations the engine runs up to eight of them per pass (each wave with its own
transmission functions) and adds their outputs thickness by thickness in configuration order, so
the results must equal those of one configuration at a time (MTB_EW_BATCH=1) bit for bit: for
real- and Fourier-space exit waves with a tilted beam, several thicknesses, the band-width limit,
electron diffraction with the coherent contribution, an HRTEM image with it, and displacements
drawn on the GPU; over batches that
divide the configurations and batches that do not (11 configurations: 8 + 3); through the graphs
of mt_multislice_run and through direct launches (tests/test_gpu_batch.py covers the recorded runs
of mt_multislice_run_batch)."""
import numpy as np
import pytest

from multem_b200 import api

pytestmark = pytest.mark.gpu


def _cases():
    from cases import ed_si001, ew_bwl_si001, ew_tilt_si001, ewfs_tilt_si001, hrtem_coherent_si001
    ew = ew_tilt_si001()
    ew.thick_type, ew.thick = 2, [10.0, 20.0, 30.0]
    ed = ed_si001()
    ed.pn_coh_contrib = 1
    hr = hrtem_coherent_si001()
    hr.pn_coh_contrib = 1
    dev = ew_tilt_si001()
    dev.pn_rng = 1  # displacements drawn on the GPU for every configuration of the batch
    return {"ewrs_tilt_3thick": ew, "ewfs_tilt": ewfs_tilt_si001(), "ewrs_bwl": ew_bwl_si001(), "ed_coh": ed,
            "hrtem_coh": hr, "ewrs_device_rng": dev}


def _arrays(out):
    keys = ("psi_coh", "m2psi_tot", "m2psi_coh")
    return {k: np.stack([np.asarray(d[k]) for d in out["data"]]) for k in keys if k in out["data"][0]}


@pytest.mark.parametrize("nconf", [5, 11])
@pytest.mark.parametrize("name", ["ewrs_tilt_3thick", "ewfs_tilt", "ewrs_bwl", "ed_coh", "hrtem_coh", "ewrs_device_rng"])
def test_batched_configurations_match_one_at_a_time(name, nconf, monkeypatch):
    p = _cases()[name]
    p.pn_model, p.pn_nconf = 3, nconf
    monkeypatch.setenv("MTB_EW_BATCH", "1")
    ref = _arrays(api.ilc_multem(None, p))
    monkeypatch.delenv("MTB_EW_BATCH")
    got = _arrays(api.ilc_multem(None, p))
    assert got.keys() == ref.keys()
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    # direct launches (no graphs) give the same
    monkeypatch.setenv("MTB_GRAPH", "0")
    direct = _arrays(api.ilc_multem(None, p))
    monkeypatch.delenv("MTB_GRAPH")
    for k in ref:
        np.testing.assert_array_equal(direct[k], ref[k], err_msg=k)

