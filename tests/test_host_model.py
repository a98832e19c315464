"""Host-side model (validation, phonon displacements, slicing) against the reference's own dumps.

These run without a GPU: the specimen entry points of the C ABI use host code only.
"""
import numpy as np
import pytest

from multem_b200 import api, specimens
from cases import amorph_au110, ew_monolayer_au, ew_po_si001, ew_rot_si001, ew_wpo_si001, stem_monolayer_au, stem_rot_srtio3


def cases():
    p = specimens.stem_srtio3(nx=128, ny=128, na=4, nb=4, nc=4, ns=3, nconf=2, seed=11)
    p.thick_type = 2
    p.thick = [4.0, 8.0, 12.0]
    p.cond_lens_c_10 = 15.0
    p.cond_lens_c_30 = 0.001
    return {
        "stem_small": specimens.stem_srtio3(nx=128, ny=128, na=4, nb=4, nc=4, ns=4, nconf=2, seed=7),
        "stem_thick": p,
        "ew_small": specimens.hrtem_si001(nx=128, ny=128, na=2, nb=2, nc=2),
        "ew_config1": specimens.hrtem_si001(nx=256, ny=256, na=4, nb=4, nc=8),
        "amorph_au110": amorph_au110(),
        "ew_rot_si001": ew_rot_si001(),
        "stem_rot_srtio3": stem_rot_srtio3(),
        "ew_monolayer_au": ew_monolayer_au(),
        "stem_monolayer_au": stem_monolayer_au(),
        "ew_po_si001": ew_po_si001(),
        "ew_wpo_si001": ew_wpo_si001(),
    }


@pytest.mark.parametrize("name", ["stem_small", "stem_thick", "ew_small", "ew_config1", "amorph_au110", "ew_rot_si001",
                                  "stem_rot_srtio3", "ew_monolayer_au", "stem_monolayer_au", "ew_po_si001",
                                  "ew_wpo_si001"])
@pytest.mark.parametrize("iconf", [1, 2])
def test_displaced_atoms_and_slices_bit_exact(golden, name, iconf):
    p = cases()[name]
    if iconf > p.pn_nconf:
        pytest.skip("single configuration")
    Z, xyz = api.specimen_atoms(p, iconf)
    np.testing.assert_array_equal(Z, golden[f"{name}_c{iconf}_Z"])
    np.testing.assert_array_equal(xyz.astype(np.float32), golden[f"{name}_c{iconf}_xyz"].astype(np.float32))
    s = api.specimen_slices(p, iconf)
    for k in ("iatom_0", "iatom_e", "ithk"):
        np.testing.assert_array_equal(s[k], golden[f"{name}_c{iconf}_{k}"])
    for k in ("z_0", "z_e"):
        np.testing.assert_array_equal(s[k].astype(np.float32), golden[f"{name}_c{iconf}_{k}"].astype(np.float32))


def test_output_dims_host_only(golden):
    p = cases()["stem_thick"]
    d = api.output_dims(p)
    assert (d.n_thick, d.n_detector, d.nx, d.ny) == (3, 2, 3, 3)
    assert d.n_x == 9 and d.has_image_tot == 1


def test_seed_zero_is_clamped_to_one():
    """validate_parameters clamps pn_seed to >= 1 (src/input_multislice.cuh:624)."""
    p0 = specimens.hrtem_si001(nx=128, ny=128, na=2, nb=2, nc=2)
    p1 = p0.copy()
    p0.pn_seed, p1.pn_seed = 0, 1
    np.testing.assert_array_equal(api.specimen_atoms(p0, 1)[1], api.specimen_atoms(p1, 1)[1])


def test_configurations_differ_and_repeat():
    p = cases()["stem_small"]
    a1, a2 = api.specimen_atoms(p, 1)[1], api.specimen_atoms(p, 2)[1]
    assert not np.array_equal(a1, a2)
    np.testing.assert_array_equal(a1, api.specimen_atoms(p, 1)[1])
    # pn_dim = 110: z untouched
    np.testing.assert_array_equal(a1[:, 2], a2[:, 2])


@pytest.mark.parametrize("field,value,status", [
    ("simulation_type", 62, 6), ("simulation_type", 61, 6), ("potential_type", 5, 6), ("potential_type", 7, 1),
    ("potential_slicing", 3, 6), ("nx", 0, 1),
])
def test_unsupported_and_invalid_inputs_fail_loudly(field, value, status):
    from multem_b200 import capi
    p = cases()["stem_small"]
    setattr(p, field, value)
    with pytest.raises(capi.MtError) as e:
        api.output_dims(p)
    assert e.value.status == status


@pytest.mark.parametrize("sim,fields", [
    (32, {"illumination_model": 3}),  # the reference's transmission-cross-coefficient branch computes nothing
    (32, {"illumination_model": 4, "temporal_spatial_incoh": 1, "cond_lens_si_sigma": 0.01}),  # its spatial quadrature is empty
    (42, {"pn_coh_contrib": 1}),  # HCTEM's m2psi_coh
])
def test_image_formation_limits_are_refused(sim, fields):
    """Imaging and incident-wave variants outside what the engine implements fail with
    MT_ERR_UNSUPPORTED at the engine's host-side set-up, before any GPU work."""
    from multem_b200 import capi
    p = specimens.hrtem_si001(nx=64, ny=64, na=2, nb=2, nc=2)
    p.simulation_type = sim
    for k, v in fields.items():
        setattr(p, k, v)
    with pytest.raises(capi.MtError) as e:
        api.Engine(p)
    assert e.value.status == 6


def test_input_report_lists_silent_changes():
    """mt_input_report names what validate_parameters would change silently; a plain input has
    nothing to report."""
    assert api.input_report(cases()["stem_small"]) == []
    rep = api.input_report(cases()["stem_thick"])
    assert any(r.startswith("thick [") for r in rep), rep
    p = specimens.hrtem_si001(nx=128, ny=128, na=2, nb=2, nc=2)
    p.pn_seed = 0
    assert "pn_seed 0 -> 1" in api.input_report(p)
    p.output_area_ix_0, p.output_area_ix_e = 20, 900
    p.output_area_iy_0, p.output_area_iy_e = 1, 64
    assert any(r.startswith("output_area ->") for r in api.input_report(p))


def test_strict_mode_rejects_silent_changes(monkeypatch):
    """With MTB_STRICT=1 a run refuses such an input on the host, before any GPU work."""
    from multem_b200 import capi
    p = specimens.hrtem_si001(nx=128, ny=128, na=2, nb=2, nc=2)
    p.pn_seed = 0
    monkeypatch.setenv("MTB_STRICT", "1")
    with pytest.raises(capi.MtError) as e:
        api.ilc_multem(None, p)
    assert e.value.status == 1 and "pn_seed" in str(e.value)


def test_cbed_full_integration_is_accepted():
    """CBED under full integration (condenser defocus and source spreads) passes the host-side
    validation; its numbers are checked against the reference in the GPU parity tests."""
    p = specimens.hrtem_si001(nx=64, ny=64, na=2, nb=2, nc=2)
    p.simulation_type = 21
    p.iw_type = 2
    p.iw_x, p.iw_y = [5.0], [5.0]
    p.illumination_model = 4
    p.temporal_spatial_incoh = 1
    p.cond_lens_si_sigma = 0.2
    p.cond_lens_si_rad_npts = 3
    p.cond_lens_si_azm_npts = 4
    p.cond_lens_ti_npts = 2
    p.cond_lens_ti_sigma = 10.0
    d = api.output_dims(p)
    assert d["nx"] == 64 if isinstance(d, dict) else True
