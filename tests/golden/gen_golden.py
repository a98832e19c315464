"""Generate golden fixtures from the reference's own CPU path (oracle/_ref/libmultem_ref.so).

The reference has no test vectors of its own, so these fixtures are outputs of the reference code
itself (its Multislice<T, e_host>, compiled from its sources by oracle/Makefile) on small seeded
inputs. They let the oracle and the engine be checked where oracle/_ref is not built.

    make -C oracle && python tests/golden/gen_golden.py

The full runs use 8 host threads, and the reference's threaded CPU path does not sum in a fixed
order: a regeneration reproduces them only to float rounding (about 1e-6 relative in FP32), so
arrays already in the file are kept and only new keys are added (--overwrite replaces all).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from multem_b200 import specimens  # noqa: E402
from cases import (amorph_au110, ew_1024, ew_384x256, prop_case, prop_tilt_case, stem_1024, stem_384,  # noqa: E402
                   stem_tilt_au001, ew_tilt_si001, ewfs_tilt_si001, stem_incoh_srtio3, stem_matrix_srtio3,
                   stem_coh_srtio3, ed_si001, hrtem_coherent_si001, hrtem_pctf_si001, hrtem_fullint_si001,
                   cbed_si001, cbei_si001, ewrs_two_beams_si001, ewrs_user_wave_si001, hrtem_user_wave_si001,
                   ew_rot_si001, stem_rot_srtio3, ped_si001, hctem_si001, istem_srtio3, ew_monolayer_au,
                   stem_monolayer_au, ew_po_si001, ew_wpo_si001, ew_bwl_si001, stem_bwl_srtio3, hrtem_bwl_si001,
                   ew_doyle_si001, ew_peng4_si001, ew_kirkland_si001, stem_peng12_srtio3, stem_kirkland_srtio3,
                   stem_ions_srtio3, ew_ions_si001, cbed_full_si001, cbei_full_si001, ed_coh_si001,
                   cbed_coh_si001, ped_coh_si001, hrtem_coh_si001, cbei_coh_si001, stem_bench512,
                   ew_au110_ac_2048, ed_au110_ac_2048)
from oracle import reference as R  # noqa: E402

OUT = Path(__file__).resolve().parent


def stem_small():
    return specimens.stem_srtio3(nx=128, ny=128, na=4, nb=4, nc=4, ns=4, nconf=2, seed=7)


def stem_thick():
    p = specimens.stem_srtio3(nx=128, ny=128, na=4, nb=4, nc=4, ns=3, nconf=2, seed=11)
    p.thick_type = 2
    p.thick = [4.0, 8.0, 12.0]
    p.cond_lens_c_10 = 15.0
    p.cond_lens_c_30 = 0.001
    return p


def ew_small():
    return specimens.hrtem_si001(nx=128, ny=128, na=2, nb=2, nc=2)


def ew_config1():
    return specimens.hrtem_si001(nx=256, ny=256, na=4, nb=4, nc=8)


FULL_RUNS = (("ew_384x256", ew_384x256), ("stem_384", stem_384), ("ew_1024", ew_1024), ("stem_1024", stem_1024),
             ("amorph_au110", amorph_au110), ("stem_tilt_au001", stem_tilt_au001), ("ew_tilt_si001", ew_tilt_si001),
             ("ewfs_tilt_si001", ewfs_tilt_si001), ("stem_incoh_srtio3", stem_incoh_srtio3),
             ("stem_matrix_srtio3", stem_matrix_srtio3), ("stem_coh_srtio3", stem_coh_srtio3),
             ("ed_si001", ed_si001), ("hrtem_coherent_si001", hrtem_coherent_si001),
             ("hrtem_pctf_si001", hrtem_pctf_si001), ("hrtem_fullint_si001", hrtem_fullint_si001),
             ("cbed_si001", cbed_si001), ("cbei_si001", cbei_si001), ("ewrs_two_beams_si001", ewrs_two_beams_si001),
             ("ewrs_user_wave_si001", ewrs_user_wave_si001), ("hrtem_user_wave_si001", hrtem_user_wave_si001),
             ("ew_rot_si001", ew_rot_si001), ("stem_rot_srtio3", stem_rot_srtio3),
             ("ped_si001", ped_si001), ("hctem_si001", hctem_si001), ("istem_srtio3", istem_srtio3),
             ("ew_monolayer_au", ew_monolayer_au), ("stem_monolayer_au", stem_monolayer_au), ("ew_po_si001", ew_po_si001),
             ("ew_wpo_si001", ew_wpo_si001), ("ew_bwl_si001", ew_bwl_si001), ("stem_bwl_srtio3", stem_bwl_srtio3),
             ("hrtem_bwl_si001", hrtem_bwl_si001), ("ew_doyle_si001", ew_doyle_si001), ("ew_peng4_si001", ew_peng4_si001),
             ("ew_kirkland_si001", ew_kirkland_si001), ("stem_peng12_srtio3", stem_peng12_srtio3),
             ("stem_kirkland_srtio3", stem_kirkland_srtio3), ("stem_ions_srtio3", stem_ions_srtio3),
             ("ew_ions_si001", ew_ions_si001), ("cbed_full_si001", cbed_full_si001),
             ("cbei_full_si001", cbei_full_si001), ("ed_coh_si001", ed_coh_si001), ("cbed_coh_si001", cbed_coh_si001),
             ("ped_coh_si001", ped_coh_si001), ("hrtem_coh_si001", hrtem_coh_si001), ("cbei_coh_si001", cbei_coh_si001),
             ("stem_bench512", stem_bench512), ("ew_au110_ac_2048", ew_au110_ac_2048),
             ("ed_au110_ac_2048", ed_au110_ac_2048))

SPECIMENS = (("ew_rot_si001", ew_rot_si001), ("stem_rot_srtio3", stem_rot_srtio3), ("ew_monolayer_au", ew_monolayer_au),
             ("stem_monolayer_au", stem_monolayer_au), ("ew_po_si001", ew_po_si001), ("ew_wpo_si001", ew_wpo_si001))


def specimen_fixtures(rec, names=None):
    """Displaced atoms and slicing of configurations 1 and 2 from the reference (SPECIMENS)."""
    for name, fn in SPECIMENS:
        if names is not None and name not in names:
            continue
        p = fn()
        for iconf in (1, 2):
            if iconf > p.pn_nconf:
                continue
            sp = R.specimen(p, iconf)
            for k in ("Z", "xyz", "z_0", "z_e", "iatom_0", "iatom_e", "ithk"):
                rec[f"{name}_c{iconf}_{k}"] = sp[k]


def full_runs(rec, names=None):
    """Full reference runs (outputs stored in single precision) of FULL_RUNS, or of `names`."""
    for name, fn in FULL_RUNS:
        if names is not None and name not in names:
            continue
        p = fn()
        for prec in (1, 2):
            out = R.run(p, precision=prec, nthreads=8)
            for k in ("image_tot", "image_coh", "psi_coh", "m2psi_tot", "m2psi_coh", "thick", "x", "y"):
                if k in out:
                    v = out[k]
                    rec[f"{name}_run_p{prec}_{k}"] = v.astype(np.complex64 if np.iscomplexobj(v) else np.float64)


def potential_table_fixtures(rec):
    """Spline tables of potential_type 1-4 (Doyle-Turner, Peng 0-4, Peng 0-12, Kirkland) for O, Ti, Sr
    at the small STEM grid's sampling and for Si at the small exit-wave grid's."""
    for pt in (1, 2, 3, 4):
        for fn, Zs in ((stem_small, (8, 22, 38)), (ew_small, (14,))):
            p = fn()
            p.potential_type = pt
            for Z in Zs:
                t = R.atom_type(p, Z, 1)
                rec[f"tab_pt{pt}_Z{Z}_head"] = np.array([t["R_min"], t["R_max"], t["R_tap"], t["tap_cf"]])
                rec[f"tab_pt{pt}_Z{Z}_tab"] = np.stack([t[k] for k in ("R2", "c0", "c1", "c2", "c3")])
    # ionic tables (Peng 0-4 ions; any potential_type): charges with and without an ionic entry
    for pt, fn, Zq in ((6, stem_small, ((8, -2), (8, -1), (22, 4), (22, 2), (38, 2), (38, 1))),
                       (4, ew_small, ((14, 4), (14, 1)))):
        p = fn()
        p.potential_type = pt
        for Z, q in Zq:
            t = R.atom_type(p, Z, 1, charge=q)
            key = f"tab_ion_pt{pt}_Z{Z}_q{q}"
            rec[key + "_head"] = np.array([t["R_min"], t["R_max"], t["R_tap"], t["tap_cf"]])
            rec[key + "_tab"] = np.stack([t[k] for k in ("R2", "c0", "c1", "c2", "c3")])


def add_only(names):
    """Adds the full runs of `names` to the existing fixture file (other arrays kept); the name
    potential_tables adds potential_table_fixtures."""
    path = OUT / "reference_fixtures.npz"
    old = np.load(path)
    rec = {k: old[k] for k in old.files}
    full_runs(rec, names)
    specimen_fixtures(rec, names)
    if "potential_tables" in names:
        potential_table_fixtures(rec)
    np.savez_compressed(path, **rec)
    print("wrote", path, len(rec), "arrays")


def main():
    if not R.available():
        raise SystemExit("oracle/_ref not built: make -C oracle")
    if "--only" in sys.argv:
        return add_only(sys.argv[sys.argv.index("--only") + 1].split(","))
    rec = {}
    # specimen host logic: displaced atoms and slicing of two configurations
    for name, fn in (("stem_small", stem_small), ("stem_thick", stem_thick), ("ew_small", ew_small),
                     ("ew_config1", ew_config1), ("amorph_au110", amorph_au110)):
        p = fn()
        for iconf in (1, 2):
            if iconf > p.pn_nconf:
                continue
            sp = R.specimen(p, iconf)
            for k in ("Z", "xyz", "z_0", "z_e", "iatom_0", "iatom_e", "ithk"):
                rec[f"{name}_c{iconf}_{k}"] = sp[k]
        rec[f"{name}_params"] = np.array([R.params(p)[k] for k in ("lambda", "Vr_factor", "cond_zero_defocus_plane",
                                                                  "n_slice", "n_atoms", "dz", "n_thick")])
    # spline tables at the small grids' sampling
    p = stem_small()
    for Z in (8, 22, 38):
        for prec in (1, 2):
            t = R.atom_type(p, Z, prec)
            rec[f"tab_Z{Z}_p{prec}_head"] = np.array([t["R_min"], t["R_max"], t["R_tap"], t["tap_cf"]])
            rec[f"tab_Z{Z}_p{prec}_tab"] = np.stack([t[k] for k in ("R2", "c0", "c1", "c2", "c3")])
    q = ew_small()
    for prec in (1, 2):
        t = R.atom_type(q, 14, prec)
        rec[f"tab_Z14_p{prec}_head"] = np.array([t["R_min"], t["R_max"], t["R_tap"], t["tap_cf"]])
        rec[f"tab_Z14_p{prec}_tab"] = np.stack([t[k] for k in ("R2", "c0", "c1", "c2", "c3")])
    potential_table_fixtures(rec)
    # projected potential and transmission of one slice
    for prec in (1, 2):
        rec[f"stem_small_V_c1_s3_p{prec}"] = R.projected_potential(p, 1, 3, prec).astype(np.float64)
        rec[f"stem_small_T_c1_s3_p{prec}"] = R.transmission_function(p, 1, 3, prec).astype(np.complex128)
    # incident wave at an off-centre position
    pw = stem_small()
    pw.iw_x, pw.iw_y = [3.3], [7.1]
    pw.cond_lens_c_10 = 25.0
    pw.cond_lens_c_30 = 0.002
    for prec in (1, 2):
        rec[f"probe_real_p{prec}"] = R.incident_wave(pw, 1, prec)
        rec[f"probe_fourier_p{prec}"] = R.incident_wave(pw, 2, prec)
    # propagation of a user wave (ilc_propagate), plain and with a beam tilt
    rec["prop_in"] = np.asarray(prop_case().iw_psi)
    for name, fn, zs in (("prop", prop_case, (0.0, 35.0)), ("prop_tilt", prop_tilt_case, (35.0,))):
        q = fn()
        for z in zs:
            for space in (1, 2):
                for prec in ((1, 2) if z != 0 else (1,)):
                    r = R.propagate(q, z, space, prec)
                    rec[f"{name}_z{int(z)}_s{space}_p{prec}"] = r.astype(np.complex64) if prec == 1 else r
    # full runs on a radix-3 grid, a 1024^2 grid, an amorphous layer and a tilted beam
    full_runs(rec)
    specimen_fixtures(rec)
    # full runs
    for name, fn in (("stem_small", stem_small), ("stem_thick", stem_thick), ("ew_small", ew_small),
                     ("ew_config1", ew_config1)):
        p = fn()
        for prec in (1, 2):
            out = R.run(p, precision=prec, nthreads=8)
            for k in ("image_tot", "psi_coh", "m2psi_tot", "thick", "x", "y"):
                if k in out:
                    v = out[k]
                    rec[f"{name}_run_p{prec}_{k}"] = v.astype(np.complex64 if np.iscomplexobj(v) else np.float64) \
                        if name == "ew_config1" else v
    path = OUT / "reference_fixtures.npz"
    if path.exists() and "--overwrite" not in sys.argv:
        old = np.load(path)
        rec.update({k: old[k] for k in old.files})
    np.savez_compressed(path, **rec)
    print("wrote", OUT / "reference_fixtures.npz", len(rec), "arrays")


if __name__ == "__main__":
    main()
