"""The CPU oracle (oracle/multislice.py) against outputs of the reference itself (tests/golden)."""
import numpy as np
import pytest

from conftest import rel_l2
from multem_b200 import specimens
from oracle import multislice as O


def small_stem():
    return specimens.stem_srtio3(nx=128, ny=128, na=4, nb=4, nc=4, ns=4, nconf=2, seed=7)


@pytest.mark.parametrize("Z", [8, 22, 38])
def test_spline_tables_float_bit_exact(golden, Z):
    p = small_stem()
    grid = O.Grid(p.nx, p.ny, p.spec_lx, p.spec_ly)
    t = O.atom_table(Z, grid.dRx)
    ref_head = golden[f"tab_Z{Z}_p1_head"]
    ref_tab = golden[f"tab_Z{Z}_p1_tab"]
    assert np.float32(t["R_max"]) == np.float32(ref_head[1])
    for i, k in enumerate(("R2", "c0", "c1", "c2", "c3")):
        np.testing.assert_array_equal(np.float32(t[k]), ref_tab[i].astype(np.float32))


def test_spline_tables_si(golden):
    p = specimens.hrtem_si001(nx=128, ny=128, na=2, nb=2, nc=2)
    grid = O.Grid(p.nx, p.ny, p.spec_lx, p.spec_ly)
    t = O.atom_table(14, grid.dRx)
    for i, k in enumerate(("R2", "c0", "c1", "c2", "c3")):
        np.testing.assert_array_equal(np.float32(t[k]), golden["tab_Z14_p1_tab"][i].astype(np.float32))


@pytest.mark.parametrize("pt", [1, 2, 3, 4])
def test_spline_tables_other_parameterisations(golden, pt):
    """Doyle-Turner, Peng (0-4, 0-12) and Kirkland tables: bit-exact in float except at the last knot,
    where the cosine taper leaves rounding noise around zero (|c0| ~ 1e-17)."""
    cases = ((small_stem(), (8, 22, 38)), (specimens.hrtem_si001(nx=128, ny=128, na=2, nb=2, nc=2), (14,)))
    for p, Zs in cases:
        grid = O.Grid(p.nx, p.ny, p.spec_lx, p.spec_ly)
        for Z in Zs:
            t = O.atom_table(Z, grid.dRx, potential_type=pt)
            assert np.float32(t["R_max"]) == np.float32(golden[f"tab_pt{pt}_Z{Z}_head"][1])
            ref = golden[f"tab_pt{pt}_Z{Z}_tab"].astype(np.float32)
            for i, k in enumerate(("R2", "c0", "c1", "c2", "c3")):
                got = np.float32(t[k])
                tiny = np.abs(ref[i]) < 1e-12 * np.abs(ref[i]).max()
                np.testing.assert_array_equal(got[~tiny], ref[i][~tiny])
                assert np.all(np.abs(got[tiny]) < 1e-12 * np.abs(ref[i]).max())


ION_TABLES = [(6, 8, -2), (6, 8, -1), (6, 22, 4), (6, 22, 2), (6, 38, 2), (6, 38, 1), (4, 14, 4), (4, 14, 1)]


@pytest.mark.parametrize("pt,Z,q", ION_TABLES)
def test_ionic_spline_tables_bit_exact(golden, pt, Z, q):
    """Peng's ionic tables (Sr 2+, Ti 2+/4+, O 1-/2-, Si 4+) and charges without an ionic entry
    (Sr 1+, Si 1+: the neutral table), with Lobato and Kirkland neutral atoms, bit-identical."""
    p = small_stem() if pt == 6 else specimens.hrtem_si001(nx=128, ny=128, na=2, nb=2, nc=2)
    grid = O.Grid(p.nx, p.ny, p.spec_lx, p.spec_ly)
    t = O.atom_table(Z, grid.dRx, potential_type=pt, charge=q)
    key = f"tab_ion_pt{pt}_Z{Z}_q{q}"
    assert np.float32(t["R_max"]) == np.float32(golden[key + "_head"][1])
    for i, k in enumerate(("R2", "c0", "c1", "c2", "c3")):
        np.testing.assert_array_equal(np.float32(t[k]), golden[key + "_tab"][i].astype(np.float32))


def test_projected_potential_float_bit_exact(golden):
    p = small_stem()
    grid = O.Grid(p.nx, p.ny, p.spec_lx, p.spec_ly)
    tabs = {Z: O.atom_table(Z, grid.dRx) for Z in (8, 22, 38)}
    Z = golden["stem_small_c1_Z"]
    xyz = golden["stem_small_c1_xyz"]
    i0, ie = golden["stem_small_c1_iatom_0"][3], golden["stem_small_c1_iatom_e"][3]
    V = O.projected_potential(grid, xyz[i0:ie + 1, :2], Z[i0:ie + 1], np.ones(ie - i0 + 1), tabs, dtype=np.float32)
    np.testing.assert_array_equal(V, golden["stem_small_V_c1_s3_p1"].T.astype(np.float32))
    V64 = O.projected_potential(grid, xyz[i0:ie + 1, :2], Z[i0:ie + 1], np.ones(ie - i0 + 1), tabs)
    assert rel_l2(V64, golden["stem_small_V_c1_s3_p1"].T) < 1e-5


@pytest.mark.parametrize("name,args", [("ew_small", (128, 128, 2, 2, 2)), ("ew_config1", (256, 256, 4, 4, 8))])
def test_exit_wave_matches_reference(golden, name, args):
    nx, ny, na, nb, nc = args
    p = specimens.hrtem_si001(nx=nx, ny=ny, na=na, nb=nb, nc=nc)
    grid = O.Grid(p.nx, p.ny, p.spec_lx, p.spec_ly)
    tabs = {14: O.atom_table(14, grid.dRx)}
    Z = golden[f"{name}_c1_Z"]
    xyz = golden[f"{name}_c1_xyz"]
    z0, ze = golden[f"{name}_c1_z_0"], golden[f"{name}_c1_z_e"]
    ia0, iae = golden[f"{name}_c1_iatom_0"], golden[f"{name}_c1_iatom_e"]
    lam, w = O.wavelength(p.E_0), O.vr_factor(p.E_0)
    Ts, dzs = [], []
    for k in range(len(z0)):
        n = max(0, iae[k] - ia0[k] + 1)
        V = O.projected_potential(grid, xyz[ia0[k]:iae[k] + 1, :2], Z[ia0[k]:iae[k] + 1], np.ones(n), tabs)
        Ts.append(O.transmission(V, float(w)))
        dzs.append(np.float32(np.float32(ze[k]) - np.float32(z0[k])))
    _, psi = O.multislice(grid, np.ones((nx, ny)), Ts, dzs, lam, {len(z0) - 1})
    # objective zero-defocus plane = first atom (obj_lens_zero_defocus_type = 1): back-propagate
    zbp = np.float32(np.float32(xyz[:, 2].min()) - 0.5 * (np.float64(z0[-1]) + np.float64(ze[-1])))
    psi = np.fft.ifft2(np.fft.fft2(psi) * O.propagator(grid, lam, zbp)) * (nx * ny)
    out = np.roll(np.roll(psi, -(nx // 2), 0), -(ny // 2), 1)
    ref64 = golden[f"{name}_run_p2_psi_coh"][0].T
    ref32 = golden[f"{name}_run_p1_psi_coh"][0].T
    assert rel_l2(out, ref64) < 1e-5
    assert rel_l2(out, ref32) < 1e-5


@pytest.mark.parametrize("name,tilt", [("prop", False), ("prop_tilt", True)])
@pytest.mark.parametrize("space", [1, 2])
def test_propagate_matches_reference(golden, name, tilt, space):
    """The numpy restatement of Propagator::operator() against the reference's own double path
    (ilc_propagate semantics) at z = 35 A, plain and with a tilted beam."""
    from cases import prop_case, prop_tilt_case
    p = prop_tilt_case() if tilt else prop_case()
    lam = float(O.wavelength(p.E_0, np.float64))
    grid = O.Grid(p.nx, p.ny, p.spec_lx, p.spec_ly)
    th = O.incident_angle(np.deg2rad(p.theta), lam, min(1 / p.spec_lx, 1 / p.spec_ly))
    ph = np.deg2rad(p.phi)
    gx0, gy0 = np.sin(th) * np.cos(ph) / lam, np.sin(th) * np.sin(ph) / lam
    out = O.propagate_wave(grid, lam, golden["prop_in"], 35.0, space, gx0, gy0)
    assert rel_l2(out, golden[f"{name}_z35_s{space}_p2"]) < 1e-6
    assert rel_l2(out, golden[f"{name}_z35_s{space}_p1"]) < 1e-5


def test_propagate_zero_distance(golden):
    """isZero(z): real space returns the wave, reciprocal space FFT2(psi)/N."""
    from cases import prop_case
    p = prop_case()
    grid = O.Grid(p.nx, p.ny, p.spec_lx, p.spec_ly)
    lam = O.wavelength(p.E_0, np.float32)
    assert rel_l2(O.propagate_wave(grid, lam, golden["prop_in"], 0.0, 1), golden["prop_z0_s1_p1"]) < 1e-7
    assert rel_l2(O.propagate_wave(grid, lam, golden["prop_in"], 0.0, 2), golden["prop_z0_s2_p1"]) < 1e-6
