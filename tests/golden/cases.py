"""Inputs of the golden cases that are not specimens (shared by gen_golden.py and the tests)."""
import numpy as np

from multem_b200 import Parameters


def prop_case():
    """A seeded smooth user wave on a 128 x 64 grid (non-square) for ilc_propagate, 200 kV."""
    p = Parameters()
    p.nx, p.ny = 128, 64
    p.spec_lx, p.spec_ly = 20.0, 10.0
    p.E_0 = 200.0
    p.iw_type = 3
    rng = np.random.default_rng(21)
    y, x = np.meshgrid(np.arange(p.ny) * p.spec_ly / p.ny, np.arange(p.nx) * p.spec_lx / p.nx, indexing="ij")
    env = np.exp(-((x - 10.0) ** 2 + (y - 5.0) ** 2) / (2 * 3.0 ** 2))
    phase = rng.standard_normal((p.ny, p.nx))
    p.iw_psi = env * np.exp(1j * 0.5 * phase)
    p.iw_x, p.iw_y = [0.0], [0.0]
    return p


def prop_tilt_case():
    """prop_case with the beam tilted by 0.5 deg at azimuth 30 deg."""
    p = prop_case()
    p.theta, p.phi = 0.5, 30.0
    return p


def ew_384x256():
    """Exit wave of Si(001) on a 384 x 256 grid (radix-3 rows against radix-2 columns), written to
    a 128 x 96 output window (cropping and fft-shift of the output area)."""
    from multem_b200 import specimens
    p = specimens.hrtem_si001(nx=384, ny=256, na=4, nb=3, nc=4)
    p.output_area_ix_0, p.output_area_ix_e = 101, 228
    p.output_area_iy_0, p.output_area_iy_e = 81, 176
    return p


def stem_384():
    """STEM ADF through SrTiO3(001) on a 384^2 grid, 3 x 3 probes, two phonon configurations."""
    from multem_b200 import specimens
    return specimens.stem_srtio3(nx=384, ny=384, na=4, nb=4, nc=4, ns=3, nconf=2, seed=5)


def ew_1024():
    """Exit wave of Si(001) on a 1024^2 grid (41.5 x 41.5 A) with a 128 x 128 output window."""
    from multem_b200 import specimens
    p = specimens.hrtem_si001(nx=1024, ny=1024, na=8, nb=8, nc=2)
    p.output_area_ix_0, p.output_area_ix_e = 449, 577
    p.output_area_iy_0, p.output_area_iy_e = 449, 577
    return p


def stem_1024():
    """STEM ADF through SrTiO3(001) on a 1024^2 grid, 2 x 2 probes, one phonon configuration."""
    from multem_b200 import specimens
    return specimens.stem_srtio3(nx=1024, ny=1024, na=8, nb=8, nc=3, ns=2, nconf=1, seed=9)


def amorph_au110():
    """Au(110) crystal (6 x 4 x 6 cells, 17.3 x 16.3 x 17.3 A) under a 10 A amorphous carbon layer
    (2.0 g/cm^3, minimum spacing 1.4 A, region 1, slices of 2 A in the layer), exit wave on a 256^2
    grid at 200 kV written to a 96 x 96 window, dz_Proj slicing of the crystal with a'/2, two
    frozen-phonon configurations."""
    import numpy as np
    from multem_b200 import Parameters, specimens
    a = 4.078
    cell = specimens.fcc_110(79, a)
    na, nb, nc = 6, 4, 6
    lx, ly = na * cell[0], nb * cell[1]
    t_am = 10.0
    xtal = specimens.crystal(cell, na, nb, nc, sigma=0.085)
    xtal[:, 3] += t_am + 0.5 * cell[2]
    am = specimens.amorphous_layer(6, lx, ly, 0.0, t_am, 2.0, 12.011, 1.4, 0.085, seed=5, region=1)
    p = Parameters()
    p.simulation_type = 52
    p.pn_model = 3
    p.pn_coh_contrib = 0
    p.pn_single_conf = 0
    p.pn_nconf = 2
    p.pn_dim = 110
    p.pn_seed = 17
    p.spec_atoms = np.vstack([am, xtal])
    p.spec_lx, p.spec_ly = lx, ly
    p.spec_lz = t_am + nc * cell[2] + cell[2]
    p.spec_dz = cell[2] / 2
    p.spec_amorp = [{"z_0": 0.0, "z_e": t_am, "dz": 2.0}]
    p.potential_slicing = 2
    p.thick_type = 1
    p.nx = p.ny = 256
    p.bwl = 0
    p.E_0 = 200.0
    p.iw_type = 1
    p.output_area_ix_0, p.output_area_ix_e = 81, 177
    p.output_area_iy_0, p.output_area_iy_e = 81, 177
    return p


def stem_tilt_au001():
    """HAADF (70-200 mrad) STEM through fcc Au(001), 6 x 6 x 5 cells, 512^2 grid, 300 kV, 25 mrad
    probe, beam tilted 1.5 deg at azimuth 30 deg, 2 x 2 probes, two phonon configurations."""
    from multem_b200 import specimens
    return specimens.haadf_fcc001(79, 4.078, 5, nx=512, ns=2, scan_cells=1, nconf=2, seed=7, theta=1.5, phi=30.0)


def ew_tilt_si001():
    """Exit wave (EWRS) of Si(001) on a 256^2 grid with the beam tilted 0.8 deg at azimuth 20 deg
    (propagator offset g0, transmission strength / cos(theta) and the output phase ramp)."""
    from multem_b200 import specimens
    p = specimens.hrtem_si001(nx=256, ny=256, na=4, nb=4, nc=4)
    p.theta, p.phi = 0.8, 20.0
    return p


def ewfs_tilt_si001():
    """ew_tilt_si001 with the exit wave in Fourier space (EWFS)."""
    p = ew_tilt_si001()
    p.simulation_type = 51
    return p


def stem_incoh_srtio3():
    """STEM ADF through SrTiO3(001) on a 256^2 grid with the condenser's defocus spread integrated
    (illumination_model 4, full integration): 5 defocus points of a Gaussian (sigma 32 A, height
    0.8) plus exponential (beta 10 A) spread around c_10 = 20 A, 3 x 3 probes, two phonon
    configurations."""
    from multem_b200 import specimens
    p = specimens.stem_srtio3(nx=256, ny=256, na=4, nb=4, nc=4, ns=3, nconf=2, seed=6)
    p.illumination_model = 4
    p.temporal_spatial_incoh = 2
    p.cond_lens_c_10 = 20.0
    p.cond_lens_ti_npts = 5
    p.cond_lens_ti_sigma = 32.0
    p.cond_lens_ti_a = 0.8
    p.cond_lens_ti_beta = 10.0
    return p


def stem_matrix_srtio3():
    """STEM through SrTiO3(001) on a 256^2 grid with two matrix detectors given on the centred
    Fourier grid (ny x nx, as detector.matrix(d).fR): a soft-edged annulus 30-90 mrad and one
    quadrant (gx > 0, gy > 0) below 60 mrad, which pins the orientation and the fft-shift; 3 x 3
    probes, one phonon configuration."""
    from multem_b200 import specimens
    p = specimens.stem_srtio3(nx=256, ny=256, na=4, nb=4, nc=4, ns=3, nconf=1, seed=8)
    lam = 0.019687  # A at 300 kV
    gx = (np.arange(p.nx) - p.nx // 2) / p.spec_lx
    gy = (np.arange(p.ny) - p.ny // 2) / p.spec_ly
    GY, GX = np.meshgrid(gy, gx, indexing="ij")  # (ny, nx)
    th = lam * np.hypot(GX, GY) * 1e3  # mrad
    ring = 1 / (1 + np.exp(-(th - 30) / 2)) * 1 / (1 + np.exp((th - 90) / 2))
    quad = ((GX > 0) & (GY > 0) & (th < 60)).astype(float)
    p.detector = {"type": 3, "matrix": [{"fR": ring}, {"fR": quad}]}
    return p


def stem_coh_srtio3():
    """STEM ADF through SrTiO3(001) on a 256^2 grid with the coherent contribution
    (pn_coh_contrib = 1: image_coh from the configuration-averaged transformed wave), 3 x 3 probes,
    three phonon configurations."""
    from multem_b200 import specimens
    p = specimens.stem_srtio3(nx=256, ny=256, na=4, nb=4, nc=4, ns=3, nconf=3, seed=10)
    p.pn_coh_contrib = 1
    return p


def ed_si001():
    """Electron diffraction (simulation_type 31) of Si(001) on a 256^2 grid: |psi_hat|^2 of the exit
    wave averaged over two phonon configurations, with a cropped output window."""
    from multem_b200 import specimens
    p = specimens.hrtem_si001(nx=256, ny=256, na=4, nb=4, nc=4)
    p.simulation_type = 31
    p.pn_nconf = 2
    p.pn_seed = 3
    p.output_area_ix_0, p.output_area_ix_e = 65, 192
    p.output_area_iy_0, p.output_area_iy_e = 65, 192
    return p


def _hrtem(illumination):
    from multem_b200 import specimens
    p = specimens.hrtem_si001(nx=256, ny=256, na=4, nb=4, nc=4)
    p.simulation_type = 32
    p.pn_nconf = 2
    p.pn_seed = 4
    p.illumination_model = illumination
    p.obj_lens_c_10 = 60.0
    p.obj_lens_c_30 = 0.002
    p.obj_lens_c_12 = 20.0
    p.obj_lens_phi_12 = 30.0
    p.obj_lens_outer_aper_ang = 22.0
    return p


def hrtem_coherent_si001():
    """HRTEM image of Si(001) (simulation_type 32), coherent transfer function: defocus 60 A,
    C3 0.002 mm, 2-fold astigmatism 20 A at 30 deg, 22 mrad aperture; two phonon configurations."""
    return _hrtem(1)


def hrtem_pctf_si001():
    """hrtem_coherent_si001 with the partially coherent transfer function (temporal and spatial
    envelopes: ti_sigma 32 A, si_sigma 0.0072 1/A)."""
    p = _hrtem(2)
    p.temporal_spatial_incoh = 1
    p.obj_lens_ti_sigma = 32.0
    p.cond_lens_si_sigma = 0.0072
    return p


def hrtem_fullint_si001():
    """hrtem_coherent_si001 integrated numerically over the objective's defocus spread (illumination
    4, temporal only): 7 Gauss-Hermite points, ti_sigma 32 A."""
    p = _hrtem(4)
    p.temporal_spatial_incoh = 2
    p.obj_lens_ti_sigma = 32.0
    p.obj_lens_ti_npts = 7
    p.cond_lens_si_sigma = 0.0
    return p


def _conv_si001(sim_type, beams):
    from multem_b200 import specimens
    p = specimens.hrtem_si001(nx=256, ny=256, na=4, nb=4, nc=4)
    p.simulation_type = sim_type
    p.pn_nconf = 2
    p.pn_seed = 5
    p.iw_type = 2
    p.iw_x = [b[0] for b in beams]
    p.iw_y = [b[1] for b in beams]
    p.cond_lens_c_10 = 30.0
    p.cond_lens_c_30 = 0.001
    p.cond_lens_outer_aper_ang = 15.0
    return p


def cbed_si001():
    """CBED (simulation_type 21) of Si(001) on a 256^2 grid: a 15 mrad probe (defocus 30 A) off the
    cell centre, |psi_hat|^2 averaged over two phonon configurations."""
    return _conv_si001(21, [(11.2, 10.5)])


def cbei_si001():
    """CBEI (simulation_type 22): the cbed_si001 wave imaged through the objective's coherent
    transfer function (defocus 40 A, 30 mrad aperture)."""
    p = _conv_si001(22, [(11.2, 10.5)])
    p.obj_lens_c_10 = 40.0
    p.obj_lens_outer_aper_ang = 30.0
    return p


def ewrs_two_beams_si001():
    """Exit wave (EWRS) of Si(001) under a convergent incident wave of two beams (the probes are
    summed, Incident_Wave::operator())."""
    return _conv_si001(52, [(8.0, 9.0), (13.5, 12.0)])


def ewrs_user_wave_si001():
    """Exit wave (EWRS) of Si(001) on a 256^2 grid under a user-defined incident wave (iw_type 3): a
    seeded smooth complex wave, placed off the cell centre by iw_x/iw_y; two phonon configurations."""
    from multem_b200 import specimens
    p = specimens.hrtem_si001(nx=256, ny=256, na=4, nb=4, nc=4)
    p.pn_nconf = 2
    p.pn_seed = 6
    p.iw_type = 3
    rng = np.random.default_rng(31)
    y, x = np.meshgrid(np.arange(p.ny) * p.spec_ly / p.ny, np.arange(p.nx) * p.spec_lx / p.nx, indexing="ij")
    env = np.exp(-((x - 0.5 * p.spec_lx) ** 2 + (y - 0.5 * p.spec_ly) ** 2) / (2 * 5.0 ** 2))
    p.iw_psi = env * np.exp(1j * 0.4 * rng.standard_normal((p.ny, p.nx)))
    p.iw_x, p.iw_y = [0.5 * p.spec_lx + 1.7], [0.5 * p.spec_ly - 2.3]
    return p


def hrtem_user_wave_si001():
    """ewrs_user_wave_si001 imaged through the objective's coherent transfer function (HRTEM)."""
    p = ewrs_user_wave_si001()
    p.simulation_type = 32
    p.illumination_model = 1
    p.obj_lens_c_10 = 40.0
    p.obj_lens_outer_aper_ang = 25.0
    return p


def ew_rot_si001():
    """Exit wave (EWRS) of Si(001), 256^2 grid, 4 x 4 x 4 cells rotated by 4 deg about (1, 0.5, 0)
    through the geometric centre (spec_rot_*), dz_Proj slices of 1.36 A (with plane slicing the
    rotated atoms fall into a single plane and the reference switches to its phase-object mode)."""
    from multem_b200 import specimens
    p = specimens.hrtem_si001(nx=256, ny=256, na=4, nb=4, nc=4)
    p.potential_slicing = 2
    p.spec_dz = 1.36
    p.spec_rot_theta = 4.0
    p.spec_rot_u0 = (1.0, 0.5, 0.0)
    p.spec_rot_center_type = 1
    return p


def stem_rot_srtio3():
    """STEM ADF through SrTiO3(001) rotated by 10 deg about z through a user point (7, 8, 5), 256^2
    grid, 3 x 3 probes, two phonon configurations."""
    from multem_b200 import specimens
    p = specimens.stem_srtio3(nx=256, ny=256, na=4, nb=4, nc=4, ns=3, nconf=2, seed=12)
    p.spec_rot_theta = 10.0
    p.spec_rot_u0 = (0.0, 0.0, 1.0)
    p.spec_rot_center_type = 2
    p.spec_rot_center_p = (7.0, 8.0, 5.0)
    return p


def ped_si001():
    """Precession electron diffraction (simulation_type 41) of Si(001), 256^2 grid: the beam tilted
    by 2 deg and turned through 8 azimuths, diffraction patterns averaged over rotations and two
    phonon configurations (the pattern is not shifted back: dp_Shift)."""
    from multem_b200 import specimens
    p = specimens.hrtem_si001(nx=256, ny=256, na=4, nb=4, nc=4)
    p.simulation_type = 41
    p.pn_nconf = 2
    p.pn_seed = 8
    p.ped_theta, p.ped_nrot = 2.0, 8
    return p


def hctem_si001():
    """Hollow-cone TEM (simulation_type 42) of Si(001), 256^2 grid: 1.5 deg cone, 6 azimuths, images
    through the objective's coherent transfer function (defocus 50 A, 25 mrad), two phonon
    configurations."""
    from multem_b200 import specimens
    p = specimens.hrtem_si001(nx=256, ny=256, na=4, nb=4, nc=4)
    p.simulation_type = 42
    p.pn_nconf = 2
    p.pn_seed = 9
    p.hci_theta, p.hci_nrot = 1.5, 6
    p.illumination_model = 1
    p.obj_lens_c_10 = 50.0
    p.obj_lens_outer_aper_ang = 25.0
    return p


def istem_srtio3():
    """ISTEM (simulation_type 12) of SrTiO3(001), 256^2 grid: 3 x 3 probes (21 mrad), each exit wave
    imaged through the objective's coherent transfer function (defocus 30 A, 25 mrad), the images
    of all probes and two phonon configurations summed."""
    from multem_b200 import specimens
    p = specimens.stem_srtio3(nx=256, ny=256, na=4, nb=4, nc=4, ns=3, nconf=2, seed=13)
    p.simulation_type = 12
    p.illumination_model = 1
    p.obj_lens_c_10 = 30.0
    p.obj_lens_outer_aper_ang = 25.0
    return p


def _au_monolayer():
    from multem_b200 import specimens
    a = 4.078
    layer = (a, a, a, [(79, 0.0, 0.0, 0.0), (79, 0.5, 0.5, 0.0)])  # the z = 0 plane of fcc(001)
    return specimens.crystal(layer, 6, 6, 1, sigma=0.085), 6 * a


def ew_monolayer_au():
    """Exit wave (EWRS) of a single Au(001) atomic plane (6 x 6 cells) on a 256^2 grid: one plane
    under plane slicing, so the reference switches to its phase-object mode (transmission only);
    two phonon configurations."""
    from multem_b200 import specimens
    p = specimens.hrtem_si001(nx=256, ny=256, na=4, nb=4, nc=4)
    p.spec_atoms, L = _au_monolayer()
    p.spec_lx = p.spec_ly = L
    p.spec_lz = 4.0
    p.pn_nconf = 2
    p.pn_seed = 14
    return p


def stem_monolayer_au():
    """STEM ADF over the single Au(001) plane (phase-object mode), 256^2 grid, 3 x 3 probes."""
    from multem_b200 import specimens
    p = specimens.stem_srtio3(nx=256, ny=256, na=4, nb=4, nc=4, ns=3, nconf=2, seed=15)
    p.spec_atoms, L = _au_monolayer()
    p.spec_lx = p.spec_ly = L
    p.spec_lz = 4.0
    p.potential_slicing = 1
    p.scanning_x0 = p.scanning_y0 = 2 * 4.078
    p.scanning_xe = p.scanning_ye = 3 * 4.078
    return p


def ew_po_si001():
    """Exit wave (EWRS) of Si(001) 4 x 4 x 4 cells in the phase-object approximation
    (interaction_model 2): the whole specimen's projected potential, transmission only."""
    from multem_b200 import specimens
    p = specimens.hrtem_si001(nx=256, ny=256, na=4, nb=4, nc=4)
    p.interaction_model = 2
    return p


def ew_wpo_si001():
    """ew_po_si001 in the weak-phase-object approximation (interaction_model 3: T = 1 + i sigma V)."""
    p = ew_po_si001()
    p.interaction_model = 3
    return p


def ew_bwl_si001():
    """Exit wave (EWRS) of Si(001), 256^2 grid, with the band-width limit (bwl = 1: the transmission
    functions and every propagation cut off smoothly at 2/3 of g_max); two phonon configurations."""
    from multem_b200 import specimens
    p = specimens.hrtem_si001(nx=256, ny=256, na=4, nb=4, nc=4)
    p.bwl = 1
    p.pn_nconf = 2
    p.pn_seed = 16
    return p


def stem_bwl_srtio3():
    """STEM ADF through SrTiO3(001) with the band-width limit, 256^2 grid, 3 x 3 probes, two
    thicknesses, two phonon configurations."""
    from multem_b200 import specimens
    p = specimens.stem_srtio3(nx=256, ny=256, na=4, nb=4, nc=4, ns=3, nconf=2, seed=17)
    p.bwl = 1
    p.thick_type = 2
    p.thick = [8.0, 15.0]
    return p


def hrtem_bwl_si001():
    """HRTEM (coherent transfer function) of Si(001) with the band-width limit."""
    p = _hrtem(1)
    p.bwl = 1
    return p


def _ew_potential(pt, seed):
    from multem_b200 import specimens
    p = specimens.hrtem_si001(nx=256, ny=256, na=4, nb=4, nc=4)
    p.potential_type = pt
    p.pn_nconf = 2
    p.pn_seed = seed
    return p


def ew_doyle_si001():
    """Exit wave (EWRS) of Si(001), 256^2 grid, two phonon configurations, with the Doyle-Turner
    (0-4) parameterisation (potential_type 1)."""
    return _ew_potential(1, 21)


def ew_peng4_si001():
    """As ew_doyle_si001 with the Peng (0-4) parameterisation (potential_type 2)."""
    return _ew_potential(2, 22)


def ew_kirkland_si001():
    """As ew_doyle_si001 with the Kirkland (0-12) parameterisation (potential_type 4)."""
    return _ew_potential(4, 24)


def _stem_potential(pt, seed):
    from multem_b200 import specimens
    p = specimens.stem_srtio3(nx=256, ny=256, na=4, nb=4, nc=4, ns=3, nconf=2, seed=seed)
    p.potential_type = pt
    p.thick_type = 2
    p.thick = [8.0, 15.0]
    return p


def stem_peng12_srtio3():
    """STEM ADF through SrTiO3(001), 256^2 grid, 3 x 3 probes, two thicknesses, two phonon
    configurations, with the Peng (0-12) parameterisation (potential_type 3)."""
    return _stem_potential(3, 23)


def stem_kirkland_srtio3():
    """As stem_peng12_srtio3 with the Kirkland (0-12) parameterisation (potential_type 4)."""
    return _stem_potential(4, 25)


def stem_ions_srtio3():
    """STEM ADF through SrTiO3(001) with ionic charges (Sr 2+, Ti 4+, O 2-, Peng's ionic
    coefficients), 256^2 grid, 3 x 3 probes, two thicknesses, two phonon configurations."""
    import numpy as np
    p = _stem_potential(6, 27)
    a = np.array(p.spec_atoms, dtype=np.float64)
    q = {38: 2, 22: 4, 8: -2}
    a[:, 7] = [q[int(z)] for z in a[:, 0]]
    p.spec_atoms = a
    return p


def ew_ions_si001():
    """Exit wave (EWRS) of Si(001) with every second atom a Si 4+ ion and a charge that has no ionic
    table (Si 2+, which the reference treats as neutral) on the others, 256^2 grid."""
    import numpy as np
    p = _ew_potential(6, 28)
    a = np.array(p.spec_atoms, dtype=np.float64)
    a[0::2, 7] = 4
    a[1::2, 7] = 2
    p.spec_atoms = a
    return p


def _full_integration(p):
    """Condenser defocus spread (3 points, sigma 20 A) and source spread (2 radial x 3 azimuthal
    points, sigma 0.15 A) under full integration (illumination_model 4, temporal_spatial_incoh 1)."""
    p.illumination_model = 4
    p.temporal_spatial_incoh = 1
    p.cond_lens_ti_sigma = 20.0
    p.cond_lens_ti_npts = 3
    p.cond_lens_si_sigma = 0.15
    p.cond_lens_si_rad_npts = 2
    p.cond_lens_si_azm_npts = 3
    return p


def cbed_full_si001():
    """cbed_si001 with the condenser's defocus and source spreads integrated (18 incident waves per
    phonon configuration, Multislice::CBED_CBEI's full-integration branch)."""
    return _full_integration(cbed_si001())


def cbei_full_si001():
    """cbei_si001 with the condenser's and the objective's defocus spreads integrated
    (temporal_spatial_incoh 2: with the source spread too, the reference's objective-lens spatial
    quadrature is empty and its images are zero, an input the engine refuses)."""
    p = _full_integration(cbei_si001())
    p.temporal_spatial_incoh = 2
    return p


def _coherent(p):
    p.pn_coh_contrib = 1
    p.pn_nconf = 4
    return p


def ed_coh_si001():
    """ed_si001 over four phonon configurations with the coherent contribution (pn_coh_contrib 1):
    m2psi_coh, |configuration-averaged psi_hat|^2, beside m2psi_tot."""
    return _coherent(ed_si001())


def cbed_coh_si001():
    """cbed_si001 over four phonon configurations with the coherent contribution."""
    return _coherent(cbed_si001())


def ped_coh_si001():
    """ped_si001 over four phonon configurations with the coherent contribution."""
    return _coherent(ped_si001())


def hrtem_coh_si001():
    """hrtem_coherent_si001 over four phonon configurations with the coherent contribution: m2psi_coh,
    the objective's image of the configuration-averaged exit wave."""
    return _coherent(hrtem_coherent_si001())


def cbei_coh_si001():
    """cbei_si001 over four phonon configurations with the coherent contribution."""
    return _coherent(cbei_si001())


def stem_bench512():
    """The benchmark workload (SrTiO3(001) 8 x 8 x 25 cells, 8000 atoms, 512^2 grid, 50 dz_Proj
    slices of 1.95 A, 300 kV, 21 mrad probe, ADF 40-80 and 80-200 mrad, seed 1) with a 16 x 16
    raster over the same unit cell: 256 probes, one full probe batch of the engine at 512^2, and
    two frozen-phonon configurations."""
    from multem_b200 import specimens
    p = specimens.stem_srtio3(nconf=2, seed=1)
    p.scanning_ns = 16
    return p


def _au110_ac_2048(sim_type):
    """Amorphous carbon (2 nm, 2.0 g/cm^3, minimum spacing 1.4 A) on Au(110) 12 x 17 x 60 cells
    (29,292 atoms), 2048^2 grid, 200 kV, 2 A slices, two frozen-phonon configurations, written to a
    256 x 256 window at the centre of the grid."""
    from multem_b200 import specimens
    p = specimens.au110_amorphous_carbon(nx=2048, ny=2048, nconf=2)
    p.simulation_type = sim_type
    p.output_area_ix_0, p.output_area_ix_e = 896, 1152
    p.output_area_iy_0, p.output_area_iy_e = 896, 1152
    return p


def ew_au110_ac_2048():
    """Exit wave (EWRS) of the large-field precision case on the 2048^2 grid (see _au110_ac_2048)."""
    return _au110_ac_2048(52)


def ed_au110_ac_2048():
    """Electron diffraction pattern (ED) of the large-field precision case on the 2048^2 grid (see
    _au110_ac_2048); the window is the centre of the shifted pattern."""
    return _au110_ac_2048(31)
