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
