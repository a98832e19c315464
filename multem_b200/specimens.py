"""Seeded synthetic specimens and the standard workloads of this engine.

Crystals are periodic tilings of a unit cell described by layers of fractional positions, the same
layer description MULTEM's crystal scripts use (e.g. crystalline_materials/SrTiO3001_xtl.m,
Si001_xtl.m, Au110_xtl.m, fcc001_xtl.m). Unlike MULTEM's Crystal_Spec builder
(src/xtl_build.hpp:37-96) no closing layer at z = nc*c and no duplicate boundary atoms are added:
na x nb x nc cells give exactly na*nb*nc*(atoms per cell) atoms. Rows are
[Z, x, y, z, sigma, occ, region, charge], the spec_atoms layout of the MATLAB input.
"""
from __future__ import annotations

import numpy as np

from .input import Parameters

# Unit cells: (a, b, c, [(Z, fx, fy, fz), ...])
SI_001 = (5.4307, 5.4307, 5.4307, [
    (14, 0.00, 0.00, 0.00), (14, 0.50, 0.50, 0.00),
    (14, 0.25, 0.25, 0.25), (14, 0.75, 0.75, 0.25),
    (14, 0.00, 0.50, 0.50), (14, 0.50, 0.00, 0.50),
    (14, 0.25, 0.75, 0.75), (14, 0.75, 0.25, 0.75)])


def srtio3_001(a: float = 3.905):
    return (a, a, a, [(38, 0.0, 0.0, 0.0), (8, 0.5, 0.5, 0.0),
                      (8, 0.0, 0.5, 0.5), (8, 0.5, 0.0, 0.5), (22, 0.5, 0.5, 0.5)])


def fcc_001(Z: int, a: float):
    return (a, a, a, [(Z, 0.0, 0.0, 0.0), (Z, 0.5, 0.5, 0.0), (Z, 0.0, 0.5, 0.5), (Z, 0.5, 0.0, 0.5)])


def haadf_fcc001(Z: int, a: float, nc: int, nx: int = 512, ns: int = 32, scan_cells: int = 2, nconf: int = 64,
                 seed: int = 1, theta: float = 0.0, phi: float = 0.0, sigma: float = 0.085) -> "Parameters":
    """HAADF STEM through fcc(001) (6 x 6 x nc cells, lattice constant a, element Z): 300 kV,
    25 mrad probe, one annular detector 70-200 mrad, ns x ns periodic raster over scan_cells x
    scan_cells unit cells, `nconf` frozen-phonon configurations (isotropic sigma), dz_Proj slices of
    a/2, beam tilt theta (deg) at azimuth phi (deg). On 512^2 the sampling is 6a/512 <= 0.048 A, so
    lambda * g_max reaches the 200 mrad detector edge."""
    p = stem_srtio3(nx=nx, ny=nx, na=6, nb=6, nc=nc, ns=ns, nconf=nconf, seed=seed)
    p.spec_atoms = crystal(fcc_001(Z, a), 6, 6, nc, sigma=sigma)
    p.spec_lx = p.spec_ly = 6 * a
    p.spec_lz = nc * a
    p.spec_dz = a / 2
    p.cond_lens_outer_aper_ang = 25.0
    x0 = (3 - scan_cells // 2) * a
    p.scanning_x0, p.scanning_y0 = x0, x0
    p.scanning_xe, p.scanning_ye = x0 + scan_cells * a, x0 + scan_cells * a
    p.detector = {"type": 1, "cir": [{"inner_ang": 70.0, "outer_ang": 200.0}]}
    p.theta, p.phi = theta, phi
    return p


def fcc_110(Z: int, a: float):
    # (110) orientation: a' = a/sqrt(2), b' = a, c' = a/sqrt(2), two layers
    ap = a / np.sqrt(2.0)
    return (ap, a, ap, [(Z, 0.0, 0.0, 0.0), (Z, 0.5, 0.5, 0.5)])


def crystal(cell, na: int, nb: int, nc: int, sigma, occ: float = 1.0) -> np.ndarray:
    """Tile `cell` na x nb x nc times. `sigma` is a scalar or a dict {Z: sigma}."""
    a, b, c, basis = cell
    rows = []
    for k in range(nc):
        for j in range(nb):
            for i in range(na):
                for (Z, fx, fy, fz) in basis:
                    s = sigma[Z] if isinstance(sigma, dict) else sigma
                    rows.append((Z, (i + fx) * a, (j + fy) * b, (k + fz) * c, s, occ, 0, 0))
    return np.asarray(rows, dtype=np.float64)


def amorphous_layer(Z: int, lx: float, ly: float, z0: float, thickness: float, density_gcm3: float,
                    mass_amu: float, d_min: float, sigma: float, seed: int, region: int = 1) -> np.ndarray:
    """Random atoms with a minimum spacing (semantics of MULTEM's Amorp_Spec, src/amorp_spec.hpp):
    positions drawn uniformly in the box and rejected when closer than d_min to an accepted atom
    (periodic in x, y)."""
    rng = np.random.default_rng(seed)
    vol = lx * ly * thickness * 1e-24  # cm^3
    n_target = int(round(density_gcm3 * vol / (mass_amu * 1.66053906660e-24)))
    cell = d_min
    grid = {}
    out = []
    tries = 0
    while len(out) < n_target and tries < 200 * max(n_target, 1):
        tries += 1
        p = rng.random(3) * (lx, ly, thickness)
        key = tuple((p // cell).astype(int))
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    kk = ((key[0] + dx) % max(1, int(lx // cell)), (key[1] + dy) % max(1, int(ly // cell)),
                          key[2] + dz)
                    for q in grid.get(kk, ()):
                        d = np.abs(p - q)
                        d[0] = min(d[0], lx - d[0])
                        d[1] = min(d[1], ly - d[1])
                        if d @ d < d_min * d_min:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            kk = (key[0] % max(1, int(lx // cell)), key[1] % max(1, int(ly // cell)), key[2])
            grid.setdefault(kk, []).append(p)
            out.append((Z, p[0], p[1], z0 + p[2], sigma, 1.0, region, 0))
    return np.asarray(out, dtype=np.float64).reshape(-1, 8)


# ---------------------------------------------------------------------------------------------
# Standard workloads


def hrtem_si001(nx: int = 256, ny: int = 256, na: int = 4, nb: int = 4, nc: int = 8) -> Parameters:
    """Plane-wave exit wave (EWRS) through Si(001), 200 kV, slices of a/4 (planes), one frozen-phonon
    configuration with sigma = 0.075 A from seed 0 (clamped to 1 by validation)."""
    cell = SI_001
    atoms = crystal(cell, na, nb, nc, sigma=0.075)
    p = Parameters()
    p.simulation_type = 52
    p.pn_model = 3
    p.pn_coh_contrib = 0
    p.pn_single_conf = 0
    p.pn_nconf = 1
    p.pn_dim = 110
    p.pn_seed = 0
    p.spec_atoms = atoms
    p.spec_lx, p.spec_ly, p.spec_lz = na * cell[0], nb * cell[1], nc * cell[2]
    p.spec_dz = cell[2] / 4
    p.potential_slicing = 1
    p.nx, p.ny = nx, ny
    p.bwl = 0
    p.E_0 = 200.0
    p.iw_type = 1
    p.thick_type = 1
    return p


def stem_srtio3(nx: int = 512, ny: int = 512, na: int = 8, nb: int = 8, nc: int = 25, ns: int = 64,
                nconf: int = 16, seed: int = 1) -> Parameters:
    """Batched STEM ADF through SrTiO3(001): 300 kV, 21 mrad probe, C3 = 0, defocus 0, dz_Proj slices
    of 1.95 A, ns x ns raster over one unit cell, frozen phonons with per-element sigma, annular
    detectors 40-80 and 80-200 mrad."""
    a = 3.905
    cell = srtio3_001(a)
    atoms = crystal(cell, na, nb, nc, sigma={38: 0.088, 22: 0.075, 8: 0.095})
    p = Parameters()
    p.simulation_type = 11
    p.pn_model = 3
    p.pn_coh_contrib = 0
    p.pn_single_conf = 0
    p.pn_nconf = nconf
    p.pn_dim = 110
    p.pn_seed = seed
    p.spec_atoms = atoms
    p.spec_lx, p.spec_ly, p.spec_lz = na * a, nb * a, nc * a
    p.spec_dz = 1.95
    p.potential_slicing = 2
    p.thick_type = 1
    p.nx, p.ny = nx, ny
    p.bwl = 0
    p.E_0 = 300.0
    p.iw_type = 2
    p.cond_lens_m = 0
    p.cond_lens_c_10 = 0.0
    p.cond_lens_c_30 = 0.0
    p.cond_lens_c_50 = 0.0
    p.cond_lens_outer_aper_ang = 21.0
    p.cond_lens_inner_aper_ang = 0.0
    p.cond_lens_zero_defocus_type = 1
    p.illumination_model = 1
    p.temporal_spatial_incoh = 1
    p.scanning_type = 2
    p.scanning_periodic = 1
    p.scanning_square_pxs = 1
    p.scanning_ns = ns
    x0 = (na // 2) * a
    p.scanning_x0, p.scanning_y0 = x0, x0
    p.scanning_xe, p.scanning_ye = x0 + a, x0 + a
    p.detector = {"type": 1, "cir": [{"inner_ang": 40.0, "outer_ang": 80.0},
                                     {"inner_ang": 80.0, "outer_ang": 200.0}]}
    return p


FCC_Z = (13, 28, 29, 46, 47, 78, 79)


def fcc_batch(n: int = 32, seed: int = 3, grids=(256, 384, 512, 1024), ns: int = 8, nconf: int = 8):
    """Seeded batch of fcc(001) specimens of uneven size: lattice constant a ~ U[3.8, 4.1] A,
    Z from FCC_Z, thickness ~ U[5, 30] nm, grids cycling through `grids` (about 0.06 A per pixel,
    so the box grows with the grid), 200 or 300 kV, alternately plane-wave exit waves (EWRS) and
    STEM ADF (ns x ns raster over one cell, 21 mrad, detectors 40-80 and 80-200 mrad), `nconf`
    frozen-phonon configurations with sigma = 0.085 A, dz_Proj slices of a/2."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        a = float(rng.uniform(3.8, 4.1))
        Z = int(rng.choice(FCC_Z))
        t_nm = float(rng.uniform(5.0, 30.0))
        nx = int(grids[i % len(grids)])
        na = max(1, int(round(nx * 0.06 / a)))
        nc = max(1, int(round(t_nm * 10.0 / a)))
        E_0 = 200.0 if rng.uniform() < 0.5 else 300.0
        cell = fcc_001(Z, a)
        atoms = crystal(cell, na, na, nc, sigma=0.085)
        p = Parameters()
        p.pn_model = 3
        p.pn_coh_contrib = 0
        p.pn_single_conf = 0
        p.pn_nconf = nconf
        p.pn_dim = 110
        p.pn_seed = 100 + i
        p.spec_atoms = atoms
        p.spec_lx = p.spec_ly = na * a
        p.spec_lz = nc * a
        p.spec_dz = a / 2
        p.potential_slicing = 2
        p.thick_type = 1
        p.nx = p.ny = nx
        p.bwl = 0
        p.E_0 = E_0
        if i % 2 == 0:
            p.simulation_type = 52
            p.iw_type = 1
        else:
            p.simulation_type = 11
            p.iw_type = 2
            p.cond_lens_outer_aper_ang = 21.0
            p.cond_lens_zero_defocus_type = 1
            p.scanning_type = 2
            p.scanning_periodic = 1
            p.scanning_square_pxs = 1
            p.scanning_ns = ns
            x0 = (na // 2) * a
            p.scanning_x0, p.scanning_y0 = x0, x0
            p.scanning_xe, p.scanning_ye = x0 + a, x0 + a
            p.detector = {"type": 1, "cir": [{"inner_ang": 40.0, "outer_ang": 80.0},
                                             {"inner_ang": 80.0, "outer_ang": 200.0}]}
        out.append(p)
    return out


def au110_amorphous_carbon(nx: int = 2048, ny: int = 2048, na: int = 12, nb: int = 17, nc: int = 60,
                           t_ac: float = 20.0, dz: float = 2.0, nconf: int = 32, seed: int = 1) -> Parameters:
    """Plane-wave exit wave (EWRS) through Au(110) (a = 4.0782 A; na x nb x nc cells of
    a/sqrt(2) x a x a/sqrt(2), 34.6 x 69.3 x 173 A at the defaults) under a t_ac-thick amorphous
    carbon layer (2.0 g/cm^3, minimum spacing 1.4 A, region 1): 200 kV, dz_Proj slices of `dz` in
    the crystal and in the layer, `nconf` frozen-phonon configurations (sigma 0.085 A)."""
    a = 4.0782
    cell = fcc_110(79, a)
    lx, ly = na * cell[0], nb * cell[1]
    xtal = crystal(cell, na, nb, nc, sigma=0.085)
    xtal[:, 3] += t_ac + 0.5 * cell[2]
    ac = amorphous_layer(6, lx, ly, 0.0, t_ac, 2.0, 12.011, 1.4, 0.085, seed=seed + 1000, region=1)
    p = Parameters()
    p.simulation_type = 52
    p.pn_model = 3
    p.pn_coh_contrib = 0
    p.pn_single_conf = 0
    p.pn_nconf = nconf
    p.pn_dim = 110
    p.pn_seed = seed
    p.spec_atoms = np.vstack([ac, xtal])
    p.spec_lx, p.spec_ly = lx, ly
    p.spec_lz = t_ac + nc * cell[2] + cell[2]
    p.spec_dz = dz
    p.spec_amorp = [{"z_0": 0.0, "z_e": t_ac, "dz": dz}]
    p.potential_slicing = 2
    p.thick_type = 1
    p.nx, p.ny = nx, ny
    p.bwl = 0
    p.E_0 = 200.0
    p.iw_type = 1
    return p
