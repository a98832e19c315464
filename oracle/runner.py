"""Whole-run CPU oracle for small cases (TEST INFRASTRUCTURE ONLY).

Runs the numpy restatement in oracle/multislice.py over a full simulation: frozen-phonon
configurations, slices, thicknesses; STEM annular detectors or the plane-wave exit wave. The
specimen of each configuration (displaced atoms, slice ranges, thickness slices) is taken from the
engine's host logic (multem_b200.api.specimen_atoms / specimen_slices), which is checked
bit-for-bit against the reference separately (tests/test_host_model.py).
"""
from __future__ import annotations

import numpy as np

from multem_b200 import api
from oracle import multislice as O


def _slices(p, iconf, grid, tabs, w, dtype):
    Z, xyz = api.specimen_atoms(p, iconf)
    s = api.specimen_slices(p, iconf)
    occ = np.ones(len(Z))
    Ts, dzs = [], []
    for k in range(len(s["z_0"])):
        i0, ie = s["iatom_0"][k], s["iatom_e"][k]
        n = max(0, ie - i0 + 1)
        V = O.projected_potential(grid, xyz[i0:i0 + n, :2], Z[i0:i0 + n], occ[i0:i0 + n], tabs, dtype=dtype)
        Ts.append(O.transmission(V, float(w), dtype=dtype))
        dzs.append(np.float32(np.float32(s["z_e"][k]) - np.float32(s["z_0"][k])))
    return Z, xyz, s, Ts, dzs


def stem(p, dtype=np.float64, confs=None):
    """image_tot[ithk][idet] as (ny, nx) arrays (MATLAB orientation), summed over the phonon
    configurations `confs` (default: all), each weighted 1/pn_nconf like the reference."""
    grid = O.Grid(p.nx, p.ny, p.spec_lx, p.spec_ly)
    Zs = sorted({int(z) % 1000 for z in np.asarray(p.spec_atoms)[:, 0]})
    tabs = {Z: O.atom_table(Z, grid.dRx) for Z in Zs}
    lam, w = O.wavelength(p.E_0), O.vr_factor(p.E_0)
    dims = api.output_dims(p)
    nconf = p.pn_nconf if p.pn_model == 3 else 1
    wconf = 1.0 / nconf
    g_in = [np.float32(np.sin(np.float32(d["inner_ang"]) * 1e-3) / lam) for d in p.detector["cir"]]
    g_out = [np.float32(np.sin(np.float32(d["outer_ang"]) * 1e-3) / lam) for d in p.detector["cir"]]
    img = np.zeros((dims.n_thick, len(g_in), dims.nx * dims.ny))
    # scan positions in the reference's order (ix*ny + iy)
    out = api.output_dims(p)
    xs = np.float32(p.scanning_x0) + np.arange(out.nx, dtype=np.float32) * np.float32(
        (np.float32(p.scanning_xe) - np.float32(p.scanning_x0)) / np.float32(p.scanning_ns if p.scanning_periodic else p.scanning_ns - 1))
    ys = np.float32(p.scanning_y0) + np.arange(out.ny, dtype=np.float32) * np.float32(
        (np.float32(p.scanning_ye) - np.float32(p.scanning_y0)) / np.float32(p.scanning_ns if p.scanning_periodic else p.scanning_ns - 1))
    for iconf in (confs if confs is not None else range(1, nconf + 1)):
        Z, xyz, s, Ts, dzs = _slices(p, iconf, grid, tabs, w, dtype)
        thk_slices = {int(k): int(s["ithk"][k]) for k in range(len(s["ithk"])) if s["ithk"][k] >= 0}
        z_init = float(np.float32(0.5 * (np.float64(s["z_0"][0]) + np.float64(s["z_e"][0]))))
        zdp = float(np.float32(xyz[:, 2].min()))  # condenser zero-defocus plane: first atom (type 1)
        c10 = float(np.float32(np.float32(p.cond_lens_c_10) - np.float32(np.float32(zdp) - np.float32(z_init))))
        for ix in range(out.nx):
            for iy in range(out.ny):
                psi_hat = O.probe_fourier(grid, lam, p.cond_lens_outer_aper_ang, p.cond_lens_inner_aper_ang, c10,
                                          p.cond_lens_c_30 * 1e7, xs[ix], ys[iy])
                psi0 = np.fft.ifft2(psi_hat) * (p.nx * p.ny)
                res, _ = O.multislice(grid, psi0, Ts, dzs, lam, set(thk_slices), dtype=dtype)
                for k, ithk in thk_slices.items():
                    for d in range(len(g_in)):
                        img[ithk, d, ix * out.ny + iy] += wconf * O.detector_sum(grid, res[k], g_in[d], g_out[d])
    return [[img[t, d].reshape(out.nx, out.ny).T for d in range(len(g_in))] for t in range(dims.n_thick)]


def exit_wave(p, dtype=np.float64):
    """Plane-wave exit wave psi_coh[ithk] (ny, nx), back-propagated to the objective's zero-defocus
    plane (first atom, obj_lens_zero_defocus_type = 1) as the reference does for EWRS."""
    grid = O.Grid(p.nx, p.ny, p.spec_lx, p.spec_ly)
    Zs = sorted({int(z) % 1000 for z in np.asarray(p.spec_atoms)[:, 0]})
    tabs = {Z: O.atom_table(Z, grid.dRx) for Z in Zs}
    lam, w = O.wavelength(p.E_0), O.vr_factor(p.E_0)
    Z, xyz, s, Ts, dzs = _slices(p, 1, grid, tabs, w, dtype)
    thk = {int(k): int(s["ithk"][k]) for k in range(len(s["ithk"])) if s["ithk"][k] >= 0}
    outs = {}
    psi = np.ones((p.nx, p.ny), dtype=np.complex128)
    for k, (T, dz) in enumerate(zip(Ts, dzs)):
        psi = psi * T
        psi = np.fft.ifft2(np.fft.fft2(psi) * O.propagator(grid, lam, dz)) * (p.nx * p.ny)
        if k in thk:
            zbp = np.float32(np.float32(xyz[:, 2].min()) - 0.5 * (np.float64(s["z_0"][k]) + np.float64(s["z_e"][k])))
            ob = psi if abs(zbp) < 1e-4 else np.fft.ifft2(np.fft.fft2(psi) * O.propagator(grid, lam, zbp)) * (p.nx * p.ny)
            outs[thk[k]] = np.roll(np.roll(ob, -(p.nx // 2), 0), -(p.ny // 2), 1).T
        if k == max(thk):
            break
    return [outs[t] for t in sorted(outs)]
