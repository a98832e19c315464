"""ctypes access to oracle/_ref/libmultem_ref.so — the reference's own CPU path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's reference /
cpu_baseline leg as the checker, never by the product. The library is the reference's
Multislice<T, e_host> compiled from its sources (oracle/Makefile) with this directory's FFTW-API
shim; see ref/ref_driver.cu for the entry points.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from multem_b200 import capi

REF_LIB = Path(__file__).resolve().parent / "_ref" / "libmultem_ref.so"
_lib = None


def available() -> bool:
    return REF_LIB.exists()


def lib():
    global _lib
    if _lib is None:
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} not built (make -C oracle)")
        L = C.CDLL(str(REF_LIB))
        P = C.POINTER
        L.mtref_last_error.restype = C.c_char_p
        L.mtref_run.argtypes = [P(capi.MtInputMultislice), C.c_int, C.c_int, P(capi.MtOutputMultislice)]
        L.mtref_output_dims.argtypes = [P(capi.MtInputMultislice), C.c_int, P(capi.MtOutputDims)]
        L.mtref_run_device.argtypes = [P(capi.MtInputMultislice), P(capi.MtOutputMultislice)]
        L.mtref_params.argtypes = [P(capi.MtInputMultislice), C.c_int, capi.P_double, C.c_int]
        L.mtref_specimen.argtypes = [P(capi.MtInputMultislice), C.c_int, C.c_int, C.c_int, capi.P_int, capi.P_int,
                                     capi.P_double, C.c_int, capi.P_int, capi.P_double, capi.P_double, capi.P_int,
                                     capi.P_int, capi.P_int, capi.P_double]
        L.mtref_projected_potential.argtypes = [P(capi.MtInputMultislice), C.c_int, C.c_int, C.c_int, C.c_int,
                                                capi.P_double]
        L.mtref_transmission_function.argtypes = [P(capi.MtInputMultislice), C.c_int, C.c_int, C.c_int, C.c_int,
                                                  capi.P_double]
        L.mtref_atom_type.argtypes = [P(capi.MtInputMultislice), C.c_int, C.c_int, capi.P_double, capi.P_double,
                                      C.c_int]
        L.mtref_atom_type_q.argtypes = [P(capi.MtInputMultislice), C.c_int, C.c_int, C.c_int, capi.P_double,
                                        capi.P_double, C.c_int]
        L.mtref_incident_wave.argtypes = [P(capi.MtInputMultislice), C.c_int, C.c_int, capi.P_double]
        L.mtref_propagate.argtypes = [P(capi.MtInputMultislice), C.c_int, C.c_int, C.c_double, capi.P_double]
        _lib = L
    return _lib


def _chk(rc):
    if rc != 0:
        raise RuntimeError("reference oracle failed: " + lib().mtref_last_error().decode())


def _dp(a):
    return a.ctypes.data_as(capi.P_double)


def _ip(a):
    return a.ctypes.data_as(capi.P_int)


def output_dims(params, precision=1):
    s, keep = params.to_c()
    d = capi.MtOutputDims()
    _chk(lib().mtref_output_dims(C.byref(s), precision, C.byref(d)))
    return d


def run(params, precision=1, nthreads=1, device=False):
    """Full simulation through the reference; returns a dict shaped like the MATLAB output struct
    (set_struct_multislice, mex_files_multem/ilc_multem.cu:382-481), arrays as numpy. device=True
    runs the reference's own GPU path (float, cuFFT) instead of its CPU path."""
    d = output_dims(params, precision)
    s, keep = params.to_c()
    nxy = d.nx * d.ny
    x = np.zeros(d.n_x)
    y = np.zeros(d.n_y)
    thick = np.zeros(d.n_thick)
    o = capi.MtOutputMultislice()
    o.x, o.y, o.thick = _dp(x), _dp(y), _dp(thick)
    res = {"x": x, "y": y, "thick": thick}
    if d.has_image_tot:
        res["image_tot"] = np.zeros((d.n_thick, d.n_detector, d.nx, d.ny))
        o.image_tot = _dp(res["image_tot"])
    if d.has_image_coh:
        res["image_coh"] = np.zeros((d.n_thick, d.n_detector, d.nx, d.ny))
        o.image_coh = _dp(res["image_coh"])
    if d.has_m2psi_tot:
        res["m2psi_tot"] = np.zeros((d.n_thick, d.nx, d.ny))
        o.m2psi_tot = _dp(res["m2psi_tot"])
    if d.has_psi_coh:
        res["psi_coh_raw"] = np.zeros((d.n_thick, d.nx, d.ny, 2))
        o.psi_coh = _dp(res["psi_coh_raw"])
    if d.has_m2psi_coh:
        res["m2psi_coh"] = np.zeros((d.n_thick, d.nx, d.ny))
        o.m2psi_coh = _dp(res["m2psi_coh"])
    if device:
        _chk(lib().mtref_run_device(C.byref(s), C.byref(o)))
    else:
        _chk(lib().mtref_run(C.byref(s), precision, nthreads, C.byref(o)))
    res["dx"], res["dy"] = o.dx, o.dy
    # arrays are column-major (ix*ny + iy): stored here as [.., ix, iy]; expose MATLAB (iy, ix) order
    if "image_tot" in res:
        res["image_tot"] = np.swapaxes(res["image_tot"], -1, -2)
    if "image_coh" in res:
        res["image_coh"] = np.swapaxes(res["image_coh"], -1, -2)
    if "m2psi_tot" in res:
        res["m2psi_tot"] = np.swapaxes(res["m2psi_tot"], -1, -2)
    if "m2psi_coh" in res:
        res["m2psi_coh"] = np.swapaxes(res["m2psi_coh"], -1, -2)
    if "psi_coh_raw" in res:
        r = res.pop("psi_coh_raw")
        res["psi_coh"] = np.swapaxes(r[..., 0] + 1j * r[..., 1], -1, -2)
    return res


def params(p, precision=1):
    s, keep = p.to_c()
    v = np.zeros(8)
    _chk(lib().mtref_params(C.byref(s), precision, _dp(v), 8))
    return {"lambda": v[0], "Vr_factor": v[1], "cond_zero_defocus_plane": v[2], "n_slice": int(v[3]),
            "n_atoms": int(v[4]), "dz": v[5], "n_thick": int(v[6]), "interaction_model": int(v[7])}


def specimen(p, iconf, precision=1):
    """Displaced z-sorted atoms and slicing of configuration iconf (reference Spec::move_atoms)."""
    s, keep = p.to_c()
    n_max = max(1, int(np.asarray(p.spec_atoms).shape[0]))
    ns_max = 100000
    n_atoms = np.zeros(1, np.int32)
    Z = np.zeros(n_max, np.int32)
    xyz = np.zeros(3 * n_max)
    n_slice = np.zeros(1, np.int32)
    z0 = np.zeros(ns_max)
    ze = np.zeros(ns_max)
    ia0 = np.zeros(ns_max, np.int32)
    iae = np.zeros(ns_max, np.int32)
    ithk = np.zeros(ns_max, np.int32)
    zbp = np.zeros(4096)
    _chk(lib().mtref_specimen(C.byref(s), precision, iconf, n_max, _ip(n_atoms), _ip(Z), _dp(xyz), ns_max,
                              _ip(n_slice), _dp(z0), _dp(ze), _ip(ia0), _ip(iae), _ip(ithk), _dp(zbp)))
    na, ns = int(n_atoms[0]), int(n_slice[0])
    return {"Z": Z[:na], "xyz": xyz[:3 * na].reshape(na, 3), "z_0": z0[:ns], "z_e": ze[:ns],
            "iatom_0": ia0[:ns], "iatom_e": iae[:ns], "ithk": ithk[:ns], "z_back_prop": zbp}


def projected_potential(p, iconf, islice, precision=1, nthreads=1):
    s, keep = p.to_c()
    V = np.zeros(p.nx * p.ny)
    _chk(lib().mtref_projected_potential(C.byref(s), precision, nthreads, iconf, islice, _dp(V)))
    return V.reshape(p.nx, p.ny).T


def transmission_function(p, iconf, islice, precision=1, nthreads=1):
    s, keep = p.to_c()
    t = np.zeros(2 * p.nx * p.ny)
    _chk(lib().mtref_transmission_function(C.byref(s), precision, nthreads, iconf, islice, _dp(t)))
    t = t[0::2] + 1j * t[1::2]
    return t.reshape(p.nx, p.ny).T


def atom_type(p, Z, precision=1, nR=128, charge=0):
    s, keep = p.to_c()
    head = np.zeros(4)
    tab = np.zeros(5 * nR)
    _chk(lib().mtref_atom_type_q(C.byref(s), precision, Z, charge, _dp(head), _dp(tab), nR))
    t = tab.reshape(5, nR)
    return {"R_min": head[0], "R_max": head[1], "R_tap": head[2], "tap_cf": head[3], "R2": t[0], "c0": t[1],
            "c1": t[2], "c2": t[3], "c3": t[4]}


def incident_wave(p, space=1, precision=1):
    s, keep = p.to_c()
    t = np.zeros(2 * p.nx * p.ny)
    _chk(lib().mtref_incident_wave(C.byref(s), precision, space, _dp(t)))
    t = t[0::2] + 1j * t[1::2]
    return t.reshape(p.nx, p.ny).T


def propagate(p, z, space=1, precision=1):
    """The reference's Propagator on the user wave p.iw_psi (ilc_propagate semantics, distance z)."""
    s, keep = p.to_c()
    t = np.zeros(2 * p.nx * p.ny)
    _chk(lib().mtref_propagate(C.byref(s), precision, space, float(z), _dp(t)))
    t = t[0::2] + 1j * t[1::2]
    return t.reshape(p.nx, p.ny).T
