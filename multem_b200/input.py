"""Python mirror of MULTEM's MATLAB input class (matlab_functions/+multem_input/parameters.m).

Attribute names, enum codes, units and defaults are the MATLAB class's, so a MULTEM script ports by
renaming `multem_input.parameters` to `multem_b200.Parameters`. `to_c()` packs the fields into the
C ABI struct of include/multem_b200.h exactly as read_input_multislice
(mex_files_multem/ilc_multem.cu:38-379) reads them from the MATLAB struct.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import capi

_LENS_KEYS = [name for name, _ in capi._LENS_FIELDS]


@dataclass
class SystemConf:
    """matlab_functions/+multem_input/system_conf.m: precision 1 float / 2 double, device 1 CPU / 2 GPU."""
    precision: int = 1
    device: int = 2
    cpu_nthread: int = 1
    gpu_device: int = 0

    def to_c(self) -> capi.MtSystemConf:
        return capi.MtSystemConf(int(self.precision), int(self.device), int(self.cpu_nthread), int(self.gpu_device))


def _lens_defaults(prefix: str) -> dict:
    # parameters.m defaults for cond_lens_* and obj_lens_*
    d = {k: 0.0 for k in _LENS_KEYS}
    d.update(m=0, c_10=14.0312, c_30=1e-3, ti_a=1.0, ti_sigma=32.0, ti_beta=0.0, ti_npts=10, si_a=1.0,
             si_sigma=0.0072, si_beta=0.0, si_rad_npts=4, si_azm_npts=4, zero_defocus_type=1,
             zero_defocus_plane=0.0, inner_aper_ang=0.0)
    d["outer_aper_ang"] = 21.0 if prefix == "cond_lens" else 24.0
    return {f"{prefix}_{k}": v for k, v in d.items()}


class Parameters:
    """Input of a multislice run; field names and defaults of multem_input.parameters."""

    def __init__(self, **kw):
        self.system_conf = SystemConf()
        self.interaction_model = 1
        self.potential_type = 6
        self.operation_mode = 1
        self.memory_size = 0
        self.reverse_multislice = 0
        self.pn_model = 1
        self.pn_coh_contrib = 0
        self.pn_single_conf = 0
        self.pn_nconf = 1
        self.pn_dim = 110
        self.pn_seed = 300183
        self.pn_rng = 0          # 0 the reference's host draws, 1 counter-based draws on the GPU
        self.spec_atoms = np.zeros((0, 8))
        self.spec_dz = 0.25
        self.spec_lx = 10.0
        self.spec_ly = 10.0
        self.spec_lz = 10.0
        self.spec_cryst_na = 1
        self.spec_cryst_nb = 1
        self.spec_cryst_nc = 1
        self.spec_cryst_a = 0.0
        self.spec_cryst_b = 0.0
        self.spec_cryst_c = 0.0
        self.spec_cryst_x0 = 0.0
        self.spec_cryst_y0 = 0.0
        self.spec_amorp = []            # list of dicts {z_0, z_e, dz}
        self.spec_rot_theta = 0.0
        self.spec_rot_u0 = (0.0, 0.0, 1.0)
        self.spec_rot_center_type = 1
        self.spec_rot_center_p = (0.0, 0.0, 0.0)
        self.thick_type = 1
        self.thick = [0.0]
        self.potential_slicing = 1
        self.nx = 256
        self.ny = 256
        self.bwl = 0
        self.simulation_type = 52
        self.iw_type = 4
        self.iw_psi = None
        self.iw_x = [0.0]
        self.iw_y = [0.0]
        self.E_0 = 300.0
        self.theta = 0.0
        self.phi = 0.0
        self.ped_theta, self.ped_nrot = 3.0, 360
        self.hci_theta, self.hci_nrot = 3.0, 360
        self.illumination_model = 3
        self.temporal_spatial_incoh = 1
        for k, v in _lens_defaults("cond_lens").items():
            setattr(self, k, v)
        for k, v in _lens_defaults("obj_lens").items():
            setattr(self, k, v)
        self.detector = {"type": 1, "cir": [{"inner_ang": 60.0, "outer_ang": 180.0}]}
        self.scanning_type = 2
        self.scanning_periodic = 0
        self.scanning_square_pxs = 1
        self.scanning_ns = 10
        self.scanning_x0 = 0.0
        self.scanning_y0 = 0.0
        self.scanning_xe = 4.078
        self.scanning_ye = 4.078
        self.output_area_ix_0 = 0
        self.output_area_iy_0 = 0
        self.output_area_ix_e = 0
        self.output_area_iy_e = 0
        for k, v in kw.items():
            if not hasattr(self, k):
                raise AttributeError(f"unknown MULTEM input field {k!r}")
            setattr(self, k, v)

    def copy(self) -> "Parameters":
        import copy
        return copy.deepcopy(self)

    def to_c(self):
        """Return (MtInputMultislice, keepalive) — keepalive owns the arrays the struct points to."""
        keep = []

        def darr(a):
            a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))
            keep.append(a)
            return a.ctypes.data_as(capi.P_double), a

        s = capi.MtInputMultislice()
        for k in ["simulation_type", "interaction_model", "potential_type", "operation_mode", "reverse_multislice",
                  "pn_model", "pn_coh_contrib", "pn_single_conf", "pn_nconf", "pn_dim", "pn_seed", "pn_rng",
                  "spec_cryst_na", "spec_cryst_nb", "spec_cryst_nc", "spec_rot_center_type", "thick_type",
                  "potential_slicing", "nx", "ny", "bwl", "iw_type", "illumination_model",
                  "temporal_spatial_incoh", "scanning_type", "scanning_periodic", "scanning_square_pxs",
                  "scanning_ns", "output_area_ix_0", "output_area_iy_0", "output_area_ix_e", "output_area_iy_e",
                  "ped_nrot", "hci_nrot"]:
            setattr(s, k, int(getattr(self, k)))
        for k in ["spec_lx", "spec_ly", "spec_lz", "spec_dz", "spec_cryst_a", "spec_cryst_b", "spec_cryst_c",
                  "spec_cryst_x0", "spec_cryst_y0", "spec_rot_theta", "E_0", "theta", "phi", "scanning_x0",
                  "scanning_y0", "scanning_xe", "scanning_ye", "ped_theta", "hci_theta"]:
            setattr(s, k, float(getattr(self, k)))
        atoms = np.atleast_2d(np.asarray(self.spec_atoms, dtype=np.float64))
        if atoms.size == 0:
            atoms = np.zeros((0, 8))
        s.spec_atoms, _ = darr(atoms)          # column-major, MATLAB layout
        s.spec_atoms_rows, s.spec_atoms_cols = atoms.shape
        amorp = [a for a in self.spec_amorp if a is not None]
        s.spec_amorp_n = len(amorp)
        s.spec_amorp_z_0, _ = darr([a["z_0"] for a in amorp] or [0.0])
        s.spec_amorp_z_e, _ = darr([a["z_e"] for a in amorp] or [0.0])
        s.spec_amorp_dz, _ = darr([a.get("dz", 2.0) for a in amorp] or [0.0])
        s.spec_rot_u0 = (C.c_double * 3)(*[float(v) for v in self.spec_rot_u0])
        s.spec_rot_center_p = (C.c_double * 3)(*[float(v) for v in self.spec_rot_center_p])
        th = np.atleast_1d(np.asarray(self.thick, dtype=np.float64))
        s.thick, _ = darr(th)
        s.n_thick = th.size
        if self.iw_psi is not None:
            psi = np.asarray(self.iw_psi, dtype=np.complex128)
            inter = np.empty(psi.size * 2)
            flat = psi.ravel(order="F")
            inter[0::2], inter[1::2] = flat.real, flat.imag
            s.iw_psi, _ = darr(inter)
        else:
            s.iw_psi = capi.P_double()
        ix = np.atleast_1d(np.asarray(self.iw_x, dtype=np.float64))
        iy = np.atleast_1d(np.asarray(self.iw_y, dtype=np.float64))
        n = min(ix.size, iy.size)
        s.iw_x, _ = darr(ix[:n])
        s.iw_y, _ = darr(iy[:n])
        s.n_iw_xy = n
        for prefix, lens in (("cond_lens", s.cond_lens), ("obj_lens", s.obj_lens)):
            for k, t in capi._LENS_FIELDS:
                v = getattr(self, f"{prefix}_{k}")
                setattr(lens, k, int(v) if t is capi.c_int else float(v))
        det = self.detector or {"type": 1, "cir": []}
        s.detector_type = int(det.get("type", 1))
        cir = det.get("cir", []) if s.detector_type == 1 else []
        mats = det.get("matrix", []) if s.detector_type == 3 else []
        s.n_detector = len(mats) if s.detector_type == 3 else len(cir)
        s.detector_inner_ang, _ = darr([c["inner_ang"] for c in cir] or [0.0])
        s.detector_outer_ang, _ = darr([c["outer_ang"] for c in cir] or [0.0])
        # matrix detectors: fR is (ny, nx) as in MATLAB; stored x-major ([ix][iy])
        fr = [np.asarray(m["fR"], dtype=np.float64).T.ravel() for m in mats]
        s.detector_fR, _ = darr(np.concatenate(fr) if fr else [0.0])
        return s, keep

    def to_struct(self) -> dict:
        """The MATLAB struct of these parameters as multem_input.parameters.toStruct builds it
        (matlab_functions/+multem_input/parameters.m:283-303): flat fields, system_conf as a nested
        struct, spec_amorp and detector.cir / detector.matrix as 1 x n struct arrays. Values are
        numpy arrays in MATLAB's shapes (column vectors and matrices as MATLAB sees them), so
        scipy.io.savemat writes a file that mt_mat_input_open (and MATLAB) reads."""
        def sarr(rows, names):
            a = np.empty((1, len(rows)), dtype=[(n, object) for n in names])
            for i, r in enumerate(rows):
                a[0, i] = tuple(np.atleast_2d(np.asarray(r[n], dtype=np.float64)) for n in names)
            return a

        d = {}
        for k, v in vars(self).items():
            if k in ("system_conf", "spec_amorp", "detector", "iw_psi"):
                continue
            d[k] = np.atleast_2d(np.asarray(v, dtype=np.float64))
        d["spec_atoms"] = np.atleast_2d(np.asarray(self.spec_atoms, dtype=np.float64))
        d["thick"] = np.atleast_2d(np.asarray(self.thick, dtype=np.float64))
        c = self.system_conf
        d["system_conf"] = {"precision": float(c.precision), "device": float(c.device),
                            "cpu_nthread": float(c.cpu_nthread), "gpu_device": float(c.gpu_device)}
        amorp = [a for a in self.spec_amorp if a is not None]
        d["spec_amorp"] = sarr([{"z_0": a["z_0"], "z_e": a["z_e"], "dz": a.get("dz", 2.0)} for a in amorp],
                               ["z_0", "z_e", "dz"])
        if self.iw_psi is not None:
            d["iw_psi"] = np.asarray(self.iw_psi, dtype=np.complex128)
        det = self.detector or {"type": 1, "cir": []}
        d["detector"] = {"type": float(det.get("type", 1)),
                         "cir": sarr(det.get("cir", []), ["inner_ang", "outer_ang"]),
                         "matrix": sarr([{"fR": m["fR"]} for m in det.get("matrix", [])], ["fR"])}
        return d

