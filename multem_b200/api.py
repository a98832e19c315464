"""MATLAB-style entry points over the C ABI (the `ilc_*` methods of multem_input.parameters,
matlab_functions/+multem_input/parameters.m:241-305).

    out = multem_b200.ilc_multem(system_conf, params)

returns a dict shaped like the MATLAB output struct of ilc_multem (set_struct_multislice,
mex_files_multem/ilc_multem.cu:382-481): dx, dy, x, y, thick and `data`, a list over thicknesses
of {"image_tot": [image per detector]} (STEM) or {"psi_coh", "m2psi_tot"} (exit wave). Images are
numpy arrays in MATLAB (ny, nx) orientation.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .input import Parameters, SystemConf


def _dp(a):
    return a.ctypes.data_as(capi.P_double)


def _conf(system_conf):
    return (system_conf or SystemConf()).to_c()


def output_dims(params: Parameters) -> capi.MtOutputDims:
    lib = capi.load()
    s, keep = params.to_c()
    d = capi.MtOutputDims()
    capi.check(lib.mt_output_query(C.byref(s), C.byref(d)))
    return d


class OutputBuffers:
    """Host buffers for mt_output_multislice sized from mt_output_dims."""

    def __init__(self, d: capi.MtOutputDims):
        self.d = d
        nxy = d.nx * d.ny
        self.x = np.zeros(max(1, d.n_x))
        self.y = np.zeros(max(1, d.n_y))
        self.thick = np.zeros(max(1, d.n_thick))
        self.image_tot = np.zeros(max(1, d.n_thick * d.n_detector * nxy)) if d.has_image_tot else None
        self.image_coh = np.zeros(max(1, d.n_thick * d.n_detector * nxy)) if d.has_image_coh else None
        self.m2psi_tot = np.zeros(max(1, d.n_thick * nxy)) if d.has_m2psi_tot else None
        self.psi_coh = np.zeros(max(1, 2 * d.n_thick * nxy)) if d.has_psi_coh else None
        self.m2psi_coh = np.zeros(max(1, d.n_thick * nxy)) if d.has_m2psi_coh else None
        o = capi.MtOutputMultislice()
        o.x, o.y, o.thick = _dp(self.x), _dp(self.y), _dp(self.thick)
        if self.image_tot is not None:
            o.image_tot = _dp(self.image_tot)
        if self.image_coh is not None:
            o.image_coh = _dp(self.image_coh)
        if self.m2psi_tot is not None:
            o.m2psi_tot = _dp(self.m2psi_tot)
        if self.psi_coh is not None:
            o.psi_coh = _dp(self.psi_coh)
        if self.m2psi_coh is not None:
            o.m2psi_coh = _dp(self.m2psi_coh)
        self.c = o

    def to_dict(self):
        d = self.d
        nx, ny = d.nx, d.ny
        res = {"dx": self.c.dx, "dy": self.c.dy, "x": self.x[:d.n_x].copy(), "y": self.y[:d.n_y].copy(),
               "thick": self.thick[:d.n_thick].copy(), "data": []}
        for it in range(d.n_thick):
            e = {}
            if self.image_tot is not None:
                imgs = self.image_tot.reshape(d.n_thick, d.n_detector, nx, ny)[it]
                e["image_tot"] = [imgs[k].T.copy() for k in range(d.n_detector)]
            if self.image_coh is not None:
                imgs = self.image_coh.reshape(d.n_thick, d.n_detector, nx, ny)[it]
                e["image_coh"] = [imgs[k].T.copy() for k in range(d.n_detector)]
            if self.m2psi_tot is not None:
                e["m2psi_tot"] = self.m2psi_tot.reshape(d.n_thick, nx, ny)[it].T.copy()
            if self.psi_coh is not None:
                r = self.psi_coh.reshape(d.n_thick, nx, ny, 2)[it]
                e["psi_coh"] = (r[..., 0] + 1j * r[..., 1]).T.copy()
            if self.m2psi_coh is not None:
                e["m2psi_coh"] = self.m2psi_coh.reshape(d.n_thick, nx, ny)[it].T.copy()
            res["data"].append(e)
        return res


def ilc_multem(system_conf: SystemConf | None, params: Parameters) -> dict:
    """Run a full simulation (mexFunction of mex_files_multem/ilc_multem.cu:520-546)."""
    lib = capi.load()
    d = output_dims(params)
    buf = OutputBuffers(d)
    s, keep = params.to_c()
    conf = _conf(system_conf)
    capi.check(lib.mt_multislice_run(C.byref(conf), C.byref(s), C.byref(buf.c)))
    return buf.to_dict()


def ilc_multem_mat(in_path, out_path, var: str | None = None, compress: bool = False) -> None:
    """File-level form of ilc_multem for MATLAB users (mt_multislice_run_mat): reads the input struct
    (variable `var`, else the first struct) from the MAT-file `in_path`, runs it on the GPU of its
    system_conf, and writes `output_multislice` to the MAT-file `out_path` (-v7 compressed when
    `compress`)."""
    lib = capi.load()
    capi.check(lib.mt_multislice_run_mat(str(in_path).encode(), var.encode() if var else None,
                                         str(out_path).encode(), int(compress)))


class MatInput:
    """An input struct read from a MAT-file (mt_mat_input_open): .conf and .c are the C ABI
    structs, valid while the object lives."""

    def __init__(self, path, var: str | None = None):
        self.lib = capi.load()
        self.h = C.c_void_p()
        self.conf = capi.MtSystemConf()
        self.c = capi.MtInputMultislice()
        capi.check(self.lib.mt_mat_input_open(str(path).encode(), var.encode() if var else None, C.byref(self.h),
                                              C.byref(self.conf), C.byref(self.c)))

    def close(self):
        if self.h:
            self.lib.mt_mat_input_close(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_output_mat(path, params: Parameters, out: dict, var: str | None = None, compress: bool = False) -> None:
    """Write an ilc_multem output dict of a run of `params` as MATLAB's output struct
    (mt_mat_output_write)."""
    lib = capi.load()
    d = output_dims(params)
    buf = OutputBuffers(d)
    buf.c.dx, buf.c.dy = float(out["dx"]), float(out["dy"])
    buf.x[:d.n_x], buf.y[:d.n_y], buf.thick[:d.n_thick] = out["x"], out["y"], out["thick"]
    nx, ny = d.nx, d.ny
    for it, e in enumerate(out["data"]):
        if buf.image_tot is not None:
            buf.image_tot.reshape(d.n_thick, d.n_detector, nx, ny)[it] = np.stack([im.T for im in e["image_tot"]])
        if buf.image_coh is not None:
            buf.image_coh.reshape(d.n_thick, d.n_detector, nx, ny)[it] = np.stack([im.T for im in e["image_coh"]])
        if buf.m2psi_tot is not None:
            buf.m2psi_tot.reshape(d.n_thick, nx, ny)[it] = e["m2psi_tot"].T
        if buf.psi_coh is not None:
            r = buf.psi_coh.reshape(d.n_thick, nx, ny, 2)[it]
            r[..., 0], r[..., 1] = e["psi_coh"].T.real, e["psi_coh"].T.imag
        if buf.m2psi_coh is not None:
            buf.m2psi_coh.reshape(d.n_thick, nx, ny)[it] = e["m2psi_coh"].T
    s, keep = params.to_c()
    capi.check(lib.mt_mat_output_write(str(path).encode(), var.encode() if var else None, C.byref(s),
                                       C.byref(buf.c), int(compress)))


def input_report(params: Parameters) -> list:
    """The changes the reference's validate_parameters would apply silently to `params`
    (mt_input_report), one string each; host only."""
    lib = capi.load()
    s, keep = params.to_c()
    buf = C.create_string_buffer(1 << 16)
    n = C.c_int()
    capi.check(lib.mt_input_report(C.byref(s), buf, len(buf), C.byref(n)))
    return [line for line in buf.value.decode().split("\n") if line][: n.value]


def ilc_multem_batch(system_conf: SystemConf | None, params_list) -> list:
    """Run several simulations in one call (mt_multislice_run_batch): largest first, overlapping
    on the GPU. Returns one output dict per input (as ilc_multem); raises on the first failure."""
    lib = capi.load()
    n = len(params_list)
    ins = (capi.MtInputMultislice * max(1, n))()
    outs = (capi.MtOutputMultislice * max(1, n))()
    keep, bufs = [], []
    for i, p in enumerate(params_list):
        s, k = p.to_c()
        keep.append((s, k))
        ins[i] = s
        b = OutputBuffers(output_dims(p))
        bufs.append(b)
        outs[i] = b.c
    status = (C.c_int * max(1, n))()
    conf = _conf(system_conf)
    capi.check(lib.mt_multislice_run_batch(C.byref(conf), n, ins, outs, status))
    res = []
    for i, b in enumerate(bufs):
        b.c = outs[i]
        res.append(b.to_dict())
    return res


class Engine:
    """Handle-based engine: set-up once, run configurations, read FP64 accumulators."""

    def __init__(self, params: Parameters, system_conf: SystemConf | None = None):
        self.lib = capi.load()
        self.params = params
        self._s, self._keep = params.to_c()
        conf = _conf(system_conf)
        h = C.c_void_p()
        capi.check(self.lib.mt_engine_create(C.byref(conf), C.byref(self._s), C.byref(h)))
        self.h = h
        self.dims = output_dims(params)

    def close(self):
        if self.h:
            self.lib.mt_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self) -> dict:
        buf = OutputBuffers(self.dims)
        capi.check(self.lib.mt_engine_run(self.h, C.byref(buf.c)))
        return buf.to_dict()

    def reset(self):
        capi.check(self.lib.mt_engine_reset(self.h))

    def run_confs(self, c0: int, c1: int):
        capi.check(self.lib.mt_engine_run_confs(self.h, c0, c1))

    def prepare_confs(self, c0: int, c1: int):
        capi.check(self.lib.mt_engine_prepare_confs(self.h, c0, c1))

    def run_prepared(self, c0: int, c1: int):
        capi.check(self.lib.mt_engine_run_prepared(self.h, c0, c1))

    def read_stem(self) -> np.ndarray:
        d = self.dims
        a = np.zeros(d.n_thick * d.n_detector * d.nx * d.ny)
        capi.check(self.lib.mt_engine_read_stem(self.h, _dp(a), a.size))
        return a.reshape(d.n_thick, d.n_detector, d.nx, d.ny)

    def launch_count(self) -> int:
        n = C.c_longlong()
        capi.check(self.lib.mt_engine_launch_count(self.h, C.byref(n)))
        return n.value

    def pass_variants(self) -> int:
        """Bit 0: bulk-copy-fed row pass, bit 1: column pass (autotuned or MTB_PIPE)."""
        v = C.c_int()
        capi.check(self.lib.mt_engine_pass_variants(self.h, C.byref(v)))
        return v.value

    def tuning(self) -> dict:
        """The autotuner's choice: row and column pass variant (0 per-thread loads, 1 bulk-copy fed,
        2 and 3 bulk-copy fed in the alternative pipeline shapes) and probes per launch."""
        r, c, b = C.c_int(), C.c_int(), C.c_int()
        capi.check(self.lib.mt_engine_tuning(self.h, C.byref(r), C.byref(c), C.byref(b)))
        return {"rows": r.value, "cols": c.value, "probes_per_launch": b.value}

    def cancel(self):
        capi.check(self.lib.mt_engine_cancel(self.h))

    def set_wait_limit(self, seconds: float):
        """Bound of every wait of a line pass for its bulk copies (0: no waiting beyond the first
        check); a wait that runs out makes the run raise MT_ERR_TIMEOUT."""
        capi.check(self.lib.mt_engine_set_wait_limit(self.h, float(seconds)))

    def set_timing(self, on: bool):
        capi.check(self.lib.mt_engine_set_timing(self.h, 1 if on else 0))

    def timing(self) -> dict:
        """Device time of the last run_prepared (CUDA events on the engine's stream)."""
        t, r, c = C.c_double(), C.c_double(), C.c_double()
        nr, nc = C.c_longlong(), C.c_longlong()
        capi.check(self.lib.mt_engine_timing(self.h, C.byref(t), C.byref(r), C.byref(nr), C.byref(c), C.byref(nc)))
        return {"total_ms": t.value, "rows_ms": r.value, "n_rows": nr.value, "cols_ms": c.value, "n_cols": nc.value}

    def progress(self):
        i, n = C.c_int(), C.c_int()
        capi.check(self.lib.mt_engine_progress(self.h, C.byref(i), C.byref(n)))
        return i.value, n.value


def ilc_projected_potential(system_conf, params: Parameters, iconf: int, islice: int) -> np.ndarray:
    lib = capi.load()
    s, keep = params.to_c()
    V = np.zeros(params.nx * params.ny)
    conf = _conf(system_conf)
    capi.check(lib.mt_projected_potential(C.byref(conf), C.byref(s), iconf, islice, _dp(V)))
    return V.reshape(params.nx, params.ny).T


def ilc_transmission_function(system_conf, params: Parameters, iconf: int, islice: int) -> np.ndarray:
    lib = capi.load()
    s, keep = params.to_c()
    t = np.zeros(2 * params.nx * params.ny)
    conf = _conf(system_conf)
    capi.check(lib.mt_transmission_function(C.byref(conf), C.byref(s), iconf, islice, _dp(t)))
    return (t[0::2] + 1j * t[1::2]).reshape(params.nx, params.ny).T


def ilc_incident_wave(system_conf, params: Parameters, space: int = 1) -> np.ndarray:
    lib = capi.load()
    s, keep = params.to_c()
    t = np.zeros(2 * params.nx * params.ny)
    conf = _conf(system_conf)
    capi.check(lib.mt_incident_wave(C.byref(conf), C.byref(s), space, _dp(t)))
    return (t[0::2] + 1j * t[1::2]).reshape(params.nx, params.ny).T


def propagate(system_conf, params: Parameters, z: float, space: int = 1) -> np.ndarray:
    """The user wave params.iw_psi ([ny, nx], iw_type 3) propagated by z (Angstrom); space 1 real,
    2 reciprocal (Propagator::operator(), src/propagator.cuh:51-103). Returns [ny, nx] complex."""
    lib = capi.load()
    s, keep = params.to_c()
    t = np.zeros(2 * params.nx * params.ny)
    conf = _conf(system_conf)
    capi.check(lib.mt_propagate(C.byref(conf), C.byref(s), int(space), float(z), _dp(t)))
    return (t[0::2] + 1j * t[1::2]).reshape(params.nx, params.ny).T


def ilc_propagate(system_conf, params: Parameters) -> dict:
    """ilc_propagate (mex_files_multem/ilc_propagate.cu:125-175): propagates iw_psi by obj_lens_c_10
    in real space; returns {dx, dy, psi}."""
    psi = propagate(system_conf, params, params.obj_lens_c_10, 1)
    return {"dx": params.spec_lx / params.nx, "dy": params.spec_ly / params.ny, "psi": psi}


def spline_tables(Z, dR_min: float, Vrl: float = 0.015, nR: int = 128, system_conf=None, potential_type: int = 6,
                  charge=None):
    """FP64 GPU build of the spline tables of `potential_type` (6 Lobato; 1-4 Doyle-Turner, Peng 0-4,
    Peng 0-12, Kirkland), optionally for ionic charges: returns (heads[n, 4], tab[n, 5, nR] float32)."""
    lib = capi.load()
    z = np.ascontiguousarray(np.asarray(Z, dtype=np.int32))
    q = None if charge is None else np.ascontiguousarray(np.asarray(charge, dtype=np.int32))
    heads = np.zeros((z.size, 4))
    tab = np.zeros((z.size, 5, nR), dtype=np.float32)
    conf = _conf(system_conf)
    capi.check(lib.mt_spline_tables_ex(C.byref(conf), int(potential_type), z.ctypes.data_as(capi.P_int),
                                       q.ctypes.data_as(capi.P_int) if q is not None else capi.P_int(), z.size,
                                       float(dR_min), float(Vrl), nR, _dp(heads),
                                       tab.ctypes.data_as(C.POINTER(C.c_float))))
    return heads, tab


def specimen_atoms(params: Parameters, iconf: int):
    """Displaced z-sorted atoms of configuration iconf (host logic, no GPU)."""
    lib = capi.load()
    s, keep = params.to_c()
    na, ns, nt = C.c_int(), C.c_int(), C.c_int()
    capi.check(lib.mt_specimen_info(C.byref(s), iconf, C.byref(na), C.byref(ns), C.byref(nt)))
    Z = np.zeros(na.value, np.int32)
    xyz = np.zeros(3 * na.value)
    capi.check(lib.mt_specimen_atoms(C.byref(s), iconf, Z.ctypes.data_as(capi.P_int), _dp(xyz), na.value))
    return Z, xyz.reshape(-1, 3)


def phonon_atoms(params: Parameters, iconf: int, system_conf=None):
    """Atoms of configuration iconf as the engine simulates them: the host draws of the reference
    (pn_rng 0, no GPU) or the device generator's (pn_rng 1)."""
    lib = capi.load()
    s, keep = params.to_c()
    na, ns, nt = C.c_int(), C.c_int(), C.c_int()
    capi.check(lib.mt_specimen_info(C.byref(s), iconf, C.byref(na), C.byref(ns), C.byref(nt)))
    Z = np.zeros(na.value, np.int32)
    xyz = np.zeros(3 * na.value)
    conf = _conf(system_conf)
    capi.check(lib.mt_phonon_atoms(C.byref(conf), C.byref(s), iconf, Z.ctypes.data_as(capi.P_int), _dp(xyz),
                                   na.value))
    return Z, xyz.reshape(-1, 3)


def philox4x32_10(ctr, key):
    """Philox4x32-10 on the device: ctr [n, 4] and key [n, 2] uint32 -> [n, 4] uint32."""
    lib = capi.load()
    c = np.ascontiguousarray(np.asarray(ctr, dtype=np.uint32).reshape(-1, 4))
    k = np.ascontiguousarray(np.asarray(key, dtype=np.uint32).reshape(-1, 2))
    out = np.zeros_like(c)
    P = C.POINTER(C.c_uint)
    capi.check(lib.mt_philox4x32_10(c.ctypes.data_as(P), k.ctypes.data_as(P), c.shape[0], out.ctypes.data_as(P)))
    return out


def specimen_slices(params: Parameters, iconf: int):
    lib = capi.load()
    s, keep = params.to_c()
    na, ns, nt = C.c_int(), C.c_int(), C.c_int()
    capi.check(lib.mt_specimen_info(C.byref(s), iconf, C.byref(na), C.byref(ns), C.byref(nt)))
    n = ns.value
    z0, ze = np.zeros(n), np.zeros(n)
    i0, ie, it = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, np.int32)
    capi.check(lib.mt_specimen_slices(C.byref(s), iconf, _dp(z0), _dp(ze), i0.ctypes.data_as(capi.P_int),
                                      ie.ctypes.data_as(capi.P_int), it.ctypes.data_as(capi.P_int), n))
    return {"z_0": z0, "z_e": ze, "iatom_0": i0, "iatom_e": ie, "ithk": it}
