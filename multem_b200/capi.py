"""ctypes mirror of the C ABI in include/multem_b200.h.

The structures here are field-for-field copies of the C structs; the library loader refuses to run
without the compiled CUDA library (there is no CPU fallback of the engine).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libmultem_b200.so"

c_int = C.c_int
c_double = C.c_double
P_double = C.POINTER(C.c_double)
P_int = C.POINTER(C.c_int)


class MtSystemConf(C.Structure):
    _fields_ = [("precision", c_int), ("device", c_int), ("cpu_nthread", c_int), ("gpu_device", c_int)]


_LENS_FIELDS = [
    ("m", c_int),
    ("c_10", c_double), ("c_12", c_double), ("phi_12", c_double),
    ("c_21", c_double), ("phi_21", c_double), ("c_23", c_double), ("phi_23", c_double),
    ("c_30", c_double), ("c_32", c_double), ("phi_32", c_double), ("c_34", c_double), ("phi_34", c_double),
    ("c_41", c_double), ("phi_41", c_double), ("c_43", c_double), ("phi_43", c_double),
    ("c_45", c_double), ("phi_45", c_double),
    ("c_50", c_double), ("c_52", c_double), ("phi_52", c_double), ("c_54", c_double), ("phi_54", c_double),
    ("c_56", c_double), ("phi_56", c_double),
    ("inner_aper_ang", c_double), ("outer_aper_ang", c_double),
    ("ti_a", c_double), ("ti_sigma", c_double), ("ti_beta", c_double), ("ti_npts", c_int),
    ("si_a", c_double), ("si_sigma", c_double), ("si_beta", c_double),
    ("si_rad_npts", c_int), ("si_azm_npts", c_int),
    ("zero_defocus_type", c_int), ("zero_defocus_plane", c_double),
]


class MtLens(C.Structure):
    _fields_ = _LENS_FIELDS


class MtInputMultislice(C.Structure):
    _fields_ = [
        ("simulation_type", c_int), ("interaction_model", c_int), ("potential_type", c_int),
        ("operation_mode", c_int), ("reverse_multislice", c_int),
        ("pn_model", c_int), ("pn_coh_contrib", c_int), ("pn_single_conf", c_int), ("pn_nconf", c_int),
        ("pn_dim", c_int), ("pn_seed", c_int), ("pn_rng", c_int),
        ("spec_atoms", P_double), ("spec_atoms_rows", c_int), ("spec_atoms_cols", c_int),
        ("spec_lx", c_double), ("spec_ly", c_double), ("spec_lz", c_double), ("spec_dz", c_double),
        ("spec_cryst_na", c_int), ("spec_cryst_nb", c_int), ("spec_cryst_nc", c_int),
        ("spec_cryst_a", c_double), ("spec_cryst_b", c_double), ("spec_cryst_c", c_double),
        ("spec_cryst_x0", c_double), ("spec_cryst_y0", c_double),
        ("spec_amorp_n", c_int), ("spec_amorp_z_0", P_double), ("spec_amorp_z_e", P_double),
        ("spec_amorp_dz", P_double),
        ("spec_rot_theta", c_double), ("spec_rot_u0", c_double * 3), ("spec_rot_center_type", c_int),
        ("spec_rot_center_p", c_double * 3),
        ("thick_type", c_int), ("thick", P_double), ("n_thick", c_int),
        ("potential_slicing", c_int),
        ("nx", c_int), ("ny", c_int), ("bwl", c_int),
        ("iw_type", c_int), ("iw_psi", P_double), ("iw_x", P_double), ("iw_y", P_double), ("n_iw_xy", c_int),
        ("E_0", c_double), ("theta", c_double), ("phi", c_double),
        ("ped_theta", c_double), ("hci_theta", c_double), ("ped_nrot", c_int), ("hci_nrot", c_int),
        ("illumination_model", c_int), ("temporal_spatial_incoh", c_int),
        ("cond_lens", MtLens), ("obj_lens", MtLens),
        ("scanning_type", c_int), ("scanning_periodic", c_int), ("scanning_square_pxs", c_int),
        ("scanning_ns", c_int), ("scanning_x0", c_double), ("scanning_y0", c_double),
        ("scanning_xe", c_double), ("scanning_ye", c_double),
        ("detector_type", c_int), ("n_detector", c_int), ("detector_inner_ang", P_double),
        ("detector_outer_ang", P_double), ("detector_fR", P_double),
        ("output_area_ix_0", c_int), ("output_area_iy_0", c_int), ("output_area_ix_e", c_int),
        ("output_area_iy_e", c_int),
    ]


class MtOutputDims(C.Structure):
    _fields_ = [("n_thick", c_int), ("n_detector", c_int), ("nx", c_int), ("ny", c_int),
                ("has_image_tot", c_int), ("has_image_coh", c_int), ("has_m2psi_tot", c_int),
                ("has_psi_coh", c_int), ("n_x", c_int), ("n_y", c_int), ("has_m2psi_coh", c_int)]


class MtOutputMultislice(C.Structure):
    _fields_ = [("dx", c_double), ("dy", c_double), ("x", P_double), ("y", P_double), ("thick", P_double),
                ("image_tot", P_double), ("image_coh", P_double), ("m2psi_tot", P_double),
                ("psi_coh", P_double), ("m2psi_coh", P_double)]


MT_OK = 0
STATUS_NAMES = {0: "MT_OK", 1: "MT_ERR_INVALID_ARG", 2: "MT_ERR_OOM", 3: "MT_ERR_CUDA",
                4: "MT_ERR_CANCELLED", 5: "MT_ERR_TIMEOUT", 6: "MT_ERR_UNSUPPORTED", 7: "MT_ERR_INTERNAL"}

# Every entry point declared in include/multem_b200.h, with its ctypes signature.
_VP = C.c_void_p
SIGNATURES = {
    "mt_abi_version": (c_int, []),
    "mt_last_error": (C.c_char_p, []),
    "mt_device_alloc_count": (c_int, [C.POINTER(C.c_longlong)]),
    "mt_output_query": (c_int, [C.POINTER(MtInputMultislice), C.POINTER(MtOutputDims)]),
    "mt_multislice_run": (c_int, [C.POINTER(MtSystemConf), C.POINTER(MtInputMultislice),
                                  C.POINTER(MtOutputMultislice)]),
    "mt_input_report": (c_int, [C.POINTER(MtInputMultislice), C.c_char_p, C.c_size_t, P_int]),
    "mt_multislice_run_batch": (c_int, [C.POINTER(MtSystemConf), c_int, C.POINTER(MtInputMultislice),
                                        C.POINTER(MtOutputMultislice), P_int]),
    "mt_mat_input_open": (c_int, [C.c_char_p, C.c_char_p, C.POINTER(_VP), C.POINTER(MtSystemConf),
                                  C.POINTER(MtInputMultislice)]),
    "mt_mat_input_close": (c_int, [_VP]),
    "mt_mat_output_write": (c_int, [C.c_char_p, C.c_char_p, C.POINTER(MtInputMultislice),
                                    C.POINTER(MtOutputMultislice), c_int]),
    "mt_multislice_run_mat": (c_int, [C.c_char_p, C.c_char_p, C.c_char_p, c_int]),
    "mt_engine_create": (c_int, [C.POINTER(MtSystemConf), C.POINTER(MtInputMultislice), C.POINTER(_VP)]),
    "mt_engine_run": (c_int, [_VP, C.POINTER(MtOutputMultislice)]),
    "mt_engine_run_confs": (c_int, [_VP, c_int, c_int]),
    "mt_engine_reset": (c_int, [_VP]),
    "mt_engine_read_stem": (c_int, [_VP, P_double, C.c_size_t]),
    "mt_engine_cancel": (c_int, [_VP]),
    "mt_engine_set_wait_limit": (c_int, [_VP, c_double]),
    "mt_engine_progress": (c_int, [_VP, P_int, P_int]),
    "mt_engine_prepare_confs": (c_int, [_VP, c_int, c_int]),
    "mt_engine_run_prepared": (c_int, [_VP, c_int, c_int]),
    "mt_engine_launch_count": (c_int, [_VP, C.POINTER(C.c_longlong)]),
    "mt_engine_pass_variants": (c_int, [_VP, P_int]),
    "mt_engine_tuning": (c_int, [_VP, P_int, P_int, P_int]),
    "mt_engine_destroy": (c_int, [_VP]),
    "mt_engine_set_timing": (c_int, [_VP, c_int]),
    "mt_engine_timing": (c_int, [_VP, P_double, P_double, C.POINTER(C.c_longlong), P_double,
                                 C.POINTER(C.c_longlong)]),
    "mt_projected_potential": (c_int, [C.POINTER(MtSystemConf), C.POINTER(MtInputMultislice), c_int, c_int,
                                       P_double]),
    "mt_transmission_function": (c_int, [C.POINTER(MtSystemConf), C.POINTER(MtInputMultislice), c_int, c_int,
                                         P_double]),
    "mt_propagate": (c_int, [C.POINTER(MtSystemConf), C.POINTER(MtInputMultislice), c_int, c_double, P_double]),
    "mt_incident_wave": (c_int, [C.POINTER(MtSystemConf), C.POINTER(MtInputMultislice), c_int, P_double]),
    "mt_spline_tables": (c_int, [C.POINTER(MtSystemConf), P_int, c_int, c_double, c_double, c_int, P_double,
                                 C.POINTER(C.c_float)]),
    "mt_spline_tables_noalloc": (c_int, [P_int, c_int, c_double, c_double, c_int, P_double, C.c_void_p,
                                         C.c_void_p]),
    "mt_phonon_atoms": (c_int, [C.POINTER(MtSystemConf), C.POINTER(MtInputMultislice), c_int, P_int, P_double,
                                c_int]),
    "mt_philox4x32_10": (c_int, [C.POINTER(C.c_uint), C.POINTER(C.c_uint), c_int, C.POINTER(C.c_uint)]),
    "mt_spline_tables_ex": (c_int, [C.POINTER(MtSystemConf), c_int, P_int, P_int, c_int, c_double, c_double, c_int,
                                    P_double, C.POINTER(C.c_float)]),
    "mt_spline_tables_noalloc_ex": (c_int, [c_int, P_int, P_int, c_int, c_double, c_double, c_int, P_double,
                                            C.c_void_p, C.c_void_p]),
    # learned surrogate kernels (include/multem_b200_surrogate.h); tensors are device pointers
    "mt_sg_conv3x3_forward": (c_int, [_VP, _VP, _VP, _VP, _VP, c_int, c_int, c_int, c_int, c_int, c_int, _VP]),
    "mt_sg_conv3x3_backward_data": (c_int, [_VP, _VP, _VP, _VP, c_int, c_int, c_int, c_int, c_int, _VP]),
    "mt_sg_conv3x3_backward_weight": (c_int, [_VP, _VP, _VP, _VP, _VP, c_int, c_int, c_int, c_int, c_int, _VP]),
    "mt_sg_loss": (c_int, [_VP, _VP, _VP, _VP, _VP, _VP, c_int, c_int, c_int, C.c_float, _VP]),
    "mt_sg_adam": (c_int, [_VP, _VP, _VP, _VP, _VP, c_int, C.c_float, C.c_float, C.c_float, C.c_float, c_int, _VP]),
    "mt_sg_to_bf16": (c_int, [_VP, _VP, c_int, _VP]),
    "mt_sg_check": (c_int, [_VP]),
    "mt_sg_pool2": (c_int, [_VP, _VP, c_int, c_int, c_int, c_int, C.c_float, _VP]),
    "mt_sg_upsample2": (c_int, [_VP, _VP, c_int, c_int, c_int, c_int, C.c_float, _VP]),
    "mt_sg_add": (c_int, [_VP, _VP, _VP, C.c_longlong, _VP]),
    "mt_specimen_info": (c_int, [C.POINTER(MtInputMultislice), c_int, P_int, P_int, P_int]),
    "mt_specimen_atoms": (c_int, [C.POINTER(MtInputMultislice), c_int, P_int, P_double, c_int]),
    "mt_specimen_slices": (c_int, [C.POINTER(MtInputMultislice), c_int, P_double, P_double, P_int, P_int, P_int,
                                   c_int]),
}

_lib = None


class MtError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load the engine library; raise if it has not been built (no silent fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"multem_b200 CUDA library not found at {p}; build it with "
                          f"`python -c 'import __graft_entry__ as g; g.build()'` or `make -C multem_b200/csrc`")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(status: int) -> None:
    if status != MT_OK:
        msg = load().mt_last_error()
        raise MtError(status, msg.decode() if msg else "")
