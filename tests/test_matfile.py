"""MATLAB files (include/multem_b200.h, mt_mat_*): the input struct MATLAB's toStruct produces,
written by scipy.io.savemat (a second, independent implementation of the level-5 format; -v6
uncompressed and -v7 compressed), read through the C ABI into the same mt_input_multislice that
Parameters.to_c() builds; the output struct written through the C ABI read back by scipy.io.loadmat
in set_struct_multislice's layout (mex_files_multem/ilc_multem.cu:382-481). Host only; the GPU run
of a MAT-file is in test_gpu_matfile.py."""
import ctypes as C

import numpy as np
import pytest

from multem_b200 import api, capi, specimens

sio = pytest.importorskip("scipy.io")


def _cases():
    stem = specimens.stem_srtio3(nx=128, ny=128, na=2, nb=2, nc=2, ns=4, nconf=2, seed=3)
    stem.detector = {"type": 1, "cir": [{"inner_ang": 40.0, "outer_ang": 80.0}, {"inner_ang": 80.0, "outer_ang": 200.0}]}
    stem.thick_type, stem.thick = 2, [3.9, 7.8]
    stem.cond_lens_c_30, stem.cond_lens_phi_12, stem.cond_lens_c_12 = 0.002, 33.0, 5.0
    stem.spec_rot_u0, stem.spec_rot_center_p = (0.0, 0.2, 1.0), (1.0, 2.0, 3.0)
    mat = specimens.stem_srtio3(nx=64, ny=64, na=2, nb=2, nc=2, ns=2, nconf=1, seed=3)
    rng = np.random.default_rng(5)
    mat.detector = {"type": 3, "matrix": [{"fR": rng.random((64, 64))}, {"fR": rng.random((64, 64))}]}
    ew = specimens.hrtem_si001(nx=64, ny=64, na=2, nb=2, nc=2)
    ew.simulation_type, ew.iw_type = 52, 3
    ew.iw_psi = rng.standard_normal((64, 64)) + 1j * rng.standard_normal((64, 64))
    ew.iw_x, ew.iw_y = [1.0, 2.5], [3.0, 4.5]
    ew.spec_amorp = [{"z_0": 0.0, "z_e": 5.0, "dz": 2.0}, {"z_0": 20.0, "z_e": 25.0, "dz": 1.5}]
    ew.system_conf.gpu_device = 3
    return {"stem": stem, "matrix": mat, "ew": ew}


def _arr(p, n):
    return np.ctypeslib.as_array(p, shape=(n,)).copy() if n > 0 else np.zeros(0)


def _fields(s):
    """Every field of an mt_input_multislice, pointers dereferenced with their lengths."""
    out = {}
    for name, typ in capi.MtInputMultislice._fields_:
        v = getattr(s, name)
        if typ is capi.P_double:
            continue
        if name in ("cond_lens", "obj_lens"):
            for k, _ in capi._LENS_FIELDS:
                out[f"{name}.{k}"] = getattr(v, k)
        elif hasattr(v, "__len__"):
            out[name] = list(v)
        else:
            out[name] = v
    out["spec_atoms"] = _arr(s.spec_atoms, s.spec_atoms_rows * s.spec_atoms_cols)
    out["thick"] = _arr(s.thick, s.n_thick)
    out["iw_x"], out["iw_y"] = _arr(s.iw_x, s.n_iw_xy), _arr(s.iw_y, s.n_iw_xy)
    for k in ("spec_amorp_z_0", "spec_amorp_z_e", "spec_amorp_dz"):
        out[k] = _arr(getattr(s, k), s.spec_amorp_n)
    if s.detector_type == 1:
        out["inner"], out["outer"] = _arr(s.detector_inner_ang, s.n_detector), _arr(s.detector_outer_ang, s.n_detector)
    else:
        out["fR"] = _arr(s.detector_fR, s.n_detector * s.nx * s.ny)
    out["iw_psi"] = _arr(s.iw_psi, 2 * s.nx * s.ny) if s.iw_psi else None
    return out


@pytest.mark.parametrize("case", ["stem", "matrix", "ew"])
@pytest.mark.parametrize("compress", [False, True])
def test_input_struct_reads_as_parameters_to_c(tmp_path, case, compress):
    p = _cases()[case]
    path = tmp_path / "in.mat"
    sio.savemat(path, {"input_multem": p.to_struct()}, do_compression=compress, format="5")
    m = api.MatInput(path)
    got = _fields(m.c)
    ref_s, keep = p.to_c()
    ref = _fields(ref_s)
    assert got.keys() == ref.keys()
    for k in ref:
        if isinstance(ref[k], np.ndarray):
            np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
        else:
            assert got[k] == ref[k], k
    c = p.system_conf
    assert (m.conf.precision, m.conf.device, m.conf.cpu_nthread, m.conf.gpu_device) == \
        (c.precision, c.device, c.cpu_nthread, c.gpu_device)
    m.close()


def test_variable_selection_and_defaults(tmp_path):
    """A named variable is picked among several; fields the struct lacks take the class defaults;
    malformed files are rejected with a message."""
    path = tmp_path / "two.mat"
    sio.savemat(path, {"a_number": np.array([[1.0]]), "prms": {"nx": 128.0, "ny": 64.0, "E_0": 200.0},
                       "other": {"nx": 32.0}}, format="5")
    m = api.MatInput(path, "prms")
    assert (m.c.nx, m.c.ny, m.c.E_0, m.c.potential_type, m.c.pn_seed) == (128, 64, 200.0, 6, 300183)
    assert (m.c.obj_lens.outer_aper_ang, m.c.cond_lens.outer_aper_ang, m.c.cond_lens.c_10) == (24.0, 21.0, 14.0312)
    assert m.conf.device == 2 and m.c.n_detector == 1
    m2 = api.MatInput(path)  # first struct variable
    assert m2.c.nx == 128
    with pytest.raises(capi.MtError) as e:
        api.MatInput(path, "missing")
    assert e.value.status == 1 and b"missing" in capi.load().mt_last_error()
    bad = tmp_path / "bad.mat"
    bad.write_bytes(b"not a mat file" * 20)
    with pytest.raises(capi.MtError):
        api.MatInput(bad)


def _fake_output(p, rng):
    d = api.output_dims(p)
    out = {"dx": 0.25, "dy": 0.5, "x": rng.random(d.n_x), "y": rng.random(d.n_y), "thick": rng.random(d.n_thick),
           "data": []}
    for _ in range(d.n_thick):
        e = {}
        if d.has_image_tot:
            e["image_tot"] = [rng.random((d.ny, d.nx)) for _ in range(d.n_detector)]
        if d.has_image_coh:
            e["image_coh"] = [rng.random((d.ny, d.nx)) for _ in range(d.n_detector)]
        if d.has_m2psi_tot:
            e["m2psi_tot"] = rng.random((d.ny, d.nx))
        if d.has_psi_coh:
            e["psi_coh"] = rng.random((d.ny, d.nx)) + 1j * rng.random((d.ny, d.nx))
        if d.has_m2psi_coh:
            e["m2psi_coh"] = rng.random((d.ny, d.nx))
        out["data"].append(e)
    return d, out


@pytest.mark.parametrize("case", ["stem", "ew", "hrtem"])
@pytest.mark.parametrize("compress", [False, True])
def test_output_struct_layout(tmp_path, case, compress):
    p = _cases()[case] if case != "hrtem" else specimens.hrtem_si001(nx=64, ny=64, na=2, nb=2, nc=2)
    if case == "stem":
        p.pn_coh_contrib = 1
    if case == "hrtem":
        p.simulation_type, p.pn_model, p.pn_nconf, p.pn_coh_contrib = 32, 3, 2, 1
        p.illumination_model = 1
    rng = np.random.default_rng(7)
    d, out = _fake_output(p, rng)
    path = tmp_path / "out.mat"
    api.write_output_mat(path, p, out, compress=compress)
    z = sio.loadmat(path, squeeze_me=False, struct_as_record=True)
    o = z["output_multislice"][0, 0]
    assert float(o["dx"][0, 0]) == 0.25 and float(o["dy"][0, 0]) == 0.5
    np.testing.assert_array_equal(o["x"][0], out["x"])
    np.testing.assert_array_equal(o["y"][0], out["y"])
    np.testing.assert_array_equal(o["thick"][0], out["thick"])
    data = o["data"]
    assert data.shape == (1, d.n_thick)
    for it in range(d.n_thick):
        e = data[0, it]
        if case == "stem":
            assert set(data.dtype.names) == {"image_tot", "image_coh"}
            for name in ("image_tot", "image_coh"):
                dets = e[name]
                assert dets.shape == (1, d.n_detector)
                for k in range(d.n_detector):
                    np.testing.assert_array_equal(dets[0, k]["image"], out["data"][it][name][k])
        elif case == "ew":
            assert set(data.dtype.names) == {"m2psi_tot", "psi_coh"}
            np.testing.assert_array_equal(e["m2psi_tot"], out["data"][it]["m2psi_tot"])
            np.testing.assert_array_equal(e["psi_coh"], out["data"][it]["psi_coh"])
        else:
            assert set(data.dtype.names) == {"m2psi_tot", "m2psi_coh"}
            np.testing.assert_array_equal(e["m2psi_tot"], out["data"][it]["m2psi_tot"])
            np.testing.assert_array_equal(e["m2psi_coh"], out["data"][it]["m2psi_coh"])


@pytest.mark.parametrize("compress", [False, True])
def test_damaged_files_are_rejected_cleanly(tmp_path, compress):
    """Truncated or corrupted files end in MT_ERR_INVALID_ARG (or, where the damage leaves a
    readable struct, a normal read), never in a crash."""
    p = _cases()["ew"]
    good = tmp_path / "good.mat"
    sio.savemat(good, {"prms": p.to_struct()}, format="5", do_compression=compress)
    data = good.read_bytes()
    rng = np.random.default_rng(11)
    bad = tmp_path / "bad.mat"
    cuts = sorted(set(int(c) for c in rng.integers(129, len(data), 12))) + [130, 136, 200]
    for cut in cuts:
        bad.write_bytes(data[:cut])
        try:
            api.MatInput(bad).close()
        except capi.MtError as e:
            assert e.status == 1
    for _ in range(20):
        b = bytearray(data)
        for i in rng.integers(128, len(b), 4):
            b[i] = int(rng.integers(0, 256))
        bad.write_bytes(bytes(b))
        try:
            api.MatInput(bad).close()
        except capi.MtError as e:
            assert e.status == 1
