"""A simulation stored in a MAT-file, run on the GPU through mt_multislice_run_mat (and the
`python -m multem_b200` command), gives the same output struct as ilc_multem on the same
parameters: every array bit-identical (same engine, same input values)."""
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from multem_b200 import api, specimens

pytestmark = pytest.mark.gpu
sio = pytest.importorskip("scipy.io")


def _stem():
    p = specimens.stem_srtio3(nx=128, ny=128, na=2, nb=2, nc=2, ns=4, nconf=2, seed=3)
    p.detector = {"type": 1, "cir": [{"inner_ang": 40.0, "outer_ang": 80.0}, {"inner_ang": 80.0, "outer_ang": 200.0}]}
    return p


def _ew():
    p = specimens.hrtem_si001(nx=128, ny=128, na=2, nb=2, nc=4)
    p.simulation_type = 52
    return p


@pytest.mark.parametrize("make", [_stem, _ew])
def test_mat_file_run_matches_ilc_multem(tmp_path, make):
    p = make()
    src, dst = tmp_path / "in.mat", tmp_path / "out.mat"
    sio.savemat(src, {"input_multem": p.to_struct()}, do_compression=True, format="5")
    api.ilc_multem_mat(src, dst)
    ref = api.ilc_multem(p.system_conf, p)
    o = sio.loadmat(dst, squeeze_me=False, struct_as_record=True)["output_multislice"][0, 0]
    np.testing.assert_array_equal(o["x"][0], ref["x"])
    np.testing.assert_array_equal(o["thick"][0], ref["thick"])
    data = o["data"]
    for it, e in enumerate(ref["data"]):
        if "image_tot" in e:
            for k, im in enumerate(e["image_tot"]):
                np.testing.assert_array_equal(data[0, it]["image_tot"][0, k]["image"], im)
        else:
            np.testing.assert_array_equal(data[0, it]["m2psi_tot"], e["m2psi_tot"])
            np.testing.assert_array_equal(data[0, it]["psi_coh"], e["psi_coh"])


def test_command_line_entry(tmp_path):
    p = _stem()
    src, dst = tmp_path / "in.mat", tmp_path / "out.mat"
    sio.savemat(src, {"prms": p.to_struct()}, format="5")
    subprocess.run([sys.executable, "-m", "multem_b200", str(src), str(dst), "--var", "prms", "--compress"],
                   check=True, cwd=str(Path(__file__).resolve().parents[1]))
    o = sio.loadmat(dst)["output_multislice"][0, 0]
    ref = api.ilc_multem(p.system_conf, p)
    np.testing.assert_array_equal(o["data"][0, 0]["image_tot"][0, 1]["image"], ref["data"][0]["image_tot"][1])
