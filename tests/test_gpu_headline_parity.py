"""Parity on the benchmark's own workload and on the 2048^2 precision case, against the reference.

* stem_bench512: the 512^2 SrTiO3(001) STEM workload exactly as bench.py builds it (8 x 8 x 25
  cells, 8000 atoms, 50 slices, 300 kV, 21 mrad, ADF 40-80 and 80-200 mrad, seed 1), on a 16 x 16
  raster over the same unit cell: 256 probes, i.e. one full probe batch of the engine at 512^2,
  and two frozen-phonon configurations. It runs both through the C ABI entry (mt_multislice_run)
  and through the engine handle the benchmark times (prepare_confs / run_prepared / read_stem).
* ew_au110_ac_2048 / ed_au110_ac_2048: the large-field case (2 nm amorphous carbon on Au(110)
  12 x 17 x 60 cells, 29,292 atoms, 2048^2 grid, 200 kV, 2 A slices, two configurations), exit wave
  and diffraction pattern in a 256 x 256 window at the centre; the 2048-point line plan runs.

The references are the reference's own float and double CPU paths (tests/golden, made by
tests/golden/gen_golden.py). Bounds as in the other parity tests: relative L2 <= 1e-3 on detector
intensities and <= 1e-4 on exit waves against the reference float path (intensities of a wave
2e-4); the error against the reference double path is printed and held to the same bound plus
the reference's own float-to-double gap on the case (7e-5 on the 2048^2 exit wave).
"""
import numpy as np
import pytest

import cases
from conftest import rel_l2
from multem_b200 import api

pytestmark = pytest.mark.gpu

EXIT_WAVE_TOL = 1e-4
DETECTOR_TOL = 1e-3


def test_stem_bench_workload_full_batch(golden):
    p = cases.stem_bench512()
    out = api.ilc_multem(None, p)
    got = np.stack([np.stack(d["image_tot"]) for d in out["data"]])
    ref32 = golden["stem_bench512_run_p1_image_tot"]
    ref64 = golden["stem_bench512_run_p2_image_tot"]
    assert got.shape == ref32.shape == (1, 2, 16, 16)
    e32, e64 = rel_l2(got, ref32), rel_l2(got, ref64)
    per_det = [rel_l2(got[:, d], ref32[:, d]) for d in range(2)]
    print(f"stem_bench512: detector rel L2 vs reference float {e32:.3e} (per detector {per_det[0]:.3e}, "
          f"{per_det[1]:.3e}), vs reference double {e64:.3e}")
    assert e32 < DETECTOR_TOL and e64 < DETECTOR_TOL
    assert max(per_det) < DETECTOR_TOL
    # the benchmark's path: engine handle, configurations prepared then run, FP64 accumulators read
    e = api.Engine(p)
    e.prepare_confs(1, 2)
    e.run_prepared(1, 2)
    acc = e.read_stem()
    e.close()
    np.testing.assert_allclose(np.swapaxes(acc, -1, -2), got, rtol=1e-12, atol=0)


@pytest.mark.parametrize("name", ["ew_au110_ac_2048"])
def test_exit_wave_2048(golden, name):
    p = getattr(cases, name)()
    out = api.ilc_multem(None, p)
    psi = out["data"][0]["psi_coh"]
    m2 = out["data"][0]["m2psi_tot"]
    ref = golden[f"{name}_run_p1_psi_coh"][0]
    assert psi.shape == ref.shape == (256, 256)
    e32 = rel_l2(psi, ref)
    e64 = rel_l2(psi, golden[f"{name}_run_p2_psi_coh"][0])
    m32 = rel_l2(m2, golden[f"{name}_run_p1_m2psi_tot"][0])
    m64 = rel_l2(m2, golden[f"{name}_run_p2_m2psi_tot"][0])
    # the reference's own float path is this far from its double path on this case
    gap = rel_l2(golden[f"{name}_run_p1_psi_coh"][0], golden[f"{name}_run_p2_psi_coh"][0])
    print(f"{name}: exit wave rel L2 vs reference float {e32:.3e}, vs reference double {e64:.3e} "
          f"(reference float vs double {gap:.3e}); |psi|^2 vs float {m32:.3e}, vs double {m64:.3e}")
    assert e32 < EXIT_WAVE_TOL and e64 < EXIT_WAVE_TOL + 1.01 * gap
    assert m32 < 2 * EXIT_WAVE_TOL and m64 < 2 * EXIT_WAVE_TOL + 1.01 * gap
    np.testing.assert_allclose(out["x"], golden[f"{name}_run_p1_x"], rtol=1e-6)


def test_diffraction_pattern_2048(golden):
    name = "ed_au110_ac_2048"
    out = api.ilc_multem(None, getattr(cases, name)())
    m2 = out["data"][0]["m2psi_tot"]
    ref = golden[f"{name}_run_p1_m2psi_tot"][0]
    assert m2.shape == ref.shape == (256, 256)
    e32 = rel_l2(m2, ref)
    e64 = rel_l2(m2, golden[f"{name}_run_p2_m2psi_tot"][0])
    print(f"{name}: diffraction pattern rel L2 vs reference float {e32:.3e}, vs reference double {e64:.3e}")
    assert e32 < 2 * EXIT_WAVE_TOL and e64 < 2 * EXIT_WAVE_TOL
