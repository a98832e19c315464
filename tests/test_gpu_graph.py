"""run_confs replays each configuration as a CUDA graph (MTB_GRAPH, on by default): the captured
launches are the ones issued directly, so results must be bit-identical to MTB_GRAPH=0, with the
same launch count and progress. Cases: STEM with several probe batches and phonon configurations
(the two configuration slots alternate, and the graphs replay), multiple output thicknesses, a
tilted beam, and exit waves."""
import numpy as np
import pytest

from multem_b200 import api, specimens

pytestmark = pytest.mark.gpu


def _run(p, graph, monkeypatch):
    monkeypatch.setenv("MTB_GRAPH", str(graph))
    monkeypatch.setenv("MTB_BATCH", "8")
    monkeypatch.setenv("MTB_PIPE", "3")  # no autotuner launches (they happen once per process and shape)
    e = api.Engine(p)
    r = e.run()
    n = e.launch_count()
    e.close()
    return r, n


def _cases():
    stem = specimens.stem_srtio3(nx=128, ny=128, na=4, nb=4, nc=6, ns=5, nconf=5, seed=2)
    thick = specimens.stem_srtio3(nx=128, ny=128, na=4, nb=4, nc=6, ns=4, nconf=3, seed=4)
    thick.thick_type = 2
    thick.thick = [4.0, 12.0, 20.0]
    tilt = specimens.haadf_fcc001(79, 4.078, 4, nx=256, ns=3, scan_cells=1, nconf=3, seed=3, theta=1.0, phi=40.0)
    ew = specimens.hrtem_si001(nx=128, ny=128, na=4, nb=4, nc=4)
    ew.pn_nconf = 4
    ew.pn_seed = 7
    stem_dev = specimens.stem_srtio3(nx=128, ny=128, na=4, nb=4, nc=6, ns=5, nconf=5, seed=2)
    stem_dev.pn_rng = 1  # configurations drawn on the device, into the slot the graph reads
    return {"stem": stem, "stem_thicknesses": thick, "stem_tilt": tilt, "ew": ew, "stem_device_rng": stem_dev}


@pytest.mark.parametrize("name", ["stem", "stem_thicknesses", "stem_tilt", "ew", "stem_device_rng"])
def test_graph_replay_is_bit_identical(name, monkeypatch):
    p = _cases()[name]
    direct, n0 = _run(p, 0, monkeypatch)
    graph, n1 = _run(p, 1, monkeypatch)
    assert n1 == n0 > 0
    for d0, d1 in zip(direct["data"], graph["data"]):
        for k in d0:
            np.testing.assert_array_equal(np.asarray(d1[k]), np.asarray(d0[k]), err_msg=k)
