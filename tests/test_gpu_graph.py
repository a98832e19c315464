"""run_confs replays each configuration as a CUDA graph (MTB_GRAPH, on by default), and run_prepared
runs a range of prepared configurations as one graph: the captured launches are the ones issued
directly, so results must be bit-identical to MTB_GRAPH=0, with the same launch count and progress.
Cases: STEM with several probe batches and phonon configurations (the two configuration slots
alternate, and the graphs replay), multiple output thicknesses, a tilted beam, exit waves, and the
512^2 benchmark grid with full 256-probe batches."""
import numpy as np
import pytest

from multem_b200 import api, specimens

pytestmark = pytest.mark.gpu


def _run(p, graph, monkeypatch, batch=8):
    monkeypatch.setenv("MTB_GRAPH", str(graph))
    monkeypatch.setenv("MTB_BATCH", str(batch))
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
    stem512 = specimens.stem_srtio3(nx=512, ny=512, na=8, nb=8, nc=4, ns=16, nconf=3, seed=6)
    return {"stem": stem, "stem_thicknesses": thick, "stem_tilt": tilt, "ew": ew, "stem_device_rng": stem_dev,
            "stem512": stem512}


@pytest.mark.parametrize("name", ["stem", "stem_thicknesses", "stem_tilt", "ew", "stem_device_rng", "stem512"])
def test_graph_replay_is_bit_identical(name, monkeypatch):
    p = _cases()[name]
    batch = 256 if name == "stem512" else 8
    direct, n0 = _run(p, 0, monkeypatch, batch)
    graph, n1 = _run(p, 1, monkeypatch, batch)
    assert n1 == n0 > 0
    for d0, d1 in zip(direct["data"], graph["data"]):
        for k in d0:
            np.testing.assert_array_equal(np.asarray(d1[k]), np.asarray(d0[k]), err_msg=k)


def test_prepared_range_runs_as_one_graph(monkeypatch):
    """run_prepared over a range of configurations as one graph (what the benchmark times) against
    direct launches: identical FP64 detector images, launch counts and progress."""
    p = specimens.stem_srtio3(nx=256, ny=256, na=4, nb=4, nc=6, ns=8, nconf=4, seed=8)
    out = {}
    for graph in ("0", "1"):
        monkeypatch.setenv("MTB_GRAPH", graph)
        monkeypatch.setenv("MTB_PIPE", "3")
        e = api.Engine(p)
        e.prepare_confs(1, 4)
        e.run_prepared(1, 1)
        e.reset()
        e.run_prepared(2, 4)
        first = e.read_stem()
        n = e.launch_count()
        e.reset()
        e.run_prepared(2, 4)  # replayed
        again = e.read_stem()
        e.close()
        np.testing.assert_array_equal(again, first)
        out[graph] = (first, n)
    np.testing.assert_array_equal(out["1"][0], out["0"][0])
    assert out["1"][1] == out["0"][1] > 0
