"""Bounded waits and cancellation of a run in progress.

The bulk-copy-fed line passes wait on mbarriers for the copies that feed them. Every such wait is
bounded: once it runs out, the pass sets the engine's error flag, stops issuing copies, waits
(bounded) for those in flight and returns; later passes return on entry, and the run reports
MT_ERR_TIMEOUT with the engine still usable. The timeout is made to happen without any fault: with
a wait limit of 0 a copy that has not landed at the first check counts as timed out, which happens
on the first item of a pass (its copy was issued microseconds earlier). mt_engine_cancel from a
second host thread stops a run between launches with MT_ERR_CANCELLED, the role of the reference's
ext_stop_sim (src/tem_simulation.cuh:47,512).
"""
import threading
import time

import numpy as np
import pytest

from multem_b200 import api, capi, specimens

pytestmark = pytest.mark.gpu


def _images(r):
    return np.stack([np.stack(d["image_tot"]) for d in r["data"]])


@pytest.mark.parametrize("nx", [512, 1024])
def test_wait_timeout_returns_error_quickly_and_engine_stays_usable(nx, monkeypatch):
    monkeypatch.setenv("MTB_PIPE", "3")  # the bulk-copy-fed passes, whose waits are bounded
    p = specimens.stem_srtio3(nx=nx, ny=nx, na=4, nb=4, nc=6, ns=8, nconf=2, seed=3)
    e = api.Engine(p)
    ref = _images(e.run())
    e.set_wait_limit(0.0)
    t0 = time.perf_counter()
    with pytest.raises(capi.MtError) as exc:
        e.run()
    dt = time.perf_counter() - t0
    assert exc.value.status == 5, exc.value  # MT_ERR_TIMEOUT
    assert dt < 1.0, f"a timed-out run took {dt:.3f} s"
    # the engine and the context are still usable, and a normal limit gives the same images
    e.set_wait_limit(2.0)
    again = _images(e.run())
    e.close()
    np.testing.assert_array_equal(again, ref)


def test_cancel_from_another_thread():
    p = specimens.stem_srtio3(nconf=6, seed=2)  # 512^2, 4096 probes, 6 configurations: seconds of work
    e = api.Engine(p)
    status = {}

    def run():
        try:
            e.run()
            status["rc"] = 0
        except capi.MtError as err:
            status["rc"] = err.status

    th = threading.Thread(target=run)
    t0 = time.perf_counter()
    th.start()
    time.sleep(0.5)
    while th.is_alive():  # repeated in case the first request came before the run reset its flag
        e.cancel()
        th.join(timeout=0.05)
    dt = time.perf_counter() - t0
    assert status.get("rc") == 4, status  # MT_ERR_CANCELLED
    # the engine runs again after a cancellation
    p1 = specimens.stem_srtio3(nx=128, ny=128, na=4, nb=4, nc=2, ns=2, nconf=1, seed=3)
    e.close()
    e1 = api.Engine(p1)
    img = _images(e1.run())
    e1.close()
    assert np.all(np.isfinite(img)) and img.sum() > 0
    assert dt < 30.0
