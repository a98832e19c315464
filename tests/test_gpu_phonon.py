"""The device phonon generator (pn_rng 1) on the GPU: the generator against the published vectors
and its CPU restatement, the displaced atoms against the restatement, and simulations with it
against the reference's host draws (statistically: the same phonon average, different
configurations)."""
import numpy as np
import pytest

from conftest import rel_l2
from multem_b200 import api, specimens
from oracle import phonon as P

pytestmark = pytest.mark.gpu


def test_device_philox_matches_known_answers_and_restatement():
    ctr = np.array([c for c, _, _ in P.KAT], np.uint32)
    key = np.array([k for _, k, _ in P.KAT], np.uint32)
    out = api.philox4x32_10(ctr, key)
    np.testing.assert_array_equal(out, np.array([r for _, _, r in P.KAT], np.uint32))
    rng = np.random.default_rng(5)
    ctr = rng.integers(0, 2 ** 32, size=(4096, 4), dtype=np.uint32)
    key = rng.integers(0, 2 ** 32, size=(4096, 2), dtype=np.uint32)
    np.testing.assert_array_equal(api.philox4x32_10(ctr, key), P.philox4x32_10(ctr, key))


def test_device_displacements_match_restatement():
    p = specimens.stem_srtio3(nx=128, ny=128, na=4, nb=4, nc=4, ns=4, nconf=3, seed=7)
    sig = {int(r[0]): float(r[4]) for r in np.asarray(p.spec_atoms)}
    p.pn_rng = 1
    for iconf in (1, 3):
        Z, got = api.phonon_atoms(p, iconf)
        q = specimens.stem_srtio3(nx=128, ny=128, na=4, nb=4, nc=4, ns=4, nconf=3, seed=7)
        q.pn_model = 1  # still atoms, in the same (z-sorted) order
        Zs, still = api.specimen_atoms(q, 1)
        np.testing.assert_array_equal(Z, Zs)
        sigma = np.array([sig[z] for z in Z], np.float32)
        want = P.displaced(still, sigma, p.pn_seed, iconf)
        got32 = got.astype(np.float32)
        np.testing.assert_array_equal(got32[:, 2], want[:, 2])
        # Box-Muller in double on both sides: equal after rounding to float, up to one float ulp
        ulp = np.spacing(np.abs(want[:, :2]))
        assert np.all(np.abs(got32[:, :2] - want[:, :2]) <= ulp)
        assert np.mean(got32[:, :2] == want[:, :2]) > 0.999
        d = (got32 - still.astype(np.float32))[:, :2] / sigma[:, None]
        assert abs(d.std() - 1) < 0.1


def _stem(rng, seed, nconf=24, pn_model=3):
    p = specimens.stem_srtio3(nx=128, ny=128, na=4, nb=4, nc=8, ns=6, nconf=nconf, seed=seed)
    p.pn_rng = rng
    p.pn_model = pn_model
    out = api.ilc_multem(None, p)
    return np.stack([np.stack(d["image_tot"]) for d in out["data"]])


def test_device_draws_give_the_reference_phonon_average():
    """24 configurations drawn on the device against 24 host draws of the reference, three seeds
    each: device averages differ from host averages no more than host averages differ among
    themselves (mean over the pairs), and all lie far closer to one another than to the still-atom
    image. The runs are deterministic, so the test is too."""
    import itertools
    seeds = (3, 11, 19)
    host = [_stem(0, s) for s in seeds]
    dev = [_stem(1, s) for s in seeds]
    still = _stem(0, 3, nconf=1, pn_model=1)
    e_hh = np.mean([rel_l2(a, b) for a, b in itertools.combinations(host, 2)])
    e_dd = np.mean([rel_l2(a, b) for a, b in itertools.combinations(dev, 2)])
    e_dh = np.mean([rel_l2(a, b) for a in dev for b in host])
    e_still = np.mean([rel_l2(still, b) for b in host])
    print(f"host-host {e_hh:.3e}, device-host {e_dh:.3e}, device-device {e_dd:.3e}, still-host {e_still:.3e}")
    assert e_dh < 2 * e_hh and e_dd < 2 * e_hh
    assert e_still > 5 * max(e_hh, e_dh)


def test_device_draws_are_deterministic_and_differ_per_configuration():
    a = _stem(1, 5, nconf=2)
    b = _stem(1, 5, nconf=2)
    np.testing.assert_array_equal(a, b)
    p = specimens.stem_srtio3(nx=128, ny=128, na=4, nb=4, nc=4, ns=4, nconf=3, seed=7)
    p.pn_rng = 1
    _, x1 = api.phonon_atoms(p, 1)
    _, x2 = api.phonon_atoms(p, 2)
    assert np.mean(x1[:, :2] != x2[:, :2]) > 0.99
