"""The device phonon generator (pn_rng 1): its CPU restatement against the published Philox4x32-10
vectors, the statistics of its displacements, and the host logic it relies on (no GPU)."""
import numpy as np
import pytest

from multem_b200 import api, capi, specimens
from oracle import phonon as P


def test_philox_known_answer_vectors():
    for ctr, key, res in P.KAT:
        out = P.philox4x32_10(np.array(ctr, np.uint32), np.array(key, np.uint32))[0]
        assert [int(v) for v in out] == list(res)


def test_normals_are_standard_and_independent():
    from scipy import stats
    n = 200_000
    x1, y1 = P.normals(n, 300183, 1)
    x2, _ = P.normals(n, 300183, 2)
    x3, _ = P.normals(n, 7, 1)
    for v in (x1, y1):
        assert abs(v.mean()) < 5 / np.sqrt(n) and abs(v.var() - 1) < 5 * np.sqrt(2 / n)
        assert stats.kstest(v, "norm").pvalue > 1e-3
    # x and y of one atom, the same atom in two configurations, two seeds: uncorrelated
    for a, b in ((x1, y1), (x1, x2), (x1, x3)):
        assert abs(np.corrcoef(a, b)[0, 1]) < 5 / np.sqrt(n)


def test_displacement_scales_with_sigma_and_respects_pn_dim():
    xyz = np.zeros((1000, 3), np.float32)
    sig = np.full(1000, 0.1, np.float32)
    d = P.displaced(xyz, sig, 5, 3)
    assert abs(d[:, 0].std() - 0.1) < 0.01 and abs(d[:, 1].std() - 0.1) < 0.01
    assert np.all(d[:, 2] == 0)
    dx = P.displaced(xyz, sig, 5, 3, pn_y=False)
    assert np.all(dx[:, 1] == 0) and np.array_equal(dx[:, 0], d[:, 0])


def test_slicing_does_not_depend_on_the_configuration():
    """The plain path never displaces z, so the device generator's single slicing (of the undisplaced
    atoms) is the slicing of every configuration the reference's host draws produce."""
    p = specimens.stem_srtio3(nx=128, ny=128, na=4, nb=4, nc=4, ns=4, nconf=3, seed=7)
    p.potential_slicing = 2
    for rng in (0, 1):
        p.pn_rng = rng
        for iconf in (1, 2, 3):
            s = api.specimen_slices(p, iconf)
            if rng == 0 and iconf == 1:
                ref = s
            for k in ref:
                np.testing.assert_array_equal(s[k], ref[k])


def test_invalid_generator_is_refused():
    p = specimens.stem_srtio3(nx=128, ny=128, na=2, nb=2, nc=2, ns=2, nconf=2, seed=7)
    p.pn_rng = 2
    with pytest.raises(capi.MtError) as e:
        api.output_dims(p)
    assert e.value.status == 1
