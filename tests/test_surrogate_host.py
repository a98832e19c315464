"""Host-side pieces of the learned surrogate (multem_b200/surrogate.py) that need no GPU: the
noise floor of the many-configuration target, the conditioned network input and the error
measures."""
import numpy as np

from multem_b200 import surrogate as S


def test_noise_floor_matches_the_known_noise():
    rng = np.random.default_rng(0)
    yy, xx = np.mgrid[0:32, 0:32] / 32.0
    truth = 1.0 + 0.3 * np.cos(2 * np.pi * xx) * np.cos(2 * np.pi * yy)
    sigma = 0.1
    im = truth[None] + sigma * rng.standard_normal((64, 32, 32))
    expect = sigma * np.sqrt(60) / 64 / np.sqrt(np.mean(im.mean(axis=0) ** 2))
    assert abs(S.noise_floor(im, 4) / expect - 1) < 0.05


def test_conditioned_input():
    img = np.full((8, 8), 3.0)
    img[0, 0] = 5.0
    for n, level in ((4, 1.0), (16, 0.5), (64, 0.25)):
        x, s = S.conditioned_input(img, n)
        assert x.shape == (4, 8, 8) and x.dtype == np.float32
        assert abs(s - img.mean()) < 1e-12
        np.testing.assert_allclose(x[0] * s, img, rtol=1e-6)
        np.testing.assert_allclose(x[1], level)
        np.testing.assert_allclose(x[2], x[0])  # no period: the image itself
        np.testing.assert_allclose(x[3], 0.0)
    x, s = S.conditioned_input(img, 4, period=4)
    np.testing.assert_allclose(x[2] * s, S.lattice_fold(img, 4), rtol=1e-6)
    np.testing.assert_allclose(x[3], 1.0)


def test_lattice_fold():
    """A lattice-periodic image is a fixed point; independent noise shrinks by the square root of
    the number of equivalent positions (2 per cell, (H/p)*(W/p) cells)."""
    p = 8
    yy, xx = np.mgrid[0:32, 0:32]
    cell = np.cos(2 * np.pi * (xx + yy) / p) + np.cos(2 * np.pi * (xx - yy) / p) + 3.0  # period p/2 diagonal
    np.testing.assert_allclose(S.lattice_fold(cell, p), cell, atol=1e-12)
    rng = np.random.default_rng(1)
    noise = rng.standard_normal((200, 32, 32))
    folded = S.lattice_fold(noise, p)
    assert abs(folded.std() * np.sqrt(2 * 16) - 1) < 0.05
    with np.testing.assert_raises(ValueError):
        S.lattice_fold(noise[0, :30], p)


def test_error_measures():
    b = np.ones((4, 4))
    assert S.rel_rms(b, b) == 0.0
    assert abs(S.rel_rms(1.02 * b, b) - 0.02) < 1e-12
    assert abs(S.error_estimate(b, 0.03 * b) - 0.03) < 1e-12
    assert S.TIERS[0] == 4 and S.TIERS[-1] == 64
