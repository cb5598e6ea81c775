"""The oracle's BSE optical functions, pinned by the reference's own tests
(quasix_core/src/bse/optical.rs:410-680).  CPU only."""
import math

import numpy as np
import pytest

from oracle import qx_oracle as O


def test_oscillator_strength_simple():
    # optical.rs:410-431
    f, _, _ = O.compute_oscillator_strengths([0.3, 0.5], np.eye(2), [[1, 0, 0], [0, 1, 0]])
    assert abs(f[0] - 0.2) < 1e-10 and abs(f[1] - 1.0 / 3.0) < 1e-10


def test_oscillator_strength_normalization():
    # optical.rs:433-456
    f, d, _ = O.compute_oscillator_strengths([0.4], [[0.6], [0.8]], [[1, 0, 0], [0, 0, 1]])
    assert abs(f[0] - 0.4 * 2.0 / 3.0) < 1e-10 and np.allclose(d, [[0.6, 0.0, 0.8]])


def test_nonnegative_and_f_sum():
    # optical.rs:458-476, 587-604
    x = np.full((3, 3), 0.1) + np.eye(3) * 0.7
    mu = np.sin(0.1 * (np.arange(3)[:, None] + np.arange(3)[None, :]))
    f, _, fs = O.compute_oscillator_strengths([0.1, 0.2, 0.3], x, mu)
    assert np.all(f >= 0.0)
    _, _, fs = O.compute_oscillator_strengths([0.2, 0.3, 0.4], np.eye(3), [[1, .5, 0], [.5, 1, .3], [.3, .2, 1]])
    assert fs > 0.0 and math.isfinite(fs)


def test_validation():
    # optical.rs:542-585
    with pytest.raises(ValueError):
        O.compute_oscillator_strengths([0.3, 0.4], np.eye(3), [[1, 0, 0], [0, 1, 0]])
    with pytest.raises(ValueError):
        O.compute_oscillator_strengths([0.3], [[1.0]], [[1.0, 0.0]])
    with pytest.raises(ValueError):
        O.compute_oscillator_strengths([-0.3], [[1.0]], [[1.0, 0.0, 0.0]])


def test_line_shapes():
    # optical.rs:642-659
    assert abs(O.absorption_lorentzian(0.0, 0.1) - 10.0) < 1e-10
    assert abs(O.absorption_lorentzian(0.1, 0.1) - 5.0) < 1e-10
    assert abs(O.absorption_gaussian(0.0, 0.1) - 1.0) < 1e-10
    assert abs(O.absorption_gaussian(0.1, 0.1) - math.exp(-0.5)) < 1e-10


def test_absorption_peaks():
    # optical.rs:478-540
    e, i = O.compute_absorption_spectrum([0.2, 0.4], [0.5, 0.3], 0.01, energy_range=(0.1, 0.5), n_points=100)
    assert e.shape == (100,) and i.shape == (100,)
    k = int(np.argmin(np.abs(e - 0.2)))
    assert i[k] > i[max(k - 5, 0)]
    e, i = O.compute_absorption_spectrum([0.3], [1.0], 0.02, gaussian=True, energy_range=(0.1, 0.5), n_points=200)
    assert abs(e[int(np.argmax(i))] - 0.3) < 0.01


def test_transition_dipoles_transform():
    rng = np.random.default_rng(0)
    nao, nmo, nocc = 9, 7, 3
    c = rng.standard_normal((nao, nmo))
    d = rng.standard_normal((3, nao, nao))
    mu = O.compute_transition_dipoles(c, d, nocc)
    i, a, k = 2, 1, 1
    ref = sum(c[m, i] * d[k, m, n] * c[n, nocc + a] for m in range(nao) for n in range(nao))
    assert abs(mu[i * (nmo - nocc) + a, k] - ref) < 1e-12
