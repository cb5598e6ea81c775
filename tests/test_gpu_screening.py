"""GPU parity of compute_screened_interaction (the S3-3 form
W = v^1/2 (I - v^1/2 P0 v^1/2)^-1 v^1/2, dielectric/screening.rs:164-236)
against the oracle, plus the reference's own property checks of that
function (screening.rs:150-157): W symmetric, W -> v as P0 -> 0, and the
Dyson equation W = v + v P0 W."""
import numpy as np
import pytest

from oracle import qx_oracle as O

pytestmark = pytest.mark.gpu


def metric(n, seed, lo=0.1, hi=10.0):
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    return (q * np.geomspace(lo, hi, n)) @ q.T


def p0_cd(nfreq, n, seed, scale=0.05):
    """Negative semidefinite P0 of the CD convention, decaying with frequency."""
    rng = np.random.default_rng(seed)
    out = np.empty((nfreq, n, n))
    for k in range(nfreq):
        b = rng.standard_normal((n, 3 * n)) * np.sqrt(scale / n)
        out[k] = -(b @ b.T) / (1.0 + k)
    return out


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("n", [37, 150, 301])
def test_screened_interaction_matches_oracle(n):
    import quasix_b200 as q
    v = metric(n, n)
    p0 = p0_cd(5, n, n + 1)
    got = q.compute_screened_interaction(p0, v, np.linspace(0.1, 2.0, 5))
    ref = O.compute_screened_interaction(p0, v)
    assert rel(got, ref) < 1e-12
    assert np.array_equal(got, np.swapaxes(got, 1, 2))


def test_screened_interaction_properties():
    import quasix_b200 as q
    n = 120
    v = metric(n, 3)
    w0 = q.compute_screened_interaction(np.zeros((2, n, n)), v)
    assert rel(w0[0], v) < 1e-12 and rel(w0[1], v) < 1e-12
    p0 = p0_cd(3, n, 4)
    w = q.compute_screened_interaction(p0, v)
    for k in range(3):
        assert rel(w[k], v + v @ p0[k] @ w[k]) < 1e-11


def test_screened_interaction_indefinite_eps_takes_pivoted_path():
    """P0 with positive directions makes eps indefinite, with a tiny leading
    minor: the reference's Cholesky fails and LU inverts it; here the guard
    sends it to the pivoted re-inversion."""
    import quasix_b200 as q
    n = 96
    v = np.eye(n)
    rng = np.random.default_rng(9)
    a = rng.standard_normal((n, n))
    eps = 0.5 * (a + a.T) + 3.0 * np.eye(n)
    eps[0, 0] = 1e-13
    p0 = (np.eye(n) - eps)[None]
    got = q.compute_screened_interaction(p0, v)
    ref = O.compute_screened_interaction(p0, v)
    assert rel(got, ref) < 1e-10


def test_screened_interaction_rejects_indefinite_metric():
    import quasix_b200 as q
    n = 40
    v = metric(n, 5)
    v -= 0.2 * np.eye(n) + np.eye(n) * np.linalg.eigvalsh(v)[0]
    with pytest.raises(RuntimeError):
        q.compute_screened_interaction(p0_cd(1, n, 6), v)
    with pytest.raises(ValueError):
        q.compute_screened_interaction(np.zeros((1, n, n + 1)), np.eye(n))
