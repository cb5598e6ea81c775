"""Device Thiele/Pade entry points and spectral functions against the oracle.

Tolerances: the Pade fit and evaluation are the same FP64 recursion as the
oracle's; the reciprocal differences amplify the last-bit differences of the
complex divisions (the device divides by b conj(b), numpy scales first), so
the coefficients and the continued fraction's values agree to 1e-11
relative; the broadened spectral sums are FP64 sums of exp / rational terms
(1e-13 relative to max|A|).
"""
import numpy as np
import pytest

from oracle import qx_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q():
    import quasix_b200
    return quasix_b200


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(1e-300, np.abs(np.asarray(b)).max())


def test_pade_thiele_known_answer(q):
    # correlation_ac.rs:775-810: Pade of 1/(1+z) from four points on the imaginary axis.
    zn = np.array([0.5j, 1j, 2j, 4j])
    c = O.thiele(1.0 / (1.0 + zn), zn)
    w = np.array([0.0, 0.1, -0.3, 2.5])
    got = q.pade_thiele(w, zn, c)
    ref = np.array([O.pade_thiele(x, zn, c) for x in w])
    assert rel(got, ref) < 1e-14
    assert abs(got[1] - 1.0 / 1.1) < 0.01 and abs(got[0].real - 1.0) < 0.01


def test_thiele_fit_on_device_matches_oracle(q):
    from quasix_b200.synth import make_system
    s = make_system(5, 19, 84, seed=0, pi_norm=2.0)
    sig, om = q.get_sigma_diag(s.mo_energy, s.lpq, list(range(s.nmo)), s.nocc, nw=32)
    for npade in (None, 4):
        c, f = q.ac_pade_thiele_diag(sig, om, npade)
        c2, f2 = O.ac_pade_thiele_diag(sig, om, npade)
        assert np.array_equal(f, f2)
        assert rel(c, c2) < 1e-11
        w = np.linspace(-1.0, 1.0, 7)
        for p in (0, 4, 5, 23):
            got = q.pade_thiele(w, f[p], c[:, p])
            ref = np.array([O.pade_thiele(x, f2[p], c2[:, p]) for x in w])
            assert rel(got, ref) < 1e-11


def test_spectral_function_matches_oracle(q):
    from quasix_b200.spectral import BroadeningParams, SpectralAnalyzer
    rng = np.random.default_rng(4)
    e = np.sort(rng.uniform(-20.0, 10.0, 700))
    z = rng.uniform(0.5, 0.95, 700)
    w = np.linspace(-25.0, 15.0, 3001)
    an = SpectralAnalyzer(e, z, -2.0)
    for mix in (0.0, 0.5, 1.0):
        an.set_broadening(BroadeningParams(0.2, 0.1, 300.0, mix))
        got = an.compute_spectral_function(w)
        ref, tw = O.spectral_function(e, z, w, 0.2, 0.1, mix)
        assert rel(got.spectral_weights, ref) < 1e-13
        assert abs(got.metadata.total_weight - tw) < 1e-12 * tw
    pes = an.generate_pes_spectrum(0.0, 20.0, 500)
    ipes = an.generate_ipes_spectrum(0.0, 15.0, 400)
    assert pes.metadata.n_states == int(np.sum(e <= -2.0)) and ipes.metadata.n_states == int(np.sum(e > -2.0))
    ref_p, _ = O.spectral_function(e, z, np.linspace(0, 20, 500), 0.2, 0.1, 1.0, -2.0, 1)
    ref_i, _ = O.spectral_function(e, z, np.linspace(0, 15, 400), 0.2, 0.1, 1.0, -2.0, 2)
    assert rel(pes.spectral_weights, ref_p) < 1e-13 and rel(ipes.spectral_weights, ref_i) < 1e-13


def test_spectral_function_validation(q):
    from quasix_b200.spectral import BroadeningParams, SpectralAnalyzer
    with pytest.raises(ValueError, match="Z-factor"):
        SpectralAnalyzer([-1.0, 0.0, 1.0], [0.5, 1.5, 0.3], 0.0)   # spectral.rs:839-847
    an = SpectralAnalyzer([-1.0, 0.0, 1.0], [0.5, 0.8, 0.3], 0.0)
    with pytest.raises(ValueError):
        an.set_broadening(BroadeningParams(gaussian_width=-1.0))  # spectral.rs:826-837
    with pytest.raises(ValueError):
        an.set_broadening(BroadeningParams(voigt_mixing=1.5))
    with pytest.raises(ValueError, match="Empty omega grid"):
        an.compute_spectral_function(np.zeros(0))
    # The C ABI applies the same checks itself.
    import ctypes as C
    from quasix_b200 import _native
    ctx = _native.context(0)
    e, z, w, out = np.array([0.0]), np.array([1.5]), np.linspace(-1, 1, 5), np.zeros(5)
    st = ctx.lib.qx_spectral_function(ctx.handle, e.ctypes.data, z.ctypes.data, 1, 0.0, 0, w.ctypes.data, 5, 0.1,
                                      0.05, 0.5, out.ctypes.data, None)
    assert st == 1 and b"Z-factor" in ctx.lib.qx_last_error(ctx.handle)


def test_spectral_states_and_pade(q):
    from quasix_b200.spectral import spectral_function_pade, spectral_function_states
    from quasix_b200.synth import make_system
    rng = np.random.default_rng(9)
    e, z = rng.uniform(-1, 1, 37), rng.uniform(0.1, 1.0, 37)
    w = np.linspace(-1.5, 1.5, 777)
    assert rel(spectral_function_states(e, z, w, 0.02), O.spectral_function_states(e, z, w, 0.02)) < 1e-13
    s = make_system(5, 19, 84, seed=0, pi_norm=2.0)
    orbs = list(range(2, 9))
    sig, om = q.get_sigma_diag(s.mo_energy, s.lpq, orbs, s.nocc, nw=32)
    c, f = q.ac_pade_thiele_diag(sig, om)
    sx = q.compute_exchange_diag(s.lpq, s.nocc)[orbs]
    ef = 0.5 * (s.mo_energy[s.nocc - 1] + s.mo_energy[s.nocc])
    vxc = 0.9 * sx
    wg = np.linspace(-3.0, 3.0, 901)
    got = spectral_function_pade(c, f, s.mo_energy[orbs], sx, wg, ef, vxc=vxc, eta=0.01)
    ref = O.spectral_function_pade(c, f, s.mo_energy[orbs], sx, vxc, ef, wg, 0.01)
    assert rel(got, ref) < 1e-12
