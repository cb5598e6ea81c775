"""The oracle's spectral functions, pinned by the reference's own tests of
quasix_core/src/analysis/spectral.rs (:849-925) and by a closed form for the
Pade-based A(w).  CPU only."""
import numpy as np

from oracle import qx_oracle as O


def test_gaussian_normalization():
    # spectral.rs:849-861
    w = np.linspace(-5.0, 5.0, 1000)
    assert abs(np.sum(O.gaussian_broadening(w, 0.0, 0.1)) * (w[1] - w[0]) - 1.0) < 0.01


def test_lorentzian_normalization():
    # spectral.rs:863-875
    w = np.linspace(-10.0, 10.0, 2000)
    assert abs(np.sum(O.lorentzian_broadening(w, 0.0, 0.1)) * (w[1] - w[0]) - 1.0) < 0.01


def test_voigt_limits():
    # spectral.rs:909-925
    g = O.gaussian_broadening(1.0, 0.0, 0.1)
    lo = O.lorentzian_broadening(1.0, 0.0, 0.05)
    assert abs(O.voigt_profile(1.0, 0.0, 0.1, 0.05, 0.0) - g) <= 1e-10 * abs(g)
    assert abs(O.voigt_profile(1.0, 0.0, 0.1, 0.05, 1.0) - lo) <= 1e-10 * abs(lo)


def test_spectral_function_creation_and_pes_ipes():
    # spectral.rs:877-907
    e = np.array([-2.0, -1.0, 0.0, 1.0, 2.0])
    z = np.array([0.8, 0.7, 0.6, 0.7, 0.8])
    w = np.linspace(-3.0, 3.0, 100)
    out, tw = O.spectral_function(e, z, w)
    assert out.shape == (100,) and tw > 0.0
    e2 = np.array([-2.0, -1.0, 0.5, 1.0, 2.0])
    pes, _ = O.spectral_function(e2, z, np.linspace(0, 3, 50), kind=1)
    ipes, _ = O.spectral_function(e2, z, np.linspace(0, 3, 50), kind=2)
    # Two occupied states at binding energies 1 and 2; three empty ones at 0.5, 1, 2.
    ref_pes, _ = O.spectral_function([2.0, 1.0], [0.8, 0.7], np.linspace(0, 3, 50))
    ref_ipes, _ = O.spectral_function([0.5, 1.0, 2.0], [0.6, 0.7, 0.8], np.linspace(0, 3, 50))
    assert np.allclose(pes, ref_pes, rtol=1e-14) and np.allclose(ipes, ref_ipes, rtol=1e-14)


def test_states_form_integrates_to_z():
    # evgw.py:124-134: each row is Z_i times a unit Lorentzian.
    w = np.linspace(-40.0, 40.0, 400001)
    a = O.spectral_function_states([0.3, -0.2], [0.9, 0.6], w, eta=0.01)
    integ = a.sum(axis=1) * (w[1] - w[0])
    assert np.allclose(integ, [0.9, 0.6], atol=1e-3)


def test_pade_form_of_a_constant_self_energy():
    """Sigma_c = c (a one-point Thiele fit is the constant): A is a Lorentzian of
    width eta centred at e + Sx - Vxc + c."""
    c = -0.2 + 0.0j
    coeff = np.array([[c]])
    ofit = np.array([[0.5j]])
    w = np.linspace(-2, 2, 41)
    a = O.spectral_function_pade(coeff, ofit, [0.1], [-0.3], [0.05], 0.0, w, 0.02)
    centre = 0.1 - 0.3 - 0.05 + c.real
    ref = 0.02 / np.pi / ((w - centre) ** 2 + 0.02 ** 2)
    assert np.allclose(a[0], ref, rtol=1e-13)
