"""BSE optical properties on the GPU against the oracle (FP64: transition
dipoles 1e-13 relative, oscillator strengths 1e-12, spectra 1e-13), and the
oscillator strengths of run_bse_tda from its own eigenvectors."""
import numpy as np
import pytest

from oracle import qx_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(1e-300, np.abs(np.asarray(b)).max())


def test_reference_known_answers():
    from quasix_b200 import bse
    r = bse.compute_oscillator_strengths([0.3, 0.5], np.eye(2), [[1, 0, 0], [0, 1, 0]])
    assert abs(r["oscillator_strengths"][0] - 0.2) < 1e-10 and abs(r["oscillator_strengths"][1] - 1 / 3) < 1e-10
    r = bse.compute_oscillator_strengths([0.4], [[0.6], [0.8]], [[1, 0, 0], [0, 0, 1]])
    assert abs(r["oscillator_strengths"][0] - 0.4 * 2 / 3) < 1e-10
    with pytest.raises(RuntimeError, match="Negative eigenvalue"):
        bse.compute_oscillator_strengths([-0.3], [[1.0]], [[1.0, 0.0, 0.0]])
    with pytest.raises(ValueError):
        bse.compute_oscillator_strengths([0.3, 0.4], np.eye(3), [[1, 0, 0], [0, 1, 0]])
    s = bse.compute_absorption_spectrum([0.3], [1.0], energy_range=(0.1, 0.5), n_points=200, broadening=0.02 * 27.2114,
                                        broadening_type="gaussian")
    assert abs(s["energies"][int(np.argmax(s["intensities"]))] - 0.3) < 0.01


def test_matches_oracle_on_random_inputs():
    from quasix_b200 import bse
    rng = np.random.default_rng(1)
    nao, nmo, nocc = 150, 130, 23
    c = rng.standard_normal((nao, nmo)) / np.sqrt(nao)
    d = rng.standard_normal((3, nao, nao))
    d = d + d.transpose(0, 2, 1)
    mu = bse.compute_transition_dipoles(c, d, nocc)
    assert rel(mu, O.compute_transition_dipoles(c, d, nocc)) < 1e-13
    nt, nr = mu.shape[0], 10
    x = rng.standard_normal((nt, nr))
    e = np.sort(rng.uniform(0.1, 0.9, nr))
    r = bse.compute_oscillator_strengths(e, x, mu)
    f, dd, fs = O.compute_oscillator_strengths(e, x, mu)
    assert rel(r["oscillator_strengths"], f) < 1e-12 and rel(r["transition_dipoles"], dd) < 1e-12
    assert abs(r["f_sum"] - fs) < 1e-12 * fs
    for kind in ("lorentzian", "gaussian"):
        for rng_ in (None, (0.0, 1.2)):
            s = bse.compute_absorption_spectrum(e, f, energy_range=rng_, n_points=777, broadening=0.2,
                                                broadening_type=kind)
            ge, gi = O.compute_absorption_spectrum(e, f, 0.2 / 27.2114, kind == "gaussian", rng_, 777)
            assert rel(s["energies"], ge) < 1e-14 and rel(s["intensities"], gi) < 1e-13


def test_run_bse_tda_oscillator_strengths():
    import quasix_b200 as q
    from quasix_b200.synth import make_system
    s = make_system(6, 30, 90, seed=11, pi_norm=2.0)
    rng = np.random.default_rng(2)
    nao = s.nmo + 4
    c = np.linalg.qr(rng.standard_normal((nao, nao)))[0][:, : s.nmo]
    d = rng.standard_normal((3, nao, nao))
    d = d + d.transpose(0, 2, 1)
    res = q.run_bse_tda(lpq=s.lpq, mo_energy=s.mo_energy, nocc=s.nocc, nstates=4, tol=1e-8, verbose=False,
                        mo_coeff=c, ao_dipoles=d)
    mu = O.compute_transition_dipoles(c, d, s.nocc)
    f, dd, fs = O.compute_oscillator_strengths(res.excitation_energies_Ha, res.eigenvectors, mu)
    assert rel(res.oscillator_strengths, f) < 1e-12 and abs(res.f_sum - fs) < 1e-12 * max(fs, 1e-30)
    bare = q.run_bse_tda(lpq=s.lpq, mo_energy=s.mo_energy, nocc=s.nocc, nstates=4, tol=1e-8, verbose=False)
    assert np.isnan(bare.oscillator_strengths).all()
