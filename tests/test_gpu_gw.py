"""GPU parity of the FP64 GW chain against the CPU oracle (same seeded inputs).

Tolerances: the plain path is all FP64; P0/Wc agree to ~1e-12 relative, Sigma_c
to 1e-10 Ha absolute, QP energies to 1e-8 Ha (the parity bar of the plain FP64 path).
"""
import numpy as np
import pytest

from oracle import qx_oracle as O
from quasix_b200.synth import make_system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q():
    import quasix_b200
    return quasix_b200


def small():
    return make_system(5, 19, 84, seed=0, pi_norm=2.0)


def medium():
    return make_system(12, 61, 250, seed=3, pi_norm=3.0)


def test_rho_response_matches_oracle(q):
    s = small()
    lov = np.ascontiguousarray(s.lpq[:, :5, 5:])
    freqs = np.array([0.0, 0.05, 0.7, 3.0, 40.0])
    got = q.get_rho_response_batch(freqs, s.mo_energy, lov)
    for k, f in enumerate(freqs):
        ref = O.get_rho_response(f, s.mo_energy, lov)
        assert np.abs(got[k] - ref).max() < 1e-13 * max(1.0, np.abs(ref).max())


def test_polarizability_prefactor_hand_case(q):
    # quasix_core/src/dielectric/polarizability.rs:432-484
    p0 = q.compute_polarizability_p0(np.full((1, 1, 2), 0.1), np.array([0.5, -0.5]), np.array([2.0, 0.0]),
                                     np.array([1.0]))
    assert np.allclose(p0, 0.02, atol=1e-15)


@pytest.mark.parametrize("naux", [7, 64, 130, 257])
def test_screened_interaction_matches_oracle(q, naux):
    rng = np.random.default_rng(naux)
    b = rng.normal(size=(naux, 3 * naux)) * 0.1
    pi = -(b @ b.T)[None].repeat(2, 0)
    pi[1] *= 0.3
    got = q.compute_epsilon_inverse_minus_identity(pi)
    for k in range(2):
        ref = O.epsilon_inverse_minus_identity(pi[k])
        assert np.abs(got[k] - ref).max() < 1e-11


def test_indefinite_and_singular_epsilon(q):
    """Indefinite eps is inverted (the reference's LU fallback); a singular eps
    gives Wc = 0 (the reference's identity fallback, correlation_ac.rs:383-399)."""
    pi = np.eye(4)[None] * 2.0  # eps = -I, indefinite but regular
    assert np.allclose(q.compute_epsilon_inverse_minus_identity(pi), -2.0 * np.eye(4))
    rng = np.random.default_rng(2)
    x = rng.normal(size=(6, 6))
    pi = (np.eye(6) - (x + x.T) / 2)[None]  # eps symmetric indefinite
    ref = np.linalg.inv(np.eye(6) - pi[0]) - np.eye(6)
    assert np.abs(q.compute_epsilon_inverse_minus_identity(pi)[0] - ref).max() < 1e-10
    pi = np.eye(3)[None]  # eps = 0, singular
    assert np.abs(q.compute_epsilon_inverse_minus_identity(pi)).max() == 0.0


def test_sigma_six_mo_fixture(q):
    # quasix_core/src/selfenergy/frequency_cache.rs:621-700 fixture
    nmo, nocc, naux = 6, 3, 15
    e = np.array([-0.5, -0.4, -0.3, 0.1, 0.2, 0.3])
    P, m, n = np.meshgrid(np.arange(naux), np.arange(nmo), np.arange(nmo), indexing="ij")
    lpq = 0.1 * np.exp(-0.2 * (m + n + P))
    s, om = q.get_sigma_diag(e, lpq, list(range(6)), nocc, nw=20)
    s2, om2 = O.get_sigma_diag(e, lpq, list(range(6)), nocc, nw=20)
    assert s.shape == s2.shape
    assert np.abs(om - om2).max() < 1e-12 * np.abs(om2).max()
    assert np.abs(s - s2).max() < 1e-12


@pytest.mark.parametrize("sysf,nw,orbs", [(small, 16, [3, 4, 5, 6]), (small, 48, None), (medium, 24, [0, 11, 12, 40])])
def test_sigma_diag_matches_oracle(q, sysf, nw, orbs):
    s = sysf()
    orbs = list(range(s.nmo)) if orbs is None else orbs
    got, om = q.get_sigma_diag(s.mo_energy, s.lpq, orbs, s.nocc, nw=nw)
    ref, om2 = O.get_sigma_diag(s.mo_energy, s.lpq, orbs, s.nocc, nw=nw)
    assert np.abs(got - ref).max() < 1e-10


def test_exchange_matches_oracle(q):
    s = medium()
    got = q.compute_exchange_diag(s.lpq, s.nocc)
    ref = np.diag(O.compute_exchange(s.miP()))
    assert np.abs(got - ref).max() < 1e-12


def test_pade_coefficients_match_oracle(q):
    s = small()
    sig, om = O.get_sigma_diag(s.mo_energy, s.lpq, list(range(s.nmo)), s.nocc, nw=48)
    for npade in (None, 4):
        c, of = q.ac_pade_thiele_diag(sig, om, npade)
        c2, of2 = O.ac_pade_thiele_diag(sig, om, npade)
        assert np.abs(of - of2).max() == 0.0
        # High-order Thiele coefficients are ill-conditioned (reciprocal
        # differences amplify rounding), so the fits are compared by value.
        assert np.allclose(c[:2], c2[:2], rtol=1e-9, atol=1e-12)
        for p in range(s.nmo):
            for w in (-0.8, -0.2, 0.0, 0.3, 1.0):
                a = q.pade_thiele(w, of[p], c[:, p])
                b = O.pade_thiele(w, of2[p], c2[:, p])
                assert abs(a - b) < 1e-9 * max(1.0, abs(b))


def _dict_inputs(s, **kw):
    naux = s.naux
    d = dict(mo_energy=s.mo_energy, mo_occ=s.mo_occ, iaP=s.iaP(), ijP=s.miP().reshape(-1, naux),
             abP=s.abP().reshape(-1, naux), chol_v=np.eye(naux), vxc_dft=np.zeros(s.nmo))
    d.update(kw)
    return d


@pytest.mark.parametrize("qp_solver", ["linearized", "newton"])
def test_run_evgw_matches_oracle(q, qp_solver):
    s = small()
    cfg = _dict_inputs(s, nfreq=32, max_cycle=6, qp_solver=qp_solver, conv_tol=1e-7)
    got = q.run_evgw(cfg)
    ref = O.run_evgw(cfg)
    assert got["n_cycles"] == ref["n_cycles"] and got["converged"] == ref["converged"]
    assert np.abs(got["qp_energies"] - ref["qp_energies"]).max() < 1e-8
    assert np.abs(got["z_factors"] - ref["z_factors"]).max() < 1e-8
    assert np.abs(got["sigma_x"] - ref["sigma_x"]).max() < 1e-12
    assert np.abs(got["sigma_c_re"] - ref["sigma_c_re"]).max() < 1e-8
    # Intermediate iterates of the DIIS loop carry rounding differences of
    # earlier iterations amplified by the mixing; they are held to 3e-8 Ha.
    for a, b in zip(got["iteration_history"], ref["iteration_history"]):
        assert np.abs(a["qp_energies"] - b["qp_energies"]).max() < 3e-8
    for k in ("ip", "ea", "gap"):
        assert abs(got[k] - ref[k]) < 1e-8


def test_evgw_medium_kk_pade(q):
    """[k/k] Pade variant on a medium system."""
    s = medium()
    # k = 4 keeps the spread 8-point Thiele fit conditioned on this grid (a 1e-15
    # perturbation of Sigma moves it by ~3e-10 Ha; k = 8 by ~1e-4 Ha).  One
    # iteration only: with this fit the second iteration already crosses QP
    # levels and the loop turns chaotic (a 1e-13 change of the input energies
    # moves the third iterate by 0.06 Ha in the oracle itself).
    kw = dict(nfreq=24, max_cycle=1, conv_tol=1e-9, npade=4, diis=True)
    cfg = _dict_inputs(s, **kw)
    got = q.run_evgw(cfg)
    ref = O.run_evgw(cfg)
    assert np.abs(got["qp_energies"] - ref["qp_energies"]).max() < 1e-7


def test_input_validation(q):
    s = small()
    with pytest.raises(ValueError):
        q.get_sigma_diag(s.mo_energy, s.lpq, [0], 0, nw=8)
    with pytest.raises(ValueError):
        q.get_sigma_diag(s.mo_energy, s.lpq, [0], s.nmo, nw=8)
    with pytest.raises(ValueError):
        q.get_sigma_diag(s.mo_energy, s.lpq[:, :, :-1], [0], s.nocc, nw=8)
    with pytest.raises(ValueError):
        q.get_sigma_diag(s.mo_energy, s.lpq, [s.nmo], s.nocc, nw=8)


def test_tiny_system(q):
    s = make_system(1, 1, 3, seed=9, pi_norm=0.5)
    got, _ = q.get_sigma_diag(s.mo_energy, s.lpq, [0, 1], 1, nw=12)
    ref, _ = O.get_sigma_diag(s.mo_energy, s.lpq, [0, 1], 1, nw=12)
    assert np.abs(got - ref).max() < 1e-12


def test_evgw_fifteen_pade_runs_without_cutoff(q):
    """[15/15] Pade on a 32-point grid (cutoff lifted so the grid holds 33 points).

    The 30-point fit is ill-conditioned: a 1e-15 relative perturbation of the
    sampled Sigma_c moves the continued fraction by up to ~0.1 Ha on this grid
    (measured with the oracle), so GPU and oracle cannot agree to 1e-8 Ha; the
    test checks the fit runs and stays finite and that both land on the same
    side of the Fermi level."""
    s = small()
    cfg = _dict_inputs(s, nfreq=32, max_cycle=1, npade=15, iw_cutoff=1e9, conv_tol=1e-12)
    got = q.run_evgw(cfg)
    ref = O.run_evgw(cfg)
    assert np.all(np.isfinite(got["qp_energies"]))
    assert np.array_equal(got["qp_energies"] < 0, ref["qp_energies"] < 0)
