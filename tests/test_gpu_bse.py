"""BSE-TDA on the GPU against the CPU oracle (quasix_core/src/bse/kernel.rs and
davidson.rs restated): matvec to 1e-12, Davidson roots to the residual
tolerance (1e-8 Ha roots at tol 1e-8 are accurate to ~tol^2/gap)."""
import numpy as np
import pytest

from oracle import qx_oracle as O
from quasix_b200.synth import make_system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q():
    import quasix_b200
    return quasix_b200


def bse_inputs(nocc, nvir, naux, seed, pi_norm=2.0):
    s = make_system(nocc, nvir, naux, seed=seed, pi_norm=pi_norm)
    dia, dij, dab = O.bse_blocks(s.lpq, nocc)
    w0 = O.bse_w0(s.lpq, s.mo_energy, nocc)
    delta = (s.mo_energy[None, nocc:] - s.mo_energy[:nocc, None]).reshape(-1)
    return s, delta, dia, dij, dab, w0


def test_screened_w0_matches_oracle(q):
    s, *_ = bse_inputs(6, 30, 80, 1)
    got = q.bse.screened_w0(s.mo_energy, np.ascontiguousarray(s.lpq[:, :6, 6:]))
    assert np.abs(got - O.bse_w0(s.lpq, s.mo_energy, 6)).max() < 1e-12


@pytest.mark.parametrize("spin,ax", [("singlet", 2.0), ("triplet", 0.0)])
@pytest.mark.parametrize("shape", [(6, 30, 80), (7, 13, 31)])
def test_matvec_matches_oracle(q, spin, ax, shape):
    nocc, nvir, naux = shape
    s, delta, dia, dij, dab, w0 = bse_inputs(nocc, nvir, naux, 2)
    k = q.BSETDAKernel(nocc, nvir, naux, delta, dia, dij, dab, w0, spin=spin)
    x = np.random.default_rng(0).normal(size=(nocc * nvir, 5))
    got = k.apply_hamiltonian_batch(x)
    ref = O.bse_apply_tda(x, delta, dia, dij, dab, w0, nocc, nvir, alpha_x=ax)
    assert np.abs(got - ref).max() < 1e-12 * max(1.0, np.abs(ref).max())
    one = k.apply_hamiltonian(x[:, 0])
    assert np.abs(one - ref[:, 0]).max() < 1e-12 * max(1.0, np.abs(ref).max())


def test_davidson_matches_dense_eigh(q):
    nocc, nvir, naux = 8, 40, 96
    s, delta, dia, dij, dab, w0 = bse_inputs(nocc, nvir, naux, 3)
    k = q.BSETDAKernel(nocc, nvir, naux, delta, dia, dij, dab, w0)
    r = k.solve_davidson(n_roots=5, max_iter=200, tol_residual=1e-8)
    H = O.bse_apply_tda(np.eye(nocc * nvir), delta, dia, dij, dab, w0, nocc, nvir)
    ev = np.linalg.eigvalsh(0.5 * (H + H.T))[:5]
    assert r["all_converged"]
    assert np.abs(r["eigenvalues"] - ev).max() < 1e-9
    X = r["eigenvectors"]
    assert np.abs(X.T @ X - np.eye(5)).max() < 1e-7
    ro = O.davidson_bse(lambda V: O.bse_apply_tda(V, delta, dia, dij, dab, w0, nocc, nvir), delta,
                        O.DavidsonConfig(n_roots=5, max_iter=200, max_space=100, tol_residual=1e-8))
    assert np.abs(r["eigenvalues"] - ro["eigenvalues"]).max() < 1e-9


def test_davidson_restart_path(q):
    """A small max_space forces the restart branch (davidson.rs:298-307)."""
    nocc, nvir, naux = 6, 30, 70
    s, delta, dia, dij, dab, w0 = bse_inputs(nocc, nvir, naux, 4)
    k = q.BSETDAKernel(nocc, nvir, naux, delta, dia, dij, dab, w0)
    cfg = dict(n_roots=3, max_iter=300, max_space=12, tol_residual=1e-8)
    r = k.solve_davidson_with_config(q.DavidsonConfig(**cfg))
    H = O.bse_apply_tda(np.eye(nocc * nvir), delta, dia, dij, dab, w0, nocc, nvir)
    ev = np.linalg.eigvalsh(0.5 * (H + H.T))[:3]
    assert r["all_converged"] and np.abs(r["eigenvalues"] - ev).max() < 1e-9
    ro = O.davidson_bse(lambda V: O.bse_apply_tda(V, delta, dia, dij, dab, w0, nocc, nvir), delta,
                        O.DavidsonConfig(**cfg))
    # Same algorithm, same restarts: the iteration counts agree up to rounding
    # of the convergence test.
    assert abs(r["iterations"] - ro["iterations"]) <= 3


def test_trivial_dimension(q):
    """n_trans <= n_roots: the full matrix is diagonalised (davidson.rs:384-387)."""
    s, delta, dia, dij, dab, w0 = bse_inputs(1, 2, 5, 5)
    k = q.BSETDAKernel(1, 2, 5, delta, dia, dij, dab, w0)
    r = k.solve_davidson(n_roots=3)
    H = O.bse_apply_tda(np.eye(2), delta, dia, dij, dab, w0, 1, 2)
    assert np.abs(r["eigenvalues"] - np.linalg.eigvalsh(0.5 * (H + H.T))).max() < 1e-12


def test_rejects_bad_inputs(q):
    s, delta, dia, dij, dab, w0 = bse_inputs(3, 5, 12, 6)
    with pytest.raises(ValueError):
        q.BSETDAKernel(3, 5, 12, delta[:-1], dia, dij, dab, w0)
    with pytest.raises(ValueError):
        q.BSETDAKernel(3, 5, 12, delta, dia, dij, dab, w0, spin="quintet")
    bad = delta.copy()
    bad[0] = np.nan
    from quasix_b200._native import QxError
    with pytest.raises(QxError):
        q.BSETDAKernel(3, 5, 12, bad, dia, dij, dab, w0)


def test_run_bse_tda(q):
    s = make_system(6, 30, 80, seed=7, pi_norm=2.0)
    res = q.run_bse_tda(nstates=4, tol=1e-8, lpq=s.lpq, mo_energy=s.mo_energy, nocc=6)
    dia, dij, dab = O.bse_blocks(s.lpq, 6)
    w0 = O.bse_w0(s.lpq, s.mo_energy, 6)
    delta = (s.mo_energy[None, 6:] - s.mo_energy[:6, None]).reshape(-1)
    H = O.bse_apply_tda(np.eye(180), delta, dia, dij, dab, w0, 6, 30)
    assert res.converged and np.abs(res.excitation_energies_Ha - np.linalg.eigvalsh(H)[:4]).max() < 1e-9


@pytest.mark.parametrize("shape", [(6, 30, 80), (7, 13, 31)])
def test_root_gradient_matches_oracle(q, shape):
    """Hellmann-Feynman gradient of the lowest root (the oracle's is checked
    against central differences in tests/test_oracle_bse_grad.py)."""
    nocc, nvir, naux = shape
    s, delta, dia, dij, dab, w0 = bse_inputs(nocc, nvir, naux, 4)
    k = q.BSETDAKernel(nocc, nvir, naux, delta, dia, dij, dab, w0)
    r = k.solve_davidson(n_roots=1, tol_residual=1e-9)
    x = r["eigenvectors"][:, 0]
    for e in (s.mo_energy, None):
        got = k.root_gradient(3.0 * x, mo_energy=e)  # any norm
        ref = O.bse_root_grad(x, dia, dij, dab, w0, nocc, nvir, mo_energy=e)
        assert np.abs(got - ref).max() < 1e-10 * np.abs(ref).max()


@pytest.mark.parametrize("precision", ["fp64", "fp16x3"])
def test_davidson_is_deterministic(q, precision):
    """Two solves from the same start take the same path: identical iteration
    counts and bit-identical roots (the norm reductions have a fixed order)."""
    nocc, nvir, naux = 12, 60, 150
    s, delta, dia, dij, dab, w0 = bse_inputs(nocc, nvir, naux, 3)
    k = q.BSETDAKernel(nocc, nvir, naux, delta, dia, dij, dab, w0, precision=precision)
    r1 = k.solve_davidson(n_roots=5, tol_residual=1e-8)
    r2 = k.solve_davidson(n_roots=5, tol_residual=1e-8)
    assert r1["iterations"] == r2["iterations"]
    assert np.array_equal(np.array(r1["eigenvalues"]), np.array(r2["eigenvalues"]))


@pytest.mark.parametrize("precision,tol", [("fp16x3", 2e-6), ("bf16x3", 3e-5)])
def test_split_precision_matvec_and_roots(q, precision, tol):
    """Split forms: the direct kernel K^d is held as hi/lo and the direct term
    is one tcgen05 GEMM (FP64 drain of each 64-wide K block); the exchange
    term and the Rayleigh-Ritz step stay FP64.  Matvec error relative to
    max|y|; roots within 1e-6 Ha of FP64."""
    nocc, nvir, naux = 6, 30, 80
    s, delta, dia, dij, dab, w0 = bse_inputs(nocc, nvir, naux, 2)
    k = q.BSETDAKernel(nocc, nvir, naux, delta, dia, dij, dab, w0, precision=precision)
    x = np.random.default_rng(0).normal(size=(nocc * nvir, 7))
    ref = O.bse_apply_tda(x, delta, dia, dij, dab, w0, nocc, nvir)
    got = k.apply_hamiltonian_batch(x)
    assert np.abs(got - ref).max() < tol * np.abs(ref).max()
    k64 = q.BSETDAKernel(nocc, nvir, naux, delta, dia, dij, dab, w0)
    r64 = k64.solve_davidson(n_roots=4, tol_residual=1e-8)
    r = k.solve_davidson(n_roots=4, tol_residual=1e-8)
    assert np.abs(np.array(r["eigenvalues"]) - np.array(r64["eigenvalues"])).max() < 1e-6
