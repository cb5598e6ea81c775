"""Guarded eps inversion: nonsingular eps that the unpivoted sweep cannot
invert (zero or tiny leading pivots, large element growth) are inverted again
with partial pivoting, as the reference's LU fallback does after a failed
Cholesky (quasix_core/src/selfenergy/correlation_ac.rs:383-399).

Every case is compared with numpy's LU inverse (the oracle's LU branch,
oracle.qx_oracle.epsilon_inverse_minus_identity) at 1e-11 relative to
max|Wc|; an exactly singular eps gives Wc = 0 (the identity fallback).
"""
import ctypes as C

import numpy as np
import pytest

from oracle import qx_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-11


@pytest.fixture(scope="module")
def q():
    import quasix_b200
    return quasix_b200


def wc_ref(eps):
    return O.epsilon_inverse_minus_identity(np.eye(eps.shape[0]) - eps)


def rel(a, b):
    return np.abs(a - b).max() / max(1.0, np.abs(b).max())


def sym(rng, n, scale=1.0):
    x = rng.standard_normal((n, n)) * scale
    return (x + x.T) / 2


def check(q, eps_list):
    eps = np.stack(eps_list)
    pi = np.eye(eps.shape[1])[None] - eps
    got = q.compute_epsilon_inverse_minus_identity(pi)
    for k, e in enumerate(eps_list):
        ref = wc_ref(e)
        assert rel(got[k], ref) < TOL, (k, rel(got[k], ref))
    return got


def test_swap_matrix(q):
    """eps = [[0, 1], [1, 0]]: the unpivoted sweep meets a zero pivot at once."""
    got = check(q, [np.array([[0.0, 1.0], [1.0, 0.0]])])
    assert np.allclose(got[0], [[-1.0, 1.0], [1.0, -1.0]], atol=1e-15)


def test_zero_and_tiny_leading_pivot(q):
    rng = np.random.default_rng(7)
    cases = []
    for lead in (0.0, 1e-12, 1e-14, -3e-9):
        e = np.eye(9) + sym(rng, 9)
        e[0, 0] = lead
        cases.append(e)
    check(q, cases)


def test_growth_without_small_pivot(q):
    """Leading pivot 2e-6 (above the 1e-6 pivot guard) with unit couplings:
    the Schur complement grows to ~5e5, which the growth guard catches."""
    rng = np.random.default_rng(8)
    e = np.eye(12) + 0.3 * sym(rng, 12)
    e[0, 0] = 2e-6
    e[0, 1:] = e[1:, 0] = 1.0
    check(q, [e])


@pytest.mark.parametrize("n,zero", [(300, 100), (257, 130), (129, 129 // 2)])
def test_singular_leading_block(q, n, zero):
    """A zero leading zero x zero block (nonsingular overall): the fallback's
    panels (32 wide) and update tiles (64) cross the sweep's 128-blocks, and n
    is no multiple of either."""
    rng = np.random.default_rng(n)
    e = sym(rng, n) + 2.0 * np.eye(n)
    e[:zero, :zero] = 0.0
    check(q, [e])


def test_mixed_batch_with_singular_member(q):
    """One call: an SPD eps (no fallback), a zero-pivot eps (fallback) and a
    singular eps (Wc = 0, the reference's identity fallback)."""
    rng = np.random.default_rng(3)
    n = 40
    b = rng.standard_normal((n, 3 * n)) * 0.1
    spd = np.eye(n) + b @ b.T
    piv = np.eye(n) + sym(rng, n)
    piv[0, 0] = 0.0
    sing = sym(rng, n)
    sing[:, 0] = 0.0
    sing[0, :] = 0.0
    eps = np.stack([spd, piv, sing])
    got = q.compute_epsilon_inverse_minus_identity(np.eye(n)[None] - eps)
    assert rel(got[0], wc_ref(spd)) < TOL
    assert rel(got[1], wc_ref(piv)) < TOL
    assert np.abs(got[2]).max() == 0.0


def test_noalloc_takes_the_same_fallback(q):
    """qx_screened_interaction_noalloc runs the same guarded sweep from its
    static scratch: it reproduces qx_screened_interaction bit for bit."""
    import torch
    from quasix_b200 import _native
    rng = np.random.default_rng(5)
    n = 200
    cases = []
    for lead in (0.0, 1e-13, None):
        e = sym(rng, n) + 3.0 * np.eye(n)
        if lead is not None:
            e[:70, :70] = 0.0
            e[0, 0] = lead
        cases.append(e)
    pi = np.ascontiguousarray(np.eye(n)[None] - np.stack(cases))
    ref = q.compute_epsilon_inverse_minus_identity(pi)
    ctx = _native.context(0)
    pd = torch.from_numpy(pi).cuda()
    wd = torch.empty_like(pd)
    torch.cuda.synchronize()
    ctx.check(ctx.lib.qx_screened_interaction_noalloc(ctx.handle, 3, n, C.c_void_p(pd.data_ptr()),
                                                      C.c_void_p(wd.data_ptr())))
    got = wd.cpu().numpy()
    assert np.array_equal(got, ref)
    for k, e in enumerate(cases):
        assert rel(got[k], wc_ref(e)) < TOL


@pytest.mark.parametrize("delta", [1e-3, 1e-6, 1e-9])
def test_cd_residue_shift_next_to_a_transition(q, delta):
    """Sigma_LUMO at w just above e_LUMO + gap: its residue eps(w_r) has a shift
    (1 + delta) x the smallest transition, where chi' of that pair is large and
    negative, so eps is indefinite and the inversion runs guarded.  The CD
    Sigma and its slope match the oracle (numpy LU solve per residue).  The
    slope reads B^T x along the resonant pair, a component ~delta of x times a
    chi' derivative ~1/delta^2: at delta = 1e-9 the oracle's own LU value of
    that residue is 1e-7 (relative) from its 50-digit value, so the slope is
    compared at 1e-6 there and at 1e-8 otherwise."""
    from quasix_b200.synth import make_system
    s = make_system(3, 9, 30, seed=21, pi_norm=2.0)
    nocc = s.nocc
    gap = s.mo_energy[nocc] - s.mo_energy[nocc - 1]
    lumo = nocc
    om = s.mo_energy[lumo] + gap * (1.0 + delta)
    nw = 16
    freqs, wts = O.get_scaled_legendre_roots(nw, 0.5)
    wci = O.wc_pairs_imag(s.mo_energy, s.lpq, nocc, [lumo], freqs)[:, 0, :]
    ref, dref = O.sigma_cd(om, lumo, s.mo_energy, s.lpq, nocc, freqs, wts, wci)
    r = q.cd_sigma(s.mo_energy, s.lpq, nocc, [lumo], [om], nw=nw)
    got, dgot = r["sigma_c"][0], r["dsigma_c"][0]
    assert abs(got - ref) <= 1e-9 * max(1.0, abs(ref)), (got, ref)
    tol = 1e-6 if delta < 1e-7 else 1e-8
    assert abs(dgot - dref) <= tol * max(1.0, abs(dref)), (dgot, dref)


def test_eps_certificate_with_crossed_levels(q):
    """Levels that crossed (an occupied level above a virtual one): eps is not
    certified >= I, so the evGW/CD inversions run guarded, and the CD Sigma
    still matches the oracle."""
    from quasix_b200.synth import make_system
    s = make_system(4, 12, 40, seed=22, pi_norm=2.0)
    e = s.mo_energy.copy()
    e[s.nocc - 1], e[s.nocc] = e[s.nocc] + 0.05, e[s.nocc - 1] - 0.05  # crossed
    lib = q._native.load()
    assert lib.qx_eps_at_least_identity(e.ctypes.data, s.nocc, s.nmo - s.nocc, 0.0) == 0
    nw = 16
    freqs, wts = O.get_scaled_legendre_roots(nw, 0.5)
    t = s.nocc - 2
    wci = O.wc_pairs_imag(e, s.lpq, s.nocc, [t], freqs)[:, 0, :]
    om = e[t] - 0.01
    ref, _ = O.sigma_cd(om, t, e, s.lpq, s.nocc, freqs, wts, wci)
    got = q.cd_sigma(e, s.lpq, s.nocc, [t], [om], nw=nw)["sigma_c"][0]
    assert abs(got - ref) <= 1e-9 * max(1.0, abs(ref)), (got, ref)
