"""Hellmann-Feynman gradient of the lowest BSE-TDA root with respect to the
orbital energies (oracle) against central differences of a dense
diagonalisation, with Delta_ia = e_a - e_i and W0 = (I - Pi(0))^-1 rebuilt from
the perturbed energies.  Small system: nocc 5, nvirt 19, naux 84, seed 0."""
import numpy as np

from oracle import qx_oracle as O
from quasix_b200.synth import make_system


def _lowest(e, s, nocc):
    nvirt = s.nmo - nocc
    df_ia, df_ij, df_ab = O.bse_blocks(s.lpq, nocc)
    w0 = O.bse_w0(s.lpq, e, nocc)
    delta = (e[None, nocc:] - e[:nocc, None]).reshape(-1)
    A = O.bse_apply_tda(np.eye(nocc * nvirt), delta, df_ia, df_ij, df_ab, w0, nocc, nvirt)
    w, v = np.linalg.eigh(0.5 * (A + A.T))
    return w[0], v[:, 0], (df_ia, df_ij, df_ab, w0)


def test_bse_lowest_root_gradient_matches_central_differences():
    s = make_system(5, 19, 84, seed=0, pi_norm=2.0)
    nocc, nvirt = 5, 19
    w, x, (df_ia, df_ij, df_ab, w0) = _lowest(s.mo_energy, s, nocc)
    g_full = O.bse_root_grad(x, df_ia, df_ij, df_ab, w0, nocc, nvirt, mo_energy=s.mo_energy)
    g_delta = O.bse_root_grad(x, df_ia, df_ij, df_ab, w0, nocc, nvirt)
    assert np.abs(g_full - g_delta).max() > 1e-4  # the W0 term matters
    h = 1e-5
    for p in [0, 2, 4, 5, 6, 11, 23]:
        ep, em = s.mo_energy.copy(), s.mo_energy.copy()
        ep[p] += h
        em[p] -= h
        fd = (_lowest(ep, s, nocc)[0] - _lowest(em, s, nocc)[0]) / (2 * h)
        assert abs(fd - g_full[p]) <= 1e-6 * max(abs(fd), 1e-2), (p, fd, g_full[p])


def _w0_from(df_ia, e, nocc):
    """W0 = (I - Pi(0))^-1, Pi(0) = 4 sum_ia B_ia B_ia^T / (e_i - e_a)."""
    e_ia = (e[:nocc, None] - e[None, nocc:]).reshape(-1)
    pi0 = 4.0 * (df_ia / e_ia[:, None]).T @ df_ia
    return np.linalg.inv(np.eye(df_ia.shape[1]) - pi0)


def _lowest_blocks(df_ia, df_ij, df_ab, e, nocc, nvirt, w0=None):
    if w0 is None:
        w0 = _w0_from(df_ia, e, nocc)
    delta = (e[None, nocc:] - e[:nocc, None]).reshape(-1)
    A = O.bse_apply_tda(np.eye(nocc * nvirt), delta, df_ia, df_ij, df_ab, w0, nocc, nvirt)
    w, v = np.linalg.eigh(0.5 * (A + A.T))
    return w[0], v[:, 0]


def test_bse_lowest_root_gradient_wrt_df_blocks_matches_central_differences():
    """dOmega/d(df_ia, df_ij, df_ab): W0 held fixed, and W0 following df_ia."""
    s = make_system(5, 19, 84, seed=0, pi_norm=2.0)
    nocc, nvirt = 5, 19
    e = s.mo_energy
    df_ia, df_ij, df_ab = O.bse_blocks(s.lpq, nocc)
    w0 = _w0_from(df_ia, e, nocc)
    _, x = _lowest_blocks(df_ia, df_ij, df_ab, e, nocc, nvirt, w0)
    h = 1e-6
    rng = np.random.default_rng(1)
    for follow in (False, True):
        g_ia, g_ij, g_ab = O.bse_root_grad_blocks(x, df_ia, df_ij, df_ab, w0, nocc, nvirt,
                                                  mo_energy=e if follow else None)
        for name, arr, g in (("ia", df_ia, g_ia), ("ij", df_ij, g_ij), ("ab", df_ab, g_ab)):
            mags = np.abs(g).reshape(-1)
            for k in rng.choice(np.argsort(mags)[-50:], 4, replace=False):
                r, c = divmod(int(k), arr.shape[1])
                vals = []
                for sgn in (1.0, -1.0):
                    blocks = {"ia": df_ia.copy(), "ij": df_ij.copy(), "ab": df_ab.copy()}
                    blocks[name][r, c] += sgn * h
                    ww = None if follow else w0
                    vals.append(_lowest_blocks(blocks["ia"], blocks["ij"], blocks["ab"], e, nocc, nvirt, ww)[0])
                fd = (vals[0] - vals[1]) / (2 * h)
                assert abs(fd - g[r, c]) <= 1e-6 * max(abs(fd), 1e-3), (follow, name, r, c, fd, g[r, c])
