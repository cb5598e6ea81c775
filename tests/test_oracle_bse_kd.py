"""The materialised direct kernel of the split-form BSE matvec, checked on the
CPU against the oracle's factored matvec (bse/kernel.rs:391-462).

In the split forms `qx_bse_create` builds C[(i,j)][(a,b)] = sum_Q
ijw[(i,j)][Q] B_ab[(a,b)][Q] with ijw = B_ij W0, and every matvec's direct term
is one GEMM with K^d[(i,a)][(j,b)] = C[(i,j)][(a,b)]; its output rows (i,a)
with the vectors as columns are the factored form's Yd[i][(a,v)].  This test
pins that index map and the layout identity in FP64 (no GPU).
"""
import numpy as np

from oracle import qx_oracle as O
from quasix_b200.synth import make_system


def _direct_kernel(df_ij, df_ab, w0, nocc, nvir):
    naux = df_ij.shape[1]
    ijw = df_ij @ w0                                   # [(i,j)][Q]
    c = ijw @ df_ab.T                                  # C[(i,j)][(a,b)]
    # K^d[(i,a)][(j,b)] = C[(i,j)][(a,b)]
    return c.reshape(nocc, nocc, nvir, nvir).transpose(0, 2, 1, 3).reshape(nocc * nvir, nocc * nvir), naux


def test_direct_kernel_reproduces_the_factored_matvec():
    nocc, nvir, naux = 5, 17, 46
    s = make_system(nocc, nvir, naux, seed=4, pi_norm=2.0)
    df_ia, df_ij, df_ab = O.bse_blocks(s.lpq, nocc)
    w0 = O.bse_w0(s.lpq, s.mo_energy, nocc)
    delta = (s.mo_energy[None, nocc:] - s.mo_energy[:nocc, None]).reshape(-1)
    kd, _ = _direct_kernel(df_ij, df_ab, w0, nocc, nvir)
    x = np.random.default_rng(1).normal(size=(nocc * nvir, 6))
    for ax in (2.0, 0.0):
        ref = O.bse_apply_tda(x, delta, df_ia, df_ij, df_ab, w0, nocc, nvir, alpha_x=ax)
        got = delta[:, None] * x + ax * (df_ia @ (df_ia.T @ x)) - kd @ x
        assert np.abs(got - ref).max() < 1e-12 * np.abs(ref).max()


def test_direct_kernel_is_symmetric():
    """K^d is symmetric (W0 symmetric, B_ij and B_ab symmetric in their pair
    index), so the materialised TDA matrix is too."""
    nocc, nvir, naux = 4, 11, 30
    s = make_system(nocc, nvir, naux, seed=9, pi_norm=3.0)
    _, df_ij, df_ab = O.bse_blocks(s.lpq, nocc)
    w0 = O.bse_w0(s.lpq, s.mo_energy, nocc)
    kd, _ = _direct_kernel(df_ij, df_ab, w0, nocc, nvir)
    assert np.abs(kd - kd.T).max() < 1e-13 * np.abs(kd).max()


def test_gemm_output_layout_is_the_factored_yd_layout():
    """The GEMM writes row (i,a), column v at (i nvir + a) nvec + v, which is
    the factored form's Yd[i][(a,v)] = Yd[i][a nvec + v]."""
    nocc, nvir, nvec = 3, 5, 4
    yd = np.arange(nocc * nvir * nvec, dtype=float).reshape(nocc, nvir * nvec)
    rows = yd.reshape(nocc * nvir, nvec)   # K^d X as [(i,a)][v] with ld = nvec
    for i in range(nocc):
        for a in range(nvir):
            for v in range(nvec):
                assert rows[i * nvir + a, v] == yd[i, a * nvec + v]
