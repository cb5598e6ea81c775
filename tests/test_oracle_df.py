"""The oracle's DF tensor build: J^-1/2 J J^-1/2 = I, the Rust ov-block
transform equals the ov block of the full build before the metric step, and
the metric step makes the RI reconstruction exact (sum_P B_pq^P B_rs^P equals
the fitted (pq|J^-1|rs)).  CPU only."""
import numpy as np

from oracle import qx_oracle as O


def system(seed=0, nao=14, nmo=12, naux=30):
    rng = np.random.default_rng(seed)
    j3 = rng.standard_normal((nao, nao, naux))
    j3 = j3 + j3.transpose(1, 0, 2)
    a = rng.standard_normal((naux, 2 * naux))
    metric = a @ a.T / naux + 0.1 * np.eye(naux)
    c = np.linalg.qr(rng.standard_normal((nao, nao)))[0][:, :nmo]
    return j3, metric, c


def test_metric_inverse_square_root():
    _, metric, _ = system()
    jm, jp = O.metric_inv_sqrt(metric)
    n = metric.shape[0]
    assert np.abs(jm @ metric @ jm - np.eye(n)).max() < 1e-12
    assert np.abs(jp @ jp - metric).max() < 1e-12 * np.abs(metric).max()


def test_ov_block_and_ri_reconstruction():
    j3, metric, c = system(1)
    nocc = 4
    ov = O.transform_mo_3center(j3, c[:, :nocc], c[:, nocc:])
    full = np.einsum("up,uvP,vq->pqP", c, j3, c)
    assert np.allclose(ov, full[:nocc, nocc:].reshape(-1, j3.shape[2]), atol=1e-12)
    lpq, _ = O.build_lpq(j3, c, metric)
    # sum_P L[P,p,q] L[P,r,s] = (pq|Q) J^-1 (Q|rs)
    lhs = np.einsum("Ppq,Prs->pqrs", lpq, lpq)
    rhs = np.einsum("pqQ,QR,rsR->pqrs", full, np.linalg.inv(metric), full)
    assert np.abs(lhs - rhs).max() < 1e-10 * np.abs(rhs).max()
