"""DF tensor build on the GPU against the oracle (FP64 DMMA GEMMs and the
Denman-Beavers J^-1/2: 1e-12 relative; for a metric of condition number
kappa both J^-1/2's are good to ~kappa 1e-16 only, so there 1e-15 kappa)."""
import numpy as np
import pytest

from oracle import qx_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def system(seed, nao, nmo, naux, cond=1e3):
    rng = np.random.default_rng(seed)
    j3 = rng.standard_normal((nao, nao, naux)) * 0.1
    j3 = j3 + j3.transpose(1, 0, 2)
    q = np.linalg.qr(rng.standard_normal((naux, naux)))[0]
    lam = np.geomspace(1.0, 1.0 / cond, naux) * 5.0
    metric = (q * lam) @ q.T
    metric = (metric + metric.T) / 2
    c = np.linalg.qr(rng.standard_normal((nao, nao)))[0][:, :nmo]
    return j3, metric, c


def test_transform_mo_3center():
    from quasix_b200 import df
    j3, _, c = system(0, 61, 57, 190)
    nocc = 9
    got = df.transform_mo_3center(j3, c[:, :nocc], c[:, nocc:])
    assert rel(got, O.transform_mo_3center(j3, c[:, :nocc], c[:, nocc:])) < 1e-12


@pytest.mark.parametrize("cond", [1e2, 1e6])
def test_metric_inv_sqrt(cond):
    from quasix_b200 import df
    _, metric, _ = system(1, 4, 4, 301, cond)
    jm, jp = df.metric_inv_sqrt(metric)
    rm, rp = O.metric_inv_sqrt(metric)
    assert rel(jm, rm) < max(1e-12, 1e-15 * cond) and rel(jp, rp) < max(1e-12, 1e-15 * cond)


def test_metric_below_threshold_is_rejected():
    from quasix_b200 import df
    from quasix_b200._native import QxError
    _, metric, _ = system(2, 4, 4, 64, cond=1e13)
    with pytest.raises(QxError, match="thresh_df"):
        df.metric_inv_sqrt(metric)


@pytest.mark.parametrize("nao,nmo,naux", [(40, 40, 110), (93, 88, 250)])
def test_build_lpq_matches_oracle(nao, nmo, naux):
    from quasix_b200 import df
    j3, metric, c = system(nao, nao, nmo, naux)
    lpq, chol = df.build_lpq(j3, c, metric=metric)
    ref, rchol = O.build_lpq(j3, c, metric)
    assert rel(lpq, ref) < 1e-12 and rel(chol, rchol) < 1e-12
    jm, _ = O.metric_inv_sqrt(metric)
    lpq2, _ = df.build_lpq(j3, c, metric_inv_sqrt=jm)
    assert rel(lpq2, ref) < 1e-12


def test_df_tensors_feed_the_gw_path():
    """build_df_tensors returns the reference's flattened blocks
    (evgw.py:1085-1100), cut from the same lpq."""
    from quasix_b200 import df
    j3, metric, c = system(5, 30, 28, 90)
    lpq, _ = df.build_lpq(j3, c, metric=metric)
    occ = np.zeros(28)
    occ[:5] = 2.0
    iaP, miP, abP, chol = df.build_df_tensors(j3, c, occ, metric)
    assert np.array_equal(iaP, np.ascontiguousarray(lpq[:, :5, 5:].transpose(1, 2, 0)).reshape(5 * 23, 90))
    assert np.array_equal(miP, np.ascontiguousarray(lpq[:, :, :5].transpose(1, 2, 0)).reshape(28 * 5, 90))
    assert abP.shape == (23 * 23, 90) and chol.shape == (90, 90)
