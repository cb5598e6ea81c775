"""lpq from stored Cholesky vectors on the GPU equals C^T L_P C (1e-12)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_lpq_from_cderi(tmp_path):
    from quasix_b200 import io as qio
    rng = np.random.default_rng(4)
    nao, nmo, naux, nocc = 17, 15, 40, 4
    full = rng.standard_normal((nao, nao, naux)) * 0.1
    full = full + full.transpose(1, 0, 2)
    il, jl = np.tril_indices(nao)
    a = rng.standard_normal((naux, naux))
    d = qio.DFTensorsS24(a @ a.T, full[il, jl, :].T.copy(), np.zeros((nocc * (nao - nocc), naux)),
                         np.zeros((nocc * nocc, naux)), qio.DFMetadata(naux, nao, nocc, nao - nocc))
    p = str(tmp_path / "df.npz")
    d.write(p)
    c = np.linalg.qr(rng.standard_normal((nao, nao)))[0][:, :nmo]
    lpq = qio.lpq_from_cderi(qio.DFTensorsS24.read(p), c)
    ref = np.einsum("up,uvP,vq->Ppq", c, full, c)
    assert np.abs(lpq - ref).max() < 1e-12 * np.abs(ref).max()
