"""DF-tensor and evGW-result files (the reference's HDF5 schema in .npz):
round trips, the reference's schema validation
(quasix_core/src/io/df_tensors.rs:381-468) and checksum detection.  CPU only."""
import io as _io
import json

import numpy as np
import pytest

from quasix_b200 import io as qio


def df_sample(naux=12, nao=5, nocc=2):
    rng = np.random.default_rng(0)
    a = rng.standard_normal((naux, naux))
    nvir = nao - nocc
    return qio.DFTensorsS24(a @ a.T, rng.standard_normal((naux, nao * (nao + 1) // 2)),
                            rng.standard_normal((nocc * nvir, naux)), rng.standard_normal((nocc * nocc, naux)),
                            qio.DFMetadata(naux=naux, nao=nao, nocc=nocc, nvir=nvir, auxbasis="def2-svp-jkfit",
                                           basis="sto-3g"))


def test_df_round_trip(tmp_path):
    d = df_sample()
    p = str(tmp_path / "df.npz")
    d.write(p)
    r = qio.DFTensorsS24.read(p)
    for a, b in ((d.metric_2c, r.metric_2c), (d.cderi_3c, r.cderi_3c), (d.ia_p, r.ia_p), (d.ij_p, r.ij_p)):
        assert np.array_equal(a, b)
    assert r.metadata.auxbasis == "def2-svp-jkfit" and r.metadata.version == "1.0" and r.metadata.timestamp


@pytest.mark.parametrize("breakage,msg", [
    (lambda d: setattr(d, "metric_2c", d.metric_2c[:-1]), "metric_2c shape"),
    (lambda d: d.metric_2c.__setitem__((0, 1), d.metric_2c[0, 1] + 1e-6), "not symmetric"),
    (lambda d: setattr(d, "cderi_3c", d.cderi_3c[:, :-1]), "cderi_3c shape"),
    (lambda d: setattr(d, "ia_p", d.ia_p[1:]), "ia_p shape"),
    (lambda d: setattr(d, "ij_p", d.ij_p[:, 1:]), "ij_p shape"),
    (lambda d: d.ia_p.__setitem__((0, 0), np.nan), "NaN"),
    (lambda d: setattr(d.metadata, "version", "2.0"), "schema version"),
])
def test_df_validation(tmp_path, breakage, msg):
    d = df_sample()
    breakage(d)
    with pytest.raises(ValueError, match=msg):
        d.write(str(tmp_path / "bad.npz"))


def test_checksum_detects_corruption(tmp_path):
    d = df_sample()
    p = str(tmp_path / "df.npz")
    d.write(p)
    with np.load(p) as z:
        files = {k: z[k].copy() for k in z.files}
    files["df_tensors/iaP"][0, 0] += 1.0
    with open(p, "wb") as f:
        np.savez(f, **files)
    with pytest.raises(ValueError, match="checksum"):
        qio.DFTensorsS24.read(p)


def test_unpack_cderi():
    nao, naux = 4, 3
    rng = np.random.default_rng(1)
    full = rng.standard_normal((nao, nao, naux))
    full = full + full.transpose(1, 0, 2)
    il, jl = np.tril_indices(nao)
    packed = full[il, jl, :].T
    assert np.array_equal(qio.unpack_cderi(packed, nao), full)


def test_evgw_results_round_trip(tmp_path):
    nmo, nocc = 6, 2
    rng = np.random.default_rng(2)
    hist = [dict(cycle=c + 1, qp_energies=rng.standard_normal(nmo), z_factors=rng.uniform(0.5, 1, nmo),
                 energy_change=0.1 / (c + 1), rms_change=0.05, damping_used=0.5, converged=c == 2) for c in range(3)]
    res = dict(qp_energies=np.sort(rng.standard_normal(nmo)), z_factors=rng.uniform(0.5, 1, nmo),
               sigma_x=rng.standard_normal(nmo), sigma_c_re=rng.standard_normal(nmo),
               sigma_c_im=rng.standard_normal(nmo), converged=True, n_cycles=3, final_error=1e-5,
               iteration_history=hist)
    p = str(tmp_path / "evgw.npz")
    qio.save_evgw_results(p, res, nocc, parameters=dict(conv_tol=1e-5, nfreq=32), total_time=1.5)
    r = qio.load_evgw_results(p)
    for k in ("qp_energies", "z_factors", "sigma_x", "sigma_c_re", "sigma_c_im"):
        assert np.array_equal(r[k], res[k])
    assert r["converged"] is True and r["n_cycles"] == 3
    assert len(r["iteration_history"]) == 3 and r["iteration_history"][1]["cycle"] == 2
    assert np.array_equal(r["iteration_history"][2]["qp_energies"], hist[2]["qp_energies"])
    assert abs(r["gap"] - (res["qp_energies"][2] - res["qp_energies"][1])) < 1e-15
    assert r["attrs"]["parameters/convergence"]["energy_tol"] == 1e-5
