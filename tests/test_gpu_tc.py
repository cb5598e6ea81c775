"""tcgen05 BF16x3 form against the FP64 oracle.

Tolerances follow the split-operand error model: each product carries a
relative error of ~2^-17 of |a||b|, so Pi and Sigma_c agree with FP64 to
~1e-5 relative; QP energies to well under 1 meV (3.7e-5 Ha).
"""
import numpy as np
import pytest

from oracle import qx_oracle as O
from quasix_b200.synth import make_system

pytestmark = pytest.mark.gpu
HA_MEV = 27211.386


@pytest.fixture(scope="module")
def q():
    import quasix_b200
    return quasix_b200


@pytest.mark.parametrize("shape", [(5, 19, 84), (12, 61, 250), (20, 130, 520)])
def test_rho_response_bf16x3(q, shape):
    nocc, nvir, naux = shape
    s = make_system(nocc, nvir, naux, seed=4, pi_norm=3.0)
    lov = np.ascontiguousarray(s.lpq[:, :nocc, nocc:])
    freqs = np.array([0.0, 0.3, 5.0])
    got = q.get_rho_response_batch(freqs, s.mo_energy, lov, precision="bf16x3")
    for k, f in enumerate(freqs):
        ref = O.get_rho_response(f, s.mo_energy, lov)
        scale = np.abs(ref).max()
        assert np.abs(got[k] - ref).max() < 5e-5 * scale
        assert np.abs(got[k] - got[k].T).max() < 1e-12 * max(scale, 1.0)


@pytest.mark.parametrize("shape,nw,orbs", [((5, 19, 84), 16, None), ((12, 61, 250), 24, [0, 11, 12, 72]),
                                           ((20, 130, 520), 20, [19, 20])])
def test_sigma_diag_bf16x3(q, shape, nw, orbs):
    nocc, nvir, naux = shape
    s = make_system(nocc, nvir, naux, seed=5, pi_norm=3.0)
    orbs = list(range(s.nmo)) if orbs is None else orbs
    got, _ = q.get_sigma_diag(s.mo_energy, s.lpq, orbs, nocc, nw=nw, precision="bf16x3")
    ref, _ = O.get_sigma_diag(s.mo_energy, s.lpq, orbs, nocc, nw=nw)
    assert np.abs(got - ref).max() < 2e-5 * max(1.0, np.abs(ref).max())


def test_evgw_bf16x3_within_one_mev(q):
    s = make_system(12, 61, 250, seed=6, pi_norm=3.0)
    kw = dict(nfreq=32, fixed_iterations=3, max_iterations=3)
    a = q.run_evgw_blocks(s.mo_energy, s.lpq, np.zeros(s.nmo), s.nocc, precision="bf16x3", **kw)
    b = q.run_evgw_blocks(s.mo_energy, s.lpq, np.zeros(s.nmo), s.nocc, precision="fp64", **kw)
    assert np.abs(a["qp_energies"] - b["qp_energies"]).max() * HA_MEV < 1.0
