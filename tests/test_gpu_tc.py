"""tcgen05 split-operand forms against the FP64 oracle.

Tolerances follow the error model: each product carries a relative error of
~2^-17 of |a||b| for bf16 hi/lo pairs and ~2^-22 for scaled fp16 pairs, so Pi
and Sigma_c agree with FP64 to ~1e-5 (BF16X3) or ~1e-6 (FP16X3) relative.
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


# Pi: split rounding plus the per-k-block FP64 drain of the accumulator
# (measured ~1e-6 relative for both forms at K up to 16384).  Sigma_c: the pair
# contraction accumulates a whole N tile in FP32 (measured ~3e-6 relative).
TOL = {"bf16x3": 5e-6, "fp16x3": 3e-6}
TOL_SIGMA = {"bf16x3": 2e-5, "fp16x3": 1e-5}


@pytest.fixture
def p0_form(q):
    """Set the split P0 form of the default context for one test."""
    from quasix_b200 import _native
    ctx = _native.context(0)

    def use(form):
        ctx.set_p0_form(form)

    yield use
    ctx.set_p0_form("auto")


@pytest.fixture
def contraction_form(q):
    """Set the split pair-contraction form of the default context for one test."""
    from quasix_b200 import _native
    ctx = _native.context(0)

    def use(form):
        ctx.set_contraction_form(form)

    yield use
    ctx.set_contraction_form("auto")


@pytest.mark.parametrize("form", ["materialised", "pair", "converter"])
@pytest.mark.parametrize("prec", ["bf16x3", "fp16x3"])
@pytest.mark.parametrize("shape", [(5, 19, 84), (12, 61, 250), (20, 130, 520)])
def test_rho_response_tc(q, p0_form, shape, prec, form):
    """The forms of the split P0: the chi-scaled operand materialised (tiles on
    one CTA, or two tiles of a column on a CTA pair: with 1, 2 and 5 tile rows
    every column count, even and odd, occurs), or built in shared memory by
    the converter warps (chi applied while staged)."""
    nocc, nvir, naux = shape
    s = make_system(nocc, nvir, naux, seed=4, pi_norm=3.0)
    lov = np.ascontiguousarray(s.lpq[:, :nocc, nocc:])
    freqs = np.array([0.0, 0.3, 5.0])
    p0_form(form)
    got = q.get_rho_response_batch(freqs, s.mo_energy, lov, precision=prec)
    for k, f in enumerate(freqs):
        ref = O.get_rho_response(f, s.mo_energy, lov)
        scale = np.abs(ref).max()
        assert np.abs(got[k] - ref).max() < TOL[prec] * scale
        assert np.abs(got[k] - got[k].T).max() < 1e-12 * max(scale, 1.0)


@pytest.mark.parametrize("cform", ["single", "pair"])
@pytest.mark.parametrize("prec", ["bf16x3", "fp16x3"])
@pytest.mark.parametrize("shape,nw,orbs", [((5, 19, 84), 16, None), ((12, 61, 250), 24, [0, 11, 12, 72]),
                                           ((20, 130, 520), 20, [19, 20])])
def test_sigma_diag_tc(q, contraction_form, shape, nw, orbs, prec, cform):
    """The pair contraction on one CTA per pair block, or on CTA pairs (the
    pair counts give odd and even numbers of 128-row pair blocks)."""
    contraction_form(cform)
    nocc, nvir, naux = shape
    s = make_system(nocc, nvir, naux, seed=5, pi_norm=3.0)
    orbs = list(range(s.nmo)) if orbs is None else orbs
    got, _ = q.get_sigma_diag(s.mo_energy, s.lpq, orbs, nocc, nw=nw, precision=prec)
    ref, _ = O.get_sigma_diag(s.mo_energy, s.lpq, orbs, nocc, nw=nw)
    assert np.abs(got - ref).max() < TOL_SIGMA[prec] * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("form", ["materialised", "pair", "converter"])
@pytest.mark.parametrize("prec", ["bf16x3", "fp16x3"])
def test_evgw_tc_within_one_mev(q, p0_form, prec, form):
    s = make_system(12, 61, 250, seed=6, pi_norm=3.0)
    kw = dict(nfreq=32, fixed_iterations=3, max_iterations=3)
    p0_form(form)
    a = q.run_evgw_blocks(s.mo_energy, s.lpq, np.zeros(s.nmo), s.nocc, precision=prec, **kw)
    b = q.run_evgw_blocks(s.mo_energy, s.lpq, np.zeros(s.nmo), s.nocc, precision="fp64", **kw)
    assert np.abs(a["qp_energies"] - b["qp_energies"]).max() * HA_MEV < 1.0
