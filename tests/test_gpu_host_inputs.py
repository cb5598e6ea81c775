"""Host-resident lpq on the evGW entry point (qx_evgw).

Page-locked host memory is read in place by the setup gathers (only the pairs
p <= q cross the host link), pageable memory is copied in full, device memory
is used as it is.  The three must give the same bits.  With every orbital a
target, B_ov is transposed out of the gathered pair tensor and the exchange
diagonal is summed from it; both are checked against the direct forms.
"""
import numpy as np
import pytest

from oracle import qx_oracle as O
from quasix_b200.synth import make_system

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["fp64", "fp16x3"])
def test_evgw_lpq_device_pinned_pageable_identical(prec):
    import torch
    import quasix_b200 as q
    s = make_system(10, 50, 200, seed=11, pi_norm=3.0)
    vx = np.zeros(s.nmo)
    kw = dict(nfreq=16, fixed_iterations=2, max_iterations=2, precision=prec)
    on_dev = q.run_evgw_blocks(s.mo_energy, torch.from_numpy(s.lpq).cuda(), vx, s.nocc, **kw)
    pinned_t = torch.from_numpy(s.lpq).pin_memory()
    assert pinned_t.is_pinned()
    pinned = q.run_evgw_blocks(s.mo_energy, pinned_t, vx, s.nocc, **kw)
    pinned_np = q.run_evgw_blocks(s.mo_energy, pinned_t.numpy(), vx, s.nocc, **kw)
    pageable = q.run_evgw_blocks(s.mo_energy, np.array(s.lpq, copy=True), vx, s.nocc, **kw)
    for r in (pinned, pinned_np, pageable):
        for k in ("qp_energies", "z_factors", "sigma_x", "sigma_c"):
            assert np.array_equal(r[k], on_dev[k]), k


def test_exchange_from_pairs_matches_direct_and_oracle():
    """Sigma_x of the evGW entry point (summed from the pair tensor) against
    the direct exchange kernel and the oracle."""
    import quasix_b200 as q
    s = make_system(9, 41, 170, seed=12, pi_norm=2.0)
    r = q.run_evgw_blocks(s.mo_energy, s.lpq, np.zeros(s.nmo), s.nocc, nfreq=8, fixed_iterations=1,
                          max_iterations=1, precision="fp64")
    direct = np.asarray(q.compute_exchange_diag(s.lpq, s.nocc))
    ref = -np.einsum("rpi,rpi->p", s.lpq[:, :, :s.nocc], s.lpq[:, :, :s.nocc])
    scale = np.abs(ref).max()
    assert np.abs(r["sigma_x"] - direct).max() < 1e-13 * scale
    assert np.abs(r["sigma_x"] - ref).max() < 1e-13 * scale


def test_sigma_all_orbitals_pinned_matches_oracle():
    """get_sigma_diag over every orbital (B_ov from the pair tensor) from
    page-locked host lpq, against the oracle."""
    import torch
    import quasix_b200 as q
    s = make_system(6, 30, 120, seed=13, pi_norm=3.0)
    orbs = list(range(s.nmo))
    pinned_t = torch.from_numpy(s.lpq).pin_memory()
    got, _ = q.get_sigma_diag(s.mo_energy, pinned_t.numpy(), orbs, s.nocc, nw=12, precision="fp64")
    ref, _ = O.get_sigma_diag(s.mo_energy, s.lpq, orbs, s.nocc, nw=12)
    assert np.abs(got - ref).max() < 1e-10 * max(1.0, np.abs(ref).max())


def test_sigma_subset_pinned_matches_device():
    """get_sigma_diag over a few targets (B_ov gathered from lpq itself, in
    place over the host link) from page-locked host lpq: the same bits as from
    device lpq."""
    import torch
    import quasix_b200 as q
    s = make_system(7, 33, 140, seed=14, pi_norm=3.0)
    orbs = [0, 5, 6, 7, 20]
    pinned_t = torch.from_numpy(s.lpq).pin_memory()
    for prec in ("fp64", "fp16x3"):
        a, _ = q.get_sigma_diag(s.mo_energy, pinned_t.numpy(), orbs, s.nocc, nw=12, precision=prec)
        b, _ = q.get_sigma_diag(s.mo_energy, torch.from_numpy(s.lpq).cuda(), orbs, s.nocc, nw=12, precision=prec)
        assert np.array_equal(a, b), prec
