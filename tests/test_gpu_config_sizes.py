"""GPU parity at the benchmark configurations' own sizes (slow: the oracle
needs tens of seconds per case on the host cores).

* nmo 300 / naux 1000 / nw 32 evGW (the precision workload): one FP64
  iteration of the GPU driver equals the oracle's (its frequency loop on a
  thread pool) to 1e-8 Ha, the plain path's bar.
* the three largest members of the 64-system batch (nmo ~400, naux ~1400,
  24-point grid, HOMO-2..LUMO+2, linearized CD): FP64 QP energies equal the
  oracle's to 1e-8 Ha.
* the BSE-TDA matrix of dimension 26 400 (naux 1800): the FP64 matvec on 4
  vectors equals the oracle's factored form to 1e-12 relative.
"""
import os

import numpy as np
import pytest

from oracle import qx_oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def cores():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


def test_evgw_nmo300_one_fp64_iteration():
    import quasix_b200 as q
    from quasix_b200.synth import make_system
    s = make_system(40, 260, 1000, seed=1, pi_norm=4.0)
    mi = np.ascontiguousarray(s.lpq[:, :, :40].transpose(1, 2, 0))
    vxc = np.diag(O.compute_exchange(mi)).copy()
    got = q.run_evgw_blocks(s.mo_energy, s.lpq, vxc, 40, nfreq=32, precision="fp64", fixed_iterations=1,
                            max_iterations=1)
    cfg = O.EvGWConfig(max_iterations=1, energy_tolerance=0.0, nfreq=32)
    w = min(32, cores())
    ref = O.run_evgw_blocks(s.mo_energy, mi, vxc, s.lpq, 40, cfg,
                            sigma_fn=lambda e: O.get_sigma_diag_threaded(e, s.lpq, range(300), 40, 32, 5.0, 0.5, w))
    assert np.abs(got["energies"][0] - ref["energies"][0]).max() < 1e-8


def largest_batch_members(k=3):
    from quasix_b200.synth import batch64_shapes
    shapes = batch64_shapes()
    return sorted(shapes, key=lambda t: t[1] + t[2], reverse=True)[:k]


@pytest.mark.parametrize("shape", largest_batch_members(), ids=lambda t: f"seed{t[0]}_nmo{t[1] + t[2]}")
def test_batch64_largest_member_linearized_cd(shape):
    import quasix_b200 as q
    from quasix_b200.synth import make_system
    seed, nocc, nvir, naux, pin = shape
    s = make_system(nocc, nvir, naux, seed=seed, pi_norm=pin)
    targets = list(range(nocc - 3, nocc + 3))
    sx = q.compute_exchange_diag(s.lpq, nocc)
    got = q.g0w0_cd(s.mo_energy, s.lpq, nocc, targets, nw=24, vxc=sx, qp_solver="linearized", precision="fp64")
    ref = O.g0w0_cd(s.mo_energy, s.lpq, nocc, targets, 24, vxc=sx, qp_solver="linearized")
    assert np.abs(got["qp_energies"] - ref["qp_energies"]).max() < 1e-8


def test_bse_dim26400_fp64_matvec():
    import quasix_b200 as q
    from quasix_b200.synth import bse_blocks, make_system
    s = make_system(60, 440, 1800, seed=11, pi_norm=5.0)
    nocc, nvir, naux = 60, 440, 1800
    dia, dij, dab = bse_blocks(s.lpq, nocc)
    w0 = q.bse.screened_w0(s.mo_energy, np.ascontiguousarray(s.lpq[:, :nocc, nocc:]))
    delta = (s.mo_energy[None, nocc:] - s.mo_energy[:nocc, None]).reshape(-1)
    k = q.BSETDAKernel(nocc, nvir, naux, delta, dia, dij, dab, w0, precision="fp64")
    x = np.random.default_rng(3).standard_normal((nocc * nvir, 4))
    got = k.apply_hamiltonian_batch(x)
    ref = O.bse_apply_tda(x, delta, dia, dij, dab, w0, nocc, nvir)
    k.close()
    assert np.abs(got - ref).max() < 1e-12 * np.abs(ref).max()
