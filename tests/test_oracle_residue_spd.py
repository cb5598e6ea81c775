"""The condition under which the grouped batch runs the split trailing update
on the residue matrices: for a real shift w below 0.9 of the smallest
transition |e_ia|, eps(w) = I - Pi(w) is SPD with eigenvalues in
[1, 1 + ||Pi(0)|| / 0.19] (checked on the CPU with the oracle's real-axis
response; above the smallest transition eps(w) is indefinite)."""
import numpy as np
import pytest

from oracle import qx_oracle as O
from quasix_b200.synth import make_system


@pytest.mark.parametrize("seed,pin", [(3, 1.5), (8, 6.0)])
def test_residue_eps_is_spd_below_the_smallest_transition(seed, pin):
    nocc, nvir, naux = 6, 22, 60
    s = make_system(nocc, nvir, naux, seed=seed, pi_norm=pin)
    lov = s.lpq[:, :nocc, nocc:]
    gap = s.mo_energy[nocc] - s.mo_energy[nocc - 1]
    pi0 = O.get_rho_response_real(0.0, s.mo_energy, lov)
    bound = 1.0 + np.linalg.norm(pi0, 2) / 0.19
    for w in np.linspace(0.0, 0.9 * gap, 7):
        ev = np.linalg.eigvalsh(np.eye(naux) - O.get_rho_response_real(w, s.mo_energy, lov))
        assert ev.min() >= 1.0 - 1e-12 and ev.max() <= bound * (1.0 + 1e-12), (w, ev.min(), ev.max())


def test_residue_eps_is_indefinite_above_the_smallest_transition():
    nocc, nvir, naux = 6, 22, 60
    s = make_system(nocc, nvir, naux, seed=3, pi_norm=4.0)
    lov = s.lpq[:, :nocc, nocc:]
    e_ia = np.sort((s.mo_energy[None, nocc:] - s.mo_energy[:nocc, None]).reshape(-1))
    w = 0.5 * (e_ia[0] + e_ia[1])  # just above the smallest transition
    ev = np.linalg.eigvalsh(np.eye(naux) - O.get_rho_response_real(w, s.mo_energy, lov))
    assert ev.min() < 0.0 < ev.max()
