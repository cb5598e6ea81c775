"""The oracle's adjoint of the CD QP roots against central finite differences
of the oracle's own forward path (no GPU).  Small system: nocc 5, nvirt 19,
naux 84, seed 0, 16-point grid, HOMO and LUMO, Vxc = diag(Sigma_x) held fixed."""
import numpy as np

from oracle import qx_oracle as O
from quasix_b200.synth import make_system


def test_oracle_cd_adjoint_matches_central_differences():
    s = make_system(5, 19, 84, seed=0, pi_norm=2.0)
    nocc, tg, nw = 5, [4, 5], 16
    vxc = np.diag(O.compute_exchange(np.ascontiguousarray(s.lpq[:, :, :nocc].transpose(1, 2, 0))))
    lam = np.array([1.0, 1.0])

    def loss(e, lpq):
        r = O.g0w0_cd(e, lpq, nocc, tg, nw, vxc=vxc, tol=1e-13, max_iter=100)
        return float(lam @ r["qp_energies"]), r

    _, r0 = loss(s.mo_energy, s.lpq)
    assert (r0["iterations"] < 100).all()
    ge, gl = O.g0w0_cd_grad(s.mo_energy, s.lpq, nocc, tg, r0["qp_energies"], lam, nw)
    assert np.allclose(gl, gl.transpose(0, 2, 1))
    h = 1e-5
    for p in [0, 3, 4, 5, 9, 20]:
        ep, em = s.mo_energy.copy(), s.mo_energy.copy()
        ep[p] += h
        em[p] -= h
        fd = (loss(ep, s.lpq)[0] - loss(em, s.lpq)[0]) / (2 * h)
        assert abs(fd - ge[p]) <= 1e-6 * max(abs(fd), 1e-3), (p, fd, ge[p])
    h = 1e-6
    # target rows, the ov block, Sigma_x entries and a diagonal element
    for (P, a, b) in [(3, 4, 9), (10, 5, 2), (20, 1, 7), (50, 4, 4), (60, 2, 4), (11, 3, 15)]:
        d = np.zeros_like(s.lpq)
        d[P, a, b] += h
        if a != b:
            d[P, b, a] += h
        fd = (loss(s.mo_energy, s.lpq + d)[0] - loss(s.mo_energy, s.lpq - d)[0]) / (2 * h)
        an = gl[P, a, b] * (2 if a != b else 1)
        assert abs(fd - an) <= 1e-5 * max(abs(fd), 1e-3), ((P, a, b), fd, an)
