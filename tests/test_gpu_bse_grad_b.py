"""Gradient of the lowest BSE-TDA root with respect to the DF blocks and,
through the torch.autograd.Function, to mo_energy and lpq.

* GPU block gradients equal the oracle's Hellmann-Feynman restatement
  (oracle.qx_oracle.bse_root_grad_blocks) to 1e-10 relative (FP64);
* the autograd gradients equal central differences of the GPU forward path
  (Davidson to 1e-11) to 1e-5 relative, at 20 seeded coordinates of
  mo_energy and lpq (steps 1e-5 Ha and 1e-6).
"""
import numpy as np
import pytest

from oracle import qx_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def small():
    from quasix_b200.synth import make_system
    return make_system(6, 30, 90, seed=12, pi_norm=2.0)


def test_block_gradients_match_oracle():
    import quasix_b200 as q
    from quasix_b200.synth import bse_blocks
    s = small()
    nocc, nvir, naux = 6, 30, 90
    dia, dij, dab = bse_blocks(s.lpq, nocc)
    w0 = q.bse.screened_w0(s.mo_energy, np.ascontiguousarray(s.lpq[:, :nocc, nocc:]))
    delta = (s.mo_energy[None, nocc:] - s.mo_energy[:nocc, None]).reshape(-1)
    for prec in ("fp64", "fp16x3"):
        k = q.BSETDAKernel(nocc, nvir, naux, delta, dia, dij, dab, w0, precision=prec)
        r = k.solve_davidson_with_config(q.DavidsonConfig(2, 300, None, 1e-10))
        x = r["eigenvectors"][:, 0]
        for e in (None, s.mo_energy):
            ge, gia, gij, gab = k.root_gradient_blocks(x, mo_energy=e)
            ria, rij, rab = O.bse_root_grad_blocks(x, dia, dij, dab, w0, nocc, nvir, mo_energy=e)
            tol = 1e-10 if prec == "fp64" else 1e-5
            assert rel(gia, ria) < tol and rel(gij, rij) < tol and rel(gab, rab) < tol, (prec, e is None)
            assert rel(ge, O.bse_root_grad(x, dia, dij, dab, w0, nocc, nvir, mo_energy=e)) < tol
        k.close()


def test_autograd_matches_central_differences():
    import torch
    import quasix_b200 as q
    s = small()
    nocc = 6
    e = torch.tensor(s.mo_energy, dtype=torch.float64, device="cuda", requires_grad=True)
    lpq = torch.tensor(s.lpq, dtype=torch.float64, device="cuda", requires_grad=True)
    om = q.bse_lowest_root(e, lpq, nocc, tol=1e-11)
    ge, gl = torch.autograd.grad(om, (e, lpq))
    ge, gl = ge.cpu().numpy(), gl.cpu().numpy()
    assert np.allclose(gl, gl.transpose(0, 2, 1), atol=0)

    def f(ev, lv):
        with torch.no_grad():
            return float(q.bse_lowest_root(ev, lv, nocc, tol=1e-11))

    rng = np.random.default_rng(3)
    an, fd = [], []
    for p in rng.choice(s.nmo, 10, replace=False):
        d = torch.zeros_like(e)
        d[p] = 1e-5
        fd.append((f(e + d, lpq) - f(e - d, lpq)) / 2e-5)
        an.append(ge[p])
    mag = np.abs(gl)
    cand = np.argwhere(mag > 1e-2 * mag.max())
    for k in rng.choice(len(cand), 10, replace=False):
        P, a, b = (int(v) for v in cand[k])
        d = torch.zeros_like(lpq)
        d[P, a, b] += 1e-6
        if a != b:
            d[P, b, a] += 1e-6
        fd.append((f(e, lpq + d) - f(e, lpq - d)) / 2e-6)
        an.append(gl[P, a, b] * (2 if a != b else 1))
    an, fd = np.array(an), np.array(fd)
    assert np.abs(an - fd).max() < 1e-5 * np.abs(fd).max(), np.abs(an - fd).max() / np.abs(fd).max()
