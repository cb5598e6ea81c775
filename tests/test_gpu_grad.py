"""Adjoint of the CD QP roots on the GPU (qx_g0w0_cd_grad).

* Against the oracle's adjoint on the small system: same mathematics, FP64,
  agreement to 1e-10 relative.
* Against central finite differences of the GPU's own FP64 forward path on the
  differentiation workload: nocc 30, nvirt 170 (nmo 200), naux 700, seed 7,
  24-point grid, L = E_QP(HOMO) + E_QP(LUMO), steps 1e-5 Ha (energies) and
  1e-6 (tensor entries, symmetric pairs), 20 seeded coordinates.  Vxc is held
  fixed at values that put the unperturbed roots 0.05 Ha inside the gap, where
  Sigma^CD is smooth and Newton converges to |f| < 1e-13 (with Vxc =
  diag(Sigma_x) these synthetic roots are satellites with Z ~ 1e-4 and the
  damped Newton converges only linearly, so differences of them measure the
  iteration, not the derivative).
* Tolerance: 1e-5 relative in the max-norm over the sampled coordinates (the
  FP64 form also entrywise with a floor of 1e-3 of the largest entry); the
  split tcgen05 forms (P0 rebuilt in FP16X3 / BF16X3) to the same max-norm
  bound.
"""
import numpy as np
import pytest

from oracle import qx_oracle as O
from quasix_b200.synth import make_system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def q():
    import quasix_b200
    return quasix_b200


def _sx(s, nocc):
    return np.diag(O.compute_exchange(np.ascontiguousarray(s.lpq[:, :, :nocc].transpose(1, 2, 0))))


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_adjoint_matches_oracle_adjoint(q):
    s = make_system(5, 19, 84, seed=0, pi_norm=2.0)
    nocc, tg, nw = 5, [4, 5], 16
    vxc = _sx(s, nocc)
    r = q.g0w0_cd(s.mo_energy, s.lpq, nocc, tg, nw=nw, vxc=vxc, tol=1e-13, max_iter=100)
    lam = np.array([1.0, 0.7])
    ge, gl, z = q.g0w0_cd_grad(s.mo_energy, s.lpq, nocc, tg, r["qp_energies"], lam, nw=nw)
    oe, ol = O.g0w0_cd_grad(s.mo_energy, s.lpq, nocc, tg, r["qp_energies"], lam, nw)
    assert _rel(ge, oe) < 1e-10
    assert _rel(gl, ol) < 1e-10
    assert np.allclose(gl, gl.transpose(0, 2, 1), rtol=0, atol=0)


@pytest.fixture(scope="module")
def c3(q):
    import torch
    s = make_system(30, 170, 700, seed=7, pi_norm=2.0)
    nocc, tg, nw = 30, [29, 30], 24
    e_d = torch.from_numpy(s.mo_energy.copy()).cuda()
    l_d = torch.from_numpy(s.lpq.copy()).cuda()
    target_e = np.array([s.mo_energy[29] + 0.05, s.mo_energy[30] - 0.05])
    cs = q.cd_sigma(e_d, l_d, nocc, tg, target_e, nw=nw)
    vxc = np.asarray(q.compute_exchange_diag(l_d, nocc))
    vxc[tg] = cs["sigma_x"] + cs["sigma_c"] - (target_e - s.mo_energy[tg])
    v_d = torch.from_numpy(vxc).cuda()

    def loss(e, lpq, precision="fp64"):
        r = q.g0w0_cd(e, lpq, nocc, tg, nw=nw, vxc=v_d, tol=1e-13, max_iter=100, precision=precision)
        return float(r["qp_energies"].sum()), r

    _, r0 = loss(e_d, l_d)
    assert np.abs(r0["qp_energies"] - target_e).max() < 1e-10
    ge, gl, _ = q.g0w0_cd_grad(e_d, l_d, nocc, tg, r0["qp_energies"], [1.0, 1.0], nw=nw)
    ge, gl = ge.cpu().numpy(), gl.cpu().numpy()
    rng = np.random.default_rng(7)
    coords_e = [int(p) for p in rng.choice(200, 10, replace=False)]
    mag = np.abs(gl)
    cand = np.argwhere(mag > 1e-3 * mag.max())
    coords_b = [tuple(int(v) for v in cand[k]) for k in rng.choice(len(cand), 10, replace=False)]
    fd_e, fd_b = [], []
    h = 1e-5
    for p in coords_e:
        ep, em = e_d.clone(), e_d.clone()
        ep[p] += h
        em[p] -= h
        fd_e.append((loss(ep, l_d)[0] - loss(em, l_d)[0]) / (2 * h))
    h = 1e-6
    for (P, a, b) in coords_b:
        d = torch.zeros_like(l_d)
        d[P, a, b] += h
        if a != b:
            d[P, b, a] += h
        fd_b.append((loss(e_d, l_d + d)[0] - loss(e_d, l_d - d)[0]) / (2 * h))
    return dict(s=s, nocc=nocc, tg=tg, nw=nw, e=e_d, l=l_d, loss=loss, ge=ge, gl=gl, coords_e=coords_e,
                coords_b=coords_b, fd_e=np.array(fd_e), fd_b=np.array(fd_b))


def _sampled(c, ge, gl):
    an_e = np.array([ge[p] for p in c["coords_e"]])
    an_b = np.array([gl[P, a, b] * (2 if a != b else 1) for (P, a, b) in c["coords_b"]])
    return an_e, an_b


def test_adjoint_vs_central_differences_fp64(c3):
    an_e, an_b = _sampled(c3, c3["ge"], c3["gl"])
    for an, fd in ((an_e, c3["fd_e"]), (an_b, c3["fd_b"])):
        assert np.abs(an - fd).max() <= 1e-5 * np.abs(fd).max()
        floor = 1e-3 * np.abs(fd).max()
        assert (np.abs(an - fd) <= 1e-5 * np.maximum(np.abs(fd), floor)).all()


@pytest.mark.parametrize("precision", ["fp16x3", "bf16x3"])
def test_split_precision_adjoint_vs_central_differences(q, c3, precision):
    _, r = c3["loss"](c3["e"], c3["l"], precision)
    ge, gl, _ = q.g0w0_cd_grad(c3["e"], c3["l"], c3["nocc"], c3["tg"], r["qp_energies"], [1.0, 1.0],
                               nw=c3["nw"], precision=precision)
    an_e, an_b = _sampled(c3, ge.cpu().numpy(), gl.cpu().numpy())
    for an, fd in ((an_e, c3["fd_e"]), (an_b, c3["fd_b"])):
        assert np.abs(an - fd).max() <= 1e-5 * np.abs(fd).max()


def test_autograd_function_matches_direct_adjoint(q):
    import torch
    s = make_system(5, 19, 84, seed=0, pi_norm=2.0)
    nocc, tg, nw = 5, [4, 5], 16
    vxc = torch.from_numpy(_sx(s, nocc).copy()).cuda()
    e = torch.from_numpy(s.mo_energy.copy()).cuda().requires_grad_(True)
    lpq = torch.from_numpy(s.lpq.copy()).cuda().requires_grad_(True)
    qp = q.g0w0_cd_qp(e, lpq, nocc, tg, nw=nw, vxc=vxc)
    (qp[0] + 0.7 * qp[1]).backward()
    ge, gl, _ = q.g0w0_cd_grad(s.mo_energy, s.lpq, nocc, tg, qp.detach().cpu().numpy(), [1.0, 0.7], nw=nw)
    assert _rel(e.grad.cpu().numpy(), ge) < 1e-14
    assert _rel(lpq.grad.cpu().numpy(), gl) < 1e-14


def test_adjoint_rejects_bad_arguments(q):
    from quasix_b200._native import QxValueError
    s = make_system(5, 19, 84, seed=0, pi_norm=2.0)
    with pytest.raises(QxValueError, match="listed twice"):
        q.g0w0_cd_grad(s.mo_energy, s.lpq, 5, [4, 4], [-0.5, -0.5], [1.0, 1.0], nw=16)
    with pytest.raises(QxValueError, match="out of range"):
        q.g0w0_cd_grad(s.mo_energy, s.lpq, 5, [4, 99], [-0.5, 0.1], [1.0, 1.0], nw=16)
