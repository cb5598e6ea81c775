"""The standalone Newton QP solver (NewtonQPSolver, qp/newton_solver.rs:124-402)
on the device against the oracle's restatement, with the same Pade
evaluator.  The Pade coefficients are taken from the oracle's fit and handed to
both sides, so the two solves differ only in the rounding of the continued
fraction (the device divides by b conj(b), numpy scales first): QP energies
agree to 1e-9 Ha and the method and iteration counts match."""
import numpy as np
import pytest

from oracle import qx_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fit():
    import quasix_b200 as q
    from quasix_b200.synth import make_system
    s = make_system(6, 22, 96, seed=4, pi_norm=2.0)
    orbs = list(range(s.nmo))
    sig, om = q.get_sigma_diag(s.mo_energy, s.lpq, orbs, s.nocc, nw=32)
    coeff, ofit = O.ac_pade_thiele_diag(sig, om)
    mi = np.ascontiguousarray(s.lpq[:, :, : s.nocc].transpose(1, 2, 0))
    sx = np.diag(O.compute_exchange(mi)).copy()
    ef = 0.5 * (s.mo_energy[s.nocc - 1] + s.mo_energy[s.nocc])
    return s, coeff, ofit, sx, ef


def oracle_solve(s, coeff, ofit, sx, vxc, ef, guess, cfg):
    out = []
    for p in range(s.nmo):
        solver = O.NewtonQPSolver(s.mo_energy[p], sx[p], vxc[p], ef, cfg)
        f = lambda w, p=p: O.pade_thiele(w, ofit[p], coeff[:, p])
        try:
            out.append(solver.solve(f, guess[p]))
        except O.ConvergenceError:
            out.append(None)
    return out


CONFIGS = {
    "default": {},
    "central_difference": {"use_richardson": False},
    "short_newton_bisection": {"max_iterations": 2},
    "no_fallback": {"max_iterations": 2, "use_bisection_fallback": False},
    "damped": {"initial_damping": 0.5, "max_step": 0.2, "energy_tolerance": 1e-10},
}


@pytest.mark.parametrize("name", list(CONFIGS))
def test_newton_qp_solve_matches_oracle(fit, name):
    import quasix_b200 as q
    s, coeff, ofit, sx, ef = fit
    kw = CONFIGS[name]
    vxc = sx.copy()  # HF reference: the QP correction is Sigma_c alone
    guess = s.mo_energy + 0.01
    got = q.newton_qp_solve(coeff, ofit, s.mo_energy, sx, vxc, ef, guess, q.NewtonSolverConfig(**kw))
    ref = oracle_solve(s, coeff, ofit, sx, vxc, ef, guess, O.NewtonSolverConfig(**kw))
    methods = {"newton": 0, "bisection": 1}
    for p, r in enumerate(ref):
        if r is None:
            assert got["method"][p] == -1
            continue
        assert got["method"][p] == methods[r.method]
        assert got["iterations"][p] == r.iterations
        assert abs(got["qp_energy"][p] - r.qp_energy) < 1e-9
        assert abs(got["z_factor"][p] - r.z_factor) < 1e-7
        assert abs(got["sigma_c"][p] - r.sigma_c) < 1e-9
    if name == "short_newton_bisection":
        assert (got["method"] == 1).any()
    if name == "no_fallback":
        assert (got["method"] == -1).any()


def test_single_orbital_solver_and_errors(fit):
    import quasix_b200 as q
    s, coeff, ofit, sx, ef = fit
    p = s.nocc - 1
    solver = q.NewtonQPSolver(s.mo_energy[p], sx[p], sx[p], ef)
    r = solver.solve((ofit[p], coeff[:, p]), s.mo_energy[p])
    ref = O.NewtonQPSolver(s.mo_energy[p], sx[p], sx[p], ef, O.NewtonSolverConfig()).solve(
        lambda w: O.pade_thiele(w, ofit[p], coeff[:, p]), s.mo_energy[p])
    assert r.converged and r.method == ref.method and abs(r.qp_energy - ref.qp_energy) < 1e-9
    strict = q.NewtonQPSolver(s.mo_energy[p], sx[p], sx[p], ef,
                              q.NewtonSolverConfig(max_iterations=1, energy_tolerance=1e-300,
                                                   use_bisection_fallback=False))
    with pytest.raises(q.gw.ConvergenceError):
        strict.solve((ofit[p], coeff[:, p]), s.mo_energy[p] + 0.3)
    with pytest.raises(ValueError):
        q.newton_qp_solve(coeff, ofit[:, :-1], s.mo_energy, sx, sx, ef, s.mo_energy)
