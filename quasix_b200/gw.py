"""GW entry points with the reference's Python/Rust API shapes, on the GPU.

Every function here calls libqxgpu through the C ABI; none has a CPU fallback.
Reference interfaces (QuasiX, by path within the project):

* ``get_scaled_legendre_roots``  quasix_core/src/selfenergy/correlation_ac.rs:94-114
* ``get_rho_response`` / ``compute_polarizability_p0``
                                 correlation_ac.rs:184-211, dielectric/polarizability.rs:169-275
* ``compute_epsilon_inverse``    correlation_ac.rs:377-401 (quasix/src/lib.rs:1694)
* ``compute_screened_interaction``  dielectric/screening.rs:164-236
* ``get_sigma_diag``             correlation_ac.rs:241-449
* ``ac_pade_thiele_diag`` / ``pade_thiele``  correlation_ac.rs:470-654
* ``compute_exchange_diag``      quasix_core/src/qp/evgw.rs:1167-1193
* ``NewtonQPSolver`` / ``newton_qp_solve``  quasix_core/src/qp/newton_solver.rs:52-402
* ``evgw`` / ``run_evgw``        quasix/src/evgw.rs:22-677
* ``g0w0_cd``                    contour deformation (imaginary-axis term of
                                 selfenergy/correlation_pyscf_cd.rs:164-259 plus residues)
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, fields
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _native as N


def _ctx(device: int = 0, *arrays) -> N.Context:
    """Context for ``device``; device tensors among ``arrays`` are made ready
    first (their producer may still be running on the framework's stream)."""
    for a in arrays:
        if hasattr(a, "is_cuda") and a.is_cuda:
            import torch
            torch.cuda.current_stream(a.device).synchronize()
    return N.context(device)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _prec(precision) -> int:
    if isinstance(precision, int):
        return precision
    try:
        return N.PREC[precision.lower()]
    except KeyError:
        raise ValueError(f"precision must be one of {list(N.PREC)}") from None


def get_scaled_legendre_roots(nw: int, x0: float = 0.5):
    lib = N.load()
    f = np.zeros(nw)
    w = np.zeros(nw)
    st = lib.qx_get_scaled_legendre_roots(int(nw), float(x0), N.ptr(f), N.ptr(w))
    if st != 0:
        raise N.QxValueError(st, "get_scaled_legendre_roots")
    return f, w


def get_rho_response_batch(freqs, mo_energy, lpq_ov, precision="fp64", device: int = 0) -> np.ndarray:
    """Pi(iw) for many imaginary frequencies: [nfreq, naux, naux]."""
    ctx = _ctx(device)
    freqs = _f64(np.atleast_1d(freqs))
    mo_energy = _f64(mo_energy)
    lpq_ov = _f64(lpq_ov)
    naux, nocc, nvir = lpq_ov.shape
    out = np.zeros((freqs.shape[0], naux, naux))
    ctx.check(ctx.lib.qx_get_rho_response(ctx.handle, freqs.shape[0], N.ptr(freqs), N.ptr(mo_energy),
                                          N.ptr(lpq_ov), naux, nocc, nvir, _prec(precision), N.ptr(out)))
    return out


def get_rho_response(omega: float, mo_energy, lpq_ov, precision="fp64", device: int = 0) -> np.ndarray:
    """Pi(iw) = 4 (L_ov chi) L_ov^T for one frequency (lpq_ov [naux, nocc, nvir])."""
    return get_rho_response_batch([omega], mo_energy, lpq_ov, precision, device)[0]


def compute_polarizability_p0(ia_P, mo_energy, mo_occ, freqs, device: int = 0) -> np.ndarray:
    """S3-2 binding: ia_P [nocc, nvir, naux] -> P0 [nfreq, naux, naux]."""
    ia_P = _f64(ia_P)
    lpq_ov = np.ascontiguousarray(ia_P.transpose(2, 0, 1))
    return get_rho_response_batch(freqs, mo_energy, lpq_ov, device=device)


def compute_epsilon_inverse_minus_identity(pi, device: int = 0) -> np.ndarray:
    """Wc = (I - Pi)^-1 - I for [nfreq, naux, naux] (or one [naux, naux])."""
    ctx = _ctx(device)
    pi = _f64(pi)
    single = pi.ndim == 2
    p = pi[None] if single else pi
    out = np.zeros_like(p)
    ctx.check(ctx.lib.qx_screened_interaction(ctx.handle, p.shape[0], p.shape[1], N.ptr(np.ascontiguousarray(p)),
                                              N.ptr(out)))
    return out[0] if single else out


def compute_screened_interaction(p0, v_aux, freqs=None, device: int = 0) -> np.ndarray:
    """W(w) = v^1/2 (I - v^1/2 P0(w) v^1/2)^-1 v^1/2 for P0 [nfreq, naux, naux]
    (or one [naux, naux]) and the metric v_aux, with the symmetric square root
    of v_aux (dielectric/screening.rs:164-236).  ``freqs`` is accepted for the
    reference's signature and, as there, not used."""
    ctx = _ctx(device)
    p0 = _f64(p0)
    v = np.ascontiguousarray(_f64(v_aux))
    single = p0.ndim == 2
    p = np.ascontiguousarray(p0[None] if single else p0)
    if v.ndim != 2 or v.shape[0] != v.shape[1]:
        raise ValueError(f"v_aux must be square, got {v.shape}")
    if p.ndim != 3 or p.shape[1] != v.shape[0] or p.shape[2] != v.shape[0]:
        raise ValueError(f"P0 dimension mismatch: expected [freq, {v.shape[0]}, {v.shape[0]}], got {p0.shape}")
    out = np.zeros_like(p)
    ctx.check(ctx.lib.qx_compute_screened_interaction(ctx.handle, p.shape[0], p.shape[1], N.ptr(p), N.ptr(v),
                                                      N.ptr(out)))
    return out[0] if single else out


def get_sigma_diag(mo_energy, lpq, orbs: Sequence[int], nocc: int, nw: int = 100, iw_cutoff: float = 5.0,
                   x0: float = 0.5, precision="fp64", device: int = 0):
    """Sigma_c(iw) [norbs, nw_sigma] and the omega grid, both complex."""
    ctx = _ctx(device, lpq)
    lpq_is_dev = hasattr(lpq, "data_ptr")
    lpq_a = lpq if lpq_is_dev else _f64(lpq)
    naux, nmo, nmo2 = tuple(lpq_a.shape)
    if nmo != nmo2:
        raise N.QxValueError(2, f"Lpq not square in MO dimensions: {nmo} x {nmo2}")
    orbs_a = np.ascontiguousarray(np.asarray(orbs, dtype=np.int32))
    e = _f64(mo_energy)
    nmax = nw + 1
    sig = np.zeros((len(orbs_a), nmax), dtype=np.complex128)
    om = np.zeros((len(orbs_a), nmax), dtype=np.complex128)
    nws = C.c_int(0)
    ctx.check(ctx.lib.qx_get_sigma_diag(ctx.handle, N.ptr(e), N.ptr(lpq_a), N.ptr(orbs_a), len(orbs_a), nmo,
                                        int(nocc), naux, int(nw), float(iw_cutoff), float(x0), _prec(precision),
                                        N.ptr(sig), N.ptr(om), nmax, C.byref(nws)))
    k = nws.value
    return np.ascontiguousarray(sig[:, :k]), np.ascontiguousarray(om[:, :k])


def ac_pade_thiele_diag(sigma, omega, npade: Optional[int] = None, device: int = 0):
    """(coeff [nfit, norbs], omega_fit [norbs, nfit]) complex."""
    ctx = _ctx(device)
    sigma = np.ascontiguousarray(sigma, dtype=np.complex128)
    omega = np.ascontiguousarray(omega, dtype=np.complex128)
    norbs, nws = sigma.shape
    nmax = nws
    coeff = np.zeros((nmax, norbs), dtype=np.complex128)
    ofit = np.zeros((norbs, nmax), dtype=np.complex128)
    nfit = C.c_int(0)
    ctx.check(ctx.lib.qx_ac_pade_thiele_diag(ctx.handle, norbs, nws, N.ptr(sigma), N.ptr(omega),
                                             -1 if npade is None else int(npade), N.ptr(coeff), N.ptr(ofit), nmax,
                                             C.byref(nfit)))
    k = nfit.value
    # coeff was written with row stride norbs for the first k rows.
    c = np.ascontiguousarray(coeff.reshape(-1)[: k * norbs].reshape(k, norbs))
    o = np.ascontiguousarray(ofit.reshape(-1)[: norbs * k].reshape(norbs, k))
    return c, o


def pade_thiele(omega, zn, coeff, device: int = 0):
    """Evaluate the continued fraction of one orbital at real omega (scalar or
    array) on the device."""
    ctx = _ctx(device)
    zn = np.ascontiguousarray(zn, dtype=np.complex128)
    coeff = np.ascontiguousarray(coeff, dtype=np.complex128)
    w = _f64(np.atleast_1d(omega))
    out = np.zeros(w.shape[0], dtype=np.complex128)
    ctx.check(ctx.lib.qx_pade_thiele(ctx.handle, coeff.shape[0], N.ptr(zn), N.ptr(coeff), w.shape[0], N.ptr(w),
                                     N.ptr(out)))
    return out[0] if np.ndim(omega) == 0 else out


@dataclass
class NewtonSolverConfig:
    """NewtonSolverConfig (qp/newton_solver.rs:52-103), same fields and
    defaults (``verbose`` has no counterpart: the solve runs on the device)."""
    max_iterations: int = 50
    energy_tolerance: float = 1e-8
    initial_damping: float = 1.0
    min_damping: float = 0.1
    max_damping: float = 1.0
    max_step: float = 1.0
    derivative_delta: float = 1e-6
    use_richardson: bool = True
    z_min: float = 0.1
    z_max: float = 0.999
    use_bisection_fallback: bool = True
    max_bisection_iterations: int = 30

    def native(self) -> N.NewtonConfig:
        return N.NewtonConfig(**{f.name: (int(v) if isinstance(v, bool) else v)
                                 for f in fields(self) for v in [getattr(self, f.name)]})


@dataclass
class NewtonSolverResult:
    """NewtonSolverResult (qp/newton_solver.rs:105-122)."""
    qp_energy: float
    residual: float
    iterations: int
    converged: bool
    sigma_c: complex
    z_factor: float
    method: str


class ConvergenceError(N.QxError):
    """The reference's QuasixError::ConvergenceError for one QP equation."""

    def __init__(self, message: str):
        super().__init__(4, message)


_METHOD = {0: "newton", 1: "bisection", -1: "none"}


def newton_qp_solve(coeff, omega_fit, epsilon_hf, sigma_x, vxc, fermi_level: float, initial_guess,
                    config: Optional[NewtonSolverConfig] = None, device: int = 0) -> Dict[str, np.ndarray]:
    """Solve E = eps + Sigma_x + Re Sigma_c(E - ef) - Vxc for every orbital at
    once, one device thread each, with Sigma_c the Pade continuation given by
    ``coeff`` [nfit, norbs] and ``omega_fit`` [norbs, nfit] (the output of
    ``ac_pade_thiele_diag``).  Returns arrays ``qp_energy``, ``residual``,
    ``iterations``, ``method`` (0 Newton, 1 bisection, -1 not converged),
    ``converged``, ``sigma_c`` and ``z_factor``."""
    cfg = (config or NewtonSolverConfig()).native()
    ctx = _ctx(device)
    coeff = np.ascontiguousarray(coeff, dtype=np.complex128)
    ofit = np.ascontiguousarray(omega_fit, dtype=np.complex128)
    if coeff.ndim != 2 or ofit.shape != (coeff.shape[1], coeff.shape[0]):
        raise ValueError(f"coeff [nfit, norbs] and omega_fit [norbs, nfit] disagree: {coeff.shape}, {ofit.shape}")
    nfit, norbs = coeff.shape
    vec = [np.ascontiguousarray(np.broadcast_to(_f64(x), (norbs,))) for x in (epsilon_hf, sigma_x, vxc,
                                                                               initial_guess)]
    qp, res, z = np.zeros(norbs), np.zeros(norbs), np.zeros(norbs)
    sc = np.zeros(norbs, dtype=np.complex128)
    its, meth = np.zeros(norbs, dtype=np.int32), np.zeros(norbs, dtype=np.int32)
    ctx.check(ctx.lib.qx_newton_qp_solve(ctx.handle, C.byref(cfg), norbs, nfit, N.ptr(coeff), N.ptr(ofit),
                                         *[N.ptr(v) for v in vec[:3]], float(fermi_level), N.ptr(vec[3]),
                                         N.ptr(qp), N.ptr(res), N.ptr(its), N.ptr(meth), N.ptr(sc), N.ptr(z)))
    return {"qp_energy": qp, "residual": res, "iterations": its, "method": meth, "converged": meth >= 0,
            "sigma_c": sc, "z_factor": z}


class NewtonQPSolver:
    """NewtonQPSolver (qp/newton_solver.rs:124-402) for one orbital.  The
    reference's evaluator is any closure Sigma_c(w); on the device it is the
    Pade continuation of that orbital, passed to ``solve`` as ``(zn, coeff)``
    (complex [nfit] each, one column of ``ac_pade_thiele_diag``'s output)."""

    def __init__(self, epsilon_hf: float, sigma_x: float, vxc: float, fermi_level: float,
                 config: Optional[NewtonSolverConfig] = None, device: int = 0):
        self.epsilon_hf, self.sigma_x, self.vxc = float(epsilon_hf), float(sigma_x), float(vxc)
        self.fermi_level = float(fermi_level)
        self.config = config or NewtonSolverConfig()
        self.device = device

    def solve(self, pade, initial_guess: float) -> NewtonSolverResult:
        zn, coeff = (np.asarray(a, dtype=np.complex128).reshape(-1) for a in pade)
        r = newton_qp_solve(coeff[:, None], zn[None, :], self.epsilon_hf, self.sigma_x, self.vxc, self.fermi_level,
                            float(initial_guess), self.config, self.device)
        m = int(r["method"][0])
        if m < 0:
            what = "Bisection fallback" if self.config.use_bisection_fallback else "Newton-Raphson"
            raise ConvergenceError(f"{what} failed to converge (residual = {r['residual'][0]:.2e})")
        return NewtonSolverResult(float(r["qp_energy"][0]), float(r["residual"][0]), int(r["iterations"][0]), True,
                                  complex(r["sigma_c"][0]), float(r["z_factor"][0]), _METHOD[m])


def compute_exchange_diag(lpq, nocc: int, device: int = 0) -> np.ndarray:
    ctx = _ctx(device, lpq)
    lpq_a = lpq if hasattr(lpq, "data_ptr") else _f64(lpq)
    naux, nmo, _ = tuple(lpq_a.shape)
    out = np.zeros(nmo)
    ctx.check(ctx.lib.qx_compute_exchange_diag(ctx.handle, N.ptr(lpq_a), naux, nmo, int(nocc), N.ptr(out)))
    return out


def evgw_config(**kw) -> N.EvgwConfig:
    lib = N.load()
    cfg = N.EvgwConfig()
    lib.qx_evgw_config_default(C.byref(cfg))
    for k, v in kw.items():
        if v is None:
            continue
        if k == "precision":
            v = _prec(v)
        setattr(cfg, k, v)
    return cfg


def run_evgw_blocks(mo_energy, lpq, vxc, nocc: int, device: int = 0, **cfg_kw) -> Dict:
    """EvGWDriver::run_evgw_blocks on lpq [naux, nmo, nmo] (host array or device tensor)."""
    ctx = _ctx(device, lpq)
    lpq_a = lpq if hasattr(lpq, "data_ptr") else _f64(lpq)
    naux, nmo, _ = tuple(lpq_a.shape)
    cfg = evgw_config(**cfg_kw)
    e = _f64(mo_energy)
    vx = _f64(vxc)
    maxit = cfg.fixed_iterations if cfg.fixed_iterations > 0 else cfg.max_iterations
    qp = np.zeros(nmo)
    z = np.zeros(nmo)
    sx = np.zeros(nmo)
    sc = np.zeros(nmo, dtype=np.complex128)
    he = np.zeros((maxit, nmo))
    hm = np.zeros(maxit)
    hr = np.zeros(maxit)
    dp = C.POINTER(C.c_double)
    res = N.EvgwResult(qp.ctypes.data_as(dp), z.ctypes.data_as(dp), sx.ctypes.data_as(dp), sc.ctypes.data_as(dp),
                       he.ctypes.data_as(dp), hm.ctypes.data_as(dp), hr.ctypes.data_as(dp), 0, 0)
    ctx.check(ctx.lib.qx_evgw(ctx.handle, N.ptr(e), N.ptr(lpq_a), N.ptr(vx), nmo, int(nocc), naux, C.byref(cfg),
                              C.byref(res)))
    n = res.n_iterations
    return dict(qp_energies=qp, z_factors=z, sigma_x=sx, sigma_c=sc, n_iterations=n, converged=bool(res.converged),
                energies=[he[i].copy() for i in range(n)], max_energy_changes=list(hm[:n]),
                rms_energy_changes=list(hr[:n]), timings=ctx.timings())


def _build_lpq(mo_energy, mo_occ, iaP, ijP, abP, naux):
    """Full DF tensor from blocks, symmetrized (quasix/src/evgw.rs:161-205),
    returned in the driver's [naux, nmo, nmo] layout (evgw.rs:539-543)."""
    nmo = len(mo_energy)
    nocc = int(np.count_nonzero(np.asarray(mo_occ) > 0.0))
    nvir = nmo - nocc
    try:
        ia = np.asarray(iaP, dtype=np.float64).reshape(nocc, nvir, naux)
        mi = np.asarray(ijP, dtype=np.float64).reshape(nmo, nocc, naux)
        ab = np.asarray(abP, dtype=np.float64).reshape(nvir, nvir, naux)
    except ValueError as e:
        raise ValueError(f"Failed to reshape DF tensor: {e}") from None
    mn = np.zeros((nmo, nmo, naux))
    mn[:, :nocc] = mi
    mn[:nocc, nocc:] = ia
    mn[nocc:, nocc:] = ab
    mn = 0.5 * (mn + mn.transpose(1, 0, 2))
    return np.ascontiguousarray(mn.transpose(2, 0, 1)), nocc


def _result_dict(res: Dict, nocc: int) -> Dict:
    qp = res["qp_energies"]
    nmo = qp.shape[0]
    hist = []
    for c, e in enumerate(res["energies"]):
        hist.append(dict(cycle=c + 1, qp_energies=e, z_factors=res["z_factors"],
                         energy_change=res["max_energy_changes"][c], rms_change=res["rms_energy_changes"][c],
                         damping_used=0.5, converged=(c + 1 == res["n_iterations"] and res["converged"])))
    out = dict(qp_energies=qp, z_factors=res["z_factors"], converged=res["converged"], n_cycles=res["n_iterations"],
               final_error=res["max_energy_changes"][-1] if res["max_energy_changes"] else 0.0,
               sigma_x=res["sigma_x"], sigma_c_re=res["sigma_c"].real.copy(), sigma_c_im=res["sigma_c"].imag.copy(),
               iteration_history=hist, ip=-qp[nocc - 1])
    if nmo > nocc:
        out["ea"] = -qp[nocc]
        out["gap"] = qp[nocc] - qp[nocc - 1]
    else:
        out["ea"] = None
        out["gap"] = None
    return out


def evgw(mo_energy, mo_occ, iaP, ijP, abP, chol_v, vxc_dft, max_cycle=12, conv_tol=0.0001, conv_tol_z=0.001,
         damping=0.5, damping_dynamic=False, diis=False, diis_space=6, _diis_start_cycle=3, _freq_int="cd",
         nfreq=48, eta=0.01, _check_stability=True, verbose=1, energy_window=2.0, frontier_convergence=True,
         frontier_window=1.0, n_occ_active=None, n_vir_active=None, qp_solver="linearized",
         newton_max_iterations=50, newton_energy_tolerance=1e-8, npade=None, iw_cutoff=5.0, precision="fp64",
         device: int = 0) -> Dict:
    """Drop-in for quasix.quasix.evgw (quasix/src/evgw.rs:22-453)."""
    naux = np.asarray(chol_v).shape[0]
    q = qp_solver.lower()
    if q in ("linearized", "linear"):
        solved = 0
    elif q in ("newton", "newton-raphson", "solved"):
        solved = 1
    else:
        raise ValueError(f"Invalid qp_solver '{qp_solver}'. Valid options: 'linearized' (default) or 'newton'")
    lpq, nocc = _build_lpq(mo_energy, mo_occ, iaP, ijP, abP, naux)
    res = run_evgw_blocks(mo_energy, lpq, vxc_dft, nocc, device=device, max_iterations=int(max_cycle),
                          energy_tolerance=float(conv_tol), damping_factor=float(damping), use_diis=int(bool(diis)),
                          diis_space_dim=int(diis_space), frontier_convergence=int(bool(frontier_convergence)),
                          frontier_window=float(frontier_window), nfreq=int(nfreq), use_solved_qp=solved,
                          newton_energy_tolerance=float(newton_energy_tolerance),
                          newton_max_iterations=int(newton_max_iterations),
                          npade=-1 if npade is None else int(npade), iw_cutoff=float(iw_cutoff),
                          precision=precision)
    return _result_dict(res, nocc)


def run_evgw(config: Dict) -> Dict:
    """Drop-in for quasix.run_evgw(dict) (quasix/src/evgw.rs:456-677)."""
    for k in ("mo_energy", "mo_occ", "iaP", "ijP", "chol_v", "vxc_dft"):
        if k not in config:
            raise KeyError(f"{k} not found")
    iaP = np.asarray(config["iaP"])
    nocc, nvir, naux = iaP.shape
    abP = config.get("abP")
    if abP is None:
        abP = np.zeros((nvir * nvir, naux))
    return evgw(config["mo_energy"], config["mo_occ"], iaP.reshape(nocc * nvir, naux), config["ijP"], abP,
                config["chol_v"], config["vxc_dft"], max_cycle=config.get("max_cycle", 12),
                conv_tol=config.get("conv_tol", 0.0001), damping=config.get("damping", 0.5),
                diis=config.get("diis", True), diis_space=config.get("diis_space", 6),
                nfreq=config.get("nfreq", 48), verbose=config.get("verbose", 1),
                energy_window=config.get("energy_window", 2.0),
                frontier_convergence=config.get("frontier_convergence", True),
                frontier_window=config.get("frontier_window", 0.1),
                n_occ_active=config.get("n_occ_active", 3), n_vir_active=config.get("n_vir_active", 3),
                qp_solver=config.get("qp_solver", "linearized"),
                newton_max_iterations=config.get("newton_max_iterations", 50),
                newton_energy_tolerance=config.get("newton_energy_tolerance", 1e-8), npade=config.get("npade"),
                iw_cutoff=config.get("iw_cutoff", 5.0), precision=config.get("precision", "fp64"), device=config.get("device", 0))


def _qp_solver(name) -> int:
    try:
        return N.QP_SOLVER[name]
    except KeyError:
        raise ValueError(f"qp_solver must be one of {list(N.QP_SOLVER)}") from None


def g0w0_cd(mo_energy, lpq, nocc: int, targets: Sequence[int], nw: int = 100, x0: float = 0.5, vxc=None,
            tol: float = 1e-8, max_iter: int = 50, precision="fp64", qp_solver: str = "newton",
            device: int = 0) -> Dict:
    """G0W0 by contour deformation (imaginary-axis GL integral + residues) with a
    Newton (damped, as NewtonQPSolver) or linearized QP step per target."""
    ctx = _ctx(device, lpq, mo_energy, vxc)
    lpq_a = lpq if hasattr(lpq, "data_ptr") else _f64(lpq)
    naux, nmo, _ = tuple(lpq_a.shape)
    e = mo_energy if hasattr(mo_energy, "data_ptr") else _f64(mo_energy)
    vx = np.zeros(nmo) if vxc is None else (vxc if hasattr(vxc, "data_ptr") else _f64(vxc))
    t = np.ascontiguousarray(np.asarray(targets, dtype=np.int32))
    qp = np.zeros(len(t))
    z = np.zeros(len(t))
    sc = np.zeros(len(t))
    sx = np.zeros(len(t))
    ctx.check(ctx.lib.qx_g0w0_cd(ctx.handle, N.ptr(e), N.ptr(lpq_a), N.ptr(vx), nmo, int(nocc), naux, N.ptr(t), len(t),
                                 int(nw), float(x0), float(tol), int(max_iter), _qp_solver(qp_solver),
                                 _prec(precision), N.ptr(qp), N.ptr(z),
                                 N.ptr(sc), N.ptr(sx)))
    return dict(qp_energies=qp, z_factors=z, sigma_c=sc, sigma_x=sx)


def cd_sigma(mo_energy, lpq, nocc: int, targets: Sequence[int], omega, nw: int = 24, x0: float = 0.5,
             precision="fp64", device: int = 0) -> Dict:
    """Sigma_c^CD_n(omega_t) and dSigma/dw per target at the given real energies
    (qx_cd_sigma), plus diag(Sigma_x) of the targets."""
    ctx = _ctx(device, lpq, mo_energy)
    lpq_a = lpq if hasattr(lpq, "data_ptr") else _f64(lpq)
    naux, nmo, _ = tuple(lpq_a.shape)
    e = mo_energy if hasattr(mo_energy, "data_ptr") else _f64(mo_energy)
    t = np.ascontiguousarray(np.asarray(targets, dtype=np.int32))
    om = _f64(omega)
    sc, ds, sx = np.zeros(len(t)), np.zeros(len(t)), np.zeros(len(t))
    ctx.check(ctx.lib.qx_cd_sigma(ctx.handle, N.ptr(e), N.ptr(lpq_a), nmo, int(nocc), naux, N.ptr(t), len(t),
                                  N.ptr(om), int(nw), float(x0), _prec(precision), N.ptr(sc), N.ptr(ds), N.ptr(sx)))
    return dict(sigma_c=sc, dsigma_c=ds, sigma_x=sx)


def g0w0_cd_batch(systems, nw: int = 24, x0: float = 0.5, tol: float = 1e-8, max_iter: int = 50,
                  precision="fp64", qp_solver: str = "newton", nworkers: int = 0, device: int = 0) -> List[Dict]:
    """G0W0-CD for many independent systems in one call (qx_g0w0_cd_batch).

    ``systems``: sequence of dicts with keys mo_energy, lpq ([naux, nmo, nmo],
    numpy or a CUDA tensor), nocc, targets and optionally vxc.  Returns one dict
    per system with the keys of :func:`g0w0_cd`.  ``nworkers=0`` (default)
    runs the grouped mode (all systems phase by phase, every inversion as one
    grouped block sweep); ``nworkers > 0`` runs each system whole on one of
    that many worker streams, largest first."""
    ctx = _ctx(device, *[s["lpq"] for s in systems])
    keep, outs = [], []
    arr = (N.CdSystem * len(systems))()
    for i, s in enumerate(systems):
        lpq = s["lpq"] if hasattr(s["lpq"], "data_ptr") else _f64(s["lpq"])
        naux, nmo, _ = tuple(lpq.shape)
        e = s["mo_energy"]
        e = e if hasattr(e, "data_ptr") else _f64(e)
        vx = s.get("vxc")
        vx = None if vx is None else (vx if hasattr(vx, "data_ptr") else _f64(vx))
        t = np.ascontiguousarray(np.asarray(s["targets"], dtype=np.int32))
        out = dict(qp_energies=np.zeros(len(t)), z_factors=np.zeros(len(t)), sigma_c=np.zeros(len(t)),
                   sigma_x=np.zeros(len(t)))
        keep += [lpq, e, vx, t]
        outs.append(out)
        arr[i] = N.CdSystem(N.ptr(e), N.ptr(lpq), N.ptr(vx), nmo, int(s["nocc"]), naux, N.ptr(t), len(t),
                            N.ptr(out["qp_energies"]), N.ptr(out["z_factors"]), N.ptr(out["sigma_c"]),
                            N.ptr(out["sigma_x"]), -1)
    ctx.check(ctx.lib.qx_g0w0_cd_batch(ctx.handle, arr, len(systems), int(nw), float(x0), float(tol), int(max_iter),
                                       _qp_solver(qp_solver), _prec(precision), int(nworkers)))
    return outs
