"""CPU FP64 oracle for the RI GW/BSE hot path (TEST INFRASTRUCTURE ONLY).

This module is the checker, not the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it.  The product path (``quasix_b200``) never calls into it and fails loudly
when its CUDA library is missing.

It restates, in numpy/scipy (FP64, LAPACK via scipy), the algorithm of the
QuasiX reference implementation (a Rust crate that cannot be built here:
there is no Rust toolchain).  Each function cites the reference file:line it
follows, by path within the QuasiX project.

Parity pinning: the reference cannot run here, so this restatement is pinned
against every known-answer test the reference's own test suite holds for this
path (Gauss-Legendre 2-point rule, Thiele of a constant, Pade of 1/(1+z),
Pi symmetry and the P0 prefactor hand case, W -> v as P0 -> 0, the 6-MO cached
fixture, the Newton/Richardson cases, the 6x6 Davidson case) plus an analytic
one-pole model with a closed-form self-energy; see tests/test_oracle_*.py.
The contour-deformation residue term has no reference implementation
(quasix_core/src/freq/contour_deformation.rs:142-239 is an unused skeleton), so
it is restated from the published formulation and pinned only by the analytic
model.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np
import scipy.linalg as sla

PI = math.pi


# ---------------------------------------------------------------------------
# a1: frequency grid
# ---------------------------------------------------------------------------
def gauss_legendre_nodes_weights(n: int) -> Tuple[np.ndarray, np.ndarray]:
    """Golub-Welsch GL rule on [-1, 1].

    quasix_core/src/selfenergy/correlation_ac.rs:122-160: Jacobi matrix with
    beta_i = i / sqrt((2i-1)(2i+1)), nodes = eigenvalues, weights = 2 v_0^2.
    """
    if n == 0:
        return np.zeros(0), np.zeros(0)
    if n == 1:
        return np.array([0.0]), np.array([2.0])
    i = np.arange(1, n, dtype=np.float64)
    beta = i / np.sqrt((2.0 * i - 1.0) * (2.0 * i + 1.0))
    J = np.diag(beta, 1) + np.diag(beta, -1)
    evals, evecs = np.linalg.eigh(J)
    return evals, 2.0 * evecs[0, :] ** 2


def get_scaled_legendre_roots(nw: int, x0: float = 0.5) -> Tuple[np.ndarray, np.ndarray]:
    """GL rule mapped to [0, inf): w = x0 (1+t)/(1-t), wt = w_t 2 x0/(1-t)^2.

    quasix_core/src/selfenergy/correlation_ac.rs:94-114.
    """
    t, w = gauss_legendre_nodes_weights(nw)
    freqs = x0 * (1.0 + t) / (1.0 - t)
    wts = w * 2.0 * x0 / (1.0 - t) ** 2
    return freqs, wts


# ---------------------------------------------------------------------------
# a2: polarizability
# ---------------------------------------------------------------------------
def get_rho_response(omega: float, mo_energy: np.ndarray, lpq_ov: np.ndarray) -> np.ndarray:
    """Pi(iw) = 4 (L_ov * chi) L_ov^T, chi_ia = e_ia / (w^2 + e_ia^2), e_ia = e_i - e_a.

    quasix_core/src/selfenergy/correlation_ac.rs:184-211.  lpq_ov is [naux, nocc, nvir].
    """
    naux, nocc, nvir = lpq_ov.shape
    e_ia = (mo_energy[:nocc, None] - mo_energy[None, nocc:nocc + nvir]).reshape(-1)
    chi = e_ia / (omega * omega + e_ia * e_ia)
    flat = lpq_ov.reshape(naux, nocc * nvir)
    return 4.0 * (flat * chi) @ flat.T


def get_rho_response_real(omega_r: float, mo_energy: np.ndarray, lpq_ov: np.ndarray) -> np.ndarray:
    """Pi at a real frequency: the continuation iw -> w_r of get_rho_response,
    chi_ia = e_ia / (e_ia^2 - w_r^2).  Used only by the contour-deformation
    residues (restated from the mathematics; no reference implementation)."""
    naux, nocc, nvir = lpq_ov.shape
    e_ia = (mo_energy[:nocc, None] - mo_energy[None, nocc:nocc + nvir]).reshape(-1)
    chi = e_ia / (e_ia * e_ia - omega_r * omega_r)
    flat = lpq_ov.reshape(naux, nocc * nvir)
    return 4.0 * (flat * chi) @ flat.T


def compute_polarizability_p0(ia_P: np.ndarray, mo_energy: np.ndarray, mo_occ: np.ndarray,
                              freqs: np.ndarray) -> np.ndarray:
    """S3-2 variant: P0[w] = sum_ia 4 e_ia/(w^2+e_ia^2) (ia|P)(ia|Q), symmetrized.

    quasix_core/src/dielectric/polarizability.rs:169-275 (weight :231).
    ia_P is [nocc, nvir, naux]; returns [nfreq, naux, naux].
    """
    nocc, nvir, naux = ia_P.shape
    out = np.empty((len(freqs), naux, naux))
    lpq_ov = np.ascontiguousarray(ia_P.transpose(2, 0, 1))
    for k, w in enumerate(freqs):
        p = get_rho_response(w, mo_energy, lpq_ov)
        out[k] = 0.5 * (p + p.T)
    return out


# ---------------------------------------------------------------------------
# a3: screened interaction
# ---------------------------------------------------------------------------
def epsilon_inverse_minus_identity(pi: np.ndarray) -> np.ndarray:
    """Wc = (I - Pi)^-1 - I via Cholesky inverse, LU fallback, identity fallback.

    quasix_core/src/selfenergy/correlation_ac.rs:377-401.
    """
    n = pi.shape[0]
    eps = np.eye(n) - pi
    try:
        c, low = sla.cho_factor(eps, lower=False, check_finite=False)
        inv = sla.cho_solve((c, low), np.eye(n), check_finite=False)
    except np.linalg.LinAlgError:
        try:
            inv = np.linalg.inv(eps)
        except np.linalg.LinAlgError:
            inv = np.eye(n)
    return inv - np.eye(n)


def compute_screened_interaction(p0: np.ndarray, v_aux: np.ndarray) -> np.ndarray:
    """S3-3 variant: W = v^1/2 (I - v^1/2 P0 v^1/2)^-1 v^1/2 per frequency, with a
    symmetric v^1/2 from eigh.  quasix_core/src/dielectric/screening.rs:164-236,
    334-410, 580-639.  p0 is [nfreq, naux, naux]."""
    lam, U = np.linalg.eigh(v_aux)
    vs = (U * np.sqrt(np.maximum(lam, 1e-14))) @ U.T   # the clamp of screening.rs:606-607
    out = np.empty_like(p0)
    n = v_aux.shape[0]
    for k in range(p0.shape[0]):
        m = np.eye(n) - vs @ p0[k] @ vs
        m = 0.5 * (m + m.T)
        w = vs @ np.linalg.inv(m) @ vs
        out[k] = 0.5 * (w + w.T)
    return out


# ---------------------------------------------------------------------------
# a4: Sigma_c on the imaginary axis
# ---------------------------------------------------------------------------
def sigma_grid(nw: int, iw_cutoff: float = 5.0, x0: float = 0.5):
    """Self-energy sample grid of get_sigma_diag: index 0 is w = 0, then every GL
    frequency below the cutoff.  correlation_ac.rs:268-302."""
    freqs, wts = get_scaled_legendre_roots(nw, x0)
    idx = [i for i in range(nw) if freqs[i] < iw_cutoff]
    nw_sigma = min(len(idx) + 1, nw + 1)
    iw = np.zeros(nw_sigma)
    for k, fi in enumerate(idx):
        if k + 1 < nw_sigma:
            iw[k + 1] = freqs[fi]
    return freqs, wts, iw


def get_sigma_diag(mo_energy: np.ndarray, lpq: np.ndarray, orbs: Sequence[int], nocc: int,
                   nw: int = 100, iw_cutoff: float = 5.0, x0: float = 0.5
                   ) -> Tuple[np.ndarray, np.ndarray]:
    """Sigma_c(iw_k) for every orbital in ``orbs``.

    quasix_core/src/selfenergy/correlation_ac.rs:241-449.  The structure is the
    reference's: per frequency, Pi by one GEMM, Wc by Cholesky inverse, then one
    GEMM per target orbital (:415-438).  Returns (sigma, omega), both complex
    [norbs, nw_sigma]; omega is -i*w for occupied targets and +i*w for virtual.
    """
    naux, nmo, nmo2 = lpq.shape
    if nmo != nmo2:
        raise ValueError(f"Lpq not square in MO dimensions: {nmo} x {nmo2}")
    if nocc == 0 or nocc >= nmo:
        raise ValueError(f"Invalid nocc={nocc}: must be in range [1, {nmo})")
    freqs, wts, iw = sigma_grid(nw, iw_cutoff, x0)
    nw_sigma = iw.shape[0]
    ef = 0.5 * (mo_energy[nocc - 1] + mo_energy[nocc])
    omega_occ = -1j * iw
    omega_vir = 1j * iw
    emo_occ = omega_occ[None, :] + ef - mo_energy[:, None]
    emo_vir = omega_vir[None, :] + ef - mo_energy[:, None]
    lpq_ov = lpq[:, :nocc, nocc:]
    orbs = list(orbs)
    norbs = len(orbs)
    sigma = np.zeros((norbs, nw_sigma), dtype=np.complex128)
    omega = np.array([omega_occ if o < nocc else omega_vir for o in orbs])
    for w in range(nw):
        pi = get_rho_response(freqs[w], mo_energy, lpq_ov)
        wc = epsilon_inverse_minus_identity(pi)
        g0_occ = wts[w] * emo_occ / (emo_occ * emo_occ + freqs[w] ** 2)
        g0_vir = wts[w] * emo_vir / (emo_vir * emo_vir + freqs[w] ** 2)
        for ni, n in enumerate(orbs):
            q = wc.T @ lpq[:, n, :]
            wmn = np.sum(q * lpq[:, :, n], axis=0)
            g0 = g0_occ if n < nocc else g0_vir
            sigma[ni] += (-1.0 / PI) * (wmn @ g0)
    return sigma, omega


def get_sigma_diag_threaded(mo_energy, lpq, orbs, nocc, nw=100, iw_cutoff=5.0, x0=0.5, workers=1):
    """get_sigma_diag with its frequency loop on a thread pool, as the reference
    runs it (rayon into_par_iter over frequencies, correlation_ac.rs:367-441):
    each worker returns the contribution of its frequencies, summed afterwards
    in frequency order.  Same arithmetic as get_sigma_diag per frequency."""
    from concurrent.futures import ThreadPoolExecutor
    naux, nmo, _ = lpq.shape
    freqs, wts, iw = sigma_grid(nw, iw_cutoff, x0)
    ef = 0.5 * (mo_energy[nocc - 1] + mo_energy[nocc])
    emo_occ = (-1j * iw)[None, :] + ef - mo_energy[:, None]
    emo_vir = (1j * iw)[None, :] + ef - mo_energy[:, None]
    lpq_ov = lpq[:, :nocc, nocc:]
    orbs = list(orbs)

    def one(w):
        pi = get_rho_response(freqs[w], mo_energy, lpq_ov)
        wc = epsilon_inverse_minus_identity(pi)
        g0_occ = wts[w] * emo_occ / (emo_occ * emo_occ + freqs[w] ** 2)
        g0_vir = wts[w] * emo_vir / (emo_vir * emo_vir + freqs[w] ** 2)
        part = np.zeros((len(orbs), iw.shape[0]), dtype=np.complex128)
        for ni, n in enumerate(orbs):
            q = wc.T @ lpq[:, n, :]
            wmn = np.sum(q * lpq[:, :, n], axis=0)
            part[ni] = (-1.0 / PI) * (wmn @ (g0_occ if n < nocc else g0_vir))
        return part

    with ThreadPoolExecutor(max(1, workers)) as ex:
        parts = list(ex.map(one, range(nw)))
    sigma = np.zeros((len(orbs), iw.shape[0]), dtype=np.complex128)
    for part in parts:
        sigma += part
    omega = np.array([-1j * iw if o < nocc else 1j * iw for o in orbs])
    return sigma, omega


# ---------------------------------------------------------------------------
# a6: Thiele / Pade analytic continuation
# ---------------------------------------------------------------------------
def thiele(fn: np.ndarray, zn: np.ndarray) -> np.ndarray:
    """Continued-fraction coefficients by reciprocal differences.

    quasix_core/src/selfenergy/correlation_ac.rs:470-509 (guard 1e-14 -> 1e10 at :493-498).
    """
    nfit = fn.shape[0]
    g = np.zeros((nfit, nfit), dtype=np.complex128)
    g[:, 0] = fn
    for j in range(1, nfit):
        for i in range(j, nfit):
            denom = (zn[i] - zn[j - 1]) * g[i, j - 1]
            if abs(denom) < 1e-14:
                g[i, j] = 1e10
            else:
                g[i, j] = (g[j - 1, j - 1] - g[i, j - 1]) / denom
    return np.diag(g).copy()


def pade_thiele(omega, zn: np.ndarray, coeff: np.ndarray) -> complex:
    """Backward continued-fraction evaluation at real (or complex) omega.

    quasix_core/src/selfenergy/correlation_ac.rs:530-566.
    """
    nfit = coeff.shape[0]
    if nfit == 0:
        return 0j
    if nfit == 1:
        return complex(coeff[0])
    z = complex(omega)
    x = coeff[nfit - 1] * (z - zn[nfit - 2])
    for i in range(nfit - 2, 0, -1):
        denom = 1.0 + x
        if abs(denom) < 1e-14:
            x = 1e10 + 0j
        else:
            x = coeff[i] * (z - zn[i - 1]) / denom
    denom = 1.0 + x
    if abs(denom) < 1e-14:
        return complex(coeff[0])
    return complex(coeff[0] / denom)


def pade_point_indices(nw_sigma: int, npade: Optional[int] = None) -> List[int]:
    """Sample points used for the fit.

    ``npade=None`` is the reference rule (correlation_ac.rs:599-622): indices
    1, 7, 13, ... (< min(40, nw)), then every 4th from the last + 4, truncated to
    an even count.  ``npade=k`` selects 2k points spread evenly over indices
    1 .. nw_sigma-1 (the [k/k] variant, e.g. k = 15); it needs nw_sigma >= 2k + 1.
    """
    if npade is None:
        idx1 = list(range(1, min(40, nw_sigma), 6))
        idx2: List[int] = []
        if idx1:
            idx2 = list(range(idx1[-1] + 4, nw_sigma, 4))
        allidx = idx1 + idx2
        nfit = (len(allidx) // 2) * 2
        return allidx[:nfit]
    if 2 * npade + 1 > nw_sigma:
        raise ValueError(f"[{npade}/{npade}] Pade needs {2 * npade + 1} sigma points, have {nw_sigma}")
    m = 2 * npade
    if m == 1:
        return [1]
    return [int(math.floor(1.0 + j * (nw_sigma - 2) / (m - 1) + 0.5)) for j in range(m)]


def ac_pade_thiele_diag(sigma: np.ndarray, omega: np.ndarray, npade: Optional[int] = None):
    """Thiele coefficients per orbital.  correlation_ac.rs:587-654.

    Returns (coeff [nfit, norbs], omega_fit [norbs, nfit]).
    """
    norbs, nw = sigma.shape
    idx = pade_point_indices(nw, npade)
    nfit = len(idx)
    if nfit == 0:
        return np.zeros((0, norbs), np.complex128), np.zeros((norbs, 0), np.complex128)
    sfit = sigma[:, idx]
    ofit = omega[:, idx]
    coeff = np.zeros((nfit, norbs), dtype=np.complex128)
    for p in range(norbs):
        coeff[:, p] = thiele(sfit[p], ofit[p])
    return coeff, ofit


# ---------------------------------------------------------------------------
# a8: Newton QP solver
# ---------------------------------------------------------------------------
@dataclass
class NewtonSolverConfig:
    """quasix_core/src/qp/newton_solver.rs:86-103."""
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


class ConvergenceError(RuntimeError):
    pass


@dataclass
class NewtonResult:
    qp_energy: float
    residual: float
    iterations: int
    converged: bool
    sigma_c: complex
    z_factor: float
    method: str


class NewtonQPSolver:
    """f(E) = E - eps - Sigma_x - Re Sigma_c(E - ef) + Vxc = 0.

    quasix_core/src/qp/newton_solver.rs:141-402.
    """

    def __init__(self, epsilon_hf: float, sigma_x: float, vxc: float, fermi_level: float,
                 config: NewtonSolverConfig):
        self.eps = epsilon_hf
        self.sx = sigma_x
        self.vxc = vxc
        self.ef = fermi_level
        self.cfg = config

    def compute_derivative(self, f: Callable[[float], complex], omega: float) -> float:
        """newton_solver.rs:282-303."""
        de = self.cfg.derivative_delta
        if self.cfg.use_richardson:
            p1 = f(omega + de).real
            m1 = f(omega - de).real
            p2 = f(omega + 2.0 * de).real
            m2 = f(omega - 2.0 * de).real
            return (8.0 * (p1 - m1) - (p2 - m2)) / (12.0 * de)
        return (f(omega + de).real - f(omega - de).real) / (2.0 * de)

    def compute_z_factor(self, f, energy: float) -> float:
        """newton_solver.rs:306-315."""
        d = self.compute_derivative(f, energy - self.ef)
        z = 1.0 / (1.0 - d)
        return min(max(z, self.cfg.z_min), self.cfg.z_max)

    def residual(self, f, energy: float) -> float:
        """newton_solver.rs:394-401."""
        return energy - self.eps - self.sx - f(energy - self.ef).real + self.vxc

    def solve(self, f, initial_guess: float) -> NewtonResult:
        """newton_solver.rs:174-280."""
        cfg = self.cfg
        energy = initial_guess
        damping = cfg.initial_damping
        prev = float("inf")
        for it in range(cfg.max_iterations):
            omega = energy - self.ef
            sc = f(omega)
            res = energy - self.eps - self.sx - sc.real + self.vxc
            ares = abs(res)
            if ares < cfg.energy_tolerance:
                z = self.compute_z_factor(f, energy)
                return NewtonResult(energy, ares, it + 1, True, sc, z, "newton")
            d = self.compute_derivative(f, omega)
            fp = 1.0 - d
            if abs(fp) < 1e-10:
                step = -math.copysign(1.0, res) * min(cfg.max_step, ares)
            else:
                step = -res / fp
            clipped = min(max(step, -cfg.max_step), cfg.max_step)
            if ares > prev:
                damping = max(damping * 0.5, cfg.min_damping)
            elif ares < 0.5 * prev and damping < cfg.max_damping:
                damping = min(damping * 1.2, cfg.max_damping)
            energy += damping * clipped
            prev = ares
        if cfg.use_bisection_fallback:
            return self.bisection_fallback(f, initial_guess)
        raise ConvergenceError("Newton-Raphson failed to converge")

    def bisection_fallback(self, f, initial_guess: float) -> NewtonResult:
        """newton_solver.rs:317-392."""
        cfg = self.cfg
        width = 2.0
        lo = initial_guess - width
        hi = initial_guess + width
        if self.residual(f, lo) * self.residual(f, hi) > 0.0:
            for e in range(1, 5):
                w = width * 2.0 ** e
                lo = initial_guess - w
                hi = initial_guess + w
                if self.residual(f, lo) * self.residual(f, hi) <= 0.0:
                    break
        for it in range(cfg.max_bisection_iterations):
            mid = 0.5 * (lo + hi)
            fm = self.residual(f, mid)
            if abs(fm) < cfg.energy_tolerance or 0.5 * (hi - lo) < cfg.energy_tolerance:
                sc = f(mid - self.ef)
                z = self.compute_z_factor(f, mid)
                return NewtonResult(mid, abs(fm), it + 1, True, sc, z, "bisection")
            fl = self.residual(f, lo)
            if fm * fl < 0.0:
                hi = mid
            else:
                lo = mid
        raise ConvergenceError("Bisection fallback failed to converge")


# ---------------------------------------------------------------------------
# a9: DIIS / convergence monitor
# ---------------------------------------------------------------------------
def _diis_solve(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Gaussian elimination with partial pivoting and the reference's guards.

    quasix_core/src/qp/convergence.rs:440-540.
    """
    PIVOT_TOL = 1e-12
    COND_TOL = 1e-10
    n = a.shape[0]
    aug = np.zeros((n, n + 1))
    aug[:, :n] = a
    aug[:, n] = b
    max_elem = np.abs(a).max()
    abs_tol = PIVOT_TOL * max(max_elem, 1.0)
    for i in range(n - 1):
        max_row = i
        max_val = abs(aug[i, i])
        for k in range(i + 1, n):
            if abs(aug[k, i]) > max_val:
                max_val = abs(aug[k, i])
                max_row = k
        if max_val < abs_tol:
            raise ConvergenceError("DIIS matrix is singular or ill-conditioned")
        if max_row != i:
            aug[[i, max_row]] = aug[[max_row, i]]
        piv = aug[i, i]
        for k in range(i + 1, n):
            if abs(aug[k, i]) > COND_TOL * abs(piv):
                fac = aug[k, i] / piv
                aug[k, i:] -= fac * aug[i, i:]
    if abs(aug[n - 1, n - 1]) < abs_tol:
        raise ConvergenceError("DIIS matrix is singular")
    x = np.zeros(n)
    for i in range(n - 1, -1, -1):
        x[i] = aug[i, n] - aug[i, i + 1:n] @ x[i + 1:n]
        if abs(aug[i, i]) < abs_tol:
            raise ConvergenceError("DIIS back-substitution failed")
        x[i] /= aug[i, i]
    if abs(x[:n - 1].sum() - 1.0) > 0.5:
        raise ConvergenceError("DIIS coefficients do not sum to ~1")
    if not np.all(np.isfinite(x)):
        raise ConvergenceError("DIIS solution not finite")
    return x


class ConvergenceMonitor:
    """History + DIIS on [E; Z].  quasix_core/src/qp/convergence.rs:96-330.

    Only the parts the evGW driver reaches are restated: check_convergence's
    history bookkeeping (:146-192) and apply_diis (:264-321).
    """

    def __init__(self, diis_max_vectors: Optional[int]):
        self.max_vectors = diis_max_vectors
        self.energy_history: List[np.ndarray] = []
        self.z_history: List[np.ndarray] = []
        self.diis_vectors: List[np.ndarray] = []
        self.diis_errors: List[np.ndarray] = []

    def check_convergence(self, energies: np.ndarray, z: np.ndarray) -> None:
        if not self.energy_history:
            self.energy_history.append(energies.copy())
            self.z_history.append(z.copy())
            return
        self.energy_history.append(energies.copy())
        self.z_history.append(z.copy())
        if self.max_vectors is not None:
            while len(self.energy_history) > self.max_vectors:
                self.energy_history.pop(0)
                self.z_history.pop(0)

    def accelerate(self, energies: np.ndarray, z: np.ndarray):
        if self.max_vectors is None:
            return energies.copy(), z.copy()
        if not self.energy_history:
            return energies.copy(), z.copy()
        # The error is taken against the newest history entry (convergence.rs:275-276).
        error = energies - self.energy_history[-1]
        combined = np.concatenate([energies, z])
        self.diis_vectors.append(combined)
        self.diis_errors.append(error)
        while len(self.diis_vectors) > self.max_vectors:
            self.diis_vectors.pop(0)
            self.diis_errors.pop(0)
        nv = len(self.diis_vectors)
        if nv < 2:
            return energies.copy(), z.copy()
        B = np.zeros((nv + 1, nv + 1))
        for i in range(nv):
            for j in range(i + 1):
                d = float(self.diis_errors[i] @ self.diis_errors[j])
                B[i, j] = d
                B[j, i] = d
            B[i, nv] = -1.0
            B[nv, i] = -1.0
        rhs = np.zeros(nv + 1)
        rhs[nv] = -1.0
        c = _diis_solve(B, rhs)
        res = np.zeros_like(combined)
        for i in range(nv):
            res = res + c[i] * self.diis_vectors[i]
        n = energies.shape[0]
        return res[:n].copy(), res[n:].copy()


# ---------------------------------------------------------------------------
# a10: exchange self-energy
# ---------------------------------------------------------------------------
def compute_exchange(mi_all_occ: np.ndarray) -> np.ndarray:
    """Sigma_x[p,q] = -sum_{i,R} (pi|R)(qi|R).  quasix_core/src/qp/evgw.rs:1167-1193.
    mi_all_occ is [nmo, nocc, naux]."""
    nmo = mi_all_occ.shape[0]
    flat = mi_all_occ.reshape(nmo, -1)
    return -(flat @ flat.T)


# ---------------------------------------------------------------------------
# a9: evGW driver
# ---------------------------------------------------------------------------
@dataclass
class EvGWConfig:
    """quasix_core/src/qp/evgw.rs:161-316, with the Python binding's overrides
    (quasix/src/evgw.rs:231-292)."""
    max_iterations: int = 12
    energy_tolerance: float = 1e-4
    damping_factor: float = 0.5
    z_min: float = 0.1
    z_max: float = 0.999
    use_diis: bool = True
    diis_space_dim: int = 6
    frontier_convergence: bool = True
    frontier_window: float = 1.0
    nfreq: int = 100
    iw_cutoff: float = 5.0
    x0: float = 0.5
    use_solved_qp: bool = False
    newton_energy_tolerance: float = 1e-8
    newton_max_iterations: int = 50
    npade: Optional[int] = None  # None = reference point rule


def determine_convergence_window(mo_energy: np.ndarray, n_occ: int, cfg: EvGWConfig) -> Tuple[int, int]:
    """quasix_core/src/qp/evgw.rs:1121-1160."""
    n_mo = mo_energy.shape[0]
    if not cfg.frontier_convergence:
        return 0, n_mo
    w = cfg.frontier_window
    homo = mo_energy[n_occ - 1]
    start = max(n_occ - 1, 0)
    for i in range(n_occ - 1, -1, -1):
        if mo_energy[i] >= homo - w:
            start = i
        else:
            break
    lumo = mo_energy[n_occ]
    end = n_occ + 1
    for i in range(n_occ, n_mo):
        if mo_energy[i] <= lumo + w:
            end = i + 1
        else:
            break
    return start, end


def run_evgw_blocks(mo_energy: np.ndarray, mi_all_occ: np.ndarray, vxc: np.ndarray,
                    lpq: np.ndarray, n_occ: int, cfg: EvGWConfig,
                    sigma_fn=None) -> Dict:
    """EvGWDriver::run_evgw_blocks, quasix_core/src/qp/evgw.rs:420-1049.

    ``lpq`` is the [naux, nmo, nmo] tensor.  ``sigma_fn(energies)`` may replace
    the imaginary-axis Sigma_c evaluation (default: get_sigma_diag).
    """
    n_mo = mo_energy.shape[0]
    ef = 0.5 * (mo_energy[n_occ - 1] + mo_energy[n_occ])
    sigma_x = compute_exchange(mi_all_occ)
    sx = np.diag(sigma_x).copy()
    qp = mo_energy.copy()
    z = np.ones(n_mo)
    final_sc = np.zeros(n_mo, dtype=np.complex128)
    monitor = ConvergenceMonitor(cfg.diis_space_dim if cfg.use_diis else None)
    history = []
    max_changes = []
    rms_changes = []
    orbs = list(range(n_mo))
    de = 1e-6
    ncfg = NewtonSolverConfig(max_iterations=cfg.newton_max_iterations,
                              energy_tolerance=cfg.newton_energy_tolerance,
                              z_min=cfg.z_min, z_max=cfg.z_max)
    for it in range(cfg.max_iterations):
        qp_old = qp.copy()
        e_p0 = mo_energy.copy() if it == 0 else qp_old.copy()
        if sigma_fn is None:
            s_iw, o_iw = get_sigma_diag(e_p0, lpq, orbs, n_occ, cfg.nfreq, cfg.iw_cutoff, cfg.x0)
        else:
            s_iw, o_iw = sigma_fn(e_p0)
        coeff, ofit = ac_pade_thiele_diag(s_iw, o_iw, cfg.npade)
        new_qp = np.zeros(n_mo)
        new_z = np.zeros(n_mo)
        for idx, p in enumerate(orbs):
            op = ofit[idx]
            cp = coeff[:, idx]
            f = (lambda w, op=op, cp=cp: pade_thiele(w, op, cp))
            if cfg.use_solved_qp:
                if it == 0:
                    we = mo_energy[p] - ef
                    s0 = f(we).real
                    s1 = f(we + de).real
                    zz = min(max(1.0 / (1.0 - (s1 - s0) / de), cfg.z_min), cfg.z_max)
                    guess = mo_energy[p] + zz * (sx[p] + s0 - vxc[p])
                else:
                    guess = qp_old[p]
                solver = NewtonQPSolver(mo_energy[p], sx[p], vxc[p], ef, ncfg)
                try:
                    r = solver.solve(f, guess)
                    new_qp[p] = r.qp_energy
                    new_z[p] = r.z_factor
                    final_sc[p] = r.sigma_c
                except ConvergenceError:
                    we = guess - ef
                    sc = f(we)
                    s1 = f(we + de)
                    zz = min(max(1.0 / (1.0 - (s1.real - sc.real) / de), cfg.z_min), cfg.z_max)
                    new_qp[p] = mo_energy[p] + zz * (sx[p] + sc.real - vxc[p])
                    new_z[p] = zz
                    final_sc[p] = sc
            else:
                ev = mo_energy[p] if it == 0 else qp_old[p]
                we = ev - ef
                sc = f(we)
                final_sc[p] = sc
                s1 = f(we + de)
                zz = min(max(1.0 / (1.0 - (s1.real - sc.real) / de), cfg.z_min), cfg.z_max)
                new_z[p] = zz
                new_qp[p] = mo_energy[p] + zz * (sx[p] + sc.real - vxc[p])
        # Mixing (evgw.rs:832-927)
        d = cfg.damping_factor
        if it == 0:
            qp = new_qp.copy()
            z = new_z.copy()
            monitor.check_convergence(qp, z)
        elif it == 1:
            qp = (1.0 - d) * qp_old + d * new_qp
            z = (1.0 - d) * z + d * new_z
            monitor.check_convergence(qp, z)
        elif cfg.use_diis:
            monitor.check_convergence(new_qp, new_z)
            try:
                de_, dz_ = monitor.accelerate(new_qp, new_z)
                if np.abs(de_ - new_qp).max() < 0.5 and np.abs(dz_ - new_z).max() < 0.2:
                    qp, z = de_, dz_
                else:
                    qp = (1.0 - d) * qp_old + d * new_qp
                    z = (1.0 - d) * z + d * new_z
            except ConvergenceError:
                qp = (1.0 - d) * qp_old + d * new_qp
                z = (1.0 - d) * z + d * new_z
            z = np.clip(z, cfg.z_min, cfg.z_max)
        else:
            qp = (1.0 - d) * qp_old + d * new_qp
            z = (1.0 - d) * z + d * new_z
        cs, ce = determine_convergence_window(mo_energy, n_occ, cfg)
        dconv = np.abs(qp[cs:ce] - qp_old[cs:ce])
        max_change = float(dconv.max())
        rms_change = float(np.sqrt((dconv ** 2).sum() / (ce - cs)))
        history.append(qp.copy())
        max_changes.append(max_change)
        rms_changes.append(rms_change)
        if max_change < cfg.energy_tolerance:
            return dict(qp_energies=qp, z_factors=z, sigma_x=sigma_x, sigma_c=final_sc,
                        n_iterations=it + 1, converged=True, energies=history,
                        max_energy_changes=max_changes, rms_energy_changes=rms_changes)
    return dict(qp_energies=qp, z_factors=z, sigma_x=sigma_x, sigma_c=final_sc,
                n_iterations=cfg.max_iterations, converged=False, energies=history,
                max_energy_changes=max_changes, rms_energy_changes=rms_changes)


def build_mn_full(mo_energy, mo_occ, iaP, ijP, abP, naux) -> Tuple[np.ndarray, int]:
    """Rebuild the full (m, n, P) tensor from blocks and symmetrize.

    quasix/src/evgw.rs:93-205.  Returns (mn_full [nmo, nmo, naux], nocc).
    """
    n_mo = mo_energy.shape[0]
    n_occ = int(np.count_nonzero(np.asarray(mo_occ) > 0.0))
    n_vir = n_mo - n_occ
    ia = np.asarray(iaP).reshape(n_occ, n_vir, naux)
    mi = np.asarray(ijP).reshape(n_mo, n_occ, naux)
    ab = np.asarray(abP).reshape(n_vir, n_vir, naux)
    mn = np.zeros((n_mo, n_mo, naux))
    mn[:, :n_occ, :] = mi
    mn[:n_occ, n_occ:, :] = ia
    mn[n_occ:, n_occ:, :] = ab
    iu, ju = np.triu_indices(n_mo, 1)
    avg = 0.5 * (mn[iu, ju, :] + mn[ju, iu, :])
    mn[iu, ju, :] = avg
    mn[ju, iu, :] = avg
    return mn, n_occ


def evgw(mo_energy, mo_occ, iaP, ijP, abP, chol_v, vxc_dft, max_cycle=12, conv_tol=1e-4,
         damping=0.5, diis=False, diis_space=6, nfreq=48, frontier_convergence=True,
         frontier_window=1.0, qp_solver="linearized", newton_max_iterations=50,
         newton_energy_tolerance=1e-8, npade=None, iw_cutoff=5.0, **_unused) -> Dict:
    """quasix.quasix.evgw, quasix/src/evgw.rs:22-453 (result dict :339-452)."""
    mo_energy = np.asarray(mo_energy, dtype=np.float64)
    naux = np.asarray(chol_v).shape[0]
    mn, n_occ = build_mn_full(mo_energy, mo_occ, iaP, ijP, abP, naux)
    q = qp_solver.lower()
    if q in ("linearized", "linear"):
        solved = False
    elif q in ("newton", "newton-raphson", "solved"):
        solved = True
    else:
        raise ValueError(f"Invalid qp_solver '{qp_solver}'")
    cfg = EvGWConfig(max_iterations=max_cycle, energy_tolerance=conv_tol, damping_factor=damping,
                     use_diis=diis, diis_space_dim=diis_space, frontier_convergence=frontier_convergence,
                     frontier_window=frontier_window, nfreq=nfreq, use_solved_qp=solved,
                     newton_energy_tolerance=newton_energy_tolerance,
                     newton_max_iterations=newton_max_iterations, npade=npade,
                     iw_cutoff=iw_cutoff)
    lpq = np.ascontiguousarray(mn.transpose(2, 0, 1))
    mi = mn[:, :n_occ, :]
    res = run_evgw_blocks(mo_energy, mi, np.asarray(vxc_dft, dtype=np.float64), lpq, n_occ, cfg)
    return evgw_result_dict(res, n_occ)


def evgw_result_dict(res: Dict, n_occ: int) -> Dict:
    """Result dictionary of quasix/src/evgw.rs:339-452."""
    qp = res["qp_energies"]
    n_mo = qp.shape[0]
    hist = []
    for c, e in enumerate(res["energies"]):
        hist.append(dict(cycle=c + 1, qp_energies=e, z_factors=res["z_factors"],
                         energy_change=res["max_energy_changes"][c],
                         rms_change=res["rms_energy_changes"][c], damping_used=0.5,
                         converged=(c + 1 == res["n_iterations"] and res["converged"])))
    out = dict(qp_energies=qp, z_factors=res["z_factors"], converged=res["converged"],
               n_cycles=res["n_iterations"],
               final_error=res["max_energy_changes"][-1] if res["max_energy_changes"] else 0.0,
               sigma_x=np.diag(res["sigma_x"]).copy(), sigma_c_re=res["sigma_c"].real.copy(),
               sigma_c_im=res["sigma_c"].imag.copy(), iteration_history=hist,
               ip=-qp[n_occ - 1])
    if n_mo > n_occ:
        out["ea"] = -qp[n_occ]
        out["gap"] = qp[n_occ] - qp[n_occ - 1]
    else:
        out["ea"] = None
        out["gap"] = None
    return out


def run_evgw(config: Dict) -> Dict:
    """quasix.run_evgw(dict), quasix/src/evgw.rs:456-677 (defaults :541-641)."""
    for k in ("mo_energy", "mo_occ", "iaP", "ijP", "chol_v", "vxc_dft"):
        if k not in config:
            raise KeyError(f"{k} not found")
    iaP = np.asarray(config["iaP"])
    nocc, nvir, naux = iaP.shape
    abP = config.get("abP")
    if abP is None:
        abP = np.zeros((nvir * nvir, naux))
    return evgw(config["mo_energy"], config["mo_occ"], iaP.reshape(nocc * nvir, naux), config["ijP"],
                abP, config["chol_v"], config["vxc_dft"], max_cycle=config.get("max_cycle", 12),
                conv_tol=config.get("conv_tol", 1e-4), damping=config.get("damping", 0.5),
                diis=config.get("diis", True), diis_space=config.get("diis_space", 6),
                nfreq=config.get("nfreq", 48),
                frontier_convergence=config.get("frontier_convergence", True),
                frontier_window=config.get("frontier_window", 0.1),
                qp_solver=config.get("qp_solver", "linearized"),
                newton_max_iterations=config.get("newton_max_iterations", 50),
                newton_energy_tolerance=config.get("newton_energy_tolerance", 1e-8),
                npade=config.get("npade"), iw_cutoff=config.get("iw_cutoff", 5.0))


# ---------------------------------------------------------------------------
# a5: contour deformation (imaginary-axis term + residues)
# ---------------------------------------------------------------------------
def wc_pairs_imag(mo_energy, lpq, nocc, targets, freqs):
    """Wc_nm(iw) for every target n, every m and every frequency: [nw, ntarget, nmo]."""
    naux = lpq.shape[0]
    out = np.zeros((len(freqs), len(targets), lpq.shape[1]))
    for w, f in enumerate(freqs):
        wc = epsilon_inverse_minus_identity(get_rho_response(f, mo_energy, lpq[:, :nocc, nocc:]))
        for t, n in enumerate(targets):
            out[w, t] = np.sum((wc.T @ lpq[:, n, :]) * lpq[:, :, n], axis=0)
    return out


def wc_pair_real(mo_energy, lpq, nocc, n, m, omega_r) -> Tuple[float, float]:
    """Wc_nm at the real frequency omega_r and its derivative d/d omega_r.

    eps(w) = I - Pi(w) with chi_ia = e_ia/(e_ia^2 - w^2); solved by LU (eps is
    not positive definite on the real axis above the lowest transition).
    dWc/dw = x^T (dPi/dw) x with x = eps^-1 B_nm.
    """
    lov = lpq[:, :nocc, nocc:]
    naux = lpq.shape[0]
    pi = get_rho_response_real(omega_r, mo_energy, lov)
    eps = np.eye(naux) - pi
    b = lpq[:, n, m]
    x = np.linalg.solve(eps, b)
    wc = float(b @ x - b @ b)
    e_ia = (mo_energy[:nocc, None] - mo_energy[None, nocc:]).reshape(-1)
    dchi = e_ia * 2.0 * omega_r / (e_ia * e_ia - omega_r * omega_r) ** 2
    flat = lov.reshape(naux, -1)
    t = flat.T @ x
    dwc = float(4.0 * np.sum(dchi * t * t))
    return wc, dwc


def sigma_cd(omega: float, n: int, mo_energy, lpq, nocc, freqs, wts, wc_imag_n
             ) -> Tuple[float, float]:
    """Sigma_c^CD(omega) for target n and its derivative d/d omega.

    Sigma = I + R with
      I(w) = -(1/pi) sum_k wts_k sum_m Wc_nm(i f_k) (w - e_m)/((w - e_m)^2 + f_k^2)
      R(w) = - sum_{m occ, e_m > w} Wc_nm(|w - e_m|) + sum_{m vir, e_m < w} Wc_nm(|w - e_m|)
    (full-frequency contour deformation, e.g. Golze et al., JCTC 14, 4856 (2018);
    the imaginary-axis integrand is the reference's, correlation_pyscf_cd.rs:164-259,
    evaluated at the real target energy with eta -> 0).  wc_imag_n is [nw, nmo].
    """
    x = omega - mo_energy
    den = x[None, :] ** 2 + freqs[:, None] ** 2
    integ = (-1.0 / PI) * np.sum(wts[:, None] * wc_imag_n * x[None, :] / den)
    dinteg = (-1.0 / PI) * np.sum(wts[:, None] * wc_imag_n * (freqs[:, None] ** 2 - x[None, :] ** 2) / den ** 2)
    res = 0.0
    dres = 0.0
    nmo = mo_energy.shape[0]
    for m in range(nmo):
        em = mo_energy[m]
        if m < nocc and em > omega:
            wr, dwr = wc_pair_real(mo_energy, lpq, nocc, n, m, em - omega)
            res -= wr
            dres += dwr  # d/dw of -Wc(e_m - w) = +Wc'(e_m - w)
        elif m >= nocc and em < omega:
            wr, dwr = wc_pair_real(mo_energy, lpq, nocc, n, m, omega - em)
            res += wr
            dres += dwr
    return integ + res, dinteg + dres


def g0w0_cd(mo_energy, lpq, nocc, targets, nw, x0=0.5, vxc=None, sigma_x=None,
            tol=1e-8, max_iter=50, qp_solver="newton", z_min=0.1, z_max=0.999) -> Dict:
    """G0W0 by contour deformation for ``targets``, f(E) = E - e_n - Sx_n -
    Sigma_c^CD(E) + Vxc_n, with the analytic slope of Sigma^CD.

    qp_solver "newton": the step rule of NewtonQPSolver::solve
    (quasix_core/src/qp/newton_solver.rs:174-280): step -f/f' (or
    -sign(f) min(1, |f|) when |f'| < 1e-10) clipped to +-1 Ha, times an
    adaptive damping that starts at 1, halves when |f| grew and grows by 1.2
    when |f| more than halved, within [0.1, 1]; converged when |f| < tol.
    qp_solver "linearized": E = e_n + Z (Sx_n + Sigma(e_n) - Vxc_n), the
    linearized QP of qp/evgw.rs:784-821.  Z = 1/(1 - dSigma/dw) clipped to
    [z_min, z_max] in both (newton_solver.rs:306-315).  Sigma_x from the
    exchange of quasix_core/src/qp/evgw.rs:1167-1193; Vxc = 0 unless given."""
    nmo = mo_energy.shape[0]
    freqs, wts = get_scaled_legendre_roots(nw, x0)
    if sigma_x is None:
        sigma_x = np.diag(compute_exchange(np.ascontiguousarray(lpq[:, :, :nocc].transpose(1, 2, 0))))
    if vxc is None:
        vxc = np.zeros(nmo)
    wci = wc_pairs_imag(mo_energy, lpq, nocc, targets, freqs)
    qp = np.zeros(len(targets))
    zf = np.zeros(len(targets))
    sc_out = np.zeros(len(targets))
    iters = np.zeros(len(targets), dtype=np.int64)
    for t, n in enumerate(targets):
        e = mo_energy[n]
        if qp_solver == "linearized":
            s, ds = sigma_cd(e, n, mo_energy, lpq, nocc, freqs, wts, wci[:, t])
            z = min(max(1.0 / (1.0 - ds), z_min), z_max)
            qp[t] = e + z * (sigma_x[n] + s - vxc[n])
            zf[t] = z
            sc_out[t] = s
            iters[t] = 1
            continue
        damping, prev = 1.0, np.inf
        it = 0
        for it in range(max_iter):
            s, ds = sigma_cd(e, n, mo_energy, lpq, nocc, freqs, wts, wci[:, t])
            f = e - mo_energy[n] - sigma_x[n] - s + vxc[n]
            if abs(f) < tol:
                break
            fp = 1.0 - ds
            step = -np.sign(f) * min(1.0, abs(f)) if abs(fp) < 1e-10 else -f / fp
            step = min(max(step, -1.0), 1.0)
            if abs(f) > prev:
                damping = max(damping * 0.5, 0.1)
            elif abs(f) < 0.5 * prev and damping < 1.0:
                damping = min(damping * 1.2, 1.0)
            e += damping * step
            prev = abs(f)
        s, ds = sigma_cd(e, n, mo_energy, lpq, nocc, freqs, wts, wci[:, t])
        qp[t] = e
        zf[t] = min(max(1.0 / (1.0 - ds), z_min), z_max)
        sc_out[t] = s
        iters[t] = it + 1
    return dict(qp_energies=qp, z_factors=zf, sigma_c=sc_out, sigma_x=sigma_x[list(targets)],
                iterations=iters)


def g0w0_cd_grad(mo_energy, lpq, nocc, targets, qp, dl_dqp, nw, x0=0.5):
    """Adjoint of the CD QP roots: gradient of L = sum_t dl_dqp[t] E_t with
    respect to the orbital energies and the symmetric tensor lpq, where E_t
    solves f_t(E) = E - e_n - Sx_n - Sigma_c^CD_n(E) + Vxc_n = 0 (Vxc held fixed).

    Implicit differentiation: dE_t = Z_t (de_n + dSx_n + dSigma_n|_E) with
    Z_t = 1 / (1 - dSigma_n/dE) unclipped, mu_t = dl_dqp[t] Z_t.  Sigma_n(E) =
    I_n + R_n (sigma_cd); through Wc_nm = b^T (eps^-1 - I) b with
    eps = I + B diag(chi) B^T, chi = -4 e_ia/(w^2 + e_ia^2) (imaginary axis) or
    -4 e_ia/(e_ia^2 - w^2) (residue shifts):
      dL/db_nm = 2 c (x - b),   dL/deps = G = -sum c x x^T,   x = eps^-1 b,
      dL/dB_ov = 2 G B_ov diag(chi),   dL/dchi_ia = b_ia^T G b_ia,
    with c the coefficient of Wc_nm in mu_t Sigma_n.  The residue shifts
    w_r = s_r (E - e_m) contribute -mu_t dWc_r/dw to e_m.  P0 and W are rebuilt
    per frequency.  Returns (grad_e [nmo], grad_lpq [naux, nmo, nmo] symmetric:
    dL = sum grad_lpq * dlpq for every symmetric dlpq)."""
    naux, nmo, _ = lpq.shape
    nvir = nmo - nocc
    freqs, wts = get_scaled_legendre_roots(nw, x0)
    B = np.ascontiguousarray(lpq[:, :nocc, nocc:]).reshape(naux, -1)
    e_ia = (mo_energy[:nocc, None] - mo_energy[None, nocc:]).reshape(-1)
    wci = wc_pairs_imag(mo_energy, lpq, nocc, targets, freqs)
    mu = np.zeros(len(targets))
    for t, n in enumerate(targets):
        _, ds = sigma_cd(qp[t], n, mo_energy, lpq, nocc, freqs, wts, wci[:, t])
        mu[t] = dl_dqp[t] / (1.0 - ds)
    g_e = np.zeros(nmo)
    g_l = np.zeros_like(lpq)
    g_b = np.zeros_like(B)
    g_eia = np.zeros_like(e_ia)
    for t, n in enumerate(targets):
        g_e[n] += mu[t]
        g_l[:, n, :nocc] += -2.0 * mu[t] * lpq[:, n, :nocc]
    eye = np.eye(naux)
    for k, f in enumerate(freqs):
        chi = -4.0 * e_ia / (f * f + e_ia * e_ia)
        dchi = -4.0 * (f * f - e_ia * e_ia) / (f * f + e_ia * e_ia) ** 2
        inv = np.linalg.inv(eye + (B * chi) @ B.T)
        G = np.zeros((naux, naux))
        for t, n in enumerate(targets):
            xr = qp[t] - mo_energy
            den = xr * xr + f * f
            c = mu[t] * (-1.0 / PI) * wts[k] * xr / den
            g_e += mu[t] * (1.0 / PI) * wts[k] * wci[k, t] * (f * f - xr * xr) / den ** 2
            bn = lpq[:, n, :]
            X = inv @ bn
            g_l[:, n, :] += 2.0 * c[None, :] * (X - bn)
            G -= (X * c[None, :]) @ X.T
        H = G @ B
        g_eia += np.sum(B * H, axis=0) * dchi
        g_b += 2.0 * H * chi[None, :]
    for t, n in enumerate(targets):
        E = qp[t]
        for m in range(nmo):
            em = mo_energy[m]
            if m < nocc and em > E:
                sgn, w = -1.0, em - E
            elif m >= nocc and em < E:
                sgn, w = 1.0, E - em
            else:
                continue
            chi = -4.0 * e_ia / (e_ia * e_ia - w * w)
            dchi_de = 4.0 * (e_ia * e_ia + w * w) / (e_ia * e_ia - w * w) ** 2
            b = lpq[:, n, m]
            x = np.linalg.solve(eye + (B * chi) @ B.T, b)
            tv = B.T @ x
            dwc = float(4.0 * np.sum(e_ia * 2.0 * w / (e_ia * e_ia - w * w) ** 2 * tv * tv))
            c = mu[t] * sgn
            g_e[m] += -mu[t] * dwc
            g_l[:, n, m] += 2.0 * c * (x - b)
            g_eia += -c * tv * tv * dchi_de
            g_b += -2.0 * c * np.outer(x, tv * chi)
    ge = g_eia.reshape(nocc, nvir)
    g_e[:nocc] += ge.sum(axis=1)
    g_e[nocc:] -= ge.sum(axis=0)
    g_l[:, :nocc, nocc:] += g_b.reshape(naux, nocc, nvir)
    g_l = 0.5 * (g_l + g_l.transpose(0, 2, 1))
    return g_e, g_l


# ---------------------------------------------------------------------------
# a11-a13: BSE-TDA
# ---------------------------------------------------------------------------
def bse_w0(lpq, mo_energy, nocc) -> np.ndarray:
    """W(w=0) = (I - Pi(0))^-1 in the RI-normalized basis (the screened-direct kernel)."""
    pi0 = get_rho_response(0.0, mo_energy, lpq[:, :nocc, nocc:])
    return epsilon_inverse_minus_identity(pi0) + np.eye(pi0.shape[0])


def bse_blocks(lpq, nocc):
    """df_ia [nov, naux], df_ij [nocc^2, naux], df_ab [nvir^2, naux] as the reference's kernel takes."""
    naux, nmo, _ = lpq.shape
    nvir = nmo - nocc
    df_ia = np.ascontiguousarray(lpq[:, :nocc, nocc:].reshape(naux, -1).T)
    df_ij = np.ascontiguousarray(lpq[:, :nocc, :nocc].reshape(naux, -1).T)
    df_ab = np.ascontiguousarray(lpq[:, nocc:, nocc:].reshape(naux, -1).T)
    return df_ia, df_ij, df_ab


def bse_apply_tda(x: np.ndarray, delta_qp, df_ia, df_ij, df_ab, w0, nocc, nvirt, alpha_x=2.0):
    """y = Delta x + alpha_x B_ia (B_ia^T x) - sum_jb (ij|W0|ab) x_jb.

    quasix_core/src/bse/kernel.rs:501-598 (exchange :344-365, direct :391-462).
    x is [nov] or [nov, nvec].
    """
    single = x.ndim == 1
    X = x[:, None] if single else x
    Y = delta_qp[:, None] * X
    if abs(alpha_x) > np.finfo(float).eps:
        Y = Y + alpha_x * (df_ia @ (df_ia.T @ X))
    naux = df_ia.shape[1]
    ijw = (df_ij @ w0).reshape(nocc, nocc, naux)
    ab = df_ab.reshape(nvirt, nvirt, naux)
    for v in range(X.shape[1]):
        xv = X[:, v].reshape(nocc, nvirt)
        t = np.einsum("abQ,jb->jaQ", ab, xv, optimize=True)
        Y[:, v] -= np.einsum("ijQ,jaQ->ia", ijw, t, optimize=True).reshape(-1)
    return Y[:, 0] if single else Y


def bse_root_grad(x, df_ia, df_ij, df_ab, w0, nocc, nvirt, mo_energy=None) -> np.ndarray:
    """dOmega/de_p for an eigenpair (Omega, x) of the BSE-TDA matrix
    A = diag(Delta) + alpha_x K^x - K^d(W0) (kernel.rs:501-598), by
    Hellmann-Feynman (no reference counterpart): dOmega = x^T dA x / x^T x.

    Delta_ia = e_a - e_i gives -sum_a x_ia^2 on e_i and +sum_i x_ia^2 on e_a.
    With mo_energy given, W0 = (I - Pi(0))^-1 is taken as built from mo_energy
    and df_ia (bse_w0): dOmega/dW0 = -M, M_PQ = sum x_ia x_jb B_ij^P B_ab^Q;
    through W0 = eps0^-1, dOmega/deps0 = W0 sym(M) W0 = G; eps0 = I + sum_ia
    chi_ia b_ia b_ia^T with chi_ia = 4/Delta_ia, so dOmega/dDelta_ia gains
    (b_ia^T G b_ia) (-4/Delta_ia^2)."""
    nov = nocc * nvirt
    x = np.asarray(x, dtype=np.float64).reshape(-1)
    xx = x / np.sqrt(x @ x)
    X = xx.reshape(nocc, nvirt)
    nmo = nocc + nvirt
    g = np.zeros(nmo)
    g[:nocc] -= np.sum(X * X, axis=1)
    g[nocc:] += np.sum(X * X, axis=0)
    if mo_energy is None:
        return g
    naux = df_ia.shape[1]
    ab = df_ab.reshape(nvirt, nvirt, naux)
    ij = df_ij.reshape(nocc, nocc, naux)
    T = np.einsum("ia,abQ,jb->ijQ", X, ab, X, optimize=True)
    M = np.einsum("ijP,ijQ->PQ", ij, T, optimize=True)
    Ms = 0.5 * (M + M.T)
    G = w0 @ Ms @ w0
    s = np.einsum("kP,PQ,kQ->k", df_ia, G, df_ia, optimize=True)
    delta = (mo_energy[None, nocc:] - mo_energy[:nocc, None]).reshape(-1)
    gd = (s * (-4.0 / delta ** 2)).reshape(nocc, nvirt)
    g[:nocc] -= gd.sum(axis=1)
    g[nocc:] += gd.sum(axis=0)
    return g


def bse_root_grad_blocks(x, df_ia, df_ij, df_ab, w0, nocc, nvirt, mo_energy=None, alpha_x=2.0):
    """dOmega/d(df_ia, df_ij, df_ab) for an eigenpair of A = diag(Delta) +
    alpha_x B_ia B_ia^T - K^d(W0) (kernel.rs:344-462), by Hellmann-Feynman on
    the normalised x (no reference counterpart):
      d/dB_ia^P = 2 alpha_x x_ia (B_ia^T x)_P [+ 8/Delta_ia (G B_ia)_P],
      d/dB_ij^P = -(T W0)_(ij)P,   T^Q_ij = sum_ab x_ia B_ab^Q x_jb,
      d/dB_ab^Q = -sum_ij x_ia (B_ij W0)^Q_ij x_jb,
    the bracket (G = W0 sym(M) W0, M_PQ = sum_ij B_ij^P T^Q_ij) when
    W0 = (I - Pi(0))^-1 follows df_ia (mo_energy given), as in bse_root_grad.
    Returns (grad_ia [nov, naux], grad_ij [nocc^2, naux], grad_ab [nvir^2, naux])."""
    x = np.asarray(x, dtype=np.float64).reshape(-1)
    xx = x / np.sqrt(x @ x)
    X = xx.reshape(nocc, nvirt)
    naux = df_ia.shape[1]
    ab = df_ab.reshape(nvirt, nvirt, naux)
    ij = df_ij.reshape(nocc, nocc, naux)
    u = df_ia.T @ xx
    g_ia = 2.0 * alpha_x * np.outer(xx, u)
    T = np.einsum("ia,abQ,jb->ijQ", X, ab, X, optimize=True)
    g_ij = -(T.reshape(nocc * nocc, naux) @ w0)
    U = (df_ij @ w0).reshape(nocc, nocc, naux)
    g_ab = -np.einsum("ia,ijQ,jb->abQ", X, U, X, optimize=True).reshape(nvirt * nvirt, naux)
    if mo_energy is not None:
        M = np.einsum("ijP,ijQ->PQ", ij, T, optimize=True)
        G = w0 @ (0.5 * (M + M.T)) @ w0
        delta = (mo_energy[None, nocc:] - mo_energy[:nocc, None]).reshape(-1)
        g_ia += (8.0 / delta)[:, None] * (df_ia @ G)
    return g_ia, g_ij, g_ab


@dataclass
class DavidsonConfig:
    """quasix_core/src/bse/davidson.rs:47-104."""
    n_roots: int = 3
    max_iter: int = 100
    max_space: int = 60
    tol_residual: float = 1e-5
    lindep_threshold: float = 1e-12
    level_shift: float = 0.001


def davidson_bse(apply_h, qp_gaps: np.ndarray, cfg: DavidsonConfig) -> Dict:
    """Block Davidson, quasix_core/src/bse/davidson.rs:372-508."""
    n = qp_gaps.shape[0]
    n_roots = min(cfg.n_roots, n)
    max_space = min(cfg.max_space, n)
    if n <= n_roots:
        h = apply_h(np.eye(n))
        h = 0.5 * (h + h.T)
        ev, vec = np.linalg.eigh(h)
        return dict(eigenvalues=ev, eigenvectors=vec, converged=[True] * n, iterations=1,
                    residual_norms=[0.0] * n)
    order = np.argsort(qp_gaps, kind="stable")
    V = np.zeros((n, n_roots))
    for i in range(n_roots):
        V[order[i], i] = 1.0
    evals = np.zeros(n_roots)
    evecs = np.zeros((n, n_roots))
    conv = [False] * n_roots
    rnorm = [float("inf")] * n_roots
    for iteration in range(cfg.max_iter):
        AV = apply_h(V)
        heff = V.T @ AV
        heff = 0.5 * (heff + heff.T)
        theta, Y = np.linalg.eigh(heff)
        nr = min(n_roots, Y.shape[1])
        X = V @ Y[:, :nr]
        AX = AV @ Y[:, :nr]
        new = []
        for j in range(n_roots):
            if j >= nr or conv[j]:
                continue
            r = AX[:, j] - theta[j] * X[:, j]
            rn = float(np.linalg.norm(r))
            rnorm[j] = rn
            if rn < cfg.tol_residual:
                conv[j] = True
                evals[j] = theta[j]
                evecs[:, j] = X[:, j]
                continue
            den = qp_gaps - theta[j] + cfg.level_shift
            den = np.where(np.abs(den) < 1e-8, np.where(den >= 0.0, 1e-8, -1e-8), den)
            t = r / den
            tn = np.linalg.norm(t)
            if tn > 1e-14:
                t = t / tn
            if np.linalg.norm(t) > cfg.lindep_threshold:
                new.append(t)
        if all(conv):
            return dict(eigenvalues=evals, eigenvectors=evecs, converged=conv,
                        iterations=iteration + 1, residual_norms=rnorm)
        if not new:
            continue
        if V.shape[1] + len(new) > max_space:
            q, _ = np.linalg.qr(X[:, :min(n_roots, X.shape[1])])
            V = q
            continue
        for t in new:
            for _ in range(2):
                t = _gs(V, t)
            nrm = np.linalg.norm(t)
            if nrm < cfg.lindep_threshold:
                continue
            V = np.column_stack([V, t / nrm])
    for j in range(n_roots):
        if not conv[j] and np.linalg.norm(evecs[:, j]) < 0.1:
            AV = apply_h(V)
            heff = V.T @ AV
            theta, Y = np.linalg.eigh(0.5 * (heff + heff.T))
            nr = min(n_roots, Y.shape[1])
            if j < nr:
                evals[j] = theta[j]
                evecs[:, j] = V @ Y[:, j]
    return dict(eigenvalues=evals, eigenvectors=evecs, converged=conv, iterations=cfg.max_iter,
                residual_norms=rnorm)


def _gs(V: np.ndarray, t: np.ndarray) -> np.ndarray:
    """One classical Gram-Schmidt pass, column by column (davidson.rs:248-252)."""
    for j in range(V.shape[1]):
        t = t - float(t @ V[:, j]) * V[:, j]
    return t


# ---------------------------------------------------------------------------
# f4: spectral functions (quasix_core/src/analysis/spectral.rs)
# ---------------------------------------------------------------------------
def gaussian_broadening(omega, energy, sigma):
    """spectral.rs:779-784 (scalar form; the reference's AVX2 path uses a fast exp)."""
    d = np.asarray(omega) - energy
    return np.exp(-d * d / (2.0 * sigma * sigma)) / (sigma * math.sqrt(2.0 * PI))


def lorentzian_broadening(omega, energy, gamma):
    """spectral.rs:796-799."""
    d = np.asarray(omega) - energy
    return (gamma / PI) / (d * d + gamma * gamma)


def voigt_profile(omega, energy, sigma, gamma, alpha):
    """spectral.rs:814-818: (1 - alpha) G + alpha L."""
    return (1.0 - alpha) * gaussian_broadening(omega, energy, sigma) + alpha * lorentzian_broadening(omega, energy,
                                                                                                   gamma)


def spectral_function(qp_energies, z_factors, omega, gaussian_width=0.1, lorentzian_width=0.05, voigt_mixing=0.5,
                      fermi_energy=0.0, kind=0):
    """SpectralAnalyzer::compute_spectral_function (spectral.rs:283-325) with the
    profile choice of :291-302 (Gaussian below mixing 0.01, Lorentzian above
    0.99, else Voigt) and, for kind 1 / 2, the state filter and energy shift of
    generate_pes_spectrum / generate_ipes_spectrum (:557-656).  Returns
    (weights [nomega], total_weight = sum * (omega[1] - omega[0]))."""
    e = np.asarray(qp_energies, float)
    z = np.asarray(z_factors, float)
    w = np.asarray(omega, float)
    if kind == 1:
        m = e <= fermi_energy
        e, z = fermi_energy - e[m], z[m]
    elif kind == 2:
        m = e > fermi_energy
        e, z = e[m] - fermi_energy, z[m]
    out = np.zeros_like(w)
    for ei, zi in zip(e, z):
        if voigt_mixing < 0.01:
            p = gaussian_broadening(w, ei, gaussian_width)
        elif voigt_mixing > 0.99:
            p = lorentzian_broadening(w, ei, lorentzian_width)
        else:
            p = voigt_profile(w, ei, gaussian_width, lorentzian_width, voigt_mixing)
        out += zi * p
    dw = w[1] - w[0] if w.shape[0] > 1 else 1.0
    return out, float(out.sum() * dw)


def spectral_function_states(qp_energies, z_factors, omega, eta=0.01):
    """EvGWResult.spectral_function (quasix/quasix/evgw.py:124-134): per state
    A[i, w] = Z_i eta / ((w - E_i)^2 + eta^2) / pi."""
    e = np.asarray(qp_energies, float)[:, None]
    z = np.asarray(z_factors, float)[:, None]
    w = np.asarray(omega, float)[None, :]
    return z * eta / ((w - e) ** 2 + eta ** 2) / PI


def spectral_function_pade(coeff, omega_fit, e_ref, sigma_x, vxc, ef, omega, eta):
    """A_t(w) = (1/pi) G / ((w - e_t - Sx_t + Vxc_t - Re S)^2 + G^2), G = |Im S| + eta,
    S = pade_thiele(w - ef) of orbital t (correlation_ac.rs:530-566 for S); no
    reference counterpart for A itself (the reference broadens QP peaks only)."""
    norbs = coeff.shape[1]
    out = np.zeros((norbs, len(omega)))
    for t in range(norbs):
        for q, w in enumerate(omega):
            s = pade_thiele(w - ef, omega_fit[t], coeff[:, t])
            re = w - e_ref[t] - sigma_x[t] + vxc[t] - s.real
            g = abs(s.imag) + eta
            out[t, q] = g / (PI * (re * re + g * g))
    return out


# ---------------------------------------------------------------------------
# f2: BSE optical properties (quasix_core/src/bse/optical.rs)
# ---------------------------------------------------------------------------
def compute_transition_dipoles(mo_coeff, ao_dipoles, nocc):
    """<i|r_c|a> = C_occ^T D_c C_vir, [nocc * nvirt, 3] (quasix/quasix/bse_driver.py:249-298)."""
    c = np.asarray(mo_coeff, float)
    out = np.zeros((nocc * (c.shape[1] - nocc), 3))
    for k in range(3):
        out[:, k] = (c[:, :nocc].T @ ao_dipoles[k] @ c[:, nocc:]).ravel()
    return out


def compute_oscillator_strengths(eigenvalues, eigenvectors, transition_dipoles):
    """optical.rs:179-247: d = X^T mu, f_n = 2/3 E_n |d_n|^2, with the
    reference's validation (dimension mismatch, 3 components, finite and
    non-negative eigenvalues)."""
    e = np.asarray(eigenvalues, float)
    x = np.asarray(eigenvectors, float)
    mu = np.asarray(transition_dipoles, float)
    if x.shape[1] != e.shape[0] or x.shape[0] != mu.shape[0] or mu.shape[1] != 3:
        raise ValueError("dimension mismatch")
    if not np.all(np.isfinite(e)) or np.any(e < 0.0):
        raise ValueError("eigenvalues must be finite and non-negative")
    d = x.T @ mu
    f = (2.0 / 3.0) * e * np.sum(d * d, axis=1)
    return f, d, float(f.sum())


def absorption_lorentzian(x, gamma):
    """optical.rs:121-123: gamma / (x^2 + gamma^2)."""
    return gamma / (x * x + gamma * gamma)


def absorption_gaussian(x, sigma):
    """optical.rs:131-133: exp(-x^2 / (2 sigma^2))."""
    return np.exp(-0.5 * x * x / (sigma * sigma))


def compute_absorption_spectrum(eigenvalues, oscillator_strengths, broadening, gaussian=False, energy_range=None,
                                n_points=1000):
    """optical.rs:305-385 (broadening in Hartree; automatic range :332-340)."""
    e = np.asarray(eigenvalues, float)
    f = np.asarray(oscillator_strengths, float)
    if energy_range is None:
        lo, hi = e.min(), e.max()
        pad = max((hi - lo) * 0.2, broadening * 5.0)
        e_min, e_max = max(lo - pad, 0.0), hi + pad
    else:
        e_min, e_max = energy_range
    de = (e_max - e_min) / (n_points - 1) if n_points > 1 else 0.0
    grid = e_min + np.arange(n_points) * de
    out = np.zeros(n_points)
    for en, fn in zip(e, f):
        x = grid - en
        out += fn * (absorption_gaussian(x, broadening) if gaussian else absorption_lorentzian(x, broadening))
    return grid, out


# ---------------------------------------------------------------------------
# f1: density-fitting tensors (quasix/quasix/evgw.py:1007-1100,
#     quasix_core/src/df/mo_transform.rs:136-282)
# ---------------------------------------------------------------------------
def metric_inv_sqrt(metric, thresh_df=1e-10):
    """J^-1/2 and J^1/2 by eigh with the eigenvalues clamped at thresh_df
    (evgw.py:1014-1046)."""
    lam, u = np.linalg.eigh(metric)
    lam = np.maximum(lam, thresh_df)
    return (u / np.sqrt(lam)) @ u.T, (u * np.sqrt(lam)) @ u.T


def transform_mo_3center(j3c_ao, c_occ, c_vir):
    """(ia|P) as [nocc*nvir, naux] (mo_transform.rs:136-282)."""
    out = np.einsum("uvP,ui,va->iaP", j3c_ao, c_occ, c_vir, optimize=True)
    return out.reshape(c_occ.shape[1] * c_vir.shape[1], j3c_ao.shape[2])


def build_lpq(j3c_ao, mo_coeff, metric, thresh_df=1e-10):
    """lpq[P, p, q] = sum_Q J^-1/2[Q, P] (C^T (uv|Q) C)[p, q] and chol_v = J^1/2:
    the J^-1/2 transformation of the AO integrals (evgw.py:1041-1050) followed
    by the per-P MO transform (:1068-1083), in the reference's order."""
    jm, jp = metric_inv_sqrt(metric, thresh_df)
    int3c = np.einsum("uvQ,QP->uvP", j3c_ao, jm, optimize=True)
    lpq = np.einsum("up,uvP,vq->Ppq", mo_coeff, int3c, mo_coeff, optimize=True)
    return lpq, jp
