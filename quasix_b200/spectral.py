"""Spectral functions on the GPU, with the reference's analysis API.

* ``SpectralAnalyzer`` / ``BroadeningParams``
      quasix_core/src/analysis/spectral.rs:115-656 (compute_spectral_function,
      generate_pes_spectrum, generate_ipes_spectrum); the broadened sum runs in
      ``qx_spectral_function``.
* ``spectral_function_states``
      EvGWResult.spectral_function, quasix/quasix/evgw.py:124-134
      (``qx_spectral_function_states``).
* ``spectral_function_pade``
      A_n(w) of each orbital from the Pade continuation of its Sigma_c
      (``qx_spectral_function_pade``; the reference has no such form).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


@dataclass
class BroadeningParams:
    """spectral.rs:115-166 (energies in the caller's unit)."""
    gaussian_width: float = 0.1
    lorentzian_width: float = 0.05
    temperature: float = 300.0
    voigt_mixing: float = 0.5

    def validate(self) -> None:
        if self.gaussian_width <= 0.0:
            raise ValueError(f"Invalid broadening parameter gaussian_width: {self.gaussian_width}")
        if self.lorentzian_width <= 0.0:
            raise ValueError(f"Invalid broadening parameter lorentzian_width: {self.lorentzian_width}")
        if self.temperature < 0.0:
            raise ValueError(f"Invalid broadening parameter temperature: {self.temperature}")
        if not 0.0 <= self.voigt_mixing <= 1.0:
            raise ValueError(f"Invalid broadening parameter voigt_mixing: {self.voigt_mixing}")


@dataclass
class SpectralMetadata:
    """spectral.rs:184-197."""
    n_states: int
    fermi_energy: float
    broadening: BroadeningParams
    total_weight: float
    energy_unit: str = "eV"


@dataclass
class SpectralFunction:
    """spectral.rs:173-182."""
    omega_grid: np.ndarray
    spectral_weights: np.ndarray
    metadata: SpectralMetadata


class SpectralAnalyzer:
    """spectral.rs:214-656: broadened quasiparticle peaks sum_n Z_n P(w - E_n)."""

    def __init__(self, qp_energies, z_factors, fermi_energy: float, device: int = 0):
        e = _f64(qp_energies)
        z = _f64(z_factors)
        if e.shape != z.shape:
            raise ValueError(f"Dimension mismatch: energies ({e.shape[0]}) != z_factors ({z.shape[0]})")
        for i, v in enumerate(z):
            if not 0.0 <= v <= 1.0:
                raise ValueError(f"Invalid Z-factor {v} at index {i}: must be in range (0, 1)")
        self.qp_energies, self.z_factors, self.fermi_energy = e, z, float(fermi_energy)
        self.broadening = BroadeningParams()
        self.device = device

    def set_broadening(self, broadening: BroadeningParams) -> None:
        broadening.validate()
        self.broadening = broadening

    def _run(self, omega_grid, kind: int) -> SpectralFunction:
        w = _f64(omega_grid)
        if w.shape[0] == 0:
            raise ValueError("Invalid omega grid: Empty omega grid")
        ctx = N.context(self.device)
        out = np.zeros_like(w)
        tw = C.c_double(0.0)
        b = self.broadening
        ctx.check(ctx.lib.qx_spectral_function(ctx.handle, N.ptr(self.qp_energies), N.ptr(self.z_factors),
                                               self.qp_energies.shape[0], self.fermi_energy, kind, N.ptr(w),
                                               w.shape[0], b.gaussian_width, b.lorentzian_width, b.voigt_mixing,
                                               N.ptr(out), C.byref(tw)))
        if kind == 0:
            n, ef = self.qp_energies.shape[0], self.fermi_energy
        elif kind == 1:
            n, ef = int(np.sum(self.qp_energies <= self.fermi_energy)), 0.0
        else:
            n, ef = int(np.sum(self.qp_energies > self.fermi_energy)), 0.0
        return SpectralFunction(w, out, SpectralMetadata(n, ef, b, tw.value))

    def compute_spectral_function(self, omega_grid) -> SpectralFunction:
        return self._run(omega_grid, 0)

    def generate_pes_spectrum(self, omega_min: float, omega_max: float, n_points: int) -> SpectralFunction:
        """Occupied states (E <= E_F) at binding energy E_F - E (spectral.rs:557-606)."""
        return self._run(np.linspace(omega_min, omega_max, n_points), 1)

    def generate_ipes_spectrum(self, omega_min: float, omega_max: float, n_points: int) -> SpectralFunction:
        """Unoccupied states (E > E_F) at E - E_F (spectral.rs:610-656)."""
        return self._run(np.linspace(omega_min, omega_max, n_points), 2)


def spectral_function_states(qp_energies, z_factors, omega, eta: float = 0.01, device: int = 0) -> np.ndarray:
    """Per-state Lorentzian peaks A [n_states, n_omega] (evgw.py:124-134)."""
    e, z, w = _f64(qp_energies), _f64(z_factors), _f64(omega)
    ctx = N.context(device)
    out = np.zeros((e.shape[0], w.shape[0]))
    ctx.check(ctx.lib.qx_spectral_function_states(ctx.handle, N.ptr(e), N.ptr(z), e.shape[0], N.ptr(w), w.shape[0],
                                                  float(eta), N.ptr(out)))
    return out


def spectral_function_pade(coeff, omega_fit, e_ref, sigma_x, omega, ef: float, vxc=None, eta: float = 0.01,
                           device: int = 0) -> np.ndarray:
    """A [norbs, n_omega] of each orbital from its Pade fit (coeff [nfit, norbs],
    omega_fit [norbs, nfit], as returned by ``ac_pade_thiele_diag``)."""
    c = np.ascontiguousarray(coeff, dtype=np.complex128)
    f = np.ascontiguousarray(omega_fit, dtype=np.complex128)
    nfit, norbs = c.shape
    e, sx, w = _f64(e_ref), _f64(sigma_x), _f64(omega)
    vx = None if vxc is None else _f64(vxc)
    ctx = N.context(device)
    out = np.zeros((norbs, w.shape[0]))
    ctx.check(ctx.lib.qx_spectral_function_pade(ctx.handle, norbs, nfit, N.ptr(c), N.ptr(f), N.ptr(e), N.ptr(sx),
                                                N.ptr(vx), float(ef), N.ptr(w), w.shape[0], float(eta), N.ptr(out)))
    return out
