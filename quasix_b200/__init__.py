"""quasix_b200: B200-native RI GW/BSE hot path of QuasiX (sm_100a CUDA behind a C ABI).

Drop-in entry points with the reference's names and argument meaning:
``run_evgw`` / ``evgw`` (quasix/src/evgw.rs), ``get_sigma_diag`` and friends
(quasix_core/src/selfenergy/correlation_ac.rs), ``g0w0_cd``, and the BSE-TDA
``bse.BSETDAKernel`` / ``run_bse_tda`` (quasix/src/bse.rs, quasix/quasix/bse_driver.py),
the spectral functions of quasix_core/src/analysis/spectral.rs (``spectral``),
the density-fitting tensor build (``df``), DF-tensor and result files (``io``),
and the adjoint of the CD QP roots (``grad``), which the reference does not have.
"""
from . import _native, bse, df, grad, io, spectral
from .bse import BSETDAConfig, BSETDAKernel, BSETDAResult, DavidsonConfig, davidson_bse, run_bse_tda
from .gw import (ac_pade_thiele_diag, compute_epsilon_inverse_minus_identity, compute_exchange_diag,
                 compute_screened_interaction, NewtonQPSolver, NewtonSolverConfig, newton_qp_solve,
                 cd_sigma, compute_polarizability_p0, evgw, g0w0_cd, g0w0_cd_batch, get_rho_response, get_rho_response_batch,
                 get_scaled_legendre_roots, get_sigma_diag, pade_thiele, run_evgw, run_evgw_blocks)
from .grad import BSELowestRoot, G0W0CDQP, bse_lowest_root, g0w0_cd_grad, g0w0_cd_qp

__all__ = [
    "bse", "df", "io", "spectral", "BSETDAConfig", "BSETDAKernel", "BSETDAResult", "DavidsonConfig", "davidson_bse", "run_bse_tda",
    "ac_pade_thiele_diag", "compute_epsilon_inverse_minus_identity", "compute_exchange_diag",
    "compute_screened_interaction", "NewtonQPSolver", "NewtonSolverConfig", "newton_qp_solve",
    "cd_sigma", "compute_polarizability_p0", "evgw", "g0w0_cd", "g0w0_cd_batch", "get_rho_response", "get_rho_response_batch",
    "get_scaled_legendre_roots", "get_sigma_diag", "pade_thiele", "run_evgw", "run_evgw_blocks",
    "grad", "G0W0CDQP", "g0w0_cd_grad", "g0w0_cd_qp", "BSELowestRoot", "bse_lowest_root",
]
