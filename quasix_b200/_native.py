"""ctypes binding of libqxgpu.so (the C ABI declared in include/qx_gw.h).

The library is built in-tree by ``quasix_b200/build.py``.  Loading fails
loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqxgpu.so")

QX_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "InvalidInput", 2: "DimensionMismatch", 3: "NumericalError", 4: "ConvergenceError",
    5: "NotImplemented", 6: "CudaError", 7: "NoDevice",
}
PREC = {"fp64": 0, "bf16x3": 1, "fp16x3": 2}
QP_SOLVER = {"newton": 0, "linearized": 1}
P0_FORM = {"auto": 0, "materialised": 1, "converter": 2, "pair": 3}
CONTRACTION_FORM = {"auto": 0, "single": 1, "pair": 2}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p


class QxError(RuntimeError):
    """Error returned through the C ABI (mirrors QuasixError variants)."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


class QxValueError(QxError, ValueError):
    pass


class EvgwConfig(C.Structure):
    _fields_ = [
        ("max_iterations", C.c_int), ("energy_tolerance", C.c_double), ("damping_factor", C.c_double),
        ("z_min", C.c_double), ("z_max", C.c_double), ("use_diis", C.c_int), ("diis_space_dim", C.c_int),
        ("frontier_convergence", C.c_int), ("frontier_window", C.c_double), ("nfreq", C.c_int),
        ("iw_cutoff", C.c_double), ("x0", C.c_double), ("use_solved_qp", C.c_int),
        ("newton_energy_tolerance", C.c_double), ("newton_max_iterations", C.c_int), ("npade", C.c_int),
        ("precision", C.c_int), ("fixed_iterations", C.c_int),
    ]


class EvgwResult(C.Structure):
    _fields_ = [
        ("qp_energies", _dp), ("z_factors", _dp), ("sigma_x", _dp), ("sigma_c", _dp),
        ("history_energies", _dp), ("history_max_change", _dp), ("history_rms_change", _dp),
        ("n_iterations", C.c_int), ("converged", C.c_int),
    ]


class DavidsonConfig(C.Structure):
    _fields_ = [("n_roots", C.c_int), ("max_iter", C.c_int), ("max_space", C.c_int),
                ("tol_residual", C.c_double), ("lindep_threshold", C.c_double), ("level_shift", C.c_double)]


class NewtonConfig(C.Structure):
    _fields_ = [
        ("max_iterations", C.c_int), ("energy_tolerance", C.c_double), ("initial_damping", C.c_double),
        ("min_damping", C.c_double), ("max_damping", C.c_double), ("max_step", C.c_double),
        ("derivative_delta", C.c_double), ("use_richardson", C.c_int), ("z_min", C.c_double),
        ("z_max", C.c_double), ("use_bisection_fallback", C.c_int), ("max_bisection_iterations", C.c_int),
    ]


class CdSystem(C.Structure):
    _fields_ = [
        ("mo_energy", _vp), ("lpq", _vp), ("vxc", _vp), ("nmo", C.c_int), ("nocc", C.c_int), ("naux", C.c_int),
        ("targets", _vp), ("ntarget", C.c_int), ("qp_energies", _vp), ("z_factors", _vp), ("sigma_c", _vp),
        ("sigma_x", _vp), ("status", C.c_int),
    ]


# qx_apply_fn: int (*)(void* user, const double* x, double* y, int nvec, int ld).
APPLY_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int)


# Every symbol the header declares, with its ctypes signature.
SIGNATURES = {
    "qx_ctx_create": (C.c_int, [C.POINTER(_vp), C.c_int]),
    "qx_ctx_destroy": (C.c_int, [_vp]),
    "qx_last_error": (C.c_char_p, [_vp]),
    "qx_ctx_set_stream": (C.c_int, [_vp, _vp]),
    "qx_ctx_last_timings": (C.c_int, [_vp, _dp, _dp, _dp, _dp, _dp]),
    "qx_ctx_last_launches": (C.c_int64, [_vp]),
    "qx_ctx_last_guard_stats": (C.c_int, [_vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "qx_ctx_set_p0_form": (C.c_int, [_vp, C.c_int]),
    "qx_ctx_set_contraction_form": (C.c_int, [_vp, C.c_int]),
    "qx_version": (C.c_char_p, []),
    "qx_get_scaled_legendre_roots": (C.c_int, [C.c_int, C.c_double, _vp, _vp]),
    "qx_get_rho_response": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp]),
    "qx_screened_interaction": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _vp]),
    "qx_screened_interaction_noalloc": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _vp]),
    "qx_eps_at_least_identity": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double]),
    "qx_compute_screened_interaction": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _vp, _vp]),
    "qx_get_sigma_diag": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                    C.c_double, C.c_int, _vp, _vp, C.c_int, _ip]),
    "qx_ac_pade_thiele_diag": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _vp, C.c_int, _vp, _vp, C.c_int, _ip]),
    "qx_pade_thiele": (C.c_int, [_vp, C.c_int, _vp, _vp, C.c_int, _vp, _vp]),
    "qx_newton_qp_solve": (C.c_int, [_vp, C.POINTER(NewtonConfig), C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp,
                                     C.c_double, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "qx_spectral_function": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_double, C.c_int, _vp, C.c_int, C.c_double,
                                       C.c_double, C.c_double, _vp, _dp]),
    "qx_spectral_function_states": (C.c_int, [_vp, _vp, _vp, C.c_int, _vp, C.c_int, C.c_double, _vp]),
    "qx_spectral_function_pade": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, C.c_double, _vp,
                                            C.c_int, C.c_double, _vp]),
    "qx_compute_exchange_diag": (C.c_int, [_vp, _vp, C.c_int, C.c_int, C.c_int, _vp]),
    "qx_evgw_config_default": (None, [C.POINTER(EvgwConfig)]),
    "qx_evgw": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.POINTER(EvgwConfig),
                          C.POINTER(EvgwResult)]),
    "qx_g0w0_cd": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_int, _vp, C.c_int, C.c_int, C.c_double,
                             C.c_double, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp]),
    "qx_g0w0_cd_batch": (C.c_int, [_vp, C.POINTER(CdSystem), C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                   C.c_int, C.c_int, C.c_int]),
    "qx_cd_sigma": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, _vp, C.c_int, _vp, C.c_int, C.c_double,
                              C.c_int, _vp, _vp, _vp]),
    "qx_g0w0_cd_grad": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, _vp, C.c_int, _vp, _vp, C.c_int,
                                  C.c_double, C.c_int, _vp, _vp, _vp]),
    "qx_bse_create": (C.c_int, [_vp, C.POINTER(_vp), C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, C.c_int,
                                C.c_int]),
    "qx_bse_destroy": (C.c_int, [_vp]),
    "qx_bse_apply": (C.c_int, [_vp, _vp, _vp, C.c_int]),
    "qx_davidson_config_default": (None, [C.POINTER(DavidsonConfig)]),
    "qx_bse_davidson": (C.c_int, [_vp, C.POINTER(DavidsonConfig), _vp, _vp, _vp, _vp, _ip]),
    "qx_davidson": (C.c_int, [_vp, C.c_int, _vp, APPLY_FN, _vp, C.POINTER(DavidsonConfig), _vp, _vp, _vp, _vp, _ip]),
    "qx_bse_root_grad": (C.c_int, [_vp, _vp, _vp, _vp]),
    "qx_bse_root_grad_b": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "qx_bse_w0": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, _vp]),
    "qx_compute_transition_dipoles": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, _vp]),
    "qx_transform_mo_3center": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp]),
    "qx_metric_inv_sqrt": (C.c_int, [_vp, _vp, C.c_int, C.c_double, _vp, _vp]),
    "qx_build_lpq": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_double, _vp, _vp]),
    "qx_compute_oscillator_strengths": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_int, _vp, _vp, _dp]),
    "qx_compute_absorption_spectrum": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, C.c_double, C.c_int, C.c_double,
                                                 C.c_double, C.c_int, _vp, _vp]),
}

_lib = None
_lock = threading.Lock()


def load(path: str = LIB_PATH):
    """Load the native library; raises if it is not built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise ImportError(f"libqxgpu.so is not built ({path}); run quasix_b200/build.py")
        lib = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def ptr(a) -> int:
    """Address of a numpy array (host) or torch tensor (host or device)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)}")


class Context:
    """One libqxgpu context (device, stream, cached workspace)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = _vp()
        st = self.lib.qx_ctx_create(C.byref(h), device)
        if st != QX_OK:
            raise QxError(st, f"qx_ctx_create(device={device}) failed")
        self.handle = h
        self.device = device

    def check(self, st: int):
        if st != QX_OK:
            msg = self.lib.qx_last_error(self.handle).decode(errors="replace")
            if st in (1, 2):
                raise QxValueError(st, msg)
            raise QxError(st, msg)

    def timings(self):
        vals = [C.c_double() for _ in range(5)]
        self.lib.qx_ctx_last_timings(self.handle, *[C.byref(v) for v in vals])
        return dict(zip(["p0", "inversion", "contraction", "sigma", "qp"], [v.value for v in vals]))

    def launches(self) -> int:
        return int(self.lib.qx_ctx_last_launches(self.handle))

    def set_p0_form(self, form: str):
        """'auto', 'materialised', 'pair' or 'converter' (qx_ctx_set_p0_form)."""
        self.check(self.lib.qx_ctx_set_p0_form(self.handle, P0_FORM[form]))

    def set_contraction_form(self, form: str):
        """'auto', 'single' or 'pair' (qx_ctx_set_contraction_form)."""
        self.check(self.lib.qx_ctx_set_contraction_form(self.handle, CONTRACTION_FORM[form]))

    def guard_stats(self):
        """(guarded, reinverted): eps inversions of the last call that ran
        guarded, and those re-inverted with pivoting."""
        g, r = C.c_int64(0), C.c_int64(0)
        self.check(self.lib.qx_ctx_last_guard_stats(self.handle, C.byref(g), C.byref(r)))
        return int(g.value), int(r.value)

    def set_stream(self, stream_handle: int | None):
        self.check(self.lib.qx_ctx_set_stream(self.handle, stream_handle))

    def close(self):
        if getattr(self, "handle", None):
            self.lib.qx_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_contexts = {}


def context(device: int = 0) -> Context:
    with _lock:
        pass
    ctx = _contexts.get(device)
    if ctx is None:
        ctx = Context(device)
        _contexts[device] = ctx
    return ctx
