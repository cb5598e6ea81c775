"""Density-fitting tensors on the GPU.

* ``transform_mo_3center``  quasix_core/src/df/mo_transform.rs:136-282
  ((uv|P) -> (ia|P) as [nocc*nvir, naux]).
* ``metric_inv_sqrt``       J^-1/2 and J^1/2 of the Coulomb metric
  (quasix/quasix/evgw.py:1014-1046).
* ``build_lpq`` / ``build_df_tensors``
                            the DF tensor build of quasix/quasix/evgw.py:
                            1007-1100 from given AO integrals: the
                            RI-normalised lpq [naux, nmo, nmo] that every GW /
                            BSE entry point takes, and the reference's
                            flattened blocks (iaP, miP, abP, chol_v).

The AO integrals (uv|P) [nao, nao, naux] and the metric (P|Q) come from the
caller (the reference takes them from PySCF, which is not part of this path).
"""
from __future__ import annotations

from typing import Optional, Tuple

import numpy as np

from . import _native as N


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def transform_mo_3center(j3c_ao, c_occ, c_vir, device: int = 0) -> np.ndarray:
    j, co, cv = _f64(j3c_ao), _f64(c_occ), _f64(c_vir)
    nao, nao2, naux = j.shape
    if nao != nao2:
        raise ValueError(f"3-center integrals must have square AO dimensions, got {list(j.shape)}")
    if co.shape[0] != nao or cv.shape[0] != nao:
        raise ValueError(f"MO coefficient dimensions don't match AO basis: AO={nao}, C_occ={co.shape[0]}, "
                         f"C_vir={cv.shape[0]}")
    ctx = N.context(device)
    out = np.zeros((co.shape[1] * cv.shape[1], naux))
    ctx.check(ctx.lib.qx_transform_mo_3center(ctx.handle, N.ptr(j), N.ptr(co), N.ptr(cv), nao, co.shape[1],
                                              cv.shape[1], naux, N.ptr(out)))
    return out


def metric_inv_sqrt(metric, thresh: float = 1e-10, device: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    """(J^-1/2, J^1/2) of the metric J."""
    m = _f64(metric)
    n = m.shape[0]
    ctx = N.context(device)
    a, b = np.zeros((n, n)), np.zeros((n, n))
    ctx.check(ctx.lib.qx_metric_inv_sqrt(ctx.handle, N.ptr(m), n, float(thresh), N.ptr(a), N.ptr(b)))
    return a, b


def build_lpq(j3c_ao, mo_coeff, metric=None, metric_inv_sqrt=None, thresh: float = 1e-10,
              device: int = 0) -> Tuple[np.ndarray, Optional[np.ndarray]]:
    """(lpq [naux, nmo, nmo], chol_v = J^1/2 or None).  Give the metric J or
    its inverse square root."""
    j, c = _f64(j3c_ao), _f64(mo_coeff)
    nao, _, naux = j.shape
    nmo = c.shape[1]
    if (metric is None) == (metric_inv_sqrt is None):
        raise ValueError("give exactly one of metric and metric_inv_sqrt")
    m = None if metric is None else _f64(metric)
    mi = None if metric_inv_sqrt is None else _f64(metric_inv_sqrt)
    ctx = N.context(device)
    lpq = np.zeros((naux, nmo, nmo))
    chol = None if m is None else np.zeros((naux, naux))
    ctx.check(ctx.lib.qx_build_lpq(ctx.handle, N.ptr(j), N.ptr(c), N.ptr(m), N.ptr(mi), nao, nmo, naux,
                                   float(thresh), N.ptr(lpq), N.ptr(chol)))
    return lpq, chol


def build_df_tensors(j3c_ao, mo_coeff, mo_occ, metric, thresh: float = 1e-10, device: int = 0):
    """The return of the reference's DF build (evgw.py:1085-1100):
    (iaP [nocc*nvir, naux], miP [nmo*nocc, naux], abP [nvir*nvir, naux], chol_v)."""
    nocc = int(np.sum(np.asarray(mo_occ) > 0))
    lpq, chol = build_lpq(j3c_ao, mo_coeff, metric=metric, thresh=thresh, device=device)
    naux, nmo, _ = lpq.shape
    nvir = nmo - nocc
    t = lpq.transpose(1, 2, 0)
    iaP = np.ascontiguousarray(t[:nocc, nocc:]).reshape(nocc * nvir, naux)
    miP = np.ascontiguousarray(t[:, :nocc]).reshape(nmo * nocc, naux)
    abP = np.ascontiguousarray(t[nocc:, nocc:]).reshape(nvir * nvir, naux)
    return iaP, miP, abP, chol
