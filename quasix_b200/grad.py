"""Gradients of contour-deformation QP energies (qx_g0w0_cd_grad) and of
the lowest BSE-TDA excitation energy (qx_bse_root_grad_b).

``g0w0_cd_grad`` returns dL/d(mo_energy) and dL/d(lpq) for L = sum_t
dl_dqp[t] E_t, where E_t are the Newton roots of qx_g0w0_cd with Vxc held
fixed.  ``G0W0CDQP`` wraps the forward root and the adjoint as a
``torch.autograd.Function``; ``g0w0_cd_qp`` is its functional form.
``BSELowestRoot`` / ``bse_lowest_root`` do the same for the lowest singlet
BSE-TDA root, with respect to mo_energy and lpq (W0 = (I - Pi(0))^-1 follows
both).

The reference (QuasiX) has no derivative code; the forward path it
differentiates is the CD self-energy of
quasix_core/src/selfenergy/correlation_pyscf_cd.rs:164-259 plus residues.
"""
from __future__ import annotations

from typing import Sequence, Tuple

import numpy as np

from . import _native as N
from .gw import _ctx, _f64, _prec, g0w0_cd


def _is_tensor(a) -> bool:
    return hasattr(a, "data_ptr")


def _dev_index(dev) -> int:
    return (dev.index or 0) if dev.type == "cuda" else 0


def g0w0_cd_grad(mo_energy, lpq, nocc: int, targets: Sequence[int], qp_energies, dl_dqp, nw: int = 24,
                 x0: float = 0.5, precision="fp64", device: int = 0, want_lpq: bool = True):
    """(grad_energy [nmo], grad_lpq [naux, nmo, nmo] or None, z_raw [ntarget]).

    Outputs are CUDA tensors when ``lpq`` is a CUDA tensor, else numpy arrays.
    grad_lpq is symmetric in its last two indices: dL = sum(grad_lpq * dlpq)
    for every symmetric perturbation dlpq."""
    ctx = _ctx(device, lpq, mo_energy)
    on_dev = _is_tensor(lpq) and lpq.is_cuda
    lpq_a = lpq if _is_tensor(lpq) else _f64(lpq)
    naux, nmo, _ = tuple(lpq_a.shape)
    e = mo_energy if _is_tensor(mo_energy) else _f64(mo_energy)
    t = np.ascontiguousarray(np.asarray(targets, dtype=np.int32))
    qp = np.ascontiguousarray(np.asarray(qp_energies.detach().cpu() if _is_tensor(qp_energies) else qp_energies,
                                         dtype=np.float64))
    lam = np.ascontiguousarray(np.asarray(dl_dqp.detach().cpu() if _is_tensor(dl_dqp) else dl_dqp,
                                          dtype=np.float64))
    if on_dev:
        import torch
        ge = torch.zeros(nmo, dtype=torch.float64, device=lpq.device)
        gl = torch.zeros((naux, nmo, nmo), dtype=torch.float64, device=lpq.device) if want_lpq else None
    else:
        ge = np.zeros(nmo)
        gl = np.zeros((naux, nmo, nmo)) if want_lpq else None
    z = np.zeros(len(t))
    ctx.check(ctx.lib.qx_g0w0_cd_grad(ctx.handle, N.ptr(e), N.ptr(lpq_a), nmo, int(nocc), naux, N.ptr(t), len(t),
                                      N.ptr(qp), N.ptr(lam), int(nw), float(x0), _prec(precision), N.ptr(ge),
                                      N.ptr(gl) if gl is not None else None, N.ptr(z)))
    return ge, gl, z


def _torch_function():
    import torch

    class G0W0CDQP(torch.autograd.Function):
        """E_t = CD QP roots (Newton) of ``targets``; backward by the adjoint.

        forward(mo_energy [nmo], lpq [naux, nmo, nmo], nocc, targets, nw, vxc,
        tol, max_iter, precision) -> qp [ntarget] (float64, on lpq's device).
        Gradients flow to mo_energy and lpq (symmetric gradient)."""

        @staticmethod
        def forward(ctx, mo_energy, lpq, nocc, targets, nw=24, vxc=None, tol=1e-12, max_iter=100,
                    precision="fp64"):
            dev = lpq.device
            r = g0w0_cd(mo_energy.detach().contiguous(), lpq.detach().contiguous(), nocc, targets, nw=nw,
                        vxc=None if vxc is None else vxc.detach().contiguous(), tol=tol, max_iter=max_iter,
                        precision=precision, device=_dev_index(dev))
            qp = torch.as_tensor(r["qp_energies"], dtype=torch.float64, device=dev)
            ctx.save_for_backward(mo_energy.detach(), lpq.detach(), qp)
            ctx.cfg = (nocc, list(targets), nw, precision)
            return qp

        @staticmethod
        def backward(ctx, grad_qp):
            mo_energy, lpq, qp = ctx.saved_tensors
            nocc, targets, nw, precision = ctx.cfg
            dev = lpq.device
            ge, gl, _ = g0w0_cd_grad(mo_energy.contiguous(), lpq.contiguous(), nocc, targets, qp, grad_qp,
                                     nw=nw, precision=precision, device=_dev_index(dev),
                                     want_lpq=ctx.needs_input_grad[1])
            ge = torch.as_tensor(ge, device=mo_energy.device) if ctx.needs_input_grad[0] else None
            gl = torch.as_tensor(gl, device=lpq.device) if gl is not None else None
            return ge, gl, None, None, None, None, None, None, None

    return G0W0CDQP


_FN = None


def G0W0CDQP():
    """The torch.autograd.Function class (created on first use: torch is optional)."""
    global _FN
    if _FN is None:
        _FN = _torch_function()
    return _FN


def g0w0_cd_qp(mo_energy, lpq, nocc: int, targets: Sequence[int], nw: int = 24, vxc=None, tol: float = 1e-12,
               max_iter: int = 100, precision="fp64"):
    """Differentiable CD QP energies of ``targets`` (torch tensors in, tensor out)."""
    return G0W0CDQP().apply(mo_energy, lpq, nocc, list(targets), nw, vxc, tol, max_iter, precision)


# ---------------------------------------------------------------------------
# Lowest BSE-TDA root with respect to the orbital energies and lpq.
# ---------------------------------------------------------------------------
def bse_blocks_t(lpq, nocc: int):
    """The DF blocks of BSETDAKernel::new (quasix_core/src/bse/kernel.rs:259-337)
    cut from lpq [naux, nmo, nmo] (torch tensor, kept on its device):
    df_ia [nocc*nvir, naux], df_ij [nocc^2, naux], df_ab [nvir^2, naux]."""
    naux = lpq.shape[0]
    t = lpq.permute(1, 2, 0)
    return (t[:nocc, nocc:].reshape(-1, naux).contiguous(), t[:nocc, :nocc].reshape(-1, naux).contiguous(),
            t[nocc:, nocc:].reshape(-1, naux).contiguous())


def bse_lpq_gradient(g_ia, g_ij, g_ab, nocc: int, nmo: int):
    """dL/dlpq [naux, nmo, nmo] from the gradients of the three blocks, in the
    symmetric convention (dL = sum(grad * dlpq) for every symmetric dlpq): the
    ia block feeds both (i, a) and (a, i); the ij and ab blocks are symmetrised."""
    import torch
    naux = g_ia.shape[1]
    nvir = nmo - nocc
    out = torch.zeros((naux, nmo, nmo), dtype=torch.float64, device=g_ia.device)
    gia = g_ia.T.reshape(naux, nocc, nvir)
    out[:, :nocc, nocc:] += 0.5 * gia
    out[:, nocc:, :nocc] += 0.5 * gia.transpose(1, 2)
    gij = g_ij.T.reshape(naux, nocc, nocc)
    out[:, :nocc, :nocc] += 0.5 * (gij + gij.transpose(1, 2))
    gab = g_ab.T.reshape(naux, nvir, nvir)
    out[:, nocc:, nocc:] += 0.5 * (gab + gab.transpose(1, 2))
    return out


def _bse_function():
    import torch

    from .bse import BSETDAKernel, DavidsonConfig, screened_w0

    class BSELowestRoot(torch.autograd.Function):
        """Omega = lowest root of the singlet BSE-TDA matrix built from
        (mo_energy, lpq): Delta_ia = e_a - e_i, K^x and K^d from lpq's blocks,
        W0 = (I - Pi(0))^-1 of mo_energy and the ov block.  Forward: device
        Davidson; backward: the Hellmann-Feynman gradients of
        qx_bse_root_grad_b, W0's dependence included.

        forward(mo_energy [nmo], lpq [naux, nmo, nmo], nocc, precision, tol,
        max_iter) -> Omega (0-d float64 tensor on lpq's device)."""

        @staticmethod
        def forward(ctx, mo_energy, lpq, nocc, precision="fp64", tol=1e-10, max_iter=300):
            dev = lpq.device
            e = mo_energy.detach().to(dev).contiguous()
            l = lpq.detach().contiguous()
            nmo = l.shape[1]
            nvir = nmo - nocc
            dia, dij, dab = bse_blocks_t(l, nocc)
            e_h = e.cpu().numpy()
            w0 = screened_w0(e_h, np.ascontiguousarray(l[:, :nocc, nocc:].cpu().numpy()), device=_dev_index(dev))
            delta = (e_h[None, nocc:] - e_h[:nocc, None]).reshape(-1)
            k = BSETDAKernel(nocc, nvir, l.shape[0], delta, dia, dij, dab, w0, precision=precision,
                             device=_dev_index(dev))
            # A block of four roots (and a subspace of 80) converges the lowest
            # one far faster than a single-root Davidson restarting every 20
            # vectors; a root short of tol would make the gradient inexact.
            nroots = min(4, nvir * nocc)
            r = k.solve_davidson_with_config(DavidsonConfig(nroots, max_iter, 20 * nroots, tol))
            if not r["converged"][0]:
                k.close()
                raise RuntimeError(f"ConvergenceError: the lowest BSE root did not reach tol {tol:g} in {max_iter} "
                                   f"iterations (residual {r['residual_norms'][0]:.2e})")
            ctx.kernel = k
            ctx.x = np.ascontiguousarray(r["eigenvectors"][:, 0])
            ctx.e = e_h
            ctx.nocc = nocc
            ctx.nmo = nmo
            return torch.as_tensor(float(r["eigenvalues"][0]), dtype=torch.float64, device=dev)

        @staticmethod
        def backward(ctx, grad_out):
            k = ctx.kernel
            ge, gia, gij, gab = k.root_gradient_blocks(ctx.x, mo_energy=ctx.e)
            k.close()
            ctx.kernel = None
            g = float(grad_out)
            dev = grad_out.device
            d_e = torch.as_tensor(ge * g, device=dev) if ctx.needs_input_grad[0] else None
            d_l = None
            if ctx.needs_input_grad[1]:
                t = [torch.as_tensor(a * g, device=dev) for a in (gia, gij, gab)]
                d_l = bse_lpq_gradient(t[0], t[1], t[2], ctx.nocc, ctx.nmo)
            return d_e, d_l, None, None, None, None

    return BSELowestRoot


_BSE_FN = None


def BSELowestRoot():
    """The torch.autograd.Function class of the lowest BSE-TDA root."""
    global _BSE_FN
    if _BSE_FN is None:
        _BSE_FN = _bse_function()
    return _BSE_FN


def bse_lowest_root(mo_energy, lpq, nocc: int, precision="fp64", tol: float = 1e-10, max_iter: int = 300):
    """Differentiable lowest singlet BSE-TDA excitation energy (torch tensors in)."""
    return BSELowestRoot().apply(mo_energy, lpq, nocc, precision, tol, max_iter)
