"""Seeded synthetic RI-GW systems.

The reference benchmarks molecules whose density-fitted tensors come from
PySCF; here those inputs are replaced by seeded synthetic systems with the
same shapes and value distributions:

* occupied orbital energies ~ U[-1.2, -0.3] Ha, virtual ~ U[0.05, 3.0] Ha,
  each block sorted ascending;
* B[P, p, q] = B[P, q, p] ~ N(0, 0.05^2): the upper triangle p <= q is drawn
  in the order (P, then row-major p <= q) and mirrored;
* B is rescaled so that the spectral norm of Pi(i*0) equals ``pi_norm``,
  where Pi(iw) = 4 * sum_ia B_ia e_ia / (w^2 + e_ia^2) B_ia^T with
  e_ia = eps_i - eps_a (the reference's sign convention,
  quasix_core/src/selfenergy/correlation_ac.rs:184-211).  Pi is quadratic in B,
  so the rescaling is exact and eps(0) = 1 - Pi(0) has eigenvalues in
  [1, 1 + pi_norm].

The tensor layout is the reference's ``lpq[naux, nmo, nmo]``
(quasix_core/src/qp/evgw.rs:539-543).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class SyntheticSystem:
    mo_energy: np.ndarray  # [nmo]
    lpq: np.ndarray  # [naux, nmo, nmo], symmetric in the last two indices
    nocc: int
    seed: int

    @property
    def nmo(self) -> int:
        return self.mo_energy.shape[0]

    @property
    def naux(self) -> int:
        return self.lpq.shape[0]

    @property
    def nvir(self) -> int:
        return self.nmo - self.nocc

    @property
    def mo_occ(self) -> np.ndarray:
        occ = np.zeros(self.nmo)
        occ[: self.nocc] = 2.0
        return occ

    # Block views in the layouts the reference's Python front ends pass in
    # (quasix/src/evgw.rs:103-140): iaP[nocc, nvir, naux], miP[nmo, nocc, naux],
    # abP[nvir, nvir, naux].
    def iaP(self) -> np.ndarray:
        o = self.nocc
        return np.ascontiguousarray(self.lpq[:, :o, o:].transpose(1, 2, 0))

    def miP(self) -> np.ndarray:
        o = self.nocc
        return np.ascontiguousarray(self.lpq[:, :, :o].transpose(1, 2, 0))

    def abP(self) -> np.ndarray:
        o = self.nocc
        return np.ascontiguousarray(self.lpq[:, o:, o:].transpose(1, 2, 0))

    def mn_full(self) -> np.ndarray:
        return np.ascontiguousarray(self.lpq.transpose(1, 2, 0))


def pi0_spectral_norm(mo_energy: np.ndarray, lpq: np.ndarray, nocc: int) -> float:
    """||Pi(i*0)||_2 for the occupied-virtual block of ``lpq``."""
    naux = lpq.shape[0]
    bov = lpq[:, :nocc, nocc:].reshape(naux, -1)
    e_ia = (mo_energy[:nocc, None] - mo_energy[None, nocc:]).reshape(-1)
    pi0 = 4.0 * (bov / e_ia) @ bov.T
    return float(np.abs(np.linalg.eigvalsh(pi0)).max())


def draw_system(nocc: int, nvir: int, naux: int, seed: int):
    """The seeded draws of one system, in the order (occupied energies, virtual
    energies, upper triangle of B by (P, then row-major p <= q)): returns
    (mo_energy [nmo], upper [naux, nmo (nmo + 1) / 2]) before the rescaling."""
    rng = np.random.default_rng(seed)
    nmo = nocc + nvir
    e_occ = np.sort(rng.uniform(-1.2, -0.3, nocc))
    e_vir = np.sort(rng.uniform(0.05, 3.0, nvir))
    upper = rng.normal(0.0, 0.05, size=(naux, nmo * (nmo + 1) // 2))
    return np.concatenate([e_occ, e_vir]), upper


def make_system(nocc: int, nvir: int, naux: int, seed: int, pi_norm: float) -> SyntheticSystem:
    """Build one seeded synthetic system (see module docstring)."""
    nmo = nocc + nvir
    mo_energy, upper = draw_system(nocc, nvir, naux, seed)
    iu, ju = np.triu_indices(nmo)
    lpq = np.empty((naux, nmo, nmo))
    lpq[:, iu, ju] = upper
    lpq[:, ju, iu] = upper
    scale = np.sqrt(pi_norm / pi0_spectral_norm(mo_energy, lpq, nocc))
    lpq *= scale
    return SyntheticSystem(mo_energy=mo_energy, lpq=lpq, nocc=nocc, seed=seed)


# Workloads, each named by what it is and its sizes.
def g0w0_cd_small() -> SyntheticSystem:
    """nocc 5, nvirt 19, naux 84, seed 0, ||Pi(0)|| = 2."""
    return make_system(5, 19, 84, seed=0, pi_norm=2.0)


def evgw_nmo300() -> SyntheticSystem:
    """nocc 40, nvirt 260, naux 1000, seed 1, ||Pi(0)|| = 4."""
    return make_system(40, 260, 1000, seed=1, pi_norm=4.0)


def batch64_shapes(seed0: int = 100, count: int = 64):
    """Shapes of the 64-system batch: nmo ~ U[40, 400] drawn from each system's seed,
    nocc = round(nmo / 6), naux = round(3.5 nmo), ||Pi(0)|| ~ U[1, 6]."""
    shapes = []
    for s in range(seed0, seed0 + count):
        rng = np.random.default_rng(s + 1_000_000)
        nmo = int(rng.integers(40, 401))
        pi_norm = float(rng.uniform(1.0, 6.0))
        nocc = int(round(nmo / 6))
        naux = int(round(3.5 * nmo))
        shapes.append((s, nocc, nmo - nocc, naux, pi_norm))
    return shapes


def batch64_system(index: int) -> SyntheticSystem:
    s, nocc, nvir, naux, pi_norm = batch64_shapes()[index]
    return make_system(nocc, nvir, naux, seed=s, pi_norm=pi_norm)


def grad_nmo200() -> SyntheticSystem:
    """nocc 30, nvirt 170, naux 700, seed 7 (pi norm as the small G0W0 case: 2)."""
    return make_system(30, 170, 700, seed=7, pi_norm=2.0)


def bse_dim26400_bov() -> SyntheticSystem:
    """nocc 60, nvirt 440, naux 1800, seed 11, ||Pi(0)|| = 5 (full tensor is 3.6 GB)."""
    return make_system(60, 440, 1800, seed=11, pi_norm=5.0)


def bse_blocks(lpq: np.ndarray, nocc: int):
    """The BSE kernel's DF blocks in the layouts of BSETDAKernel::new
    (quasix_core/src/bse/kernel.rs:259-337): df_ia [nocc*nvir, naux],
    df_ij [nocc*nocc, naux], df_ab [nvir*nvir, naux]."""
    naux = lpq.shape[0]
    t = lpq.transpose(1, 2, 0)
    dia = np.ascontiguousarray(t[:nocc, nocc:]).reshape(-1, naux)
    dij = np.ascontiguousarray(t[:nocc, :nocc]).reshape(-1, naux)
    dab = np.ascontiguousarray(t[nocc:, nocc:]).reshape(-1, naux)
    return dia, dij, dab


def systems_on_device(shapes, device: int = 0, threads: int = 8):
    """make_system for many shapes, resident on the GPU: the seeded numpy draws
    of draw_system (the same numbers make_system uses) run on a thread pool
    (numpy's generators release the GIL), and each system is mirrored and
    rescaled on the device.  shapes: (seed, nocc, nvir, naux, pi_norm) tuples.
    Returns [(mo_energy, lpq)] as CUDA float64 tensors; the rescaling's
    spectral norm comes from the device eigensolver, so lpq equals
    make_system's to rounding."""
    from concurrent.futures import ThreadPoolExecutor

    import torch
    dev = torch.device("cuda", device)
    out = [None] * len(shapes)

    def draw(i):
        seed, nocc, nvir, naux, _ = shapes[i]
        return i, draw_system(nocc, nvir, naux, seed)

    with ThreadPoolExecutor(max(1, threads)) as ex:
        for i, (e, upper) in ex.map(draw, range(len(shapes))):
            seed, nocc, nvir, naux, pin = shapes[i]
            nmo = nocc + nvir
            up = torch.from_numpy(upper).to(dev)
            del upper
            iu, ju = torch.triu_indices(nmo, nmo, device=dev)
            lpq = torch.empty((naux, nmo, nmo), dtype=torch.float64, device=dev)
            lpq[:, iu, ju] = up
            lpq[:, ju, iu] = up
            del up
            ed = torch.from_numpy(e).to(dev)
            bov = lpq[:, :nocc, nocc:].reshape(naux, -1)
            e_ia = (ed[:nocc, None] - ed[None, nocc:]).reshape(-1)
            pi0 = 4.0 * (bov / e_ia) @ bov.T
            lpq *= torch.sqrt(pin / torch.linalg.eigvalsh(pi0).abs().max())
            out[i] = (ed, lpq)
    return out


def make_system_device(nocc: int, nvir: int, naux: int, seed: int, pi_norm: float, device: int = 0):
    """The same distributions as :func:`make_system`, drawn on the GPU with
    torch's seeded device generator (the draws differ from numpy's).  Returns
    (mo_energy, lpq) as CUDA float64 tensors.  Used where the host draw is too
    slow (the 64-system batch holds ~32 GB of lpq)."""
    import torch
    dev = torch.device("cuda", device)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    nmo = nocc + nvir
    kw = dict(generator=g, device=dev, dtype=torch.float64)
    e_occ = torch.sort(torch.rand(nocc, **kw) * 0.9 - 1.2).values
    e_vir = torch.sort(torch.rand(nvir, **kw) * 2.95 + 0.05).values
    e = torch.cat([e_occ, e_vir])
    lpq = torch.randn(naux, nmo, nmo, **kw) * 0.05
    lpq = torch.triu(lpq) + torch.triu(lpq, 1).transpose(1, 2)
    bov = lpq[:, :nocc, nocc:].reshape(naux, -1)
    e_ia = (e[:nocc, None] - e[None, nocc:]).reshape(-1)
    pi0 = 4.0 * (bov / e_ia) @ bov.T
    norm = torch.linalg.eigvalsh(pi0).abs().max()
    lpq *= torch.sqrt(pi_norm / norm)
    return e.contiguous(), lpq.contiguous()
