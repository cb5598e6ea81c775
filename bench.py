#!/usr/bin/env python
"""Benchmark: evGW iterations per second on one B200 (replicas on N GPUs).

Workload (one "step" = one evGW iteration over all orbitals):
  nocc 40, nvirt 260 (nmo 300), naux 1000, seed 1, ||Pi(0)||_2 = 4, 32-point
  imaginary-frequency GL grid, linearized QP, reference Pade point rule.
  Inputs are synthetic (seeded), far larger than L2 (lpq is 720 MB), so no
  explicit L2 flush is needed between steps.

The headline value is the split-precision tcgen05 form (FP16x3 by default);
the plain FP64 GPU path is timed in the same run and the QP-energy error of
the split form against it is reported in meV.  The same line carries the
64-system batched G0W0 (batch64_g0w0_cd), the differentiation workload
(grad_nmo200) and the BSE-TDA Davidson (bse_dim26400).  ``--impl reference`` times the reference's
algorithm on the host cores (the CPU oracle restatement; the Rust reference
cannot be built here).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "evGW iter/s: mixed-prec vs FP64 GPU at ≤1 meV QP err; TC util %; CPU ref"
NOCC, NVIR, NAUX, SEED, PINORM, NW = 40, 260, 1000, 1, 4.0, 32
CONFIG_ITERS = 5  # evGW iterations of the configuration
WORKLOAD = "evgw_nmo300_naux1000_nw32"
HA_TO_MEV = 27211.386


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    # 50 evGW iterations (10 calls of 5): long enough that a driver stall
    # under the nvidia-smi clock sampler (up to ~0.1 s) cannot dominate.
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--precision", choices=["fp16x3", "bf16x3", "fp64"], default=None)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-batch64", action="store_true")
    p.add_argument("--no-grad", action="store_true")
    p.add_argument("--no-bse", action="store_true")
    p.add_argument("--batch-workers", type=int, default=0)
    p.add_argument("--batch-largest", type=int, default=0,
                   help="profiling aid: run the batch leg on its K largest systems only (0: all 64)")
    p.add_argument("--bse-fd-points", type=int, default=4)
    p.add_argument("--p0-form", choices=["auto", "materialised", "pair", "converter"], default="auto",
                   help="form of the split P0 (chi-scaled operand materialised, or built while staged)")
    p.add_argument("--contraction-form", choices=["auto", "single", "pair"], default="auto",
                   help="tiles of the split pair contraction (one CTA, or CTA pairs)")
    return p.parse_args()


def dist_setup(n):
    import torch
    import torch.distributed as dist
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        from datetime import timedelta
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        return dist.get_rank(), dist.get_world_size(), local
    return 0, 1, 0


def max_over_ranks(values, world, device):
    """Element-wise maximum of per-rank timings (seconds) over the job: every
    rank takes part in the same all-reduce, in the same order."""
    if world == 1:
        return [float(v) for v in values]
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t]


def job_rate(units_per_rank, world, seconds_max):
    """Whole-job throughput: units of all ranks over the slowest rank's time."""
    return world * units_per_rank / seconds_max


class Clocks:
    """nvidia-smi sampler for the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None
        # nvidia-smi's start-up (NVML init) can stall CUDA calls of this
        # process; start timing once it is sampling.
        t0 = time.time()
        while self.p is not None and time.time() - t0 < 10.0:
            self.f.flush()
            with open(self.f.name) as fh:
                if len(fh.read().splitlines()) >= 3:
                    break
            time.sleep(0.1)
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for name, val in zip(names, parts[3:7]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def fp64_dgemm_peak_tflops():
    """cuBLAS DGEMM rate on this GPU (the FP64 tensor-pipe denominator)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def contraction_flops(nmo, naux, nw):
    """Algorithmic FLOPs of the Sigma_c contraction per iteration (all orbitals):
    2 naux^2 norbs nmo per frequency (the per-unit figure of the reference's
    per-orbital dgemm), norbs = nmo."""
    return 2.0 * naux * naux * nmo * nmo * nw


def contraction_mma_flops(nmo, naux, nw):
    """MMA FLOPs the split tcgen05 contraction issues: unique pairs padded to
    128 rows, N tiles of 256 over naux padded to 64, the half-lower K range
    [0, n0 + 256) of each N tile, three products."""
    npair = nmo * (nmo + 1) // 2
    m_pad = -(-npair // 128) * 128
    kb = -(-naux // 64)
    kn = sum(min(kb, -(-(n0 + 256) // 64)) * 64 for n0 in range(0, naux, 256))
    return 3 * 2.0 * m_pad * 256 * kn * nw


# DRAM bytes (read + write) of one pair-contraction launch at nmo 300 / naux 1000 /
# nw 32, from one ncu capture of the bench's own command (dram__bytes_read.sum +
# dram__bytes_write.sum of the launch the bench keeps).
# DRAM bytes of one pair-contraction launch at nmo 300 / naux 1000 / nw 32 (ncu,
# the frequency grouping the autotuner keeps): CTA-pair and single-CTA tiles.
CONTRACTION_DRAM_BYTES = {"pair": 1.617387e9 + 0.015371e9, "single": 1.563380e9 + 0.015538e9}
CONTRACTION_KERNEL = {"pair": "k_rowdot_pair (pair contraction on CTA pairs, cta_group::2)",
                      "single": "k_tc_gemm<256,EPI_ROWDOT> (pair contraction, one CTA per pair block)"}


def iteration_flops(nocc, nvir, naux, nw):
    nmo = nocc + nvir
    nov = nocc * nvir
    p0 = 2.0 * nov * naux * naux * nw / 2.0  # lower-triangle tiles of the symmetric product
    inv = 2.0 * naux ** 3 * nw
    return p0 + inv + contraction_flops(nmo, naux, nw)


def qp_step_map(q, e_in, e_hf, lpq_d, nocc, sx, vxc, prec, dev):
    """One evGW step's QP energies before mixing, from input energies e_in
    (qp/evgw.rs:688-821): Sigma_c(iw) with e_in in P0 and G (all orbitals, the
    NW-point grid), the Pade fit by the reference point rule, then the
    linearized QP E = e_hf + Z (Sx + Re S(e_in - ef_hf) - Vxc) with Z from the
    1e-6 forward difference, clipped to [0.1, 0.999].  Sigma, Pade fit and
    Pade evaluations run on the device in form `prec`."""
    nmo = e_hf.shape[0]
    sig, om = q.get_sigma_diag(e_in, lpq_d, list(range(nmo)), nocc, nw=NW, precision=prec, device=dev)
    c, f = q.ac_pade_thiele_diag(sig, om, device=dev)
    ef = 0.5 * (e_hf[nocc - 1] + e_hf[nocc])
    out = np.empty(nmo)
    for p in range(nmo):
        we = e_in[p] - ef
        s0, s1 = q.pade_thiele(np.array([we, we + 1e-6]), f[p], c[:, p], device=dev)
        z = min(max(1.0 / (1.0 - (s1.real - s0.real) / 1e-6), 0.1), 0.999)
        out[p] = e_hf[p] + z * (sx[p] + s0.real - vxc[p])
    return out


def host_cores() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


class CpuEvgw:
    """The reference's evGW iteration on the host cores, by the CPU oracle (its
    restatement of the reference's algorithm; the Rust reference cannot be
    built here): per frequency P0 by one GEMM, the Cholesky inverse and one
    GEMM per orbital for all orbitals (correlation_ac.rs:241-449), then the
    Pade fit and the linearized QP of every orbital (qp/evgw.rs:784-821).  The
    frequency loop runs on a thread pool of one worker per core with one BLAS
    thread each (the reference's rayon into_par_iter, correlation_ac.rs:367)."""

    def __init__(self, sysm, vxc):
        from oracle import qx_oracle as O
        self.O, self.s, self.vxc = O, sysm, np.asarray(vxc, dtype=np.float64)
        self.cores = host_cores()
        self.workers = min(NW, self.cores)
        self.mi = np.ascontiguousarray(sysm.lpq[:, :, :sysm.nocc].transpose(1, 2, 0))

    def _sigma(self, e, nw=NW):
        return self.O.get_sigma_diag_threaded(e, self.s.lpq, range(self.s.nmo), self.s.nocc, nw, 5.0, 0.5,
                                              self.workers)

    def iteration(self) -> float:
        """Seconds of one full evGW iteration (all NW frequencies, all orbitals)."""
        from threadpoolctl import threadpool_limits
        cfg = self.O.EvGWConfig(max_iterations=1, energy_tolerance=0.0, nfreq=NW)
        with threadpool_limits(limits=max(1, self.cores // self.workers)):
            t0 = time.perf_counter()
            self.O.run_evgw_blocks(self.s.mo_energy, self.mi, self.vxc, self.s.lpq, self.s.nocc, cfg,
                                   sigma_fn=self._sigma)
            return time.perf_counter() - t0

    def warm(self):
        """One frequency of an iteration (loads the BLAS threads)."""
        from threadpoolctl import threadpool_limits
        with threadpool_limits(limits=max(1, self.cores // self.workers)):
            self.O.get_sigma_diag_threaded(self.s.mo_energy, self.s.lpq, range(8), self.s.nocc, 1, 5.0, 0.5, 1)

    def threads(self) -> int:
        return self.workers * max(1, self.cores // self.workers)


def cpu_baseline(sysm, vxc):
    """One full evGW iteration of the reference's algorithm on the host cores
    (CpuEvgw), timed whole: no frequency sampling, no extrapolation."""
    c = CpuEvgw(sysm, vxc)
    c.warm()
    t = c.iteration()
    return {"value": 1.0 / t, "unit": "evGW iter/s", "cores": c.threads(), "kind": "port", "extrapolated": False,
            "seconds": t,
            "sample": f"one full evGW iteration: all {NW} frequencies (P0 GEMM, Cholesky inverse, one GEMM per "
                      f"orbital for all {sysm.nmo} orbitals), Pade and linearized QP; {c.workers} frequency "
                      f"workers x {max(1, c.cores // c.workers)} BLAS threads; {t:.1f} s"}


def batch64_flops(shapes, nw):
    """Algorithmic FLOPs of one pass over the batch (imaginary axis): per system
    and frequency 2 nov naux^2 (P0) + naux^3 (inverse) + 2 naux^2 norbs nmo."""
    tot = 0.0
    for _, nocc, nvir, naux, _ in shapes:
        nmo = nocc + nvir
        tot += nw * (2.0 * nocc * nvir * naux ** 2 + naux ** 3 + 2.0 * naux ** 2 * 6 * nmo)
    return tot


def bench_batch64(q, dev, precision, steps, warmup, nworkers, largest=0):
    """64 independent G0W0-CD systems (nmo ~ U[40, 400], nocc = round(nmo/6),
    naux = round(3.5 nmo), ||Pi(0)|| ~ U[1, 6], 24-point grid, HOMO-2..LUMO+2,
    HF reference Vxc = diag(Sigma_x), linearized QP step: batched G0W0 = one
    evGW iteration per system), all resident in HBM; one step = one pass over
    the batch.  The systems are make_system's seeded numpy draws (the ones
    the parity tests rebuild).  Returns systems/s for the mixed and the FP64
    forms and the QP error of the mixed form in meV."""
    import torch
    from quasix_b200.synth import batch64_shapes, systems_on_device
    shapes = batch64_shapes()
    if largest:
        # A small case of the same kernels (profiling): the largest systems only.
        shapes = sorted(shapes, key=lambda sh: -(sh[1] + sh[2]))[:largest]
    systems = []
    t_draw = time.perf_counter()
    drawn = systems_on_device(shapes, device=dev, threads=min(16, host_cores()))
    t_draw = time.perf_counter() - t_draw
    for (seed, nocc, nvir, naux, pin), (e, lpq) in zip(shapes, drawn):
        vxc = q.compute_exchange_diag(lpq, nocc, device=dev)
        systems.append(dict(mo_energy=e, lpq=lpq, nocc=nocc, targets=list(range(nocc - 3, nocc + 3)), vxc=vxc))
    torch.cuda.synchronize()
    nw = 24

    def timed(prec):
        for _ in range(warmup):
            q.g0w0_cd_batch(systems, nw=nw, precision=prec, nworkers=nworkers, qp_solver="linearized", device=dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s.record()
        for _ in range(steps):
            r = q.g0w0_cd_batch(systems, nw=nw, precision=prec, nworkers=nworkers, qp_solver="linearized", device=dev)
        e.record()
        torch.cuda.synchronize()
        return r, s.elapsed_time(e) * 1e-3

    res_mixed, t_mixed = timed(precision)
    res_fp64, t_fp64 = timed("fp64")
    err = max(float(np.abs(a["qp_energies"] - b["qp_energies"]).max()) for a, b in zip(res_mixed, res_fp64))
    n = len(systems)
    flops = batch64_flops(shapes, nw)
    del systems
    torch.cuda.empty_cache()
    return {"workload": ("g0w0_cd_batch64_nmo40-400_nw24" if not largest
                         else f"g0w0_cd_batch64_largest{largest}_nw24 (profiling subset)"),
            "systems": n, "nworkers": nworkers,
            "mode": "grouped (every inversion one grouped block sweep)" if nworkers == 0
            else f"{nworkers} per-system worker streams", "qp": "linearized",
            "precision": precision, "steps": steps, "warmup": warmup,
            "systems_per_s": n * steps / t_mixed, "fp64_systems_per_s": n * steps / t_fp64,
            "speedup_vs_fp64_gpu": t_fp64 / t_mixed, "max_qp_err_meV_vs_fp64": err * HA_TO_MEV,
            "imag_axis_flop_per_pass": flops,
            "data": f"synthetic: make_system's numpy draws for seeds 100-163 (drawn on {min(16, host_cores())} "
                    f"host threads in {t_draw:.1f} s, mirrored and rescaled on the device)"}


def bench_grad_nmo200(q, dev, precision, steps=3, warmup=1):
    """Differentiation workload: nocc 30, nvirt 170, naux 700, seed 7, 24-point
    grid, L = E_QP(HOMO) + E_QP(LUMO) by the CD Newton root, gradient with
    respect to all orbital energies and lpq by the adjoint (P0/W rebuilt per
    frequency).  Vxc is held fixed at values that put the roots 0.05 Ha inside
    the gap.  One step = forward root + adjoint.  Also reports the max-norm
    relative deviation from FP64 central differences at 8 seeded coordinates."""
    import torch
    from quasix_b200.synth import make_system
    s = make_system(30, 170, 700, seed=7, pi_norm=2.0)
    nocc, tg, nw = 30, [29, 30], 24
    e_d = torch.from_numpy(s.mo_energy.copy()).to(f"cuda:{dev}")
    l_d = torch.from_numpy(s.lpq.copy()).to(f"cuda:{dev}")
    target = np.array([s.mo_energy[29] + 0.05, s.mo_energy[30] - 0.05])
    cs = q.cd_sigma(e_d, l_d, nocc, tg, target, nw=nw, device=dev)
    vxc = np.asarray(q.compute_exchange_diag(l_d, nocc, device=dev))
    vxc[tg] = cs["sigma_x"] + cs["sigma_c"] - (target - s.mo_energy[tg])
    v_d = torch.from_numpy(vxc).to(f"cuda:{dev}")

    def step(prec, e=e_d, lpq=l_d, tol=1e-13, grad=True):
        r = q.g0w0_cd(e, lpq, nocc, tg, nw=nw, vxc=v_d, tol=tol, max_iter=100, precision=prec, device=dev)
        if not grad:
            return float(r["qp_energies"].sum())
        return q.g0w0_cd_grad(e, lpq, nocc, tg, r["qp_energies"], [1.0, 1.0], nw=nw, precision=prec, device=dev)

    out = {"workload": "g0w0_cd_grad_nmo200_naux700_nw24", "loss": "E_QP(HOMO) + E_QP(LUMO)", "steps": steps,
           "vxc": "fixed; roots 0.05 Ha inside the gap"}
    grads = {}
    for prec in (precision, "fp64"):
        for _ in range(warmup):
            step(prec)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(steps):
            g = step(prec)
        ev1.record()
        torch.cuda.synchronize()
        grads[prec] = (g[0].cpu().numpy(), g[1].cpu().numpy())
        out[("" if prec == precision else "fp64_") + "ms_per_gradient"] = ev0.elapsed_time(ev1) / steps
    out["precision"] = precision
    out["speedup_vs_fp64_gpu"] = out["fp64_ms_per_gradient"] / out["ms_per_gradient"]
    rng = np.random.default_rng(7)
    ge64, gl64 = grads["fp64"]
    fd, an = [], {precision: [], "fp64": []}
    for p in rng.choice(200, 4, replace=False):
        ep, em = e_d.clone(), e_d.clone()
        ep[p] += 1e-5
        em[p] -= 1e-5
        fd.append((step("fp64", e=ep, grad=False) - step("fp64", e=em, grad=False)) / 2e-5)
        for k in an:
            an[k].append(grads[k][0][p])
    mag = np.abs(gl64)
    cand = np.argwhere(mag > 1e-3 * mag.max())
    for k in rng.choice(len(cand), 4, replace=False):
        P, a, b = (int(v) for v in cand[k])
        d = torch.zeros_like(l_d)
        d[P, a, b] += 1e-6
        if a != b:
            d[P, b, a] += 1e-6
        fd.append((step("fp64", lpq=l_d + d, grad=False) - step("fp64", lpq=l_d - d, grad=False)) / 2e-6)
        for kk in an:
            an[kk].append(grads[kk][1][P, a, b] * (2 if a != b else 1))
    fd = np.array(fd)
    for k in an:
        key = ("" if k == precision else "fp64_") + "fd_max_rel_err"
        out[key] = float(np.abs(np.array(an[k]) - fd).max() / np.abs(fd).max())
    return out


def bench_bse_dim26400(q, precision, fd_points=4):
    """BSE-TDA: nocc 60, nvirt 440 (dimension 26 400), naux 1800, seed 11,
    ||Pi(0)|| = 5, singlet, W0 = (I - Pi(0))^-1; the 10 lowest roots to a
    1e-8 Ha residual by the device Davidson (max_space 200).  One step = one
    Davidson solve from the unit-vector start, after one untimed solve.  Reports seconds to converge
    for the split form and FP64 and the largest root difference in meV."""
    import torch
    from quasix_b200.synth import bse_blocks, make_system
    s = make_system(60, 440, 1800, seed=11, pi_norm=5.0)
    nocc, nvir, naux = 60, 440, 1800
    dia, dij, dab = bse_blocks(s.lpq, nocc)
    w0 = q.bse.screened_w0(s.mo_energy, np.ascontiguousarray(s.lpq[:, :nocc, nocc:]))
    delta = (s.mo_energy[None, nocc:] - s.mo_energy[:nocc, None]).reshape(-1)
    out = {"workload": "bse_tda_dim26400_naux1800_10roots", "tol_residual": 1e-8, "precision": precision}
    roots = {}
    for prec in (precision, "fp64"):
        k = q.BSETDAKernel(nocc, nvir, naux, delta, dia, dij, dab, w0, precision=prec)
        cfg = q.DavidsonConfig(10, 400, 200, 1e-8)
        # One untimed solve first: the kernel object allocates its subspace and
        # matvec buffers on its first solve (the solves themselves are
        # deterministic, so the timed one repeats the same path).
        k.solve_davidson_with_config(cfg)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record()
        r = k.solve_davidson_with_config(cfg)
        ev1.record()
        torch.cuda.synchronize()
        pre = "" if prec == precision else "fp64_"
        out[pre + "s_to_converge"] = ev0.elapsed_time(ev1) * 1e-3
        out[pre + "iterations"] = r["iterations"]
        out[pre + "all_converged"] = r["all_converged"]
        roots[prec] = np.array(r["eigenvalues"])
        # Adjoint of the lowest root: dOmega/de and dOmega/d(df_ia, df_ij,
        # df_ab) with W0's dependence (qx_bse_root_grad_b), after one untimed call.
        x0 = r["eigenvectors"][:, 0]
        k.root_gradient_blocks(x0, mo_energy=s.mo_energy)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        k.root_gradient_blocks(x0, mo_energy=s.mo_energy)
        torch.cuda.synchronize()
        out[pre + "s_adjoint_lowest_root"] = time.perf_counter() - t0
        k.close()
    out["speedup_vs_fp64_gpu"] = out["fp64_s_to_converge"] / out["s_to_converge"]
    out["max_root_err_meV_vs_fp64"] = float(np.abs(roots[precision] - roots["fp64"]).max() * HA_TO_MEV)
    out["roots_Ha"] = [float(v) for v in roots["fp64"]]
    if fd_points > 0:
        out["grad_fd_check"] = bse_grad_fd_check(q, s, nocc, fd_points)
    return out


def bse_grad_fd_check(q, s, nocc, npoints):
    """The lowest-root gradient of the torch.autograd.Function (FP64) against
    FP64 central differences of its own forward path at npoints seeded
    coordinates, half orbital energies (step 1e-5 Ha), half lpq entries
    (symmetric step 1e-6)."""
    import torch
    e = torch.tensor(s.mo_energy, dtype=torch.float64, device="cuda", requires_grad=True)
    lpq = torch.tensor(s.lpq, dtype=torch.float64, device="cuda", requires_grad=True)
    t0 = time.perf_counter()
    om = q.bse_lowest_root(e, lpq, nocc, tol=1e-10, max_iter=600)
    ge, gl = torch.autograd.grad(om, (e, lpq))
    t_fwd_bwd = time.perf_counter() - t0

    def f(ev, lv):
        with torch.no_grad():
            return float(q.bse_lowest_root(ev, lv, nocc, tol=1e-10, max_iter=600))

    rng = np.random.default_rng(11)
    an, fd, where = [], [], []
    # Coordinates with gradients within 1e-2 of the largest (the others are
    # below the FD resolution of a 1e-10-converged root).
    gmag = ge.abs().cpu().numpy()
    top = np.flatnonzero(gmag > 1e-2 * gmag.max())
    for p in rng.choice(top, min(npoints // 2, len(top)), replace=False):
        d = torch.zeros_like(e)
        d[p] = 1e-5
        fd.append((f(e + d, lpq) - f(e - d, lpq)) / 2e-5)
        an.append(float(ge[p]))
        where.append(f"e[{int(p)}]")
    mag = gl.abs()
    cand = torch.nonzero(mag > 1e-2 * mag.max()).cpu().numpy()
    for k in rng.choice(len(cand), npoints - npoints // 2, replace=False):
        P, a, b = (int(v) for v in cand[k])
        d = torch.zeros_like(lpq)
        d[P, a, b] += 1e-6
        if a != b:
            d[P, b, a] += 1e-6
        fd.append((f(e, lpq + d) - f(e, lpq - d)) / 2e-6)
        # The symmetric step moves both entries: its derivative is the sum of
        # the two gradient entries (the forward reads one triangle of some blocks).
        an.append(float(gl[P, a, b]) + (float(gl[P, b, a]) if a != b else 0.0))
        where.append(f"lpq[{P},{a},{b}]")
    an, fd = np.array(an), np.array(fd)
    return {"points": npoints, "max_rel_err": float(np.abs(an - fd).max() / np.abs(fd).max()),
            "coordinates": where, "analytic": an.tolist(), "central_difference": fd.tolist(),
            "s_forward_and_backward_fp64": t_fwd_bwd,
            "note": "bse_lowest_root (torch.autograd.Function) vs FP64 central differences of the same forward"}


# Wall-clock budget of the reference arm's timed region: full evGW iterations
# are timed until this is spent or --steps are done, whichever comes first.
REFERENCE_BUDGET_S = 150.0


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from quasix_b200.synth import make_system
    sysm = make_system(NOCC, NVIR, NAUX, seed=SEED, pi_norm=PINORM)
    # The same HF-reference Vxc = diag(Sigma_x) as the GPU arm.
    mi = sysm.lpq[:, :, :NOCC]
    vxc = -np.einsum("Ppi,Ppi->p", mi, mi)
    c = CpuEvgw(sysm, vxc)
    # Warm-up: W samples of one frequency each (BLAS thread start-up).
    for _ in range(args.warmup):
        c.warm()
    times = []
    t_all = time.perf_counter()
    while len(times) < max(1, args.steps):
        times.append(c.iteration())
        if time.perf_counter() - t_all + times[-1] > REFERENCE_BUDGET_S:
            break
    t_all = time.perf_counter() - t_all
    steps = len(times)
    v = steps / sum(times)
    base = {"value": v, "unit": "evGW iter/s", "cores": c.threads(), "kind": "port", "extrapolated": False,
            "sample": f"{steps} full evGW iteration(s) (all {NW} frequencies, all {sysm.nmo} orbitals, Pade and "
                      f"linearized QP) of the requested {args.steps}, {t_all:.1f} s; {c.workers} frequency workers x "
                      f"{max(1, c.cores // c.workers)} BLAS threads"}
    line = {"metric": METRIC, "value": v, "unit": "evGW iter/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": steps, "steps_requested": args.steps, "warmup": args.warmup,
            "warmup_unit": "one frequency of an iteration", "ms_per_step": 1e3 * sum(times) / steps,
            "timed_s": sum(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "nocc": NOCC, "nvirt": NVIR, "naux": NAUX, "nw": NW, "seed": SEED,
                       "orbitals": "all", "qp": "linearized"},
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": "evGW iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch

    import quasix_b200 as q
    from quasix_b200 import _native as N
    from quasix_b200.synth import make_system

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = local
    sysm = make_system(NOCC, NVIR, NAUX, seed=SEED, pi_norm=PINORM)
    nmo = sysm.nmo
    lpq_d = torch.from_numpy(sysm.lpq).to(f"cuda:{dev}")
    # HF reference: the mean-field potential is the exchange operator itself,
    # so Vxc = diag(Sigma_x) and the QP correction is Sigma_c.  (With Vxc = 0
    # this synthetic system shifts the QP levels by ~-3 Ha, the levels cross in
    # the second evGW iteration and the loop turns chaotic.)
    vxc = q.compute_exchange_diag(lpq_d, sysm.nocc, device=dev)
    ctx = N.context(dev)
    ctx.set_p0_form(args.p0_form)
    ctx.set_contraction_form(args.contraction_form)
    have_tc = True
    prec_main = args.precision or "fp16x3"

    def run(prec, iters, lpq):
        return q.run_evgw_blocks(sysm.mo_energy, lpq, vxc, sysm.nocc, device=dev, nfreq=NW, precision=prec,
                                 fixed_iterations=iters, max_iterations=iters)

    # One step is one evGW iteration; the timed region runs the configuration's
    # own call length, calls of CONFIG_ITERS iterations from the HF start
    # (each with its per-call setup: pair gather and splits), K / 5 of them.
    ncalls = max(1, -(-args.steps // CONFIG_ITERS))
    steps = ncalls * CONFIG_ITERS

    def timed(prec, lpq):
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        t0 = time.perf_counter()
        for _ in range(ncalls):
            r = run(prec, CONFIG_ITERS, lpq)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        el = time.perf_counter() - t0
        return r, el

    # Warm-up: one call of 5 iterations (>= 3 steps) for each form, then the
    # timed calls.
    try:
        run(prec_main, CONFIG_ITERS, lpq_d)
    except N.QxError as e:
        if prec_main == "fp64":
            raise
        have_tc = False
        prec_main = "fp64"
        if rank == 0:
            print(f"# mixed-precision form unavailable ({e}); timing FP64 only", file=sys.stderr)
        run(prec_main, CONFIG_ITERS, lpq_d)
    with Clocks(dev) as clk:
        res_main, t_main = timed(prec_main, lpq_d)
        launches = ctx.launches() * ncalls
        stage = ctx.timings()  # the last call's stages (5 iterations)
        guarded, reinverted = ctx.guard_stats()
    clocks = clk.summary()
    res_fp64, t_fp64 = (res_main, t_main)
    if prec_main != "fp64":
        run("fp64", CONFIG_ITERS, lpq_d)
        res_fp64, t_fp64 = timed("fp64", lpq_d)
    t_main, t_fp64 = max_over_ranks([t_main, t_fp64], world, f"cuda:{dev}")
    value = job_rate(steps, world, t_main)
    fp64_rate = job_rate(steps, world, t_fp64)
    err_iter = [float(np.abs(a - b).max() * HA_TO_MEV) for a, b in zip(res_main["energies"], res_fp64["energies"])]
    # Conditioning of the FP64 path itself: the same FP64 evGW on lpq
    # perturbed by ~1e-14 relative (symmetric noise).
    gen = torch.Generator(device=f"cuda:{dev}")
    gen.manual_seed(7)
    noise = torch.rand(lpq_d.shape, generator=gen, device=f"cuda:{dev}", dtype=torch.float64) - 0.5
    lpq_p = lpq_d * (1.0 + 1e-14 * (noise + noise.transpose(1, 2)))
    del noise
    res_p = run("fp64", CONFIG_ITERS, lpq_p)
    sens_iter = [float(np.abs(a - b).max() * HA_TO_MEV) for a, b in zip(res_p["energies"], res_fp64["energies"])]
    # Precision per evGW step: the mixed and the FP64 step map from the same
    # FP64 iterate (HF energies, then the FP64 run's iterates), for each of
    # the configuration's 5 iterations.  This separates the precision error of
    # one step from the trajectory's sensitivity once levels cross.  Per
    # orbital, the FP64 step map's own movement under the 1e-14 perturbation
    # of lpq tells whether that orbital's step is numerically meaningful.
    sx_h = np.asarray(vxc.cpu().numpy() if hasattr(vxc, "cpu") else vxc, dtype=np.float64)
    inputs = [sysm.mo_energy] + [np.asarray(e) for e in res_fp64["energies"][:CONFIG_ITERS - 1]]
    step_err, step_sens, step_err_cond, step_excluded, step_cause = [], [], [], [], []
    step_check = None
    for k, e_in in enumerate(inputs):
        m64 = qp_step_map(q, e_in, sysm.mo_energy, lpq_d, sysm.nocc, sx_h, sx_h, "fp64", dev)
        mmx = qp_step_map(q, e_in, sysm.mo_energy, lpq_d, sysm.nocc, sx_h, sx_h, prec_main, dev)
        m64p = qp_step_map(q, e_in, sysm.mo_energy, lpq_p, sysm.nocc, sx_h, sx_h, "fp64", dev)
        err = np.abs(mmx - m64) * HA_TO_MEV
        sens = np.abs(m64p - m64) * HA_TO_MEV
        ok = sens < 1e-3
        step_err.append(float(err.max()))
        step_sens.append(float(sens.max()))
        step_err_cond.append(float(err[ok].max()) if ok.any() else None)
        step_excluded.append(int((~ok).sum()))
        homo, lumo = float(e_in[:sysm.nocc].max()), float(e_in[sysm.nocc:].min())
        step_cause.append("input levels ordered" if lumo > homo else
                          f"input levels crossed (max occupied {homo:.4f} Ha > min virtual {lumo:.4f} Ha)")
        if k == 0:
            # Iteration 0 has no mixing: the step map must reproduce the driver.
            step_check = float(np.abs(m64 - res_fp64["energies"][0]).max() * HA_TO_MEV)
    del lpq_p
    conditioned = [v for v in step_err_cond if v is not None]
    err_mev = max(conditioned) if conditioned else None

    # End to end through the C ABI with host (pinned) inputs: every call
    # reads lpq from host memory (in place: the setup gathers its upper
    # triangle, the pairs p <= q, 361 MB of its 720 MB) and the energies, and
    # returns the results.
    lpq_h = torch.from_numpy(sysm.lpq).pin_memory()
    naux_l = sysm.lpq.shape[0]
    lpq_triangle_bytes = naux_l * nmo * (nmo + 1) // 2 * 8
    run(prec_main, CONFIG_ITERS, lpq_h.numpy())
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(ncalls):
        run(prec_main, CONFIG_ITERS, lpq_h.numpy())
    torch.cuda.synchronize()
    t_e2e = max_over_ranks([time.perf_counter() - t0], world, f"cuda:{dev}")[0]
    e2e = {"value": job_rate(steps, world, t_e2e), "unit": "evGW iter/s",
           "h2d_bytes_per_step": int((lpq_triangle_bytes + 2 * nmo * 8) / CONFIG_ITERS + nmo * 8 * 2),
           "h2d_note": "pinned host lpq is read in place; its upper triangle crosses the link once per call",
           "d2h_bytes_per_step": int(nmo * 8 * 4 / CONFIG_ITERS),
           "calls": ncalls, "iterations_per_call": CONFIG_ITERS}

    peaks, peak_src = measured_peaks()
    cflops = contraction_flops(nmo, NAUX, NW)
    ms_contract = stage["contraction"] / CONFIG_ITERS
    achieved = cflops / (ms_contract * 1e-3) / 1e12
    executed = contraction_mma_flops(nmo, NAUX, NW) / (ms_contract * 1e-3) / 1e12
    if prec_main == "fp64":
        dpeak = fp64_dgemm_peak_tflops()
        roof = {"bound": "tensor", "achieved": achieved, "peak": dpeak, "unit": "TFLOP/s", "frac": achieved / dpeak,
                "traffic": None, "kernel": "k_pair_contract_f64",
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 has no entry in MEASURED_PEAKS.json)"}
    else:
        pk = peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops"))
        cform = "single" if args.contraction_form == "single" else "pair"
        burst = peaks.get("bf16_tflops")
        roof = {"bound": "tensor", "achieved": achieved, "peak": pk, "unit": "TFLOP/s", "frac": achieved / pk,
                "traffic": CONTRACTION_DRAM_BYTES[cform], "kernel": CONTRACTION_KERNEL[cform],
                "peak_source": f"bf16_tflops_sustained, {peak_src} (the kernel runs inside a seconds-long step)",
                "frac_of_burst_peak": achieved / burst if burst else None,
                "algorithmic_flops_per_launch": cflops,
                "executed_mma_tflops": executed, "executed_mma_frac": executed / pk,
                "note": "algorithmic = 2 naux^2 norbs nmo nw; executed = 3 split products over the "
                        "half-lower K range of unique pairs; stage time includes the Wc split"}

    line = {"metric": METRIC, "value": value, "unit": "evGW iter/s", "n_gpus": world, "steps": steps,
            "warmup": CONFIG_ITERS, "ms_per_step": 1e3 * t_main / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": {"fp16x3": "f16x3->f32(TMEM)->f64", "bf16x3": "bf16x3->f32(TMEM)->f64"}.get(prec_main, "f64"),
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "nocc": NOCC, "nvirt": NVIR, "naux": NAUX, "nw": NW, "seed": SEED,
                       "orbitals": "all", "qp": "linearized", "vxc": "diag(Sigma_x) (HF reference)",
                       "precision": prec_main, "p0_form": args.p0_form, "contraction_form": args.contraction_form,
                       "parallelism": f"replicas{world}" if world > 1 else "single",
                       "l2": "inputs larger than L2 (lpq 720 MB, pair tensor 361 MB); no flush"},
            "fp64_gpu_iter_per_s": fp64_rate, "speedup_vs_fp64_gpu": value / fp64_rate,
            "max_qp_err_meV_vs_fp64": err_mev,
            "per_step_qp_err_meV": step_err, "per_step_qp_err_meV_conditioned": step_err_cond,
            "per_step_fp64_sensitivity_1e-14_meV": step_sens, "per_step_orbitals_excluded": step_excluded,
            "per_step_input": step_cause, "per_step_map_check_meV": step_check,
            "qp_err_note": "per_step: mixed vs FP64 step map from the same FP64 iterate, iterations 0-4; "
                           "conditioned: over the orbitals whose FP64 step moves < 1e-3 meV under a 1e-14 "
                           "relative perturbation of lpq (the others' step carries no precision information); "
                           "max_qp_err_meV_vs_fp64 is the max of the conditioned values; trajectory: the two "
                           "runs' iterates",
            "guarded_inversions_last_call": guarded, "pivoted_reinversions_last_call": reinverted,
            "trajectory_qp_err_meV_per_iteration": err_iter, "fp64_perturbation_1e-14_meV_per_iteration": sens_iter,
            "stage_ms_per_step": {k: v / CONFIG_ITERS for k, v in stage.items()},
            "roofline": roof, "clocks": clocks, "e2e": e2e, "gpu_launches": launches}
    if prec_main != "fp64":
        # Tensor-core utilisation of the dominant kernel: the MMA work it issues
        # per second over the measured sustained tcgen05 (bf16/fp16) peak.
        line["tc_util_pct"] = 100.0 * roof["executed_mma_frac"]
    if not args.no_grad:
        line["grad_nmo200"] = bench_grad_nmo200(q, dev, prec_main)
    if not args.no_bse:
        line["bse_dim26400"] = bench_bse_dim26400(q, prec_main, fd_points=args.bse_fd_points)
    if not args.no_batch64:
        line["batch64_g0w0_cd"] = bench_batch64(q, dev, prec_main, steps=3, warmup=1, nworkers=args.batch_workers,
                                                    largest=args.batch_largest)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(sysm, vxc.cpu().numpy() if hasattr(vxc, "cpu") else vxc)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
