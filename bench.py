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
WORKLOAD = "evgw_nmo300_naux1000_nw32"
HA_TO_MEV = 27211.386


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    # 50 evGW iterations (~0.6 s): long enough that a driver stall under the
    # nvidia-smi clock sampler (up to ~0.1 s) cannot dominate the timed region.
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--precision", choices=["fp16x3", "bf16x3", "fp64"], default=None)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-batch64", action="store_true")
    p.add_argument("--no-grad", action="store_true")
    p.add_argument("--no-bse", action="store_true")
    p.add_argument("--batch-workers", type=int, default=0)
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
CONTRACTION_DRAM_BYTES = 1.563380e9 + 0.015538e9


def iteration_flops(nocc, nvir, naux, nw):
    nmo = nocc + nvir
    nov = nocc * nvir
    p0 = 2.0 * nov * naux * naux * nw / 2.0  # lower-triangle tiles of the symmetric product
    inv = 2.0 * naux ** 3 * nw
    return p0 + inv + contraction_flops(nmo, naux, nw)


def cpu_reference_sample(sysm, budget_s=15.0):
    """The reference's per-frequency algorithm (oracle restatement, BLAS threads
    on every host core) on a bounded sample of one evGW iteration: frequencies
    are processed until the budget is spent, then scaled to all NW."""
    from oracle import qx_oracle as O
    e = sysm.mo_energy
    lpq = sysm.lpq
    nocc = sysm.nocc
    freqs, wts, iw = O.sigma_grid(NW)
    orbs = list(range(sysm.nmo))
    lov = lpq[:, :nocc, nocc:]
    t0 = time.perf_counter()
    done = 0
    for w in range(NW):
        pi = O.get_rho_response(freqs[w], e, lov)
        wc = O.epsilon_inverse_minus_identity(pi)
        for n in orbs:
            q = wc.T @ lpq[:, n, :]
            np.sum(q * lpq[:, :, n], axis=0)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    per_iter = el * NW / done
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    return {"value": 1.0 / per_iter, "unit": "evGW iter/s", "cores": cores, "kind": "port",
            "sample": f"{done} of {NW} frequencies of one evGW iteration (P0, Cholesky inverse, one GEMM per "
                      f"orbital for all {sysm.nmo} orbitals), {el:.1f} s, scaled by {NW}/{done}"}


def batch64_flops(shapes, nw):
    """Algorithmic FLOPs of one pass over the batch (imaginary axis): per system
    and frequency 2 nov naux^2 (P0) + naux^3 (inverse) + 2 naux^2 norbs nmo."""
    tot = 0.0
    for _, nocc, nvir, naux, _ in shapes:
        nmo = nocc + nvir
        tot += nw * (2.0 * nocc * nvir * naux ** 2 + naux ** 3 + 2.0 * naux ** 2 * 6 * nmo)
    return tot


def bench_batch64(q, dev, precision, steps, warmup, nworkers):
    """64 independent G0W0-CD systems (nmo ~ U[40, 400], nocc = round(nmo/6),
    naux = round(3.5 nmo), ||Pi(0)|| ~ U[1, 6], 24-point grid, HOMO-2..LUMO+2,
    HF reference Vxc = diag(Sigma_x), linearized QP step: batched G0W0 = one
    evGW iteration per system), all resident in HBM; one step = one pass over
    the batch.  Returns systems/s for the mixed and the FP64 forms and the
    QP error of the mixed form in meV."""
    import torch
    from quasix_b200.synth import batch64_shapes, make_system_device
    shapes = batch64_shapes()
    systems = []
    for seed, nocc, nvir, naux, pin in shapes:
        e, lpq = make_system_device(nocc, nvir, naux, seed, pin, device=dev)
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
    return {"workload": "g0w0_cd_batch64_nmo40-400_nw24", "systems": n, "nworkers": nworkers,
            "mode": "grouped (every inversion one grouped block sweep)" if nworkers == 0
            else f"{nworkers} per-system worker streams", "qp": "linearized",
            "precision": precision, "steps": steps, "warmup": warmup,
            "systems_per_s": n * steps / t_mixed, "fp64_systems_per_s": n * steps / t_fp64,
            "speedup_vs_fp64_gpu": t_fp64 / t_mixed, "max_qp_err_meV_vs_fp64": err * HA_TO_MEV,
            "imag_axis_flop_per_pass": flops,
            "data": "synthetic, drawn on the device (torch generator, seeds 100-163)"}


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


def bench_bse_dim26400(q, precision):
    """BSE-TDA: nocc 60, nvirt 440 (dimension 26 400), naux 1800, seed 11,
    ||Pi(0)|| = 5, singlet, W0 = (I - Pi(0))^-1; the 10 lowest roots to a
    1e-8 Ha residual by the device Davidson (max_space 200).  One step = one
    Davidson solve from the unit-vector start, after one untimed solve.  Reports seconds to converge
    for the split form and FP64 and the largest root difference in meV."""
    import torch
    from oracle import qx_oracle as O
    from quasix_b200.synth import make_system
    s = make_system(60, 440, 1800, seed=11, pi_norm=5.0)
    nocc, nvir, naux = 60, 440, 1800
    dia, dij, dab = O.bse_blocks(s.lpq, nocc)
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
        k.close()
    out["speedup_vs_fp64_gpu"] = out["fp64_s_to_converge"] / out["s_to_converge"]
    out["max_root_err_meV_vs_fp64"] = float(np.abs(roots[precision] - roots["fp64"]).max() * HA_TO_MEV)
    out["roots_Ha"] = [float(v) for v in roots["fp64"]]
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from quasix_b200.synth import make_system
    sysm = make_system(NOCC, NVIR, NAUX, seed=SEED, pi_norm=PINORM)
    # Warm-up: one frequency.
    cpu_reference_sample(sysm, budget_s=0.0)
    vals = []
    for _ in range(max(1, args.steps)):
        vals.append(cpu_reference_sample(sysm, budget_s=max(2.0, 20.0 / max(1, args.steps))))
    v = statistics.median([x["value"] for x in vals])
    base = vals[0]
    base["value"] = v
    line = {"metric": METRIC, "value": v, "unit": "evGW iter/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
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
    have_tc = True
    prec_main = args.precision or "fp16x3"

    def run(prec, iters, lpq):
        return q.run_evgw_blocks(sysm.mo_energy, lpq, vxc, sysm.nocc, device=dev, nfreq=NW, precision=prec,
                                 fixed_iterations=iters, max_iterations=iters)

    def timed(prec, iters, lpq):
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        t0 = time.perf_counter()
        r = run(prec, iters, lpq)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        el = time.perf_counter() - t0
        return r, el

    # Warm-up (W steps) for each form, then the timed K steps.
    try:
        run(prec_main, args.warmup, lpq_d)
    except N.QxError as e:
        if prec_main == "fp64":
            raise
        have_tc = False
        prec_main = "fp64"
        if rank == 0:
            print(f"# mixed-precision form unavailable ({e}); timing FP64 only", file=sys.stderr)
        run(prec_main, args.warmup, lpq_d)
    with Clocks(dev) as clk:
        res_main, t_main = timed(prec_main, args.steps, lpq_d)
        launches = ctx.launches()
        stage = ctx.timings()
    clocks = clk.summary()
    res_fp64, t_fp64 = (res_main, t_main)
    if prec_main != "fp64":
        run("fp64", min(args.warmup, 1), lpq_d)
        res_fp64, t_fp64 = timed("fp64", args.steps, lpq_d)
    t_main, t_fp64 = max_over_ranks([t_main, t_fp64], world, f"cuda:{dev}")
    value = job_rate(args.steps, world, t_main)
    fp64_rate = job_rate(args.steps, world, t_fp64)
    err_iter = [float(np.abs(a - b).max() * HA_TO_MEV) for a, b in zip(res_main["energies"], res_fp64["energies"])]
    # Conditioning of the FP64 path itself: the same FP64 evGW on lpq
    # perturbed by ~1e-14 relative (symmetric noise).  Iterations whose FP64
    # energies move by more than 1 micro-eV under that perturbation are
    # ill-conditioned (levels cross in this synthetic system) and carry no
    # precision information; the headline error is taken over the others.
    gen = torch.Generator(device=f"cuda:{dev}")
    gen.manual_seed(7)
    noise = torch.rand(lpq_d.shape, generator=gen, device=f"cuda:{dev}", dtype=torch.float64) - 0.5
    lpq_p = lpq_d * (1.0 + 1e-14 * (noise + noise.transpose(1, 2)))
    del noise
    res_p = run("fp64", args.steps, lpq_p)
    del lpq_p
    sens_iter = [float(np.abs(a - b).max() * HA_TO_MEV) for a, b in zip(res_p["energies"], res_fp64["energies"])]
    stable = [i for i, v in enumerate(sens_iter) if v < 1e-3]
    err_mev = max(err_iter[i] for i in stable) if stable else None

    # End to end through the C ABI with host (pinned) inputs: H2D of lpq and the
    # energies and D2H of the results happen inside the call.
    lpq_h = torch.from_numpy(sysm.lpq).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    run(prec_main, args.steps, lpq_h.numpy())
    torch.cuda.synchronize()
    t_e2e = max_over_ranks([time.perf_counter() - t0], world, f"cuda:{dev}")[0]
    e2e = {"value": job_rate(args.steps, world, t_e2e), "unit": "evGW iter/s",
           "h2d_bytes_per_step": int((sysm.lpq.nbytes + 2 * nmo * 8) / args.steps + nmo * 8 * 2),
           "d2h_bytes_per_step": int(nmo * 8 * 4)}

    peaks, peak_src = measured_peaks()
    cflops = contraction_flops(nmo, NAUX, NW)
    ms_contract = stage["contraction"] / args.steps
    achieved = cflops / (ms_contract * 1e-3) / 1e12
    executed = contraction_mma_flops(nmo, NAUX, NW) / (ms_contract * 1e-3) / 1e12
    if prec_main == "fp64":
        dpeak = fp64_dgemm_peak_tflops()
        roof = {"bound": "tensor", "achieved": achieved, "peak": dpeak, "unit": "TFLOP/s", "frac": achieved / dpeak,
                "traffic": None, "kernel": "k_pair_contract_f64",
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 has no entry in MEASURED_PEAKS.json)"}
    else:
        pk = peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops"))
        roof = {"bound": "tensor", "achieved": achieved, "peak": pk, "unit": "TFLOP/s", "frac": achieved / pk,
                "traffic": CONTRACTION_DRAM_BYTES, "kernel": "k_tc_gemm<256,EPI_ROWDOT> (pair contraction)",
                "peak_source": f"bf16_tflops_sustained, {peak_src}",
                "algorithmic_flops_per_launch": cflops,
                "executed_mma_tflops": executed, "executed_mma_frac": executed / pk,
                "note": "algorithmic = 2 naux^2 norbs nmo nw; executed = 3 split products over the "
                        "half-lower K range of unique pairs; stage time includes the Wc split"}

    line = {"metric": METRIC, "value": value, "unit": "evGW iter/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_main / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": {"fp16x3": "f16x3->f32(TMEM)->f64", "bf16x3": "bf16x3->f32(TMEM)->f64"}.get(prec_main, "f64"),
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "nocc": NOCC, "nvirt": NVIR, "naux": NAUX, "nw": NW, "seed": SEED,
                       "orbitals": "all", "qp": "linearized", "vxc": "diag(Sigma_x) (HF reference)",
                       "precision": prec_main,
                       "parallelism": f"replicas{world}" if world > 1 else "single",
                       "l2": "inputs larger than L2 (lpq 720 MB, pair tensor 361 MB); no flush"},
            "fp64_gpu_iter_per_s": fp64_rate, "speedup_vs_fp64_gpu": value / fp64_rate,
            "max_qp_err_meV_vs_fp64": err_mev, "qp_err_iterations": stable,
            "max_qp_err_meV_per_iteration": err_iter, "fp64_perturbation_1e-14_meV_per_iteration": sens_iter,
            "stage_ms_per_step": {k: v / args.steps for k, v in stage.items()},
            "roofline": roof, "clocks": clocks, "e2e": e2e, "gpu_launches": launches}
    if prec_main != "fp64":
        # Tensor-core utilisation of the dominant kernel: the MMA work it issues
        # per second over the measured sustained tcgen05 (bf16/fp16) peak.
        line["tc_util_pct"] = 100.0 * roof["executed_mma_frac"]
    if not args.no_grad:
        line["grad_nmo200"] = bench_grad_nmo200(q, dev, prec_main)
    if not args.no_bse:
        line["bse_dim26400"] = bench_bse_dim26400(q, prec_main)
    if not args.no_batch64:
        line["batch64_g0w0_cd"] = bench_batch64(q, dev, prec_main, steps=3, warmup=1, nworkers=args.batch_workers)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_reference_sample(sysm, budget_s=12.0)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
