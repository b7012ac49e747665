"""Benchmark of the linear-solve hot path on one B200 (or N independent replicas).

Workload (one step = one complete solve): 3D Poisson, trilinear Q1 hexahedra on
128^3 cells of the unit cube (2,146,689 DoFs, 57,066,625 nonzeros, int32 CSR),
kappa = exp(smoothed unit-variance Gaussian field), RHS uniform [-1, 1] (seed 0),
homogeneous Dirichlet boundary by symmetric elimination, Jacobi-preconditioned CG
to ||r||/||b|| <= 1e-10 from x = 0.  Matrix assembled on the GPU (untimed set-up).

Metric: PCG time-to-1e-10 in seconds (lower is better); value = the headline
solver's device time per solve with inputs resident in HBM (inputs are larger than
L2, so no flush is needed); e2e = the same through the public API with host
buffers (H2D of CSR + RHS from pinned memory and D2H of the solution inside the
timed region).  The line also carries the FP64 solver's time, the roofline of the
dominant kernel (CSR SpMV, timed live with CUDA events) and of the whole PCG
iteration, and the reference's threaded CPU solver on a bounded sample.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cie_b200|reference]
"""
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

WORKLOAD = {"workload": "poisson3d_q1_128^3_lognormal_kappa_jacobi_pcg_rel1e-10", "cells": [128, 128, 128],
            "dofs": 2146689, "nnz": 57066625, "seed": 0, "tolerance": 1e-10, "index": "int32",
            "l2": "inputs larger than L2 (no flush needed)"}
METRIC = "PCG time-to-1e-10 (s), 3D Q1 128^3 Poisson"


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.file = None

    def start(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.file.flush()
        self.file.seek(0)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.file:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        os.unlink(self.file.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_problem_arrays(prob):
    rp, col, val = prob.host_csr()
    return rp, col, val, prob.rhs.cpu().numpy()


def cpu_reference_sample(rp, col, val, b, full_iterations, budget_s=15.0, threads=None):
    """The reference's threaded FP64 CG (oracle/_ref) on a bounded number of
    iterations of the same system; the per-iteration time is scaled to the
    iteration count of a complete solve."""
    from oracle.oracle import Reference, reference_available
    if not reference_available():
        return None
    ref = Reference(threads=threads)
    try:
        _, _, err, t_probe = ref.pcg(rp, col, val, b, maxit=2, reltol=1e-10)
        per_it = max(t_probe / 3.0, 1e-6)
        m = int(max(3, min(full_iterations, budget_s / per_it - 1)))
        _, stats, err, t = ref.pcg(rp, col, val, b, maxit=m, reltol=1e-10)
        per_it = t / (stats[0] + 1)
        est = per_it * (full_iterations + 1)
        return {"value": est, "unit": "s", "cores": ref.threads, "kind": "reference",
                "sample": "%d CG iterations of the reference's ConjugateGradients<DefaultSpace<double>> + "
                          "CSROperator + DiagonalOperator (oracle/_ref) on the same system: %.3f s, i.e. %.2f ms per "
                          "iteration, scaled to the %d iterations of a complete solve"
                          % (stats[0] + 1, t, 1e3 * per_it, full_iterations + 1),
                "seconds_per_iteration": per_it}
    finally:
        ref.close()


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import torch  # noqa: F401  (only for problem construction on the GPU, not timed)
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import CUDASpace
    space = CUDASpace()
    prob = make_poisson(space, 3, 1, WORKLOAD["cells"], seed=WORKLOAD["seed"])
    rp, col, val, b = cpu_problem_arrays(prob)
    del prob, space
    from oracle.oracle import Reference
    ref = Reference()
    full = FULL_ITERATIONS_FP64
    times = []
    per_its = []
    budget = max(2.0, 150.0 / max(1, args.steps + args.warmup))
    _, _, _, t_probe = ref.pcg(rp, col, val, b, maxit=2, reltol=1e-10)
    m = int(max(3, min(full, budget / max(t_probe / 3.0, 1e-6) - 1)))
    for step in range(args.warmup + args.steps):
        _, stats, err, t = ref.pcg(rp, col, val, b, maxit=m, reltol=1e-10)
        if step >= args.warmup:
            per_its.append(t / (stats[0] + 1))
    ref.close()
    per_it = statistics.median(per_its)
    value = per_it * (full + 1)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * value, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": dict(WORKLOAD, parallelism="replicas"),
            "cpu_baseline": {"value": value, "unit": "s", "cores": ref.threads, "kind": "reference",
                             "sample": "each step: %d CG iterations of the reference's CPU solver (oracle/_ref), "
                                       "per-iteration time scaled to the %d iterations of a complete solve"
                                       % (m + 1, full + 1)},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# Iterations of the FP64 Jacobi-PCG on this seeded system (GPU solver; the compiled
# reference agrees within +-2 on the parity cases); used to scale CPU samples.
FULL_ITERATIONS_FP64 = 1000


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cie_b200", choices=["cie_b200", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
        return

    import torch
    import torch.distributed as dist
    from cie_b200 import _lib
    from cie_b200.fem import make_poisson
    from cie_b200.linalg import (CUDASpace, CSRMatrix, CSROperator, ConjugateGradients, Statistics,
                                 launch_count, makeDiagonalOperator)

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    space = CUDASpace()
    prob = make_poisson(space, 3, 1, WORKLOAD["cells"], seed=WORKLOAD["seed"])
    n, nnz = prob.mesh.ndofs, prob.matrix.nnz()
    A = CSROperator(prob.matrix, space)
    D = makeDiagonalOperator(prob.matrix, space, csr_handle=A.csr)
    settings = Statistics(20000, 0.0, WORKLOAD["tolerance"])
    cg = ConjugateGradients(A, space, D, settings)
    x = torch.zeros_like(prob.rhs)
    stream = torch.cuda.ExternalStream(space.stream.cuda_stream)

    def solve():
        x.zero_()
        cg.product(0.0, prob.rhs, 1.0, x)

    for _ in range(args.warmup):
        solve()
    iters = cg.getStats().iterationCount
    hbm, peak_kind = peaks()
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = launch_count()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        solve()
    e1.record(stream)
    barrier()
    t_solve = e0.elapsed_time(e1) / 1e3 / args.steps
    launches = launch_count() - launches0

    # dominant kernel: the CSR row pass (SpMV), timed live with CUDA events
    y = torch.empty_like(prob.rhs)
    spmv_reps = 20
    for _ in range(3):
        A.product(0.0, x, 1.0, y)
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(spmv_reps):
        A.product(0.0, x, 1.0, y)
    s1.record(stream)
    torch.cuda.synchronize()
    t_spmv = s0.elapsed_time(s1) / 1e3 / spmv_reps
    clocks = sampler.stop()

    t_tensor = torch.tensor([t_solve, t_spmv], device="cuda", dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t_tensor, op=dist.ReduceOp.MAX)
    t_solve, t_spmv = t_tensor.tolist()

    spmv_bytes = 12 * nnz + 4 * (n + 1) + 16 * n
    iter_bytes = 12 * nnz + 4 * (n + 1) + 104 * n
    solve_bytes = (iters + 1) * iter_bytes + (12 * nnz + 4 * (n + 1) + 24 * n)
    spmv_gbs = spmv_bytes / t_spmv / 1e9
    iter_gbs = solve_bytes / t_solve / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get("spmv_f64_poisson3d_q1_128", None)

    # end to end through the public API with host buffers
    rp_h, col_h, val_h = [t.cpu().pin_memory() for t in (prob.matrix.rowExtents, prob.matrix.columnIndices,
                                                          prob.matrix.entries)]
    rhs_h = prob.rhs.cpu().pin_memory()
    sol_h = torch.empty(n, dtype=torch.float64).pin_memory()
    e2e_times = []
    for step in range(2 + max(1, min(args.steps, 3))):
        barrier()
        t0 = time.perf_counter()
        m = CSRMatrix(n, rp_h.to("cuda", non_blocking=True), col_h.to("cuda", non_blocking=True),
                      val_h.to("cuda", non_blocking=True))
        b = rhs_h.to("cuda", non_blocking=True)
        A2 = CSROperator(m, space)
        cg2 = ConjugateGradients(A2, space, makeDiagonalOperator(m, space, csr_handle=A2.csr), settings)
        xe = torch.zeros(n, dtype=torch.float64, device="cuda")
        cg2.product(0.0, b, 1.0, xe)
        sol_h.copy_(xe, non_blocking=True)
        torch.cuda.synchronize()
        if step >= 2:
            e2e_times.append(time.perf_counter() - t0)
        del cg2, A2, m
    e2e = statistics.median(e2e_times)
    h2d = 4 * (n + 1) + 12 * nnz + 8 * n
    d2h = 8 * n

    # parity of the timed solve: true residual in FP64 on the GPU
    r = prob.rhs.clone()
    A.product(1.0, x, -1.0, r)
    true_rel = float(torch.linalg.norm(r) / torch.linalg.norm(prob.rhs))

    cpu = None
    if rank == 0 and not args.no_cpu:
        rp, col, val, bh = cpu_problem_arrays(prob)
        cpu = cpu_reference_sample(rp, col, val, bh, iters, budget_s=args.cpu_budget)

    if rank == 0:
        line = {
            "metric": METRIC, "value": t_solve, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_solve, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded mt19937_64 RHS and kappa field)",
            "config": dict(WORKLOAD, parallelism="replicas" if world > 1 else "single_gpu",
                           solver="fp64 jacobi-pcg", iterations=iters, true_relative_residual=true_rel),
            "fp64": {"seconds": t_solve, "iterations": iters, "true_relative_residual": true_rel},
            "roofline": {"bound": "hbm", "kernel": "csr spmv (ciecu spmv_kernel, schedule %d)" % A.csr.kernel(),
                         "achieved": spmv_gbs, "peak": hbm, "unit": "GB/s", "frac": spmv_gbs / hbm,
                         "peak_kind": peak_kind, "traffic": traffic, "algorithmic_bytes": spmv_bytes,
                         "launch_ms": 1e3 * t_spmv},
            "pcg_iteration_roofline": {"achieved": iter_gbs, "peak": hbm, "unit": "GB/s", "frac": iter_gbs / hbm,
                                       "algorithmic_bytes_per_iteration": iter_bytes,
                                       "us_per_iteration": 1e6 * t_solve / (iters + 1)},
            "clocks": clocks,
            "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
