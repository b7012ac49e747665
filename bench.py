"""Benchmark of the linear-solve hot path on one B200 (or N independent replicas).

Workload (one step = one complete solve): 3D Poisson, trilinear Q1 hexahedra on
128^3 cells of the unit cube (2,146,689 DoFs, 57,066,625 nonzeros, int32 CSR),
kappa = exp(smoothed unit-variance Gaussian field), RHS uniform [-1, 1] (seed 0),
homogeneous Dirichlet boundary by symmetric elimination, Jacobi-preconditioned CG
to ||r||/||b|| <= 1e-10 from x = 0.  Matrix assembled on the GPU (untimed set-up).

Metric: PCG time-to-1e-10 in seconds (lower is better).  value = the headline
mixed-precision solver (FP32 inner CG with FP64 reliable updates, stopping on the
true FP64 residual) per solve with inputs resident in HBM (inputs are larger than
L2, so no flush is needed); the plain FP64 PCG (the drop-in) is timed beside it.
e2e = the mixed solve through the public API with host buffers (H2D of CSR + RHS
from pinned memory, operator set-up, solve, D2H of the solution, all timed).
roofline = the headline's dominant kernel (the FP32 inner SpMV: over the diagonal-
storage copy for this 27-diagonal matrix, else SELL-32) timed live with CUDA
events; the FP64 CSR operator SpMV and whole-iteration rooflines are reported
beside it, and the reference's threaded CPU solver is timed on the same system.

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
# Smaller case of the same workload for ncu captures (matrix 290 MB, still above L2).
PROFILE_CELLS = [96, 96, 96]
# Reliable-update trigger of the mixed solver: replace the FP32 residual by the FP64
# one when it has fallen below DELTA times its running maximum.  On the 128^3 system
# 0.1 gives 10 replacements and a solution 2e-11 from the FP64 solver's; 0.01 saves
# 5 replacements but lands 1.1e-9 away, outside the 1e-9 parity bar.
DELTA = 0.1
# Inner-iteration form of the mixed solver (MixedPrecisionCG fuseDirection): 1 = the
# search direction and its product formed by recurrence inside the inner SpMV (two
# kernels per inner iteration), 2 = one kernel per inner iteration over the FP32 DIA
# copy (pending step, direction and product in one row pass), 0 = a separate
# direction kernel (three).  OTHER_FORM is timed beside it on the same system: at
# 128^3 the one-kernel form measured 38.0 ms against 27.7 ms for the two-kernel
# form (its row pass forms each operand entry from r, q, p and D^-1, where the
# two-kernel pass gathers z).
FUSE = 1
OTHER_FORM = 2
FORM_NAMES = {0: "three kernels per inner iteration (separate direction kernel)",
              1: "two kernels per inner iteration (fused direction)",
              2: "one kernel per inner iteration (single pass)"}
# Two-level CG on the finite-cell Q3 sphere: (smoothing precision, Chebyshev
# degree, pipelined coarse PCG iterations per cycle)
TWO_LEVEL = (("f64", 4, 80), ("f32", 6, 80))
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


def common_config(world):
    """The config both arms print (the workload, nothing about either solver)."""
    return dict(WORKLOAD, parallelism="replicas" if world > 1 else "single_gpu")


def compact(v, digits=4):
    """Floats rounded to `digits` significant digits, recursively (keeps the line short)."""
    if isinstance(v, float):
        return float("%.*g" % (digits, v)) if np.isfinite(v) else v
    if isinstance(v, dict):
        return {k: compact(x, digits) for k, x in v.items()}
    if isinstance(v, (list, tuple)):
        return [compact(x, digits) for x in v]
    return v


def oracle_system():
    """The workload's system built on the host by the oracle (no CUDA library):
    the arrays the reference arm solves."""
    from oracle.oracle import Restatement, system_digest
    rp, col, val, b, _, _ = Restatement().poisson_system(3, 1, WORKLOAD["cells"], seed=WORKLOAD["seed"])
    return (rp, col, val, b), system_digest(rp, col, val, b)


def reference_solve(rp, col, val, b, full_iterations, budget_s=15.0, threads=None):
    """The reference's threaded FP64 CG (oracle/_ref) on the same system.  Returns
    (cpu_baseline, x_ref, iterations): a complete solve when it is expected to
    end within max(budget, 120 s) -- its solution then anchors the parity of the
    GPU solutions -- else a bounded number of iterations scaled to a complete
    solve (no solution)."""
    from oracle.oracle import Reference, reference_available
    if not reference_available():
        return None, None, None
    ref = Reference(threads=threads)
    try:
        _, _, err, t_probe = ref.pcg(rp, col, val, b, maxit=2, reltol=1e-10)
        per_it = max(t_probe / 3.0, 1e-6)
        if per_it * (full_iterations + 1) <= max(budget_s, 120.0):
            x, stats, err, t = ref.pcg(rp, col, val, b, maxit=20000, reltol=1e-10)
            if err:
                raise RuntimeError(err)
            base = {"value": t, "unit": "s", "cores": ref.threads, "kind": "reference",
                    "sample": "one complete solve to 1e-10 (%d iterations) with the reference's ConjugateGradients"
                              "<DefaultSpace<double>> + CSROperator + DiagonalOperator built from its sources "
                              "(oracle/_ref), same system" % int(stats[0])}
            return base, x, int(stats[0])
        m = int(max(3, budget_s / per_it - 1))
        _, stats, err, t = ref.pcg(rp, col, val, b, maxit=m, reltol=1e-10)
        per_it = t / (stats[0] + 1)
        return ({"value": per_it * (full_iterations + 1), "unit": "s", "cores": ref.threads, "kind": "reference",
                 "sample": "%d CG iterations of the reference's CPU solver (oracle/_ref) on the same system, "
                           "scaled to the %d iterations of a complete solve" % (stats[0] + 1, full_iterations + 1)},
                None, None)
    finally:
        ref.close()


def run_reference_arm(args):
    """The reference's own threaded FP64 CPU solver (oracle/_ref: ConjugateGradients<
    DefaultSpace<double>> + CSROperator + DiagonalOperator over mp::ThreadPoolBase with
    every host thread) on the workload's system, built on the host by the oracle
    (bit-identical to the GPU-assembled one: same digest); each step is a complete
    solve.  No CUDA library is loaded on this arm."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    (rp, col, val, b), digest = oracle_system()
    from oracle.oracle import Reference
    ref = Reference()
    times, its = [], []
    for step in range(args.warmup + args.steps):
        _, stats, err, t = ref.pcg(rp, col, val, b, maxit=20000, reltol=WORKLOAD["tolerance"])
        if err:
            raise RuntimeError(err)
        if step >= args.warmup:
            times.append(t)
            its.append(int(stats[0]))
    ref.close()
    value = statistics.median(times)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * value, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded mt19937_64 RHS and "
            "kappa field)", "config": common_config(world),
            "system_digest": digest, "iterations": its[-1],
            "cpu_baseline": {"value": value, "unit": "s", "cores": ref.threads, "kind": "reference",
                             "sample": "each step: one complete solve to 1e-10 (%d iterations) with the reference's "
                                       "CPU solver built from its own sources (oracle/_ref)" % its[-1]},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(compact(line, 6)), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cie_b200", choices=["cie_b200", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the other workloads (2D Q1 256^2, batched Q2 systems, 32 right-hand sides, adjoint)")
    ap.add_argument("--profile", action="store_true",
                    help="ncu target: solves only (no e2e, no CPU baseline, no clock sampling)")
    ap.add_argument("--profile-kernels", action="store_true",
                    help="with --profile: no solves, only three launches each of the FP32 SELL and FP64 CSR SpMV "
                         "after set-up (a short target for a full ncu capture)")
    ap.add_argument("--pin", default=None,
                    help="with --profile: FP64-solver,mixed-unroll,CSR schedules to use instead of autotuning "
                         "(the choices a bench run without the profiler reports), e.g. 4,1,4")
    ap.add_argument("--mixed-form", type=int, default=None, choices=[0, 1, 2],
                    help="with --profile: inner-iteration form of the mixed solver (fuseDirection) instead of the "
                         "benchmarked one")
    ap.add_argument("--profile-target", default="pcg",
                    choices=["pcg", "batch", "spmm", "spmm32", "embedded", "cut", "twolevel", "gradient"],
                    help="with --profile: the solver the ncu target runs (pcg: the headline solves; batch: a "
                         "batched solve of 128 Q2 systems; spmm: a 32-RHS solve on the Q1 grid of --profile-cells "
                         "(spmm32: its FP32 form with FP64 reliable updates); "
                         "embedded: the finite-cell Q3 assembly (FP64 and FP32) on --profile-cells^3 cells when that "
                         "is at most 32, else 16^3; twolevel: three iterations of the two-level CG with FP32 "
                         "smoothing on that system; cut: 30 FP64 Jacobi-PCG iterations "
                         "on that finite-cell system, on --profile-cells^3 cells when that is at most 24 "
                         "(--pin's first value pins the SpMV schedule); gradient: one "
                         "adjoint gradient on the Q1 grid of --profile-cells)")
    ap.add_argument("--profile-cells", type=int, default=PROFILE_CELLS[0],
                    help="cells per axis of the --profile case (96: 290 MB matrix; 128: the full workload)")
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
    from cie_b200.linalg import (CUDASpace, CSRMatrix, CSROperator, ConjugateGradients, MixedPrecisionCG,
                                 Statistics, launch_count, makeDiagonalOperator)

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    space = CUDASpace()
    if args.profile and args.profile_target != "pcg":
        profile_target(space, args.profile_target, args.profile_cells,
                       int(args.pin.split(",")[0]) if args.pin else 0)
        return
    cells = [args.profile_cells] * 3 if args.profile else WORKLOAD["cells"]
    prob = make_poisson(space, 3, 1, cells, seed=WORKLOAD["seed"])
    n, nnz = prob.mesh.ndofs, prob.matrix.nnz()
    settings = Statistics(20000, 0.0, WORKLOAD["tolerance"])
    if not args.profile:
        # host copies of the system (pinned) for the end-to-end runs and the CPU leg
        rp_h, col_h, val_h = [t.cpu().pin_memory() for t in (prob.matrix.rowExtents, prob.matrix.columnIndices,
                                                              prob.matrix.entries)]
        rhs_h = prob.rhs.cpu().pin_memory()
        sol_h = torch.empty(n, dtype=torch.float64).pin_memory()

        def e2e_solve():
            """The public API with host buffers: H2D of the CSR arrays and RHS, operator
            and solver set-up, the mixed solve, D2H of the solution."""
            m = CSRMatrix(n, rp_h.to("cuda", non_blocking=True), col_h.to("cuda", non_blocking=True),
                          val_h.to("cuda", non_blocking=True))
            b = rhs_h.to("cuda", non_blocking=True)
            A2 = CSROperator(m, space)
            D2 = makeDiagonalOperator(m, space, csr_handle=A2.csr)
            M2 = MixedPrecisionCG(A2, D2, settings, mode=0, delta=DELTA, fuseDirection=FUSE)
            xe = torch.zeros(n, dtype=torch.float64, device="cuda")
            M2.product(0.0, b, 1.0, xe)
            sol_h.copy_(xe, non_blocking=True)
            torch.cuda.synchronize()
            del M2, D2, A2, m

        # first call of the process on a matrix of this shape: includes the one-off
        # autotuning and the build of the inner-matrix copy, cached per shape after it
        barrier()
        t0 = time.perf_counter()
        e2e_solve()
        e2e_cold = time.perf_counter() - t0
    A = CSROperator(prob.matrix, space)
    D = makeDiagonalOperator(prob.matrix, space, csr_handle=A.csr)
    cg = ConjugateGradients(A, space, D, settings)
    form = args.mixed_form if (args.profile and args.mixed_form is not None) else FUSE
    if args.profile and args.pin:
        pin_fp64, pin_unroll, pin_csr = (int(v) for v in args.pin.split(","))
        A.csr.set_kernel(pin_csr)
        cg.set_schedule(pin_fp64)
        mixed = MixedPrecisionCG(A, D, settings, mode=0, delta=DELTA, innerKernel=pin_unroll, fuseDirection=form)
    else:
        mixed = MixedPrecisionCG(A, D, settings, mode=0, delta=DELTA, fuseDirection=FUSE)
    x64 = torch.zeros_like(prob.rhs)
    xmx = torch.zeros_like(prob.rhs)
    stream = torch.cuda.ExternalStream(space.stream.cuda_stream)

    def solve_fp64():
        x64.zero_()
        cg.product(0.0, prob.rhs, 1.0, x64)

    def solve_mixed():
        xmx.zero_()
        mixed.product(0.0, prob.rhs, 1.0, xmx)

    if args.profile and args.profile_kernels:
        from cie_b200.linalg import _ptr
        lib = _lib.load()
        x32, y32 = torch.rand(n, dtype=torch.float32, device="cuda"), torch.empty(n, dtype=torch.float32,
                                                                                   device="cuda")
        xr, yr = torch.rand(n, dtype=torch.float64, device="cuda"), torch.empty_like(prob.rhs)
        _lib.check(lib.ciecu_csr_spmv_f64(A.csr.handle, 0.0, _ptr(xr), 1.0, _ptr(yr)))  # schedule tuned here
        space.synchronize()
        torch.cuda.nvtx.range_push("profile_kernels")  # ncu --nvtx --nvtx-include "profile_kernels/"
        for _ in range(3):
            _lib.check(lib.ciecu_mixed_apply_f32(mixed._solver, _ptr(x32), _ptr(y32)))
            _lib.check(lib.ciecu_csr_spmv_f64(A.csr.handle, 0.0, _ptr(xr), 1.0, _ptr(yr)))
        space.synchronize()
        torch.cuda.nvtx.range_pop()
        print(json.dumps({"profile": True, "kernels_only": True, "cells": cells, "fp64_info": cg.info(),
                          "mixed_info": mixed.info()}), flush=True)
        return
    for _ in range(args.warmup):
        solve_mixed()
        solve_fp64()
    it64 = cg.getStats().iterationCount
    mst = mixed.getStats()
    if args.profile:
        from cie_b200.linalg import _ptr
        lib = _lib.load()
        x32, y32 = xmx.float(), torch.empty(n, dtype=torch.float32, device="cuda")
        for _ in range(args.steps):
            solve_mixed()
            solve_fp64()
            for _ in range(3):
                lib.ciecu_mixed_apply_f32(mixed._solver, _ptr(x32), _ptr(y32))
                lib.ciecu_csr_spmv_f64(A.csr.handle, 0.0, _ptr(x64), 1.0, _ptr(prob.rhs.clone()))
        torch.cuda.synchronize()
        print(json.dumps({"profile": True, "cells": cells, "fp64_iterations": it64, "fp64_info": cg.info(),
                          "mixed_info": mixed.info(),
                          "mixed_inner": mst.innerIterations, "mixed_refinements": mst.refinements}), flush=True)
        return
    hbm, peak_kind = peaks()

    def timed(fn, reps):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        barrier()
        return e0.elapsed_time(e1) / 1e3 / reps

    sampler = ClockSampler(local)
    sampler.start()
    launches0 = launch_count()
    t_mixed = timed(solve_mixed, args.steps)
    t_fp64 = timed(solve_fp64, args.steps)
    launches = launch_count() - launches0

    # the other inner-iteration form on the same system (reported, not the headline)
    other = MixedPrecisionCG(A, D, settings, mode=0, delta=DELTA, fuseDirection=OTHER_FORM)
    xother = torch.zeros_like(prob.rhs)

    def solve_other():
        xother.zero_()
        other.product(0.0, prob.rhs, 1.0, xother)

    for _ in range(2):
        solve_other()
    t_other = timed(solve_other, args.steps)
    ost = other.getStats()

    # dominant kernels, timed live with CUDA events on the launching stream
    lib = _lib.load()
    from cie_b200.linalg import _ptr
    y64 = torch.empty_like(prob.rhs)
    x32 = xmx.float()
    y32 = torch.empty_like(x32)
    reps = 50

    def apply32():
        for _ in range(reps):
            lib.ciecu_mixed_apply_f32(mixed._solver, _ptr(x32), _ptr(y32))

    def apply64():
        for _ in range(reps):
            lib.ciecu_csr_spmv_f64(A.csr.handle, 0.0, _ptr(x64), 1.0, _ptr(y64))

    apply32()  # warm-up launches of both kernels
    apply64()
    t_spmv32 = timed(apply32, 1) / reps
    t_spmv64 = timed(apply64, 1) / reps
    clocks = sampler.stop()

    from cie_b200.sharding import max_over_ranks
    t_mixed, t_fp64, t_spmv32, t_spmv64, t_other = max_over_ranks([t_mixed, t_fp64, t_spmv32, t_spmv64, t_other])
    info = mixed.info()

    ndiag = A.csr.diagonals()
    dia32 = info.get("format") == "dia"
    dia64 = cg.info().get("spmv_schedule") == 64
    idx_bytes = 2 if info.get("compressed_columns") else 4
    if dia32:
        # FP32 DIA SpMV: the stored diagonals (nonzeros and the zeros that pad the
        # diagonals), x read, y written; no column indices
        spmv32_bytes = 4 * ndiag * n + 8 * n
        inner_bytes = 4 * ndiag * n + 52 * n
    else:
        # FP32 SELL-32 SpMV: values + column offsets of the nonzeros, x read, y written
        # (padding entries and the per-slice descriptors are reported, not counted)
        spmv32_bytes = (4 + idx_bytes) * nnz + 8 * n
        inner_bytes = (4 + idx_bytes) * nnz + 52 * n
    spmv64_bytes = 12 * nnz + 4 * (n + 1) + 16 * n
    stored64 = cg.info().get("dia_stored_diagonals") or ndiag
    iter64_bytes = (8 * stored64 * n if dia64 else 12 * nnz + 4 * (n + 1)) + 104 * n
    fp64_solve_bytes = (it64 + 1) * iter64_bytes + (12 * nnz + 4 * (n + 1) + 24 * n)
    refine_bytes = 12 * nnz + 4 * (n + 1) + 28 * n  # FP64 residual pass: x64, b read, r32 written, dinv32
    mixed_solve_bytes = mst.innerIterations * inner_bytes + (mst.refinements + 1) * refine_bytes
    # DRAM bytes per launch from the committed ncu capture of the same kernel on the same workload
    traffic = traffic64 = None
    tpath = os.path.join(ROOT, "profiles", "dram_traffic_poisson3d_q1_128.txt")
    if os.path.exists(tpath) and cells == [128, 128, 128]:
        figures = dict(line.split() for line in open(tpath) if line.strip() and not line.startswith("#"))
        if dia32:
            key = "mixed_apply_dia_kernel_f32" + ("_triples" if info.get("dia_triples") else "")
            traffic = int(figures.get(key, 0)) or None
        elif info["compressed_columns"] and info["group_unroll"] > 0:
            traffic = int(figures.get("mixed_apply_kernel_f32_sell16", 0)) or None
        traffic64 = int(figures.get("spmv_kernel_f64_csr", 0)) or None

    # end to end through the public API with host buffers (warm: the shape's tuning is cached)
    e2e_times = []
    for step in range(max(1, min(args.steps, 3))):
        barrier()
        t0 = time.perf_counter()
        e2e_solve()
        e2e_times.append(time.perf_counter() - t0)
    e2e = statistics.median(e2e_times)
    h2d = 4 * (n + 1) + 12 * nnz + 8 * n
    d2h = 8 * n

    # accuracy of the timed solves: true FP64 residuals and agreement of the two solvers
    def true_rel(x):
        r = prob.rhs.clone()
        A.product(1.0, x, -1.0, r)
        return float(torch.linalg.norm(r) / torch.linalg.norm(prob.rhs))
    rel_mixed, rel_fp64, rel_other = true_rel(xmx), true_rel(x64), true_rel(xother)
    agree = float(torch.linalg.norm(xmx - x64) / torch.linalg.norm(x64))

    extra = None
    if not args.no_extra:
        extra = extra_workloads(space, A, D, settings, t_fp64, it64, rank, world)

    # CPU leg (rank 0): the oracle rebuilds the system on the host without the CUDA
    # library (the reference arm's input; same digest = same bits), the reference's
    # threaded CPU CG solves it, and its solution anchors the parity of both GPU solves
    cpu = parity = None
    if rank == 0 and not args.no_cpu:
        rp, col, val, bh = (t.numpy() for t in (rp_h, col_h, val_h, rhs_h))
        from oracle.oracle import system_digest
        digest = system_digest(rp, col, val, bh)
        (orp, ocol, oval, ob), odigest = oracle_system()
        same = digest == odigest
        cpu, x_ref, it_ref = reference_solve(orp, ocol, oval, ob, it64, budget_s=args.cpu_budget)
        parity = {"system_digest": digest, "oracle_system_digest": odigest, "bit_identical_to_oracle": same}
        if not same:
            parity["max_entry_rel_diff"] = float(np.abs(val - oval).max() / np.abs(oval).max())
        del orp, ocol, oval, ob
        if x_ref is not None:
            xr = np.linalg.norm(x_ref)
            parity.update({"reference_iterations": it_ref,
                           "mixed_rel_err_vs_reference": float(np.linalg.norm(xmx.cpu().numpy() - x_ref) / xr),
                           "fp64_rel_err_vs_reference": float(np.linalg.norm(x64.cpu().numpy() - x_ref) / xr)})

    if rank == 0:
        g32 = spmv32_bytes / t_spmv32 / 1e9
        # key order: the long blocks first, the headline blocks last (the end of the
        # line is what a log tail shows)
        line = {
            "metric": METRIC, "value": t_mixed, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_mixed, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 inner / f64 refinement",
            "data": "synthetic (seeded mt19937_64 RHS and kappa field)",
            "config": common_config(world),
            "solver": {"mixed": "jacobi-pcg, FP32 inner over %s, FP64 reliable updates delta=%g, %s" % (
                           info["format"], DELTA, FORM_NAMES[3 - mixed.kernels_per_iteration]),
                       "fp64": "jacobi-pcg over %s" % (("dia, symmetric upper half" if cg.info().get(
                           "dia_symmetric") else "dia") if dia64 else "csr")},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "workloads": extra,
            "fp64_spmv_roofline": {"kernel": "spmv_kernel (FP64 CSR, schedule %d)" % A.csr.kernel(),
                                   "achieved": spmv64_bytes / t_spmv64 / 1e9, "peak": hbm,
                                   "frac": spmv64_bytes / t_spmv64 / 1e9 / hbm, "algorithmic_bytes": spmv64_bytes,
                                   "traffic": traffic64, "launch_ms": 1e3 * t_spmv64},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "cold_first_call_s": e2e_cold, "solver": "mixed"},
            "fp64": {"seconds": t_fp64, "iterations": it64, "true_relative_residual": rel_fp64,
                     "us_per_iteration": 1e6 * t_fp64 / (it64 + 1), "achieved_gbs": fp64_solve_bytes / t_fp64 / 1e9},
            "mixed": {"seconds": t_mixed, "inner_iterations": mst.innerIterations,
                      "refinements": mst.refinements, "true_relative_residual": rel_mixed,
                      "rel_diff_vs_fp64_solution": agree, "achieved_gbs": mixed_solve_bytes / t_mixed / 1e9},
            "mixed_other_form": {"form": FORM_NAMES[3 - other.kernels_per_iteration],
                                 "seconds": t_other, "inner_iterations": ost.innerIterations,
                                 "refinements": ost.refinements, "true_relative_residual": rel_other,
                                 "achieved_gbs": (ost.innerIterations * inner_bytes +
                                                  (ost.refinements + 1) * refine_bytes) / t_other / 1e9},
            "speedup_mixed_vs_fp64": t_fp64 / t_mixed,
            "pcg_iteration_roofline": {"fp64_frac": fp64_solve_bytes / t_fp64 / 1e9 / hbm,
                                       "mixed_frac": mixed_solve_bytes / t_mixed / 1e9 / hbm},
            "parity": parity,
            "roofline": {"bound": "hbm", "kernel": (
                             "mixed_apply_dia_kernel (FP32 DIA SpMV, %d diagonals%s)" % (
                                 ndiag, ", triple pass" if info.get("dia_triples") else "")) if dia32 else (
                             "%s (FP32 SELL-32 SpMV)" % ("mixed_apply_kernel<%d>" % info["group_unroll"]
                                                         if info["group_unroll"] > 0 else "mixed_apply_tma_kernel")),
                         "achieved": g32, "peak": hbm, "unit": "GB/s", "frac": g32 / hbm, "peak_kind": peak_kind,
                         "traffic": traffic, "algorithmic_bytes": spmv32_bytes, "launch_ms": 1e3 * t_spmv32},
        }
        print(json.dumps(compact(line)), flush=True)
    if world > 1:
        dist.destroy_process_group()


def profile_target(space, target, cells, schedule=0):
    """Short runs of the other solvers for ncu (inputs built first, one solve or
    assembly, no timing)."""
    import torch
    from cie_b200.fem import kappa_field, make_embedded_poisson, make_poisson, random_uniform
    from cie_b200.linalg import (BatchedConjugateGradients, ConjugateGradients, CSROperator,
                                 MultiRHSConjugateGradients, Statistics, block_diagonal, makeDiagonalOperator)
    tight = Statistics(20000, 0.0, 1e-10)
    if target == "batch":
        rng = np.random.default_rng(0)
        sizes = rng.integers(16, 129, 128)
        probs = [make_poisson(space, 2, 2, [int(m), int(m)], seed=1000 + 3 * i) for i, m in enumerate(sizes)]
        bd, offsets = block_diagonal([p.matrix for p in probs])
        rhs = torch.cat([p.rhs for p in probs])
        solver = BatchedConjugateGradients(bd, offsets, space, makeDiagonalOperator(bd, space), tight)
        x = torch.zeros_like(rhs)
        solver.product(0.0, rhs, 1.0, x)
        info = solver.info()
    elif target in ("spmm", "spmm32"):
        prob = make_poisson(space, 3, 1, [cells] * 3, seed=0)
        n = prob.rhs.numel()
        A = CSROperator(prob.matrix, space)
        D = makeDiagonalOperator(prob.matrix, space, csr_handle=A.csr)
        B = torch.as_tensor(np.stack([random_uniform(2000 + c, n) for c in range(32)], axis=1)).cuda().contiguous()
        solver = MultiRHSConjugateGradients(A, D, 32, tight)
        if target == "spmm32":
            solver.set_refinement(DELTA)
        X = torch.zeros_like(B)
        solver.product(0.0, B, 1.0, X)
        info = solver.info()
    elif target == "embedded":
        # the FP64 (DMMA) assembly inside the set-up, then the FP32 (split-BF16) one
        c = cells if cells <= 32 else 16
        prob = make_embedded_poisson(space, 3, 3, [c, c, c], radius=0.4, alpha=1e-6, depth=2)
        v32 = torch.zeros(prob.matrix.entries.numel(), dtype=torch.float32, device="cuda")
        prob.assembler.assemble_embedded_f32(v32, [0.5] * 3, 0.4, 1e-6, 2)
        info = {"cut_cells": prob.cut_cells, "cells": c}
    elif target == "twolevel":
        # three outer iterations of the device two-level CG (FP32 smoothing) on the
        # finite-cell sphere of --profile-cells^3 cells (at most 32)
        from cie_b200.twolevel import make_two_level_cg
        c = cells if cells <= 32 else 16
        prob = make_embedded_poisson(space, 3, 3, [c, c, c], radius=0.4, alpha=1e-6, depth=2)
        precision, degree, coarse = TWO_LEVEL[-1]
        solver = make_two_level_cg(space, prob, Statistics(3, 0.0, 1e-10), degree=degree, coarseIterations=coarse,
                                   precision=precision)
        x = torch.zeros_like(prob.rhs)
        solver.product(0.0, prob.rhs, 1.0, x)
        info = dict(solver.info(), cells=c, degree=degree, coarse=coarse)
    elif target == "cut":
        c = cells if cells <= 24 else 16
        prob = make_embedded_poisson(space, 3, 3, [c, c, c], radius=0.4, alpha=1e-6, depth=2)
        A = CSROperator(prob.matrix, space)
        cg = ConjugateGradients(A, space, makeDiagonalOperator(prob.matrix, space, csr_handle=A.csr),
                                Statistics(30, 0.0, 1e-10))
        cg.set_loop(1)
        if schedule:
            cg.set_schedule(schedule)
        x = torch.zeros_like(prob.rhs)
        cg.product(0.0, prob.rhs, 1.0, x)
        info = dict(cg.info(), nnz=prob.matrix.nnz(), dofs=prob.rhs.numel())
    else:
        from cie_b200.adjoint import DifferentiablePoisson
        prob = DifferentiablePoisson(space, 3, 1, [cells] * 3, settings=tight)
        kappa = torch.as_tensor(kappa_field(1, [cells] * 3)).cuda().requires_grad_(True)
        b = torch.as_tensor(random_uniform(0, prob.n)).cuda()
        u = prob(kappa, b)
        (0.5 * torch.sum(u ** 2)).backward()
        info = {"adjoint_iterations": prob.adjoint_stats.iterationCount}
    torch.cuda.synchronize()
    print(json.dumps({"profile": True, "target": target, "info": info}), flush=True)


def extra_workloads(space, A, D, settings, t_fp64, it64, rank=0, world=1):
    """The other workloads of the path, each timed with CUDA events around complete
    solves (inputs resident on the device):
      * 2D Q1 Poisson 256^2, kappa = 1: FP64 Jacobi-PCG to 1e-10;
      * 512 independent 2D Q2 systems on n x n meshes, n ~ U{16..128} (seeded), each
        with its own log-normal kappa: one batched solve vs the same systems solved
        one after another with the single-system solver;
      * 32 right-hand sides (uniform [-1, 1]) on the 128^3 Q1 matrix: one SpMM-CG
        vs 32 single solves (the FP64 time measured above, times 32);
      * adjoint gradient of J = 1/2 ||u - u_t||^2 on 3D Q1 64^3: forward solve and
        backward (transposed solve + per-element gradient).
    Under torchrun (world > 1) only the batched solve runs: the 512 systems are
    dealt out to the ranks by nonzero count, each rank solves its share, and the
    time is the max over ranks (total work fixed)."""
    import torch
    from cie_b200.adjoint import DifferentiablePoisson
    from cie_b200.fem import kappa_field, make_poisson, random_uniform
    from cie_b200.linalg import (BatchedConjugateGradients, CSROperator, ConjugateGradients,
                                 MultiRHSConjugateGradients, Statistics, block_diagonal, makeDiagonalOperator)
    stream = torch.cuda.current_stream()

    def timed(fn, reps, warm=1):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps

    out = {}
    tight = Statistics(5000, 0.0, 1e-10)
    if world > 1:
        from cie_b200.sharding import max_over_ranks, shard_by_weight
        rng = np.random.default_rng(0)
        sizes = rng.integers(16, 129, 512)
        mine = shard_by_weight((8 * sizes + 1) ** 2, world, rank)
        probs = [make_poisson(space, 2, 2, [int(sizes[i]), int(sizes[i])], seed=1000 + 3 * i) for i in mine]
        bd, offsets = block_diagonal([p.matrix for p in probs])
        rhs = torch.cat([p.rhs for p in probs])
        batch = BatchedConjugateGradients(bd, offsets, space, makeDiagonalOperator(bd, space), tight)
        xb = torch.zeros_like(rhs)

        def solve_shard():
            xb.zero_()
            batch.product(0.0, rhs, 1.0, xb)
        ts = timed(solve_shard, 3)
        tmax, = max_over_ranks([ts])
        out["batched_512_poisson2d_q2_fp64_pcg"] = {
            "seconds": tmax, "systems": 512, "ranks": world, "systems_this_rank": len(mine),
            "scaling": "strong (the 512 systems split over the ranks by nonzero count, no exchange)"}
        return out
    # 2D Q1 256^2
    p1 = make_poisson(space, 2, 1, [256, 256], seed=0, kappa="one")
    A1 = CSROperator(p1.matrix, space)
    cg1 = ConjugateGradients(A1, space, makeDiagonalOperator(p1.matrix, space, csr_handle=A1.csr), tight)
    x1 = torch.zeros_like(p1.rhs)

    def solve1():
        x1.zero_()
        cg1.product(0.0, p1.rhs, 1.0, x1)
    t1 = timed(solve1, 5, warm=3)
    out["poisson2d_q1_256^2_fp64_pcg"] = {"seconds": t1, "iterations": cg1.getStats().iterationCount,
                                         "dofs": p1.rhs.numel(), "nnz": p1.matrix.nnz(),
                                         "us_per_iteration": 1e6 * t1 / (cg1.getStats().iterationCount + 1)}
    del cg1, A1, p1, x1

    # 512 uneven 2D Q2 systems
    rng = np.random.default_rng(0)
    sizes = rng.integers(16, 129, 512)
    probs = [make_poisson(space, 2, 2, [int(m), int(m)], seed=1000 + 3 * i) for i, m in enumerate(sizes)]
    bd, offsets = block_diagonal([p.matrix for p in probs])
    rhs = torch.cat([p.rhs for p in probs])
    Dbd = makeDiagonalOperator(bd, space)
    batch = BatchedConjugateGradients(bd, offsets, space, Dbd, tight)
    xb = torch.zeros_like(rhs)

    def solveb():
        xb.zero_()
        batch.product(0.0, rhs, 1.0, xb)
    tb = timed(solveb, 3)
    its = [s.iterationCount for s in batch.getStats()]
    rels = [s.relativeResidual for s in batch.getStats()]
    # the same batch in FP32 with FP64 reliable updates per system (the Krylov space
    # kept across replacements), and with restarted FP32 inner solves to 1e-4 per
    # FP64 refinement round for comparison
    xr = torch.zeros_like(rhs)
    refined = BatchedConjugateGradients(bd, offsets, space, Dbd, tight)
    refined.set_reliable_updates(DELTA)

    def solve_reliable():
        xr.zero_()
        refined.product(0.0, rhs, 1.0, xr)
    tr = timed(solve_reliable, 3)
    rits = [s.iterationCount for s in refined.getStats()]
    rreps = refined.refinements()
    rrel = max(s.relativeResidual for s in refined.getStats())
    rdiff = float(torch.linalg.norm(xr - xb) / torch.linalg.norm(xb))
    refined.set_reliable_updates(0.0)
    refined.set_refinement(1e-4)

    def solve_restarted():
        xr.zero_()
        refined.product(0.0, rhs, 1.0, xr)
    t_restart = timed(solve_restarted, 1)
    del refined
    # the same systems one after another (one solver object per system)
    singles = []
    for p in probs:
        Ap = CSROperator(p.matrix, space)
        singles.append((ConjugateGradients(Ap, space, makeDiagonalOperator(p.matrix, space, csr_handle=Ap.csr),
                                           tight), p, torch.zeros_like(p.rhs), Ap))

    def solve_each():
        for cg, p, xs, _ in singles:
            xs.zero_()
            cg.product(0.0, p.rhs, 1.0, xs)
    ts = timed(solve_each, 1)
    agree = float(torch.linalg.norm(xb - torch.cat([xs for _, _, xs, _ in singles])) / torch.linalg.norm(xb))
    out["batched_512_poisson2d_q2_fp64_pcg"] = {
        "seconds": tb, "systems": len(probs), "total_dofs": int(rhs.numel()), "total_nnz": bd.nnz(),
        "iterations_min": int(min(its)), "iterations_max": int(max(its)), "max_relative_residual": max(rels),
        "sequential_single_solves_seconds": ts, "speedup_vs_sequential": ts / tb,
        "rel_diff_vs_single_solves": agree, "solver": batch.info(),
        "fp32_refined_seconds": tr, "fp32_refined_form": "FP32 iterations, FP64 reliable updates delta=%g" % DELTA,
        "fp32_refined_iterations_max": int(max(rits)), "fp32_refined_replacements_max": int(max(rreps)),
        "fp32_refined_max_relative_residual": rrel, "fp32_refined_rel_diff_vs_fp64": rdiff,
        "fp32_refined_speedup_vs_fp64": tb / tr, "fp32_restarted_refinement_1e-4_seconds": t_restart}
    del singles, batch, Dbd, bd, rhs, xb, xr, probs

    # 32 right-hand sides on the 128^3 matrix
    n = A.lhs.rowCount()
    k = 32
    B = torch.as_tensor(np.stack([random_uniform(2000 + c, n) for c in range(k)], axis=1)).cuda().contiguous()
    mrhs = MultiRHSConjugateGradients(A, D, k, settings)
    X = torch.zeros_like(B)

    def solvem():
        X.zero_()
        mrhs.product(0.0, B, 1.0, X)
    tm = timed(solvem, 2)
    its = [s.iterationCount for s in mrhs.getStats()]
    fmt = mrhs.info()["spmm_format"]
    X64 = X.clone()
    # the FP32-refined form of the same 32 solves (FP32 SpMM iterations, FP64
    # reliable updates per column)
    mrhs.set_refinement(DELTA)
    solvem()
    tmr = timed(solvem, 2)
    rits = [s.iterationCount for s in mrhs.getStats()]
    refs = mrhs.refinements()
    rres = max(s.relativeResidual for s in mrhs.getStats())
    rdiff = max(float(torch.linalg.norm(X[:, c] - X64[:, c]) / torch.linalg.norm(X64[:, c])) for c in range(k))
    mrhs.set_refinement(0.0)
    solvem()
    out["multi_rhs_32_poisson3d_q1_128^3_fp64_pcg"] = {
        "seconds": tm, "rhs": k, "spmm_format": fmt, "iterations_min": int(min(its)), "iterations_max": int(max(its)),
        "max_relative_residual": max(s.relativeResidual for s in mrhs.getStats()),
        "seconds_per_rhs": tm / k, "single_solve_seconds": t_fp64, "speedup_vs_32_single_solves": 32 * t_fp64 / tm,
        "fp32_refined_seconds": tmr, "fp32_refined_iterations_max": int(max(rits)),
        "fp32_refined_replacements_max": int(max(refs)), "fp32_refined_max_relative_residual": rres,
        "fp32_refined_max_rel_diff_vs_fp64": rdiff, "fp32_refined_speedup_vs_fp64": tm / tmr,
        "note": "random right-hand sides, boundary rows included (identity rows of the eliminated system)"}
    del mrhs, X, B, X64

    # embedded (finite-cell) Q3 sphere on 32^3 cells: set-up (pattern on the host and
    # on the device, FP64 and FP32 tensor-core assembly), FP64 Jacobi-PCG, and the
    # device two-level CG with FP64 and with FP32 smoothing (outer iteration FP64)
    from cie_b200.fem import make_embedded_poisson, csr_pattern
    from cie_b200.graph import csr_pattern_device
    from cie_b200.twolevel import make_two_level_cg
    pe = make_embedded_poisson(space, 3, 3, [32, 32, 32], radius=0.4, alpha=1e-6, depth=2, seed=0)
    torch.cuda.synchronize()
    em = pe.mesh
    t0 = time.perf_counter()
    csr_pattern(em.ncells, em.nb, em.dofmap, em.ndofs)
    t_pattern_host = time.perf_counter() - t0
    d_dofmap = pe.assembler.d_dofmap
    csr_pattern_device(space, em.ncells, em.nb, d_dofmap, em.ndofs)  # warm-up (module load)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    csr_pattern_device(space, em.ncells, em.nb, d_dofmap, em.ndofs)
    torch.cuda.synchronize()
    t_pattern_dev = time.perf_counter() - t0
    t0 = time.perf_counter()
    pe.assembler.assemble_embedded([0.5] * 3, 0.4, 1e-6, 2)
    pe.assembler.dirichlet(pe.boundary)
    torch.cuda.synchronize()
    t_asm = time.perf_counter() - t0
    v32 = torch.zeros(pe.matrix.entries.numel(), dtype=torch.float32, device="cuda")
    t0 = time.perf_counter()
    pe.assembler.assemble_embedded_f32(v32, [0.5] * 3, 0.4, 1e-6, 2)
    torch.cuda.synchronize()
    t_asm32 = time.perf_counter() - t0
    pe.assembler.dirichlet_f32(pe.boundary, v32)
    asm32_err = float((v32.double() - pe.matrix.entries).abs().max() / pe.matrix.entries.abs().max())
    del v32
    Ae = CSROperator(pe.matrix, space)
    cge = ConjugateGradients(Ae, space, makeDiagonalOperator(pe.matrix, space, csr_handle=Ae.csr),
                             Statistics(200000, 0.0, 1e-10))
    xe = torch.zeros_like(pe.rhs)

    def solve_jacobi():
        xe.zero_()
        cge.product(0.0, pe.rhs, 1.0, xe)
    tj = timed(solve_jacobi, 1, warm=0)
    itj = cge.getStats().iterationCount
    emb = {"dofs": pe.rhs.numel(), "nnz": pe.matrix.nnz(), "cut_cells": pe.cut_cells,
           "pattern_host_seconds": t_pattern_host, "pattern_device_seconds": t_pattern_dev,
           "assembly_fp64_seconds": t_asm, "assembly_fp32_tensor_core_seconds": t_asm32,
           "fp32_matrix_max_rel_entry_error": asm32_err,
           "jacobi_pcg_seconds": tj, "jacobi_pcg_iterations": itj, "jacobi_us_per_iteration": 1e6 * tj / (itj + 1)}
    del cge
    for precision, degree, coarse in TWO_LEVEL:
        solver = make_two_level_cg(space, pe, Statistics(20000, 0.0, 1e-10), degree=degree, coarseIterations=coarse,
                                   precision=precision)
        xm = torch.zeros_like(pe.rhs)

        def solve_mg():
            xm.zero_()
            solver.product(0.0, pe.rhs, 1.0, xm)
        tmg = timed(solve_mg, 1, warm=1)
        st = solver.getStats()
        info = solver.info()
        r = pe.rhs.clone()
        Ae.product(1.0, xm, -1.0, r)
        entry = {
            "seconds": tmg, "iterations": st.iterationCount, "chebyshev_degree": degree, "coarse_iterations": coarse,
            "coarse_cluster_ctas": info["coarse_cluster_ctas"] if info["coarse_cluster_active"] else 0,
            "true_relative_residual": float(torch.linalg.norm(r) / torch.linalg.norm(pe.rhs)),
            "rel_diff_vs_jacobi": float(torch.linalg.norm(xm - xe) / torch.linalg.norm(xe)),
            "speedup_vs_jacobi": tj / tmg}
        if info["coarse_cluster_active"] and precision == TWO_LEVEL[-1][0]:
            # the same solver with the pipelined coarse kernels (one launch per coarse iteration)
            solver.set_coarse_cluster(False)
            tp = timed(solve_mg, 1, warm=0)
            entry["pipelined_coarse_seconds"] = tp
            entry["pipelined_coarse_iterations"] = solver.getStats().iterationCount
            solver.set_coarse_cluster(True)
        emb["two_level_%s_smoothing" % precision] = entry
        del solver, xm
    out["embedded_sphere_q3_32^3"] = emb
    del Ae, pe, xe

    # adjoint gradient, 3D Q1 64^3
    cells = [64, 64, 64]
    prob = DifferentiablePoisson(space, 3, 1, cells, settings=Statistics(20000, 0.0, 1e-10))
    kappa = torch.as_tensor(kappa_field(1, cells)).cuda()
    kappa_t = torch.as_tensor(kappa_field(2, cells)).cuda()
    b = torch.as_tensor(random_uniform(0, prob.n)).cuda()
    u_t = prob(kappa_t, b).detach()
    k_req = kappa.clone().requires_grad_(True)

    def forward():
        return 0.5 * torch.sum((prob(k_req, b) - u_t) ** 2)
    tf = timed(forward, 3)
    J = forward()

    def backward():
        k_req.grad = None
        J.backward(retain_graph=True)
    tbk = timed(backward, 3)
    out["adjoint_poisson3d_q1_64^3"] = {
        "forward_seconds": tf, "backward_seconds": tbk, "cells": int(np.prod(cells)), "dofs": prob.n,
        "forward_iterations": prob.forward_stats.iterationCount,
        "adjoint_iterations": prob.adjoint_stats.iterationCount}
    return out


if __name__ == "__main__":
    main()
