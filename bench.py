#!/usr/bin/env python
"""Benchmark: MGCG solves/s of the structured SIMP elasticity solve, one JSON line.

Headline workload (default ``cantilever_256x128x128``): 256x128x128 H8 cantilever,
12,830,211 DOF, E0=1, Emin=1e-9, nu=0.3, penal=3, densities seeded uniform(0.001,1)
Gaussian-smoothed (sigma=2); MultiGrid-preconditioned CG with 5 coarse levels, 2 pre/post
damped-Jacobi sweeps (omega=0.6, reference adaptive schedule), relative residual 1e-8.
The timed form (default ``mixed_learned``) is the mixed-precision solver (FP32 V-cycle
inside the FP64 CG) with the learned coarse space: the network's predicted field (64x32x32
pooled cell grid) spans a deflation space that gives the initial guess (the energy-optimal
combination of its three components) and the coarse-grid correction of every PCG
iteration; its inference is inside the timed solve.  One step = one complete solve
including the hierarchy setup (the densities change every SIMP iteration, so the hierarchy
is rebuilt every solve, as in the reference).  The plain FP64 MGCG and the other forms are
timed beside it (``forms``), with their compliance and displacement errors against FP64,
and the SIMP loops of the 192x96x96 (BF16 densities, 20 iterations) and 256x128x128
(learned coarse space, 30 iterations) configurations report per-iteration errors against
FP64.

Arms
  default          this library on N GPUs (one process per GPU, replicas: a solve does not
                   shard; ranks run independent solves, ``scaling: weak``).
  --impl reference the reference algorithm on the host CPU: the C/OpenMP restatement of the
                   reference MultiGrid solve (FP64, all host threads), same workload and
                   metric, timed on a bounded sample (hierarchy setup + K PCG iterations,
                   extrapolated to the iteration count of the complete solve).

Timing: W untimed warm-up solves, then K solves, each bracketed by CUDA events on the
solve stream with a 512 MB L2 flush before each (the inputs exceed L2 as well); max over
ranks.  ``e2e`` repeats the measurement through the public API (FiniteElement.solve) with
the loads and densities in pinned host memory (host->device copies and the device->host
copy of U inside the timed region).
"""
from __future__ import annotations

import argparse
import csv
import ctypes
import io
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

WORKLOADS = {
    "cantilever_96x48x48": dict(nel=(96, 48, 48), n_level=4),
    "cantilever_192x96x96": dict(nel=(192, 96, 96), n_level=5),
    "cantilever_256x128x128": dict(nel=(256, 128, 128), n_level=5),
}
# form -> (MultiGrid precision, learned initial guess)
# form -> (V-cycle precision, learned coarse space, fixed Jacobi weight).  "fp64" is the
# reference's MGCG (its residual-driven Jacobi weight); "mixed_learned" is this library's
# fastest form; the others separate the contributions.
FIXED_OMEGA = 0.5
FORMS = {"fp64": ("fp64", False, False), "fp64_fixed": ("fp64", False, True), "mixed": ("mixed", False, False),
         "mixed_bf16": ("mixed_bf16", False, False), "mixed_learned_ref": ("mixed", True, False),
         "mixed_learned": ("mixed", True, True)}
METRIC = "MGCG solves/sec and matvec HBM GB/s, mixed+learned vs plain FP64 at rel-res 1e-8"
KNOWN = os.path.join(ROOT, "tests", "golden", "known_answers.json")


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def full_iterations(workload):
    """PCG iterations of the complete FP64 solve of the workload (the oracle's complete
    solve, recorded in the known answers), or None."""
    try:
        return int(json.load(open(KNOWN))[workload + "_oracle"]["pcg_iterations"])
    except (OSError, KeyError, ValueError):
        return None


# -----------------------------------------------------------------------------------------
# clocks sampler
# -----------------------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None
        self.skip = 0

    def mark(self):
        """Start of the timed region: samples written before now are not reported."""
        try:
            self.skip = len(open(self.f.name).read().splitlines())
        except OSError:
            self.skip = 0

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = list(csv.reader(io.StringIO(open(self.f.name).read())))[self.skip:]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# -----------------------------------------------------------------------------------------
# our arm
# -----------------------------------------------------------------------------------------
_NET = None


def coarse_space_for(learned):
    global _NET
    if not learned:
        return None
    from pyfantom_b200 import learned as L
    if _NET is None:
        _NET = L.WarmStartNet.load()
    return L.LearnedCoarseSpace(_NET, pool=4)


def build_problem(nel, n_level, form="fp64", tol=1e-8):
    import torch
    from pyfantom_b200 import workloads
    from pyfantom_b200.CUDA import FiniteElement, MultiGrid, StructuredMesh3D, StructuredStiffnessKernel
    from pyfantom_b200.physics import LinearElasticity
    prec, learned, fixed = FORMS[form]
    wl = workloads.cantilever3d(*nel)
    mesh = StructuredMesh3D(*nel, *nel, physics=LinearElasticity(E=1.0, nu=0.3))
    kern = StructuredStiffnessKernel(mesh)
    sol = MultiGrid(mesh, kern, maxiter=1000, tol=tol, n_smooth=2, omega=0.6, n_level=n_level, precision=prec,
                    coarse_correction=coarse_space_for(learned), fixed_omega=FIXED_OMEGA if fixed else None)
    fe = FiniteElement(mesh, kern, sol)
    fe.add_dirichlet_boundary_condition(node_ids=torch.as_tensor(wl["fixed_nodes"], device="cuda"), rhs=0.0)
    fe.add_point_forces(forces=wl["load_forces"], node_ids=torch.as_tensor(wl["load_nodes"], device="cuda"))
    E = torch.as_tensor(wl["E"], device="cuda")
    return wl, mesh, kern, sol, fe, E


def _flush_buffer():
    import torch
    return torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")


def replica_max(ms, world, device):
    """Max over ranks of one rank's device time: replicas run independent solves and the job
    ends with the slowest rank (no data-path collective; this all-reduce is timing only)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, steps, max_ms):
    """Whole-job solves/s: every rank solved `steps` times within the slowest rank's time."""
    return round(world * steps / (max_ms / 1e3), 4)


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from pyfantom_b200 import _lib

    torch.cuda.set_device(local_rank)
    lib = _lib.load()
    spec = WORKLOADS[args.workload]
    nel, nl = spec["nel"], spec["n_level"]
    wl, mesh, kern, sol, fe, E = build_problem(nel, nl, args.form)
    D, Ne = kern.shape[0], int(np.prod(nel))
    flush = _flush_buffer()
    stream = torch.cuda.current_stream()

    def solve_once():
        kern.set_rho(E)
        return sol.solve(fe.rhs, use_last=False)

    # the clock sampler runs from the warm-up on; only its samples of the timed region count
    clocks = Clocks()
    if rank == 0:
        clocks.start()
    t_w = time.time()
    for i in range(args.warmup):
        U, res = solve_once()
    torch.cuda.synchronize()
    while time.time() - t_w < 1.0:  # let the clocks settle: untimed solves for at least 1 s
        U, res = solve_once()
        torch.cuda.synchronize()
    iters = sol.last_info["iterations"]
    status = sol.last_info["status"]
    compliance = float(torch.dot(fe.rhs, U))

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    if rank == 0:
        clocks.mark()
    launches0 = lib.pf_launch_count()
    total_ms = 0.0
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        U, res = solve_once()
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    launches = lib.pf_launch_count() - launches0
    if world > 1:
        dist.barrier()
    max_ms = replica_max(total_ms, world, "cuda")
    clk = clocks.stop() if rank == 0 else None

    # ---- end to end through the public API with host buffers --------------------------
    rhs_h = torch.from_numpy(fe.rhs.cpu().numpy()).pin_memory()
    E_h = torch.from_numpy(wl["E"]).pin_memory()
    U_h = torch.empty(D, dtype=torch.float64).pin_memory()
    E_dev = torch.empty(Ne, dtype=torch.float64, device="cuda")
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fe.rhs.copy_(rhs_h, non_blocking=True)
        E_dev.copy_(E_h, non_blocking=True)
        fe.solver.last_x0 = None  # every timed solve starts cold (x0 = 0, or the learned space's guess)
        U2, _ = fe.solve(E_dev)
        U_h.copy_(U2, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
    e2e_max = replica_max(e2e_ms, world, "cuda")

    # ---- roofline of the dominant kernel: the fine-level matvec of the V-cycle (FP32 in
    # the mixed forms, FP64 in the FP64 form), every launch of one solve timed live with
    # CUDA events on the solve's stream --------------------------------------------------
    fp32 = FORMS[args.form][0] != "fp64"
    lib.pf_mg_set_profiling(sol._mg, 20000)
    lib.pf_mg_profile_select(sol._mg, 2 if fp32 else 1)
    flush.fill_(1.0)
    solve_once()
    ms, n_l, byts = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_double()
    lib.pf_mg_profile(sol._mg, ctypes.byref(ms), ctypes.byref(n_l), ctypes.byref(byts))
    lib.pf_mg_set_profiling(sol._mg, 0)
    avg_us = ms.value / max(n_l.value, 1) * 1e3
    achieved = byts.value / max(ms.value, 1e-12) / 1e6  # GB/s
    hbm, peak_kind = peaks()
    kname = "k_matvec_h8r<float>" if fp32 else "k_matvec_h8r<double>"
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
            "frac": round(achieved / hbm, 4), "traffic": None, "peak_kind": peak_kind,
            "kernel": f"{kname} (fine-level stiffness matvec of the V-cycle, register x-march, fused epilogues)",
            "launches_in_solve": int(n_l.value), "avg_launch_us": round(avg_us, 2),
            "algorithmic_bytes_per_launch": round(byts.value / max(n_l.value, 1))}
    prof_path = os.path.join(ROOT, "profiles", "matvec_h8_traffic.json")
    if os.path.exists(prof_path):
        tr = json.load(open(prof_path)).get(f"{args.workload}/{args.form}")
        if tr:
            roof["traffic"] = tr.get("dram_bytes_per_launch")
            roof["traffic_source"] = tr.get("source")

    dtype = {"fp64": "f64", "mixed": "f64 outer / f32 V-cycle", "mixed_bf16": "f64 outer / f32 V-cycle / bf16 E"}[
        FORMS[args.form][0]]
    result = {
        "metric": METRIC, "value": replica_throughput(world, args.steps, max_ms), "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(max_ms / args.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": dtype,
        "data": "synthetic (seeded smoothed-random densities, cantilever loads)",
        "config": {"workload": args.workload, "form": args.form, "nel": list(nel), "dof": D, "n_level": nl,
                   "n_smooth": 2, "omega": 0.6, "tol": 1e-8,
                   "jacobi_weight": (f"fixed {FIXED_OMEGA} (the same preconditioner every iteration)"
                                     if FORMS[args.form][2] else "the reference's residual-driven schedule"),
                   "start": ("learned coarse space (network on nel/4 cells): deflated start and coarse-grid correction"
                             if FORMS[args.form][1] else "cold (x0 = 0)"),
                   "l2": "512 MB L2 flush before every timed solve; inputs exceed L2",
                   "parallelism": f"replicas x{world}",
                   "warmup_extra": "untimed solves until 1 s has passed, so the clocks settle"},
        "pcg_iterations": iters, "status": status, "compliance": compliance,
        "e2e": {"value": replica_throughput(world, args.steps, e2e_max), "unit": "solves/s",
                "h2d_bytes_per_step": int(8 * (D + Ne)), "d2h_bytes_per_step": int(8 * D)},
        "gpu_launches": int(launches),
        "roofline": roof,
    }
    if rank == 0:
        result["clocks"] = clk
    del wl, mesh, kern, sol, fe, E, U, flush
    torch.cuda.empty_cache()
    return result


def time_form(nel, nl, form, reps=3, ref=None):
    """Median of `reps` cold solves (after one warm-up) of one form, L2 flushed before each,
    with the true residual and (given the FP64 reference (compliance, U)) the errors."""
    import torch
    flush = _flush_buffer()
    wl, mesh, kern, sol, fe, E = build_problem(nel, nl, form)
    kern.set_rho(E)
    U, _ = sol.solve(fe.rhs, use_last=False)
    t = []
    for _ in range(reps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        kern.set_rho(E)
        U, _ = sol.solve(fe.rhs, use_last=False)
        e1.record()
        e1.synchronize()
        t.append(e0.elapsed_time(e1))
    r = fe.rhs - kern.dot(U)
    c = float(torch.dot(fe.rhs, U))
    ms = statistics.median(t)
    out = {"solves_per_s": round(1e3 / ms, 3), "ms": round(ms, 2), "pcg_iterations": sol.last_info["iterations"],
           "setup_ms": round(sol.last_info["setup_ms"], 2),
           "true_rel_residual": float(torch.linalg.norm(r) / torch.linalg.norm(fe.rhs)), "compliance": c}
    if ref is not None:
        out["rel_compliance_err_vs_fp64"] = abs(c - ref[0]) / abs(ref[0])
        out["rel_displacement_err_vs_fp64"] = float(torch.linalg.norm(U - ref[1]) / torch.linalg.norm(ref[1]))
    keep = (c, U.clone())
    del wl, mesh, kern, sol, fe, E, U, r, flush
    torch.cuda.empty_cache()
    return out, keep


def forms_at(workload, names=("fp64", "fp64_fixed", "mixed", "mixed_bf16", "mixed_learned_ref", "mixed_learned")):
    """The solver forms at one workload; speed-ups and errors against the plain FP64 MGCG."""
    spec = WORKLOADS[workload]
    out, ref = {}, None
    for name in names:
        o, keep = time_form(spec["nel"], spec["n_level"], name, ref=ref)
        if ref is None:
            ref = keep
        else:
            o["speedup_vs_fp64"] = round(out["fp64"]["ms"] / o["ms"], 3)
        out[name] = o
    for name, o in out.items():
        prec, learned, fixed = FORMS[name]
        o["form"] = (f"{prec} V-cycle" + (", learned coarse space (network on nel/4 cells)" if learned else "") +
                     (f", fixed Jacobi weight {FIXED_OMEGA}" if fixed else ", reference Jacobi-weight schedule"))
    return out


def matvec_probe(workload, reps=8, warm=2, fp32_variant=0):
    """The fine matvec alone (FP64, FP32, FP32 with BF16 element scales), L2 flushed before
    every launch: microseconds, algorithmic bytes and GB/s, DOF-matvecs/s."""
    import torch
    from pyfantom_b200 import _lib, workloads
    from pyfantom_b200.CUDA import StructuredMesh3D, StructuredStiffnessKernel
    from pyfantom_b200.physics import LinearElasticity
    nel = WORKLOADS[workload]["nel"]
    w = workloads.cantilever3d(*nel)
    mesh = StructuredMesh3D(*nel, *nel, physics=LinearElasticity(E=1.0, nu=0.3))
    kern = StructuredStiffnessKernel(mesh)
    _lib.check(_lib.load().pf_op_set_variant(kern._op, int(fp32_variant)))
    kern.add_constraints(torch.as_tensor(w["fixed_dofs"], device="cuda"))
    D, Ne, Nn = kern.shape[0], int(np.prod(nel)), kern.n_nodes
    flush = _flush_buffer()
    lib = _lib.load()
    hbm, kind = peaks()
    out = {}
    E64 = torch.as_tensor(w["E"], device="cuda")
    for prec in ("fp64", "fp32", "fp32_bf16E"):
        dt = torch.float64 if prec == "fp64" else torch.float32
        if prec == "fp32_bf16E":
            Et, esz = E64.to(torch.bfloat16), 2
            f = lib.pf_matvec_f32_bf16
        else:
            Et, esz = E64.to(dt), (8 if prec == "fp64" else 4)
            f = lib.pf_matvec_f64 if prec == "fp64" else lib.pf_matvec_f32
        u = torch.randn(D, dtype=dt, device="cuda")
        y = torch.empty_like(u)
        ts = []
        for i in range(warm + reps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _lib.check(f(kern._op, _lib.ptr(Et), _lib.ptr(u), _lib.ptr(kern.node_mask), _lib.ptr(y), _lib.stream()))
            e1.record()
            e1.synchronize()
            if i >= warm:
                ts.append(e0.elapsed_time(e1))
        ms = statistics.median(ts)
        sz = 8 if prec == "fp64" else 4
        byts = 2 * D * sz + Ne * esz + Nn
        out[prec] = {"us": round(ms * 1e3, 1), "algorithmic_bytes": byts, "GB_per_s": round(byts / ms / 1e6, 1),
                     "frac_of_hbm": round(byts / ms / 1e6 / hbm, 4), "dof_matvecs_per_s": round(D / ms * 1e3, 1)}
    out["peak"] = {"GB_per_s": hbm, "kind": kind}
    del kern, mesh, u, y, Et, flush
    torch.cuda.empty_cache()
    return out


def simp_loop(workload, form, n_iter, vf=0.3, r_min=2.0, move=0.2):
    """SIMP minimum compliance with OC on the workload, the displacement solves by `form`
    (the learned form starts from the previous solution corrected inside the network's
    deflation space, and keeps that space as its coarse-grid correction).  Each iteration's
    stiffness is also solved by the plain FP64 MGCG (warm-started from its own previous
    solution, same tolerance) to give the relative
    compliance and displacement errors of the form; the time per SIMP iteration (filter,
    penalisation, solve, sensitivity, adjoint filter, OC update) excludes those checks.  The
    check solver keeps its Jacobi weight fixed: on the 0/1 designs of later iterations the
    reference's schedule can stall short of the tolerance, and the check must converge."""
    import torch
    from pyfantom_b200.CUDA import MinimumCompliance, MultiGrid, OC, StructuredFilter3D
    spec = WORKLOADS[workload]
    nel, nl = spec["nel"], spec["n_level"]
    wl, mesh, kern, sol, fe, E = build_problem(nel, nl, form)
    ref = MultiGrid(mesh, kern, maxiter=2000, tol=1e-8, n_smooth=2, omega=0.6, n_level=nl, precision="fp64",
                    fixed_omega=0.5)
    prob = MinimumCompliance(fe, StructuredFilter3D(mesh, r_min), E_mul=[1.0], void=1e-9, penalty=3.0,
                             volume_fraction=[vf], heavyside=False)
    oc = OC(prob, move=move)
    x0 = torch.as_tensor(wl["x"], device="cuda")
    prob.set_desvars(x0)
    oc.last_desvars = x0.clone()
    oc.last_f = prob.f()
    rows, t_iter, its = [], [], []

    def check(row):
        U = prob._U
        Ur, _ = ref.solve(fe.rhs, use_last=True)
        cr = float(torch.dot(fe.rhs, Ur))
        c = float(prob.f())
        row.update(compliance=c, rel_compliance_err=abs(c - cr) / abs(cr),
                   rel_displacement_err=float(torch.linalg.norm(U - Ur) / torch.linalg.norm(Ur)),
                   pcg_iterations=sol.last_info["iterations"], fp64_pcg_iterations=ref.last_info["iterations"],
                   status=sol.last_info["status"], fp64_status=ref.last_info["status"])
        rows.append(row)

    check({"iteration": 0})
    for it in range(n_iter):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        oc.iter()
        e1.record()
        e1.synchronize()
        t_iter.append(e0.elapsed_time(e1))
        its.append(sol.last_info["iterations"])
        check({"iteration": it + 1, "ms": round(t_iter[-1], 2)})
    ok = [r for r in rows if r["fp64_status"] == "PF_OK"] or rows
    out = {"workload": workload, "form": form, "iterations": n_iter, "volfrac": vf, "r_min": r_min,
           "ms_per_simp_iteration": round(statistics.mean(t_iter), 2),
           "mean_pcg_iterations": round(statistics.mean(its), 2),
           "max_rel_compliance_err": max(r["rel_compliance_err"] for r in ok),
           "max_rel_displacement_err": max(r["rel_displacement_err"] for r in ok),
           "errors_over": "iterations where the FP64 check solve converged",
           "iterations_fp64_not_converged": [r["iteration"] for r in rows if r["fp64_status"] != "PF_OK"],
           "iterations_form_not_converged": [r["iteration"] for r in rows if r["status"] != "PF_OK"],
           "per_iteration": [{k: (float(f"{v:.4g}") if isinstance(v, float) else v) for k, v in r.items()}
                             for r in rows]}
    del wl, mesh, kern, sol, fe, E, ref, prob, oc
    torch.cuda.empty_cache()
    return out


def extras(args):
    """Secondary measurements on one GPU: the forms at the workload, the fine matvec alone,
    the forms at 192x96x96, and the two SIMP loops."""
    out = {"forms": forms_at(args.workload), "matvec": matvec_probe(args.workload)}
    if args.workload != "cantilever_192x96x96":
        out["forms_192x96x96"] = forms_at("cantilever_192x96x96", ("fp64", "mixed", "mixed_bf16"))
    if not args.no_simp:
        out["simp_192x96x96_mixed_bf16"] = simp_loop("cantilever_192x96x96", "mixed_bf16", 20)
        out["simp_256x128x128_mixed_learned"] = simp_loop("cantilever_256x128x128", "mixed_learned", 30)
    return out


def probe_matvec(args):
    """Time the fine-level matvec alone (for ncu captures)."""
    return {"probe": "matvec", "workload": args.workload, "fp32_variant": args.fp32_variant,
            **matvec_probe(args.workload, reps=args.steps, warm=args.warmup, fp32_variant=args.fp32_variant)}


def probe_level1(args):
    """The level-1 operator of the V-cycle alone in the form's precision, element-level and
    assembled stencil (STORE epilogue, L2 flushed before every launch): microseconds and
    algorithmic bytes (u and y once, the 8 Ehat per coarse element or the 126-value half
    stencil per coarse node, one flag byte per coarse node)."""
    import torch
    from pyfantom_b200.CUDA import MultiGrid
    spec = WORKLOADS[args.workload]
    nel, nl = spec["nel"], spec["n_level"]
    prec = FORMS[args.form][0]
    wl, mesh, kern, sol, fe, E = build_problem(nel, nl, "fp64")
    kern.set_rho(E)
    flush = _flush_buffer()
    dt, sz = (torch.float64, 8) if prec == "fp64" else (torch.float32, 4)
    cnel = [n // 2 for n in nel]
    Nn1, Ne1 = int(np.prod([n + 1 for n in cnel])), int(np.prod(cnel))
    hbm, kind = peaks()
    out = {"probe": "level1", "workload": args.workload, "precision": prec}
    for op in ("element", "stencil"):
        s = MultiGrid(mesh, kern, maxiter=10, tol=1e-8, n_smooth=2, omega=0.6, n_level=nl, precision=prec,
                      coarse_op=op)
        s.setup()
        u = torch.randn(3 * Nn1, dtype=dt, device="cuda")
        ts = []
        for i in range(args.warmup + args.steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            s.level_matvec(1, u)
            e1.record()
            e1.synchronize()
            if i >= args.warmup:
                ts.append(e0.elapsed_time(e1))
        ms = statistics.median(ts)
        byts = 2 * 3 * Nn1 * sz + (8 * Ne1 * sz + Nn1 if op == "element" else 126 * Nn1 * sz)
        out[op] = {"us": round(ms * 1e3, 1), "algorithmic_bytes": byts, "GB_per_s": round(byts / ms / 1e6, 1),
                   "frac_of_hbm": round(byts / ms / 1e6 / hbm, 4), "dirty": s.level_info()[1]}
        del s
    out["peak"] = {"GB_per_s": hbm, "kind": kind}
    return out


def probe_solve(args):
    """One solve of the workload after two warm-up solves, bracketed by
    cudaProfilerStart/Stop (for `ncu --profile-from-start off`: the launch list of exactly
    one solve, hierarchy setup included)."""
    import torch
    spec = WORKLOADS[args.workload]
    wl, mesh, kern, sol, fe, E = build_problem(spec["nel"], spec["n_level"], args.form)
    kern.set_rho(E)
    for _ in range(2):
        sol.solve(fe.rhs, use_last=False)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    U, res = sol.solve(fe.rhs, use_last=False)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    return {"probe": "solve", "workload": args.workload, "form": args.form,
            "iterations": sol.last_info["iterations"], "status": sol.last_info["status"],
            "solve_ms": sol.last_info["solve_ms"], "setup_ms": sol.last_info["setup_ms"]}


# -----------------------------------------------------------------------------------------
# reference arm and CPU baseline: the oracle (C/OpenMP restatement of the reference solve)
# -----------------------------------------------------------------------------------------
def cpu_sample(workload, k_iters):
    """The oracle's FP64 MGCG on the workload: hierarchy setup plus k PCG iterations, timed
    separately; the complete solve's time is extrapolated to its iteration count."""
    from oracle import oracle as O
    from pyfantom_b200 import workloads
    from pyfantom_b200.geom import _unit_element
    from pyfantom_b200.physics import LinearElasticity
    spec = WORKLOADS[workload]
    wl = workloads.cantilever3d(*spec["nel"])
    K0 = LinearElasticity(E=1.0, nu=0.3).K(_unit_element((1.0, 1.0, 1.0)))
    x, it, res, st, setup_s, iter_s = O.mgcg_solve_timed(spec["nel"], K0, wl["E"], wl["fixed_dofs"], wl["rhs"],
                                                         n_level=spec["n_level"], n_smooth=2, omega=0.6, tol=1e-8,
                                                         maxiter=k_iters)
    n_full = full_iterations(workload)
    complete = st == 0  # converged inside the sample: a complete solve
    if complete or n_full is None:
        n_full = it
    solve_s = setup_s + iter_s / max(it, 1) * n_full
    return dict(solve_s=solve_s, setup_s=setup_s, iter_s_each=iter_s / max(it, 1), iters_sampled=it,
                iters_full=n_full, complete=complete, threads=O.num_threads(),
                compliance=float(wl["rhs"] @ x) if complete else None)


def run_reference(args):
    spec = WORKLOADS[args.workload]
    # one sample: the setup and K PCG iterations (compiled C needs no warm-up); the complete
    # solve's time is extrapolated from it
    s = cpu_sample(args.workload, args.steps)
    v = 1.0 / s["solve_s"]
    sample = (f"hierarchy setup + {s['iters_sampled']} PCG iterations of the FP64 MGCG solve "
              f"({s['setup_s']:.2f} s + {s['iter_s_each']:.3f} s per iteration), extrapolated to the "
              f"{s['iters_full']} iterations of the complete solve")
    if s["complete"]:
        sample = f"one complete solve ({s['iters_full']} PCG iterations)"
    return {
        "metric": METRIC, "value": round(v, 6), "unit": "solves/s", "n_gpus": 0, "steps": args.steps,
        "warmup": 0, "ms_per_step": round(s["solve_s"] * 1e3, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": args.workload, "form": "fp64", "nel": list(spec["nel"]), "n_level": spec["n_level"],
                   "n_smooth": 2, "omega": 0.6, "tol": 1e-8,
                   "jacobi_weight": (f"fixed {FIXED_OMEGA} (the same preconditioner every iteration)"
                                     if FORMS[args.form][2] else "the reference's residual-driven schedule"), "start": "cold (x0 = 0)"},
        "pcg_iterations": s["iters_full"],
        "cpu_baseline": {"value": round(v, 6), "unit": "solves/s", "cores": s["threads"], "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(v, 6), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    global FIXED_OMEGA
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cantilever_256x128x128", choices=sorted(WORKLOADS))
    ap.add_argument("--form", default="mixed_learned", choices=sorted(FORMS))
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-simp", action="store_true", help="skip the SIMP loops in the extras")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-iters", type=int, default=3, help="PCG iterations of the CPU-baseline sample")
    ap.add_argument("--fp32-variant", type=int, default=0, choices=[0, 1],
                    help="FP32 fine matvec of cube elements in the matvec probe (pf_op_set_variant)")
    ap.add_argument("--probe", choices=["matvec", "level1", "solve"], default=None,
                    help="only time the fine matvec, the level-1 operator, or bracket one solve (for ncu captures)")
    ap.add_argument("--fixed-omega", type=float, default=FIXED_OMEGA,
                    help="Jacobi weight of the forms that keep it fixed (fp64_fixed, mixed_learned)")
    args = ap.parse_args()
    FIXED_OMEGA = args.fixed_omega
    args.warmup = max(args.warmup, 3) if args.impl == "ours" and not args.probe else args.warmup
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
            print(json.dumps(run_reference(args)), flush=True)
        return

    import torch
    if args.probe == "matvec":
        print(json.dumps(probe_matvec(args)), flush=True)
        return
    if args.probe == "solve":
        print(json.dumps(probe_solve(args)), flush=True)
        return
    if args.probe == "level1":
        print(json.dumps(probe_level1(args)), flush=True)
        return
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    result = run_ours(args, rank, world, local_rank)
    if rank == 0 and world == 1 and not args.no_extras:
        ex = extras(args)
        result["forms"] = ex
        f = ex["forms"]
        if "fp64" in f and args.form in f:
            result["fp64_solves_per_s"] = f["fp64"]["solves_per_s"]
            result["speedup_vs_fp64"] = round(f["fp64"]["ms"] / f[args.form]["ms"], 3)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
        s = cpu_sample(args.workload, args.cpu_iters)
        result["cpu_baseline"] = {
            "value": round(1.0 / s["solve_s"], 6), "unit": "solves/s", "cores": s["threads"], "kind": "port",
            "sample": (f"C/OpenMP oracle FP64 MGCG: hierarchy setup + {s['iters_sampled']} PCG iterations "
                       f"({s['setup_s']:.2f} s + {s['iter_s_each']:.3f} s per iteration), extrapolated to the "
                       f"{s['iters_full']} iterations of the complete solve")}
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


if __name__ == "__main__":
    main()
