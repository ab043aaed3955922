"""Benchmark of the B200 assembly + Jacobi-PCG path.

Default workload: 3D vector-P1 linear elasticity on the box [0,4]x[0,1]x[0,1],
128x32x32 hexahedra split into 6 tetrahedra each (786,432 tets, 421,443 dofs),
E = 210e9, nu = 0.3, clamped at x = 0, body force (0, 0, -7.8e4); solved to
1e-8 relative residual with mixed-precision refined PCG (FP32 SpMV/axpy inside
FP64 residual replacement), next to the plain FP64 PCG on the same card.

One step = assemble the stiffness (FP64 + FP32 values) + body force +
Dirichlet elimination + mixed PCG to 1e-8, inputs resident in HBM. The
metric is dofs / step time (DOF/s). Inputs are synthetic (generated meshes).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]
                    [--config c2|c2p] [--no-cpu-baseline] [--no-extra]

After the headline measurement, rank 0 of a 1-GPU run also measures the
other configurations (2D Poisson 64^2, elasticity at 1.57M dofs with stress
recovery, P2 Poisson with random coefficient, adjoint sensitivities, the
256-problem batch, the C2 mass matrix, block-Jacobi PCG on C2, a 1M-dof
transient heat run and a cantilever's vibration modes) and reports them
under "workloads".

--impl reference times the CPU restatement of the reference path (the
reference itself is Rust and cannot be built here) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "fenics-rs_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "DOF/s to 1e-8 rel. residual: mixed-prec vs FP64 CG on 1 B200; assembly GB/s"

CONFIGS = {
    # name: (description, builder kwargs)
    "c2": dict(workload="3D vector-P1 elasticity, box [0,4]x[0,1]x[0,1], 128x32x32 hexes x 6 tets "
                        "(786,432 tets, 421,443 dofs), E=210e9, nu=0.3, clamped x=0, body force (0,0,-7.8e4), "
                        "mixed-precision refined PCG to 1e-8 vs FP64 PCG",
               L=4.0, W=1.0, H=1.0, nx=128, ny=32, nz=32),
    "c2p": dict(workload="3D vector-P1 elasticity, box [0,4]x[0,1]x[0,1], 200x50x50 hexes x 6 tets "
                         "(3,000,000 tets, 1,568,403 dofs), E=210e9, nu=0.3, clamped x=0, body force (0,0,-7.8e4), "
                         "mixed-precision refined PCG to 1e-8 vs FP64 PCG",
                L=4.0, W=1.0, H=1.0, nx=200, ny=50, nz=50),
}


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _profile_traffic(name: str):
    """DRAM bytes per launch recorded by an ncu capture summary under profiles/."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU (oracle) timing — the reference arm and the cpu_baseline leg
# ---------------------------------------------------------------------------

def config_dict(cfg):
    """The workload description both arms print (identical dicts)."""
    nx, ny, nz = cfg["nx"], cfg["ny"], cfg["nz"]
    return {"workload": cfg["workload"], "ndofs": 3 * (nx + 1) * (ny + 1) * (nz + 1), "cells": 6 * nx * ny * nz,
            "tol": 1e-8, "l2": "GPU: 256 MiB written between steps (L2 is 126 MB); CPU: the 113M-triplet assembly "
                              "and the 218 MB matrix exceed every host cache"}


class CpuPath:
    """The reference path on the host, through the CPU restatement under
    oracle/: OpenMP cell loop (rayon par_iter in elasticity.rs:88) with the
    faer-style triplet -> CSC build, body force, vector Dirichlet elimination,
    then Jacobi-PCG to 1e-8 with cg.rs's recurrence and stopping rules."""

    def __init__(self, cfg, threads=None):
        import oracle as O
        self.O = O
        self.cfg = cfg
        self.om = O.box_beam(cfg["L"], cfg["W"], cfg["H"], cfg["nx"], cfg["ny"], cfg["nz"])
        self.dofs = O.clamp_dofs(self.om)
        self.threads = threads or (os.cpu_count() or 1)
        self.n = 3 * self.om.nv

    def setup(self):
        O = self.O
        K = O.assemble_elasticity_3d(self.om, 210e9, 0.3, threads=self.threads)
        f = O.body_force_3d(self.om, [0.0, 0.0, -7.8e4])
        return O.apply_dirichlet_bc(K, f, self.dofs, np.zeros(len(self.dofs)))

    def full_step(self):
        """One complete step: setup + PCG to 1e-8 on all host threads (the
        CG's SpMV, vector loops and dot products in parallel; cg.rs itself is
        sequential). Nothing is extrapolated."""
        t0 = time.perf_counter()
        Kb, fb = self.setup()
        t1 = time.perf_counter()
        x, it, res = self.O.solve_cg_mt(Kb, fb, None, 1e-8, 1000000, self.threads)
        t2 = time.perf_counter()
        return {"s": t2 - t0, "setup_s": t1 - t0, "cg_s": t2 - t1, "iterations": it,
                "rel_residual": res / float(np.linalg.norm(fb)), "system": (Kb, fb), "x": x}

    def sequential_cg_sample(self, Kb, fb, iters_full: int, sample_iters: int = 40):
        """cg.rs as written (one thread, column-scatter SpMV): a sample of
        `sample_iters` iterations scaled to the measured iteration count."""
        t0 = time.perf_counter()
        self.O.cg_fixed_iters(Kb, fb, sample_iters)
        per_it = (time.perf_counter() - t0) / sample_iters
        return per_it, per_it * iters_full


def cpu_baseline_leg(cfg, x_ref=None):
    """The GPU arm's cpu_baseline: one complete, unextrapolated host step of
    the same workload (about 10-20 s on 16 threads), the faithful sequential
    cg.rs timed on a sample, and the FP64 reference solution's residual on
    the oracle's own matrix."""
    cp = CpuPath(cfg)
    r = cp.full_step()
    Kb, fb = r.pop("system")
    r.pop("x")
    per_it, seq_cg = cp.sequential_cg_sample(Kb, fb, r["iterations"])
    out = {
        "value": cp.n / r["s"], "unit": "DOF/s", "cores": cp.threads, "kind": "port",
        "sample": f"one complete step of the same workload, not extrapolated: oracle assembly ({cp.threads} "
                  f"threads for the cell loop, sequential faer-style triplet build) + body force + Dirichlet "
                  f"{r['setup_s']:.2f} s, then Jacobi-PCG to 1e-8 with the SpMV, vector loops and dot products "
                  f"on {cp.threads} threads: {r['iterations']} iterations, {r['cg_s']:.2f} s",
        "seconds": r["s"], "iterations": r["iterations"],
        "sequential_cg": {
            "value": cp.n / (r["setup_s"] + seq_cg), "unit": "DOF/s", "cores": 1,
            "sample": f"cg.rs as written (sequential column-scatter SpMV): 40 iterations timed "
                      f"({per_it * 1e3:.1f} ms each), scaled to the {r['iterations']} iterations the full step "
                      f"took, plus the same setup"},
    }
    if x_ref is not None:
        out["fp64_reference_rel_residual_on_oracle_matrix"] = float(
            np.linalg.norm(fb - cp.O.spmv(Kb, x_ref)) / np.linalg.norm(fb))
    return out


# ---------------------------------------------------------------------------
# GPU run
# ---------------------------------------------------------------------------

def run_cuda(args, cfg):
    import torch
    import fenics_cuda as fcu

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = world > 1
    if dist:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = local if dist else 0
    torch.cuda.set_device(dev)
    ctx = fcu.Context(dev)
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{dev}")

    mesh = fcu.box_beam(cfg["L"], cfg["W"], cfg["H"], cfg["nx"], cfg["ny"], cfg["nz"])
    nv, nc = mesh.nv, mesh.nc
    n = 3 * nv
    clamp_v = np.nonzero(mesh.coords[:, 0] < 1e-6)[0]
    dofs = (3 * clamp_v[:, None] + np.arange(3)).ravel().astype(np.int64)
    fbody = np.array([0.0, 0.0, -7.8e4])

    # setup (untimed): mesh upload, pattern, matrix storage, device inputs
    t_setup0 = time.perf_counter()
    V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1_VEC3)
    M = fcu.Matrix(ctx, V)
    t_setup = time.perf_counter() - t_setup0
    dofs_d = torch.from_numpy(dofs).to(f"cuda:{dev}")
    vals_d = torch.zeros(len(dofs), dtype=torch.float64, device=f"cuda:{dev}")
    b_d = torch.empty(n, dtype=torch.float64, device=f"cuda:{dev}")
    x_d = torch.empty(n, dtype=torch.float64, device=f"cuda:{dev}")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{dev}")  # 256 MiB > L2
    torch.cuda.synchronize()  # the inputs above were written on torch's stream, the library runs on its own

    def step(precision):
        M.assemble_elasticity(210e9, 0.3)
        V.body_force(fbody, out=b_d)
        M.apply_dirichlet(b_d, dofs_d, vals_d)
        _, info = M.pcg(b_d, x=x_d, tol=1e-8, max_iter=100000, precision=precision)
        return info

    def timed_steps(k, precision):
        times, infos = [], []
        for _ in range(k):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            infos.append(step(precision))
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        return times, infos

    # warm-up (also captures the CUDA graphs)
    for _ in range(args.warmup):
        step(fcu.FCU_MIXED)
        step(fcu.FCU_FP64)

    if dist:
        tdist.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.kernel_launches
    with ClockSampler(dev) as clk:
        t_mixed, info_mixed = timed_steps(args.steps, fcu.FCU_MIXED)
    torch.cuda.synchronize()
    launches = ctx.kernel_launches - launches0
    if dist:
        tdist.barrier()
    t_fp64, info_fp64 = timed_steps(max(1, args.steps), fcu.FCU_FP64)

    ctx.synchronize()
    x_fp64 = x_d.cpu().numpy()
    # the mixed step again, so its solution can be kept too (untimed)
    step(fcu.FCU_MIXED)
    ctx.synchronize()
    x_mixed = x_d.cpu().numpy()

    ms_mixed = sum(t_mixed) / len(t_mixed)
    ms_fp64 = sum(t_fp64) / len(t_fp64)
    if dist:
        tt = torch.tensor([ms_mixed, ms_fp64], device=f"cuda:{dev}")
        tdist.all_reduce(tt, op=tdist.ReduceOp.MAX)
        ms_mixed, ms_fp64 = tt.tolist()

    # error of each mode's solution against a tight FP64 reference solution
    # (PCG to 1e-13 on the same eliminated system; its true residual is
    # measured here with the FP64 SpMV, and in the cpu_baseline leg on the
    # oracle's own matrix)
    # (on b scaled by 2^40, exact: unscaled, p^T A p of this system falls
    # below cg.rs's absolute breakdown bound 1e-30 before a 1e-13 residual;
    # two restarts from the iterate recompute the residual as b - A x, since
    # one pass's recurrence residual drifts from the true one)
    x_ref_d = torch.empty_like(b_d)
    x_tmp_d = torch.empty_like(b_d)
    with torch.cuda.stream(stream):
        b_scaled = b_d * 2.0 ** 40
    _, info_ref = M.pcg(b_scaled, x=x_ref_d, tol=1e-13, max_iter=1000000, precision=fcu.FCU_FP64)
    ref_iters = info_ref.iterations
    for _ in range(2):
        _, info2 = M.pcg(b_scaled, x0=x_ref_d, x=x_tmp_d, tol=1e-13, max_iter=1000000, precision=fcu.FCU_FP64)
        ref_iters += info2.iterations
        x_ref_d, x_tmp_d = x_tmp_d, x_ref_d
    ctx.synchronize()
    x_ref_d /= 2.0 ** 40
    ax = torch.empty_like(b_d)
    M.spmv(x_ref_d, ax)
    ctx.synchronize()
    x_ref = x_ref_d.cpu().numpy()
    ref_res = float(torch.linalg.norm(b_d - ax) / torch.linalg.norm(b_d))
    nref = float(np.linalg.norm(x_ref))
    errors = {
        "reference_solution": f"FP64 PCG to 1e-13 in three passes, each restarted from the last iterate "
                              f"({ref_iters} iterations), true relative residual {ref_res:.2e}",
        "mixed": float(np.linalg.norm(x_mixed - x_ref) / nref),
        "fp64": float(np.linalg.norm(x_fp64 - x_ref) / nref),
        "metric": "relative L2 error ||x - x_ref|| / ||x_ref||",
    }

    # assembly alone: FP64 + FP32 values of the raw pattern, events on the ctx stream
    reps = 10
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        flush.fill_(2.0)
    e0.record(stream)
    for _ in range(reps):
        M.assemble_elasticity(210e9, 0.3)
    e1.record(stream)
    e1.synchronize()
    ms_asm = e0.elapsed_time(e1) / reps
    nnzb = V.nnz // 9
    asm_bytes = nc * (4 * 4 + 4 * 16 + 8) + nv * 3 * 8 + (nnzb * 9) * (8 + 4)
    # re-establish the solved system for the SpMV timing
    step(fcu.FCU_MIXED)

    # dominant kernel: the FP32 3x3-block SpMV of the mixed PCG, timed cold
    # (L2 evicted by a read sweep before each launch, as inside a solve whose
    # operator exceeds L2, and as an ncu capture starts) and warm (back-to-back launches: the 85 MB operator then
    # partly stays in the 126 MB L2, as it does inside the C2 solve)
    spmv_ms, spmv_bytes = M.time_spmv(fcu.FCU_MIXED, reps=20, cold=True)
    spmv_warm_ms, _ = M.time_spmv(fcu.FCU_MIXED, reps=50)
    spmv64_ms, spmv64_bytes = M.time_spmv(fcu.FCU_FP64, reps=20, cold=True)
    spmv64_warm_ms, _ = M.time_spmv(fcu.FCU_FP64, reps=20)
    peak, peak_kind = _peaks()
    traffic = _profile_traffic("spmv_bsr3_fp32_elasticity_c2.txt")
    traffic64 = _profile_traffic("spmv_bsr3_fp64_elasticity_c2.txt")
    # dominant kernel: the mixed solve's persistent loop (the whole iteration:
    # FP32 SpMV, vector update, grid barriers), one launch of exactly 300
    # iterations after an L2 read sweep, as the profiling case pcg_c2 runs it
    pcg_iters = 300
    pcg_ms, pcg_bytes = M.time_pcg(fcu.FCU_MIXED, iterations=pcg_iters, reps=5)
    achieved = pcg_bytes / (pcg_ms * 1e-3) / 1e9
    traffic_pcg = _profile_traffic("pcg_persistent_fp32_elasticity_c2.txt")

    # e2e through the public API from pinned host buffers, every timed step
    e2e_ms = []
    host_coords = torch.from_numpy(mesh.coords).pin_memory()
    host_cells = torch.from_numpy(mesh.cells).pin_memory()
    bc = fcu.VectorDirichletBC([(int(d), 0.0) for d in dofs])
    material = fcu.ElasticMaterial(210e9, 0.3)
    for k in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m_h = fcu.Mesh(host_coords.numpy(), host_cells.numpy())
        sol = fcu.solve_elasticity_3d(m_h, material, fbody, bc, 1e-8, 100000, ctx=ctx, precision=fcu.FCU_MIXED)
        if k >= args.warmup:
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
        m_h.release()
    h2d = mesh.coords.nbytes + mesh.cells.nbytes + len(dofs) * 16 + 24
    d2h = n * 8

    it_m = info_mixed[-1].iterations
    it_f = info_fp64[-1].iterations
    res = {
        "metric": METRIC,
        "value": n * world / (ms_mixed * 1e-3),
        "unit": "DOF/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_mixed,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 SpMV/axpy + f64 residual/dots (mixed); f64 assembly",
        "data": "synthetic (generated box mesh, no dataset)",
        "config": config_dict(cfg),
        "parallelism": "replicas" if world > 1 else "single GPU",
        "fp64": {"value": n * world / (ms_fp64 * 1e-3), "ms_per_step": ms_fp64, "iterations": it_f},
        "mixed": {"iterations": it_m, "residual_replacements": info_mixed[-1].outer_updates,
                  "rel_residual_fp64": info_mixed[-1].rel_residual},
        "speedup_mixed_vs_fp64": ms_fp64 / ms_mixed,
        "error_vs_fp64_ref": errors,
        "assembly": {"ms": ms_asm, "gbs": asm_bytes / (ms_asm * 1e-3) / 1e9, "bytes": asm_bytes,
                     "frac_of_" + peak_kind + "_hbm": asm_bytes / (ms_asm * 1e-3) / 1e9 / peak},
        "spmv_fp64": {"ms_cold": spmv64_ms, "ms_warm": spmv64_warm_ms,
                      "gbs_cold": spmv64_bytes / (spmv64_ms * 1e-3) / 1e9, "bytes": spmv64_bytes,
                      "frac_cold": spmv64_bytes / (spmv64_ms * 1e-3) / 1e9 / peak,
                      "frac_warm": spmv64_bytes / (spmv64_warm_ms * 1e-3) / 1e9 / peak, "traffic": traffic64},
        "roofline": {"kernel": "k_pcg_persistent<1,float,64> (the mixed PCG loop: FP32 3x3-block SpMV from "
                               "bulk-copy staged tiles, vector update, grid barriers; one cooperative launch)",
                     "bound": "hbm", "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic_pcg, "bytes_per_launch": pcg_bytes,
                     "iterations_per_launch": pcg_iters, "ms_per_launch": pcg_ms,
                     "us_per_iteration": pcg_ms * 1e3 / pcg_iters,
                     "timing": f"mean of 5 launches of {pcg_iters} iterations, each after a 256 MiB read sweep "
                               "that evicts L2",
                     "spmv_fp32": {"kernel": "k_spmv_tiled<1,float> (the same product as a standalone launch)",
                                   "bytes_per_launch": spmv_bytes, "traffic": traffic,
                                   "ms_cold": spmv_ms, "frac_cold": spmv_bytes / (spmv_ms * 1e-3) / 1e9 / peak,
                                   "ms_warm": spmv_warm_ms,
                                   "frac_warm": spmv_bytes / (spmv_warm_ms * 1e-3) / 1e9 / peak,
                                   "timing": "cold: mean of 20 single launches each after a 256 MiB read sweep; "
                                             "warm: mean of 50 back-to-back launches"}},
        "clocks": clk.summary(),
        "gpu_launches": launches,
        "e2e": {"value": n / (statistics.mean(e2e_ms) * 1e-3), "unit": "DOF/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms": statistics.mean(e2e_ms), "steps": len(e2e_ms),
                "what": "fenics_cuda.solve_elasticity_3d from pinned host mesh/BC arrays: mesh upload, pattern "
                        "build, assembly, body force, Dirichlet, mixed PCG, solution download; mean of the timed "
                        "steps"},
        "setup_s": t_setup,
    }
    if rank == 0 and world == 1 and not args.no_extra:
        res["workloads"] = run_workloads(ctx, stream, peak)
        c2p = res["workloads"].get("c2p", {})
        if "mixed" in c2p:
            sp = c2p["mixed"]["spmv"]
            res["roofline_c2p"] = {"kernel": "k_spmv_tiled<1,float> at C2' (1,568,403 dofs: the FP32 operator "
                                             "exceeds L2)", "bound": "hbm", "achieved": sp["gbs_cold"],
                                   "peak": peak, "unit": "GB/s", "frac": sp["frac_cold"],
                                   "bytes_per_launch": sp["bytes"],
                                   "traffic": _profile_traffic("spmv_bsr3_fp32_elasticity_c2p.txt")}
    if dist and not args.no_extra:
        c5 = run_c5_sharded(ctx, stream, rank, world, tdist)
        if rank == 0:
            res["c5_sharded"] = c5
    if rank == 0 and not args.no_cpu_baseline:
        res["cpu_baseline"] = cpu_baseline_leg(cfg, x_ref)
    if dist:
        tdist.barrier()
        tdist.destroy_process_group()
    ctx.close()
    return res if rank == 0 else None


def run_c5_sharded(ctx, stream, rank, world, tdist):
    """The 256-instance batch (C5) split over the ranks by instance
    (shard_instances: largest estimated cost first onto the least-loaded
    rank). Each rank assembles and solves its shard with the batched PCG on
    its own GPU; nothing is exchanged during the solve. Device time per rank
    by CUDA events, the maximum over ranks by one all_reduce; the solve is
    timed after one untimed warm-up (tuning and graph capture)."""
    import torch
    import fenics_cuda as fcu
    rng = np.random.default_rng(2024)
    ns = rng.integers(32, 257, size=256)
    meshes = [fcu.unit_square(int(n), int(n)) for n in ns]
    kap = [np.exp(rng.standard_normal(m.nc)) for m in meshes]
    fs = [rng.uniform(-1.0, 1.0, m.nv) for m in meshes]
    mine = fcu.shard_instances(fcu.batch_costs(meshes), world)[rank]
    mesh, offs = fcu.concat_meshes([meshes[i] for i in mine])
    V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1)
    M = fcu.Matrix(ctx, V).assemble_stiffness(np.concatenate([kap[i] for i in mine]))
    b = V.rhs_source(fcu.FCU_SRC_NODAL, nodal=np.concatenate([fs[i] for i in mine]))
    bd = V.boundary_dofs()
    M.apply_dirichlet(b, bd, np.zeros(len(bd)))
    M.batch_pcg(offs, b, tol=1e-8, max_iter=100000, precision=fcu.FCU_MIXED)
    tdist.barrier()
    torch.cuda.synchronize()
    ms, (x, it, rel, st, info) = _events_ms(
        stream, lambda: M.batch_pcg(offs, b, tol=1e-8, max_iter=100000, precision=fcu.FCU_MIXED))
    dev = torch.device("cuda", torch.cuda.current_device())
    t = torch.tensor([ms, float(V.ndofs), float((st != 0).sum())], dtype=torch.float64, device=dev)
    tmax = t.clone()
    tdist.all_reduce(tmax, op=tdist.ReduceOp.MAX)
    tsum = t.clone()
    tdist.all_reduce(tsum, op=tdist.ReduceOp.SUM)
    M.close()
    V.close()
    return {"workload": "the 256-problem C5 batch split over the ranks by instance, mixed PCG to 1e-8",
            "ms_max_over_ranks": float(tmax[0]), "dofs_total": int(tsum[1]),
            "dof_per_s": float(tsum[1]) / (float(tmax[0]) * 1e-3), "unconverged": int(tsum[2]),
            "instances_on_rank0": len(mine), "scaling": "strong"}


def _events_ms(stream, fn):
    """Device time of fn() on `stream` (CUDA events on both sides)."""
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1), out


def _best_ms(stream, fn, k=2):
    """Best of k device-timed runs (host stalls on a shared host only add time)."""
    best, out = None, None
    for _ in range(k):
        ms, out = _events_ms(stream, fn)
        best = ms if best is None else min(best, ms)
    return best, out


def run_workloads(ctx, stream, peak):
    """The scope table's other configurations, each measured on this GPU:
    C1 (the reference's own CPU-runnable case), C2' (the 1.5M-dof elasticity),
    C3 (P2 Poisson with a random per-cell coefficient), C4 (adjoint
    sensitivities) and C5 (the batch of 256 uneven Poisson problems). One
    warm-up and one timed run each; inputs resident in HBM."""
    import fenics_cuda as fcu
    out = {}

    # C1: 2D P1 Poisson 64x64, f = 2 pi^2 sin(pi x) sin(pi y), u = 0, FP64 PCG to 1e-10
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())

    def d64(a):
        return torch.as_tensor(np.ascontiguousarray(a), device=dev)

    mesh = fcu.unit_square(64, 64)
    V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1)
    M = fcu.Matrix(ctx, V)
    bd = d64(V.boundary_dofs().astype(np.int64))
    z = torch.zeros(len(bd), dtype=torch.float64, device=dev)
    b = torch.empty(V.ndofs, dtype=torch.float64, device=dev)
    x = torch.empty_like(b)

    def c1():
        M.assemble_stiffness(None)
        V.rhs_source(fcu.FCU_SRC_SIN_PRODUCT, params=(2 * math.pi ** 2, math.pi), out=b)
        M.apply_dirichlet(b, bd, z)
        return M.pcg(b, x=x, tol=1e-10, max_iter=10000, precision=fcu.FCU_FP64)
    c1()
    ms, (x, info) = _best_ms(stream, c1)
    out["c1"] = {"workload": "2D P1 Poisson, unit square 64x64 x 2 triangles (8,192 cells, 4,225 dofs), "
                             "f = 2 pi^2 sin(pi x) sin(pi y), u = 0 on the boundary, FP64 PCG to 1e-10",
                 "ms": ms, "dof_per_s": V.ndofs / (ms * 1e-3), "iterations": int(info.iterations),
                 "u_center": float(x[32 * 65 + 32]), "note": "launch-bound at this size"}
    del x
    M.close(); V.close()

    # C2': 3D vector-P1 elasticity 200x50x50 (1,568,403 dofs), mixed vs FP64
    mesh = fcu.box_beam(4.0, 1.0, 1.0, 200, 50, 50)
    V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1_VEC3)
    M = fcu.Matrix(ctx, V)
    cv = np.nonzero(mesh.coords[:, 0] < 1e-6)[0]
    dofs = d64((3 * cv[:, None] + np.arange(3)).ravel().astype(np.int64))
    zz = torch.zeros(len(dofs), dtype=torch.float64, device=dev)
    fb = np.array([0.0, 0.0, -7.8e4])
    b = torch.empty(V.ndofs, dtype=torch.float64, device=dev)
    x = torch.empty_like(b)
    c2p = {"workload": CONFIGS["c2p"]["workload"], "ndofs": V.ndofs}
    for name, prec in (("mixed", fcu.FCU_MIXED), ("fp64", fcu.FCU_FP64)):
        def step():
            M.assemble_elasticity(210e9, 0.3)
            V.body_force(fb, out=b)
            M.apply_dirichlet(b, dofs, zz)
            return M.pcg(b, x=x, tol=1e-8, max_iter=100000, precision=prec)
        step()
        ms, (_, info) = _best_ms(stream, step)
        c2p[name] = {"ms": ms, "solve_ms": info.kernel_ms, "dof_per_s": V.ndofs / (ms * 1e-3),
                     "iterations": int(info.iterations),
                     "rel_residual": info.rel_residual}
        sms, sbytes = M.time_spmv(prec, reps=20, cold=True)
        wms, _ = M.time_spmv(prec, reps=20)
        c2p[name]["spmv"] = {"ms_cold": sms, "ms_warm": wms, "bytes": sbytes,
                             "gbs_cold": sbytes / (sms * 1e-3) / 1e9,
                             "frac_cold": sbytes / (sms * 1e-3) / 1e9 / peak,
                             "frac_warm": sbytes / (wms * 1e-3) / 1e9 / peak}
    c2p["speedup_mixed_vs_fp64"] = c2p["fp64"]["ms"] / c2p["mixed"]["ms"]
    # stress recovery on the solution (compute_element_stresses / compute_vertex_von_mises)
    cvm = torch.empty(mesh.nc, dtype=torch.float64, device=dev)
    vvm = torch.empty(mesh.nv, dtype=torch.float64, device=dev)
    V.element_stresses(210e9, 0.3, x, von_mises=cvm)
    ms_s, _ = _best_ms(stream, lambda: V.element_stresses(210e9, 0.3, x, von_mises=cvm), k=3)
    ms_v, _ = _best_ms(stream, lambda: V.vertex_von_mises(cvm, out=vvm), k=3)
    sbytes = mesh.nc * (16 + 8) + mesh.nv * (24 + 24)
    # vertex average: per cell its 4 contribution entries (16 B), von Mises value and cached volume
    # (8 B each); per vertex its row bound (4 B) and the result (8 B)
    vbytes = mesh.nc * (16 + 8 + 8) + mesh.nv * (4 + 8)
    c2p["stress_recovery"] = {
        "element_von_mises": {"ms": ms_s, "gbs": sbytes / (ms_s * 1e-3) / 1e9, "bytes": sbytes,
                              "frac_of_hbm": sbytes / (ms_s * 1e-3) / 1e9 / peak},
        "vertex_von_mises": {"ms": ms_v, "gbs": vbytes / (ms_v * 1e-3) / 1e9, "bytes": vbytes,
                             "frac_of_hbm": vbytes / (ms_v * 1e-3) / 1e9 / peak},
        "max_vertex_von_mises_pa": float(vvm.max())}
    out["c2p"] = c2p
    M.close(); V.close()

    # C3: P2 Poisson on the unit cube 64^3 x 6 tets, kappa = exp(g), g ~ N(0,1) per cell, f = 1, u = 0
    mesh = fcu.unit_cube(64, 64, 64)
    V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P2)
    M = fcu.Matrix(ctx, V)
    kappa = d64(np.exp(np.random.default_rng(3).standard_normal(mesh.nc)))
    bd = d64(V.boundary_dofs().astype(np.int64))
    z = torch.zeros(len(bd), dtype=torch.float64, device=dev)
    b = torch.empty(V.ndofs, dtype=torch.float64, device=dev)
    x = torch.empty_like(b)
    c3 = {"workload": "3D P2 Poisson, unit cube 64^3 hexes x 6 tets (1,572,864 tets, 2,146,689 dofs), "
                      "kappa = exp(g), g ~ N(0,1) i.i.d. per cell (seed 3), f = 1, u = 0 on the boundary, "
                      "mixed-precision refined PCG to 1e-8 vs FP64 PCG", "ndofs": V.ndofs, "nnz": M.nnz}
    M.assemble_stiffness(kappa)
    ms_asm, _ = _best_ms(stream, lambda: M.assemble_stiffness(kappa), k=3)
    # the scope table's model, as for C2: per cell its connectivity (4k B), the
    # cell -> slot map (4k^2 B) and the coefficient (8 B); coordinates once;
    # every stored value written once in FP64 and FP32
    asm_bytes = mesh.nc * (10 * 4 + 10 * 10 * 4 + 8) + mesh.nv * 24 + M.nnz * (8 + 4)
    c3["assembly"] = {"ms": ms_asm, "gbs": asm_bytes / (ms_asm * 1e-3) / 1e9, "bytes": asm_bytes,
                      "frac_of_hbm": asm_bytes / (ms_asm * 1e-3) / 1e9 / peak}
    for name, prec in (("mixed", fcu.FCU_MIXED), ("fp64", fcu.FCU_FP64)):
        def step():
            M.assemble_stiffness(kappa)
            V.rhs_source(fcu.FCU_SRC_CONSTANT, params=(1.0,), out=b)
            M.apply_dirichlet(b, bd, z)
            return M.pcg(b, x=x, tol=1e-8, max_iter=100000, precision=prec)
        step()
        ms, (_, info) = _best_ms(stream, step)
        c3[name] = {"ms": ms, "solve_ms": info.kernel_ms, "dof_per_s": V.ndofs / (ms * 1e-3),
                    "iterations": int(info.iterations),
                    "rel_residual": info.rel_residual, "replacements": int(info.outer_updates)}
        sms, sbytes = M.time_spmv(prec, reps=20)
        c3[name]["spmv"] = {"ms": sms, "gbs": sbytes / (sms * 1e-3) / 1e9,
                            "frac_of_hbm": sbytes / (sms * 1e-3) / 1e9 / peak}
    c3["speedup_mixed_vs_fp64"] = c3["fp64"]["ms"] / c3["mixed"]["ms"]
    out["c3"] = c3
    M.close(); V.close()

    # C4: adjoint sensitivities, box [0,3]x[0,1]x[0,1] 96x32x32 x 6 tets, E_e = theta_e^3, nu = 0.3
    L = 3.0
    mesh = fcu.box_beam(L, 1.0, 1.0, 96, 32, 32)
    theta = np.random.default_rng(4).uniform(0.01, 1.0, mesh.nc)
    facets = fcu.facets_on_plane(mesh, 0, L, ctx)
    cv = np.nonzero(mesh.coords[:, 0] < 1e-6)[0]
    dofs = (3 * cv[:, None] + np.arange(3)).ravel().astype(np.int64)
    Vt = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1_VEC3)
    f = fcu.traction_load(Vt, facets, (0.0, 0.0, -1.0))
    Vt.close()
    verts, cells, _ = fcu.extract_boundary_facets(mesh, ctx)
    tipc = cells[np.all(np.abs(mesh.coords[verts][..., 0] - L) < 1e-9, axis=1)]
    tipv = np.unique(mesh.cells[tipc])
    cz = np.zeros(3 * mesh.nv)
    cz[3 * tipv + 2] = 1.0 / len(tipv)
    c4 = {"workload": "adjoint sensitivities, 3D vector-P1 elasticity on [0,3]x[0,1]x[0,1], 96x32x32 hexes x 6 "
                      "tets (589,824 tets, 316,899 dofs), theta ~ U[0.01,1] per cell (seed 4), E = theta^3, "
                      "nu = 0.3, clamped x = 0, unit downward traction on x = 3; objectives compliance and mean "
                      "u_z over the vertices of the cells touching x = 3; mixed PCG to 1e-8"}
    for name, obj in (("compliance", "compliance"), ("tip_uz", cz)):
        adj = fcu.ElasticityAdjoint(mesh, 0.3, f, dofs, objective=obj, ctx=ctx, tol=1e-8,
                                    precision=fcu.FCU_MIXED)
        adj.forward(theta)
        adj.backward()
        ms_f, J = _best_ms(stream, lambda: adj.forward(theta))
        ms_b, g = _best_ms(stream, lambda: adj.backward())
        c4[name] = {"J": J, "forward_ms": ms_f, "forward_solve_ms": adj.info.kernel_ms, "backward_ms": ms_b,
                    "forward_iterations": int(adj.info.iterations), "grad_norm": float(np.linalg.norm(g)),
                    "inputs": "host arrays (theta, load) staged per call"}
        if name == "compliance":
            th_d, u_d = d64(theta), d64(adj.u)
            gd = torch.empty(mesh.nc, dtype=torch.float64, device=dev)
            ms_g, _ = _best_ms(stream, lambda: adj.V.adjoint_gradient(1.0, 0.3, th_d, u_d, u_d, out=gd), k=3)
            gbytes = mesh.nc * (16 + 8 + 8) + mesh.nv * (24 + 2 * 24)
            c4["gradient_kernel"] = {"ms": ms_g, "gbs": gbytes / (ms_g * 1e-3) / 1e9, "bytes": gbytes,
                                     "frac_of_hbm": gbytes / (ms_g * 1e-3) / 1e9 / peak}
        else:
            c4[name]["adjoint_iterations"] = int(adj.adjoint_info.iterations)
        adj.close()
    out["c4"] = c4

    # C5: 256 independent 2D P1 Poisson problems on N x N unit squares, N ~ U{32..256}
    rng = np.random.default_rng(2024)
    ns = rng.integers(32, 257, size=256)
    meshes = [fcu.unit_square(int(n), int(n)) for n in ns]
    kap = np.concatenate([np.exp(rng.standard_normal(m.nc)) for m in meshes])
    fs = np.concatenate([rng.uniform(-1.0, 1.0, m.nv) for m in meshes])
    mesh, offs = fcu.concat_meshes(meshes)
    V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1)
    M = fcu.Matrix(ctx, V).assemble_stiffness(kap)
    b = V.rhs_source(fcu.FCU_SRC_NODAL, nodal=fs)
    bd = V.boundary_dofs()
    M.apply_dirichlet(b, bd, np.zeros(len(bd)))
    c5 = {"workload": "256 independent 2D P1 Poisson problems, instance i on an N_i x N_i right-diagonal unit "
                      "square, N_i ~ U{32..256} (seed 2024), kappa = exp(N(0,1)) per cell, nodal f ~ U[-1,1], "
                      "u = 0 on each boundary, one persistent graph-captured launch, PCG to 1e-8 per instance",
          "instances": 256, "ndofs": V.ndofs, "nnz": M.nnz}
    for name, prec in (("mixed", fcu.FCU_MIXED), ("fp64", fcu.FCU_FP64)):
        M.batch_pcg(offs, b, tol=1e-8, max_iter=100000, precision=prec)  # tunes, captures the graph
        ms, (x, it, rel, st, info) = _best_ms(
            stream, lambda: M.batch_pcg(offs, b, tol=1e-8, max_iter=100000, precision=prec))
        c5[name] = {"ms": info.kernel_ms, "ms_call": ms, "dof_per_s": V.ndofs / (info.kernel_ms * 1e-3),
                    "iterations_max": int(it.max()), "iterations_mean": float(it.mean()),
                    "unconverged": int((st != 0).sum()), "rel_residual_max": float(rel.max()),
                    "effective_gbs": info.effective_bw_gbps, "frac_of_hbm": info.effective_bw_gbps / peak,
                    "tuned": dict(zip(("lanes_per_row", "threads_per_cta", "ctas_per_instance"),
                                      M.batch_config(prec)))}
    c5["speedup_mixed_vs_fp64"] = c5["fp64"]["ms"] / c5["mixed"]["ms"]
    out["c5"] = c5
    M.close(); V.close()

    # Mass matrix of the C2 mesh (assemble_elasticity_mass_3d, density 7850)
    mesh = fcu.box_beam(4.0, 1.0, 1.0, 128, 32, 32)
    V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1_VEC3)
    M = fcu.Matrix(ctx, V).assemble_mass(7850.0)
    ms_m, _ = _best_ms(stream, lambda: M.assemble_mass(7850.0), k=3)
    stored = V.nnz  # scalar entries of the 3x3 blocks the kernel writes
    mbytes = mesh.nc * (4 * 4 + 4 * 16) + mesh.nv * 24 + stored * (8 + 4)
    out["mass_c2"] = {"workload": "vector-P1 mass matrix of the C2 mesh (786,432 tets), density 7850",
                      "ms": ms_m, "gbs": mbytes / (ms_m * 1e-3) / 1e9, "bytes": mbytes,
                      "frac_of_hbm": mbytes / (ms_m * 1e-3) / 1e9 / peak}
    M.close()

    # 3x3 block-Jacobi PCG on the C2 system (solve_bsr3_pcg_gpu's preconditioner) vs point Jacobi, FP64
    K = fcu.Matrix(ctx, V).assemble_elasticity(210e9, 0.3)
    cv = np.nonzero(mesh.coords[:, 0] < 1e-6)[0]
    dofs = d64((3 * cv[:, None] + np.arange(3)).ravel().astype(np.int64))
    b = torch.empty(V.ndofs, dtype=torch.float64, device=dev)
    V.body_force(np.array([0.0, 0.0, -7.8e4]), out=b)
    K.apply_dirichlet(b, dofs, torch.zeros(len(dofs), dtype=torch.float64, device=dev))
    x = torch.empty_like(b)
    bj = {"workload": "C2 system after Dirichlet elimination, FP64 PCG to 1e-8: 3x3 block-Jacobi (inverse "
                      "diagonal blocks, recomputed per solve) vs point Jacobi"}
    for name, on in (("block_jacobi", True), ("point_jacobi", False)):
        K.block_jacobi(on)
        K.pcg(b, x=x, tol=1e-8, max_iter=100000)
        ms, (_, info) = _best_ms(stream, lambda: K.pcg(b, x=x, tol=1e-8, max_iter=100000))
        bj[name] = {"ms": ms, "iterations": int(info.iterations), "dof_per_s": V.ndofs / (ms * 1e-3),
                    "effective_gbs": info.effective_bw_gbps}
    out["bsr3_block_jacobi_c2"] = bj
    K.close(); V.close()

    # Transient heat: unit square 1024^2, Crank-Nicolson, dt = 1e-4, u = 0 on the boundary
    mesh = fcu.unit_square(1024, 1024)
    V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1)
    Mm = fcu.Matrix(ctx, V).assemble_mass(1.0)
    K = fcu.Matrix(ctx, V).assemble_stiffness(None)
    bd = V.boundary_dofs().astype(np.int64)
    u0 = d64(np.sin(math.pi * mesh.coords[:, 0]) * np.sin(math.pi * mesh.coords[:, 1]))
    tr = {"workload": "2D transient heat, unit square 1024x1024 x 2 triangles (1,050,625 dofs), diffusivity 1, "
                      "Crank-Nicolson dt = 1e-4, u0 = sin(pi x) sin(pi y), u = 0 on the boundary, no source, "
                      "20 steps, each solved by PCG from the previous state to 1e-10",
          "ndofs": V.ndofs}
    nsteps = 20
    for name, prec in (("fp64", fcu.FCU_FP64), ("mixed", fcu.FCU_MIXED)):
        st = fcu._Stepper(ctx, Mm, K, fcu.FCU_CRANK_NICOLSON, 1e-4)
        st.set_dirichlet(bd, np.zeros(len(bd)))
        ua, ub = u0.clone(), torch.empty_like(u0)
        st.step(ua, None, None, ub, 1e-10, 100000, prec)   # warm-up: tuning and graph capture

        def run():
            a, b2 = u0.clone(), torch.empty_like(u0)
            its = []
            for _ in range(nsteps):
                its.append(int(st.step(a, None, None, b2, 1e-10, 100000, prec).iterations))
                a, b2 = b2, a
            return a, its
        ms, (uf, its) = _best_ms(stream, run)
        exact = math.exp(-2 * math.pi ** 2 * nsteps * 1e-4)
        tr[name] = {"ms": ms, "ms_per_step": ms / nsteps, "iterations_per_step": float(np.mean(its)),
                    "dof_steps_per_s": V.ndofs * nsteps / (ms * 1e-3),
                    "center_over_exact": float(uf[512 * 1025 + 512]) / exact}
        st.close()
    out["transient_heat"] = tr
    Mm.close(); K.close(); V.close()

    # Vibration modes: steel cantilever [0,4]x[0,1]x[0,1], 64x16x16 x 6 tets, clamped x = 0
    mesh = fcu.box_beam(4.0, 1.0, 1.0, 64, 16, 16)
    V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1_VEC3)
    K = fcu.Matrix(ctx, V).assemble_elasticity(210e9, 0.3)
    Mm = fcu.Matrix(ctx, V).assemble_mass(7850.0)
    cv = np.nonzero(mesh.coords[:, 0] < 1e-6)[0]
    fixed = (3 * cv[:, None] + np.arange(3)).ravel().astype(np.int64)
    md = {"workload": "lowest 3 vibration modes of a steel cantilever [0,4]x[0,1]x[0,1], 64x16x16 hexes x 6 tets "
                      "(56,355 dofs), E = 210e9, nu = 0.3, density 7850, clamped x = 0; inverse power iteration, "
                      "30 iterations at most, tol 1e-6, inner PCG to 1e-9 from the previous iterate",
          "ndofs": V.ndofs}
    for name, prec in (("fp64", fcu.FCU_FP64), ("mixed", fcu.FCU_MIXED)):
        def run():
            return fcu.solve_vibration_modes(K, Mm, fixed, 3, 30, 1e-6, ctx, precision=prec, inner_tol=1e-9,
                                             inner_max_iter=50000, return_stats=True)
        run()
        ms, (modes, pit, info) = _best_ms(stream, run)
        md[name] = {"ms": ms, "frequencies_hz": [m.frequency_hz for m in modes],
                    "power_iterations": [int(p) for p in pit], "inner_iterations": int(info.iterations)}
    out["modes"] = md
    K.close(); Mm.close(); V.close()
    return out


def run_reference(args, cfg):
    """The reference arm: the reference's path on the host cores (its Rust
    build is not possible in this image, so the CPU restatement under
    oracle/), on the same workload, config and metric as the GPU arm. Every
    timed step is one complete solve to 1e-8 (no extrapolation); warm-up
    steps run the setup and 50 CG iterations. Under torchrun only rank 0
    runs it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    cp = CpuPath(cfg)
    for _ in range(args.warmup):
        Kb, fb = cp.setup()
        cp.O.cg_fixed_iters_mt(Kb, fb, 50, cp.threads)
        del Kb, fb
    steps = []
    for _ in range(args.steps):
        r = cp.full_step()
        last = r.pop("system")
        r.pop("x")
        steps.append(r)
    ms = 1e3 * statistics.mean(r["s"] for r in steps)
    per_it, seq_cg = cp.sequential_cg_sample(*last, steps[-1]["iterations"])
    v = cp.n / (ms * 1e-3)
    sample = (f"each step one complete solve of the workload: oracle assembly ({cp.threads} threads for the cell "
              f"loop, sequential faer-style triplet build) + body force + Dirichlet "
              f"({statistics.mean(r['setup_s'] for r in steps):.2f} s) and Jacobi-PCG to 1e-8 with its SpMV, "
              f"vector loops and dot products on {cp.threads} threads ({steps[-1]['iterations']} iterations, "
              f"{statistics.mean(r['cg_s'] for r in steps):.2f} s); mean of {len(steps)} steps")
    return {
        "metric": METRIC, "value": v, "unit": "DOF/s", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (generated box mesh)",
        "config": config_dict(cfg), "impl": "reference",
        "cpu_baseline": {"value": v, "unit": "DOF/s", "cores": cp.threads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "DOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "iterations": steps[-1]["iterations"], "rel_residual": steps[-1]["rel_residual"],
        "sequential_cg": {"value": cp.n / (statistics.mean(r["setup_s"] for r in steps) + seq_cg),
                          "unit": "DOF/s", "cores": 1,
                          "sample": f"cg.rs as written (sequential column-scatter SpMV): 40 iterations "
                                    f"({per_it * 1e3:.1f} ms each) scaled to the measured "
                                    f"{steps[-1]['iterations']} iterations, plus the same setup"},
        "note": "the reference (Rust) cannot be built in this image; its path runs through the C++ "
                "restatement under oracle/ on the host cores",
    }


PROFILE_CASES = ("elasticity_c2", "mass_c2", "block_update_c2", "transient_1024", "batch_c5", "p2_cube40",
                 "spmv_c2p", "spmv_c2", "p2_c3", "pcg_c2", "pcg_c2_small", "solve_c2_mixed", "solve_c2_fp64")


def profile_case(name):
    """A short run of one kernel on one workload, for profiler captures: no
    timing, a few launches, a few hundred MB on the device.
      elasticity_c2    elasticity stiffness of the C2 mesh, assembled 3 times
      mass_c2          vector-P1 mass of the C2 mesh, assembled 3 times
      block_update_c2  12 block-Jacobi FP64 PCG iterations on the C2 system
      transient_1024   3 Crank-Nicolson steps of the 1024^2 heat problem,
                       12 PCG iterations each
      batch_c5         the C5 batch of 256 Poisson problems, mixed PCG capped
                       at 60 iterations per instance, 3 launches of the
                       persistent batch kernel (shape fixed by FCU_BATCH_* if
                       set, else tuned first)
      p2_cube40        P2 stiffness on the unit cube 40^3 x 6 tets (384,000
                       cells, 531,441 dofs), random kappa, assembled 3 times
                       (the C3 kernel on a quarter of its cells)
      spmv_c2p         the mixed PCG's FP32 block SpMV on the C2' system
                       (1,568,403 dofs, operator larger than L2), 3 launches
                       each after an L2 flush, shape tuning off
      spmv_c2          the same on the C2 system (421,443 dofs)
      p2_c3            P2 stiffness of the C3 cube (64^3 x 6 tets, random
                       kappa), assembled 3 times (for one-pass metrics only)
      pcg_c2           the mixed PCG's persistent loop on the C2 system: one
                       launch of exactly 300 iterations after an L2 flush
                       (the launch the bench's roofline times; shape tuning
                       off)
      pcg_c2_small     the same loop on the 32x8x8 beam (24k dofs), 20
                       iterations, for the full-section capture
      solve_c2_mixed   one complete mixed PCG solve of the C2 system to 1e-8
                       (assembly, load and Dirichlet before it; shape tuning
                       off), for the launch list of a solve
      solve_c2_fp64    the FP64 PCG of the C2 system, 100 iterations"""
    import torch
    if name in ("spmv_c2p", "spmv_c2", "pcg_c2", "pcg_c2_small", "solve_c2_mixed", "solve_c2_fp64"):
        os.environ["FCU_TUNE"] = "0"   # no shape-tuning launches before the captured ones
    import fenics_cuda as fcu
    ctx = fcu.Context(0)
    if name in ("spmv_c2p", "spmv_c2"):
        cfg = CONFIGS["c2p" if name == "spmv_c2p" else "c2"]
        mesh = fcu.box_beam(cfg["L"], cfg["W"], cfg["H"], cfg["nx"], cfg["ny"], cfg["nz"])
        V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1_VEC3)
        M = fcu.Matrix(ctx, V).assemble_elasticity(210e9, 0.3)
        cv = np.nonzero(mesh.coords[:, 0] < 1e-6)[0]
        dofs = (3 * cv[:, None] + np.arange(3)).ravel().astype(np.int64)
        b = V.body_force([0.0, 0.0, -7.8e4])
        M.apply_dirichlet(b, dofs, np.zeros(len(dofs)))
        M.time_spmv(fcu.FCU_MIXED, reps=3, cold=True)
        ctx.synchronize()
        M.close(); V.close()
    elif name in ("solve_c2_mixed", "solve_c2_fp64"):
        mesh = fcu.box_beam(4.0, 1.0, 1.0, 128, 32, 32)
        V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1_VEC3)
        M = fcu.Matrix(ctx, V).assemble_elasticity(210e9, 0.3)
        cv = np.nonzero(mesh.coords[:, 0] < 1e-6)[0]
        dofs = (3 * cv[:, None] + np.arange(3)).ravel().astype(np.int64)
        b = V.body_force([0.0, 0.0, -7.8e4])
        M.apply_dirichlet(b, dofs, np.zeros(len(dofs)))
        if name == "solve_c2_mixed":
            M.pcg(b, tol=1e-8, max_iter=100000, precision=fcu.FCU_MIXED)
        else:
            M.pcg(b, tol=1e-30, max_iter=100, precision=fcu.FCU_FP64, raise_on_error=False)
        ctx.synchronize()
        M.close(); V.close()
    elif name in ("pcg_c2", "pcg_c2_small"):
        dims = (128, 32, 32) if name == "pcg_c2" else (32, 8, 8)
        mesh = fcu.box_beam(4.0, 1.0, 1.0, *dims)
        V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1_VEC3)
        M = fcu.Matrix(ctx, V).assemble_elasticity(210e9, 0.3)
        cv = np.nonzero(mesh.coords[:, 0] < 1e-6)[0]
        dofs = (3 * cv[:, None] + np.arange(3)).ravel().astype(np.int64)
        b = V.body_force([0.0, 0.0, -7.8e4])
        M.apply_dirichlet(b, dofs, np.zeros(len(dofs)))
        M.time_pcg(fcu.FCU_MIXED, iterations=300 if name == "pcg_c2" else 20, reps=1)
        ctx.synchronize()
        M.close(); V.close()
    elif name in ("elasticity_c2", "mass_c2", "block_update_c2"):
        mesh = fcu.box_beam(4.0, 1.0, 1.0, 128, 32, 32)
        V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1_VEC3)
        if name in ("elasticity_c2", "mass_c2"):
            M = fcu.Matrix(ctx, V)
            for _ in range(3):
                if name == "mass_c2":
                    M.assemble_mass(7850.0)
                else:
                    M.assemble_elasticity(210e9, 0.3)
        else:
            M = fcu.Matrix(ctx, V).assemble_elasticity(210e9, 0.3)
            cv = np.nonzero(mesh.coords[:, 0] < 1e-6)[0]
            dofs = (3 * cv[:, None] + np.arange(3)).ravel().astype(np.int64)
            b = V.body_force([0.0, 0.0, -7.8e4])
            M.apply_dirichlet(b, dofs, np.zeros(len(dofs)))
            M.block_jacobi(True)
            M.pcg(b, tol=1e-30, max_iter=12, raise_on_error=False)
        ctx.synchronize()
        M.close(); V.close()
    elif name in ("p2_cube40", "p2_c3"):
        mesh = fcu.unit_cube(40, 40, 40) if name == "p2_cube40" else fcu.unit_cube(64, 64, 64)
        kap = np.exp(np.random.default_rng(3).standard_normal(mesh.nc))
        V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P2)
        M = fcu.Matrix(ctx, V)
        for _ in range(3):
            M.assemble_stiffness(kap)
        ctx.synchronize()
        M.close(); V.close()
    elif name == "batch_c5":
        rng = np.random.default_rng(2024)
        ns = rng.integers(32, 257, size=256)
        meshes = [fcu.unit_square(int(n), int(n)) for n in ns]
        kap = np.concatenate([np.exp(rng.standard_normal(m.nc)) for m in meshes])
        fs = np.concatenate([rng.uniform(-1.0, 1.0, m.nv) for m in meshes])
        mesh, offs = fcu.concat_meshes(meshes)
        V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1)
        M = fcu.Matrix(ctx, V).assemble_stiffness(kap)
        b = V.rhs_source(fcu.FCU_SRC_NODAL, nodal=fs)
        bd = V.boundary_dofs()
        M.apply_dirichlet(b, bd, np.zeros(len(bd)))
        for _ in range(3):
            M.batch_pcg(offs, b, tol=1e-8, max_iter=60, precision=fcu.FCU_MIXED, raise_on_error=False)
        ctx.synchronize()
        M.close(); V.close()
    elif name == "transient_1024":
        mesh = fcu.unit_square(1024, 1024)
        V = fcu.FunctionSpace(ctx, mesh, fcu.FCU_SPACE_P1)
        Mm = fcu.Matrix(ctx, V).assemble_mass(1.0)
        K = fcu.Matrix(ctx, V).assemble_stiffness(None)
        st = fcu._Stepper(ctx, Mm, K, fcu.FCU_CRANK_NICOLSON, 1e-4)
        dev = torch.device("cuda", 0)
        u = torch.as_tensor(np.sin(math.pi * mesh.coords[:, 0]) * np.sin(math.pi * mesh.coords[:, 1])).to(dev)
        un = torch.empty_like(u)
        for _ in range(3):
            try:
                st.step(u, None, None, un, 1e-30, 12, fcu.FCU_FP64)
            except fcu.CgError:
                pass   # 12 iterations, no convergence: the point is the kernels
            u, un = un, u
        ctx.synchronize()
        st.close(); Mm.close(); K.close(); V.close()
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the C1/C2'/C3/C4/C5 workload measurements")
    ap.add_argument("--profile", choices=PROFILE_CASES, help="run one kernel's short profiling case and exit")
    args = ap.parse_args()
    if args.profile:
        profile_case(args.profile)
        return
    cfg = CONFIGS[args.config]
    res = run_reference(args, cfg) if args.impl == "reference" else run_cuda(args, cfg)
    if res is not None:
        print(json.dumps(res))


if __name__ == "__main__":
    main()
