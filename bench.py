"""Benchmark of the B200 implicit hot path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload flow|solve] [--cells 1000000] [--precision fp32_refine|fp64]

Workload "flow" (default): implicit time steps (flow_imp + flow_update) of the
three-level telescoping tidal inlet of about 1.0M active cells (40/20/10 m,
M2 + K1 tide on the north edge, dt = 300 s), every linear solve (u, v, pp;
ILU(0)-BiCGStab) driven to a 1e-6 relative L2 residual.  One step = one
implicit time step (all SIMPLEC outer iterations until check_conv).  The
headline runs the solves in FP32 inside FP64 iterative refinement; the plain
FP64 drop-in runs the same steps in the same process for comparison.

Workload "solvers": one solve() call per MATRIX_SOLVER option (Gauss-Seidel,
SGS, BiCGStab, GMRES, SIP, ICCG, ICCGSTAB) on a symmetric Cartesian system of
--cells unknowns, FP64, at the reference's default nswp(n); ms per call.

Workload "solve": the pressure-correction system of the solver sweep at 1M
unknowns (telescoping 5-point stencil with up to two extra neighbours per face
at refinement interfaces, seeded off-diagonals in [-1,-0.1], diagonal 1.02 x
the off-diagonal sum, N(0,1) right-hand side), solved by ILU(0)-BiCGStab to a
1e-6 relative FP64 residual.  One step = one solve from phi = 0.

Multi-GPU: the path does not shard (the ILU(0) sweeps are global
recurrences), so N ranks run N independent replicas and `value` counts the
solves of all ranks over the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "timesteps/s at 1M cells, FP32+refine vs plain FP64 GPU @1e-6 resid; HBM GB/s"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1])); mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def build_solve_case(cells: int, seed: int):
    from cms2d_b200 import grid as G
    g = G.solver_test_grid(cells)
    acoef, ss, sp, phi = G.random_system(g, seed=seed)
    return g, acoef, ss, sp, phi


def run_solve_ours(args):
    import torch
    import torch.distributed as dist
    from cms2d_b200 import solver as S

    world, rank, local = dist_setup()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    g, acoef, ss, sp, phi = build_solve_case(args.cells, seed=17 + rank)
    N = g.ncells
    solver = S.Solver(g, precision=args.precision, tol=1e-6, norm=2, verify=False, inner_tol=args.inner_tol,
                      inner_max=args.inner_max, nsolv=3, multi_kernel=args.multi_kernel,
                      reduced_layout=args.reduced_layout)
    nswp = 5000
    # device-resident inputs
    t_acoef = torch.from_numpy(acoef).to(dev)
    t_sp = torch.from_numpy(sp).to(dev)
    t_ss0 = torch.from_numpy(ss).to(dev)
    t_phi0 = torch.from_numpy(phi).to(dev)
    t_ss = t_ss0.clone(); t_phi = t_phi0.clone(); t_res = torch.zeros_like(t_ss)
    sstream = torch.cuda.ExternalStream(solver.stream_handle, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    def step():
        t_ss.copy_(t_ss0); t_phi.copy_(t_phi0)
        torch.cuda.synchronize(dev)
        return solver.solve(t_acoef, t_ss, t_sp, t_res, t_phi, relax=1.0, nswp=nswp, nsolv=3)

    for _ in range(args.warmup):
        info = step()
    # timed: K steps, per-step CUDA events on the solver stream, L2 flushed between steps
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    launches0 = solver.launches
    ms_total = 0.0
    infos = []
    if args.ncu:  # a profiler started with --profile-from-start off sees the timed steps only
        torch.cuda.profiler.start()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            t_ss.copy_(t_ss0); t_phi.copy_(t_phi0)
            flush.fill_(1.0)
            torch.cuda.synchronize(dev)
            e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
            e0.record(sstream)
            infos.append(solver.solve(t_acoef, t_ss, t_sp, t_res, t_phi, relax=1.0, nswp=nswp, nsolv=3))
            e1.record(sstream)
            e1.synchronize()
            ms_total += e0.elapsed_time(e1)
    torch.cuda.synchronize(dev)
    if args.ncu:
        torch.cuda.profiler.stop()
    launches = solver.launches - launches0
    if world > 1:
        t = torch.tensor([ms_total], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total = float(t.item())
        dist.barrier()
    ms_step = ms_total / args.steps
    value = world * args.steps / (ms_total / 1e3)  # solves/s over all ranks
    if args.ncu:  # profiler pass: the timed steps only
        if world > 1:
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"ncu_pass": True, "ms_per_step": ms_step, "iters": infos[-1]["iters"]}), flush=True)
        return

    # true residual of the last solve (device-resident inputs unchanged)
    solver.set_options(verify=True)
    chk = step()
    solver.set_options(verify=False)

    # e2e: host (pinned) buffers through the C-ABI host entry point, copies included
    h_acoef = torch.from_numpy(acoef).pin_memory().numpy()
    h_sp = torch.from_numpy(sp).pin_memory().numpy()
    h_ss = torch.from_numpy(ss).pin_memory().numpy()
    h_phi = torch.from_numpy(phi).pin_memory().numpy()
    h_res = torch.zeros(g.ncellsD, dtype=torch.float64).pin_memory().numpy()
    e2e_ms = 0.0
    ne2e = max(1, min(args.steps, 5))
    for q in range(ne2e + 1):
        h_ss[:] = ss; h_phi[:] = phi
        flush.fill_(1.0); torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        solver.solve(h_acoef, h_ss, h_sp, h_res, h_phi, relax=1.0, nswp=nswp, nsolv=3)
        t1 = time.perf_counter()
        if q > 0:
            e2e_ms += (t1 - t0) * 1e3
    e2e_ms /= ne2e
    h2d = acoef.nbytes + ss.nbytes + sp.nbytes + phi.nbytes
    d2h = 3 * N * 8

    # roofline: per-kernel-class events on the solver stream over K profiled steps
    solver.profile(True)
    solver.profile_read(reset=True)
    for _ in range(args.steps):
        t_ss.copy_(t_ss0); t_phi.copy_(t_phi0); flush.fill_(1.0); torch.cuda.synchronize(dev)
        solver.solve(t_acoef, t_ss, t_sp, t_res, t_phi, relax=1.0, nswp=nswp, nsolv=3)
    prof = solver.profile_read(reset=True)
    solver.profile(False)
    top = max(prof, key=lambda k: prof[k]["ms"])
    peak, peak_kind = _peaks()
    tot_ms = sum(v["ms"] for v in prof.values())
    ach = prof[top]["bytes"] / (prof[top]["ms"] / 1e3) / 1e9 if prof[top]["ms"] > 0 else 0.0
    kernels = {k: {"share": round(v["ms"] / tot_ms, 4) if tot_ms else 0, "launches": v["launches"],
                   "avg_us": round(1e3 * v["ms"] / v["launches"], 2) if v["launches"] else 0,
                   "GBps": round(v["bytes"] / (v["ms"] / 1e3) / 1e9, 1) if v["ms"] > 0 else 0}
               for k, v in prof.items() if v["launches"]}

    out = {
        "metric": METRIC,
        "value": round(value, 4),
        "unit": "solves/s (1M-unknown pressure-correction system to 1e-6)",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64 refine" if args.precision == "fp32_refine" else args.precision.replace("fp", "f"),
        "data": "synthetic (seeded solver-sweep system)",
        "config": {"workload": f"pp-system solve, {N} unknowns, telescoping 5-point+interfaces, "
                               f"ILU0-BiCGStab to ||r||2/||r0||2<=1e-6 ({args.precision})",
                   "cells": N, "precision": args.precision, "ordering": "multicolor",
                   "colours": solver.ncolors, "parallelism": f"replicas x{world}",
                   "l2": "flushed between steps (256 MB write)"},
        "iters_per_step": infos[-1]["iters"], "refine_steps": infos[-1].get("refine_steps", 0),
        "true_relres": chk["true_relres"],
        "e2e": {"value": round(world * 1e3 / e2e_ms, 4), "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": round(e2e_ms, 3)},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": top, "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(ach / peak, 4), "peak_kind": peak_kind,
                     "traffic": None, "traffic_note": "not captured for the solve workload"},
        "kernels": kernels,
    }
    out["clocks"] = clk.summary()
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        out["cpu_baseline"] = cpu_baseline(args, g, acoef, ss, sp, phi)
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def cpu_baseline(args, g, acoef, ss, sp, phi, threads=None):
    """The oracle port (the reference's algorithm restated) on host cores."""
    from oracle import oracle as O
    threads = threads or os.cpu_count()
    O.set_threads(threads)
    o = O.OracleSolver(g)
    a, b, c, p = [x.copy() for x in (acoef, ss, sp, phi)]
    r = np.zeros_like(b)
    t0 = time.perf_counter()
    out = o.solve(a, b, c, r, p, relax=1.0, nswp=5000, nsolv=3, precond=O.PC_ILU0, tol=1e-6, norm=2)
    dt = time.perf_counter() - t0
    return {"value": round(1.0 / dt, 4), "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": f"1 full solve of the same {g.ncells}-unknown system, natural-order ILU0-BiCGStab "
                      f"(serial factor/sweeps as in the reference), {out['iters']} iterations",
            "iters": out["iters"]}


# MATRIX_SOLVER options timed by the "solvers" workload: (nsolv, n, ordering),
# nswp(n) at the reference's defaults for that solver (flow.F90:752-821)
SOLVER_OPTIONS = [(3, 1, "multicolor"), (4, 1, "multicolor"), (1, 1, "multicolor"), (1, 1, "natural"),
                  (2, 2, "multicolor"), (2, 2, "natural"), (6, 1, "natural"), (7, 1, "multicolor"),
                  (7, 1, "natural"), (8, 2, "multicolor"), (8, 2, "natural")]
SOLVER_LABEL = {1: "Gauss-Seidel", 2: "SGS", 3: "BiCGStab", 4: "GMRES", 6: "SIP", 7: "ICCG", 8: "ICCGSTAB"}


def symmetric_cartesian_system(nx: int, ny: int, seed: int):
    """Cartesian grid with the solver-sweep values made symmetric (the face
    coefficient of a cell pair is shared), so that every option, ICCG included,
    sees a symmetric positive definite pressure-correction-like system."""
    from cms2d_b200 import grid as G
    g = G.cartesian_grid(nx, ny)
    acoef, ss, sp, phi = G.random_system(g, seed=seed)
    n = g.ncells
    for k, kb in ((2, 0), (3, 1)):  # south face = the south neighbour's north face; west = west's east
        j = g.cell2cell[:n, k].astype(np.int64) - 1
        m = j < n
        acoef[:n, k][m] = acoef[j[m], kb]
    sp[:n] = -0.02 * acoef[:n].sum(axis=1)
    return g, acoef, ss, sp, phi


def run_solvers_ours(args):
    """ms per solve() call for each MATRIX_SOLVER option on one system."""
    import torch
    from cms2d_b200 import solver as S
    world, rank, local = dist_setup()
    if rank != 0:
        return
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    side = int(round(args.cells ** 0.5))
    g, acoef, ss, sp, phi = symmetric_cartesian_system(side, side, seed=17)
    N = g.ncells
    t_acoef = torch.from_numpy(acoef).to(dev)
    t_sp = torch.from_numpy(sp).to(dev)
    t_ss0 = torch.from_numpy(ss).to(dev)
    t_phi0 = torch.from_numpy(phi).to(dev)
    t_ss = t_ss0.clone(); t_phi = t_phi0.clone(); t_res = torch.zeros_like(t_ss)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    rows = []
    with ClockSampler(local) as clk:
        for nsolv, n, ordering in SOLVER_OPTIONS:
            solver = S.Solver(g, ordering=ordering, precision="fp64", verify=False, nsolv=nsolv)
            sstream = torch.cuda.ExternalStream(solver.stream_handle, device=dev)
            nswp = S.NSWP_DEFAULT[nsolv][n]
            ms, info = 0.0, None
            for q in range(args.warmup + args.steps):
                t_ss.copy_(t_ss0); t_phi.copy_(t_phi0); flush.fill_(1.0)
                torch.cuda.synchronize(dev)
                e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
                e0.record(sstream)
                info = solver.solve(t_acoef, t_ss, t_sp, t_res, t_phi, n=n, relax=1.0, nswp=nswp, nsolv=nsolv,
                                    raise_on_error=False)
                e1.record(sstream)
                e1.synchronize()
                if q >= args.warmup:
                    ms += e0.elapsed_time(e1)
            solver.set_options(verify=True)
            t_ss.copy_(t_ss0); t_phi.copy_(t_phi0)
            chk = solver.solve(t_acoef, t_ss, t_sp, t_res, t_phi, n=n, relax=1.0, nswp=nswp, nsolv=nsolv,
                               raise_on_error=False)
            rows.append({"nsolv": nsolv, "solver": SOLVER_LABEL[nsolv], "n": n, "ordering": ordering,
                         "nswp": nswp, "groups": solver.ncolors, "ms_per_solve": round(ms / args.steps, 3),
                         "iters": info["iters"], "status": info["status"],
                         "true_relres": chk["true_relres"]})
            solver.close()
    out = {"metric": "ms per solve() call by MATRIX_SOLVER option (FP64, nswp(n) of the reference defaults)",
           "value": None, "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded symmetric solver-sweep values on a Cartesian grid)",
           "config": {"workload": f"solve() of a {side}x{side} Cartesian system ({N} unknowns), every "
                                  f"MATRIX_SOLVER option", "cells": N,
                      "l2": "flushed between solves (256 MB write)"},
           "options": rows, "clocks": clk.summary()}
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        O.set_threads(1)
        o = O.OracleSolver(g)
        cpu = []
        for nsolv, n, ordering in SOLVER_OPTIONS:
            if ordering != "natural" and nsolv not in (3, 4):
                continue
            a, b, c, p = [x.copy() for x in (acoef, ss, sp, phi)]
            t0 = time.perf_counter()
            r = o.solve(a, b, c, np.zeros_like(b), p, relax=1.0, nswp=S.NSWP_DEFAULT[nsolv][n], nsolv=nsolv, n=n,
                        precond=O.PC_ILU0)
            cpu.append({"nsolv": nsolv, "n": n, "ms_per_solve": round(1e3 * (time.perf_counter() - t0), 1),
                        "iters": r["iters"]})
        out["cpu_baseline"] = {"unit": "ms per solve", "cores": 1, "kind": "port",
                               "sample": "one solve per option, natural order (the reference's serial loops, "
                                         "ILU0 for BiCGStab/GMRES)", "options": cpu}
    print(json.dumps(out), flush=True)


def inlet_systems(cells: int, seed: int = 11):
    """The u, v and pressure-correction systems of the tidal inlet as the
    oracle's flow step assembles them (natural order): two time steps of one
    outer iteration each from the cold start, then the u system of the next
    step's first outer iteration, the v system of the one after, and the pp
    system of the third."""
    from cms2d_b200 import cases
    from oracle import oracle as O
    case = cases.tidal_inlet(cells, seed=seed)
    f = O.FlowOracle(case)
    f.set_solver(nsolv=3, precond=O.PC_ILU0, tol=1e-6, nswp_pp=200, nswp_uv=200, norm=2)
    f.init()
    for _ in range(2):
        f.step(maxit=1)
    out = {}
    for var, name in ((2, "u"), (3, "v"), (1, "pp")):
        f.capture(var)
        f.step(maxit=1)
        out[name] = (f.captured(), 1.0 if var == 1 else 0.8)
    return case.grid, out


def run_iterations(args):
    """Krylov iteration counts of one solve() per system and preconditioner
    (the report of ILU(0) orderings against the reference's ordering and its
    actual preconditioner): BiCGStab to the reference's stopping test (L1
    ratio 1e-3, pbicgstab.f90:95) and to a 1e-6 relative L2 residual with
    multicolour ILU(0) (GPU), natural-order ILU(0) (GPU and oracle) and ILUTP
    (lfil 35, droptol 1e-3, permtol 0.5: solvers.f90:26-28,195-199, oracle);
    GMRES(3) restarts with ILUTP(lfil 8) at the reference default 1e-3 (oracle);
    and the inner iterations of FP32 + FP64 refinement (reduced inner form) to
    1e-6 L2.  Systems: the solver sweep at 0.25M and 1M unknowns and the
    1M-cell inlet's u, v and pp systems.  --iter-part gpu / cpu runs only the
    GPU or only the oracle columns (the oracle's serial factor and sweeps need
    no GPU; the two halves merge on the system names)."""
    from oracle import oracle as O
    world, rank, local = dist_setup()
    if rank != 0:
        return
    O.set_threads(os.cpu_count())
    systems = []
    for cells in (250_000, 1_000_000):
        g, acoef, ss, sp, phi = build_solve_case(cells, seed=17)
        systems.append((f"sweep {g.ncells}", g, (acoef, ss, sp, phi), 1.0))
    g_in, sy = inlet_systems(args.cells)
    for name in ("u", "v", "pp"):
        (a, b, c, p), relax = sy[name]
        systems.append((f"inlet {g_in.ncells} {name}", g_in, (a, b, c, p), relax))
    rows = []
    do_gpu, do_cpu = args.iter_part in ("all", "gpu"), args.iter_part in ("all", "cpu")
    for label, g, arrs, relax in systems:
        row = {"system": label, "unknowns": g.ncells, "relax": relax}

        def gpu(ordering, tol, norm, precision="fp64"):
            from cms2d_b200 import solver as S
            s = S.Solver(g, ordering=ordering, precision=precision, tol=tol, norm=norm, verify=True, nsolv=3)
            a, b, c, p = [np.array(x, copy=True) for x in arrs]
            info = s.solve(a, b, c, np.zeros_like(b), p, relax=relax, nswp=5000, nsolv=3)
            s.close()
            return info

        def orc(precond, tol, norm, nsolv=3, lfil=None):
            o = O.OracleSolver(g)
            a, b, c, p = [np.array(x, copy=True) for x in arrs]
            t0 = time.perf_counter()
            r = o.solve(a, b, c, np.zeros_like(b), p, relax=relax, nswp=5000, nsolv=nsolv, precond=precond, tol=tol,
                        norm=norm, lfil=lfil)
            return r, time.perf_counter() - t0

        for tag, tol, norm in (("1e-3_L1", 1e-3, 1), ("1e-6_L2", 1e-6, 2)):
            r = {}
            if do_gpu:
                i_mc = gpu("multicolor", tol, norm)
                i_nat = gpu("natural", tol, norm)
                r.update(gpu_multicolour_ilu0=i_mc["iters"], colours=i_mc["ncolors"],
                         gpu_natural_ilu0=i_nat["iters"], levels=i_nat["ncolors"])
            if do_cpu:
                o_nat, t_nat = orc(O.PC_ILU0, tol, norm)
                o_tp, t_tp = orc(O.PC_ILUTP, tol, norm, lfil=35)
                r.update(oracle_natural_ilu0=o_nat["iters"], oracle_ilutp35=o_tp["iters"],
                         oracle_s={"ilu0": round(t_nat, 2), "ilutp35": round(t_tp, 2)})
            row[tag] = r
        if do_cpu:
            o_gm, t_gm = orc(O.PC_ILUTP, 1e-3, 1, nsolv=4, lfil=8)
            row["gmres3_ilutp8_1e-3_restarts"] = o_gm["iters"]
        if do_gpu:
            i_ref = gpu("multicolor", 1e-6, 2, precision="fp32_refine")
            row["fp32_refine_reduced_1e-6_L2"] = {"inner_iters": i_ref["iters"],
                                                  "refine_steps": i_ref["refine_steps"],
                                                  "true_relres": i_ref["true_relres"]}
        rows.append(row)
        print(json.dumps(row), flush=True)
    print(json.dumps({"metric": "Krylov iterations per solve by preconditioner and ordering", "value": None,
                      "unit": "iterations", "rows": rows}), flush=True)


def run_solve_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return
    g, acoef, ss, sp, phi = build_solve_case(args.cells, seed=17)
    for _ in range(args.warmup):
        cpu_baseline(args, g, acoef, ss, sp, phi)
    times = []
    for _ in range(args.steps):
        cb = cpu_baseline(args, g, acoef, ss, sp, phi)
        times.append(1.0 / cb["value"])
    v = args.steps / sum(times)
    out = {"impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": "solves/s",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(1e3 * sum(times) / args.steps, 3), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded solver-sweep system)",
           "config": {"workload": f"pp-system solve, {g.ncells} unknowns, CPU oracle port", "cells": g.ncells},
           "cpu_baseline": {"value": round(v, 4), "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
                            "sample": "full solves of the same system"},
           "e2e": {"value": round(v, 4), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


FLOW_SOLVER = dict(nsolv=3, tol=1e-6, norm=2)

# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one launch
# of the reduced inner BiCGStab kernel on the 999,678-cell inlet flow step:
# the mean over 30 consecutive launches of this workload captured by ncu
# (velocity solves at 130-137 MB each, pressure-correction solves at
# 765-969 MB; replayed from a cold L2).  The kernel's working set (~70 MB)
# stays mostly in the 126 MB L2, so a launch's DRAM traffic is a few reads of
# it, far below its algorithmic bytes.
REDUCED_DRAM_BYTES_PER_LAUNCH = 369_075_183
REDUCED_CAPTURE_CELLS = 999_678


def reduced_traffic(prof, top, unknowns):
    """(DRAM bytes of a captured launch of the top kernel, how obtained), or
    (None, why) when no capture of this kernel on this workload exists."""
    if top != "bicgstab_reduced" or not prof[top]["launches"]:
        return None, "not measured for this kernel"
    if unknowns != REDUCED_CAPTURE_CELLS:
        return None, "captured on the 999,678-cell inlet only"
    return REDUCED_DRAM_BYTES_PER_LAUNCH, (
        "ncu dram__bytes_read.sum + dram__bytes_write.sum of this kernel on this workload, mean of 30 consecutive "
        "launches (velocity and pressure-correction solves; cold L2 under ncu replay): the ~70 MB working set stays "
        "mostly in L2, so a launch's DRAM traffic is far below its algorithmic bytes")


def flow_case(args, seed: int):
    """--case inlet: the telescoping tidal inlet of about --cells cells;
    --case basin: the 200 x 100 Cartesian tidal basin at 20 m;
    --case flat: a Cartesian intertidal flat of about --cells cells at 20 m
    (1.6:1), stepped from 2 h after high water so that cells dry every step."""
    from cms2d_b200 import cases
    if args.case == "basin":
        return cases.tidal_basin(200, 100, 20.0, seed=seed)
    if args.case == "flat":
        ny = max(8, int(round(np.sqrt(args.cells / 1.6))))
        nx = max(8, int(round(args.cells / ny)))
        return cases.tidal_flat(nx, ny, 20.0, seed=seed, dt=300.0, t0_hours=2.0)
    return cases.tidal_inlet(args.cells, seed=seed)


def case_label(case):
    g = case.grid
    if case.name == "tidal_basin":
        return f"Cartesian tidal basin {g.ncells} cells (20 m), dt={case.dt:g} s"
    if case.name == "tidal_flat":
        return (f"Cartesian intertidal flat {g.ncells} cells (20 m), dt={case.dt:g} s, falling tide "
                f"(wetting and drying every step)")
    return f"telescoping tidal inlet {g.ncells} cells (40/20/10 m), dt={case.dt:g} s"


PARITY_FIXTURE = os.path.join(ROOT, "tests", "golden", "inlet_1m_oracle.npz")


def flow_parity(case, seed, settings, precs):
    """Error of the first steps of this workload against the FP64 oracle:
    the committed fixture holds the oracle's water level and velocities
    (natural order, every solve to a 1e-9 relative residual) at seeded
    sample cells after each of its first steps on the same case.  Each
    precision re-runs those steps from the cold start with the bench's own
    settings, and the headline precision once more at the oracle's solver
    tolerance (1e-9 or 600 iterations: the difference that is left is the
    arithmetic's, not the stopping rule's); errors are the largest difference
    over the sample cells and steps relative to the largest oracle value
    (|eta| and |(u, v)|), plus the relative difference of the fixture's
    whole-grid statistics."""
    if not os.path.exists(PARITY_FIXTURE):
        return None
    from cms2d_b200.flow import FlowModel
    z = np.load(PARITY_FIXTURE)
    if int(z["cells"]) != case.grid.ncells or int(z["seed"]) != seed:
        return None
    idx, steps, n = z["sample"], z["eta"].shape[0], case.grid.ncells
    out = {"vs": "FP64 oracle, natural order, solves to 1e-9 or 600 iterations (committed fixture of the same case)",
           "steps": int(steps), "sample_cells": int(idx.size)}
    at_oracle = dict(settings, tol=float(z["tol"]), nswp_pp=int(z["nswp"]), nswp_uv=int(z["nswp"]))
    runs = [(p, p, settings) for p in precs] + [(precs[0] + "_at_oracle_tol", precs[0], at_oracle)]
    for key, prec, sett in runs:
        m = FlowModel(case, precision=prec, **sett)
        m.init()
        e_eta = e_vel = e_stat = 0.0
        niter = []
        for s in range(steps):
            info = m.step()
            niter.append(int(info["niter"]))
            eta, u, v, h = (m.get(k)[:n] for k in ("eta", "u", "v", "h"))
            eo, uo, vo = z["eta"][s], z["u"][s], z["v"][s]
            e_eta = max(e_eta, float(np.abs(eta[idx] - eo).max() / np.abs(eo).max()))
            e_vel = max(e_vel, float(np.hypot(u[idx] - uo, v[idx] - vo).max() / np.hypot(uo, vo).max()))
            st = np.array([eta.mean(), eta.min(), eta.max(), np.sqrt(np.mean(eta * eta)), np.abs(u).max(),
                           np.abs(v).max(), h.sum()])
            so = z["stats"][s]
            e_stat = max(e_stat, float(np.max(np.abs(st - so) / np.maximum(np.abs(so), 1e-30))))
        m.close()
        out[key] = {"eta_max_rel": e_eta, "vel_max_rel": e_vel, "stats_max_rel": e_stat,
                     "eta_max_abs_m": e_eta * float(np.abs(z["eta"]).max()),
                     "outer_iters": niter, "oracle_outer_iters": [int(q) for q in z["niter"]]}
    return out


def other_configs(args, dev, flush):
    """Short measurements of configs 1 and 3 in the default run: the 200 x 100
    Cartesian tidal basin (dt = 600 s) stepped by the GPU in both precisions
    and by the oracle (whole steps, one thread and all cores), and the
    solver-sweep systems at 0.25M and 1M unknowns solved to 1e-6 in both
    precisions (device-resident inputs, L2 flushed before each solve)."""
    import torch
    from cms2d_b200 import cases
    from cms2d_b200 import solver as S
    from cms2d_b200.flow import FlowModel
    from oracle import oracle as O
    out = {}
    basin = cases.tidal_basin(200, 100, 20.0, seed=11)
    c1 = {"workload": f"config 1: Cartesian tidal basin {basin.grid.ncells} cells (20 m), dt=600 s, "
                      f"ILU0-BiCGStab solves to 1e-6 (L2)"}
    for prec in ("fp32_refine", "fp64"):
        m = FlowModel(basin, precision=prec, **dict(FLOW_SOLVER, nswp_pp=args.nswp, nswp_uv=args.nswp))
        m.init()
        for _ in range(3):
            m.step()
        st = torch.cuda.ExternalStream(_lib_stream(m), device=dev)
        ms, nstep = 0.0, 12
        for _ in range(nstep):
            flush.fill_(1.0)
            torch.cuda.synchronize(dev)
            e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st); m.step(); e1.record(st); e1.synchronize()
            ms += e0.elapsed_time(e1)
        c1[prec] = {"timesteps_per_s": round(nstep / (ms / 1e3), 3), "steps": nstep}
        m.close()
    if not args.no_cpu_baseline:
        for th in (1, os.cpu_count()):
            O.set_threads(th)
            f = O.FlowOracle(basin)
            f.set_solver(nsolv=3, precond=O.PC_ILU0, tol=1e-6, nswp_pp=args.nswp, nswp_uv=args.nswp, norm=2)
            f.init()
            f.step()
            t0 = time.perf_counter()
            for _ in range(3):
                f.step()
            c1[f"cpu_{th}_threads"] = {"timesteps_per_s": round(3 / (time.perf_counter() - t0), 3), "steps": 3,
                                        "kind": "port (oracle)"}
    out["config1"] = c1
    c3 = {"workload": "config 3: solver-sweep pressure-correction systems, ILU0-BiCGStab to ||r||2/||r0||2 <= 1e-6"}
    for cells in (250_000, 1_000_000):
        g, acoef, ss, sp, phi = build_solve_case(cells, seed=17)
        ta, tsp, tss0, tph0 = (torch.from_numpy(x).to(dev) for x in (acoef, sp, ss, phi))
        row = {"unknowns": g.ncells}
        for prec in ("fp32_refine", "fp64"):
            s = S.Solver(g, precision=prec, tol=1e-6, norm=2, verify=False, nsolv=3)
            st = torch.cuda.ExternalStream(s.stream_handle, device=dev)
            res = torch.zeros_like(tss0)
            ms, info = 0.0, None
            for q in range(5):
                tss = tss0.clone(); tph = tph0.clone(); flush.fill_(1.0); torch.cuda.synchronize(dev)
                e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
                e0.record(st)
                info = s.solve(ta, tss, tsp, res, tph, relax=1.0, nswp=5000, nsolv=3)
                e1.record(st); e1.synchronize()
                if q >= 2:
                    ms += e0.elapsed_time(e1)
            row[prec] = {"ms_per_solve": round(ms / 3, 3), "iters": info["iters"], "status": info["status"]}
            s.close()
        c3[str(g.ncells)] = row
    out["config3"] = c3
    # config 4 in small: 8 uneven basins of 50k-100k cells in batched launches
    # with graph-replayed stages, against the same members one after another
    from cms2d_b200.ensemble import EnsembleModel
    cs = cases.ensemble_basins(8, seed=23, nmin=50_000, nmax=100_000)
    e = EnsembleModel(cs, **dict(FLOW_SOLVER, nswp_pp=args.nswp, nswp_uv=args.nswp))
    e.init()
    for _ in range(2):
        e.step()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(3):
        e.step()
    torch.cuda.synchronize(dev)
    t_ens = (time.perf_counter() - t0) / 3
    from cms2d_b200 import _lib
    for m in e.members:
        _lib.lib().cms_solver_set_tiles(m.solver_handle, 0)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for m in e.members:
        m.step()
    torch.cuda.synchronize(dev)
    t_seq = time.perf_counter() - t0
    out["config4_small"] = {"workload": f"8 uneven tidal basins, {e.ncells} cells in all (50k-100k each), dt=600 s, "
                                        f"FP32+refine, batched solves, graph-replayed stages (the full config 4 is 64 "
                                        f"basins of 50k-400k)",
                            "member_timesteps_per_s": round(8 / t_ens, 3),
                            "sequential_member_timesteps_per_s": round(8 / t_seq, 3),
                            "timing": "wall clock of 3 ensemble steps after 2 warm-up steps, host synchronised"}
    e.close()
    return out


def _lib_stream(m):
    from cms2d_b200 import _lib
    return _lib.lib().cms_solver_stream(m.solver_handle)


def _profile_read(L, h):
    import ctypes as C
    from cms2d_b200.solver import Solver
    names = Solver.PROFILE_CLASSES
    k = len(names)
    ms = np.zeros(k); by = np.zeros(k); cnt = np.zeros(k, np.int64)
    L.cms_solver_profile_read(h, 1, ms.ctypes.data_as(C.c_void_p), by.ctypes.data_as(C.c_void_p),
                              cnt.ctypes.data_as(C.c_void_p))
    return {nm: {"ms": float(ms[q]), "bytes": float(by[q]), "launches": int(cnt[q])} for q, nm in enumerate(names)}


def run_flow_ours(args):
    import torch
    import torch.distributed as dist
    from cms2d_b200 import _lib
    from cms2d_b200.flow import FlowModel

    world, rank, local = dist_setup()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    L = _lib.lib()
    case = flow_case(args, seed=11 + rank)
    g = case.grid
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2
    settings = dict(FLOW_SOLVER, nswp_pp=args.nswp, nswp_uv=args.nswp, inner_tol=args.inner_tol,
                    inner_max=args.inner_max, multi_kernel=args.multi_kernel, reduced_layout=args.reduced_layout)
    precs = [args.precision]
    if not args.no_companion:
        precs.append("fp64" if args.precision == "fp32_refine" else "fp32_refine")
    res = {}
    for prec in precs:
        m = FlowModel(case, precision=prec, **settings)
        m.init()
        h_solver = m.solver_handle
        stream = torch.cuda.ExternalStream(L.cms_solver_stream(h_solver), device=dev)
        for _ in range(args.warmup):
            m.step()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        launches0 = m.launches
        ms_total = 0.0
        t_wall = 0.0
        infos = []
        # host buffers of the public API: boundary water levels in (pinned),
        # the new water level out; the device time of each step is taken with
        # events on the solver stream, the end-to-end time around the call and
        # the read-back of the result
        wse_h = torch.zeros(case.th_cells.size, dtype=torch.float64).pin_memory().numpy()
        eta_h = torch.zeros(g.ncellsD, dtype=torch.float64).pin_memory().numpy()
        eta_p = eta_h.ctypes.data_as(__import__("ctypes").c_void_p)
        if args.ncu and prec == args.precision:  # the profiler sees the timed steps only
            torch.cuda.profiler.start()
        with ClockSampler(local) as clk:
            for _ in range(args.steps):
                wse_h[:] = case.wsebnd(m.t + case.dt)
                flush.fill_(1.0)
                torch.cuda.synchronize(dev)
                e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
                t0 = time.perf_counter()
                e0.record(stream)
                infos.append(m.step(wsebnd=wse_h))
                e1.record(stream)
                L.cms_flow_get(m._h, 4, eta_p)
                t_wall += time.perf_counter() - t0
                e1.synchronize()
                ms_total += e0.elapsed_time(e1)
        torch.cuda.synchronize(dev)
        if args.ncu and prec == args.precision:
            torch.cuda.profiler.stop()
        launches = m.launches - launches0
        wd_stats = m.wetdry_stats()
        if world > 1:
            t = torch.tensor([ms_total], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_total = float(t.item())
        r = {"ms_per_step": ms_total / args.steps, "value": world * args.steps / (ms_total / 1e3),
             "outer_iters": float(np.mean([i["niter"] for i in infos])),
             "krylov_iters_per_step": float(np.mean([i["krylov_iters"] for i in infos])),
             "status": sorted({i["status"] for i in infos}), "gpu_launches": int(launches),
             "wetdry": {"wet_cells": float(np.mean([i["nwet"] for i in infos])),
                        "cells_changed_per_step": float(np.mean([i["nchanged"] for i in infos])),
                        "host_update": wd_stats},
             "clocks": clk.summary()}
        if world > 1:
            t = torch.tensor([t_wall], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_wall = float(t.item())
        r["e2e"] = {"value": round(world * args.steps / t_wall, 5), "unit": "timesteps/s",
                    "h2d_bytes_per_step": int(wse_h.nbytes), "d2h_bytes_per_step": int(eta_h.nbytes),
                    "ms_per_step": round(1e3 * t_wall / args.steps, 2),
                    "timing": "wall clock around cms_flow_step and the water-level read-back, same steps"}
        if prec == args.precision and not args.ncu:
            # roofline: kernel classes timed with events over K profiled steps
            L.cms_solver_profile(h_solver, 1)
            _profile_read(L, h_solver)
            for _ in range(args.steps):
                flush.fill_(1.0); torch.cuda.synchronize(dev)
                m.step()
            r["profile"] = _profile_read(L, h_solver)
            L.cms_solver_profile(h_solver, 0)
        res[prec] = r
        m.close()
    if args.ncu:
        if world > 1:
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"ncu_pass": True, "ms_per_step": res[args.precision]["ms_per_step"],
                              "gpu_launches": res[args.precision]["gpu_launches"]}), flush=True)
        return
    head = res[args.precision]
    prof = head["profile"]
    peak, peak_kind = _peaks()
    tot = sum(v["ms"] for v in prof.values())
    top = max(prof, key=lambda k: prof[k]["ms"])
    ach = prof[top]["bytes"] / (prof[top]["ms"] / 1e3) / 1e9 if prof[top]["ms"] > 0 else 0.0
    kernels = {k: {"share": round(v["ms"] / tot, 4), "launches": v["launches"],
                   "avg_us": round(1e3 * v["ms"] / v["launches"], 2) if v["launches"] else 0,
                   "GBps": round(v["bytes"] / (v["ms"] / 1e3) / 1e9, 1) if v["ms"] > 0 else 0}
               for k, v in prof.items() if v["launches"]}
    all_bytes = sum(v["bytes"] for v in prof.values())
    traffic, traffic_note = reduced_traffic(prof, top, g.ncells)
    out = {
        "metric": METRIC,
        "value": round(head["value"], 5),
        "unit": "timesteps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(head["ms_per_step"], 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64 refine" if args.precision == "fp32_refine" else "f64",
        "data": f"synthetic (seeded {case.name.replace('_', ' ')})",
        "config": {"workload": f"implicit flow step, {case_label(case)}, "
                               f"ILU0-BiCGStab solves to 1e-6 rel. L2 residual",
                   "cells": g.ncells, "precision": args.precision, "ordering": "multicolor",
                   "solver": "BiCGStab + ILU(0)", "parallelism": f"replicas x{world}",
                   "solver_kernels": "per-phase launches" if args.multi_kernel else "persistent cooperative",
                   "inner_solves": (f"tol {args.inner_tol:g}" if args.inner_tol > 0 else "adaptive tol")
                                   + (f", cap {args.inner_max}" if args.inner_max > 0 else ", cap = remaining budget"),
                   "l2": "flushed between steps (256 MB write)"},
        "outer_iters_per_step": head["outer_iters"],
        "krylov_iters_per_step": head["krylov_iters_per_step"],
        "step_status": head["status"],
        "wetdry": head["wetdry"],
        "cells_steps_per_s": round(head["value"] * g.ncells, 1),
        "e2e": head["e2e"],
        "gpu_launches": head["gpu_launches"],
        "roofline": {"bound": "hbm", "kernel": top, "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(ach / peak, 4), "peak_kind": peak_kind,
                     "traffic": traffic, "traffic_note": traffic_note,
                     "step_GBps": round(all_bytes / (tot / 1e3) / 1e9, 1) if tot else 0},
        "kernels": kernels,
        "clocks": head["clocks"],
    }
    comp = [p for p in precs if p != args.precision]
    if comp:
        c = res[comp[0]]
        out["companion"] = {"precision": comp[0], "value": round(c["value"], 5), "unit": "timesteps/s",
                            "ms_per_step": round(c["ms_per_step"], 3), "outer_iters_per_step": c["outer_iters"],
                            "krylov_iters_per_step": c["krylov_iters_per_step"], "status": c["status"],
                            "speedup_of_headline": round(head["value"] / c["value"], 4)}
    if rank == 0 and not args.no_parity:
        out["parity"] = flow_parity(case, 11 + rank, settings, precs)
    if rank == 0 and world == 1 and not args.no_other_configs and args.case == "inlet":
        out["other_configs"] = other_configs(args, dev, flush)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = flow_cpu_sample(case, head["outer_iters"], args.cpu_outer)
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def flow_cpu_sample(case, outer_per_step, n_outer, threads=None):
    """The flow oracle (the reference's algorithm restated) on the host cores:
    the first n_outer outer iterations of a time step, scaled to a full step."""
    from oracle import oracle as O
    threads = threads or os.cpu_count()
    O.set_threads(threads)
    f = O.FlowOracle(case)
    f.set_solver(nsolv=3, precond=O.PC_ILU0, tol=1e-6, nswp_pp=200, nswp_uv=200, norm=2)
    f.init()
    t0 = time.perf_counter()
    r = f.step(maxit=n_outer)
    dt = time.perf_counter() - t0
    per_outer = dt / max(r["niter"], 1)
    t_step = per_outer * max(outer_per_step, 1.0)
    return {"value": round(1.0 / t_step, 6), "unit": "timesteps/s", "cores": threads, "kind": "port",
            "sample": f"{r['niter']} outer SIMPLEC iterations of time step 1 on the same case ({case.name}, "
                      f"{case.grid.ncells} cells; natural-order ILU0-BiCGStab, serial factor/sweeps as in the "
                      f"reference), "
                      f"{dt:.1f} s, scaled to {outer_per_step:.1f} outer iterations per step",
            "s_per_outer_iter": round(per_outer, 3)}


def run_flow_reference(args):
    """The oracle (the reference's algorithm restated: natural-order ILU(0),
    serial factor and sweeps as in the reference, other loops OpenMP on all
    host cores) on the same case.  Warm-up: W bounded samples of one outer
    iteration each.  Timed: whole time steps, every outer iteration until
    check_conv ends the step, as many as fit in --ref-budget seconds (at least
    one; a step of the 1M inlet takes minutes), reported in "steps"."""
    world, rank, local = dist_setup()
    if rank != 0:
        return
    from oracle import oracle as O
    case = flow_case(args, seed=11)
    threads = os.cpu_count()
    O.set_threads(threads)
    f = O.FlowOracle(case)
    f.set_solver(nsolv=3, precond=O.PC_ILU0, tol=1e-6, nswp_pp=200, nswp_uv=200, norm=2)
    f.init()
    small = case.grid.ncells <= 100_000
    for _ in range(args.warmup):
        f.step() if small else f.step(maxit=1)
    times, outer = [], []
    t_all = time.perf_counter()
    while True:
        t0 = time.perf_counter()
        r = f.step()
        times.append(time.perf_counter() - t0)
        outer.append(r["niter"])
        elapsed = time.perf_counter() - t_all
        if len(times) >= args.steps or elapsed + np.mean(times) > args.ref_budget:
            break
    t_step = float(np.mean(times))
    v = 1.0 / t_step
    # the reference's default thread count is one (NUM_THREADS, flow.F90:98):
    # the same bounded sample (the first 2 outer iterations of a step) on all
    # cores and on one thread, the whole-step time scaled by their ratio
    one = None
    if not small:
        per = {}
        for th in (threads, 1):
            O.set_threads(th)
            t0 = time.perf_counter()
            r1 = f.step(maxit=2)
            per[th] = (time.perf_counter() - t0) / max(r1["niter"], 1)
        ratio = per[1] / per[threads]
        one = {"value": round(v / ratio, 6), "unit": "timesteps/s", "cores": 1,
               "s_per_outer_iter_1": round(per[1], 3), f"s_per_outer_iter_{threads}": round(per[threads], 3),
               "sample": f"the first 2 outer iterations of the next two steps, one on {threads} threads and one on "
                         f"one thread; the measured whole-step rate divided by their time ratio {ratio:.2f} "
                         f"(estimate)"}
        O.set_threads(threads)
    warm = "whole steps" if small else "steps of one outer iteration (untimed)"
    sample = (f"{args.warmup} warm-up {warm}, then {len(times)} whole timed steps (every outer iteration until "
              f"check_conv; {np.mean(outer):.1f} outer iterations per step), {sum(times):.1f} s")
    out = {"impl": "reference", "metric": METRIC, "value": round(v, 6), "unit": "timesteps/s",
           "n_gpus": world, "steps": len(times), "requested_steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(1e3 * t_step, 1), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": f"synthetic (seeded {case.name.replace('_', ' ')})",
           "config": {"workload": f"implicit flow step, {case_label(case)}, ILU0-BiCGStab solves to 1e-6 "
                                  f"rel. L2 residual",
                      "cells": case.grid.ncells, "precision": "fp64", "ordering": "natural",
                      "implementation": "CPU restatement of the reference path (oracle), OpenMP"},
           "outer_iters_per_step": float(np.mean(outer)),
           "cpu_baseline": {"value": round(v, 6), "unit": "timesteps/s", "cores": threads, "kind": "port",
                            "sample": sample},
           "cpu_1thread": one,
           "e2e": {"value": round(v, 6), "unit": "timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def ensemble_cpu_sample(specs, args, nsample: int = 2):
    """Config 4's CPU baseline: the oracle (natural-order ILU(0)-BiCGStab to
    1e-6, serial factor and sweeps, OpenMP elsewhere) steps the nsample
    smallest members one whole step each; their time per cell-step, times the
    cells of all members, estimates the sum of the member times of one
    ensemble step."""
    from cms2d_b200 import cases
    from oracle import oracle as O
    threads = os.cpu_count()
    O.set_threads(threads)
    sizes = [s["nx"] * s["ny"] for s in specs]
    pick = sorted(range(len(specs)), key=lambda k: sizes[k])[:nsample]
    t_cells, t_sec = 0, 0.0
    for c in cases.ensemble_basins(len(specs), seed=23, nmin=args.ens_min, nmax=args.ens_max, members=pick):
        f = O.FlowOracle(c)
        f.set_solver(nsolv=3, precond=O.PC_ILU0, tol=1e-6, nswp_pp=200, nswp_uv=200, norm=2)
        f.init()
        t0 = time.perf_counter()
        f.step()
        t_sec += time.perf_counter() - t0
        t_cells += c.grid.ncells
    per_step = t_sec / t_cells * sum(sizes)
    return {"value": round(len(specs) / per_step, 6), "unit": "member-timesteps/s", "cores": threads, "kind": "port",
            "sample": f"one whole step of each of the {nsample} smallest members ({t_cells} cells, {t_sec:.1f} s), "
                      f"scaled by cells to all {len(specs)} members (estimate of the sum of member times)"}


def run_ensemble_ours(args):
    """Config 4: independent basins of uneven size stepped together, the
    solves of every outer iteration batched into one persistent launch each.
    With N ranks the members are partitioned by LPT on their cell counts
    (each rank builds and steps its share only; no collective until the
    final gather of per-member records)."""
    import torch
    import torch.distributed as dist
    from cms2d_b200 import _lib, cases
    from cms2d_b200.ensemble import EnsembleModel
    from cms2d_b200.partition import gather_results, lpt

    world, rank, local = dist_setup()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    L = _lib.lib()
    t_setup = time.perf_counter()
    if args.members < world:
        raise SystemExit(f"--members {args.members} is smaller than the {world} ranks")
    specs = cases.ensemble_specs(args.members, seed=23, nmin=args.ens_min, nmax=args.ens_max)
    mine = lpt([s["nx"] * s["ny"] for s in specs], world)[rank]
    cs = cases.ensemble_basins(args.members, seed=23, nmin=args.ens_min, nmax=args.ens_max, members=mine)
    e = EnsembleModel(cs, **dict(FLOW_SOLVER, nswp_pp=args.nswp, nswp_uv=args.nswp, inner_tol=args.inner_tol,
                                 inner_max=args.inner_max))
    e.init()
    t_setup = time.perf_counter() - t_setup
    ncells = e.ncells
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    streams = [torch.cuda.ExternalStream(L.cms_solver_stream(m.solver_handle), device=dev) for m in e.members]
    sync = lambda: torch.cuda.synchronize(dev)
    # warm-up: the layout autotuner's trial steps, then the remaining warm-up steps
    e.tune(steps=1, sync=sync)
    nwarm = len(e.tuning["candidates"])
    for _ in range(max(0, args.warmup - nwarm)):
        e.step()
        nwarm += 1
    if world > 1:
        dist.barrier()
    sync()
    ms_total, t_wall, infos = 0.0, 0.0, []
    launches0 = e.launches
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            sync()
            e0 = torch.cuda.Event(enable_timing=True)
            e0.record(streams[0])
            t0 = time.perf_counter()
            infos.append(e.step())
            t_wall += time.perf_counter() - t0
            ends = []
            for st in streams:  # the step has completed on every member stream (host synchronised)
                e1 = torch.cuda.Event(enable_timing=True)
                e1.record(st)
                ends.append(e1)
            for e1 in ends:
                e1.synchronize()
            ms_total += max(e0.elapsed_time(e1) for e1 in ends)
    if world > 1:
        t = torch.tensor([ms_total, t_wall], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total, t_wall = float(t[0]), float(t[1])
    kry = float(np.mean([sum(i["krylov_iters"] for i in step) for step in infos]))
    outer = float(np.mean([np.mean([i["niter"] for i in step]) for step in infos]))
    status = sorted({i["status"] for step in infos for i in step})
    steps_per_s = args.steps / (ms_total / 1e3)
    # per-member records of this rank's share, gathered on every rank
    recs = {k: {"rank": rank, "cells": c.grid.ncells,
                "krylov_iters": int(sum(step[j]["krylov_iters"] for step in infos)),
                "eta_mean": float(np.mean(e.members[j].get("eta")[: c.grid.ncells]))}
            for j, (k, c) in enumerate(zip(mine, cs))}
    allrecs = gather_results(recs)
    tot_cells = int(sum(s["nx"] * s["ny"] for s in specs))
    out = {
        "metric": "member-timesteps/s of a 64-basin ensemble (FP32+refine, batched persistent solves)",
        "value": round(args.members * steps_per_s, 4), "unit": "member-timesteps/s",
        "n_gpus": world, "steps": args.steps, "warmup": nwarm, "ms_per_step": round(ms_total / args.steps, 2),
        "higher_is_better": True, "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
        "dtype": "f32+f64 refine", "data": "synthetic (seeded uneven tidal basins)",
        "config": {"workload": f"ensemble of {args.members} tidal basins, {tot_cells} cells in all, "
                               f"dt=600 s, ILU0-BiCGStab solves to 1e-6",
                   "members": args.members, "cells": tot_cells, "layout_blocks": int(e.tiles()[0]),
                   "autotuner": e.tuning,
                   "parallelism": f"members partitioned over {world} ranks by LPT on cells (rank 0: "
                                  f"{len(mine)} members, {ncells} cells)" if world > 1 else "one GPU",
                   "l2": "flushed between steps (256 MB write)"},
        "cells_steps_per_s": round(tot_cells * steps_per_s, 1),
        "krylov_iters_per_step": kry, "outer_iters_per_step": outer, "step_status": status,
        "members_gathered": len(allrecs),
        "batched_launches_per_step": (e.launches - launches0) / args.steps,
        "e2e": {"value": round(args.members * args.steps / t_wall, 4), "unit": "member-timesteps/s",
                "h2d_bytes_per_step": int(sum(c.th_cells.size for c in cs) * 8), "d2h_bytes_per_step": 0},
        "gpu_launches": int(sum(m.launches for m in e.members)),
        "setup_s": round(t_setup, 1),
        "device_gb": round(sum(m.device_bytes for m in e.members) / 1e9, 2),
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = ensemble_cpu_sample(specs, args)
    if args.ens_sequential and world == 1:
        # the same members stepped one after another with their own solver launches
        for m in e.members:  # each member's solver on the whole GPU again
            L.cms_solver_set_tiles(m.solver_handle, 0)
        t0 = time.perf_counter()
        for m in e.members:
            m.step()
        sync()
        out["sequential_member_steps_per_s"] = round(args.members / (time.perf_counter() - t0), 4)
        out["sequential"] = "one step of each member after the timed steps, members one after another"
    if world > 1:
        dist.destroy_process_group()
    e.close()
    if rank == 0:
        print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="flow", choices=["flow", "solve", "ensemble", "solvers", "iterations"])
    ap.add_argument("--members", type=int, default=64, help="ensemble: basins")
    ap.add_argument("--ens-min", type=int, default=50_000, help="ensemble: smallest basin (cells)")
    ap.add_argument("--ens-max", type=int, default=400_000, help="ensemble: largest basin (cells)")
    ap.add_argument("--ens-sequential", action="store_true",
                    help="ensemble: also time one step of the members one after another")
    ap.add_argument("--nswp", type=int, default=200, help="iteration cap of each flow solve")
    ap.add_argument("--no-companion", action="store_true", help="flow: skip the other-precision run")
    ap.add_argument("--cpu-outer", type=int, default=3, help="flow CPU sample: outer iterations timed")
    ap.add_argument("--cells", type=int, default=1_000_000)
    ap.add_argument("--case", default="inlet", choices=["inlet", "basin", "flat"],
                    help="flow workload: 1M telescoping inlet (default), the 200x100 basin or an intertidal flat")
    ap.add_argument("--precision", default="fp32_refine", choices=["fp32_refine", "fp64"])
    ap.add_argument("--inner-tol", type=float, default=0.0,
                    help="refinement: relative residual reduction asked of each FP32 inner solve "
                         "(0: adaptive, cms_solver_opts.inner_tol)")
    ap.add_argument("--inner-max", type=int, default=0,
                    help="refinement: iteration cap of each FP32 inner solve (0: the solve's remaining budget)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="flow: skip the error check against the oracle fixture")
    ap.add_argument("--no-other-configs", action="store_true",
                    help="flow: skip the short config 1 and config 3 measurements")
    ap.add_argument("--iter-part", default="all", choices=["all", "gpu", "cpu"],
                    help="iterations workload: the GPU columns, the oracle columns, or both")
    ap.add_argument("--ref-budget", type=float, default=400.0,
                    help="reference arm: seconds of whole timed CPU steps (at least one step)")
    ap.add_argument("--ncu", action="store_true", help="warm-up and timed steps only (profiler runs)")
    ap.add_argument("--reduced-layout", type=int, default=0,
                    help="threads x rows layout and form of the reduced inner solve (0 auto, 1-7; cms_solver_opts.reduced_layout)")
    ap.add_argument("--multi-kernel", action="store_true",
                    help="BiCGStab as one launch per phase instead of one persistent launch per solve")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "iterations":
        if args.impl != "reference":
            run_iterations(args)
        return
    if args.workload == "solvers":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the solvers workload reports its CPU arm "
                                                                  "in its own line (cpu_baseline)"}))
            return
        run_solvers_ours(args)
    elif args.workload == "ensemble":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the ensemble workload has no CPU arm"}))
            return
        run_ensemble_ours(args)
    elif args.workload == "flow":
        (run_flow_reference if args.impl == "reference" else run_flow_ours)(args)
    else:
        (run_solve_reference if args.impl == "reference" else run_solve_ours)(args)


if __name__ == "__main__":
    main()
