"""Benchmark: multigrid-preconditioned GMRES solve of the 3D 64^3 Q1
variable-coefficient diffusion problem (274,625 DoFs) to a true relative
residual of 1e-8, on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one complete solve from x = 0 (mixed precision: FP32 V(2,2)-Jacobi
multigrid cycle inside FP64 flexible GMRES with refinement). The FP64 variant
(same kernels, FP64 cycle) and the reference-semantics left-preconditioned FP64
GMRES are timed beside it and reported as extra keys. Inputs are synthetic and
seeded: kappa = exp(N(0,1)) per cell (seed 1001), f ~ U[-1,1] per node (seed
1002), assembled like the reference's CGDisc Q1 (checked by the tests).

Multi-GPU: the path does not shard on one problem in this build (replicas
only): each rank solves its own copy; value = DoFs solved by all ranks / max
over ranks of the device time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solve DoF/s to 1e-8 rel. residual, mixed vs FP64 on GPU; SpMV % of HBM peak"
WORKLOAD = ("3D scalar diffusion -div(kappa grad u)=f, unit cube, Q1 hex 64^3 cells "
            "(274,625 DoFs), kappa log-normal per cell (mu 0, sigma 1, seed 1001), "
            "f~U[-1,1] per node (seed 1002); 6-level V(2,2) damped Jacobi (omega 0.8) "
            "multigrid preconditioning GMRES(20), tol 1e-8")
DIM, COARSE, REFINE = 3, 1, 6
PARAMS = dict(iterpre=2, iterpost=2, iterexact=10, omega=0.8, mgomega=1.0, mgtype="V",
              gmressize=21, tol=1e-8, globaltol=1e-300, maxiter=200)


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                r = subprocess.run(["nvidia-smi", "-i", str(self.index),
                                    f"--query-gpu={self.Q}", "--format=csv,noheader,nounits"],
                                   capture_output=True, text=True, timeout=5)
                if r.returncode == 0 and r.stdout.strip():
                    self.samples.append([x.strip() for x in r.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 3 + i and s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def cpu_baseline(kappa_rhs, ndof, threads):
    """The reference's own FP64 CPU solver (compiled from its sources into
    oracle/_ref) on the same workload; one bounded sample (one mesh build +
    assembly, then `repeat` solves). Falls back to the C restatement."""
    from oracle.oracle import REF_HARNESS, Oracle, run_reference, write_inputs
    kappa, rhs = kappa_rhs
    if os.path.exists(REF_HARNESS):
        d = tempfile.mkdtemp(prefix="gb_cpu_")
        env_threads = os.environ.get("OMP_NUM_THREADS")
        os.environ["OMP_NUM_THREADS"] = str(threads)
        try:
            t0 = time.time()
            out, s = run_reference(d, dim=DIM, coarse=COARSE, refine=REFINE, repeat=3,
                                   tol=1e-8, globaltol=1e-16, gmressize=21, iterpre=2,
                                   iterpost=2, omega=0.8, **write_inputs(d, kappa, rhs))
            wall = time.time() - t0
        finally:
            if env_threads is None:
                os.environ.pop("OMP_NUM_THREADS", None)
            else:
                os.environ["OMP_NUM_THREADS"] = env_threads
        times = [float(t) for t in s["solve_s"]]
        med = statistics.median(times)
        return {"value": ndof / med, "unit": "DoF/s", "cores": threads, "kind": "reference",
                "sample": (f"reference CPU StdMultiLevelSolver GMRES+V-cycle on the same "
                           f"64^3 problem, median of {len(times)} solves after assembly "
                           f"({med:.3f} s/solve, {s['iterations'][0]} iterations, true rel "
                           f"residual {float(s['true_rel_residual'][0]):.2e}; "
                           f"harness wall {wall:.1f} s incl. mesh+assembly)"),
                "solve_s": med, "iterations": int(s["iterations"][0]),
                "assemble_s": float(s["assemble_s"][0]) if "assemble_s" in s else None}
    from gascoignelib_b200.problem import structured_problem
    P = structured_problem(DIM, COARSE, REFINE, kappa, rhs)
    O = Oracle(P)
    t0 = time.time()
    x, info = O.gmres(vmax=21, tol=1e-8)
    dt = time.time() - t0
    return {"value": ndof / dt, "unit": "DoF/s", "cores": 1, "kind": "port",
            "sample": f"oracle C restatement, one solve ({dt:.2f} s, {info['iterations']} it)",
            "solve_s": dt, "iterations": info["iterations"]}


def run_reference_arm(args, world, rank):
    from gascoignelib_b200.problem import seeded_inputs
    if rank != 0:
        return
    kappa, rhs = seeded_inputs(DIM, COARSE, REFINE)
    ndof = (((COARSE << REFINE) + 1) ** DIM)
    threads = os.cpu_count() or 1
    from oracle.oracle import REF_HARNESS, run_reference, write_inputs
    line = {"metric": METRIC, "impl": "reference", "unit": "DoF/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "precision": "fp64 (reference CPU)"}}
    if not os.path.exists(REF_HARNESS):
        # oracle port: the C restatement, single thread
        cb = cpu_baseline((kappa, rhs), ndof, threads)
        line.update(value=cb["value"], ms_per_step=1e3 * cb["solve_s"], cpu_baseline=cb,
                    e2e={"value": cb["value"], "unit": "DoF/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0})
        print(json.dumps(line))
        return
    d = tempfile.mkdtemp(prefix="gb_refarm_")
    os.environ["OMP_NUM_THREADS"] = str(threads)
    out, s = run_reference(d, dim=DIM, coarse=COARSE, refine=REFINE,
                           repeat=args.warmup + args.steps, tol=1e-8, globaltol=1e-16,
                           gmressize=21, iterpre=2, iterpost=2, omega=0.8,
                           **write_inputs(d, kappa, rhs))
    times = [float(t) for t in s["solve_s"]][args.warmup:]
    tot = sum(times)
    value = ndof * len(times) / tot
    line.update(value=value, ms_per_step=1e3 * tot / len(times),
                cpu_baseline={"value": value, "unit": "DoF/s", "cores": threads,
                              "kind": "reference",
                              "sample": f"{len(times)} timed solves after {args.warmup} "
                                        f"warm-up, {s['iterations'][0]} iterations, true "
                                        f"rel residual {float(s['true_rel_residual'][0]):.2e}"},
                e2e={"value": value, "unit": "DoF/s", "h2d_bytes_per_step": 0,
                     "d2h_bytes_per_step": 0})
    print(json.dumps(line))


def assembly_leg(c, P, kappa, steps, warmup, flush, dev):
    """Device assembly of every level from the finest level's kappa (a CUDA
    tensor): element matrices, their sum into the SELL values (FP64 + FP32),
    Dirichlet rows/columns, block-diagonal inverse, kappa coarsening. Device
    time with CUDA events on the solver's stream, L2 flushed before each."""
    import torch

    from gascoignelib_b200.problem import structured_meshes

    for l, (cells, coord, par) in enumerate(structured_meshes(P)):
        c.set_mesh(l, P.dim, cells, coord, par)
    kd = torch.tensor(kappa, dtype=torch.float64, device=dev)
    st = torch.cuda.ExternalStream(c.stream(), device=dev)
    for _ in range(warmup):
        c.assemble_levels(kd)
    ms = []
    for _ in range(steps):
        flush.random_(0, 255)
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        c.assemble_levels(kd)
        e1.record(st)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    # algorithmic bytes: per cell 2^d node indices, kappa, element matrix
    # written and read back, its entry list; per stored entry column, entry
    # pointer, FP64 + FP32 value; per row mask, diagonal, inverse (FP64 + FP32)
    nl = 1 << P.dim
    by = 0
    for L in P.levels:
        nc = (round(L.n ** (1.0 / P.dim)) - 1) ** P.dim
        by += nc * (4 * nl + 8 + 2 * 8 * nl * nl + 4 * nl * nl)
        by += L.val.size * (4 + 4 + 8 + 4) + L.n * (1 + 4 + 8 + 8 + 8 + 4 + 8 * P.dim)
    t = sorted(ms)[len(ms) // 2]
    # matrix-free Newton residual y = b - Form(x) on the finest level (max-norm
    # read back), against the assembled matrix's residual SpMV beside it
    import numpy as np
    fl = P.nlevels - 1
    x, b, y = c.vec(), c.vec(), c.vec()
    c.upload(fl, x, np.random.default_rng(7).uniform(-1.0, 1.0, P.finest.ndof))
    c.upload(fl, b, P.rhs)
    for _ in range(warmup):
        c.newton_residual(y, x, b)
    msr = []
    for _ in range(steps):
        flush.random_(0, 255)
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        c.newton_residual(y, x, b)
        e1.record(st)
        e1.synchronize()
        msr.append(e0.elapsed_time(e1))
    for v in (x, b, y):
        c.free(v)
    return {"ms": t, "levels": P.nlevels, "cells_finest": int(nc),
            "algorithmic_bytes": by, "achieved_gbs": by / (t * 1e-3) / 1e9,
            "newton_residual_ms": sorted(msr)[len(msr) // 2]}


def adjoint_c5(local, steps, warmup, flush):
    """Forward + adjoint + coefficient gradient at 96^3 cells (912,673 dofs):
    mixed forward solve, J = int u^2 and dJ/du = 2 M u on the device, mixed
    adjoint solve, per-cell dJ/dkappa. Device time with CUDA events on the
    solver's stream, L2 flushed before every step."""
    import numpy as np
    import torch

    from gascoignelib_b200.native import GB_FP32, Context
    from gascoignelib_b200.problem import seeded_inputs, structured_problem

    kappa, rhs = seeded_inputs(3, 3, 5)
    P = structured_problem(3, 3, 5, kappa, rhs)
    c = Context(local)
    c.load_problem(P)
    c.set_params(**PARAMS)
    l = P.nlevels - 1
    u, b, g, lam = c.vec(), c.vec(), c.vec(), c.vec()
    c.upload(l, b, P.rhs)
    dev = torch.device(f"cuda:{local}")
    st = torch.cuda.ExternalStream(c.stream(), device=dev)
    out = {}

    def step():
        fi = c.fgmres(u, b, GB_FP32)
        c.functional(l, u, g, read=False)
        ai = c.adjoint_fgmres(lam, g, GB_FP32)
        c.coeff_gradient(l, u, lam, download=False)
        return fi, ai

    for _ in range(warmup):
        step()
    ms = []
    for _ in range(steps):
        flush.random_(0, 255)
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fi, ai = step()
        e1.record(st)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    J = c.functional(l, u, g)
    grad = c.coeff_gradient(l, u, lam)
    t = sum(ms) / len(ms)
    # one design step with a new kappa: device assembly of all levels, then
    # the same forward + adjoint + gradient
    asm = assembly_leg(c, P, kappa, steps, warmup, flush, dev)
    kd = torch.tensor(kappa, dtype=torch.float64, device=dev)
    for _ in range(warmup):
        c.assemble_levels(kd)
        step()
    ms2 = []
    for _ in range(steps):
        flush.random_(0, 255)
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        c.assemble_levels(kd)
        step()
        e1.record(st)
        e1.synchronize()
        ms2.append(e0.elapsed_time(e1))
    asm["assemble_forward_adjoint_gradient_ms"] = sum(ms2) / len(ms2)
    out = {"workload": "3D diffusion, kappa = exp(N(0,1)) per cell, 96^3 Q1 cells, "
                       "J = int u^2: forward solve + dJ/du + adjoint solve + dJ/dkappa",
           "dofs": P.finest.ndof, "cells": P.cells.ncells, "ms_per_step": t,
           "value": P.finest.ndof / (t * 1e-3), "unit": "DoF/s (forward+adjoint+gradient)",
           "forward": {"ms": fi["device_ms"], "iterations": fi["iterations"],
                       "true_rel_residual": fi["true_rel_residual"]},
           "adjoint": {"ms": ai["device_ms"], "iterations": ai["iterations"],
                       "true_rel_residual": ai["true_rel_residual"]},
           "J": J, "grad_norm": float(np.linalg.norm(grad)),
           "assembly": asm,
           "l2": "flushed (256 MB write) before every step"}
    c.close()
    return out


def stokes_c3(local, steps, warmup, flush):
    """C3: 2D Q1/Q1 Stokes on 512^2 cells (789,507 dofs, ncomp 3), Vanka
    V(2,2) smoother with the pressure filter, GMRES(30) to 1e-8: mixed
    (FP32 Vanka cycle in FP64 flexible GMRES) and FP64 solves, device time
    with the L2 flushed before every solve; and the finest-level Vanka local
    solve timed alone (its LU factors dominate the traffic)."""
    import torch

    from gascoignelib_b200.native import GB_FP32, GB_FP64, Context
    from gascoignelib_b200.problem import structured_stokes

    P = structured_stokes(2, 2, 8)
    c = Context(local)
    c.load_problem(P)
    c.set_params(iterpre=2, iterpost=2, iterexact=10, omega=1.0, mgomega=1.0,
                 mgtype="V", gmressize=31, tol=1e-8, globaltol=1e-300, maxiter=300)
    l = P.nlevels - 1
    x, b = c.vec(), c.vec()
    c.upload(l, b, P.rhs)
    out = {}
    for name, prec in (("mixed", GB_FP32), ("fp64", GB_FP64)):
        for _ in range(warmup):
            c.fgmres(x, b, prec)
        ms = []
        for _ in range(steps):
            flush.random_(0, 255)
            torch.cuda.synchronize()
            info = c.fgmres(x, b, prec)
            ms.append(info["device_ms"])
        t = sum(ms) / len(ms)
        out[name] = {"value": P.finest.ndof / (t * 1e-3), "unit": "DoF/s",
                     "ms_per_step": t, "iterations": info["iterations"],
                     "restarts": info["restarts"],
                     "true_rel_residual": info["true_rel_residual"]}
    c.close()
    # the 12 x 12 variant: Vanka on single cells (4 nodes x 3 components)
    Pc = structured_stokes(2, 2, 8, patches="cell")
    c = Context(local)
    c.load_problem(Pc)
    c.set_params(iterpre=2, iterpost=2, iterexact=10, omega=1.0, mgomega=1.0,
                 mgtype="V", gmressize=31, tol=1e-8, globaltol=1e-300, maxiter=300)
    x, b = c.vec(), c.vec()
    c.upload(l, b, Pc.rhs)
    for _ in range(warmup):
        c.fgmres(x, b, GB_FP32)
    ms = []
    for _ in range(steps):
        flush.random_(0, 255)
        torch.cuda.synchronize()
        info = c.fgmres(x, b, GB_FP32)
        ms.append(info["device_ms"])
    t = sum(ms) / len(ms)
    out["mixed_cell_patches_12x12"] = {
        "value": Pc.finest.ndof / (t * 1e-3), "unit": "DoF/s", "ms_per_step": t,
        "iterations": info["iterations"], "true_rel_residual": info["true_rel_residual"]}
    c.close()
    out["workload"] = ("2D Stokes Q1/Q1 (Brezzi-Pitkaranta), 512^2 cells, 789,507 dofs, "
                       "Vanka 3x3-node patches (27x27 local systems), pressure filter, "
                       "V(2,2), GMRES(30), tol 1e-8; 12x12 variant: single-cell patches")
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def ilu_c2(local, P, steps, warmup, flush, threads, with_ref):
    """The C2 solve with the block ILU smoother (linear_smooth ilu, omega 1):
    mixed and FP64 flexible solves, device time, L2 flushed; and, when asked,
    the reference's own CPU solve with its SparseBlockIlu on the same problem
    (the harness's identity ILU order)."""
    import torch

    from gascoignelib_b200.native import GB_FP32, GB_FP64, Context

    c = Context(local)
    c.load_problem(P)
    c.set_params(**dict(PARAMS, smoother="ilu", omega=1.0))
    l = P.nlevels - 1
    x, b = c.vec(), c.vec()
    c.upload(l, b, P.rhs)
    out = {"workload": "C2 (3D Q1 64^3, log-normal kappa) with linear_smooth ilu, omega 1"}
    for name, prec in (("mixed", GB_FP32), ("fp64", GB_FP64)):
        for _ in range(warmup):
            c.fgmres(x, b, prec, check=False)
        ms = []
        for _ in range(steps):
            flush.random_(0, 255)
            torch.cuda.synchronize()
            info = c.fgmres(x, b, prec, check=False)
            ms.append(info["device_ms"])
        t = sum(ms) / len(ms)
        out[name] = {"value": P.finest.ndof / (t * 1e-3), "unit": "DoF/s", "ms_per_step": t,
                     "iterations": info["iterations"],
                     "true_rel_residual": info["true_rel_residual"],
                     "kernel_launches": info["kernel_launches"]}
    c.close()
    if with_ref:
        from oracle.oracle import REF_HARNESS, run_reference, write_inputs
        if os.path.exists(REF_HARNESS):
            from gascoignelib_b200.problem import seeded_inputs
            kappa, rhs = seeded_inputs(DIM, COARSE, REFINE)
            d = tempfile.mkdtemp(prefix="gb_ilu_")
            env = os.environ.get("OMP_NUM_THREADS")
            os.environ["OMP_NUM_THREADS"] = str(threads)
            try:
                _, s = run_reference(d, dim=DIM, coarse=COARSE, refine=REFINE, repeat=1,
                                     tol=1e-8, globaltol=1e-16, gmressize=21, iterpre=2,
                                     iterpost=2, omega=1.0, smoother="ilu",
                                     **write_inputs(d, kappa, rhs))
            finally:
                if env is None:
                    os.environ.pop("OMP_NUM_THREADS", None)
                else:
                    os.environ["OMP_NUM_THREADS"] = env
            out["reference_cpu"] = {"solve_s": float(s["solve_s"][0]),
                                    "iterations": int(s["iterations"][0]),
                                    "cores": threads}
    return out


def q2_c4(local, steps, warmup, flush):
    """C4: 3D CGQ2 convection-diffusion -0.01 Laplace u + (1, 0.5, 0.25) .
    grad u = f on 80^3 cells (40^3 Q2 patches, 531,441 dofs), refined once more
    inside the ball |x - 0.5| < 0.25 (patches whose centre is inside: 779,481
    dofs, 22,752 hanging nodes on edges and faces, 47.6 M matrix entries, rows
    of up to 125), five levels, Jacobi V(2,2) with omega 0.3 (0.5 and above
    stall on this convection-dominated Q2 operator), GMRES(30) to 1e-8: mixed
    and FP64 solves, device time, L2 flushed before every solve. The same solve
    without the ball (531,441 dofs, four levels) is reported beside it."""
    import torch

    from gascoignelib_b200.native import GB_FP32, GB_FP64, Context
    from gascoignelib_b200.problem import q2_meshes, structured_q2, structured_q2_ball

    def run(P):
        c = Context(local)
        c.load_problem(P)
        c.set_params(iterpre=2, iterpost=2, iterexact=10, omega=0.3, mgomega=1.0,
                     mgtype="V", gmressize=31, tol=1e-8, globaltol=1e-300, maxiter=600)
        l = P.nlevels - 1
        x, b = c.vec(), c.vec()
        c.upload(l, b, P.rhs)
        res = {}
        for name, prec in (("mixed", GB_FP32), ("fp64", GB_FP64)):
            for _ in range(warmup):
                c.fgmres(x, b, prec, check=False)
            ms = []
            for _ in range(steps):
                flush.random_(0, 255)
                torch.cuda.synchronize()
                info = c.fgmres(x, b, prec, check=False)
                ms.append(info["device_ms"])
            t = sum(ms) / len(ms)
            res[name] = {"value": P.finest.ndof / (t * 1e-3), "unit": "DoF/s",
                         "ms_per_step": t, "iterations": info["iterations"],
                         "restarts": info["restarts"], "status": info["status_name"],
                         "true_rel_residual": info["true_rel_residual"]}
        c.close()
        res["mixed_over_fp64"] = res["mixed"]["value"] / res["fp64"]["value"]
        return res

    def assembly_ms(P):
        """Median device time of assembling every level (Q2 elements, the
        finest level's hanging nodes condensed) from a per-element
        coefficient, L2 flushed before each."""
        c = Context(local)
        c.load_problem(P)
        meshes = q2_meshes(P)
        for l, (el, par) in enumerate(meshes):
            c.set_mesh(l, 3, el, P.levels[l].coord, par, degree=2)
        dev = torch.device(f"cuda:{local}")
        kd = torch.full((meshes[-1][0].shape[0],), 1e-2, dtype=torch.float64, device=dev)
        st = torch.cuda.ExternalStream(c.stream(), device=dev)
        for _ in range(warmup):
            c.assemble_levels(kd, (1.0, 0.5, 0.25))
        ms = []
        for _ in range(steps):
            flush.random_(0, 255)
            torch.cuda.synchronize(dev)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            c.assemble_levels(kd, (1.0, 0.5, 0.25))
            e1.record(st)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        c.close()
        return sorted(ms)[len(ms) // 2]

    P = structured_q2_ball(5, 4, eps=1e-2, beta=(1.0, 0.5, 0.25), radius=0.25)
    out = run(P)
    out["workload"] = ("3D CGQ2 convection-diffusion eps 1e-2, beta (1,0.5,0.25), 80^3 cells "
                       "refined once inside |x-0.5|<0.25, %d dofs, %d hanging, 5 levels, "
                       "Jacobi V(2,2) omega 0.3, GMRES(30), tol 1e-8"
                       % (P.finest.ndof, P.info["hanging"]))
    # device assembly of the ball hierarchy (5 levels; 93,568 elements of 27
    # nodes on the finest, 6,896 of them with hanging nodes condensed)
    out["assembly_ms"] = assembly_ms(P)
    del P
    U = structured_q2(3, 5, 4, eps=1e-2, beta=(1.0, 0.5, 0.25))
    out["uniform_no_ball"] = run(U)
    out["uniform_no_ball"]["workload"] = "the same on the uniform 80^3 cells, 531,441 dofs"
    # device assembly of the uniform Q2 hierarchy (4 levels, 40^3 elements of
    # 27 nodes on the finest)
    out["uniform_no_ball"]["assembly_ms"] = assembly_ms(U)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the 96^3 forward+adjoint+gradient measurement")
    ap.add_argument("--no-stokes", action="store_true",
                    help="skip the 512^2 Stokes/Vanka measurement")
    ap.add_argument("--no-q2", action="store_true",
                    help="skip the 80^3 Q2 convection-diffusion measurement")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        return

    import numpy as np
    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from gascoignelib_b200.build import build_library
    from gascoignelib_b200.native import GB_FP32, GB_FP64, Context
    from gascoignelib_b200.problem import seeded_inputs, structured_problem

    if rank == 0:
        build_library()
    if dist:
        dist.barrier()
    kappa, rhs = seeded_inputs(DIM, COARSE, REFINE)
    P = structured_problem(DIM, COARSE, REFINE, kappa, rhs)
    ndof = P.finest.ndof
    ctx = Context(local)
    ctx.load_problem(P)
    ctx.set_params(**PARAMS)
    fl = P.nlevels - 1
    xv, bv = ctx.vec(), ctx.vec()
    ctx.upload(fl, bv, P.rhs)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def run_steps(prec, k, timed):
        ms, infos = [], []
        for _ in range(k):
            flush.random_(0, 255)            # L2 (126 MB) flush between steps
            torch.cuda.synchronize()
            info = ctx.fgmres(xv, bv, prec) if prec is not None else ctx.gmres(xv, bv)
            ms.append(info["device_ms"])
            infos.append(info)
        return ms, infos

    # warm-up
    run_steps(GB_FP32, args.warmup, False)
    run_steps(GB_FP64, max(1, args.warmup // 2), False)
    run_steps(None, 1, False)

    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    k0 = ctx.kernel_count()
    with ClockSampler(local) as clk:
        ms32, info32 = run_steps(GB_FP32, args.steps, True)
    launches = ctx.kernel_count() - k0
    ms64, info64 = run_steps(GB_FP64, args.steps, True)
    msleft, infoleft = run_steps(None, args.steps, True)
    torch.cuda.synchronize()

    t32 = sum(ms32)
    tmax = t32
    if dist:
        t = torch.tensor([t32], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tmax = float(t.item())
    value = ndof * args.steps * world / (tmax / 1e3)
    v64 = ndof * args.steps / (sum(ms64) / 1e3)
    vleft = ndof * args.steps / (sum(msleft) / 1e3)

    # e2e: the C-ABI call with host buffers (pinned), H2D + solve + D2H timed
    b_host = torch.from_numpy(P.rhs.copy()).pin_memory()
    x_host = torch.empty_like(b_host).pin_memory()
    e2e_ms = []
    for _ in range(args.steps):
        flush.random_(0, 255)
        torch.cuda.synchronize()
        bn = b_host.numpy()
        xn = x_host.numpy()
        _, info = ctx.solve_host(bn, method=2, out=xn)
        e2e_ms.append(info["device_ms"])
    e2e_val = ndof * args.steps * world / (sum(e2e_ms) / 1e3)

    # roofline: finest-level SpMV timed alone (CUDA events on the solver's
    # stream), the L2 emptied before each launch by reading a 256 MB buffer
    # (a write flush would leave dirty lines whose write-back the SpMV pays;
    # that figure is reported too)
    peak, peak_kind = _peaks()
    spmv_ms64, spmv_b64 = ctx.bench_spmv(fl, GB_FP64, reps=20, flush_l2=2)
    spmv_ms32, spmv_b32 = ctx.bench_spmv(fl, GB_FP32, reps=20, flush_l2=2)
    spmv_ms64w, _ = ctx.bench_spmv(fl, GB_FP64, reps=20, flush_l2=1)
    ach64 = spmv_b64 / (spmv_ms64 * 1e-3) / 1e9
    ach32 = spmv_b32 / (spmv_ms32 * 1e-3) / 1e9
    prof = {}
    pj = os.path.join(ROOT, "profiles", "spmv_fp64_c2_finest.json")
    if os.path.exists(pj):
        prof = json.load(open(pj))

    asm = assembly_leg(ctx, P, kappa, min(args.steps, 5), 2, flush, torch.device(f"cuda:{local}"))

    adj = None
    if not args.no_adjoint:
        adj = adjoint_c5(local, min(args.steps, 5), 2, flush)
    stk = None
    if not args.no_stokes:
        stk = stokes_c3(local, min(args.steps, 5), 2, flush)
    q2 = None
    if not args.no_q2:
        q2 = q2_c4(local, min(args.steps, 3), 1, flush)
    ilu = ilu_c2(local, P, min(args.steps, 3), 1, flush, os.cpu_count() or 1,
                 rank == 0 and not args.no_cpu_baseline)

    if rank == 0:
        cb = None
        if not args.no_cpu_baseline:
            cb = cpu_baseline((kappa, rhs), ndof, os.cpu_count() or 1)
        i32 = info32[-1]
        line = {
            "metric": METRIC, "value": value, "unit": "DoF/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": tmax / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 cycle / f64 outer",
            "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "dofs": ndof, "levels": P.nlevels,
                       "nnz_finest": int(P.finest.nnzb), "parallelism": f"replicas x{world}",
                       "l2": "flushed (256 MB write) before every step",
                       "precision": "FP32 V-cycle in FP64 flexible GMRES + refinement"},
            "fp64": {"value": v64, "unit": "DoF/s", "ms_per_step": sum(ms64) / args.steps,
                     "iterations": info64[-1]["iterations"],
                     "true_rel_residual": info64[-1]["true_rel_residual"]},
            "mixed_over_fp64": value / world / v64,
            "reference_semantics_fp64_left_gmres": {
                "value": vleft, "unit": "DoF/s", "ms_per_step": sum(msleft) / args.steps,
                "iterations": infoleft[-1]["iterations"],
                "true_rel_residual": infoleft[-1]["true_rel_residual"]},
            "iterations": i32["iterations"], "restarts": i32["restarts"],
            "true_rel_residual": i32["true_rel_residual"],
            "e2e": {"value": e2e_val, "unit": "DoF/s",
                    "h2d_bytes_per_step": ndof * 8, "d2h_bytes_per_step": ndof * 8},
            "roofline": {"bound": "hbm", "kernel": "k_spmv<kAx,double> finest level",
                         "achieved": ach64, "peak": peak, "unit": "GB/s",
                         "frac": ach64 / peak,
                         "traffic": prof.get("traffic_bytes"),
                         "peak_kind": peak_kind + " (burst copy)",
                         "ms_per_launch": spmv_ms64, "algorithmic_bytes": spmv_b64,
                         "ms_per_launch_write_flush": spmv_ms64w,
                         "ncu_duration_us": prof.get("ncu_duration_us"),
                         "traffic_source": "profiles/spmv_fp64_c2_finest.md (ncu)",
                         "fp32": {"achieved": ach32, "frac": ach32 / peak,
                                  "ms_per_launch": spmv_ms32,
                                  "algorithmic_bytes": spmv_b32}},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "cpu_baseline": cb,
            "assembly_c2": dict(asm, workload="Q1 matrices of all 6 levels of the 64^3 "
                                "problem from the per-cell kappa (device)",
                                reference_cpu_s=(cb or {}).get("assemble_s"),
                                reference_cpu_note="reference AssembleMatrix + ComputeIlu "
                                "on all levels, host threads as cpu_baseline.cores"),
            "adjoint_c5": adj,
            "stokes_c3": stk,
            "q2_c4": q2,
            "ilu_c2": ilu,
        }
        print(json.dumps(line))
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
