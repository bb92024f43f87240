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
    """SM clocks and throttle reasons during the timed region, read (never set)
    through NVML every 5 ms, with one reading on entry and one on exit; the GPU
    is found by its UUID. Falls back to nvidia-smi every 200 ms when NVML is
    not available."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index, period=0.005):
        self.index = index
        self.period = period
        self.samples = []
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        self._h = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(index).uuid)
            self._h = pynvml.nvmlDeviceGetHandleByUUID(
                uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            self._nvml = pynvml
        except Exception:
            self._nvml = None

    def _sample_nvml(self):
        n, h = self._nvml, self._h
        try:
            r = n.nvmlDeviceGetCurrentClocksEventReasons(h)
            bits = (n.nvmlClocksEventReasonHwSlowdown, n.nvmlClocksEventReasonHwThermalSlowdown,
                    n.nvmlClocksEventReasonSwThermalSlowdown, n.nvmlClocksEventReasonSwPowerCap)
            self.samples.append([str(n.nvmlDeviceGetClockInfo(h, n.NVML_CLOCK_SM)),
                                 str(n.nvmlDeviceGetMaxClockInfo(h, n.NVML_CLOCK_SM)),
                                 str(n.nvmlDeviceGetPowerUsage(h) / 1000.0)] +
                                ["Active" if r & b else "Not Active" for b in bits])
        except Exception:
            pass

    def _sample_smi(self):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        idx = ids[self.index] if self.index < len(ids) else str(self.index)
        try:
            r = subprocess.run(["nvidia-smi", "-i", idx,
                                f"--query-gpu={self.Q}", "--format=csv,noheader,nounits"],
                               capture_output=True, text=True, timeout=5)
            if r.returncode == 0 and r.stdout.strip():
                self.samples.append([x.strip() for x in r.stdout.strip().split(",")])
        except Exception:
            pass

    def _sample(self):
        if self._nvml is not None:
            self._sample_nvml()
        else:
            self._sample_smi()

    def _run(self):
        while not self._stop.is_set():
            self._sample()
            self._stop.wait(self.period if self._nvml is not None else 0.2)

    def __enter__(self):
        self._sample()
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)
        self._sample()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 3 + i and s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_min_mhz": min(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples),
                "source": "nvml" if self._nvml is not None else "nvidia-smi"}


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
                                   iterpost=2, omega=0.8, savesol=1, functional=1,
                                   **write_inputs(d, kappa, rhs))
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
                "assemble_s": float(s["assemble_s"][0]) if "assemble_s" in s else None,
                "solution_lex": _reference_solution_lex(out, DIM, COARSE << REFINE),
                "J": float(s["functional_l2"][0])}
    from gascoignelib_b200.problem import structured_problem
    P = structured_problem(DIM, COARSE, REFINE, kappa, rhs)
    O = Oracle(P)
    t0 = time.time()
    x, info = O.gmres(vmax=21, tol=1e-8)
    dt = time.time() - t0
    return {"value": ndof / dt, "unit": "DoF/s", "cores": 1, "kind": "port",
            "sample": f"oracle C restatement, one solve ({dt:.2f} s, {info['iterations']} it)",
            "solve_s": dt, "iterations": info["iterations"]}


def _reference_solution_lex(out, dim, N, name="solution.f64", ncomp=1):
    """A solution the reference harness wrote (its node numbering), in the
    lexicographic order of the structured problems."""
    import numpy as np

    from gascoignelib_b200.problem import to_lex
    coord = np.fromfile(os.path.join(out, "coord.f64")).reshape(-1, dim)
    return to_lex(np.fromfile(os.path.join(out, name)), coord, N, ncomp)


def _rel(a, b):
    import numpy as np
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def max_over_ranks(ms, dist, device):
    """The whole job's time of a timed region: the largest of the ranks' device
    times (all-reduce MAX, the same collective on every rank); the local time
    on one rank."""
    if not dist:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(ndof, steps, world, ms):
    """DoF/s of the whole job: every replica solves ndof unknowns per step."""
    return ndof * steps * world / (ms / 1e3)


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


def adjoint_c5(local, steps, warmup, flush, with_ref=False, threads=1):
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
    u_dev, g_dev, lam_dev = c.download(l, u), c.download(l, g), c.download(l, lam)
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
    if with_ref:
        out.update(_adjoint_reference(kappa, rhs, g_dev, u_dev, lam_dev, grad, J,
                                      P.finest.ndof, t, threads))
    return out


def _adjoint_reference(kappa, rhs, g_dev, u_dev, lam_dev, grad, J, ndof, t_dev, threads):
    """The reference's FP64 CPU forward solve and dual solve (AssembleDualMatrix
    + the same Gmres, right-hand side the device's dJ/du = 2 M u) of the 96^3
    problem: its time is the CPU baseline of the adjoint line, its solutions
    the FP64 oracle for u, J, lambda and dJ/dkappa."""
    import numpy as np

    from gascoignelib_b200.problem import boundary_lex, q1_cell_gradient
    from oracle.oracle import REF_HARNESS, run_reference, write_inputs
    if not os.path.exists(REF_HARNESS):
        return {}
    d = tempfile.mkdtemp(prefix="gb_c5ref_")
    kw = write_inputs(d, kappa, rhs)
    gp = os.path.join(d, "dual_in.f64")
    np.ascontiguousarray(g_dev).tofile(gp)
    env = os.environ.get("OMP_NUM_THREADS")
    os.environ["OMP_NUM_THREADS"] = str(threads)
    try:
        t0 = time.time()
        out, s = run_reference(d, dim=3, coarse=3, refine=5, tol=1e-8, globaltol=1e-16,
                               gmressize=21, iterpre=2, iterpost=2, omega=0.8, savesol=1,
                               functional=1, dualrhs=gp, **kw)
        wall = time.time() - t0
    finally:
        if env is None:
            os.environ.pop("OMP_NUM_THREADS", None)
        else:
            os.environ["OMP_NUM_THREADS"] = env
    ds = {}
    with open(os.path.join(out, "dual_summary.txt")) as f:
        for line in f:
            k, *v = line.split()
            ds[k] = v
    N = 96
    u_ref = _reference_solution_lex(out, 3, N)
    lam_ref = _reference_solution_lex(out, 3, N, "dual_solution.f64")
    g_ref = q1_cell_gradient(u_ref, lam_ref, 3, N, boundary_lex(3, N))
    J_ref = float(s["functional_l2"][0])
    t_cpu = float(s["solve_s"][0]) + float(ds["dual_solve_s"][0])
    return {
        "cpu_baseline": {"value": ndof / t_cpu, "unit": "DoF/s (forward+adjoint)",
                         "cores": threads, "kind": "reference",
                         "sample": (f"reference CPU forward solve ({float(s['solve_s'][0]):.2f} "
                                    f"s, {s['iterations'][0]} it) + AssembleDualMatrix + dual "
                                    f"solve ({float(ds['dual_solve_s'][0]):.2f} s, "
                                    f"{ds['dual_iterations'][0]} it), one run; harness wall "
                                    f"{wall:.0f} s incl. mesh + assembly")},
        "speedup_vs_cpu": t_cpu / (t_dev * 1e-3),
        "accuracy": {"reference": "the reference's FP64 CPU forward and dual solutions",
                     "rel_err_u": _rel(u_dev, u_ref),
                     "rel_err_J": abs(J - J_ref) / abs(J_ref),
                     "rel_err_lambda": _rel(lam_dev, lam_ref),
                     "rel_err_grad": _rel(grad, g_ref)}}


def stokes_c3(local, steps, warmup, flush, threads=1):
    """C3: 2D equal-order Stokes, ncomp 3 (p, u, v), on 512^2 cells (789,507
    dofs): the reference's NavierStokesLps at u = 0 (CGQ1Lps: LPS pressure
    stabilisation) with the lid-driven cavity data (u = (1, 0) on the top,
    0 elsewhere; right-hand side -Form(u_D)), Vanka V(2,2) on 3x3-node
    patches (27x27 local systems), pressure filter, GMRES(30) to 1e-8.
    The reference builds the problem (its mesh, numbering and assembled block
    matrices, written by the harness) and solves it on the host cores (the CPU
    baseline and the FP64 oracle of u and J); the device runs the mixed solve
    (FP32 Vanka cycle in FP64 flexible GMRES), its FP64 twin and the
    reference-semantics left GMRES of the same system, device time with the L2
    flushed before every solve; the finest level's FP32 Vanka sweep is timed
    alone for the roofline. The 12x12 variant repeats the mixed solve with
    single-cell patches."""
    import shutil

    import numpy as np
    import torch

    from gascoignelib_b200.native import GB_FP32, GB_FP64, Context
    from gascoignelib_b200.problem import (cell_patches, lex_index, load_reference_dump,
                                           q1_l2_squared, to_lex)
    from oracle.oracle import REF_HARNESS, run_reference

    if not os.path.exists(REF_HARNESS):
        return {"unavailable": "the reference harness (oracle/_ref) is not built"}
    d = tempfile.mkdtemp(prefix="gb_c3_")
    env = os.environ.get("OMP_NUM_THREADS")
    os.environ["OMP_NUM_THREADS"] = str(threads)
    try:
        t0 = time.time()
        out, s = run_reference(d, dim=2, coarse=2, refine=8, problem="stokeslps",
                               smoother="vanka", omega=1.0, gmressize=31, stab=0.1,
                               tol=1e-8, globaltol=1e-16, maxiter=300, dump=1,
                               functional=1)
        wall = time.time() - t0
    finally:
        if env is None:
            os.environ.pop("OMP_NUM_THREADS", None)
        else:
            os.environ["OMP_NUM_THREADS"] = env
    P = load_reference_dump(out)
    P.info["smoother"] = "vanka"
    u_ref = np.fromfile(os.path.join(out, "solution.f64"))
    J_ref = float(s["functional_l2"][0])
    t_cpu = float(s["solve_s"][0])
    shutil.rmtree(d, ignore_errors=True)
    N = 512
    coord = P.finest.coord

    def J_of(u):
        return q1_l2_squared(to_lex(u, coord, N, 3), 2, N, ncomp=3, comps=(1, 2))

    keys = dict(iterpre=2, iterpost=2, iterexact=10, omega=1.0, mgomega=1.0, mgtype="V",
                gmressize=31, tol=1e-8, globaltol=1e-300, maxiter=300, smoother="vanka")
    c = Context(local)
    c.load_problem(P)
    c.set_params(**keys)
    l = P.nlevels - 1
    x, b = c.vec(), c.vec()
    c.upload(l, b, P.rhs)
    out = {}
    sols = {}
    for name, prec in (("mixed", GB_FP32), ("fp64", GB_FP64)):
        for _ in range(warmup):
            c.fgmres(x, b, prec)
        ms = []
        for _ in range(steps):
            flush.random_(0, 255)
            torch.cuda.synchronize()
            info = c.fgmres(x, b, prec)
            ms.append(info["device_ms"])
        sols[name] = c.download(l, x)
        t = sum(ms) / len(ms)
        out[name] = {"value": P.finest.ndof / (t * 1e-3), "unit": "DoF/s",
                     "ms_per_step": t, "iterations": info["iterations"],
                     "restarts": info["restarts"],
                     "true_rel_residual": info["true_rel_residual"]}
    info = c.gmres(x, b)
    sols["fp64_left"] = c.download(l, x)
    out["fp64_left"] = {"ms_per_step": info["device_ms"], "iterations": info["iterations"],
                        "reference_iterations": int(s["iterations"][0])}
    peak, peak_kind = _peaks()
    sw_ms, sw_b = c.bench_sweep(l, GB_FP32, reps=10, flush_l2=2)
    ach = sw_b / (sw_ms * 1e-3) / 1e9
    out["roofline"] = {"bound": "hbm", "kernel": "k_vanka_inv_ct<27,float> patch solves + "
                       "k_vanka_gather<3,float>, finest level (one FP32 Vanka sweep)",
                       "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                       "ms_per_launch": sw_ms, "algorithmic_bytes": sw_b,
                       "peak_kind": peak_kind + " (burst copy)"}
    c.close()
    acc = {"reference": "the reference's FP64 CPU solution (same assembled system)",
           "functional": "J(u) = int |v|^2 over the velocity update (reference: its own "
                         "ComputeDomainFunctional; device: exact Q1 mass)",
           "J_reference": J_ref}
    for name, u in sols.items():
        acc[f"rel_err_u_{name}"] = _rel(u, u_ref)
        acc[f"rel_err_J_{name}"] = abs(J_of(u) - J_ref) / abs(J_ref)
    out["accuracy"] = acc
    out["cpu_baseline"] = {"value": P.finest.ndof / t_cpu, "unit": "DoF/s", "cores": threads,
                           "kind": "reference",
                           "sample": (f"reference CPU StdMultiLevelSolver GMRES + Vanka "
                                      f"V-cycle on the same system, one solve "
                                      f"({t_cpu:.2f} s, {s['iterations'][0]} iterations; "
                                      f"harness wall {wall:.0f} s incl. mesh, assembly, "
                                      f"dump)")}
    out["speedup_vs_cpu_mixed"] = t_cpu / (out["mixed"]["ms_per_step"] * 1e-3)
    # the 12 x 12 variant: Vanka on single cells (4 nodes x 3 components)
    for lv in P.levels:
        Nl = round(lv.n ** 0.5) - 1
        inv = np.empty(lv.n, dtype=np.int64)
        inv[lex_index(lv.coord, Nl)] = np.arange(lv.n)
        lv.patches = inv[cell_patches(2, Nl)]
    c = Context(local)
    c.load_problem(P)
    c.set_params(**keys)
    x, b = c.vec(), c.vec()
    c.upload(l, b, P.rhs)
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
        "value": P.finest.ndof / (t * 1e-3), "unit": "DoF/s", "ms_per_step": t,
        "iterations": info["iterations"], "true_rel_residual": info["true_rel_residual"],
        "rel_err_u": _rel(c.download(l, x), u_ref)}
    c.close()
    out["workload"] = ("2D Stokes Q1/Q1, NavierStokesLps at u=0 (CGQ1Lps, alpha0 0.1, visc 1), "
                       "lid-driven cavity, 512^2 cells, 789,507 dofs, the reference's own mesh "
                       "and matrices, Vanka 3x3-node patches (27x27), pressure filter, V(2,2), "
                       "GMRES(30), tol 1e-8; 12x12 variant: single-cell patches")
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


def q2_c4_reference_mesh(steps, threads):
    """C4 on the reference's own mesh, through the reference-side binding: the
    binding harness (oracle/_ref/ref_harness_b200) builds the 80^3-cell CGQ2
    mesh and refines, with MeshAgent::refine_cells, the leaf cells whose
    centroid lies within 0.25 of the centre (1,017,329 dofs on the finest of 5
    levels, hanging nodes on edges and faces), assembles -0.01 Laplace u +
    (1, 0.5, 0.25) . grad u = f (f ~ U[-1, 1], seed 1002) with the reference's
    CGDisc, and hands it to B200MultiLevelSolver. On the device: the
    reference-semantics FP64 GMRES (one cycle of up to 127 steps: the FP64
    oracle of this line, pinned to the reference's CPU solve by the tests),
    then `steps` flexible solves with the same Krylov memory (128: restarted
    flexible GMRES(30) stalls on this operator, over 600 steps) and an FP64
    cycle, and `steps` in mixed precision (FP32 cycle), each timed by CUDA
    events inside the
    binding (the finest matrix, about 0.9 GB in FP64, is larger than L2); the
    finest level's SpMV and FP32 Jacobi sweep timed alone. The reference's CPU
    solver runs 3 GMRES steps on the same mesh and right-hand side (the
    bounded CPU baseline sample)."""
    import numpy as np

    from oracle.oracle import REF_HARNESS_B200, run_reference, write_inputs
    if not os.path.exists(REF_HARNESS_B200):
        return {"unavailable": "the binding harness (oracle/_ref/ref_harness_b200) is not built"}
    res = 2 * (5 << 4)
    d = tempfile.mkdtemp(prefix="gb_c4_")
    rhs = np.random.default_rng(1002).uniform(-1.0, 1.0, size=(res + 1) ** 3)
    env = os.environ.get("OMP_NUM_THREADS")
    os.environ["OMP_NUM_THREADS"] = str(threads)
    try:
        t0 = time.time()
        out, s = run_reference(d, harness=REF_HARNESS_B200, backend="b200", dim=3, coarse=5,
                               refine=4, disc="Q2", ball=0.25, diff=0.01, conv="1,0.5,0.25",
                               rhsres=res, tol=1e-8, globaltol=1e-16, gmressize=128,
                               maxiter=600, iterpre=2, iterpost=2, omega=0.3, functional=1,
                               flexreps=steps, flexgmressize=0, benchspmv=1, cpusample=3,
                               savesol=1, **write_inputs(d, None, rhs))
        wall = time.time() - t0
    finally:
        if env is None:
            os.environ.pop("OMP_NUM_THREADS", None)
        else:
            os.environ["OMP_NUM_THREADS"] = env
    ndof = int(s["nnodes_L4"][0])
    u64 = np.fromfile(os.path.join(out, "solution.f64"))
    um = np.fromfile(os.path.join(out, "solution_mixed.f64"))
    J64 = float(s["functional_l2"][0])
    peak, peak_kind = _peaks()

    def med(key):
        v = sorted(float(t) for t in s[key])
        return v[len(v) // 2]

    res_ = {}
    for tag, name in (("mixed", "mixed"), ("flex64", "fp64")):
        t = med(f"{tag}_device_ms_all")
        res_[name] = {"value": ndof / (t * 1e-3), "unit": "DoF/s", "ms_per_step": t,
                      "iterations": int(s[f"{tag}_iterations"][0]),
                      "restarts": int(s[f"{tag}_restarts"][0]),
                      "kernel_launches": int(s[f"{tag}_launches"][0]),
                      "true_rel_residual": float(s[f"{tag}_true_rel_residual"][0])}
    sw_ms, sw_b = float(s["sweep32_ms"][0]), float(s["sweep32_bytes"][0])
    sp_ms, sp_b = float(s["spmv64_ms"][0]), float(s["spmv64_bytes"][0])
    it_ref = int(s["iterations"][0])
    cpu_it = int(s["cpu_sample_iterations"][0])
    cpu_s = float(s["cpu_sample_s"][0])
    cpu_est = cpu_s / max(cpu_it, 1) * it_ref
    res_.update({
        "workload": ("3D CGQ2 convection-diffusion eps 1e-2, beta (1,0.5,0.25), 80^3 cells "
                     "refined once by the reference (MeshAgent::refine_cells on leaf cells "
                     "whose centroid is in |x-0.5|<0.25), %d dofs, 5 levels, the reference's "
                     "mesh and CGDisc matrices through the binding, Jacobi V(2,2) omega 0.3, "
                     "flexible GMRES with Krylov memory 128, tol 1e-8" % ndof),
        "dofs": ndof,
        "mixed_over_fp64": res_["mixed"]["value"] / res_["fp64"]["value"],
        "fp64_reference_semantics": {"ms_per_step": med("device_ms_all"),
                                     "iterations": it_ref, "status": s["status"][0],
                                     "true_rel_residual": float(s["true_rel_residual"][0])},
        "accuracy": {"reference": "the reference-semantics FP64 device solve of the same "
                                  "system (within 1e-8 of the reference's CPU solve: "
                                  "tests/test_gpu_binding.py)",
                     "functional": "J(u) = int u^2 (the reference's ComputeDomainFunctional "
                                   "on each solution)",
                     "rel_err_u_mixed": _rel(um, u64),
                     "rel_err_J_mixed":
                         abs(float(s["mixed_functional_l2"][0]) - J64) / abs(J64),
                     "rel_err_J_fp64_flexible":
                         abs(float(s["flex64_functional_l2"][0]) - J64) / abs(J64)},
        "roofline": {"bound": "hbm", "kernel": "k_spmv<kJacobi,float> FP32 Jacobi sweep, "
                     "finest level (ball-refined, hanging nodes)",
                     "achieved": sw_b / (sw_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": sw_b / (sw_ms * 1e-3) / 1e9 / peak, "ms_per_launch": sw_ms,
                     "algorithmic_bytes": sw_b, "peak_kind": peak_kind + " (burst copy)",
                     "fp64_spmv": {"ms_per_launch": sp_ms, "algorithmic_bytes": sp_b,
                                   "frac": sp_b / (sp_ms * 1e-3) / 1e9 / peak}},
        "cpu_baseline": {"value": ndof / cpu_est, "unit": "DoF/s", "cores": threads,
                         "kind": "reference",
                         "sample": (f"reference CPU StdMultiLevelSolver on the same mesh and "
                                    f"right-hand side: {cpu_it} GMRES steps in {cpu_s:.2f} s, "
                                    f"scaled to the {it_ref} steps its one-cycle solve takes "
                                    f"({cpu_est:.1f} s); binding harness wall {wall:.0f} s "
                                    f"incl. mesh, two CPU assemblies and the device runs")},
        "speedup_vs_cpu_mixed": cpu_est / (res_["mixed"]["ms_per_step"] * 1e-3),
    })
    return res_


def q2_c4(local, steps, warmup, flush, with_ref=True, threads=1):
    """C4: 3D CGQ2 convection-diffusion -0.01 Laplace u + (1, 0.5, 0.25) .
    grad u = f on 80^3 cells refined once more inside the ball |x - 0.5| <
    0.25: on the reference's own mesh through the binding
    (q2_c4_reference_mesh). Beside it, the same operator on the uniform 80^3
    cells (531,441 dofs, four levels, this package's generator): Jacobi V(2,2)
    with omega 0.3 (the reference's cycle stalls with 0.5 and above on this
    convection-dominated Q2 operator), GMRES(30) to 1e-8, mixed and FP64
    solves, device time, L2 flushed before every solve."""
    import torch

    from gascoignelib_b200.native import GB_FP32, GB_FP64, Context
    from gascoignelib_b200.problem import q2_meshes, structured_q2

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

    out = q2_c4_reference_mesh(steps, threads) if with_ref else {}
    U = structured_q2(3, 5, 4, eps=1e-2, beta=(1.0, 0.5, 0.25))
    out["uniform_no_ball"] = run(U)
    out["uniform_no_ball"]["workload"] = ("the same operator on the uniform 80^3 cells "
                                          "(531,441 dofs, this package's generator)")
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
    ap.add_argument("--no-ilu", action="store_true",
                    help="skip the C2 solves with the block ILU smoother")
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

    tmax = max_over_ranks(sum(ms32), dist, f"cuda:{local}")
    value = replica_value(ndof, args.steps, world, tmax)
    v64 = ndof * args.steps / (sum(ms64) / 1e3)
    vleft = ndof * args.steps / (sum(msleft) / 1e3)

    # e2e: the C-ABI call with host buffers (pinned), H2D + solve + D2H timed
    b_host = torch.from_numpy(P.rhs.copy()).pin_memory()
    x_host = torch.empty_like(b_host).pin_memory()
    bn = b_host.numpy()
    xn = x_host.numpy()
    for _ in range(args.warmup):  # untimed, as for the device-resident steps
        ctx.solve_host(bn, method=2, out=xn)
    e2e_ms = []
    for _ in range(args.steps):
        flush.random_(0, 255)
        torch.cuda.synchronize()
        _, info = ctx.solve_host(bn, method=2, out=xn)
        e2e_ms.append(info["device_ms"])
    e2e_val = replica_value(ndof, args.steps, world,
                            max_over_ranks(sum(e2e_ms), dist, f"cuda:{local}"))

    # the solutions of the three solvers, for the accuracy keys (untimed)
    ctx.fgmres(xv, bv, GB_FP32)
    u_mixed = ctx.download(fl, xv)
    ctx.fgmres(xv, bv, GB_FP64)
    u_fp64 = ctx.download(fl, xv)
    ctx.gmres(xv, bv)
    u_left = ctx.download(fl, xv)

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
    # the mixed solve's dominant kernel: the finest level's FP32 Jacobi sweep
    sw_ms32, sw_b32 = ctx.bench_sweep(fl, GB_FP32, reps=20, flush_l2=2)
    sw_ms64, sw_b64 = ctx.bench_sweep(fl, GB_FP64, reps=20, flush_l2=2)
    achsw32 = sw_b32 / (sw_ms32 * 1e-3) / 1e9
    achsw64 = sw_b64 / (sw_ms64 * 1e-3) / 1e9
    prof32 = {}
    pj32 = os.path.join(ROOT, "profiles", "sweep_fp32_c2_finest.json")
    if os.path.exists(pj32):
        prof32 = json.load(open(pj32))
    prof = {}
    pj = os.path.join(ROOT, "profiles", "spmv_fp64_c2_finest.json")
    if os.path.exists(pj):
        prof = json.load(open(pj))

    asm = assembly_leg(ctx, P, kappa, min(args.steps, 5), 2, flush, torch.device(f"cuda:{local}"))

    adj = None
    if not args.no_adjoint:
        adj = adjoint_c5(local, min(args.steps, 5), 2, flush,
                         with_ref=rank == 0 and not args.no_cpu_baseline,
                         threads=os.cpu_count() or 1)
    stk = None
    if not args.no_stokes:
        stk = stokes_c3(local, min(args.steps, 5), 2, flush, threads=os.cpu_count() or 1)
    q2 = None
    if not args.no_q2:
        q2 = q2_c4(local, min(args.steps, 3), 1, flush,
                   with_ref=rank == 0 and not args.no_cpu_baseline,
                   threads=os.cpu_count() or 1)
    ilu = None
    if not args.no_ilu:
        ilu = ilu_c2(local, P, min(args.steps, 3), 1, flush, os.cpu_count() or 1,
                     rank == 0 and not args.no_cpu_baseline)

    if rank == 0:
        cb = None
        acc = None
        if not args.no_cpu_baseline:
            from gascoignelib_b200.problem import q1_l2_squared
            cb = cpu_baseline((kappa, rhs), ndof, os.cpu_count() or 1)
            uref = cb.pop("solution_lex", None)
            Jref = cb.pop("J", None)
            if uref is not None:
                N = COARSE << REFINE
                acc = {"reference": "the reference's FP64 CPU solution of the same problem "
                                    "(cpu_baseline run, its node numbering mapped by "
                                    "coordinates)",
                       "functional": "J(u) = int u^2 (reference: its own "
                                     "ComputeDomainFunctional; device solutions: exact "
                                     "Q1 mass)",
                       "J_reference": Jref}
                for name, u in (("mixed", u_mixed), ("fp64", u_fp64), ("fp64_left", u_left)):
                    J = q1_l2_squared(u, DIM, N)
                    acc[f"rel_err_u_{name}"] = _rel(u, uref)
                    acc[f"rel_err_J_{name}"] = abs(J - Jref) / abs(Jref)
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
            # the headline (mixed) solve's dominant kernel: the finest level's
            # fused FP32 Jacobi sweep; the FP64 SpMV and sweep beside it
            "roofline": {"bound": "hbm",
                         "kernel": "k_spmv<kJacobi,float> fused FP32 Jacobi sweep, finest "
                                   "level (the mixed solve's largest share)",
                         "achieved": achsw32, "peak": peak, "unit": "GB/s",
                         "frac": achsw32 / peak,
                         "traffic": prof32.get("traffic_bytes"),
                         "peak_kind": peak_kind + " (burst copy)",
                         "ms_per_launch": sw_ms32, "algorithmic_bytes": sw_b32,
                         "ncu_duration_us": prof32.get("ncu_duration_us"),
                         "traffic_source": "profiles/sweep_fp32_c2_finest.md (ncu)",
                         "fp64_spmv": {"kernel": "k_spmv<kAx,double> finest level",
                                       "achieved": ach64, "frac": ach64 / peak,
                                       "traffic": prof.get("traffic_bytes"),
                                       "ms_per_launch": spmv_ms64,
                                       "algorithmic_bytes": spmv_b64,
                                       "ms_per_launch_write_flush": spmv_ms64w,
                                       "ncu_duration_us": prof.get("ncu_duration_us"),
                                       "traffic_source": "profiles/spmv_fp64_c2_finest.md (ncu)"},
                         "fp32_spmv": {"achieved": ach32, "frac": ach32 / peak,
                                       "ms_per_launch": spmv_ms32,
                                       "algorithmic_bytes": spmv_b32},
                         "fp64_sweep": {"achieved": achsw64, "frac": achsw64 / peak,
                                        "ms_per_launch": sw_ms64,
                                        "algorithmic_bytes": sw_b64}},
            "accuracy": acc,
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
