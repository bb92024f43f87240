"""Fixed workloads for profiling runs (ncu launch lists and kernel captures).

    python -m gascoignelib_b200.workload --method mixed --solves 2 [--refine 6]
    python -m gascoignelib_b200.workload --spmv 3 [--precision fp64]
    python -m gascoignelib_b200.workload --sweep 3 [--precision fp32]

--method: mixed (FP32 cycle, flexible FP64 GMRES), fp64 (FP64 cycle, flexible),
left (reference-semantics left-preconditioned FP64 GMRES). --spmv K runs only K
finest-level SpMV launches (L2 flushed before each) after the set-up.
The problem is the seeded 3D Q1 diffusion problem (refine 6: 64^3 cells).
"""
from __future__ import annotations

import argparse
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--method", default="mixed", choices=["mixed", "fp64", "left"])
    ap.add_argument("--solves", type=int, default=2)
    ap.add_argument("--refine", type=int, default=6)
    ap.add_argument("--spmv", type=int, default=0)
    ap.add_argument("--smooth", type=int, default=0,
                    help="only K FP64 smoothing sweeps on the finest level (StdSolver::smooth "
                         "with the problem's smoother), after the set-up")
    ap.add_argument("--sweep", type=int, default=0,
                    help="only K finest-level sweeps of the smoother's dominant kernel "
                         "(the fused Jacobi sweep, or Vanka's patch solves and gather), "
                         "timed alone with the L2 flushed before each (gb_bench_sweep)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--problem", default="diffusion", choices=["diffusion", "stokes", "q2", "q2ball"],
                    help="stokes: 2D Q1/Q1 Stokes with Vanka on (2*2^(refine-1))^2 cells")
    ap.add_argument("--smoother", default=None, choices=["jacobi", "vanka", "ilu"],
                    help="override the problem's smoother (ilu: omega 1)")
    ap.add_argument("--assemble", type=int, default=0,
                    help="only K device assemblies of every level (diffusion, q2, q2ball)")
    ap.add_argument("--ktime", action="store_true",
                    help="per-kernel CUDA-event times of the last solve (GB_GRAPH=0)")
    a = ap.parse_args(argv)

    from gascoignelib_b200.build import build_library
    from gascoignelib_b200.native import GB_FP32, GB_FP64, Context
    from gascoignelib_b200.problem import (seeded_inputs, structured_problem,
                                           structured_stokes)

    build_library()
    if a.problem == "stokes":
        P = structured_stokes(2, 2, a.refine)
        keys = dict(gmressize=31, omega=1.0)
    elif a.problem in ("q2", "q2ball"):
        from gascoignelib_b200.problem import structured_q2, structured_q2_ball
        P = (structured_q2(3, 5, a.refine - 2) if a.problem == "q2"
             else structured_q2_ball(5, a.refine - 2))
        keys = dict(gmressize=31, omega=0.3, maxiter=600)
    else:
        kappa, rhs = seeded_inputs(3, 1, a.refine)
        P = structured_problem(3, 1, a.refine, kappa, rhs)
        keys = dict(gmressize=21, omega=0.8)
    with Context(0) as ctx:
        ctx.load_problem(P)
        keys.setdefault("maxiter", 200)
        if a.smoother:
            keys["smoother"] = a.smoother
            if a.smoother == "ilu":
                keys["omega"] = 1.0
        ctx.set_params(tol=1e-8, globaltol=1e-300, iterpre=2, iterpost=2, **keys)
        fl = P.nlevels - 1
        if a.assemble:
            import time
            beta = None
            if a.problem in ("q2", "q2ball"):  # Q2 elements (ball: hanging nodes condensed)
                import numpy as np
                from gascoignelib_b200.problem import q2_meshes
                meshes = q2_meshes(P)
                for l, (el, par) in enumerate(meshes):
                    ctx.set_mesh(l, P.dim, el, P.levels[l].coord, par, degree=2)
                kappa = np.full(meshes[-1][0].shape[0], P.info["eps"])
                beta = P.info.get("beta") or (1.0, 0.5, 0.25)
            else:
                from gascoignelib_b200.problem import structured_meshes
                for l, (cells, coord, par) in enumerate(structured_meshes(P)):
                    ctx.set_mesh(l, P.dim, cells, coord, par)
            ctx.assemble_levels(kappa, beta)  # set-up outside the count
            ctx.synchronize()
            k0 = ctx.kernel_count()
            t0 = time.time()
            for _ in range(a.assemble):
                ctx.assemble_levels(kappa, beta)
            ctx.synchronize()
            print(json.dumps({"assemblies": a.assemble, "kernels": ctx.kernel_count() - k0,
                              "wall_ms_each": 1e3 * (time.time() - t0) / a.assemble}))
            return
        if a.smooth:
            x, y, h = ctx.vec(), ctx.vec(), ctx.vec()
            ctx.upload(fl, y, P.rhs)
            ctx.smooth(fl, 1, x, y, h)  # set-up (Vanka factors) outside the count
            ctx.synchronize()
            k0 = ctx.kernel_count()
            ctx.smooth(fl, a.smooth, x, y, h)
            ctx.synchronize()
            print(json.dumps({"sweeps": a.smooth, "kernels": ctx.kernel_count() - k0}))
            return
        if a.sweep:
            prec = GB_FP32 if a.precision == "fp32" else GB_FP64
            ms, by = ctx.bench_sweep(fl, prec, reps=a.sweep, flush_l2=2)
            print(json.dumps({"sweep_ms": ms, "bytes": by, "GBps": by / ms / 1e6}))
            return
        if a.spmv:
            prec = GB_FP32 if a.precision == "fp32" else GB_FP64
            ms, by = ctx.bench_spmv(fl, prec, reps=a.spmv, flush_l2=2)
            print(json.dumps({"spmv_ms": ms, "bytes": by, "GBps": by / ms / 1e6}))
            return
        x, b = ctx.vec(), ctx.vec()
        ctx.upload(fl, b, P.rhs)
        for it in range(a.solves):
            if a.ktime and it == a.solves - 1:
                ctx.set_timing(True)
            if a.method == "left":
                info = ctx.gmres(x, b)
            else:
                info = ctx.fgmres(x, b, GB_FP32 if a.method == "mixed" else GB_FP64,
                                  check=False)
            print(json.dumps({k: info[k] for k in ("iterations", "restarts", "device_ms",
                                                   "true_rel_residual", "kernel_launches")}))
        if a.ktime:
            kt = ctx.kernel_times()
            tot = sum(v[1] for v in kt.values())
            for name, (cnt, ms) in sorted(kt.items(), key=lambda kv: -kv[1][1]):
                print(f"{cnt:6d} {1e3 * ms:10.1f} us {1e3 * ms / cnt:8.2f} us/launch "
                      f"{100 * ms / tot:5.1f}%  {name[:90]}")
            print(f"kernel time total {1e3 * tot:.1f} us")


if __name__ == "__main__":
    main()
