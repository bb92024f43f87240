"""Generates the golden fixtures in this directory by running the reference's own
CPU solver (oracle/_ref/ref_harness, compiled from the reference's sources by
oracle/ref/Makefile) on small seeded problems and saving what it assembled and
solved: per-level matrices, Dirichlet lists and transfer maps in the
reference's node numbering, the right-hand side, the solution, the iteration
count and its CGInfo residuals. The "_dual" cases add a convection term (a
nonsymmetric operator) and the reference's dual solve
(StdMultiLevelSolver::AssembleDualMatrix + the same Gmres): the dual matrices'
values, the dual right-hand side dJ/du = 2 M u of J(u) = integral of u^2 (M the
Q1 mass matrix, u the forward solution of a first run) and the dual solution.
The "stokes_" cases are the Q1/Q1 Stokes system (ncomp = dim+1, block
matrices) with the pressure filter and the Vanka or block-Jacobi smoother
("_lps_lid": the reference's NavierStokesLps at u = 0, CGQ1Lps, with the
lid-driven cavity data, right-hand side -Form(u_D)); the
harness runs them on one OpenMP thread, so Vanka's patch contributions are
summed in patch order. The "hn_" cases refine a ball once more (hanging
nodes, Q1 or Q2 elements) and also record the reference's HNAverage,
HNDistribute and HNZero of a test vector on the finest level. The "q2_"
cases are CGQ2 elements with the seeded per-cell kappa. The "ilu_"
cases use linear_smooth ilu with matrixtype block (SparseBlockIlu). The "form_"
cases also record StdSolver::Form and StdMultiLevelSolver::NewtonResidual of a
seeded vector and the solution as written by WriteBackUp (.bup) and
WriteBackUpBinary (.bip); cases with "vtk" the solution as StdSolver::Visu
writes it (VTK). The "lps_" cases are CGQ2Lps / CGQ1Lps: Q2 or patch-Q1
convection-diffusion with local projection stabilisation of the convection
(constant coefficient).

    python tests/golden/make_golden.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from gascoignelib_b200.problem import (cell_nodes, load_reference_dump,  # noqa: E402
                                       seeded_inputs, _q1_local_mass)
from oracle.oracle import run_reference, write_inputs  # noqa: E402

# name: (dim, coarse, refine, seeded, tol, extra harness keys)
CASES = {
    "q1_2d_c2_r3_seeded": (2, 2, 3, True, 1e-10, {}),
    "q1_2d_c2_r4_poisson": (2, 2, 4, False, 1e-10, {}),
    "q1_3d_c1_r3_seeded": (3, 1, 3, True, 1e-8, {}),
    "q1_3d_c1_r3_wcycle": (3, 1, 3, True, 1e-8, {"mgtype": "W", "iterpre": 1,
                                                  "iterpost": 3, "omega": 0.7}),
    "q1_2d_c2_r3_fcycle": (2, 2, 3, True, 1e-10, {"mgtype": "F", "mgomega": 0.9}),
    "q1_3d_c1_r3_conv_dual": (3, 1, 3, True, 1e-8, {"conv": "1,0.5,0.25"}),
    "q1_2d_c2_r4_conv_dual": (2, 2, 4, True, 1e-10, {"conv": "4,2"}),
    "stokes_2d_c2_r4_vanka": (2, 2, 4, True, 1e-8,
                              {"problem": "stokes", "smoother": "vanka", "omega": 1.0,
                               "gmressize": 31}),
    "stokes_2d_c2_r3_jacobi": (2, 2, 3, True, 1e-8,
                               {"problem": "stokes", "smoother": "jacobi", "omega": 0.5,
                                "gmressize": 31}),
    "stokes_2d_c2_r4_lps_lid": (2, 2, 4, False, 1e-8,
                                {"problem": "stokeslps", "smoother": "vanka", "omega": 1.0,
                                 "gmressize": 31, "stab": 0.1}),
    "stokes_3d_c1_r3_vanka": (3, 1, 3, True, 1e-8,
                              {"problem": "stokes", "smoother": "vanka", "omega": 1.0,
                               "gmressize": 31}),
    "ilu_3d_c1_r3_seeded": (3, 1, 3, True, 1e-10, {"smoother": "ilu", "omega": 1.0}),
    "ilu_2d_c2_r4_conv": (2, 2, 4, True, 1e-10, {"smoother": "ilu", "omega": 1.0,
                                                 "conv": "4,2"}),
    "q2_3d_c1_r3_kappa_conv": (3, 1, 3, True, 1e-8, {"disc": "Q2", "conv": "1,0.5,0.25"}),
    "q2_2d_c2_r3_kappa": (2, 2, 3, True, 1e-10, {"disc": "Q2", "formx": 1009}),
    "form_3d_c1_r3_conv": (3, 1, 3, True, 1e-8, {"conv": "1,0.5,0.25", "backup": 1,
                                                 "formx": 1005, "vtk": 1}),
    "form_2d_c2_r3": (2, 2, 3, True, 1e-10, {"backup": 1, "formx": 1006, "vtk": 1}),
    "lps_2d_q2_c2_r3_conv": (2, 2, 3, True, 1e-10, {"disc": "Q2", "diff": 0.01, "lps": 0.5,
                                                    "omega": 0.3, "gmressize": 41,
                                                    "conv": "1,0.5"}),
    "lps_3d_q2_c1_r3_conv": (3, 1, 3, True, 1e-8, {"disc": "Q2", "diff": 0.01, "lps": 0.5,
                                                   "omega": 0.3, "gmressize": 41,
                                                   "formx": 1010,
                                                   "conv": "1,0.5,0.25"}),
    "lps_2d_q1_c2_r3_conv": (2, 2, 3, True, 1e-10, {"disc": "Q1", "diff": 0.01, "lps": 0.5,
                                                    "omega": 0.3, "gmressize": 41,
                                                    "formx": 1011,
                                                    "conv": "1,0.5"}),
    "lps_3d_q1_c1_r3_conv": (3, 1, 3, True, 1e-8, {"disc": "Q1", "diff": 0.01, "lps": 0.5,
                                                   "omega": 0.3, "gmressize": 41,
                                                   "conv": "1,0.5,0.25"}),
    "hn_2d_q1_c2_r3_ball": (2, 2, 3, True, 1e-10,
                            {"disc": "Q1", "ball": 0.25, "diff": 1.0, "vtk": 1,
                             "formx": 1007}),
    "hn_2d_q2_c2_r3_conv_ball": (2, 2, 3, True, 1e-10,
                                 {"disc": "Q2", "ball": 0.25, "diff": 0.1,
                                  "conv": "1,0.5", "formx": 1008}),
}


def stokes_rhs(dim, coarse, refine, seed=1002):
    """f ~ U[-1, 1] per node and component (p, v_1..v_dim), the pressure part
    made algebraically mean-free so that the system with its constant-pressure
    null space is consistent."""
    n1 = (coarse << refine) + 1
    r = np.random.default_rng(seed).uniform(-1.0, 1.0, size=(n1 ** dim, dim + 1))
    r[:, 0] -= r[:, 0].mean()
    return r.ravel()


def lex_permutation(coord, N):
    """Reference node -> lexicographic node index (x fastest) on N cells per
    dimension."""
    c = np.rint(coord * N).astype(np.int64)
    idx = np.zeros(c.shape[0], dtype=np.int64)
    for d in reversed(range(c.shape[1])):
        idx = idx * (N + 1) + c[:, d]
    return idx


def l2_dual_rhs(P, u_ref):
    """2 M u on the lexicographic node order (what the harness reads)."""
    import scipy.sparse as sp
    dim = P.dim
    N = round(P.finest.n ** (1.0 / dim)) - 1
    perm = lex_permutation(P.finest.coord, N)
    u = np.empty_like(u_ref)
    u[perm] = u_ref
    nodes = cell_nodes(dim, N)
    ml = _q1_local_mass(dim, 1.0 / N)
    nl = nodes.shape[1]
    M = sp.coo_matrix((np.tile(ml.ravel(), nodes.shape[0]),
                       (np.repeat(nodes, nl, axis=1).ravel(),
                        np.tile(nodes, (1, nl)).ravel())),
                      shape=(u.size, u.size)).tocsr()
    return 2.0 * (M @ u)


def make(name, dim, coarse, refine, seeded, tol, extra):
    d = tempfile.mkdtemp(prefix="gb_golden_")
    kw = {}
    stokes = extra.get("problem") in ("stokes", "stokeslps")
    if extra.get("problem") == "stokeslps":
        kw = {}  # the harness forms the right-hand side from the lid data
    elif stokes:
        kw = write_inputs(d, None, stokes_rhs(dim, coarse, refine))
    elif "ball" in extra:
        # nodes of the extra refinement sit on the twice finer lexicographic grid
        res = 2 * (coarse << refine)
        rhs = np.random.default_rng(1002).uniform(-1.0, 1.0, size=(res + 1) ** dim)
        kw = write_inputs(d, None, rhs)
        kw["rhsres"] = res
    elif seeded:
        kappa, rhs = seeded_inputs(dim, coarse, refine)
        kw = write_inputs(d, kappa, rhs)
    keys = dict(dim=dim, coarse=coarse, refine=refine, dump=1, tol=tol,
                gmressize=21, iterpre=2, iterpost=2, iterexact=10, omega=0.8)
    keys.update(extra)
    formx = None
    if "formx" in keys:  # a seeded vector on the finest nodes (any numbering)
        n1 = (coarse << refine) + 1
        if "ball" in extra:  # more nodes than that: the harness reads its first n
            n1 = 2 * (coarse << refine) + 1
        formx = np.random.default_rng(keys["formx"]).uniform(-1.0, 1.0, size=n1 ** dim)
        keys["formx"] = os.path.join(d, "formx.f64")
        formx.tofile(keys["formx"])
    dual = name.endswith("_dual")
    if dual:
        out0, _ = run_reference(d, **keys, **kw)
        P0 = load_reference_dump(out0)
        g = l2_dual_rhs(P0, np.fromfile(os.path.join(out0, "solution.f64")))
        gp = os.path.join(d, "dual_in.f64")
        g.tofile(gp)
        kw["dualrhs"] = gp
    out, summ = run_reference(d, threads=1, **keys, **kw)
    P = load_reference_dump(out)
    arrs = {"dim": P.dim, "nlevels": P.nlevels, "rhs": P.rhs,
            "solution": np.fromfile(os.path.join(out, "solution.f64")),
            "iterations": int(summ["iterations"][0]),
            "firstresidual": float(summ["firstresidual"][0]),
            "residual": float(summ["residual"][0]),
            "status": summ["status"][0] if len(summ["status"]) == 1
            else " ".join(summ["status"])}
    for k, v in keys.items():
        if k != "formx":
            arrs["key_" + k] = v
    if formx is not None:
        arrs["formx"] = formx[:P.finest.ndof]
        arrs["form"] = np.fromfile(os.path.join(out, "form.f64"))
        arrs["newton_residual"] = np.fromfile(os.path.join(out, "newton_residual.f64"))
        with open(os.path.join(out, "newton.txt")) as f:
            arrs["newton_norm"] = float(f.read().split()[1])
    if keys.get("vtk"):
        with open(os.path.join(out, "solution.00000.vtk"), "rb") as f:
            arrs["vtk"] = np.frombuffer(f.read(), dtype=np.uint8)
    if keys.get("backup"):
        for ext in ("bup", "bip"):
            with open(os.path.join(out, "solution." + ext), "rb") as f:
                arrs["backup_" + ext] = np.frombuffer(f.read(), dtype=np.uint8)
    if dual:
        ds = {}
        with open(os.path.join(out, "dual_summary.txt")) as f:
            for line in f:
                k, *v = line.split()
                ds[k] = v
        arrs["dual_rhs"] = np.fromfile(os.path.join(out, "dual_rhs.f64"))
        arrs["dual_solution"] = np.fromfile(os.path.join(out, "dual_solution.f64"))
        arrs["dual_iterations"] = int(ds["dual_iterations"][0])
        arrs["dual_firstresidual"] = float(ds["dual_firstresidual"][0])
        arrs["dual_residual"] = float(ds["dual_residual"][0])
        arrs["dual_status"] = " ".join(ds["dual_status"])
        for l in range(P.nlevels):
            arrs[f"L{l}_dualval"] = np.fromfile(os.path.join(out, f"L{l}_dualval.f64"))
    arrs["B"] = P.finest.B
    arrs["dircomp_mask"] = P.finest.dircomp_mask
    if "ball" in extra:
        for op in ("average", "distribute", "zero"):
            arrs["hn_" + op] = np.fromfile(os.path.join(out, f"hn_{op}.f64"))
    for l, lv in enumerate(P.levels):
        if lv.hn_edges is not None:
            arrs[f"L{l}_hnedge"] = lv.hn_edges.astype(np.int32)
            arrs[f"L{l}_hnface"] = lv.hn_faces.astype(np.int32)
            arrs[f"L{l}_hndisc"] = lv.hn_disc
        if lv.pf_mask:
            arrs[f"L{l}_pfw"] = lv.pf_weights
            arrs[f"L{l}_pfdomain"] = lv.pf_domain
        if lv.patches is not None:
            arrs[f"L{l}_patches"] = lv.patches.astype(np.int32)
        arrs[f"L{l}_rowptr"] = lv.rowptr.astype(np.int32)
        arrs[f"L{l}_col"] = lv.col.astype(np.int32)
        arrs[f"L{l}_diag"] = lv.diag.astype(np.int32)
        arrs[f"L{l}_val"] = lv.val
        arrs[f"L{l}_dirichlet"] = lv.dirichlet.astype(np.int32)
        arrs[f"L{l}_coord"] = lv.coord
    for l, t in enumerate(P.transfers):
        arrs[f"T{l}_c2f"] = t.c2f.astype(np.int32)
        arrs[f"T{l}_zweier"] = t.zweier.astype(np.int32)
        arrs[f"T{l}_vierer"] = t.vierer.astype(np.int32)
        arrs[f"T{l}_achter"] = t.achter.astype(np.int32)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrs)
    print(name, summ["iterations"], summ["status"])


if __name__ == "__main__":
    only = sys.argv[1:]
    for name, spec in CASES.items():
        if not only or name in only:
            make(name, *spec)
