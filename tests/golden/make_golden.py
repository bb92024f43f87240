"""Generates the golden fixtures in this directory by running the reference's own
CPU solver (oracle/_ref/ref_harness, compiled from the reference's sources by
oracle/ref/Makefile) on small seeded problems and saving what it assembled and
solved: per-level matrices, Dirichlet lists and transfer maps in the
reference's node numbering, the right-hand side, the solution, the iteration
count and its CGInfo residuals.

    python tests/golden/make_golden.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from gascoignelib_b200.problem import load_reference_dump, seeded_inputs  # noqa: E402
from oracle.oracle import run_reference, write_inputs  # noqa: E402

# name: (dim, coarse, refine, seeded, tol, extra harness keys)
CASES = {
    "q1_2d_c2_r3_seeded": (2, 2, 3, True, 1e-10, {}),
    "q1_2d_c2_r4_poisson": (2, 2, 4, False, 1e-10, {}),
    "q1_3d_c1_r3_seeded": (3, 1, 3, True, 1e-8, {}),
    "q1_3d_c1_r3_wcycle": (3, 1, 3, True, 1e-8, {"mgtype": "W", "iterpre": 1,
                                                  "iterpost": 3, "omega": 0.7}),
    "q1_2d_c2_r3_fcycle": (2, 2, 3, True, 1e-10, {"mgtype": "F", "mgomega": 0.9}),
}


def make(name, dim, coarse, refine, seeded, tol, extra):
    d = tempfile.mkdtemp(prefix="gb_golden_")
    kw = {}
    if seeded:
        kappa, rhs = seeded_inputs(dim, coarse, refine)
        kw = write_inputs(d, kappa, rhs)
    keys = dict(dim=dim, coarse=coarse, refine=refine, dump=1, tol=tol,
                gmressize=21, iterpre=2, iterpost=2, iterexact=10, omega=0.8)
    keys.update(extra)
    out, summ = run_reference(d, **keys, **kw)
    P = load_reference_dump(out)
    arrs = {"dim": P.dim, "nlevels": P.nlevels, "rhs": P.rhs,
            "solution": np.fromfile(os.path.join(out, "solution.f64")),
            "iterations": int(summ["iterations"][0]),
            "firstresidual": float(summ["firstresidual"][0]),
            "residual": float(summ["residual"][0]),
            "status": summ["status"][0] if len(summ["status"]) == 1
            else " ".join(summ["status"])}
    for k, v in keys.items():
        arrs["key_" + k] = v
    for l, lv in enumerate(P.levels):
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
    for name, spec in CASES.items():
        make(name, *spec)
