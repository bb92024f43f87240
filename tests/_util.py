"""Shared helpers of the test suite (fixture loading, tolerances)."""
import glob
import os

import numpy as np

from gascoignelib_b200.problem import (Cells, Level, Problem, Transfer, _q1_local_mass,
                                       _q1_local_stiffness, cell_nodes)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_cases():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    """Returns (Problem in the reference's numbering, reference results dict)."""
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    nl = int(z["nlevels"])
    B = int(z["B"]) if "B" in z.files else 1
    dmask = int(z["dircomp_mask"]) if "dircomp_mask" in z.files else 1
    levels, transfers = [], []
    for l in range(nl):
        rp = z[f"L{l}_rowptr"].astype(np.int64)
        lv = Level(n=rp.shape[0] - 1, B=B, rowptr=rp,
                   col=z[f"L{l}_col"].astype(np.int64),
                   diag=z[f"L{l}_diag"].astype(np.int64),
                   val=z[f"L{l}_val"],
                   dirichlet=z[f"L{l}_dirichlet"].astype(np.int64),
                   dircomp_mask=dmask, coord=z[f"L{l}_coord"])
        if f"L{l}_pfw" in z.files:
            lv.pf_mask = 1
            lv.pf_weights = z[f"L{l}_pfw"]
            lv.pf_domain = float(z[f"L{l}_pfdomain"])
        if f"L{l}_patches" in z.files:
            lv.patches = z[f"L{l}_patches"].astype(np.int64)
        if f"L{l}_hnedge" in z.files:
            lv.hn_edges = z[f"L{l}_hnedge"].astype(np.int64).reshape(-1, 4)
            lv.hn_faces = z[f"L{l}_hnface"].astype(np.int64).reshape(-1, 10)
            lv.hn_disc = int(z[f"L{l}_hndisc"])
        levels.append(lv)
    for l in range(nl - 1):
        transfers.append(Transfer(c2f=z[f"T{l}_c2f"].astype(np.int64),
                                  zweier=z[f"T{l}_zweier"].astype(np.int64),
                                  vierer=z[f"T{l}_vierer"].astype(np.int64),
                                  achter=z[f"T{l}_achter"].astype(np.int64)))
    keys = {k[4:]: z[k].item() for k in z.files if k.startswith("key_")}
    P = Problem(dim=int(z["dim"]), levels=levels, transfers=transfers,
                rhs=z["rhs"].copy(), info={"smoother": keys.get("smoother", "jacobi")})
    ref = {"solution": z["solution"], "iterations": int(z["iterations"]),
           "firstresidual": float(z["firstresidual"]), "residual": float(z["residual"]),
           "status": str(z["status"]), "keys": keys}
    if "hn_average" in z.files:
        ref.update(hn_average=z["hn_average"], hn_distribute=z["hn_distribute"],
                   hn_zero=z["hn_zero"])
    if "dual_solution" in z.files:
        ref.update(dual_rhs=z["dual_rhs"], dual_solution=z["dual_solution"],
                   dual_iterations=int(z["dual_iterations"]),
                   dual_firstresidual=float(z["dual_firstresidual"]),
                   dual_residual=float(z["dual_residual"]),
                   dual_status=str(z["dual_status"]),
                   dualval=[z[f"L{l}_dualval"] for l in range(nl)])
    for k in ("formx", "form", "newton_residual", "backup_bup", "backup_bip", "vtk"):
        if k in z.files:
            ref[k] = z[k]
    if "newton_norm" in z.files:
        ref["newton_norm"] = float(z["newton_norm"])
    return P, ref


def golden_hn_cases():
    return [n for n in golden_cases() if n.startswith("hn_")]


def golden_stokes_cases():
    return [n for n in golden_cases() if n.startswith("stokes_")]


def golden_dual_cases():
    return [n for n in golden_cases() if n.endswith("_dual")]


def dual_problem(P, ref):
    """P with the reference's own dual matrices (transpose, Dirichlet rows)."""
    import copy
    D = copy.copy(P)
    D.levels = []
    for L, dv in zip(P.levels, ref["dualval"]):
        Lt = copy.copy(L)
        Lt.val = dv
        D.levels.append(Lt)
    return D


def reference_cells(P):
    """Finest-level cells of a uniform unit square/cube mesh in the
    reference's node numbering (mapped through the node coordinates)."""
    dim = P.dim
    N = round(P.finest.n ** (1.0 / dim)) - 1
    c = np.rint(P.finest.coord * N).astype(np.int64)
    lex = np.zeros(c.shape[0], dtype=np.int64)
    for d in reversed(range(dim)):
        lex = lex * (N + 1) + c[:, d]
    inv = np.empty_like(lex)
    inv[lex] = np.arange(lex.size)
    return Cells(nodes=inv[cell_nodes(dim, N)], kloc=_q1_local_stiffness(dim, 1.0 / N),
                 mloc=_q1_local_mass(dim, 1.0 / N))


def solver_keys(keys):
    """Harness keys -> Oracle / Context.set_params keyword arguments."""
    return dict(iterpre=int(keys.get("iterpre", 2)), iterpost=int(keys.get("iterpost", 2)),
                iterexact=int(keys.get("iterexact", 10)),
                omega=float(keys.get("omega", 0.8)),
                mgomega=float(keys.get("mgomega", 1.0)),
                mgtype=str(keys.get("mgtype", "V")))


def rel(a, b):
    """max |a - b| / max |b| (0 when both are zero)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.abs(b).max() if b.size else 0.0
    d = np.abs(a - b).max() if a.size else 0.0
    return d / s if s > 0 else d


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a - b)


def uniform_meshes(P):
    """Per level (cells, parents) of a uniform unit square/cube hierarchy in the
    problem's node numbering, for gb_level_set_mesh (parents None on level 0)."""
    from oracle.assembly import uniform_cells, uniform_parents
    out = []
    for l, L in enumerate(P.levels):
        cells = uniform_cells(L.coord, P.dim)
        N = round(cells.shape[0] ** (1.0 / P.dim))
        out.append((cells, uniform_parents(P.dim, N) if l > 0 else None))
    return out


def set_uniform_meshes(ctx, P):
    for l, (cells, parents) in enumerate(uniform_meshes(P)):
        ctx.set_mesh(l, P.dim, cells, P.levels[l].coord, parents)


def oracle_level_values(P, kappa_fine, beta=None):
    """The oracle's assembled values of every level from the finest kappa
    (coarse kappa: mean of the children)."""
    from oracle.assembly import assemble, coarsen_kappa, q1_element_matrices
    meshes = uniform_meshes(P)
    kap = [None] * P.nlevels
    kap[-1] = np.asarray(kappa_fine, dtype=np.float64)
    for l in range(P.nlevels - 2, -1, -1):
        kap[l] = coarsen_kappa(kap[l + 1], meshes[l + 1][1], meshes[l][0].shape[0])
    vals = []
    for l, L in enumerate(P.levels):
        cells = meshes[l][0]
        E = q1_element_matrices(P.dim, L.coord[cells], kap[l], beta)
        vals.append(assemble(L.n, L.rowptr, L.col, cells, E, L.dirichlet))
    return vals, kap


def golden_assembly_cases():
    """Golden Q1 cases whose matrices the device assembly rebuilds: (name,
    finest kappa, beta)."""
    from gascoignelib_b200.problem import seeded_inputs
    out = []
    for name, seeded in (("q1_2d_c2_r3_seeded", True), ("q1_3d_c1_r3_seeded", True),
                         ("q1_2d_c2_r4_poisson", False), ("q1_3d_c1_r3_conv_dual", True),
                         ("q1_2d_c2_r4_conv_dual", True)):
        z = np.load(os.path.join(GOLDEN, name + ".npz"))
        dim, coarse, refine = int(z["key_dim"]), int(z["key_coarse"]), int(z["key_refine"])
        kap = (seeded_inputs(dim, coarse, refine)[0] if seeded
               else np.ones((coarse << refine) ** dim))
        beta = ([float(t) for t in str(z["key_conv"]).split(",")] if "key_conv" in z.files
                else None)
        out.append((name, kap, beta))
    return out


def golden_form_cases():
    return [n for n in golden_cases() if n.startswith("form_")]


def golden_kappa_beta(name):
    """Finest kappa and beta of a seeded golden case."""
    from gascoignelib_b200.problem import seeded_inputs
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    dim, coarse, refine = int(z["key_dim"]), int(z["key_coarse"]), int(z["key_refine"])
    beta = ([float(t) for t in str(z["key_conv"]).split(",")] if "key_conv" in z.files
            else None)
    return seeded_inputs(dim, coarse, refine)[0], beta


def uniform_meshes_q2(P):
    """Per level (elements, parents) of a uniform CGQ2 hierarchy (elements =
    patches of 2^dim cells) in the problem's node numbering."""
    from oracle.assembly import uniform_parents, uniform_patches
    out = []
    for l, L in enumerate(P.levels):
        el = uniform_patches(L.coord, P.dim)
        N = round(el.shape[0] ** (1.0 / P.dim))
        out.append((el, uniform_parents(P.dim, N) if l > 0 else None))
    return out


def q2_element_kappa(dim, kappa_cells, Ncells):
    """kappa per finest Q2 element: the mean of its 2^dim cells (the harness's
    coefficient at the element's resolution)."""
    from oracle.assembly import coarsen_kappa, uniform_parents
    return coarsen_kappa(np.asarray(kappa_cells), uniform_parents(dim, Ncells),
                         (Ncells // 2) ** dim)


def oracle_level_values_q2(P, kappa_elements, beta=None):
    from oracle.assembly import assemble, coarsen_kappa, q2_element_matrices
    meshes = uniform_meshes_q2(P)
    kap = [None] * P.nlevels
    kap[-1] = np.asarray(kappa_elements, dtype=np.float64)
    for l in range(P.nlevels - 2, -1, -1):
        kap[l] = coarsen_kappa(kap[l + 1], meshes[l + 1][1], meshes[l][0].shape[0])
    vals = []
    for l, L in enumerate(P.levels):
        el = meshes[l][0]
        E = q2_element_matrices(P.dim, L.coord[el], kap[l], beta)
        vals.append(assemble(L.n, L.rowptr, L.col, el, E, L.dirichlet))
    return vals, kap


def ball_meshes(P, degree):
    """Per level (elements, parents) of a hierarchy whose finest level is a
    uniform mesh with some cells (Q1) or patches (Q2) refined once (hanging
    nodes), the coarser levels uniform."""
    import copy
    from oracle.assembly import refined_elements
    below = copy.copy(P)
    below.levels = P.levels[:-1]
    um = uniform_meshes(below) if degree == 1 else uniform_meshes_q2(below)
    Nc = round(P.levels[-2].n ** (1.0 / P.dim)) - 1      # cells per dim below the ball level
    el, par = refined_elements(P.finest.coord, P.dim, degree, Nc)
    return um + [(el, par)]


def oracle_ball_values(P, degree, kappa_elements, beta=None):
    """The oracle's values of every level of a ball hierarchy (kappa per finest
    element, coarser levels the mean of the children), the finest condensed."""
    from oracle.assembly import (assemble, assemble_hn, coarsen_kappa, condense, hn_maps,
                                 q1_element_matrices, q2_element_matrices)
    meshes = ball_meshes(P, degree)
    f = q1_element_matrices if degree == 1 else q2_element_matrices
    kap = [None] * P.nlevels
    kap[-1] = np.asarray(kappa_elements, dtype=np.float64)
    for l in range(P.nlevels - 2, -1, -1):
        kap[l] = coarsen_kappa(kap[l + 1], meshes[l + 1][1], meshes[l][0].shape[0])
    vals = []
    for l, L in enumerate(P.levels):
        el = meshes[l][0]
        E = f(P.dim, L.coord[el], kap[l], beta)
        if L.hn_edges is not None:
            hn = hn_maps(L, P.dim)
            Ec, ic = condense(E, el, hn)
            vals.append(assemble_hn(L.n, L.rowptr, L.col, ic, Ec, L.dirichlet,
                                    list(hn[0]) + list(hn[1])))
        else:
            vals.append(assemble(L.n, L.rowptr, L.col, el, E, L.dirichlet))
    return vals, kap


def with_condensed_pattern(P, degree):
    """P with the finest level's pattern replaced by the couplings of the
    condensed elements plus every diagonal (the reference's SparseStructure of
    a level with hanging nodes, CGDisc::Structure) and its values carried over
    (zero where P had no entry)."""
    import copy
    import scipy.sparse as sp
    from oracle.assembly import condense, hn_maps
    el = ball_meshes(P, degree)[-1][0]
    L = P.finest
    hn = hn_maps(L, P.dim)
    _, ic = condense(np.zeros((el.shape[0], el.shape[1], el.shape[1])), el, hn)
    nl = ic.shape[1]
    r = np.concatenate([np.repeat(ic, nl, axis=1).ravel(), np.arange(L.n)])
    c = np.concatenate([np.tile(ic, (1, nl)).ravel(), np.arange(L.n)])
    S = sp.coo_matrix((np.ones(r.size), (r, c)), shape=(L.n, L.n)).tocsr()
    S.sum_duplicates()
    S.sort_indices()
    A = sp.csr_matrix((L.val, L.col, L.rowptr), shape=(L.n, L.n))
    out = (abs(A) > 0).astype(np.int8) - (abs(A) > 0).multiply(S > 0).astype(np.int8)
    out.eliminate_zeros()
    assert out.nnz == 0, "an entry outside the element couplings"
    rr = np.repeat(np.arange(L.n), np.diff(S.indptr))
    vals = np.asarray(A[rr, S.indices]).ravel()
    Q = copy.deepcopy(P)
    F = Q.levels[-1]
    F.rowptr = S.indptr.astype(np.int64)
    F.col = S.indices.astype(np.int64)
    F.val = vals
    F.diag = np.nonzero(rr == S.indices)[0].astype(np.int64)
    return Q


def golden_hn_assembly_cases():
    """Golden ball cases (hanging nodes) whose matrices the device assembly
    rebuilds: (name, degree, constant kappa, beta)."""
    out = []
    for name in golden_hn_cases():
        z = np.load(os.path.join(GOLDEN, name + ".npz"))
        beta = ([float(t) for t in str(z["key_conv"]).split(",")] if "key_conv" in z.files
                else None)
        out.append((name, 2 if str(z["key_disc"]) == "Q2" else 1, float(z["key_diff"]), beta))
    return out


def reference_ball_3d(disc, diff, conv=None):
    """Runs the compiled reference on the 3D ball case (coarse 2, refine 3,
    ball 0.25: edge and face hanging nodes) and returns (problem, summary,
    output directory). A ball on a coarser 3D mesh refines every cell (the
    mesh's patch rules), so no smaller 3D case has hanging nodes."""
    import tempfile
    from gascoignelib_b200.problem import load_reference_dump
    from oracle.oracle import run_reference, write_inputs
    d = tempfile.mkdtemp()
    res = 2 * (2 << 3)
    rhs = np.random.default_rng(1002).uniform(-1.0, 1.0, size=(res + 1) ** 3)
    keys = dict(threads=1, dim=3, coarse=2, refine=3, disc=disc, ball=0.25, diff=diff,
                rhsres=res, dump=1, tol=1e-8)
    if conv is not None:
        keys["conv"] = ",".join(str(c) for c in conv)
    out, summ = run_reference(d, **keys, **write_inputs(d, None, rhs))
    return load_reference_dump(out), summ, out


def golden_vtk_cases():
    """Golden cases that hold the reference's VTK file of the solution."""
    out = []
    for n in golden_cases():
        with np.load(os.path.join(GOLDEN, n + ".npz")) as z:
            if "vtk" in z.files:
                out.append(n)
    return out


def vtk_cells(vtk_bytes):
    """The CELLS section of a legacy VTK file: int64 [ncells, nodes per cell]."""
    lines = bytes(vtk_bytes).decode().split("\n")
    i = next(k for k, s in enumerate(lines) if s.startswith("CELLS "))
    ne = int(lines[i].split()[1])
    rows = [[int(t) for t in lines[i + 1 + c].split()][1:] for c in range(ne)]
    return np.array(rows, dtype=np.int64)


def golden_lps_cases():
    """Golden CGQ2Lps / CGQ1Lps cases: (name, mesh degree code for
    set_mesh - 2 Q2 patches, 3 Q1 patches - constant kappa, beta,
    (sdelta0, xeta0))."""
    out = []
    for n in golden_cases():
        if n.startswith("lps_"):
            z = np.load(os.path.join(GOLDEN, n + ".npz"))
            out.append((n, 2 if str(z["key_disc"]) == "Q2" else 3, float(z["key_diff"]),
                        [float(t) for t in str(z["key_conv"]).split(",")],
                        (float(z["key_lps"]), 6.0)))
    return out


def stokes_rhs(dim, coarse, refine, seed=1002):
    """f ~ U[-1, 1] per node and component (p, v_1..v_dim) on the lexicographic
    grid the harness reads, the pressure part made algebraically mean-free so
    that the system with its constant-pressure null space is consistent."""
    n1 = (coarse << refine) + 1
    r = np.random.default_rng(seed).uniform(-1.0, 1.0, size=(n1 ** dim, dim + 1))
    r[:, 0] -= r[:, 0].mean()
    return r.ravel()
