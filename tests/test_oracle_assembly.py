"""The oracle's Q1 assembly (oracle/assembly.py) against the matrices the
reference assembled (golden fixtures: every level, seeded per-cell kappa,
with and without convection), and against the generator's assembly."""
import os

import numpy as np
import pytest

from _util import (ball_meshes, golden_assembly_cases, golden_hn_assembly_cases, golden_lps_cases,
                   golden_vtk_cases,
                   load_golden, oracle_ball_values, oracle_level_values, reference_ball_3d,
                   vtk_cells, with_condensed_pattern)
from gascoignelib_b200.problem import seeded_inputs, structured_problem, structured_q2_ball
from oracle.assembly import q1_element_matrices
from oracle.oracle import REF_HARNESS


@pytest.mark.parametrize("name,kappa,beta", golden_assembly_cases(),
                         ids=[c[0] for c in golden_assembly_cases()])
def test_oracle_assembly_matches_reference(name, kappa, beta):
    P, _ = load_golden(name)
    vals, _ = oracle_level_values(P, kappa, beta)
    for L, v in zip(P.levels, vals):
        assert np.abs(v - L.val).max() <= 1e-13 * np.abs(L.val).max()


def test_element_matrix_of_a_distorted_cell():
    """A non-affine hexahedron: rows of the diffusion part sum to zero (constants
    are in its kernel) and the matrix is symmetric; an affine map of the unit
    cube gives the tensor-product matrix of a box."""
    rng = np.random.default_rng(3)
    corners = np.array([[(a >> d) & 1 for d in range(3)] for a in range(8)], dtype=float)
    x = corners + 0.15 * rng.uniform(-1, 1, size=corners.shape)
    E = q1_element_matrices(3, x[None], np.array([2.0]))[0]
    assert np.abs(E.sum(axis=1)).max() < 1e-14
    assert np.abs(E - E.T).max() < 1e-14
    box = corners * np.array([0.5, 0.25, 2.0])
    Eb = q1_element_matrices(3, box[None], np.array([1.0]))[0]
    m = lambda h: np.array([[1 / 3, 1 / 6], [1 / 6, 1 / 3]]) * h
    s = lambda h: np.array([[1.0, -1.0], [-1.0, 1.0]]) / h
    ref = (np.kron(np.kron(m(2.0), m(0.25)), s(0.5)) + np.kron(np.kron(m(2.0), s(0.25)), m(0.5))
           + np.kron(np.kron(s(2.0), m(0.25)), m(0.5)))
    assert np.abs(Eb - ref).max() < 1e-14 * np.abs(ref).max()


def test_oracle_assembly_matches_generator():
    kappa, rhs = seeded_inputs(3, 1, 4)
    P = structured_problem(3, 1, 4, kappa, rhs, beta=(1.0, -0.5, 0.25))
    vals, _ = oracle_level_values(P, kappa, (1.0, -0.5, 0.25))
    for L, v in zip(P.levels, vals):
        assert np.abs(v - L.val).max() <= 1e-13 * np.abs(L.val).max()


@pytest.mark.parametrize("name", __import__("_util").golden_form_cases())
def test_oracle_form_and_newton_residual_match_reference(name):
    """StdSolver::Form and StdMultiLevelSolver::NewtonResidual of a seeded
    vector, restated as the sum of the element matrices applied per cell."""
    from _util import golden_kappa_beta, uniform_meshes
    P, ref = load_golden(name)
    kappa, beta = golden_kappa_beta(name)
    L = P.finest
    cells = uniform_meshes(P)[-1][0]
    E = q1_element_matrices(P.dim, L.coord[cells], kappa, beta)
    x = ref["formx"]
    F = np.zeros(L.n)
    for c in range(cells.shape[0]):
        F[cells[c]] += E[c] @ x[cells[c]]
    assert np.abs(F - ref["form"]).max() <= 1e-13 * np.abs(ref["form"]).max()
    y = P.rhs - F
    y[L.dirichlet] = 0.0
    assert np.abs(y - ref["newton_residual"]).max() <= 1e-13 * np.abs(y).max()
    assert abs(np.abs(y).max() - ref["newton_norm"]) <= 1e-13 * ref["newton_norm"]


@pytest.mark.parametrize("name", __import__("_util").golden_form_cases())
def test_backup_formats_match_reference_files(name):
    """WriteBackUp / WriteBackUpBinary layouts restated in numpy reproduce the
    reference's files byte for byte (the library's writer is checked against
    the same bytes on the GPU)."""
    P, ref = load_golden(name)
    u = ref["solution"]
    B = P.finest.B
    txt = f"{P.finest.n} {B}\n" + "".join(
        "".join(f"{u[i * B + c]:.16e} " for c in range(B)) + "\n" for i in range(P.finest.n))
    txt += "BackUpEnd\n"
    assert txt.encode() == ref["backup_bup"].tobytes()
    bip = f"{B} {P.finest.n}\n[".encode() + u.astype("<f8").tobytes() + b"]BackUpEnd\n"
    assert bip == ref["backup_bip"].tobytes()


def _q2_golden():
    from _util import golden_cases
    return [n for n in golden_cases() if n.startswith("q2_")]


@pytest.mark.parametrize("name", _q2_golden())
def test_oracle_q2_assembly_matches_reference(name):
    """CGQ2 elements with the per-cell kappa (per element: the mean of its
    cells) and LineGauss3 as the reference states it."""
    from _util import golden_kappa_beta, oracle_level_values_q2, q2_element_kappa
    P, _ = load_golden(name)
    kappa, beta = golden_kappa_beta(name)
    Nc = round(len(kappa) ** (1.0 / P.dim))
    vals, _ = oracle_level_values_q2(P, q2_element_kappa(P.dim, kappa, Nc), beta)
    for L, v in zip(P.levels, vals):
        assert np.abs(v - L.val).max() <= 1e-13 * np.abs(L.val).max()


@pytest.mark.parametrize("name,degree,diff,beta", golden_hn_assembly_cases(),
                         ids=[c[0] for c in golden_hn_assembly_cases()])
def test_oracle_hn_assembly_matches_reference(name, degree, diff, beta):
    """The condensed element matrices of a ball-refined level (hanging nodes)
    and the uniform levels below it reproduce the reference's matrices."""
    P, _ = load_golden(name)
    ne = ball_meshes(P, degree)[-1][0].shape[0]
    vals, _ = oracle_ball_values(P, degree, np.full(ne, diff), beta)
    for l, L in enumerate(P.levels):
        assert np.abs(vals[l] - L.val).max() <= 1e-13 * np.abs(L.val).max(), l


def test_oracle_hn_condensation_matches_generator():
    """3D Q2 with hanging edge and face nodes: the oracle's element condensation
    equals the generator's global C^T A C (whose Gauss weights are exact, hence
    1e-12), and the generator's pattern lies inside the condensed couplings."""
    P = with_condensed_pattern(structured_q2_ball(1, 3, eps=0.1), 2)
    assert P.finest.hn_faces.shape[0] > 0 and P.finest.hn_edges.shape[0] > 0
    ne = ball_meshes(P, 2)[-1][0].shape[0]
    vals, _ = oracle_ball_values(P, 2, np.full(ne, 0.1), (1.0, 0.5, 0.25))
    for l, L in enumerate(P.levels):
        assert np.abs(vals[l] - L.val).max() <= 1e-12 * np.abs(L.val).max(), l


def test_condense_plants():
    """A planted wrong weight changes the condensed matrix (the comparison is
    sensitive to the condensation), and a cell holding every parent of its
    hanging node is rejected."""
    from oracle.assembly import condense
    E = np.arange(16.0).reshape(1, 4, 4) + 1.0
    cells = np.array([[0, 1, 2, 3]])
    Eg, ig = condense(E, cells, ({1: [(0, 0.5), (7, 0.5)]}, {}))
    Eb, _ = condense(E, cells, ({1: [(0, 0.5), (7, 0.25)]}, {}))
    assert ig.tolist() == [[0, 7, 2, 3]] and not np.allclose(Eg, Eb)
    # C^T E C with u_1 = (u_0 + u_7) / 2, the element now on (0, 7, 2, 3)
    C = np.zeros((4, 4))
    C[0, 0] = C[2, 2] = C[3, 3] = 1.0
    C[1, 0] = C[1, 1] = 0.5
    assert np.allclose(Eg[0], C.T @ E[0] @ C)
    with pytest.raises(AssertionError):
        condense(E, cells, ({1: [(0, 0.5), (2, 0.5)]}, {}))


@pytest.mark.skipif(not os.path.exists(REF_HARNESS), reason="compiled reference not present")
@pytest.mark.parametrize("disc,diff,conv", [("Q1", 1.0, None), ("Q2", 0.1, (1.0, 0.5, 0.25))])
def test_oracle_hn_assembly_3d_live(disc, diff, conv):
    """3D ball refinement (edge and face hanging nodes, HNStructureQ13d /
    Q23d condensation): the oracle's levels against the reference's matrices."""
    P, _, _ = reference_ball_3d(disc, diff, conv)
    assert P.finest.hn_faces.shape[0] > 0 and P.finest.hn_edges.shape[0] > 0
    degree = 2 if disc == "Q2" else 1
    ne = ball_meshes(P, degree)[-1][0].shape[0]
    vals, _ = oracle_ball_values(P, degree, np.full(ne, diff), conv)
    for l, L in enumerate(P.levels):
        assert np.abs(vals[l] - L.val).max() <= 1e-13 * np.abs(L.val).max(), l


@pytest.mark.parametrize("name", golden_vtk_cases())
def test_vtk_layout_matches_reference_file(name):
    """Visualization::vtk's layout (Discretization/Q1/vtk.cc) restated in
    Python reproduces the reference's file byte for byte from the level's
    coordinates, the file's cells and the HN-averaged solution (the library's
    writer is checked against the same bytes on the GPU)."""
    from oracle.oracle import Oracle
    P, ref = load_golden(name)
    F = P.finest
    u = ref["solution"]
    if F.hn_edges is not None:
        u = Oracle(P).hn("average", P.nlevels - 1, u)
    cells = vtk_cells(ref["vtk"])
    dim = P.dim
    t = ("# vtk DataFile Version 2.0 \noutput from GascoigneStd, \nASCII\n"
         "DATASET UNSTRUCTURED_GRID\nFIELD FieldData 1\nTIME 1 1 double\n0\n")
    t += f"POINTS {F.n} DOUBLE \n"
    t += "".join("".join(f"{x:g}\t" for x in F.coord[i]) + (" 0\n" if dim == 2 else "\n")
                 for i in range(F.n))
    t += f"\n\nCELLS {cells.shape[0]} {cells.size + cells.shape[0]}\n"
    t += "".join(f"{cells.shape[1]} " + "".join(f"{v} " for v in c) + "\n" for c in cells)
    t += f"\nCELL_TYPES {cells.shape[0]}\n" + ("9 " if dim == 2 else "12 ") * cells.shape[0]
    t += f"\nPOINT_DATA {F.n}\n"
    for comp in range(F.B):
        t += f"SCALARS u{comp:03d} DOUBLE \nLOOKUP_TABLE default\n"
        t += "".join(f"{u[i * F.B + comp]:g}\n" for i in range(F.n)) + "\n\n"
    assert t.encode() == ref["vtk"].tobytes()


@pytest.mark.parametrize("name,kind,diff,beta,lps", golden_lps_cases(),
                         ids=[c[0] for c in golden_lps_cases()])
def test_oracle_lps_assembly_matches_reference(name, kind, diff, beta, lps):
    """CGQ2Lps / CGQ1Lps (local projection stabilisation of the convection):
    the oracle's patch element matrices (Q2, or Q1 functions on patches) with
    the projected LPS term reproduce the reference's matrices on every level;
    without the term they do not."""
    from _util import uniform_meshes_q2
    from oracle.assembly import assemble, q1patch_element_matrices, q2_element_matrices
    f = q2_element_matrices if kind == 2 else q1patch_element_matrices
    P, _ = load_golden(name)
    for l, (el, _) in enumerate(uniform_meshes_q2(P)):
        L = P.levels[l]
        kap = np.full(el.shape[0], diff)
        v = assemble(L.n, L.rowptr, L.col, el, f(P.dim, L.coord[el], kap, beta, lps),
                     L.dirichlet)
        assert np.abs(v - L.val).max() <= 1e-13 * np.abs(L.val).max(), l
        w = assemble(L.n, L.rowptr, L.col, el, f(P.dim, L.coord[el], kap, beta), L.dirichlet)
        assert np.abs(w - L.val).max() > 1e-3 * np.abs(L.val).max(), l


def _patch_form_cases():
    from _util import golden_cases
    out = []
    for n in golden_cases():
        if not n.startswith("form_"):
            with np.load(os.path.join(os.path.dirname(__file__), "golden", n + ".npz")) as z:
                if "formx" in z.files:
                    out.append(n)
    return out


@pytest.mark.parametrize("name", _patch_form_cases())
def test_oracle_form_on_patch_and_hanging_levels_matches_reference(name):
    """StdSolver::Form restated (Solver/stdsolver.cc:1041-1063): HNAverage of x,
    the uncondensed element matrices times the local values added at the
    cells' own nodes, HNDistribute of the result; the reference's Form of a
    seeded vector within 1e-13 (Q2, Q1 on patches with LPS, hanging nodes)."""
    from _util import golden_kappa_beta, golden_lps_cases, q2_element_kappa, uniform_meshes_q2
    from oracle.assembly import (q1_element_matrices, q1patch_element_matrices,
                                 q2_element_matrices)
    from oracle.oracle import Oracle
    P, ref = load_golden(name)
    keys = ref["keys"]
    F = P.finest
    lps = None
    if name.startswith("hn_"):
        deg = 2 if str(keys["disc"]) == "Q2" else 1
        el = ball_meshes(P, deg)[-1][0]
        kap = np.full(el.shape[0], float(keys["diff"]))
        beta = ([float(t) for t in str(keys["conv"]).split(",")] if "conv" in keys else None)
    elif name.startswith("lps_"):
        _, deg, diff, beta, lps = next(c for c in golden_lps_cases() if c[0] == name)
        el = uniform_meshes_q2(P)[-1][0]
        kap = np.full(el.shape[0], diff)
    else:
        deg = 2
        kappa, beta = golden_kappa_beta(name)
        el = uniform_meshes_q2(P)[-1][0]
        kap = q2_element_kappa(P.dim, kappa, round(len(kappa) ** (1.0 / P.dim)))
    f = {1: q1_element_matrices, 2: q2_element_matrices, 3: q1patch_element_matrices}[deg]
    E = f(P.dim, F.coord[el], kap, beta) if lps is None else f(P.dim, F.coord[el], kap, beta,
                                                               lps)
    x = ref["formx"]
    O = Oracle(P)
    fl = P.nlevels - 1
    if F.hn_edges is not None:
        x = O.hn("average", fl, x)
    y = np.zeros(F.n)
    np.add.at(y, el, np.einsum("cab,cb->ca", E, x[el]))
    if F.hn_edges is not None:
        y = O.hn("distribute", fl, y)
    assert np.abs(y - ref["form"]).max() <= 1e-13 * np.abs(ref["form"]).max()
