"""The oracle (C restatement) against the reference's own results.

Golden fixtures were produced by the reference's CPU solver (tests/golden/
make_golden.py); where the compiled reference is present (oracle/_ref), more
cases are run against it directly.
"""
import os
import tempfile

import numpy as np
import pytest

from _util import golden_cases, load_golden, rel, rel_l2, solver_keys
from gascoignelib_b200.problem import (load_reference_dump, seeded_inputs,
                                       structured_problem)
from oracle.oracle import REF_HARNESS, Oracle, run_reference, write_inputs

HAVE_REF = os.path.exists(REF_HARNESS)


@pytest.mark.parametrize("name", golden_cases())
def test_oracle_matches_reference_golden(name):
    P, ref = load_golden(name)
    O = Oracle(P, **solver_keys(ref["keys"]))
    x, info = O.gmres(vmax=int(ref["keys"]["gmressize"]), tol=float(ref["keys"]["tol"]))
    assert info["iterations"] == ref["iterations"]
    assert info["status"] == ref["status"]
    # same operations in the same order as the reference: bit-identical
    assert np.array_equal(x, ref["solution"]), rel_l2(x, ref["solution"])
    assert info["firstresidual"] == ref["firstresidual"]


@pytest.mark.skipif(not HAVE_REF, reason="compiled reference not present")
@pytest.mark.parametrize("dim,coarse,refine", [(2, 1, 5), (3, 1, 4), (3, 2, 2)])
def test_oracle_matches_reference_live(dim, coarse, refine):
    kappa, rhs = seeded_inputs(dim, coarse, refine, kappa_seed=7, rhs_seed=8)
    d = tempfile.mkdtemp()
    out, summ = run_reference(d, dim=dim, coarse=coarse, refine=refine, dump=1,
                              tol=1e-9, **write_inputs(d, kappa, rhs))
    P = load_reference_dump(out)
    x, info = Oracle(P).gmres(vmax=21, tol=1e-9)
    assert info["iterations"] == int(summ["iterations"][0])
    assert np.array_equal(x, np.fromfile(os.path.join(out, "solution.f64")))


@pytest.mark.skipif(not HAVE_REF, reason="compiled reference not present")
@pytest.mark.parametrize("dim,smoother,omega", [(2, "vanka", 1.0), (2, "jacobi", 0.5),
                                                (3, "jacobi", 0.5)])
def test_oracle_matches_reference_live_stokes(dim, smoother, omega):
    """Block systems (ncomp = dim+1), pressure filter, Vanka / block Jacobi."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_golden import stokes_rhs
    coarse, refine = (2, 3) if dim == 2 else (1, 3)
    d = tempfile.mkdtemp()
    out, summ = run_reference(d, threads=1, dim=dim, coarse=coarse, refine=refine,
                              dump=1, tol=1e-9, problem="stokes", smoother=smoother,
                              omega=omega, gmressize=31, maxiter=200,
                              **write_inputs(d, None, stokes_rhs(dim, coarse, refine, 9)))
    P = load_reference_dump(out)
    P.info["smoother"] = smoother
    x, info = Oracle(P, omega=omega).gmres(vmax=31, tol=1e-9, maxiter=200)
    assert info["iterations"] == int(summ["iterations"][0])
    assert np.array_equal(x, np.fromfile(os.path.join(out, "solution.f64")))


def _lex_permutation(level, N, dim):
    idx = np.rint(level.coord * N).astype(np.int64)
    lex = np.zeros(level.n, np.int64)
    for d in reversed(range(dim)):
        lex = lex * (N + 1) + idx[:, d]
    return lex


@pytest.mark.parametrize("name", ["q1_2d_c2_r3_seeded", "q1_3d_c1_r3_seeded",
                                  "q1_2d_c2_r4_poisson"])
def test_structured_generator_matches_reference_assembly(name):
    """The synthetic generator assembles the reference's operators (same values
    up to rounding, same sparsity, same Dirichlet and transfer maps) in
    lexicographic numbering."""
    import scipy.sparse as sp
    P, ref = load_golden(name)
    dim = P.dim
    coarse = 2 if dim == 2 else 1
    refine = P.nlevels
    seeded = "seeded" in name
    kappa, rhs = seeded_inputs(dim, coarse, refine) if seeded else (None, None)
    G = structured_problem(dim, coarse, refine, kappa, rhs)
    assert G.nlevels == P.nlevels
    perms = []
    for l in range(P.nlevels):
        N = (2 * coarse) << l
        lex = _lex_permutation(P.levels[l], N, dim)
        perms.append(lex)
        lr, lg = P.levels[l], G.levels[l]
        rows = np.repeat(np.arange(lr.n), np.diff(lr.rowptr))
        # permute by index arithmetic (keeps the explicit zeros of the stencil)
        Arl = sp.coo_matrix((lr.val, (lex[rows], lex[lr.col])), shape=(lr.n, lr.n)).tocsr()
        Arl.sort_indices()
        assert lr.nnzb == lg.nnzb
        assert np.array_equal(Arl.indptr, lg.rowptr) and np.array_equal(Arl.indices, lg.col)
        assert rel(Arl.data, lg.val) < 1e-13
        assert np.array_equal(np.sort(lex[lr.dirichlet]), np.sort(lg.dirichlet))
    # transfers: the same (fine, coarse) couplings
    for l, (tr, tg) in enumerate(zip(P.transfers, G.transfers)):
        pc, pf = perms[l], perms[l + 1]

        def pairs(t, mc, mf):
            s = {(int(mf[f]), int(mc[c])) for c, f in enumerate(t.c2f)}
            for arr in (t.zweier, t.vierer, t.achter):
                for row in arr:
                    s |= {(int(mf[row[0]]), int(mc[q])) for q in row[1:]}
            return s
        ident_c = np.arange(G.levels[l].n)
        ident_f = np.arange(G.levels[l + 1].n)
        assert pairs(tr, pc, pf) == pairs(tg, ident_c, ident_f)
    # rhs and solution: same problem => same solution after permutation
    x, info = Oracle(G).gmres(vmax=21, tol=float(ref["keys"]["tol"]))
    xr = np.empty_like(ref["solution"])
    xr[perms[-1]] = ref["solution"]
    assert abs(info["iterations"] - ref["iterations"]) <= 1
    assert rel_l2(x, xr) < 1e-8


def test_oracle_operator_identities():
    """Adjoint identity of the transposed product and of R = P^T."""
    kappa, rhs = seeded_inputs(3, 1, 3)
    P = structured_problem(3, 1, 3, kappa, rhs)
    O = Oracle(P)
    rng = np.random.default_rng(3)
    fl = P.nlevels - 1
    n = P.finest.n
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    Ax = O.vmult(fl, np.zeros(n), x)
    ATy = O.vmult_transpose(fl, np.zeros(n), y)
    assert abs(y @ Ax - x @ ATy) < 1e-12 * np.linalg.norm(Ax) * np.linalg.norm(y)
    nc = P.levels[fl - 1].n
    xc = rng.standard_normal(nc)
    Rx = O.restrict_zero(fl - 1, x)
    Pxc = O.prolongate_add(fl - 1, np.zeros(n), xc)
    assert abs(xc @ Rx - x @ Pxc) < 1e-12 * np.linalg.norm(Rx) * np.linalg.norm(xc)


def test_oracle_zero_rhs_returns_immediately():
    P = structured_problem(2, 2, 3)
    x, info = Oracle(P).gmres(b=np.zeros(P.finest.n))
    assert info["reached"] == 1 and info["iterations"] == 0
    assert not x.any()


def test_oracle_maxiter_stops():
    kappa, rhs = seeded_inputs(2, 2, 4)
    P = structured_problem(2, 2, 4, kappa, rhs)
    x, info = Oracle(P).gmres(vmax=21, tol=1e-14, maxiter=3)
    assert info["status"] == "too many iterations" and info["iterations"] == 4


@pytest.mark.parametrize("name", ["stokes_2d_c2_r4_vanka", "stokes_3d_c1_r3_vanka"])
def test_structured_stokes_matches_reference_assembly(name):
    """problem.structured_stokes (lexicographic numbering) builds the
    reference's Stokes matrices, Dirichlet masks, pressure-filter weights and
    Vanka patches."""
    from gascoignelib_b200.problem import structured_stokes
    P, ref = load_golden(name)
    keys = ref["keys"]
    S = structured_stokes(P.dim, int(keys["coarse"]), int(keys["refine"]))
    assert S.nlevels == P.nlevels
    for Lr, Ls in zip(P.levels, S.levels):
        N = round(Ls.n ** (1.0 / P.dim)) - 1
        perm = _lex_permutation(Lr, N, P.dim)
        B = Ls.B
        assert Lr.B == B and Lr.dircomp_mask == Ls.dircomp_mask
        # same blocks at the same (row, col) node pairs
        kr = perm[np.repeat(np.arange(Lr.n), np.diff(Lr.rowptr))] * Lr.n + perm[Lr.col]
        ks = np.repeat(np.arange(Ls.n), np.diff(Ls.rowptr)) * Ls.n + Ls.col
        orr, oss = np.argsort(kr), np.argsort(ks)
        assert np.array_equal(kr[orr], ks[oss])
        vr = Lr.val.reshape(-1, B, B)[orr]
        vs = Ls.val.reshape(-1, B, B)[oss]
        assert np.abs(vr - vs).max() <= 1e-13 * np.abs(vr).max()
        w = np.empty(Lr.n)
        w[perm] = Lr.pf_weights
        assert np.abs(w - Ls.pf_weights).max() <= 1e-15
        assert Lr.pf_domain == pytest.approx(Ls.pf_domain, rel=1e-14)
        assert {tuple(sorted(perm[p])) for p in Lr.patches} == \
            {tuple(sorted(p)) for p in Ls.patches}
        dr = np.zeros(Lr.n, bool)
        dr[perm[Lr.dirichlet]] = True
        ds = np.zeros(Ls.n, bool)
        ds[Ls.dirichlet] = True
        assert np.array_equal(dr, ds)


def _hn_test_vector(P):
    n, B = P.finest.n, P.finest.B
    return np.sin(1.0 + np.arange(n * B))


@pytest.mark.parametrize("name", [n for n in golden_cases() if n.startswith("hn_")])
def test_oracle_hanging_node_ops_match_reference(name):
    """HNAverage / HNDistribute / HNZero of the reference's HNStructure on the
    finest level (ball refinement), bit for bit."""
    P, ref = load_golden(name)
    O = Oracle(P, **solver_keys(ref["keys"]))
    t = _hn_test_vector(P)
    l = P.nlevels - 1
    assert P.finest.hn_edges.shape[0] > 0
    for op in ("average", "distribute", "zero"):
        assert np.array_equal(O.hn(op, l, t), ref["hn_" + op]), op


@pytest.mark.skipif(not HAVE_REF, reason="compiled reference not present")
@pytest.mark.parametrize("disc", ["Q1", "Q2"])
def test_oracle_hanging_nodes_3d_live(disc):
    """3D ball refinement (edge and face hanging nodes; Q13d / Q23d weights):
    HN operations and the solve against the compiled reference."""
    d = tempfile.mkdtemp()
    res = 2 * (2 << 3)
    rhs = np.random.default_rng(1002).uniform(-1.0, 1.0, size=(res + 1) ** 3)
    kw = write_inputs(d, None, rhs)
    out, summ = run_reference(d, threads=1, dim=3, coarse=2, refine=3, disc=disc,
                              ball=0.25, diff=1.0, rhsres=res, dump=1, tol=1e-8, **kw)
    P = load_reference_dump(out)
    assert P.finest.hn_faces.shape[0] > 0 and P.finest.hn_edges.shape[0] > 0
    O = Oracle(P)
    t = _hn_test_vector(P)
    l = P.nlevels - 1
    for op in ("average", "distribute", "zero"):
        assert np.array_equal(O.hn(op, l, t), np.fromfile(os.path.join(out, f"hn_{op}.f64")))
    x, info = O.gmres(vmax=21, tol=1e-8)
    assert info["iterations"] == int(summ["iterations"][0])
    assert np.array_equal(x, np.fromfile(os.path.join(out, "solution.f64")))


@pytest.mark.skipif(not HAVE_REF, reason="compiled reference not present")
@pytest.mark.parametrize("dim,coarse,refine", [(2, 2, 3), (3, 1, 3)])
def test_structured_q2_matches_reference_assembly(dim, coarse, refine):
    """problem.structured_q2 builds the reference's CGQ2 convection-diffusion
    matrices (the bench's Q2 workload) in lexicographic numbering."""
    import scipy.sparse as sp
    from gascoignelib_b200.problem import structured_q2
    N = coarse << refine
    rhs = np.random.default_rng(1002).uniform(-1, 1, size=(N + 1) ** dim)
    d = tempfile.mkdtemp()
    out, summ = run_reference(d, threads=1, dim=dim, coarse=coarse, refine=refine,
                              disc="Q2", diff=0.1, conv="1,0.5,0.25", dump=1,
                              **write_inputs(d, None, rhs))
    R = load_reference_dump(out)
    P = structured_q2(dim, coarse, refine, eps=0.1, rhs=rhs)
    for Lr, Lp in zip(R.levels, P.levels):
        Nl = round(Lp.n ** (1.0 / dim)) - 1
        perm = _lex_permutation(Lr, Nl, dim)
        Ar = sp.csr_matrix((Lr.val, Lr.col, Lr.rowptr), shape=(Lr.n, Lr.n)).tocoo()
        Ar = sp.csr_matrix((Ar.data, (perm[Ar.row], perm[Ar.col])), shape=(Lr.n, Lr.n))
        Ap = sp.csr_matrix((Lp.val, Lp.col, Lp.rowptr), shape=(Lp.n, Lp.n))
        assert Ar.nnz == Ap.nnz
        assert abs(Ar - Ap).max() <= 1e-12 * abs(Ap).max()
    x, info = Oracle(P).gmres(vmax=21, tol=1e-8)
    u_ref = np.empty(P.finest.n)
    u_ref[_lex_permutation(R.finest, N, dim)] = np.fromfile(os.path.join(out, "solution.f64"))
    assert abs(info["iterations"] - int(summ["iterations"][0])) <= 1
    assert rel_l2(x, u_ref) < 1e-7


def test_oracle_direct_coarse_solve_is_exact():
    """The coarsest-level direct solve (ndirect, the reference's UMFPACK
    branch of smooth_exact): on a one-level problem the preconditioner is the
    exact inverse, so the first GMRES iterate already solves the system."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    from gascoignelib_b200.problem import Problem, seeded_inputs, structured_problem

    kappa, rhs = seeded_inputs(3, 1, 4)
    P = structured_problem(3, 1, 4, kappa, rhs)
    L = P.levels[2]
    b = np.random.default_rng(0).uniform(-1.0, 1.0, L.n)
    b[L.dirichlet] = 0.0
    P1 = Problem(dim=3, levels=[L], transfers=[], rhs=b, info={})
    A = sp.csr_matrix((L.val, L.col, L.rowptr), shape=(L.n, L.n)).tocsc()
    x, info = Oracle(P1, ndirect=1000).gmres(vmax=21, tol=1e-8)
    assert info["status"] == "converged"
    assert info["firstresidual"] < 1e-12 * np.linalg.norm(b)
    assert np.linalg.norm(x - spl.spsolve(A, b)) < 1e-13 * np.linalg.norm(x)
    # below the threshold the iterexact sweeps run (a different preconditioner)
    _, info2 = Oracle(P1, ndirect=L.n).gmres(vmax=21, tol=1e-8)
    assert info2["firstresidual"] > 1e-6 * np.linalg.norm(b)
