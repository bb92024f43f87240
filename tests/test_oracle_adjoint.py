"""The adjoint side of the oracle, pinned to the reference's dual solve.

The "_dual" golden fixtures hold what the reference's own CPU solver did for
a nonsymmetric (convection-diffusion) operator: StdMultiLevelSolver::
AssembleDualMatrix (transpose, Dirichlet rows) on every level, then the same
Gmres/LinearMg on it, for the right-hand side dJ/du = 2 M u of J = int u^2.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as sla

from _util import (dual_problem, golden_dual_cases, load_golden, reference_cells, rel_l2,
                   solver_keys)
from gascoignelib_b200.problem import seeded_inputs, structured_problem
from oracle.oracle import Oracle, coeff_gradient, transposed_problem


def _csr(L):
    return sp.csr_matrix((L.val, L.col, L.rowptr), shape=(L.n, L.n))


@pytest.mark.parametrize("name", golden_dual_cases())
def test_oracle_dual_solve_is_the_reference_dual_solve(name):
    """On the reference's own dual matrices the oracle's GMRES reproduces the
    reference's dual solution bit for bit."""
    P, ref = load_golden(name)
    keys = ref["keys"]
    O = Oracle(dual_problem(P, ref), **solver_keys(keys))
    lam, info = O.gmres(ref["dual_rhs"], vmax=int(keys["gmressize"]), tol=float(keys["tol"]))
    assert info["iterations"] == ref["dual_iterations"]
    assert info["firstresidual"] == ref["dual_firstresidual"]
    assert np.array_equal(lam, ref["dual_solution"])


@pytest.mark.parametrize("name", golden_dual_cases())
def test_in_stencil_transpose_matches_reference_dual_matrix(name):
    """The transpose of the uploaded forward matrices is the reference's dual
    matrix on every non-Dirichlet column (up to the last bit of the
    reference's re-assembly), and solving with it gives the reference's dual
    solution."""
    P, ref = load_golden(name)
    PT = transposed_problem(P)
    for l, (L, Lt) in enumerate(zip(P.levels, PT.levels)):
        dm = np.zeros(L.n, dtype=bool)
        dm[L.dirichlet] = True
        keep = ~dm[L.col]
        dv = ref["dualval"][l]
        scale = np.abs(dv).max()
        assert np.abs(Lt.val[keep] - dv[keep]).max() <= 4e-16 * scale
        assert np.array_equal(_csr(Lt).toarray(), _csr(L).toarray().T)
    # nonsymmetric: the dual differs from the forward operator
    A = _csr(P.finest)
    assert abs(A - A.T).max() > 1e-3
    keys = ref["keys"]
    O = Oracle(PT, **solver_keys(keys))
    lam, info = O.gmres(ref["dual_rhs"], vmax=int(keys["gmressize"]), tol=float(keys["tol"]))
    assert abs(info["iterations"] - ref["dual_iterations"]) <= 1
    assert rel_l2(lam, ref["dual_solution"]) < 1e-10


@pytest.mark.parametrize("name", golden_dual_cases())
def test_dual_rhs_is_l2_functional_derivative(name):
    """The fixture's dual right-hand side is 2 M u (zeroed on Dirichlet
    nodes) for the reference's forward solution."""
    P, ref = load_golden(name)
    cells = reference_cells(P)
    M = cells.assemble(cells.mloc, P.finest.n)
    g = 2.0 * (M @ ref["solution"])
    g[P.finest.dirichlet] = 0.0
    assert rel_l2(g, ref["dual_rhs"]) < 1e-12


@pytest.mark.parametrize("name", golden_dual_cases())
def test_gradient_from_reference_dual_matches_direct_fd(name):
    """dJ/dkappa from the reference's u and dual lambda agrees with central
    differences (h = 1e-6) of J = u^T M u through direct sparse solves of the
    reference's own matrices rebuilt with kappa_c perturbed."""
    P, ref = load_golden(name)
    cells = reference_cells(P)
    g = coeff_gradient(cells, ref["solution"], ref["dual_solution"], P.finest.dirichlet)
    A = _csr(P.finest).tolil()
    M = cells.assemble(cells.mloc, P.finest.n)
    dm = np.zeros(P.finest.n, dtype=bool)
    dm[P.finest.dirichlet] = True
    b = P.rhs

    def J(c, h):
        # A(kappa_c + h): add h * kloc on the cell's non-Dirichlet rows/cols
        Ah = A.copy()
        nd = cells.nodes[c]
        for a in range(nd.size):
            for e in range(nd.size):
                if not dm[nd[a]] and not dm[nd[e]]:
                    Ah[nd[a], nd[e]] += h * cells.kloc[a, e]
        u = sla.spsolve(Ah.tocsc(), b)
        return u @ (M @ u)

    rng = np.random.default_rng(1003)
    pick = rng.choice(cells.ncells, size=8, replace=False)
    h = 1e-6
    fd = np.array([(J(c, h) - J(c, -h)) / (2 * h) for c in pick])
    # reference solves stop at tol, so agreement is at that level
    assert np.abs(fd - g[pick]).max() <= 1e-4 * np.abs(g).max()


def test_adjoint_oracle_structured_nonsymmetric():
    """Oracle on the transposed structured problem solves A^T lam = g
    (checked against a direct solve)."""
    kappa, rhs = seeded_inputs(2, 2, 4)
    P = structured_problem(2, 2, 4, kappa, rhs, beta=(4.0, 2.0))
    PT = transposed_problem(P)
    g = np.random.default_rng(11).uniform(-1, 1, P.finest.n)
    g[P.finest.dirichlet] = 0.0
    lam, info = Oracle(PT).gmres(g, vmax=21, tol=1e-12, globaltol=1e-300)
    A = _csr(P.finest)
    lam_d = sla.spsolve(A.T.tocsc(), g)
    assert info["status"] == "converged"
    assert rel_l2(lam, lam_d) < 1e-9


def test_coeff_gradient_masks_dirichlet_and_scales():
    kappa, rhs = seeded_inputs(2, 2, 3)
    P = structured_problem(2, 2, 3, kappa, rhs)
    c = P.cells
    rng = np.random.default_rng(3)
    u = rng.normal(size=P.finest.n)
    lam = rng.normal(size=P.finest.n)
    g = coeff_gradient(c, u, lam, P.finest.dirichlet)
    u0, l0 = u.copy(), lam.copy()
    u0[P.finest.dirichlet] = 0
    l0[P.finest.dirichlet] = 0
    K = c.assemble(c.kloc, P.finest.n)
    # sum over cells of the gradient = -lam^T K u (masked)
    assert abs(g.sum() + l0 @ (K @ u0)) < 1e-12 * abs(l0 @ (K @ u0)) + 1e-14
    c.scale = np.full(c.ncells, 2.0)
    assert np.allclose(coeff_gradient(c, u, lam, P.finest.dirichlet), 2 * g, rtol=0,
                       atol=1e-15)
