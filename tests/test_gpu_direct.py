"""The coarsest-level direct solve (the ndirect key: StdSolver::smooth_exact's
exact solve on a direct level) on the GPU: the FP64 inverse applied in the
forward and transposed cycles, in the single-CTA coarse program, the dense
coarse maps and the per-level kernels, against the oracle's LU solve."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from _util import rel_l2
from gascoignelib_b200.native import GB_FP32, GB_FP64, GBError
from gascoignelib_b200.problem import (Problem, seeded_inputs, structured_problem,
                                       structured_q2_ball, structured_stokes)
from oracle.oracle import Oracle, transposed_problem

pytestmark = pytest.mark.gpu


def _solve_pair(ctx, P, keys, oracle_problem=None, adjoint=False):
    O = Oracle(oracle_problem or P, ndirect=keys["ndirect"], omega=keys["omega"])
    xo, io = O.gmres(vmax=keys["gmressize"], tol=1e-8, globaltol=1e-300)
    ctx.load_problem(P)
    ctx.set_params(tol=1e-8, globaltol=1e-300, maxiter=200, **keys)
    l = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(l, b, P.rhs)
    info = ctx.adjoint_gmres(x, b) if adjoint else ctx.gmres(x, b)
    xg = ctx.download(l, x)
    ctx.free(x)
    ctx.free(b)
    return xo, io, xg, info


@pytest.mark.parametrize("env", [{}, {"GB_COARSE_DENSE": "0"}, {"GB_COARSE_KERNEL": "0"}])
def test_direct_coarse_q2_ball_matches_oracle(monkeypatch, env):
    """Q2 with the refined ball (hanging nodes: the generic dense map carries the
    direct solve), and the scalar Jacobi Q1 problem (single-CTA program, its
    dense map, or the per-level kernels)."""
    from gascoignelib_b200.build import build_library
    from gascoignelib_b200.native import Context

    for k, v in env.items():
        monkeypatch.setenv(k, v)
    build_library()
    kappa, rhs = seeded_inputs(3, 2, 4)
    cases = [(structured_q2_ball(2, 3, eps=0.1), dict(omega=0.3, gmressize=31)),
             (structured_problem(3, 2, 4, kappa, rhs), dict(omega=0.8, gmressize=21))]
    with Context(0) as ctx:
        for P, keys in cases:
            keys = dict(keys, ndirect=1000, iterpre=2, iterpost=2)
            xo, io, xg, info = _solve_pair(ctx, P, keys)
            assert io["status"] == "converged" and info["status_name"] == "converged"
            assert abs(info["iterations"] - io["iterations"]) <= 1
            assert rel_l2(xg, xo) < 1e-8
            # and the mixed / FP64 flexible solvers
            ctx.set_params(tol=1e-10, globaltol=1e-300, maxiter=300,
                           **dict(keys, gmressize=21))
            l = P.nlevels - 1
            x, b = ctx.vec(), ctx.vec()
            ctx.upload(l, b, P.rhs)
            for prec in (GB_FP64, GB_FP32):
                fi = ctx.fgmres(x, b, prec)
                assert fi["true_rel_residual"] <= 1e-10
                assert rel_l2(ctx.download(l, x), xo) < 1e-6
            ctx.free(x)
            ctx.free(b)


def test_direct_coarse_one_level_is_exact(ctx):
    kappa, rhs = seeded_inputs(3, 1, 4)
    L = structured_problem(3, 1, 4, kappa, rhs).levels[2]
    b = np.random.default_rng(0).uniform(-1.0, 1.0, L.n)
    b[L.dirichlet] = 0.0
    P = Problem(dim=3, levels=[L], transfers=[], rhs=b, info={})
    xo, io, xg, info = _solve_pair(ctx, P, dict(ndirect=1000, omega=0.8, gmressize=21))
    A = sp.csr_matrix((L.val, L.col, L.rowptr), shape=(L.n, L.n)).tocsc()
    assert info["firstresidual"] < 1e-12 * np.linalg.norm(b)
    assert np.linalg.norm(xg - spl.spsolve(A, b)) < 1e-12 * np.linalg.norm(xg)
    assert abs(info["iterations"] - io["iterations"]) <= 1


def test_direct_coarse_adjoint_matches_oracle(ctx):
    """The transposed cycle uses (A^T)^-1 on the coarsest level."""
    kappa, rhs = seeded_inputs(3, 2, 4)
    P = structured_problem(3, 2, 4, kappa, rhs, beta=(4.0, 2.0, 1.0))
    keys = dict(ndirect=1000, omega=0.8, gmressize=21, iterpre=2, iterpost=2)
    xo, io, xg, info = _solve_pair(ctx, P, keys, oracle_problem=transposed_problem(P),
                                   adjoint=True)
    assert info["status_name"] == "converged"
    assert abs(info["iterations"] - io["iterations"]) <= 1
    assert rel_l2(xg, xo) < 1e-8


def test_direct_coarse_singular_level_fails_loudly(ctx):
    """A Stokes coarsest level (pressure fixed only up to a constant) has no
    inverse: the solve reports an error instead of running."""
    P = structured_stokes(2, 2, 3)
    ctx.load_problem(P)
    ctx.set_params(ndirect=1000, omega=1.0, gmressize=21)
    l = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(l, b, P.rhs)
    with pytest.raises(GBError, match="singular"):
        ctx.gmres(x, b)
    ctx.free(x)
    ctx.free(b)
