"""Adjoint path on the GPU: transposed operators, adjoint GMRES and the
per-cell coefficient gradient, against the reference's dual solve (golden
fixtures), the oracle, and central differences through a
torch.autograd.Function that wraps the C-ABI.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from _util import (dual_problem, golden_dual_cases, load_golden, reference_cells, rel,
                   rel_l2, solver_keys)
from gascoignelib_b200.native import GB_FP32, GB_FP64
from gascoignelib_b200.problem import seeded_inputs, structured_problem
from oracle.oracle import Oracle, coeff_gradient, transposed_problem

pytestmark = pytest.mark.gpu


def _csr(L):
    return sp.csr_matrix((L.val, L.col, L.rowptr), shape=(L.n, L.n))


@pytest.mark.parametrize("name", golden_dual_cases())
def test_adjoint_gmres_matches_reference_dual_solve(ctx, name):
    P, ref = load_golden(name)
    keys = ref["keys"]
    ctx.load_problem(P)
    ctx.set_params(**solver_keys(keys), gmressize=int(keys["gmressize"]),
                   tol=float(keys["tol"]), globaltol=1e-16, maxiter=100)
    l = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(l, b, ref["dual_rhs"])
    info = ctx.adjoint_gmres(x, b)
    lam = ctx.download(l, x)
    assert ctx.get_operator() == 0  # restored
    assert info["status_name"] == "converged"
    assert abs(info["iterations"] - ref["dual_iterations"]) <= 1
    assert rel_l2(lam, ref["dual_solution"]) < 1e-8
    assert abs(info["firstresidual"] - ref["dual_firstresidual"]) <= 1e-10 * ref[
        "dual_firstresidual"]
    # and the oracle on the reference's own dual matrices
    lo, io = Oracle(dual_problem(P, ref), **solver_keys(keys)).gmres(
        ref["dual_rhs"], vmax=int(keys["gmressize"]), tol=float(keys["tol"]))
    assert rel_l2(lam, lo) < 1e-9
    ctx.free(x)
    ctx.free(b)


@pytest.mark.parametrize("name", golden_dual_cases())
def test_adjoint_gradient_matches_reference_dual_gradient(ctx, name):
    """dJ/dkappa from the GPU forward + adjoint solves and gradient kernel
    within 1e-6 relative of the gradient from the reference's FP64 forward and
    dual solutions."""
    P, ref = load_golden(name)
    cells = reference_cells(P)
    g_ref = coeff_gradient(cells, ref["solution"], ref["dual_solution"], P.finest.dirichlet)
    keys = ref["keys"]
    ctx.load_problem(P)
    ctx.set_cells(P.nlevels - 1, cells)
    ctx.set_params(**solver_keys(keys), gmressize=21, tol=1e-12, globaltol=1e-300,
                   maxiter=200)
    l = P.nlevels - 1
    u, b, lam, gv = ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec()
    ctx.upload(l, b, P.rhs)
    assert ctx.fgmres(u, b, GB_FP32)["status_name"] == "converged"
    ctx.upload(l, gv, ref["dual_rhs"])
    assert ctx.adjoint_fgmres(lam, gv, GB_FP32)["status_name"] == "converged"
    g = ctx.coeff_gradient(l, u, lam)
    assert np.linalg.norm(g - g_ref) <= 1e-6 * np.linalg.norm(g_ref)
    for v in (u, b, lam, gv):
        ctx.free(v)


def test_operator_switch_semantics(ctx):
    kappa, rhs = seeded_inputs(2, 2, 4)
    P = structured_problem(2, 2, 4, kappa, rhs, beta=(4.0, 2.0))
    ctx.load_problem(P)
    l = P.nlevels - 1
    A = _csr(P.finest)
    xv = np.random.default_rng(1).normal(size=P.finest.n)
    x, y = ctx.vec(), ctx.vec()
    ctx.upload(l, x, xv)
    ctx.zero(l, y)
    ctx.vmult(l, y, x, 1.0)
    assert rel(ctx.download(l, y), A @ xv) < 1e-14
    ctx.set_operator(1)
    try:
        assert ctx.get_operator() == 1
        ctx.zero(l, y)
        ctx.vmult(l, y, x, 1.0)
        assert rel(ctx.download(l, y), A.T @ xv) < 1e-14
        ctx.zero(l, y)
        ctx.vmult_transpose(l, y, x, 1.0)
        assert rel(ctx.download(l, y), A @ xv) < 1e-14
    finally:
        ctx.set_operator(0)
    ctx.zero(l, y)
    ctx.vmult_transpose(l, y, x, 1.0)
    assert rel(ctx.download(l, y), A.T @ xv) < 1e-14
    ctx.free(x)
    ctx.free(y)


@pytest.mark.parametrize("prec", [GB_FP64, GB_FP32])
def test_adjoint_solvers_match_oracle_transposed(ctx, prec):
    """3D convection-diffusion: reference-semantics adjoint GMRES against the
    oracle on the transposed hierarchy (iterations +-1, 1e-8), and the
    flexible adjoint solver to a true residual of A^T below tol."""
    kappa, rhs = seeded_inputs(3, 1, 5)
    P = structured_problem(3, 1, 5, kappa, rhs, beta=(1.0, 0.5, 0.25))
    gvec = np.random.default_rng(1004).uniform(-1, 1, P.finest.n)
    gvec[P.finest.dirichlet] = 0.0
    lo, io = Oracle(transposed_problem(P)).gmres(gvec, vmax=21, tol=1e-8)
    ctx.load_problem(P)
    ctx.set_params(gmressize=21, tol=1e-8, globaltol=1e-16, maxiter=100)
    l = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(l, b, gvec)
    if prec == GB_FP64:
        info = ctx.adjoint_gmres(x, b)
        assert abs(info["iterations"] - io["iterations"]) <= 1
        assert rel_l2(ctx.download(l, x), lo) < 1e-8
    ctx.set_params(gmressize=21, tol=1e-8, globaltol=1e-300, maxiter=200)
    info = ctx.adjoint_fgmres(x, b, prec)
    lam = ctx.download(l, x)
    At = _csr(P.finest).T
    assert info["status_name"] == "converged"
    assert np.linalg.norm(gvec - At @ lam) / np.linalg.norm(gvec) <= 1.0001e-8
    # the forward solve still uses A afterwards
    ctx.upload(l, b, P.rhs)
    ctx.fgmres(x, b, prec)
    u = ctx.download(l, x)
    assert np.linalg.norm(P.rhs - _csr(P.finest) @ u) / np.linalg.norm(P.rhs) <= 1.0001e-8
    ctx.free(x)
    ctx.free(b)


def test_coeff_gradient_kernel_matches_oracle(ctx):
    for dim, coarse, refine in ((2, 2, 5), (3, 1, 4)):
        kappa, rhs = seeded_inputs(dim, coarse, refine)
        P = structured_problem(dim, coarse, refine, kappa, rhs)
        ctx.load_problem(P)
        l = P.nlevels - 1
        rng = np.random.default_rng(5)
        uv, lv = rng.normal(size=P.finest.n), rng.normal(size=P.finest.n)
        u, lam = ctx.vec(), ctx.vec()
        ctx.upload(l, u, uv)
        ctx.upload(l, lam, lv)
        g = ctx.coeff_gradient(l, u, lam)
        go = coeff_gradient(P.cells, uv, lv, P.finest.dirichlet)
        assert rel(g, go) < 1e-13
        # per-cell scale and the generic (runtime nloc) kernel path
        c = P.cells
        c.scale = rng.uniform(0.5, 2.0, c.ncells)
        ctx.set_cells(l, c)
        assert rel(ctx.coeff_gradient(l, u, lam),
                   coeff_gradient(c, uv, lv, P.finest.dirichlet)) < 1e-13
        ctx.free(u)
        ctx.free(lam)


def test_coeff_gradient_generic_nloc(ctx):
    """nloc outside the specialised set (here 6: an arbitrary node subset)
    uses the runtime-nloc kernel."""
    from gascoignelib_b200.problem import Cells
    kappa, rhs = seeded_inputs(3, 1, 3)
    P = structured_problem(3, 1, 3, kappa, rhs)
    ctx.load_problem(P)
    l = P.nlevels - 1
    rng = np.random.default_rng(8)
    c = Cells(nodes=P.cells.nodes[:, :6].copy(), kloc=rng.normal(size=(6, 6)))
    ctx.set_cells(l, c)
    uv, lv = rng.normal(size=P.finest.n), rng.normal(size=P.finest.n)
    u, lam = ctx.vec(), ctx.vec()
    ctx.upload(l, u, uv)
    ctx.upload(l, lam, lv)
    assert rel(ctx.coeff_gradient(l, u, lam),
               coeff_gradient(c, uv, lv, P.finest.dirichlet)) < 1e-13
    ctx.free(u)
    ctx.free(lam)


# ------------------------------------------------ autograd wrapper (tests only)

class _Solve(torch.autograd.Function):
    """u = A(kappa)^{-1} b through the C-ABI: forward = flexible GMRES, backward
    = adjoint GMRES (A^T lam = dL/du, zero on Dirichlet nodes) and the
    per-cell gradient kernel."""

    @staticmethod
    def forward(fctx, kappa, env):
        ctx, dim, coarse, refine, rhs, beta, prec = env
        P = structured_problem(dim, coarse, refine, kappa.detach().cpu().numpy(), rhs,
                               beta=beta)
        ctx.load_problem(P)
        l = P.nlevels - 1
        u, b = ctx.vec(), ctx.vec()
        ctx.upload(l, b, P.rhs)
        info = ctx.fgmres(u, b, prec)
        assert info["status_name"] == "converged"
        fctx.env = env
        fctx.state = (P, u, b)
        return torch.from_numpy(ctx.download(l, u))

    @staticmethod
    def backward(fctx, grad_u):
        ctx = fctx.env[0]
        P, u, b = fctx.state
        l = P.nlevels - 1
        g = grad_u.detach().cpu().numpy().astype(np.float64).copy()
        g[P.finest.dirichlet] = 0.0
        lam = ctx.vec()
        ctx.upload(l, b, g)
        info = ctx.adjoint_fgmres(lam, b, fctx.env[6])
        assert info["status_name"] == "converged"
        gk = ctx.coeff_gradient(l, u, lam)
        for v in (u, b, lam):
            ctx.free(v)
        return torch.from_numpy(gk), None


def _functional(kappa, env, M):
    u = _Solve.apply(kappa, env)
    return u @ torch.sparse.mm(M, u.unsqueeze(1)).squeeze(1)


@pytest.mark.parametrize("dim,coarse,refine,beta",
                         [(2, 2, 4, (4.0, 2.0)), (3, 1, 4, None)])
def test_autograd_gradient_matches_central_fd(ctx, dim, coarse, refine, beta):
    """J(kappa) = int u^2: autograd (adjoint) gradient against central
    differences with h = 1e-6 on cells drawn with seed 1003, every solve on
    the GPU (FP64 cycle, true relative residual 1e-13)."""
    kappa0, rhs = seeded_inputs(dim, coarse, refine)
    P0 = structured_problem(dim, coarse, refine, kappa0, rhs, beta=beta)
    Mc = P0.cells.assemble(P0.cells.mloc, P0.finest.n).tocoo()
    M = torch.sparse_coo_tensor(np.vstack([Mc.row, Mc.col]), Mc.data, Mc.shape,
                                check_invariants=True).coalesce()
    ctx.set_params(gmressize=21, tol=1e-13, globaltol=1e-300, maxiter=400)
    env = (ctx, dim, coarse, refine, rhs, beta, GB_FP64)
    k = torch.tensor(kappa0, dtype=torch.float64, requires_grad=True)
    J = _functional(k, env, M)
    J.backward()
    grad = k.grad.numpy()
    pick = np.random.default_rng(1003).choice(kappa0.size, size=16, replace=False)
    h = 1e-6
    fd = []
    with torch.no_grad():
        for c in pick:
            kp = torch.tensor(kappa0)
            km = torch.tensor(kappa0)
            kp[c] += h
            km[c] -= h
            fd.append((_functional(kp, env, M) - _functional(km, env, M)).item() / (2 * h))
    fd = np.array(fd)
    assert np.abs(fd - grad[pick]).max() <= 1e-4 * np.abs(grad).max()
    # the mixed-precision solve gives the same gradient to its tolerance
    ctx.set_params(gmressize=21, tol=1e-10, globaltol=1e-300, maxiter=400)
    k2 = torch.tensor(kappa0, dtype=torch.float64, requires_grad=True)
    _functional(k2, (ctx, dim, coarse, refine, rhs, beta, GB_FP32), M).backward()
    assert np.linalg.norm(k2.grad.numpy() - grad) <= 1e-7 * np.linalg.norm(grad)


def test_c5_adjoint_gradient_full_size(ctx):
    """96^3 cells (912,673 dofs), kappa = exp(N(0,1)), J = int u^2: GPU
    forward and adjoint solves with the FP32 cycle in FP64 flexible GMRES and
    the gradient kernel, against the oracle's FP64 reference-semantics forward
    and dual solves (1e-6 relative in the gradient)."""
    kappa, rhs = seeded_inputs(3, 3, 5)
    P = structured_problem(3, 3, 5, kappa, rhs)
    assert P.finest.n == 912673 and P.cells.ncells == 884736
    O = Oracle(P)
    uo, io = O.gmres(vmax=21, tol=1e-10)
    M = P.cells.assemble(P.cells.mloc, P.finest.n)
    g = 2.0 * (M @ uo)
    g[P.finest.dirichlet] = 0.0
    # the diffusion operator is symmetric: its dual system is the forward one
    A = _csr(P.finest)
    assert abs(A - A.T).max() == 0.0
    lo, _ = O.gmres(g, vmax=21, tol=1e-10)
    go = coeff_gradient(P.cells, uo, lo, P.finest.dirichlet)
    O.close()
    ctx.load_problem(P)
    ctx.set_params(gmressize=21, tol=1e-10, globaltol=1e-300, maxiter=200)
    l = P.nlevels - 1
    u, b, lam, gv = ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec()
    ctx.upload(l, b, P.rhs)
    assert ctx.fgmres(u, b, GB_FP32)["true_rel_residual"] <= 1e-10
    Jg = ctx.functional(l, u, gv)  # J = u^T M u and the dual rhs 2 M u on the device
    assert ctx.adjoint_fgmres(lam, gv, GB_FP32)["true_rel_residual"] <= 1e-10
    grad = ctx.coeff_gradient(l, u, lam)
    assert np.linalg.norm(grad - go) <= 1e-6 * np.linalg.norm(go)
    Jo = uo @ (M @ uo)
    assert abs(Jg - Jo) <= 1e-8 * abs(Jo)
    for v in (u, b, lam, gv):
        ctx.free(v)


def test_device_functional_and_stream(ctx):
    kappa, rhs = seeded_inputs(3, 1, 4)
    P = structured_problem(3, 1, 4, kappa, rhs)
    ctx.load_problem(P)
    l = P.nlevels - 1
    M = P.cells.assemble(P.cells.mloc, P.finest.n)
    uv = np.random.default_rng(9).normal(size=P.finest.n)
    u, g = ctx.vec(), ctx.vec()
    ctx.upload(l, u, uv)
    J = ctx.functional(l, u, g)
    assert abs(J - uv @ (M @ uv)) <= 1e-13 * abs(J)
    gr = 2.0 * (M @ uv)
    gr[P.finest.dirichlet] = 0.0
    assert rel(ctx.download(l, g), gr) < 1e-14
    assert ctx.stream() != 0
    ctx.free(u)
    ctx.free(g)


class _DeviceSolve(torch.autograd.Function):
    """u = A(kappa)^{-1} b with the matrices of every level assembled on the
    device from kappa (gb_assemble_levels): forward = flexible GMRES with a
    fixed number of Arnoldi steps (no tolerance test, so that u is a smooth
    function of kappa and finite differences of J see no stopping jumps),
    backward = adjoint GMRES + the per-cell gradient kernel."""

    @staticmethod
    def forward(fctx, kappa, env):
        ctx, P, u, b, lam, g = env
        ctx.assemble_levels(kappa.detach().cpu().numpy())
        l = P.nlevels - 1
        ctx.fgmres(u, b, GB_FP64, check=False)
        fctx.env = env
        return torch.from_numpy(ctx.download(l, u))

    @staticmethod
    def backward(fctx, grad_u):
        ctx, P, u, b, lam, g = fctx.env
        l = P.nlevels - 1
        gu = grad_u.detach().cpu().numpy().astype(np.float64).copy()
        gu[P.finest.dirichlet] = 0.0
        ctx.upload(l, g, gu)
        ctx.adjoint_fgmres(lam, g, GB_FP64, check=False)
        return torch.from_numpy(ctx.coeff_gradient(l, u, lam)), None


def test_c5_autograd_gradient_matches_central_fd_full_size(ctx):
    """The C5 check as the benchmark states it: 96^3 cells (912,673 dofs),
    kappa = exp(N(0,1)) per cell (seed 1001), J(u) = int u^2; dJ/dkappa from the
    autograd Function (adjoint solve + gradient kernel) against central
    differences with h = 1e-6 on 32 cells drawn with seed 1003. Every solve
    assembles all 5 levels on the device from the perturbed kappa and runs 60
    FP64 flexible GMRES steps (relative residual about 1e-15).

    Noise bound: per-cell gradients are about 1e-2 against J about 1e3, so
    2 h dJ/dkappa_c is about 2e-11 J, while the rounding of the two solves
    leaves J uncertain by roughly 1e-14 J; the differences therefore carry a
    relative error of about 1e-3, and the test allows 1e-2 of the largest of
    the 32 gradient entries."""
    from gascoignelib_b200.problem import structured_meshes
    kappa0, rhs = seeded_inputs(3, 3, 5)
    P = structured_problem(3, 3, 5, kappa0, rhs)
    assert P.finest.n == 912673 and kappa0.size == 884736
    ctx.load_problem(P)
    for l, (cells, coord, par) in enumerate(structured_meshes(P)):
        ctx.set_mesh(l, 3, cells, coord, par)
    ctx.set_params(gmressize=21, tol=1e-300, globaltol=1e-300, maxiter=60)
    l = P.nlevels - 1
    u, b, lam, g = ctx.vec(), ctx.vec(), ctx.vec(), ctx.vec()
    ctx.upload(l, b, P.rhs)
    Mc = P.cells.assemble(P.cells.mloc, P.finest.n).tocoo()
    M = torch.sparse_coo_tensor(np.vstack([Mc.row, Mc.col]), Mc.data, Mc.shape,
                                check_invariants=True).coalesce()
    env = (ctx, P, u, b, lam, g)

    def J_of(k):
        uu = _DeviceSolve.apply(k, env)
        return uu @ torch.sparse.mm(M, uu.unsqueeze(1)).squeeze(1)

    k = torch.tensor(kappa0, dtype=torch.float64, requires_grad=True)
    J = J_of(k)
    J.backward()
    grad = k.grad.numpy().copy()
    pick = np.random.default_rng(1003).choice(kappa0.size, size=32, replace=False)
    h = 1e-6
    fd = []
    with torch.no_grad():
        for c in pick:
            kp = torch.tensor(kappa0)
            km = torch.tensor(kappa0)
            kp[c] += h
            km[c] -= h
            fd.append((J_of(kp) - J_of(km)).item() / (2 * h))
    fd = np.array(fd)
    scale = np.abs(grad[pick]).max()
    assert scale > 0
    assert np.abs(fd - grad[pick]).max() <= 1e-2 * scale, (fd, grad[pick])
    for v in (u, b, lam, g):
        ctx.free(v)
