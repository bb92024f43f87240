"""Device-side Q1 assembly (gb_level_set_mesh, gb_assemble, gb_assemble_levels)
against the matrices the reference assembled (golden fixtures), the oracle's
assembly, and the solver results that follow from them."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from _util import (golden_assembly_cases, load_golden, oracle_level_values, rel_l2,
                   set_uniform_meshes, solver_keys, uniform_meshes)
from gascoignelib_b200.native import GB_FP32, GB_FP64, GBError
from gascoignelib_b200.problem import seeded_inputs, structured_problem
from oracle.oracle import Oracle, transposed_problem

pytestmark = pytest.mark.gpu


def _zero_values(P):
    """The problem with every matrix value replaced by zero (pattern and
    Dirichlet lists kept), so that only the device assembly can fill them."""
    import copy
    Q = copy.deepcopy(P)
    for L in Q.levels:
        L.val = np.zeros_like(L.val)
    return Q


def _with_values(P, vals):
    import copy
    Q = copy.deepcopy(P)
    for L, v in zip(Q.levels, vals):
        L.val = np.array(v)
    return Q


@pytest.mark.parametrize("name,kappa,beta", golden_assembly_cases(),
                         ids=[c[0] for c in golden_assembly_cases()])
def test_assembly_matches_reference_and_solves(ctx, name, kappa, beta):
    """Every level assembled on the device from the finest kappa equals the
    reference's matrices within 1e-13 of the largest entry; the solve on them
    reproduces the reference's iteration count and solution."""
    P, ref = load_golden(name)
    ctx.load_problem(_zero_values(P))
    set_uniform_meshes(ctx, P)
    ctx.assemble_levels(kappa, beta)
    for l, L in enumerate(P.levels):
        v = ctx.level_values(l, L.val.size)
        assert np.abs(v - L.val).max() <= 1e-13 * np.abs(L.val).max(), l
    keys = ref["keys"]
    ctx.set_params(**solver_keys(keys), gmressize=int(keys["gmressize"]),
                   tol=float(keys["tol"]), globaltol=1e-16, maxiter=100)
    fl = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(fl, b, P.rhs)
    info = ctx.gmres(x, b)
    assert abs(info["iterations"] - ref["iterations"]) <= 1
    assert rel_l2(ctx.download(fl, x), ref["solution"]) < 1e-8
    ctx.free(x)
    ctx.free(b)


def test_reassembly_device_kappa_mixed_adjoint_direct(ctx):
    """A second kappa given as a CUDA tensor: the same bits as from host memory,
    the oracle's values, and the forward (mixed and FP64), adjoint and
    direct-coarse solves on the new matrices against the oracle."""
    kappa, rhs = seeded_inputs(3, 1, 4)
    beta = (1.0, 0.5, 0.25)
    P = structured_problem(3, 1, 4, kappa, rhs, beta=beta)
    ctx.load_problem(P)
    set_uniform_meshes(ctx, P)
    k2 = kappa ** 2 + 0.5
    ctx.assemble_levels(k2, beta)
    host = [ctx.level_values(l, L.val.size) for l, L in enumerate(P.levels)]
    ctx.assemble_levels(torch.tensor(k2, dtype=torch.float64, device="cuda"), beta)
    dev = [ctx.level_values(l, L.val.size) for l, L in enumerate(P.levels)]
    for a, b in zip(host, dev):
        assert np.array_equal(a, b)
    ovals, okap = oracle_level_values(P, k2, beta)
    for l, (v, o) in enumerate(zip(dev, ovals)):
        assert np.abs(v - o).max() <= 1e-13 * np.abs(o).max(), l
        assert np.array_equal(ctx.level_kappa(l, okap[l].size), okap[l])
    Q = _with_values(P, ovals)
    fl = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(fl, b, P.rhs)
    keys = dict(iterpre=2, iterpost=2, omega=0.8, gmressize=21)
    for nd in (0, 1000):
        ctx.set_params(tol=1e-8, globaltol=1e-300, maxiter=100, ndirect=nd, **keys)
        O = Oracle(Q, ndirect=nd, omega=0.8)
        xo, io = O.gmres(vmax=21, tol=1e-8, globaltol=1e-300)
        info = ctx.gmres(x, b)
        assert abs(info["iterations"] - io["iterations"]) <= 1
        assert rel_l2(ctx.download(fl, x), xo) < 1e-8
        lo, jo = Oracle(transposed_problem(Q), ndirect=nd, omega=0.8).gmres(
            vmax=21, tol=1e-8, globaltol=1e-300)
        ai = ctx.adjoint_gmres(x, b)
        assert abs(ai["iterations"] - jo["iterations"]) <= 1
        assert rel_l2(ctx.download(fl, x), lo) < 1e-8
    ctx.set_params(tol=1e-10, globaltol=1e-300, maxiter=300, **keys)
    A = sp.csr_matrix((ovals[-1], P.finest.col, P.finest.rowptr), shape=(P.finest.n,) * 2)
    for prec in (GB_FP32, GB_FP64):
        fi = ctx.fgmres(x, b, prec)
        assert fi["true_rel_residual"] <= 1e-10
        u = ctx.download(fl, x)
        assert np.linalg.norm(P.rhs - A @ u) <= 1e-9 * np.linalg.norm(P.rhs)
    ctx.free(x)
    ctx.free(b)


def test_assembly_errors(ctx):
    kappa, rhs = seeded_inputs(2, 2, 3)
    P = structured_problem(2, 2, 3, kappa, rhs)
    ctx.load_problem(P)
    with pytest.raises(GBError, match="no mesh"):
        ctx.assemble(P.nlevels - 1, kappa)
    meshes = uniform_meshes(P)
    cells, par = meshes[-1]
    bad = cells.copy()
    bad[0, 3] = bad[-1, 0]  # a node far outside the cell's stencil
    with pytest.raises(GBError, match="pattern"):
        ctx.set_mesh(P.nlevels - 1, 2, bad, P.finest.coord, par)
    with pytest.raises(GBError, match="parent"):
        ctx.set_mesh(P.nlevels - 1, 2, cells, P.finest.coord, None)
    ctx.set_mesh(P.nlevels - 1, 2, cells, P.finest.coord, par)
    with pytest.raises(GBError, match="no mesh"):
        ctx.assemble_levels(kappa)  # the coarser levels have none
    ctx.assemble(P.nlevels - 1, kappa)
    v = ctx.level_values(P.nlevels - 1, P.finest.val.size)
    assert np.abs(v - P.finest.val).max() <= 1e-13 * np.abs(P.finest.val).max()
    # setting the matrix again drops the mesh
    ctx.load_problem(P)
    with pytest.raises(GBError, match="no mesh"):
        ctx.assemble(P.nlevels - 1, kappa)


def test_assembly_full_size_against_generator(ctx):
    """The 64^3 hierarchy (the solve benchmark's problem): the generator's
    matrices (whose assembly the reference pins) from the seeded kappa."""
    kappa, rhs = seeded_inputs(3, 1, 6)
    P = structured_problem(3, 1, 6, kappa, rhs)
    ctx.load_problem(_zero_values(P))
    set_uniform_meshes(ctx, P)
    ctx.assemble_levels(torch.tensor(kappa, device="cuda"))
    for l, L in enumerate(P.levels):
        v = ctx.level_values(l, L.val.size)
        assert np.abs(v - L.val).max() <= 1e-13 * np.abs(L.val).max(), l
    ctx.set_params(tol=1e-8, globaltol=1e-300, maxiter=200, gmressize=21, omega=0.8)
    fl = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(fl, b, P.rhs)
    info = ctx.fgmres(x, b, GB_FP32)
    assert info["status_name"] == "converged" and info["iterations"] <= 12
    ctx.free(x)
    ctx.free(b)


@pytest.mark.parametrize("nd", [0, 1000])
def test_reassembly_after_solves(ctx, nd):
    """Solves (captured solver graphs, dense coarse maps, the transpose, the
    direct coarse inverse) first, then a new kappa assembled on the device: the
    next forward, adjoint and mixed solves use the new matrices."""
    kappa, rhs = seeded_inputs(3, 1, 4)
    beta = (1.0, 0.5, 0.25)
    P = structured_problem(3, 1, 4, kappa, rhs, beta=beta)
    ctx.load_problem(P)
    set_uniform_meshes(ctx, P)
    keys = dict(iterpre=2, iterpost=2, omega=0.8, gmressize=21, ndirect=nd)
    ctx.set_params(tol=1e-8, globaltol=1e-300, maxiter=100, **keys)
    fl = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(fl, b, P.rhs)
    ctx.assemble_levels(kappa, beta)
    ctx.gmres(x, b)
    ctx.adjoint_gmres(x, b)
    ctx.fgmres(x, b, GB_FP32)
    ctx.adjoint_fgmres(x, b, GB_FP32)
    k2 = 1.0 / kappa
    ctx.assemble_levels(torch.tensor(k2, device="cuda"), beta)
    ovals, _ = oracle_level_values(P, k2, beta)
    Q = _with_values(P, ovals)
    xo, io = Oracle(Q, ndirect=nd, omega=0.8).gmres(vmax=21, tol=1e-8, globaltol=1e-300)
    info = ctx.gmres(x, b)
    assert abs(info["iterations"] - io["iterations"]) <= 1
    assert rel_l2(ctx.download(fl, x), xo) < 1e-8
    lo, jo = Oracle(transposed_problem(Q), ndirect=nd, omega=0.8).gmres(
        vmax=21, tol=1e-8, globaltol=1e-300)
    ai = ctx.adjoint_gmres(x, b)
    assert abs(ai["iterations"] - jo["iterations"]) <= 1
    assert rel_l2(ctx.download(fl, x), lo) < 1e-8
    ctx.set_params(tol=1e-10, globaltol=1e-300, maxiter=300, **keys)
    A = sp.csr_matrix((ovals[-1], P.finest.col, P.finest.rowptr), shape=(P.finest.n,) * 2)
    fi = ctx.fgmres(x, b, GB_FP32)
    u = ctx.download(fl, x)
    assert np.linalg.norm(P.rhs - A @ u) <= 1e-9 * np.linalg.norm(P.rhs)
    af = ctx.adjoint_fgmres(x, b, GB_FP32)
    lam = ctx.download(fl, x)
    assert np.linalg.norm(P.rhs - A.T @ lam) <= 1e-9 * np.linalg.norm(P.rhs)
    assert fi["status_name"] == "converged" and af["status_name"] == "converged"
    ctx.free(x)
    ctx.free(b)


@pytest.mark.parametrize("name", [n for n in __import__("_util").golden_cases()
                                  if n.startswith("q2_")])
def test_q2_assembly_matches_reference_and_solves(ctx, name):
    """CGQ2 (27-node hexahedra, 9-node quadrilaterals) assembled on the device:
    the reference's matrices on every level, and its solve."""
    from _util import golden_kappa_beta, q2_element_kappa, uniform_meshes_q2
    P, ref = load_golden(name)
    kappa, beta = golden_kappa_beta(name)
    Nc = round(len(kappa) ** (1.0 / P.dim))
    ctx.load_problem(_zero_values(P))
    for l, (el, par) in enumerate(uniform_meshes_q2(P)):
        ctx.set_mesh(l, P.dim, el, P.levels[l].coord, par, degree=2)
    ctx.assemble_levels(q2_element_kappa(P.dim, kappa, Nc), beta)
    for l, L in enumerate(P.levels):
        v = ctx.level_values(l, L.val.size)
        assert np.abs(v - L.val).max() <= 1e-13 * np.abs(L.val).max(), l
    keys = ref["keys"]
    ctx.set_params(**solver_keys(keys), gmressize=int(keys["gmressize"]),
                   tol=float(keys["tol"]), globaltol=1e-16, maxiter=100)
    fl = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(fl, b, P.rhs)
    info = ctx.gmres(x, b)
    assert abs(info["iterations"] - ref["iterations"]) <= 1
    assert rel_l2(ctx.download(fl, x), ref["solution"]) < 1e-8
    ctx.free(x)
    ctx.free(b)


def test_q2_assembly_c4_size_against_generator(ctx):
    """The 40^3-element Q2 hierarchy of the C4 bench line (constant eps, beta):
    the generator's exact-integral matrices within the reference's own 12-digit
    Gauss weights (1e-12)."""
    from gascoignelib_b200.problem import structured_q2
    from _util import uniform_meshes_q2
    P = structured_q2(3, 5, 4, eps=1e-2, beta=(1.0, 0.5, 0.25))
    ctx.load_problem(_zero_values(P))
    for l, (el, par) in enumerate(uniform_meshes_q2(P)):
        ctx.set_mesh(l, 3, el, P.levels[l].coord, par, degree=2)
    ne = uniform_meshes_q2(P)[-1][0].shape[0]
    ctx.assemble_levels(np.full(ne, 1e-2), (1.0, 0.5, 0.25))
    for l, L in enumerate(P.levels):
        v = ctx.level_values(l, L.val.size)
        assert np.abs(v - L.val).max() <= 1e-12 * np.abs(L.val).max(), l


@pytest.mark.parametrize("name,kind,diff,beta,lps", __import__("_util").golden_lps_cases(),
                         ids=[c[0] for c in __import__("_util").golden_lps_cases()])
def test_lps_assembly_matches_reference_and_solves(ctx, name, kind, diff, beta, lps):
    """CGQ2Lps / CGQ1Lps (LPS of the convection; Q2 or Q1 functions on
    patches) assembled on the device: the reference's matrices on every level,
    the oracle's, and the reference's solve; then the same assembly with the
    stabilisation off differs, and LPS on a level of Q1 cells is refused."""
    from _util import uniform_meshes_q2
    from oracle.assembly import assemble, q1patch_element_matrices, q2_element_matrices
    f = q2_element_matrices if kind == 2 else q1patch_element_matrices
    P, ref = load_golden(name)
    ctx.load_problem(_zero_values(P))
    meshes = uniform_meshes_q2(P)
    for l, (el, par) in enumerate(meshes):
        ctx.set_mesh(l, P.dim, el, P.levels[l].coord, par, degree=kind)
    kap = np.full(meshes[-1][0].shape[0], diff)
    try:
        ctx.set_assembly_lps(*lps)
        ctx.assemble_levels(kap, beta)
    finally:
        ctx.set_assembly_lps(0.0)
    for l, L in enumerate(P.levels):
        v = ctx.level_values(l, L.val.size)
        el = meshes[l][0]
        o = assemble(L.n, L.rowptr, L.col, el,
                     f(P.dim, L.coord[el], np.full(el.shape[0], diff), beta, lps), L.dirichlet)
        assert np.abs(v - L.val).max() <= 1e-13 * np.abs(L.val).max(), l
        assert np.abs(v - o).max() <= 1e-13 * np.abs(L.val).max(), l
    keys = ref["keys"]
    ctx.set_params(**solver_keys(keys), gmressize=int(keys["gmressize"]),
                   tol=float(keys["tol"]), globaltol=1e-16, maxiter=100)
    fl = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(fl, b, P.rhs)
    info = ctx.gmres(x, b)
    assert abs(info["iterations"] - ref["iterations"]) <= 1
    assert rel_l2(ctx.download(fl, x), ref["solution"]) < 1e-8
    ctx.free(x)
    ctx.free(b)
    ctx.assemble_levels(kap, beta)  # stabilisation off again
    v = ctx.level_values(fl, P.finest.val.size)
    assert np.abs(v - P.finest.val).max() > 1e-3 * np.abs(P.finest.val).max()
    # LPS on a Q1 level is refused
    Q, _ = load_golden("q1_2d_c2_r3_seeded")
    ctx.load_problem(Q)
    set_uniform_meshes(ctx, Q)
    try:
        ctx.set_assembly_lps(*lps)
        with pytest.raises(GBError, match="patch elements only"):
            ctx.assemble(Q.nlevels - 1, np.ones(uniform_meshes(Q)[-1][0].shape[0]), beta)
    finally:
        ctx.set_assembly_lps(0.0)
