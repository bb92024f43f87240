"""Device assembly on levels with hanging nodes (one more refinement of a
ball): the element matrices of the cells with hanging nodes condensed on the
device, against the reference's matrices (2D golden ball cases; 3D cases run
on the compiled reference; Q1 and Q2), the oracle's condensation, the 3D Q2
ball generator, and the solves on the assembled levels."""
import copy
import os

import numpy as np
import pytest

from _util import (ball_meshes, golden_hn_assembly_cases, load_golden, oracle_ball_values,
                   reference_ball_3d, rel_l2, solver_keys, with_condensed_pattern)
from gascoignelib_b200.native import GB_FP32, GBError
from gascoignelib_b200.problem import q2_meshes, structured_q2_ball
from oracle.oracle import REF_HARNESS

pytestmark = pytest.mark.gpu


def _zero_values(P):
    Q = copy.deepcopy(P)
    for L in Q.levels:
        L.val = np.zeros_like(L.val)
    return Q


def _set_ball_meshes(ctx, P, degree):
    meshes = ball_meshes(P, degree)
    for l, (el, par) in enumerate(meshes):
        ctx.set_mesh(l, P.dim, el, P.levels[l].coord, par if l > 0 else None, degree=degree)
    return meshes


@pytest.mark.parametrize("name,degree,diff,beta", golden_hn_assembly_cases(),
                         ids=[c[0] for c in golden_hn_assembly_cases()])
def test_hn_assembly_matches_reference_and_solves(ctx, name, degree, diff, beta):
    """Every level assembled on the device (the finest with hanging nodes)
    equals the reference's matrices and the oracle's within 1e-13 of the
    largest entry; the solve on them reproduces the reference's iteration count
    and solution."""
    P, ref = load_golden(name)
    ctx.load_problem(_zero_values(P))
    meshes = _set_ball_meshes(ctx, P, degree)
    kap = np.full(meshes[-1][0].shape[0], diff)
    ctx.assemble_levels(kap, beta)
    ovals, _ = oracle_ball_values(P, degree, kap, beta)
    for l, L in enumerate(P.levels):
        v = ctx.level_values(l, L.val.size)
        scale = np.abs(L.val).max()
        assert np.abs(v - L.val).max() <= 1e-13 * scale, l
        assert np.abs(v - ovals[l]).max() <= 1e-13 * scale, l
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


@pytest.mark.skipif(not os.path.exists(REF_HARNESS), reason="compiled reference not present")
@pytest.mark.parametrize("disc,diff,conv", [("Q1", 1.0, None), ("Q2", 0.1, (1.0, 0.5, 0.25))])
def test_hn_assembly_3d_against_reference(ctx, disc, diff, conv):
    """3D ball refinement (edge and face hanging nodes, Q13d / Q23d): the
    device-assembled levels against the reference's matrices, then the solve
    against the reference's iteration count and solution."""
    P, summ, out = reference_ball_3d(disc, diff, conv)
    assert P.finest.hn_faces.shape[0] > 0 and P.finest.hn_edges.shape[0] > 0
    degree = 2 if disc == "Q2" else 1
    ctx.load_problem(_zero_values(P))
    meshes = _set_ball_meshes(ctx, P, degree)
    ctx.assemble_levels(np.full(meshes[-1][0].shape[0], diff), conv)
    for l, L in enumerate(P.levels):
        v = ctx.level_values(l, L.val.size)
        assert np.abs(v - L.val).max() <= 1e-13 * np.abs(L.val).max(), l
    ctx.set_params(gmressize=21, tol=1e-8, globaltol=1e-16, maxiter=100)
    fl = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(fl, b, P.rhs)
    info = ctx.gmres(x, b)
    assert abs(info["iterations"] - int(summ["iterations"][0])) <= 1
    assert rel_l2(ctx.download(fl, x), np.fromfile(os.path.join(out, "solution.f64"))) < 1e-8
    ctx.free(x)
    ctx.free(b)


@pytest.mark.parametrize("coarse,refine", [(1, 4), (2, 5)])
def test_hn_assembly_matches_q2_ball_generator(ctx, coarse, refine):
    """3D Q2 with hanging edge and face nodes: the device's condensed element
    matrices equal the generator's global C^T A C (exact Gauss weights there,
    hence 1e-12), up to 404,065 rows; then a mixed-precision solve."""
    P = with_condensed_pattern(structured_q2_ball(coarse, refine, eps=0.1), 2)
    ctx.load_problem(_zero_values(P))
    meshes = _set_ball_meshes(ctx, P, 2)
    ctx.assemble_levels(np.full(meshes[-1][0].shape[0], 0.1), (1.0, 0.5, 0.25))
    first = []
    for l, L in enumerate(P.levels):
        v = ctx.level_values(l, L.val.size)
        assert np.abs(v - L.val).max() <= 1e-12 * np.abs(L.val).max(), l
        first.append(v)
    # the generator's own element lists (q2_meshes, the bench's meshes)
    for l, (el, par) in enumerate(q2_meshes(P)):
        ctx.set_mesh(l, 3, el, P.levels[l].coord, par, degree=2)
    ctx.assemble_levels(np.full(P.info["elements"].shape[0], 0.1), (1.0, 0.5, 0.25))
    for l, L in enumerate(P.levels):
        v = ctx.level_values(l, L.val.size)
        assert np.abs(v - first[l]).max() <= 1e-13 * np.abs(first[l]).max(), l
    ctx.set_params(tol=1e-8, globaltol=1e-300, maxiter=300, gmressize=21, omega=0.8)
    fl = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(fl, b, P.rhs)
    info = ctx.fgmres(x, b, GB_FP32)
    assert info["true_rel_residual"] <= 1e-8
    ctx.free(x)
    ctx.free(b)


def test_hn_reassembly_and_mesh_rules(ctx):
    """A second kappa (per element, varying) on the hanging-node level against
    the oracle; the hanging-node lists set again drop the mesh."""
    name, degree, diff, beta = golden_hn_assembly_cases()[0]
    P, _ = load_golden(name)
    ctx.load_problem(P)
    meshes = _set_ball_meshes(ctx, P, degree)
    ne = meshes[-1][0].shape[0]
    kap = 0.5 + np.random.default_rng(7).uniform(size=ne)
    ctx.assemble_levels(kap, beta)
    ovals, okap = oracle_ball_values(P, degree, kap, beta)
    for l, L in enumerate(P.levels):
        v = ctx.level_values(l, L.val.size)
        assert np.abs(v - ovals[l]).max() <= 1e-13 * np.abs(ovals[l]).max(), l
        assert np.array_equal(ctx.level_kappa(l, okap[l].size), okap[l])
    fl = P.nlevels - 1
    ctx.load_problem(P)  # the matrix and hanging nodes again: the mesh is gone
    with pytest.raises(GBError, match="no mesh"):
        ctx.assemble(fl, kap)
