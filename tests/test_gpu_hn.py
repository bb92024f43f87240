"""Hanging nodes on the GPU (ball refinement, Q1 and Q2): the HNStructure
operations bit for bit against the reference, and solves against the
reference and the oracle."""
import os
import tempfile

import numpy as np
import pytest

from _util import golden_hn_cases, load_golden, rel_l2, solver_keys
from gascoignelib_b200.native import GB_FP32, GB_FP64
from gascoignelib_b200.problem import load_reference_dump
from oracle.oracle import REF_HARNESS, Oracle, run_reference, write_inputs

pytestmark = pytest.mark.gpu


def _ops_match(ctx, P, ref_ops):
    l = P.nlevels - 1
    t = np.sin(1.0 + np.arange(P.finest.ndof))
    v = ctx.vec()
    for op in ("average", "distribute", "zero"):
        ctx.upload(l, v, t)
        ctx.hn(op, l, v)
        assert np.array_equal(ctx.download(l, v), ref_ops[op]), op
    ctx.free(v)


@pytest.mark.parametrize("name", golden_hn_cases())
def test_hn_ops_and_solve_match_reference(ctx, name):
    P, ref = load_golden(name)
    keys = ref["keys"]
    ctx.load_problem(P)
    _ops_match(ctx, P, {op: ref["hn_" + op] for op in ("average", "distribute", "zero")})
    ctx.set_params(**solver_keys(keys), gmressize=int(keys["gmressize"]),
                   tol=float(keys["tol"]), globaltol=1e-16, maxiter=100)
    l = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(l, b, P.rhs)
    info = ctx.gmres(x, b)
    assert info["status_name"] == "converged"
    assert abs(info["iterations"] - ref["iterations"]) <= 1
    assert rel_l2(ctx.download(l, x), ref["solution"]) < 1e-8
    ctx.set_params(**solver_keys(keys), gmressize=21, tol=1e-10, globaltol=1e-300,
                   maxiter=300)
    for prec in (GB_FP64, GB_FP32):
        info = ctx.fgmres(x, b, prec)
        assert info["true_rel_residual"] <= 1e-10
        assert rel_l2(ctx.download(l, x), ref["solution"]) < 1e-6
    ctx.free(x)
    ctx.free(b)


@pytest.mark.skipif(not os.path.exists(REF_HARNESS), reason="compiled reference not present")
@pytest.mark.parametrize("disc", ["Q1", "Q2"])
def test_hn_3d_against_reference(ctx, disc):
    """3D ball refinement (edge and face hanging nodes, Q13d / Q23d):
    HN operations bit for bit, reference-semantics solve within 1e-8."""
    d = tempfile.mkdtemp()
    res = 2 * (2 << 3)
    rhs = np.random.default_rng(1002).uniform(-1.0, 1.0, size=(res + 1) ** 3)
    out, summ = run_reference(d, threads=1, dim=3, coarse=2, refine=3, disc=disc,
                              ball=0.25, diff=1.0, rhsres=res, dump=1, tol=1e-8,
                              **write_inputs(d, None, rhs))
    P = load_reference_dump(out)
    ctx.load_problem(P)
    _ops_match(ctx, P, {op: np.fromfile(os.path.join(out, f"hn_{op}.f64"))
                        for op in ("average", "distribute", "zero")})
    ctx.set_params(gmressize=21, tol=1e-8, globaltol=1e-16, maxiter=100)
    l = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(l, b, P.rhs)
    info = ctx.gmres(x, b)
    assert abs(info["iterations"] - int(summ["iterations"][0])) <= 1
    assert rel_l2(ctx.download(l, x), np.fromfile(os.path.join(out, "solution.f64"))) < 1e-8
    ctx.free(x)
    ctx.free(b)


def test_q2_ball_generator_solve_matches_oracle(ctx):
    """The bench's Q2 workload with the refined ball (edge and face hanging
    nodes of Q23d on generated meshes): the reference-semantics solve against
    the oracle, and the mixed / FP64 flexible solves to 1e-10."""
    from gascoignelib_b200.problem import structured_q2_ball

    P = structured_q2_ball(2, 3, eps=0.1)
    O = Oracle(P, omega=0.3)
    xo, io = O.gmres(vmax=31, tol=1e-8, globaltol=1e-300)
    assert io["status"] == "converged"
    ctx.load_problem(P)
    ctx.set_params(iterpre=2, iterpost=2, iterexact=10, omega=0.3, mgomega=1.0,
                   mgtype="V", gmressize=31, tol=1e-8, globaltol=1e-300, maxiter=100)
    l = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(l, b, P.rhs)
    info = ctx.gmres(x, b)
    assert abs(info["iterations"] - io["iterations"]) <= 1
    assert rel_l2(ctx.download(l, x), xo) < 1e-8
    ctx.set_params(iterpre=2, iterpost=2, iterexact=10, omega=0.3, mgomega=1.0,
                   mgtype="V", gmressize=31, tol=1e-10, globaltol=1e-300, maxiter=300)
    for prec in (GB_FP64, GB_FP32):
        info = ctx.fgmres(x, b, prec)
        assert info["status_name"] == "converged"
        assert info["true_rel_residual"] <= 1e-10
        assert rel_l2(ctx.download(l, x), xo) < 1e-6
    ctx.free(x)
    ctx.free(b)


def _context_with(env):
    from gascoignelib_b200.native import Context
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return Context(0)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def test_locality_slot_order_leaves_results_unchanged():
    """The slots of pattern-free scalar levels ordered by each row's smallest
    column (the default) against the mesh's own order (GB_ROW_ORDER=0): every
    row keeps its entries and their order, so the SpMV, a smoothing sweep and
    the reference-semantics and flexible solves give the same bits. The ball
    mesh's refined levels have no column patterns."""
    from gascoignelib_b200.problem import structured_q2_ball

    P = structured_q2_ball(2, 3, eps=0.1)
    l = P.nlevels - 1
    rng = np.random.default_rng(7)
    xv = rng.standard_normal(P.levels[l].ndof)
    out = {}
    for tag, env in (("mesh", {"GB_ROW_ORDER": "0"}), ("locality", {})):
        c = _context_with(env)
        try:
            c.load_problem(P)
            c.set_params(iterpre=2, iterpost=2, iterexact=10, omega=0.3, mgomega=1.0,
                         mgtype="V", gmressize=31, tol=1e-8, globaltol=1e-300, maxiter=100)
            x, y, h = c.vec(), c.vec(), c.vec()
            res = []
            c.upload(l, x, xv)
            c.vmult(l, y, x, 1.0)
            res.append(c.download(l, y))
            c.upload(l, y, P.rhs)
            c.smooth(l, 2, x, y, h)
            res.append(c.download(l, x))
            c.upload(l, x, np.zeros_like(xv))
            res.append((c.gmres(x, y)["iterations"], c.download(l, x)))
            for prec in (GB_FP64, GB_FP32):
                c.fgmres(x, y, prec)
                res.append(c.download(l, x))
            out[tag] = res
        finally:
            c.close()
    a, b = out["mesh"], out["locality"]
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1], b[1])
    assert a[2][0] == b[2][0] and np.array_equal(a[2][1], b[2][1])
    assert np.array_equal(a[3], b[3])
    assert np.array_equal(a[4], b[4])
