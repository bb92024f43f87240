"""The block ILU smoother (linear_smooth ilu, matrixtype block: SparseBlockIlu)
on the GPU: the level-scheduled triangular solves equal the sequential
substitutions of the oracle bit for bit, and the multigrid solves match the
reference's."""
import numpy as np
import pytest

from _util import golden_cases, load_golden, rel, rel_l2, solver_keys
from gascoignelib_b200.native import GB_FP32, GB_FP64
from gascoignelib_b200.problem import structured_stokes
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def _ilu_cases():
    return [n for n in golden_cases() if n.startswith("ilu_")]


def _sweeps_match(ctx, P, O):
    """One sweep from x = 0 (residual = y exactly, so the ILU solve alone is
    compared) bit for bit; sweeps from a general x within 1e-11 (the residual
    SpMV contracts multiply-adds, the oracle does not)."""
    rng = np.random.default_rng(11)
    x, y, h = ctx.vec(), ctx.vec(), ctx.vec()
    for l in range(P.nlevels):
        n = P.levels[l].ndof
        xv, yv = rng.standard_normal(n), rng.standard_normal(n)
        ctx.upload(l, x, np.zeros(n))
        ctx.upload(l, y, yv)
        ctx.smooth(l, 1, x, y, h)
        if not P.levels[l].pf_mask:
            assert np.array_equal(ctx.download(l, x), O.smooth(l, 1, np.zeros(n), yv)), l
        for niter in (1, 3):
            ctx.upload(l, x, xv)
            ctx.upload(l, y, yv)
            ctx.smooth(l, niter, x, y, h)
            assert rel(ctx.download(l, x), O.smooth(l, niter, xv, yv)) < 1e-11, (l, niter)
    for v in (x, y, h):
        ctx.free(v)


@pytest.mark.parametrize("name", _ilu_cases())
def test_ilu_smoothing_bitexact_and_solves(ctx, name):
    P, ref = load_golden(name)
    keys = ref["keys"]
    ctx.load_problem(P)
    ctx.set_params(**solver_keys(keys), gmressize=int(keys["gmressize"]),
                   tol=float(keys["tol"]), globaltol=1e-16, maxiter=100, smoother="ilu")
    O = Oracle(P, **solver_keys(keys), smoother="ilu")
    _sweeps_match(ctx, P, O)
    fl = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(fl, b, P.rhs)
    info = ctx.gmres(x, b)
    assert info["status_name"] == "converged"
    assert abs(info["iterations"] - ref["iterations"]) <= 1
    assert rel_l2(ctx.download(fl, x), ref["solution"]) < 1e-8
    ctx.set_params(**solver_keys(keys), gmressize=21, tol=1e-10, globaltol=1e-300,
                   maxiter=300, smoother="ilu")
    for prec in (GB_FP64, GB_FP32):
        fi = ctx.fgmres(x, b, prec)
        assert fi["true_rel_residual"] <= 1e-10
        assert rel_l2(ctx.download(fl, x), ref["solution"]) < 1e-6
    ctx.free(x)
    ctx.free(b)


def test_block_ilu_stokes_bitexact(ctx):
    """3x3 blocks (Q1/Q1 Stokes with the pressure filter): block products,
    block inverses and the filter in the sweep, against the oracle."""
    P = structured_stokes(2, 2, 3)
    ctx.load_problem(P)
    ctx.set_params(omega=1.0, smoother="ilu", gmressize=31, tol=1e-8, globaltol=1e-300,
                   maxiter=200)
    O = Oracle(P, omega=1.0, smoother="ilu")
    _sweeps_match(ctx, P, O)
    fl = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(fl, b, P.rhs)
    xo, io = O.gmres(vmax=31, tol=1e-8, globaltol=1e-300)
    info = ctx.gmres(x, b)
    assert abs(info["iterations"] - io["iterations"]) <= 1
    assert rel_l2(ctx.download(fl, x), xo) < 1e-8
    ctx.free(x)
    ctx.free(b)


def _context_with(env):
    import os

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


@pytest.mark.parametrize("cta_rows", ["4096", "600"])
def test_single_cta_level_runs_equal_level_launches(cta_rows):
    """The substitution levels run inside one CTA (a block barrier between
    levels) give the same results as one launch per level (the default), bit
    for bit: FP64 sweeps on the 33^3 and 65^3 Q1 levels (225 and 449
    dependency levels of up to 1073 rows) and FP32 and FP64 flexible solves,
    with every level in single-CTA runs (4096) and with a mix of single-CTA
    runs and wide-level launches (600)."""
    from gascoignelib_b200.problem import seeded_inputs, structured_problem
    kappa, rhs = seeded_inputs(3, 1, 6)
    P = structured_problem(3, 1, 6, kappa, rhs)
    fl = P.nlevels - 1
    out = {}
    for tag, env in (("launches", {"GB_ILU_CTA_ROWS": "0"}),
                     ("cta", {"GB_ILU_CTA_ROWS": cta_rows})):
        c = _context_with(env)
        try:
            c.load_problem(P)
            c.set_params(omega=1.0, smoother="ilu", gmressize=11, tol=1e-30,
                         globaltol=1e-300, maxiter=10)
            x, y, h = c.vec(), c.vec(), c.vec()
            res = []
            for l in (fl - 1, fl):
                n = P.levels[l].ndof
                r = np.random.default_rng(100 + l)
                c.upload(l, x, r.standard_normal(n))
                c.upload(l, y, r.standard_normal(n))
                c.smooth(l, 2, x, y, h)
                res.append(c.download(l, x))
            c.upload(fl, y, P.rhs)
            for prec in (GB_FP64, GB_FP32):
                c.fgmres(x, y, prec, check=False)
                res.append(c.download(fl, x))
            out[tag] = res
        finally:
            c.close()
    for a, b in zip(out["launches"], out["cta"]):
        assert np.array_equal(a, b)
