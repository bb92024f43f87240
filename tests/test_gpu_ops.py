"""Per-operator parity of the CUDA path (through the C-ABI) with the oracle.

Tolerances: FP64 products and smoothing sweeps accumulate in the reference's
column order but with fused multiply-adds, so they agree to a few ulps
(rel 1e-13); transfers use exact power-of-two weights in the reference's order
and agree bit for bit; FP32 operators agree to FP32 rounding (rel 1e-5).
"""
import numpy as np
import pytest

from _util import golden_cases, load_golden, rel, solver_keys
from gascoignelib_b200.native import GB_FP32, GB_FP64
from gascoignelib_b200.problem import seeded_inputs, structured_problem
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def _problems():
    out = [("golden:" + n, load_golden(n)[0], solver_keys(load_golden(n)[1]["keys"]))
           for n in golden_cases()]
    for dim, coarse, refine in [(2, 1, 2), (2, 2, 5), (3, 1, 4), (3, 2, 2)]:
        k, r = seeded_inputs(dim, coarse, refine, kappa_seed=11, rhs_seed=12)
        out.append((f"struct:{dim}d_c{coarse}_r{refine}",
                    structured_problem(dim, coarse, refine, k, r), solver_keys({})))
    return out


PROBLEMS = _problems()
IDS = [p[0] for p in PROBLEMS]


@pytest.fixture(params=range(len(PROBLEMS)), ids=IDS)
def loaded(request, ctx):
    name, P, keys = PROBLEMS[request.param]
    ctx.load_problem(P)
    ctx.set_params(**keys)
    return P, keys, Oracle(P, **keys)


def test_spmv_and_transpose(ctx, loaded):
    P, keys, O = loaded
    rng = np.random.default_rng(5)
    x, y = ctx.vec(), ctx.vec()
    for l in range(P.nlevels):
        n = P.levels[l].ndof
        xv, y0 = rng.standard_normal(n), rng.standard_normal(n)
        ctx.upload(l, x, xv)
        ctx.upload(l, y, y0)
        ctx.vmult(l, y, x, -0.7)
        assert rel(ctx.download(l, y), O.vmult(l, y0, xv, -0.7)) < 1e-13
        ctx.vmulteq(l, y, x, 1.3)
        assert rel(ctx.download(l, y), O.vmult(l, np.zeros(n), xv, 1.3)) < 1e-13
        ctx.upload(l, y, y0)
        ctx.vmult_transpose(l, y, x, 0.5)
        assert rel(ctx.download(l, y), O.vmult_transpose(l, y0, xv, 0.5)) < 1e-13
    ctx.free(x)
    ctx.free(y)


def test_residuals_and_dirichlet(ctx, loaded):
    P, keys, O = loaded
    rng = np.random.default_rng(6)
    x, b, y = ctx.vec(), ctx.vec(), ctx.vec()
    for l in range(P.nlevels):
        n = P.levels[l].ndof
        xv, bv = rng.standard_normal(n), rng.standard_normal(n)
        ctx.upload(l, x, xv)
        ctx.upload(l, b, bv)
        ctx.matrix_residual(l, y, x, b)
        r = O.matrix_residual(l, xv, bv)
        assert rel(ctx.download(l, y), r) < 1e-13
        # residualgmres: b - A x, Dirichlet-zeroed, no pressure filter
        ctx.residualgmres(l, y, x, b)
        assert rel(ctx.download(l, y), O.dirichlet_zero(l, O.vmult(l, bv, xv, -1.0))) < 1e-13
        ctx.dirichlet_zero(l, x)
        assert np.array_equal(ctx.download(l, x), O.dirichlet_zero(l, xv))
    for v in (x, b, y):
        ctx.free(v)


def test_inverse_diagonal_bitexact(ctx, loaded):
    P, keys, O = loaded
    for l in range(P.nlevels):
        assert np.array_equal(ctx.inverse_diagonal(l), O.blockdiag_inverse(l))


def test_smoothing(ctx, loaded):
    """StdSolver::smooth with the problem's smoother (Jacobi, block Jacobi or
    Vanka; with the pressure filter where the problem has one)."""
    P, keys, O = loaded
    rng = np.random.default_rng(7)
    x, y, h = ctx.vec(), ctx.vec(), ctx.vec()
    for l in range(P.nlevels):
        n = P.levels[l].ndof
        lv = P.levels[l]
        if (P.info.get("smoother") == "vanka" and lv.patches is not None
                and lv.patches.shape[0] == 1):
            continue  # one patch = the whole singular level (test_gpu_stokes)
        xv, yv = rng.standard_normal(n), rng.standard_normal(n)
        for niter in (1, 2, 3):
            ctx.upload(l, x, xv)
            ctx.upload(l, y, yv)
            ctx.smooth(l, niter, x, y, h)
            assert rel(ctx.download(l, x), O.smooth(l, niter, xv, yv)) < 1e-11
    for v in (x, y, h):
        ctx.free(v)


def test_transfers_bitexact(ctx, loaded):
    P, keys, O = loaded
    rng = np.random.default_rng(8)
    c, f = ctx.vec(), ctx.vec()
    for l in range(P.nlevels - 1):
        fv = rng.standard_normal(P.levels[l + 1].ndof)
        cv = rng.standard_normal(P.levels[l].ndof)
        ctx.upload(l + 1, f, fv)
        ctx.restrict_zero(l, c, f)
        assert np.array_equal(ctx.download(l, c), O.restrict_zero(l, fv))
        ctx.upload(l, c, cv)
        ctx.upload(l + 1, f, np.zeros_like(fv))
        ctx.prolongate_add(l, f, c)
        assert np.array_equal(ctx.download(l + 1, f), O.prolongate_add(l, np.zeros_like(fv), cv))
        ctx.upload(l + 1, f, fv)
        ctx.prolongate_add(l, f, c)
        assert rel(ctx.download(l + 1, f), O.prolongate_add(l, fv, cv)) < 1e-15
    ctx.free(c)
    ctx.free(f)


def test_vector_ops(ctx, loaded):
    P, keys, O = loaded
    rng = np.random.default_rng(9)
    a, b = ctx.vec(), ctx.vec()
    l = P.nlevels - 1
    n = P.levels[l].ndof
    av, bv = rng.standard_normal(n), rng.standard_normal(n)
    ctx.upload(l, a, av)
    ctx.upload(l, b, bv)
    assert abs(ctx.dot(l, a, b) - av @ bv) <= 1e-13 * np.abs(av * bv).sum()
    assert abs(ctx.norm(l, a) - np.linalg.norm(av)) <= 1e-14 * np.linalg.norm(av)
    ctx.add(l, a, 0.25, b)
    assert rel(ctx.download(l, a), av + 0.25 * bv) < 1e-15
    ctx.equ(l, a, -2.0, b)
    assert np.array_equal(ctx.download(l, a), -2.0 * bv)
    ctx.zero(l, a)
    assert not ctx.download(l, a).any()
    ctx.free(a)
    ctx.free(b)


def test_one_cycle_fp64_and_fp32(ctx, loaded):
    """StdMultiLevelSolver::precondition: one cycle from the current x."""
    P, keys, O = loaded
    rng = np.random.default_rng(10)
    l = P.nlevels - 1
    n = P.levels[l].ndof
    x, y = ctx.vec(), ctx.vec()
    for x0 in (np.zeros(n), rng.standard_normal(n)):
        yv = O.dirichlet_zero(l, rng.standard_normal(n))
        ref = O.precondition(x0, yv)
        ctx.upload(l, x, x0)
        ctx.upload(l, y, yv)
        ctx.precondition(x, y, GB_FP64)
        assert rel(ctx.download(l, x), ref) < 1e-11
        ctx.upload(l, x, x0)
        ctx.precondition(x, y, GB_FP32)
        # FP32 cycle: FP32 rounding, amplified in block systems by the Vanka
        # local solves (the 3D coarsest level is one singular patch)
        assert rel(ctx.download(l, x), ref) < (2e-5 if P.finest.B == 1 else 1e-3)
    ctx.free(x)
    ctx.free(y)


def test_bad_arguments_return_codes(ctx):
    from gascoignelib_b200.native import GB_EINVAL, GBError
    P = structured_problem(2, 1, 2)
    ctx.load_problem(P)
    v = ctx.vec()
    with pytest.raises(GBError) as e:
        ctx.upload(0, v, np.zeros(P.levels[0].ndof + 1))
    assert e.value.code == GB_EINVAL
    with pytest.raises(GBError):
        ctx.vmult(5, v, v)
    with pytest.raises(GBError):
        ctx.set_params(gmressize=1000)
    with pytest.raises(GBError):
        ctx.set_params(mgtype="X")
    ctx.free(v)
