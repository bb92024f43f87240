"""Block systems on the GPU (Stokes, ncomp = dim + 1): block SpMV, block
Jacobi, Vanka, the pressure filter, block transfers and the solvers, against
the oracle and the reference's golden Stokes fixtures."""
import numpy as np
import pytest

from _util import golden_stokes_cases, load_golden, rel, rel_l2, solver_keys
from gascoignelib_b200.native import GB_FP32, GB_FP64
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def _single_patch_vanka(P, l):
    """A Vanka level whose one patch is the whole level: its local matrix is
    the level's Stokes matrix, singular (constant pressure), so the local
    solve's pressure part is rounding noise that the filter only partly
    removes; the LU solves and the inverse then agree on the velocities only."""
    lv = P.levels[l]
    return (P.info.get("smoother") == "vanka" and lv.patches is not None
            and lv.patches.shape[0] == 1)


def _setup(ctx, name):
    P, ref = load_golden(name)
    keys = ref["keys"]
    ctx.load_problem(P)
    ctx.set_params(**solver_keys(keys), gmressize=int(keys["gmressize"]),
                   tol=float(keys["tol"]), globaltol=1e-16, maxiter=200)
    return P, ref, keys


@pytest.mark.parametrize("name", golden_stokes_cases())
def test_block_operators_match_oracle(ctx, name):
    P, ref, keys = _setup(ctx, name)
    O = Oracle(P, **solver_keys(keys))
    rng = np.random.default_rng(4)
    for l in range(P.nlevels):
        lv = P.levels[l]
        n = lv.ndof
        xv, bv = rng.normal(size=n), rng.normal(size=n)
        x, y, b = ctx.vec(), ctx.vec(), ctx.vec()
        ctx.upload(l, x, xv)
        ctx.upload(l, b, bv)
        ctx.zero(l, y)
        ctx.vmult(l, y, x, 1.0)
        assert rel(ctx.download(l, y), O.vmult(l, np.zeros(n), xv)) < 1e-13
        # MatrixResidual with SubtractMeanAlgebraic
        ctx.matrix_residual(l, y, x, b)
        assert rel(ctx.download(l, y), O.matrix_residual(l, xv, bv)) < 1e-12
        # inverse diagonal blocks: NodeMatrix::gauss_jordan, bit for bit
        assert np.array_equal(ctx.inverse_diagonal(l), O.blockdiag_inverse(l))
        # pressure filter
        ctx.upload(l, y, xv)
        ctx.subtract_mean(l, y)
        assert rel(ctx.download(l, y), O.subtract_mean(l, xv)) < 1e-13
        ctx.upload(l, y, xv)
        ctx.subtract_mean(l, y, algebraic=True)
        assert rel(ctx.download(l, y), O.subtract_mean(l, xv, algebraic=True)) < 1e-13
        if l > 0:
            c = ctx.vec()
            ctx.restrict_zero(l - 1, c, x)
            assert np.array_equal(ctx.download(l - 1, c), O.restrict_zero(l - 1, xv))
            cv = rng.normal(size=P.levels[l - 1].ndof)
            ctx.upload(l - 1, c, cv)
            ctx.upload(l, y, xv)
            ctx.prolongate_add(l - 1, y, c)
            assert np.array_equal(ctx.download(l, y), O.prolongate_add(l - 1, xv, cv))
            ctx.free(c)
        for v in (x, y, b):
            ctx.free(v)


@pytest.mark.parametrize("name", golden_stokes_cases())
def test_smoother_sweeps_match_oracle(ctx, name):
    """Vanka or block-Jacobi sweeps with the pressure filter, from a nonzero
    start, within rounding of the oracle."""
    P, ref, keys = _setup(ctx, name)
    O = Oracle(P, **solver_keys(keys))
    rng = np.random.default_rng(5)
    for l in range(P.nlevels):
        n = P.levels[l].ndof
        if _single_patch_vanka(P, l):
            continue
        xv, yv = rng.normal(size=n), rng.normal(size=n)
        x, y, h = ctx.vec(), ctx.vec(), ctx.vec()
        ctx.upload(l, x, xv)
        ctx.upload(l, y, yv)
        ctx.smooth(l, 3, x, y, h)
        assert rel(ctx.download(l, x), O.smooth(l, 3, xv, yv)) < 1e-11
        for v in (x, y, h):
            ctx.free(v)


@pytest.mark.parametrize("name", golden_stokes_cases())
def test_stokes_gmres_matches_reference(ctx, name):
    P, ref, keys = _setup(ctx, name)
    l = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(l, b, P.rhs)
    info = ctx.gmres(x, b)
    u = ctx.download(l, x)
    assert info["status_name"] == "converged"
    assert abs(info["iterations"] - ref["iterations"]) <= 1
    assert rel_l2(u, ref["solution"]) < 1e-8
    ctx.free(x)
    ctx.free(b)


@pytest.mark.parametrize("prec", [GB_FP64, GB_FP32])
@pytest.mark.parametrize("name", golden_stokes_cases())
def test_stokes_flexible_gmres(ctx, name, prec):
    """Flexible GMRES with an FP64 or FP32 Vanka/Jacobi cycle: true residual
    at tol and the reference's solution (its pressure mean fixed by the
    filter) within the solve tolerance."""
    P, ref, keys = _setup(ctx, name)
    ctx.set_params(**solver_keys(keys), gmressize=int(keys["gmressize"]), tol=1e-10,
                   globaltol=1e-300, maxiter=300)
    l = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(l, b, P.rhs)
    info = ctx.fgmres(x, b, prec)
    u = ctx.download(l, x)
    assert info["status_name"] == "converged"
    assert info["true_rel_residual"] <= 1e-10
    O = Oracle(P, **solver_keys(keys))
    r = O.matrix_residual(l, u, P.rhs)
    assert rel_l2(u, ref["solution"]) < 1e-6
    ctx.free(x)
    ctx.free(b)


def test_c3_stokes_vanka_full_size(ctx):
    """C3 shape: 512^2 Q1/Q1 Stokes (789,507 dofs), Vanka V(2,2), GMRES(30):
    reference-semantics FP64 solve against the oracle (iterations +-1, 1e-8),
    then the mixed solve (FP32 Vanka cycle) to a true residual of 1e-8."""
    from gascoignelib_b200.problem import structured_stokes
    P = structured_stokes(2, 2, 8)
    assert P.finest.ndof == 789507
    O = Oracle(P, omega=1.0)
    xo, io = O.gmres(vmax=31, tol=1e-8, maxiter=200)
    O.close()
    ctx.load_problem(P)
    ctx.set_params(gmressize=31, tol=1e-8, globaltol=1e-16, maxiter=200, omega=1.0)
    l = P.nlevels - 1
    x, b = ctx.vec(), ctx.vec()
    ctx.upload(l, b, P.rhs)
    info = ctx.gmres(x, b)
    assert info["status_name"] == "converged"
    assert abs(info["iterations"] - io["iterations"]) <= 1
    assert rel_l2(ctx.download(l, x), xo) < 1e-8
    ctx.set_params(gmressize=31, tol=1e-8, globaltol=1e-300, maxiter=300, omega=1.0)
    for prec in (GB_FP32, GB_FP64):
        info = ctx.fgmres(x, b, prec)
        assert info["status_name"] == "converged"
        assert info["true_rel_residual"] <= 1e-8
        assert rel_l2(ctx.download(l, x), xo) < 1e-5
    ctx.free(x)
    ctx.free(b)


def test_vanka_cell_patches_match_oracle(ctx):
    """The 12 x 12 variant (Vanka on single cells, 4 nodes x 3 components):
    sweeps and the GMRES solve against the oracle with the same patches."""
    from gascoignelib_b200.problem import structured_stokes
    P = structured_stokes(2, 2, 5, patches="cell")
    assert P.finest.patches.shape[1] == 4
    O = Oracle(P, omega=1.0)
    ctx.load_problem(P)
    ctx.set_params(gmressize=31, tol=1e-8, globaltol=1e-16, maxiter=200, omega=1.0)
    rng = np.random.default_rng(6)
    l = P.nlevels - 1
    xv, yv = rng.normal(size=P.finest.ndof), rng.normal(size=P.finest.ndof)
    x, y, h = ctx.vec(), ctx.vec(), ctx.vec()
    ctx.upload(l, x, xv)
    ctx.upload(l, y, yv)
    ctx.smooth(l, 2, x, y, h)
    assert rel(ctx.download(l, x), O.smooth(l, 2, xv, yv)) < 1e-11
    xo, io = O.gmres(vmax=31, tol=1e-8, maxiter=200)
    ctx.upload(l, y, P.rhs)
    info = ctx.gmres(x, y)
    assert info["status_name"] == "converged"
    assert abs(info["iterations"] - io["iterations"]) <= 1
    assert rel_l2(ctx.download(l, x), xo) < 1e-8
    for v in (x, y, h):
        ctx.free(v)


@pytest.mark.parametrize("name", golden_stokes_cases())
def test_vanka_factors_on_device_equal_host_factors(name):
    """The patch inverses formed on the device (k_vanka_factor: gather from the
    SELL values, partial-pivot LU, substitutions) equal, bit for bit, those of
    the same arithmetic on the host (GB_VANKA_HOST=1), on every level."""
    import os

    from gascoignelib_b200.native import Context
    P, ref = load_golden(name)
    if P.levels[-1].patches is None:
        pytest.skip("no Vanka patches")
    inv = {}
    for mode in ("device", "host"):
        old = os.environ.get("GB_VANKA_HOST")
        os.environ["GB_VANKA_HOST"] = "1" if mode == "host" else "0"
        try:
            c = Context(0)
        finally:
            if old is None:
                os.environ.pop("GB_VANKA_HOST", None)
            else:
                os.environ["GB_VANKA_HOST"] = old
        try:
            c.load_problem(P)
            c.set_params(smoother="vanka")
            inv[mode] = [c.vanka_inverse(l, L.patches.shape[0], L.patches.shape[1] * L.B)
                         for l, L in enumerate(P.levels)]
        finally:
            c.close()
    for a, b in zip(inv["device"], inv["host"]):
        assert np.array_equal(a, b)
