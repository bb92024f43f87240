"""Matrix-free Form, the Newton residual and the solution files on the GPU:
StdSolver::Form / StdMultiLevelSolver::NewtonResidual of a seeded vector and
the WriteBackUp / WriteBackUpBinary files and the StdSolver::Visu VTK file,
against what the reference itself computed and wrote (golden fixtures)."""
import os
import tempfile

import numpy as np
import pytest

from _util import (golden_form_cases, golden_kappa_beta, golden_vtk_cases, load_golden,
                   set_uniform_meshes, vtk_cells)
from gascoignelib_b200.native import GBError

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", golden_form_cases())
def test_form_and_newton_residual_match_reference(ctx, name):
    P, ref = load_golden(name)
    kappa, beta = golden_kappa_beta(name)
    ctx.load_problem(P)
    set_uniform_meshes(ctx, P)
    ctx.assemble_levels(kappa, beta)
    fl = P.nlevels - 1
    x, y, b = ctx.vec(), ctx.vec(), ctx.vec()
    ctx.upload(fl, x, ref["formx"])
    ctx.upload(fl, y, np.zeros(P.finest.n))
    ctx.form(fl, y, x, 1.0)
    f = ctx.download(fl, y)
    assert np.abs(f - ref["form"]).max() <= 1e-13 * np.abs(ref["form"]).max()
    # y += d Form(x) accumulates: d = -1 on top gives zero up to rounding
    ctx.form(fl, y, x, -1.0)
    assert np.abs(ctx.download(fl, y)).max() <= 1e-13 * np.abs(ref["form"]).max()
    ctx.upload(fl, b, P.rhs)
    nr = ctx.newton_residual(y, x, b)
    r = ctx.download(fl, y)
    scale = np.abs(ref["newton_residual"]).max()
    assert np.abs(r - ref["newton_residual"]).max() <= 1e-13 * scale
    assert abs(nr - ref["newton_norm"]) <= 1e-13 * ref["newton_norm"]
    # at the solution the residual equals b - A u on the interior rows
    ctx.upload(fl, x, ref["solution"])
    ctx.newton_residual(y, x, b)
    import scipy.sparse as sp
    L = P.finest
    A = sp.csr_matrix((L.val, L.col, L.rowptr), shape=(L.n, L.n))
    res = P.rhs - A @ ref["solution"]
    res[L.dirichlet] = 0.0
    assert np.abs(ctx.download(fl, y) - res).max() <= 1e-12 * np.abs(P.rhs).max()
    for v in (x, y, b):
        ctx.free(v)


@pytest.mark.parametrize("name", golden_form_cases())
def test_backup_files_match_reference(ctx, name):
    """The library writes the reference's .bup / .bip bytes for the same
    vector, reads the reference's files back bit for bit, and adds on request."""
    P, ref = load_golden(name)
    ctx.load_problem(P)
    fl = P.nlevels - 1
    u = ctx.vec()
    ctx.upload(fl, u, ref["solution"])
    d = tempfile.mkdtemp()
    for ext, binary in (("bup", False), ("bip", True)):
        mine = os.path.join(d, "mine." + ext)
        ctx.write_backup(fl, u, mine, binary=binary)
        assert open(mine, "rb").read() == ref["backup_" + ext].tobytes()
        theirs = os.path.join(d, "solution." + ext)
        with open(theirs, "wb") as f:
            f.write(ref["backup_" + ext].tobytes())
        v = ctx.vec()
        ctx.upload(fl, v, np.full(P.finest.ndof, 7.0))
        ctx.read_backup(fl, v, theirs, binary=binary)
        assert np.array_equal(ctx.download(fl, v), ref["solution"])
        ctx.read_backup(fl, v, theirs, binary=binary, add=True)
        assert np.array_equal(ctx.download(fl, v), 2.0 * ref["solution"])
        ctx.free(v)
    # a file of another level's size is refused
    with pytest.raises(GBError, match="does not hold"):
        ctx.read_backup(0, u, os.path.join(d, "solution.bup"))
    with pytest.raises(GBError, match="not found"):
        ctx.read_backup(fl, u, os.path.join(d, "missing.bup"))
    ctx.free(u)


@pytest.mark.parametrize("name", golden_vtk_cases())
def test_vtk_file_matches_reference(ctx, name):
    """gb_vec_write_vtk writes the reference's VTK file (StdSolver::Visu) byte
    for byte from the device vector, the level's coordinates and the mesh's
    cells; on a level with hanging nodes the written values are averaged and
    the vector is left as it was."""
    P, ref = load_golden(name)
    ctx.load_problem(P)
    fl = P.nlevels - 1
    u = ctx.vec()
    ctx.upload(fl, u, ref["solution"])
    d = tempfile.mkdtemp()
    ctx.write_vtk(fl, u, os.path.join(d, "mine"), 0, P.dim, vtk_cells(ref["vtk"]),
                  P.finest.coord)
    assert open(os.path.join(d, "mine.00000.vtk"), "rb").read() == ref["vtk"].tobytes()
    assert np.array_equal(ctx.download(fl, u), ref["solution"])
    with pytest.raises(GBError, match="out of range"):
        bad = vtk_cells(ref["vtk"])
        bad[0, 0] = P.finest.n
        ctx.write_vtk(fl, u, os.path.join(d, "bad"), 0, P.dim, bad, P.finest.coord)
    ctx.free(u)
