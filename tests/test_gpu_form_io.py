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


def _form_cases():
    from _util import golden_cases
    out = []
    for n in golden_cases():
        if n.startswith("form_"):
            continue
        with np.load(os.path.join(os.path.dirname(__file__), "golden", n + ".npz")) as z:
            if "formx" in z.files:
                out.append(n)
    return out


@pytest.mark.parametrize("name", _form_cases())
def test_form_on_patch_and_hanging_levels_matches_reference(ctx, name):
    """StdSolver::Form and NewtonResidual on levels of Q2 elements, of Q1
    functions on patches with LPS, and with hanging nodes (HNAverage of x, the
    residuals at the cells' own nodes, HNZero of x, HNDistribute of y): the
    reference's vectors within 1e-13."""
    from _util import (ball_meshes, golden_kappa_beta, golden_lps_cases, q2_element_kappa,
                       uniform_meshes_q2)
    P, ref = load_golden(name)
    ctx.load_problem(P)
    keys = ref["keys"]
    lps = None
    if name.startswith("hn_"):
        deg = 2 if str(keys["disc"]) == "Q2" else 1
        meshes = ball_meshes(P, deg)
        kap = np.full(meshes[-1][0].shape[0], float(keys["diff"]))
        beta = ([float(t) for t in str(keys["conv"]).split(",")] if "conv" in keys else None)
    elif name.startswith("lps_"):
        _, deg, diff, beta, lps = next(c for c in golden_lps_cases() if c[0] == name)
        meshes = uniform_meshes_q2(P)
        kap = np.full(meshes[-1][0].shape[0], diff)
    else:  # q2_: the seeded per-cell kappa, per element the mean of its cells
        deg = 2
        kappa, beta = golden_kappa_beta(name)
        meshes = uniform_meshes_q2(P)
        kap = q2_element_kappa(P.dim, kappa, round(len(kappa) ** (1.0 / P.dim)))
    for l, (el, par) in enumerate(meshes):
        ctx.set_mesh(l, P.dim, el, P.levels[l].coord, par if l else None, degree=deg)
    try:
        if lps:
            ctx.set_assembly_lps(*lps)
        ctx.assemble_levels(kap, beta)
    finally:
        ctx.set_assembly_lps(0.0)
    fl = P.nlevels - 1
    x, y, b = ctx.vec(), ctx.vec(), ctx.vec()
    ctx.upload(fl, x, ref["formx"])
    ctx.upload(fl, y, np.zeros(P.finest.ndof))
    ctx.form(fl, y, x, 1.0)
    scale = np.abs(ref["form"]).max()
    assert np.abs(ctx.download(fl, y) - ref["form"]).max() <= 1e-13 * scale
    ctx.upload(fl, x, ref["formx"])
    ctx.upload(fl, b, P.rhs)
    nr = ctx.newton_residual(y, x, b)
    scale = np.abs(ref["newton_residual"]).max()
    assert np.abs(ctx.download(fl, y) - ref["newton_residual"]).max() <= 1e-13 * scale
    assert abs(nr - ref["newton_norm"]) <= 1e-13 * ref["newton_norm"]
    for v in (x, y, b):
        ctx.free(v)
