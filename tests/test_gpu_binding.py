"""The reference's own solver run through the compiled reference-side binding
(gascoignelib_b200/binding/b200solver.{h,cc}).

oracle/_ref/ref_harness_b200 builds each problem with the reference's classes
(MeshAgent, CGDisc assembly, StdMultiLevelSolver set-up and
NewtonLinearSolve), but constructs B200MultiLevelSolver in place of
StdMultiLevelSolver, the way CudaLoop::BasicInit installs
CudaMultiLevelSolver (cuda/cudaloop.cc:24-31). Its B200Solver levels upload the
reference's assembled matrices, Dirichlet nodes, hanging nodes, Vanka patches
and pressure filter; its B200MgInterpolatorNested transfers upload the mesh
transfer maps. NewtonLinearSolve then runs on the GPU:
  backend=b200      the whole GMRES solve as one C-ABI call (gb_gmres);
  backend=b200host  the reference's GMRES::solve, LinearMg and mgstep on the
                    host, every vector and level operation on the device.
Each result is compared with the same harness run on the CPU
(StdMultiLevelSolver): iteration count within +-1 and the solution within
1e-8 relative L2, the criterion for the FP64 path. The dual solve
(AssembleDualMatrix, then the same NewtonLinearSolve) is checked the same way.
"""
import os
import tempfile

import numpy as np
import pytest

from _util import stokes_rhs
from gascoignelib_b200.problem import seeded_inputs
from oracle.oracle import REF_HARNESS, REF_HARNESS_B200, run_reference, write_inputs

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(REF_HARNESS_B200),
                                 reason="binding harness not built")]

# name: (dim, coarse, refine, seeded kappa/rhs, tol, extra keys, threads)
CASES = {
    "q1_2d_poisson": (2, 2, 4, False, 1e-10, {}, None),
    "q1_3d_seeded": (3, 1, 3, True, 1e-8, {}, None),
    "q1_3d_wcycle": (3, 1, 3, True, 1e-8, {"mgtype": "W", "iterpre": 1, "iterpost": 3,
                                           "omega": 0.7}, None),
    "q1_2d_fcycle": (2, 2, 3, True, 1e-10, {"mgtype": "F", "mgomega": 0.9}, None),
    "q1_3d_conv": (3, 1, 3, True, 1e-8, {"conv": "1,0.5,0.25"}, None),
    "stokes_2d_vanka": (2, 2, 4, True, 1e-8, {"problem": "stokes", "smoother": "vanka",
                                              "omega": 1.0, "gmressize": 31}, 1),
    "stokes_2d_jacobi": (2, 2, 3, True, 1e-8, {"problem": "stokes", "smoother": "jacobi",
                                               "omega": 0.5, "gmressize": 31}, None),
    "ilu_2d_conv": (2, 2, 4, True, 1e-10, {"smoother": "ilu", "omega": 1.0,
                                           "conv": "4,2"}, None),
    "q2_3d_conv": (3, 1, 3, True, 1e-8, {"disc": "Q2", "conv": "1,0.5,0.25"}, None),
    "hn_2d_q1_ball": (2, 2, 3, False, 1e-10, {"ball": 0.25, "diff": 1.0,
                                              "rhsres": 2 * (2 << 3)}, None),
    "hn_3d_q2_ball": (3, 2, 3, False, 1e-8, {"disc": "Q2", "ball": 0.25, "diff": 1.0,
                                             "rhsres": 2 * (2 << 3)}, 1),
    "lps_2d_q2_conv": (2, 2, 3, False, 1e-10, {"disc": "Q2", "diff": 0.01, "lps": 0.5,
                                               "omega": 0.3, "gmressize": 41,
                                               "conv": "1,0.5"}, None),
}


def _inputs(d, dim, coarse, refine, seeded, keys):
    if keys.get("problem") == "stokes":
        return write_inputs(d, None, stokes_rhs(dim, coarse, refine))
    if seeded:
        kap, rhs = seeded_inputs(dim, coarse, refine)
        return write_inputs(d, kap, rhs)
    res = int(keys.get("rhsres", coarse << refine))
    rhs = np.random.default_rng(1002).uniform(-1.0, 1.0, size=(res + 1) ** dim)
    if "ball" not in keys:
        rhs = np.ones_like(rhs)
    return write_inputs(d, None, rhs)


def _run(case, backend, extra=None):
    dim, coarse, refine, seeded, tol, keys, threads = CASES[case]
    d = tempfile.mkdtemp(prefix=f"gb_bind_{case}_{backend}_")
    kw = dict(dim=dim, coarse=coarse, refine=refine, tol=tol, savesol=1, **keys)
    kw.update(extra or {})
    kw.update(_inputs(d, dim, coarse, refine, seeded, keys))
    harness = REF_HARNESS if backend == "cpu" else REF_HARNESS_B200
    if backend != "cpu":
        kw["backend"] = backend
    out, s = run_reference(d, threads=threads, harness=harness, **kw)
    u = np.fromfile(os.path.join(out, "solution.f64"))
    return out, s, u


def _check(s_cpu, u_cpu, s_dev, u_dev):
    it_c, it_d = int(s_cpu["iterations"][0]), int(s_dev["iterations"][0])
    assert abs(it_c - it_d) <= 1, (it_c, it_d)
    assert s_dev["status"][0] == s_cpu["status"][0]
    err = np.linalg.norm(u_dev - u_cpu) / np.linalg.norm(u_cpu)
    assert err < 1e-8, err
    return err


@pytest.mark.parametrize("case", sorted(CASES))
def test_binding_device_solve_matches_reference(case):
    _, s_cpu, u_cpu = _run(case, "cpu")
    _, s_dev, u_dev = _run(case, "b200")
    assert s_dev["backend"][0] == "b200"
    assert float(s_dev["device_ms"][0]) > 0.0   # the device solver ran
    _check(s_cpu, u_cpu, s_dev, u_dev)


@pytest.mark.parametrize("case", ["q1_2d_poisson", "q1_3d_wcycle", "stokes_2d_vanka",
                                  "hn_2d_q1_ball", "q1_2d_fcycle"])
def test_binding_host_driven_solve_matches_reference(case):
    """The reference's GMRES::solve / LinearMg / mgstep drive the device
    operations (vmulteq, residuals, smoothers, transfers, HN, Dirichlet,
    filter, vector ops) through the binding's virtual overrides."""
    _, s_cpu, u_cpu = _run(case, "cpu")
    _, s_dev, u_dev = _run(case, "b200host")
    assert s_dev["backend"][0] == "b200host"
    _check(s_cpu, u_cpu, s_dev, u_dev)


@pytest.mark.parametrize("backend", ["b200", "b200host"])
def test_binding_dual_solve_matches_reference(backend):
    """StdMultiLevelSolver::AssembleDualMatrix through B200Solver (the
    transposed, Dirichlet-row matrices uploaded), then the dual solve."""
    dim, coarse, refine = 3, 1, 3
    kap, rhs = seeded_inputs(dim, coarse, refine)
    g = np.random.default_rng(1004).uniform(-1.0, 1.0, size=((coarse << refine) + 1) ** dim)
    outs = {}
    for be in ("cpu", backend):
        d = tempfile.mkdtemp(prefix=f"gb_bind_dual_{be}_")
        kw = dict(dim=dim, coarse=coarse, refine=refine, tol=1e-8, savesol=1,
                  conv="1,0.5,0.25", **write_inputs(d, kap, rhs))
        p = os.path.join(d, "dual_in.f64")
        g.tofile(p)
        kw["dualrhs"] = p
        if be != "cpu":
            kw["backend"] = be
        out, s = run_reference(d, harness=REF_HARNESS if be == "cpu" else REF_HARNESS_B200,
                               **kw)
        ds = {}
        with open(os.path.join(out, "dual_summary.txt")) as f:
            for line in f:
                k, *v = line.split()
                ds[k] = v
        outs[be] = (s, np.fromfile(os.path.join(out, "solution.f64")), ds,
                    np.fromfile(os.path.join(out, "dual_solution.f64")))
    sc, uc, dc, zc = outs["cpu"]
    sd, ud, dd, zd = outs[backend]
    _check(sc, uc, sd, ud)
    assert abs(int(dc["dual_iterations"][0]) - int(dd["dual_iterations"][0])) <= 1
    assert np.linalg.norm(zd - zc) / np.linalg.norm(zc) < 1e-8


@pytest.mark.parametrize("dim,coarse,refine,tol", [(2, 2, 6, 1e-10), (3, 1, 6, 1e-8)])
def test_binding_full_size_c1_c2(dim, coarse, refine, tol):
    """The two smallest benchmark configurations at full size (2D Poisson
    128^2; 3D 64^3 with the seeded log-normal kappa) through the binding."""
    d = tempfile.mkdtemp(prefix="gb_bind_full_")
    if dim == 2:
        kw = write_inputs(d, None, np.ones(((coarse << refine) + 1) ** 2))
    else:
        kw = write_inputs(d, *seeded_inputs(dim, coarse, refine))
    res = {}
    for be in ("cpu", "b200"):
        k = dict(dim=dim, coarse=coarse, refine=refine, tol=tol, savesol=1, **kw)
        if be != "cpu":
            k["backend"] = be
        out, s = run_reference(tempfile.mkdtemp(prefix=f"gb_bind_full_{be}_"),
                               harness=REF_HARNESS if be == "cpu" else REF_HARNESS_B200, **k)
        res[be] = (s, np.fromfile(os.path.join(out, "solution.f64")))
    _check(res["cpu"][0], res["cpu"][1], res["b200"][0], res["b200"][1])


def _popen_reference(harness, out_dir, threads=None, **kw):
    import subprocess
    args = [harness, f"out={out_dir}"] + [f"{k}={v}" for k, v in kw.items()]
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    return subprocess.Popen(args, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, env=env)


def _summary(out_dir):
    s = {}
    with open(os.path.join(out_dir, "summary.txt")) as f:
        for line in f:
            k, *v = line.split()
            s[k] = v
    return s


def test_binding_c4_reference_mesh_full_size():
    """The C4 configuration on the reference's own mesh: 3D CGQ2
    convection-diffusion (eps 1e-2, beta (1, 0.5, 0.25)) on 80^3 cells, refined
    once more where MeshAgent::refine_cells refines the leaf cells whose
    centroid lies in |x - 0.5| < 0.25 (1,017,329 dofs on the finest of 5
    levels, edge and face hanging nodes), f ~ U[-1, 1] (seed 1002), Jacobi
    V(2,2) with omega 0.3, one GMRES cycle of up to 127 steps to 1e-8. The
    reference's CPU solve and the binding's device solve (FP64, and mixed
    precision) of the same assembled system run side by side."""
    res = 2 * (5 << 4)
    d = tempfile.mkdtemp(prefix="gb_bind_c4_")
    rhs = np.random.default_rng(1002).uniform(-1.0, 1.0, size=(res + 1) ** 3)
    kw = dict(dim=3, coarse=5, refine=4, disc="Q2", ball=0.25, diff=0.01,
              conv="1,0.5,0.25", rhsres=res, tol=1e-8, globaltol=1e-16, gmressize=128,
              maxiter=200, iterpre=2, iterpost=2, omega=0.3, savesol=1, functional=1,
              **write_inputs(d, None, rhs))
    outs = {be: tempfile.mkdtemp(prefix=f"gb_bind_c4_{be}_")
            for be in ("cpu", "b200", "b200mixed")}
    procs = {"cpu": _popen_reference(REF_HARNESS, outs["cpu"], **kw)}
    # the device runs one after the other, the CPU reference beside them
    for be in ("b200", "b200mixed"):
        p = _popen_reference(REF_HARNESS_B200, outs[be], backend=be, **kw)
        _, err = p.communicate(timeout=1800)
        assert p.returncode == 0, err.decode()[-2000:]
    _, err = procs["cpu"].communicate(timeout=1800)
    assert procs["cpu"].returncode == 0, err.decode()[-2000:]
    s = {be: _summary(o) for be, o in outs.items()}
    u = {be: np.fromfile(os.path.join(o, "solution.f64")) for be, o in outs.items()}
    assert int(s["cpu"]["nnodes_L4"][0]) == 1017329
    assert s["cpu"]["status"][0] == "converged"
    _check(s["cpu"], u["cpu"], s["b200"], u["b200"])
    # mixed: the true residual reaches the tolerance; u and J agree with the
    # reference's FP64 solution to the accuracy that tolerance allows
    assert float(s["b200mixed"]["true_rel_residual"][0]) <= 1e-8
    err = np.linalg.norm(u["b200mixed"] - u["cpu"]) / np.linalg.norm(u["cpu"])
    assert err < 1e-6, err
    J = {be: float(s[be]["functional_l2"][0]) for be in s}
    assert abs(J["b200"] - J["cpu"]) <= 1e-8 * abs(J["cpu"])
    assert abs(J["b200mixed"] - J["cpu"]) <= 1e-6 * abs(J["cpu"])


def test_binding_c3_lps_lid_mixed():
    """The C3 operator as the benchmark states it on a reduced grid (64^2
    cells): the reference's NavierStokesLps at u = 0 (CGQ1Lps), lid-driven
    data, Vanka, pressure filter, through the binding in FP64 (parity) and in
    mixed precision (true residual)."""
    kw = dict(dim=2, coarse=2, refine=5, problem="stokeslps", smoother="vanka",
              omega=1.0, gmressize=31, stab=0.1, tol=1e-8, savesol=1, functional=1)
    res = {}
    for be in ("cpu", "b200", "b200mixed"):
        d = tempfile.mkdtemp(prefix=f"gb_bind_c3_{be}_")
        k = dict(kw)
        if be != "cpu":
            k["backend"] = be
        out, s = run_reference(d, threads=1, harness=REF_HARNESS if be == "cpu"
                               else REF_HARNESS_B200, **k)
        res[be] = (s, np.fromfile(os.path.join(out, "solution.f64")))
    _check(res["cpu"][0], res["cpu"][1], res["b200"][0], res["b200"][1])
    assert float(res["b200mixed"][0]["true_rel_residual"][0]) <= 1e-8
    um, uc = res["b200mixed"][1], res["cpu"][1]
    assert np.linalg.norm(um - uc) / np.linalg.norm(uc) < 1e-6
