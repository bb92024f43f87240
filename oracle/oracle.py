"""ORACLE - TEST INFRASTRUCTURE ONLY.

ctypes binding of the C restatement in ``gascoigne_oracle.c`` (built by
``oracle/Makefile`` into ``oracle/_lib``) and a runner for the compiled reference
harness (``oracle/_ref/ref_harness``, built from the reference's own sources by
``oracle/ref/Makefile``). Only the tests, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg use this module, as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libgascoigne_oracle.so")
REF_HARNESS = os.path.join(HERE, "_ref", "ref_harness")
REF_HARNESS_B200 = os.path.join(HERE, "_ref", "ref_harness_b200")

_P64 = C.POINTER(C.c_int64)
_PD = C.POINTER(C.c_double)


class _Level(C.Structure):
    _fields_ = [("n", C.c_int64), ("B", C.c_int), ("rowptr", _P64), ("col", _P64),
                ("diag", _P64), ("val", _PD), ("ndir", C.c_int64), ("dir", _P64),
                ("dircomp_mask", C.c_int), ("pf_mask", C.c_int), ("pf_w", _PD),
                ("pf_domain", C.c_double), ("nhanging", C.c_int64),
                ("npatch", C.c_int64), ("npp", C.c_int), ("patches", _P64),
                ("hn_disc", C.c_int), ("nhedge", C.c_int64), ("hnedge", _P64),
                ("nhface", C.c_int64), ("hnface", _P64)]


class _Transfer(C.Structure):
    _fields_ = [("ncoarse", C.c_int64), ("nfine", C.c_int64),
                ("r_ptr", _P64), ("r_col", _P64), ("r_w", _PD),
                ("p_ptr", _P64), ("p_col", _P64), ("p_w", _PD)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, "_lib/libgascoigne_oracle.so"],
                           check=True, capture_output=True)
        L = C.CDLL(LIB_PATH)
        L.or_mg_create.restype = C.c_void_p
        L.or_mg_create.argtypes = [C.c_int, C.POINTER(_Level), C.POINTER(_Transfer),
                                   C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                   C.c_char, C.c_int]
        L.or_mg_free.argtypes = [C.c_void_p]
        L.or_mg_set_direct.argtypes = [C.c_void_p, C.c_int]
        L.or_transfer_build.argtypes = [C.POINTER(_Transfer), C.c_int64, _P64,
                                        C.c_int64, _P64, C.c_int64, _P64, C.c_int64,
                                        _P64]
        L.or_transfer_free.argtypes = [C.POINTER(_Transfer)]
        L.or_gmres_solve.argtypes = [C.c_void_p, _PD, _PD, C.c_int, C.c_double,
                                     C.c_double, C.c_int, C.POINTER(C.c_int),
                                     C.POINTER(C.c_int), _PD, _PD, _PD]
        L.or_precondition.argtypes = [C.c_void_p, _PD, _PD]
        L.or_bsr_vmult.argtypes = [C.POINTER(_Level), _PD, _PD, C.c_double]
        L.or_bsr_vmult_transpose.argtypes = [C.POINTER(_Level), _PD, _PD, C.c_double]
        L.or_jacobi.argtypes = [C.POINTER(_Level), _PD]
        L.or_blockdiag_inverse.argtypes = [C.POINTER(_Level), _PD]
        L.or_smooth.argtypes = [C.c_void_p, C.c_int, C.c_int, _PD, _PD, _PD]
        L.or_restrict_zero.argtypes = [C.POINTER(_Transfer), C.c_int, _PD, _PD]
        L.or_prolongate_add.argtypes = [C.POINTER(_Transfer), C.c_int, _PD, _PD]
        L.or_dirichlet_zero.argtypes = [C.POINTER(_Level), _PD]
        L.or_matrix_residual.argtypes = [C.POINTER(_Level), _PD, _PD, _PD]
        L.or_subtract_mean.argtypes = [C.POINTER(_Level), _PD]
        L.or_subtract_mean_algebraic.argtypes = [C.POINTER(_Level), _PD]
        L.or_vanka_factor.argtypes = [C.POINTER(_Level), C.c_int64, _PD,
                                      C.POINTER(C.c_int)]
        L.or_vanka_solve.argtypes = [C.POINTER(_Level), _PD, C.POINTER(C.c_int), _PD,
                                     _PD, C.POINTER(C.c_int)]
        for f in ("or_hn_average", "or_hn_distribute", "or_hn_zero"):
            getattr(L, f).argtypes = [C.POINTER(_Level), _PD]
        L.or_dot.restype = C.c_double
        L.or_dot.argtypes = [C.c_int64, _PD, _PD]
        _lib = L
    return _lib


def _p64(a):
    return a.ctypes.data_as(_P64)


def _pd(a):
    return a.ctypes.data_as(_PD)


class Oracle:
    """FP64 CPU restatement of the reference's multilevel GMRES on a Problem."""

    def __init__(self, prob, iterpre=2, iterpost=2, iterexact=10, omega=0.8,
                 mgomega=1.0, mgtype="V", smoother=None, ndirect=0):
        """ndirect: the coarsest level is solved exactly (dense LU) when it has
        fewer nodes (the reference's ndirect key with UMFPACK compiled in);
        0 keeps the iterexact sweeps."""
        L = lib()
        self.prob = prob
        self._keep = []
        nl = prob.nlevels
        self.levels = (_Level * nl)()
        for l, lv in enumerate(prob.levels):
            arrs = [np.ascontiguousarray(a) for a in
                    (lv.rowptr, lv.col, lv.diag, lv.val, lv.dirichlet)]
            self._keep += arrs
            rp, cl, dg, vl, dr = arrs
            lev = _Level(lv.n, lv.B, _p64(rp), _p64(cl), _p64(dg), _pd(vl),
                         dr.shape[0], _p64(dr), lv.dircomp_mask)
            if lv.pf_mask:
                w = np.ascontiguousarray(lv.pf_weights, dtype=np.float64)
                self._keep.append(w)
                lev.pf_mask, lev.pf_w, lev.pf_domain = lv.pf_mask, _pd(w), lv.pf_domain
            if lv.patches is not None:
                pt = np.ascontiguousarray(lv.patches, dtype=np.int64)
                self._keep.append(pt)
                lev.npatch, lev.npp, lev.patches = pt.shape[0], pt.shape[1], _p64(pt)
            if lv.hn_edges is not None or lv.hn_faces is not None:
                he = np.ascontiguousarray(
                    lv.hn_edges if lv.hn_edges is not None else np.zeros((0, 4)),
                    dtype=np.int64).reshape(-1, 4)
                hf = np.ascontiguousarray(
                    lv.hn_faces if lv.hn_faces is not None else np.zeros((0, 10)),
                    dtype=np.int64).reshape(-1, 10)
                self._keep += [he, hf]
                lev.hn_disc = lv.hn_disc
                lev.nhedge, lev.hnedge = he.shape[0], _p64(he)
                lev.nhface, lev.hnface = hf.shape[0], _p64(hf)
            self.levels[l] = lev
        self.transfers = (_Transfer * max(nl - 1, 1))()
        for l, t in enumerate(prob.transfers):
            arrs = [np.ascontiguousarray(a, dtype=np.int64) for a in
                    (t.c2f, t.zweier, t.vierer, t.achter)]
            self._keep += arrs
            c2f, z, v, a = arrs
            rc = L.or_transfer_build(C.byref(self.transfers[l]), c2f.shape[0],
                                     _p64(c2f), z.shape[0], _p64(z), v.shape[0],
                                     _p64(v), a.shape[0], _p64(a))
            if rc != 0:
                raise MemoryError("or_transfer_build")
        if smoother is None:
            smoother = prob.info.get("smoother", "jacobi")
        self.smoother = smoother
        self.mg = L.or_mg_create(nl, self.levels, self.transfers, iterpre, iterpost,
                                 iterexact, omega, mgomega, mgtype.encode()[:1],
                                 {"vanka": 1, "ilu": 2}.get(smoother, 0))
        if not self.mg:
            raise ValueError("or_mg_create failed (Vanka needs patches on every level)")
        if ndirect and L.or_mg_set_direct(self.mg, int(ndirect)) != 0:
            raise ValueError("coarsest level too large (> 8192 dofs) or singular")

    def close(self):
        if getattr(self, "mg", None):
            L = lib()
            L.or_mg_free(self.mg)
            for l in range(self.prob.nlevels - 1):
                L.or_transfer_free(C.byref(self.transfers[l]))
            self.mg = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # single operations -----------------------------------------------------
    def vmult(self, level, y, x, s=1.0):
        y = np.array(y, dtype=np.float64)
        lib().or_bsr_vmult(C.byref(self.levels[level]), _pd(y),
                           _pd(np.ascontiguousarray(x, dtype=np.float64)), s)
        return y

    def vmult_transpose(self, level, y, x, s=1.0):
        y = np.array(y, dtype=np.float64)
        lib().or_bsr_vmult_transpose(C.byref(self.levels[level]), _pd(y),
                                     _pd(np.ascontiguousarray(x, dtype=np.float64)), s)
        return y

    def blockdiag_inverse(self, level):
        lv = self.prob.levels[level]
        out = np.zeros(lv.n * lv.B * lv.B)
        lib().or_blockdiag_inverse(C.byref(self.levels[level]), _pd(out))
        return out

    def smooth(self, level, niter, x, y):
        x = np.array(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        h = np.zeros_like(x)
        lib().or_smooth(self.mg, level, niter, _pd(x), _pd(y), _pd(h))
        return x

    def restrict_zero(self, level, fine):
        B = self.prob.levels[level].B
        out = np.zeros(self.prob.levels[level].n * B)
        lib().or_restrict_zero(C.byref(self.transfers[level]), B, _pd(out),
                               _pd(np.ascontiguousarray(fine, dtype=np.float64)))
        return out

    def prolongate_add(self, level, fine, coarse):
        B = self.prob.levels[level].B
        fine = np.array(fine, dtype=np.float64)
        lib().or_prolongate_add(C.byref(self.transfers[level]), B, _pd(fine),
                                _pd(np.ascontiguousarray(coarse, dtype=np.float64)))
        return fine

    def hn(self, op, level, u):
        """op: "average", "distribute" or "zero" (HNStructure*::Average ...)."""
        u = np.array(u, dtype=np.float64)
        getattr(lib(), "or_hn_" + op)(C.byref(self.levels[level]), _pd(u))
        return u

    def subtract_mean(self, level, u, algebraic=False):
        u = np.array(u, dtype=np.float64)
        f = lib().or_subtract_mean_algebraic if algebraic else lib().or_subtract_mean
        f(C.byref(self.levels[level]), _pd(u))
        return u

    def dirichlet_zero(self, level, u):
        u = np.array(u, dtype=np.float64)
        lib().or_dirichlet_zero(C.byref(self.levels[level]), _pd(u))
        return u

    def matrix_residual(self, level, x, b):
        y = np.zeros_like(np.asarray(b, dtype=np.float64))
        lib().or_matrix_residual(C.byref(self.levels[level]), _pd(y),
                                 _pd(np.ascontiguousarray(x, dtype=np.float64)),
                                 _pd(np.ascontiguousarray(b, dtype=np.float64)))
        return y

    def precondition(self, x, y):
        x = np.array(x, dtype=np.float64)
        lib().or_precondition(self.mg, _pd(x),
                              _pd(np.ascontiguousarray(y, dtype=np.float64)))
        return x

    def gmres(self, b=None, vmax=21, tol=1e-8, globaltol=1e-16, maxiter=100):
        b = np.ascontiguousarray(self.prob.rhs if b is None else b, dtype=np.float64)
        x = np.zeros_like(b)
        it, st = C.c_int(), C.c_int()
        f, r = C.c_double(), C.c_double()
        hist = np.zeros(vmax)
        reached = lib().or_gmres_solve(self.mg, _pd(b), _pd(x), vmax, tol, globaltol,
                                       maxiter, C.byref(it), C.byref(st), C.byref(f),
                                       C.byref(r), _pd(hist))
        status = {0: "waiting", 1: "running", 2: "converged", 3: "too many iterations",
                  4: "exploded", 5: "diverging"}[st.value]
        return x, {"reached": reached, "iterations": it.value, "status": status,
                   "firstresidual": f.value, "residual": r.value,
                   "history": hist[:max(it.value, 0)]}


def run_reference(out_dir=None, threads=None, harness=None, **kw):
    """Runs the compiled reference harness; returns (out_dir, summary dict).
    threads: OpenMP threads (1 makes Vanka's patch sums ordered); harness:
    REF_HARNESS_B200 runs the build that links the B200 binding (key
    backend=b200 or b200host selects B200MultiLevelSolver)."""
    exe = harness or REF_HARNESS
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    if out_dir is None:
        out_dir = tempfile.mkdtemp(prefix="gb_ref_")
    args = [exe, f"out={out_dir}"] + [f"{k}={v}" for k, v in kw.items()]
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    r = subprocess.run(args, capture_output=True, env=env)
    if r.returncode != 0:
        raise RuntimeError(f"{os.path.basename(exe)} failed ({r.returncode}): "
                           + r.stderr.decode(errors="replace")[-2000:])
    summ = {}
    with open(os.path.join(out_dir, "summary.txt")) as f:
        for line in f:
            k, *v = line.split()
            summ[k] = v
    return out_dir, summ


def write_inputs(d, kappa=None, rhs=None):
    """Writes kappa/rhs arrays for the harness; returns harness keyword args."""
    kw = {}
    if kappa is not None:
        p = os.path.join(d, "kappa_in.f64")
        np.ascontiguousarray(kappa, dtype=np.float64).tofile(p)
        kw["kappa"] = p
    if rhs is not None:
        p = os.path.join(d, "rhs_in.f64")
        np.ascontiguousarray(rhs, dtype=np.float64).tofile(p)
        kw["rhs"] = p
    return kw


# ------------------------------------------------------------------ adjoint

def transposed_problem(prob):
    """The dual system of ``StdSolver::AssembleDualMatrix``
    (Solver/stdsolver.cc:1815-1834) on every level: each level matrix
    transposed inside its own stencil, entry (i, j) taking the value of (j, i)
    as ``SparseBlockMatrix::transpose`` swaps them
    (LinAlg/sparseblockmatrix.xx:478-491), so row i keeps its column order.
    The uploaded matrices have Dirichlet rows and columns both set to identity,
    so their transposes are the reference's transpose-then-Dirichlet-rows
    matrices on every vector that is zero on the Dirichlet dofs. Transfers and
    the right-hand side are shared with ``prob``."""
    import copy
    out = copy.copy(prob)
    out.levels = []
    for L in prob.levels:
        assert L.B == 1
        n = L.n
        rowidx = np.repeat(np.arange(n), np.diff(L.rowptr))
        # position of (j, i) for every entry (i, j): sort the entries by key
        key = rowidx * n + L.col
        tkey = L.col * n + rowidx
        order = np.argsort(key)
        pos = np.searchsorted(key[order], tkey)
        if np.any(pos >= key.size) or np.any(key[order][np.minimum(pos, key.size - 1)] != tkey):
            raise ValueError("level matrix is not structurally symmetric")
        Lt = copy.copy(L)
        Lt.val = L.val[order[pos]].copy()
        out.levels.append(Lt)
    return out


def coeff_gradient(cells, u, lam, dirichlet):
    """dJ/dkappa_c = -scale_c * lam_c^T kloc u_c with u, lam zero on the
    Dirichlet nodes: the derivative of the per-cell element assembly
    (DofHandler/cgdisc.h:599-635 with a per-cell coefficient) restricted to the
    non-Dirichlet rows and columns of the strongly constrained matrix
    (LinAlg/sparseblockmatrix.xx:205-218), contracted with the dual and primal
    solutions. Plain numpy; the reference has no such gradient
    (Solver/stdsolver.cc:1080)."""
    u = np.array(u, dtype=np.float64)
    lam = np.array(lam, dtype=np.float64)
    u[dirichlet] = 0.0
    lam[dirichlet] = 0.0
    uc = u[cells.nodes]
    lc = lam[cells.nodes]
    g = -np.einsum("ci,ij,cj->c", lc, cells.kloc, uc)
    if cells.scale is not None:
        g = g * cells.scale
    return g
