"""ctypes binding of the C-ABI in include/gascoigne_b200.h.

The shared library is built in-tree (gascoignelib_b200/_lib/libgascoigne_b200.so,
see build.py). There is no fallback: if the library cannot be loaded, or no GPU
is visible, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libgascoigne_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "gascoigne_b200.h")

GB_OK, GB_EINVAL, GB_ENOMEM, GB_ECUDA, GB_ENOTCONV, GB_ESTATE, GB_ETIMEOUT = range(7)
GB_FP64, GB_FP32 = 0, 1
STATUS = {0: "waiting", 1: "running", 2: "converged", 3: "too many iterations",
          4: "exploded"}

_P64 = C.POINTER(C.c_int64)
_PD = C.POINTER(C.c_double)


class GbParams(C.Structure):
    _fields_ = [("iterpre", C.c_int), ("iterpost", C.c_int), ("iterexact", C.c_int),
                ("omega", C.c_double), ("mgomega", C.c_double), ("mgtype", C.c_char),
                ("gmressize", C.c_int), ("tol", C.c_double), ("globaltol", C.c_double),
                ("maxiter", C.c_int), ("smoother", C.c_int), ("ndirect", C.c_int)]


class GbSolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("status", C.c_int), ("restarts", C.c_int),
                ("firstresidual", C.c_double), ("residual", C.c_double),
                ("true_residual", C.c_double), ("rhs_norm", C.c_double),
                ("kernel_launches", C.c_int), ("device_ms", C.c_double)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["status_name"] = STATUS.get(self.status, str(self.status))
        d["true_rel_residual"] = (self.true_residual / self.rhs_norm
                                  if self.rhs_norm else 0.0)
        return d


class GBError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"gascoigne_b200 error {code}: {msg}")
        self.code = code


_lib = None

_SIGS = {
    "gb_ctx_create": [C.POINTER(C.c_void_p), C.c_int],
    "gb_ctx_destroy": [C.c_void_p],
    "gb_ctx_synchronize": [C.c_void_p],
    "gb_set_params": [C.c_void_p, C.POINTER(GbParams)],
    "gb_get_params": [C.c_void_p, C.POINTER(GbParams)],
    "gb_set_nlevels": [C.c_void_p, C.c_int],
    "gb_level_set_matrix": [C.c_void_p, C.c_int, C.c_int64, C.c_int, _P64, _P64, _P64, _PD],
    "gb_level_set_dirichlet": [C.c_void_p, C.c_int, C.c_int64, _P64, C.c_int],
    "gb_level_set_dirichlet_masks": [C.c_void_p, C.c_int, C.c_int64, _P64,
                                     C.POINTER(C.c_int)],
    "gb_level_set_transfer": [C.c_void_p, C.c_int, C.c_int64, _P64, C.c_int64, _P64,
                              C.c_int64, _P64, C.c_int64, _P64],
    "gb_level_size": [C.c_void_p, C.c_int, _P64, C.POINTER(C.c_int), _P64],
    "gb_vec_create": [C.c_void_p, C.POINTER(C.c_int)],
    "gb_vec_free": [C.c_void_p, C.c_int],
    "gb_vec_upload": [C.c_void_p, C.c_int, C.c_int, _PD, C.c_int64],
    "gb_vec_download": [C.c_void_p, C.c_int, C.c_int, _PD, C.c_int64],
    "gb_vec_zero": [C.c_void_p, C.c_int, C.c_int],
    "gb_vec_equ": [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int],
    "gb_vec_add": [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int],
    "gb_vec_norm": [C.c_void_p, C.c_int, C.c_int, _PD],
    "gb_vec_dot": [C.c_void_p, C.c_int, C.c_int, C.c_int, _PD],
    "gb_vmult": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double],
    "gb_vmulteq": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double],
    "gb_vmult_transpose": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double],
    "gb_matrix_residual": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int],
    "gb_residualgmres": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int],
    "gb_smooth_jacobi": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int],
    "gb_smooth_vanka": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int],
    "gb_smooth": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int],
    "gb_subtract_mean": [C.c_void_p, C.c_int, C.c_int],
    "gb_subtract_mean_algebraic": [C.c_void_p, C.c_int, C.c_int],
    "gb_level_set_patches": [C.c_void_p, C.c_int, C.c_int64, C.c_int, _P64],
    "gb_level_set_pfilter": [C.c_void_p, C.c_int, C.c_int, _PD, C.c_double, C.c_int64],
    "gb_level_set_hn": [C.c_void_p, C.c_int, C.c_int, C.c_int64, _P64, C.c_int64, _P64],
    "gb_hn_average": [C.c_void_p, C.c_int, C.c_int],
    "gb_hn_distribute": [C.c_void_p, C.c_int, C.c_int],
    "gb_hn_zero": [C.c_void_p, C.c_int, C.c_int],
    "gb_dirichlet_zero": [C.c_void_p, C.c_int, C.c_int],
    "gb_level_get_inverse_diagonal": [C.c_void_p, C.c_int, _PD, C.c_int64],
    "gb_restrict_zero": [C.c_void_p, C.c_int, C.c_int, C.c_int],
    "gb_prolongate_add": [C.c_void_p, C.c_int, C.c_int, C.c_int],
    "gb_precondition": [C.c_void_p, C.c_int, C.c_int, C.c_int],
    "gb_gmres": [C.c_void_p, C.c_int, C.c_int, C.POINTER(GbSolveInfo)],
    "gb_fgmres": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(GbSolveInfo)],
    "gb_solve_host": [C.c_void_p, C.c_int, _PD, _PD, C.c_int64, C.POINTER(GbSolveInfo)],
    "gb_set_operator": [C.c_void_p, C.c_int],
    "gb_get_operator": [C.c_void_p, C.POINTER(C.c_int)],
    "gb_adjoint_gmres": [C.c_void_p, C.c_int, C.c_int, C.POINTER(GbSolveInfo)],
    "gb_adjoint_fgmres": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(GbSolveInfo)],
    "gb_level_set_cells": [C.c_void_p, C.c_int, C.c_int64, C.c_int, _P64, _PD, _PD],
    "gb_coeff_gradient": [C.c_void_p, C.c_int, C.c_int, C.c_int, _PD, C.c_int64],
    "gb_level_set_functional": [C.c_void_p, C.c_int, _PD, _PD],
    "gb_functional": [C.c_void_p, C.c_int, C.c_int, C.c_int, _PD],
    "gb_level_set_mesh": [C.c_void_p, C.c_int, C.c_int, C.c_int64, _P64, _PD, _P64],
    "gb_level_set_mesh_degree": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int64, _P64, _PD,
                                 _P64],
    "gb_set_assembly_lps": [C.c_void_p, C.c_double, C.c_double],
    "gb_assemble": [C.c_void_p, C.c_int, C.c_void_p, C.c_int, _PD],
    "gb_assemble_levels": [C.c_void_p, C.c_void_p, C.c_int, _PD],
    "gb_level_get_kappa": [C.c_void_p, C.c_int, _PD],
    "gb_level_get_values": [C.c_void_p, C.c_int, _PD],
    "gb_form": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double],
    "gb_newton_residual": [C.c_void_p, C.c_int, C.c_int, C.c_int, _PD],
    "gb_vec_write_backup": [C.c_void_p, C.c_int, C.c_int, C.c_char_p, C.c_int],
    "gb_vec_read_backup": [C.c_void_p, C.c_int, C.c_int, C.c_char_p, C.c_int, C.c_int],
    "gb_vec_write_vtk": [C.c_void_p, C.c_int, C.c_int, C.c_char_p, C.c_int, C.c_int,
                         C.c_int64, C.c_int, _P64, _PD, C.c_double, C.c_char_p],
    "gb_ctx_get_stream": [C.c_void_p, C.POINTER(C.c_void_p)],
    "gb_set_timing": [C.c_void_p, C.c_int],
    "gb_get_kernel_count": [C.c_void_p, _P64],
    "gb_bench_spmv": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, _PD, _PD],
    "gb_bench_sweep": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, _PD, _PD],
    "gb_level_get_vanka_inverse": [C.c_void_p, C.c_int, _PD, C.c_int64],
    "gb_set_wait_limit": [C.c_void_p, C.c_uint64, C.c_int],
    "gb_debug_fail_alloc": [C.c_int64],
    "gb_kernel_arch": [C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "gb_dot_noalloc": [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p],
    "gb_get_kernel_times": [C.c_void_p, C.c_char_p, C.c_int64],
}


def lib():
    """Loads the in-tree CUDA library; raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with gascoignelib_b200.build.build()")
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.gb_last_error_string.argtypes = [C.c_void_p]
        L.gb_last_error_string.restype = C.c_char_p
        _lib = L
    return _lib


def _p64(a):
    return a.ctypes.data_as(_P64)


def _pd(a):
    return a.ctypes.data_as(_PD)


class Context:
    """One device context: levels, transfers, named vectors, solver keys."""

    def __init__(self, device: int = 0):
        self._L = lib()
        h = C.c_void_p()
        rc = self._L.gb_ctx_create(C.byref(h), device)
        if rc != GB_OK:
            raise GBError(rc, "gb_ctx_create failed (no usable CUDA device?)")
        self.h = h
        self.nlevels = 0
        self.sizes = []
        self.blocks = []

    # ------------------------------------------------------------ plumbing
    def _chk(self, rc):
        if rc != GB_OK:
            msg = self._L.gb_last_error_string(self.h)
            raise GBError(rc, msg.decode() if msg else "")
        return rc

    def close(self):
        if getattr(self, "h", None):
            self._L.gb_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------- set-up
    def set_params(self, iterpre=2, iterpost=2, iterexact=10, omega=0.8, mgomega=1.0,
                   mgtype="V", gmressize=21, tol=1e-8, globaltol=1e-16, maxiter=100,
                   smoother=None, ndirect=0):
        """smoother: "jacobi", "vanka" (or 0/1); default: the loaded problem's.
        ndirect: the coarsest level is solved exactly (FP64 inverse) when it has
        fewer nodes; 0 keeps the iterexact sweeps."""
        if smoother is None:
            smoother = getattr(self, "smoother", "jacobi")
        sm = {"jacobi": 0, "vanka": 1, "ilu": 2}.get(smoother, smoother)
        p = GbParams(iterpre, iterpost, iterexact, omega, mgomega, mgtype.encode()[:1],
                     gmressize, tol, globaltol, maxiter, int(sm), int(ndirect))
        self._chk(self._L.gb_set_params(self.h, C.byref(p)))

    def get_params(self):
        p = GbParams()
        self._chk(self._L.gb_get_params(self.h, C.byref(p)))
        return {k: getattr(p, k) for k, _ in p._fields_}

    def load_problem(self, prob):
        """Uploads every level's matrix, Dirichlet list, Vanka patches, pressure
        filter and transfer maps; the problem's smoother becomes the default of
        set_params."""
        self.smoother = prob.info.get("smoother", "jacobi")
        nl = prob.nlevels
        self._chk(self._L.gb_set_nlevels(self.h, nl))
        self.nlevels = nl
        self.sizes = []
        self.blocks = []
        for l, lv in enumerate(prob.levels):
            rp, cl, dg = (np.ascontiguousarray(a, dtype=np.int64)
                          for a in (lv.rowptr, lv.col, lv.diag))
            vl = np.ascontiguousarray(lv.val, dtype=np.float64)
            self._chk(self._L.gb_level_set_matrix(self.h, l, lv.n, lv.B, _p64(rp),
                                                  _p64(cl), _p64(dg), _pd(vl)))
            dr = np.ascontiguousarray(lv.dirichlet, dtype=np.int64)
            self._chk(self._L.gb_level_set_dirichlet(self.h, l, dr.shape[0], _p64(dr),
                                                     lv.dircomp_mask))
            if getattr(lv, "patches", None) is not None:
                pt = np.ascontiguousarray(lv.patches, dtype=np.int64)
                self._chk(self._L.gb_level_set_patches(self.h, l, pt.shape[0], pt.shape[1],
                                                       _p64(pt)))
            if getattr(lv, "hn_edges", None) is not None:
                he = np.ascontiguousarray(lv.hn_edges, dtype=np.int64).reshape(-1, 4)
                hf = np.ascontiguousarray(
                    lv.hn_faces if lv.hn_faces is not None else np.zeros((0, 10)),
                    dtype=np.int64).reshape(-1, 10)
                self._chk(self._L.gb_level_set_hn(self.h, l, lv.hn_disc, he.shape[0],
                                                  _p64(he), hf.shape[0], _p64(hf)))
            if getattr(lv, "pf_mask", 0):
                w = np.ascontiguousarray(lv.pf_weights, dtype=np.float64)
                self._chk(self._L.gb_level_set_pfilter(self.h, l, lv.pf_mask, _pd(w),
                                                       lv.pf_domain, 0))
            self.sizes.append(lv.n * lv.B)
            self.blocks.append(lv.B)
        for l, t in enumerate(prob.transfers):
            c2f, z, v, a = (np.ascontiguousarray(x, dtype=np.int64)
                            for x in (t.c2f, t.zweier, t.vierer, t.achter))
            self._chk(self._L.gb_level_set_transfer(
                self.h, l, c2f.shape[0], _p64(c2f), z.shape[0], _p64(z), v.shape[0],
                _p64(v), a.shape[0], _p64(a)))
        cells = getattr(prob, "cells", None)
        if cells is not None:
            self.set_cells(nl - 1, cells)

    def set_cells(self, level, cells):
        """Cells of `level` for gb_coeff_gradient (a problem.Cells)."""
        nd = np.ascontiguousarray(cells.nodes, dtype=np.int64)
        kl = np.ascontiguousarray(cells.kloc, dtype=np.float64)
        sc = (None if cells.scale is None
              else np.ascontiguousarray(cells.scale, dtype=np.float64))
        self._chk(self._L.gb_level_set_cells(
            self.h, level, nd.shape[0], nd.shape[1], _p64(nd), _pd(kl),
            _pd(sc) if sc is not None else None))
        self.ncells = nd.shape[0]
        if cells.mloc is not None:
            ml = np.ascontiguousarray(cells.mloc, dtype=np.float64)
            self._chk(self._L.gb_level_set_functional(self.h, level, _pd(ml), None))

    # ------------------------------------------------------- device assembly
    def set_mesh(self, level, dim, cells, coords, parent=None, degree=1):
        """Elements (int64 [ncells, nloc]: Q1 cells, local node a at corner
        bits (a&1, a>>1&1, a>>2&1); degree 2: Q2 patches of 3^dim nodes,
        x fastest), node coordinates [n, dim] and, above level 0, the parent
        element on level-1 of every element (gb_level_set_mesh_degree). On a
        level whose hanging nodes are set (load_problem does), the elements
        hold the hanging nodes themselves; the assembly condenses them. Call it
        after load_problem: setting the matrix or the hanging nodes again
        drops the mesh."""
        nd = np.ascontiguousarray(cells, dtype=np.int64)
        xy = np.ascontiguousarray(coords, dtype=np.float64)
        pa = None if parent is None else np.ascontiguousarray(parent, dtype=np.int64)
        self._chk(self._L.gb_level_set_mesh_degree(self.h, level, dim, degree, nd.shape[0],
                                                   _p64(nd), _pd(xy),
                                                   _p64(pa) if pa is not None else None))

    @staticmethod
    def _kappa_arg(kappa):
        """(pointer, where) for a numpy array (host) or a CUDA torch tensor."""
        if hasattr(kappa, "data_ptr"):
            if kappa.is_cuda:
                import torch
                assert kappa.dtype == torch.float64 and kappa.is_contiguous()
                # the library reads it on its own stream: finish torch's writes
                torch.cuda.current_stream(kappa.device).synchronize()
                return C.c_void_p(kappa.data_ptr()), 1, None
            kappa = kappa.numpy()
        k = np.ascontiguousarray(kappa, dtype=np.float64)
        return k.ctypes.data_as(C.c_void_p), 0, k

    def set_assembly_lps(self, sdelta0, xeta0=6.0):
        """gb_set_assembly_lps: LPS of the convection in later Q2 assemblies
        (sdelta0 = 0: off)."""
        self._chk(self._L.gb_set_assembly_lps(self.h, float(sdelta0), float(xeta0)))

    def assemble(self, level, kappa, beta=None):
        """gb_assemble: the level's matrix from per-cell kappa (numpy: host,
        CUDA tensor: device) and an optional convection vector."""
        p, where, keep = self._kappa_arg(kappa)
        b = None if beta is None else np.ascontiguousarray(beta, dtype=np.float64)
        self._chk(self._L.gb_assemble(self.h, level, p, where,
                                      _pd(b) if b is not None else None))
        del keep

    def assemble_levels(self, kappa, beta=None):
        """gb_assemble_levels: every level from the finest level's kappa."""
        p, where, keep = self._kappa_arg(kappa)
        b = None if beta is None else np.ascontiguousarray(beta, dtype=np.float64)
        self._chk(self._L.gb_assemble_levels(self.h, p, where,
                                             _pd(b) if b is not None else None))
        del keep

    def form(self, level, y, x, d=1.0):
        """gb_form: y += d * Form(x) on the level (its last assembled equation)."""
        self._chk(self._L.gb_form(self.h, level, y, x, d))

    def newton_residual(self, y, x, b):
        """gb_newton_residual on the finest level; returns max |y|."""
        nr = C.c_double()
        self._chk(self._L.gb_newton_residual(self.h, y, x, b, C.byref(nr)))
        return nr.value

    def write_backup(self, level, vid, path, binary=False):
        self._chk(self._L.gb_vec_write_backup(self.h, level, vid, path.encode(), int(binary)))

    def write_vtk(self, level, vid, name, step, dim, cells, coords, time=0.0, title=""):
        """gb_vec_write_vtk: <name>.<step %05d>.vtk with the mesh's cells
        (int64 [ncells, 2^dim], the mesh's vertex order) and node coordinates."""
        cl = np.ascontiguousarray(cells, dtype=np.int64)
        xy = np.ascontiguousarray(coords, dtype=np.float64)
        self._chk(self._L.gb_vec_write_vtk(self.h, level, vid, name.encode(), int(step), dim,
                                           cl.shape[0], cl.shape[1], _p64(cl), _pd(xy),
                                           float(time), title.encode()))

    def read_backup(self, level, vid, path, binary=False, add=False):
        self._chk(self._L.gb_vec_read_backup(self.h, level, vid, path.encode(), int(binary),
                                             int(add)))

    def level_values(self, level, nvals):
        v = np.zeros(nvals)
        self._chk(self._L.gb_level_get_values(self.h, level, _pd(v)))
        return v

    def level_kappa(self, level, ncells):
        k = np.zeros(ncells)
        self._chk(self._L.gb_level_get_kappa(self.h, level, _pd(k)))
        return k

    # ------------------------------------------------------------ vectors
    def vec(self):
        i = C.c_int()
        self._chk(self._L.gb_vec_create(self.h, C.byref(i)))
        return i.value

    def free(self, vid):
        self._chk(self._L.gb_vec_free(self.h, vid))

    def upload(self, level, vid, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        self._chk(self._L.gb_vec_upload(self.h, level, vid, _pd(a), a.shape[0]))

    def download(self, level, vid):
        out = np.empty(self.sizes[level])
        self._chk(self._L.gb_vec_download(self.h, level, vid, _pd(out), out.shape[0]))
        return out

    def zero(self, level, vid):
        self._chk(self._L.gb_vec_zero(self.h, level, vid))

    def equ(self, level, dst, s, src):
        self._chk(self._L.gb_vec_equ(self.h, level, dst, s, src))

    def add(self, level, dst, s, src):
        self._chk(self._L.gb_vec_add(self.h, level, dst, s, src))

    def norm(self, level, vid):
        out = C.c_double()
        self._chk(self._L.gb_vec_norm(self.h, level, vid, C.byref(out)))
        return out.value

    def dot(self, level, a, b):
        out = C.c_double()
        self._chk(self._L.gb_vec_dot(self.h, level, a, b, C.byref(out)))
        return out.value

    # ----------------------------------------------------------- operators
    def vmult(self, level, y, x, d=1.0):
        self._chk(self._L.gb_vmult(self.h, level, y, x, d))

    def vmulteq(self, level, y, x, d=1.0):
        self._chk(self._L.gb_vmulteq(self.h, level, y, x, d))

    def vmult_transpose(self, level, y, x, d=1.0):
        self._chk(self._L.gb_vmult_transpose(self.h, level, y, x, d))

    def matrix_residual(self, level, y, x, b):
        self._chk(self._L.gb_matrix_residual(self.h, level, y, x, b))

    def residualgmres(self, level, y, x, b):
        self._chk(self._L.gb_residualgmres(self.h, level, y, x, b))

    def smooth_jacobi(self, level, niter, x, y, h):
        self._chk(self._L.gb_smooth_jacobi(self.h, level, niter, x, y, h))

    def smooth_vanka(self, level, niter, x, y, h):
        self._chk(self._L.gb_smooth_vanka(self.h, level, niter, x, y, h))

    def smooth(self, level, niter, x, y, h):
        self._chk(self._L.gb_smooth(self.h, level, niter, x, y, h))

    def hn(self, op, level, vid):
        """op: "average", "distribute" or "zero"."""
        self._chk(getattr(self._L, "gb_hn_" + op)(self.h, level, vid))

    def subtract_mean(self, level, vid, algebraic=False):
        f = self._L.gb_subtract_mean_algebraic if algebraic else self._L.gb_subtract_mean
        self._chk(f(self.h, level, vid))

    def dirichlet_zero(self, level, vid):
        self._chk(self._L.gb_dirichlet_zero(self.h, level, vid))

    def inverse_diagonal(self, level):
        out = np.empty(self.sizes[level] * self.blocks[level])
        self._chk(self._L.gb_level_get_inverse_diagonal(self.h, level, _pd(out),
                                                        out.shape[0]))
        return out

    def restrict_zero(self, level, coarse, fine):
        self._chk(self._L.gb_restrict_zero(self.h, level, coarse, fine))

    def prolongate_add(self, level, fine, coarse):
        self._chk(self._L.gb_prolongate_add(self.h, level, fine, coarse))

    def precondition(self, x, y, precision=GB_FP64):
        self._chk(self._L.gb_precondition(self.h, x, y, precision))

    def gmres(self, x, b):
        info = GbSolveInfo()
        self._chk(self._L.gb_gmres(self.h, x, b, C.byref(info)))
        return info.as_dict()

    def fgmres(self, x, b, precision=GB_FP32, check=True):
        info = GbSolveInfo()
        rc = self._L.gb_fgmres(self.h, x, b, precision, C.byref(info))
        if check or rc not in (GB_OK, GB_ENOTCONV):
            self._chk(rc)
        return info.as_dict()

    # ------------------------------------------------------------ adjoint
    def set_operator(self, transposed):
        self._chk(self._L.gb_set_operator(self.h, int(transposed)))

    def get_operator(self):
        v = C.c_int()
        self._chk(self._L.gb_get_operator(self.h, C.byref(v)))
        return v.value

    def adjoint_gmres(self, x, b):
        info = GbSolveInfo()
        self._chk(self._L.gb_adjoint_gmres(self.h, x, b, C.byref(info)))
        return info.as_dict()

    def adjoint_fgmres(self, x, b, precision=GB_FP32, check=True):
        info = GbSolveInfo()
        rc = self._L.gb_adjoint_fgmres(self.h, x, b, precision, C.byref(info))
        if check or rc not in (GB_OK, GB_ENOTCONV):
            self._chk(rc)
        return info.as_dict()

    def coeff_gradient(self, level, u, lam, download=True):
        if not download:  # computed and kept on the device
            self._chk(self._L.gb_coeff_gradient(self.h, level, u, lam, None, self.ncells))
            return None
        g = np.empty(self.ncells, dtype=np.float64)
        self._chk(self._L.gb_coeff_gradient(self.h, level, u, lam, _pd(g), g.shape[0]))
        return g

    def functional(self, level, u, g, read=True):
        """J = u^T M u and g = 2 M u (0 on Dirichlet dofs) on the device."""
        J = C.c_double()
        self._chk(self._L.gb_functional(self.h, level, u, g, C.byref(J) if read else None))
        return J.value if read else None

    def stream(self):
        """The context's CUDA stream handle (cudaStream_t as an int)."""
        s = C.c_void_p()
        self._chk(self._L.gb_ctx_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def solve_host(self, b, method=2, out=None, check=True):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.empty_like(b) if out is None else out
        info = GbSolveInfo()
        rc = self._L.gb_solve_host(self.h, method, _pd(b), _pd(x), b.shape[0],
                                   C.byref(info))
        if check or rc not in (GB_OK, GB_ENOTCONV):
            self._chk(rc)
        return x, info.as_dict()

    def synchronize(self):
        self._chk(self._L.gb_ctx_synchronize(self.h))

    def kernel_count(self):
        v = C.c_int64()
        self._chk(self._L.gb_get_kernel_count(self.h, C.byref(v)))
        return v.value

    def set_timing(self, on=True):
        self._chk(self._L.gb_set_timing(self.h, int(on)))

    def kernel_times(self):
        """{kernel name: (launches, total ms)} since set_timing(True)."""
        import json
        buf = C.create_string_buffer(1 << 20)
        self._chk(self._L.gb_get_kernel_times(self.h, buf, len(buf)))
        return {k: tuple(v) for k, v in json.loads(buf.value.decode()).items()}

    def bench_spmv(self, level, precision=GB_FP64, reps=10, flush_l2=2):
        """flush_l2: 0 none, 1 write-flush, 2 read-flush (clean lines)."""
        ms, by = C.c_double(), C.c_double()
        self._chk(self._L.gb_bench_spmv(self.h, level, precision, reps, int(flush_l2),
                                        C.byref(ms), C.byref(by)))
        return ms.value, by.value

    def vanka_inverse(self, level, npatch, M):
        """The level's patch inverses [npatch, M, M] (row j = column j of the
        inverse), formed from its current values."""
        out = np.empty(int(npatch) * M * M)
        self._chk(self._L.gb_level_get_vanka_inverse(self.h, level, _pd(out), out.size))
        return out.reshape(int(npatch), M, M)

    def bench_sweep(self, level, precision=GB_FP32, reps=10, flush_l2=2):
        """One fused damped-Jacobi sweep of a scalar level, timed alone."""
        ms, by = C.c_double(), C.c_double()
        self._chk(self._L.gb_bench_sweep(self.h, level, precision, reps, int(flush_l2),
                                         C.byref(ms), C.byref(by)))
        return ms.value, by.value


def declared_symbols(header: str = HEADER):
    """Function names declared in the public header."""
    import re
    txt = open(header).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(gb_\w+)\s*\(", txt,
                                 flags=re.M)))
