"""CPU restatement (numpy) of the reference's Q1 and Q2 matrix assembly, for the
device assembly's tests. Test infrastructure: nothing in the library imports it.

What it restates:
- CGDisc::Matrix (DofHandler/cgdisc.h:599-635): a loop over the cells in
  ascending order; per cell the element matrix of the equation, added into the
  global matrix (LocalToGlobal, :353-366; no hanging nodes here).
- ElementIntegrator::Matrix (DofHandler/elementintegrator.xx:350-395) with the
  matrix formula of ElementIntegratorQ12d / Q13d (QuadGauss4 / HexGauss8,
  DofHandler/elementintegrator.h:214-222): Gauss-Legendre points, weight =
  w_k * det J, and at every point E(test a, trial b) += the equation's entry.
- The harness equation -div(kappa grad u) + beta . grad u
  (oracle/ref/ref_harness.cc, DiffusionEquation::Matrix): kappa grad phi_b .
  grad phi_a + (beta . grad phi_b) phi_a, kappa the cell's value.
- The harness's kappa on coarser levels: the mean of the 2^dim children
  (oracle/ref/ref_harness.cc, build_kappa).
- StdSolver's strong Dirichlet condition on the matrix
  (SparseBlockMatrix::dirichlet, LinAlg/sparseblockmatrix.xx:207-218): the
  Dirichlet row and column are zeroed and the diagonal set to 1.

The element matrices are formed with the multilinear map of each cell and its
Jacobian at the Gauss points, so they match the reference up to rounding (the
tests use 1e-13 relative to the largest entry), not bit for bit.
"""
from __future__ import annotations

import numpy as np

_G = 0.5 / np.sqrt(3.0)


def gauss_points(dim: int):
    """2-point Gauss-Legendre rule per direction on the unit cell [0, 1]^dim:
    points [2^dim, dim] (x fastest) and weights [2^dim]."""
    p1 = np.array([0.5 - _G, 0.5 + _G])
    if dim == 2:
        y, x = np.meshgrid(p1, p1, indexing="ij")
        pts = np.stack([x.ravel(), y.ravel()], 1)
    else:
        z, y, x = np.meshgrid(p1, p1, p1, indexing="ij")
        pts = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    return pts, np.full(pts.shape[0], 0.5 ** dim)


def q1_shape(dim: int, xi: np.ndarray):
    """Q1 basis values [nloc] and reference gradients [nloc, dim] at xi;
    local node a has corner bits (a & 1, a >> 1 & 1, a >> 2 & 1)."""
    nloc = 1 << dim
    phi = np.ones(nloc)
    grad = np.ones((nloc, dim))
    for a in range(nloc):
        for d in range(dim):
            bit = (a >> d) & 1
            f = xi[d] if bit else 1.0 - xi[d]
            df = 1.0 if bit else -1.0
            phi[a] *= f
            for e in range(dim):
                grad[a, e] *= df if e == d else f
    return phi, grad


def q1_element_matrices(dim: int, xcell: np.ndarray, kappa: np.ndarray,
                        beta=None) -> np.ndarray:
    """E[c, a, b] = sum over Gauss points of w |J| (kappa_c grad phi_b . grad
    phi_a + (beta . grad phi_b) phi_a) for cells with corner coordinates
    xcell[c, a, :] (local order as q1_shape)."""
    pts, wts = gauss_points(dim)
    nc, nloc = xcell.shape[0], 1 << dim
    E = np.zeros((nc, nloc, nloc))
    b = np.zeros(dim) if beta is None else np.asarray(beta, dtype=np.float64)[:dim]
    for q in range(pts.shape[0]):
        phi, gref = q1_shape(dim, pts[q])
        J = np.einsum("cad,ae->cde", xcell, gref)          # dx_d / dxi_e
        det = np.linalg.det(J)
        Jinv = np.linalg.inv(J)                             # dxi / dx
        g = np.einsum("ae,ced->cad", gref, Jinv)            # d phi_a / dx_d
        w = wts[q] * det
        E += (w * kappa)[:, None, None] * np.einsum("cad,cbd->cab", g, g)
        conv = np.einsum("cbd,d->cb", g, b)                 # beta . grad phi_b
        E += w[:, None, None] * phi[None, :, None] * conv[:, None, :]
    return E


def uniform_cells(coord: np.ndarray, dim: int) -> np.ndarray:
    """Cells of a uniform mesh of the unit square/cube in a given node
    numbering (found through the node coordinates): [N^dim, 2^dim], cells
    lexicographic (x fastest), local nodes as q1_shape."""
    n = coord.shape[0]
    N = int(round(n ** (1.0 / dim))) - 1
    c = np.rint(coord * N).astype(np.int64)
    lex = np.zeros(n, dtype=np.int64)
    for d in reversed(range(dim)):
        lex = lex * (N + 1) + c[:, d]
    inv = np.empty_like(lex)
    inv[lex] = np.arange(n)
    n1 = N + 1
    if dim == 3:
        k, j, i = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
        base = ((k * n1 + j) * n1 + i).ravel()
        offs = np.array([((a >> 2) * n1 + ((a >> 1) & 1)) * n1 + (a & 1) for a in range(8)])
    else:
        j, i = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
        base = (j * n1 + i).ravel()
        offs = np.array([((a >> 1) & 1) * n1 + (a & 1) for a in range(4)])
    return inv[base[:, None] + offs[None, :]]


def uniform_parents(dim: int, N: int) -> np.ndarray:
    """Parent cell (on the N/2 mesh) of every cell of the uniform N mesh,
    both lexicographic."""
    i = np.arange(N)
    if dim == 3:
        k, j, ii = np.meshgrid(i, i, i, indexing="ij")
        return (((k // 2) * (N // 2) + j // 2) * (N // 2) + ii // 2).ravel()
    j, ii = np.meshgrid(i, i, indexing="ij")
    return ((j // 2) * (N // 2) + ii // 2).ravel()


def coarsen_kappa(kappa: np.ndarray, parent: np.ndarray, ncoarse: int) -> np.ndarray:
    """kappa of each coarse cell = (sum of its children in ascending order) /
    their count, the harness's build_kappa."""
    order = np.argsort(parent, kind="stable")
    s = np.zeros(ncoarse)
    cnt = np.zeros(ncoarse)
    for f in order:
        s[parent[f]] += kappa[f]
        cnt[parent[f]] += 1
    return s / cnt


def assemble(n: int, rowptr, col, cells, E, dirichlet) -> np.ndarray:
    """Values in the given CSR pattern: element matrices added cell by cell in
    ascending order, then the strong Dirichlet rows and columns."""
    val = np.zeros(col.shape[0])
    pos = {}
    for r in range(n):
        for k in range(rowptr[r], rowptr[r + 1]):
            pos[(r, int(col[k]))] = k
    for c in range(cells.shape[0]):
        nd = cells[c]
        for a in range(nd.size):
            for b in range(nd.size):
                val[pos[(int(nd[a]), int(nd[b]))]] += E[c, a, b]
    dm = np.zeros(n, dtype=bool)
    dm[dirichlet] = True
    ri = np.repeat(np.arange(n), np.diff(rowptr))
    val[dm[ri] | dm[col]] = 0.0
    val[(ri == col) & dm[ri]] = 1.0
    return val


# ------------------------------------------------------------------ Q2

# LineGauss3 as the reference states it (Discretization/Q1/integrationformula1d.cc
# :82-92): points to 20 digits, weights rounded to 12 (so 5/18, 8/18 are off by
# about 2e-13 relative; the tensor rules QuadGauss9 / HexGauss27 inherit it)
_P3 = (0.11270166537925831148, 0.5, 0.88729833462074168852)
_W3 = (0.277777777778, 0.444444444444, 0.277777777778)


def gauss_points_q2(dim: int):
    """The reference's 3-point Gauss rule per direction on [0, 1]^dim
    (QuadGauss9 / HexGauss27): points [3^dim, dim] (x fastest), weights."""
    p1 = np.array(_P3)
    w1 = np.array(_W3)
    grids = np.meshgrid(*([np.arange(3)] * dim), indexing="ij")
    idx = np.stack([g.ravel() for g in reversed(grids)], 1)     # x fastest
    return p1[idx], np.prod(w1[idx], axis=1)


def q2_shape(dim: int, xi: np.ndarray):
    """Q2 (tensor quadratic Lagrange, nodes 0, 1/2, 1) values [3^dim] and
    reference gradients [3^dim, dim]; local node a = sum_d a_d 3^d."""
    def L(k, t):
        return (2 * (t - 0.5) * (t - 1.0), -4.0 * t * (t - 1.0), 2.0 * t * (t - 0.5))[k]

    def dL(k, t):
        return (4.0 * t - 3.0, -8.0 * t + 4.0, 4.0 * t - 1.0)[k]

    nloc = 3 ** dim
    phi = np.ones(nloc)
    grad = np.ones((nloc, dim))
    for a in range(nloc):
        digits = [(a // 3 ** d) % 3 for d in range(dim)]
        for d in range(dim):
            f, df = L(digits[d], xi[d]), dL(digits[d], xi[d])
            phi[a] *= f
            for e in range(dim):
                grad[a, e] *= df if e == d else f
    return phi, grad


def q2_element_matrices(dim: int, xcell: np.ndarray, kappa: np.ndarray,
                        beta=None) -> np.ndarray:
    """As q1_element_matrices for Q2 elements (3^dim nodes, the isoparametric
    quadratic map) with the 3-point Gauss rule."""
    pts, wts = gauss_points_q2(dim)
    nc, nloc = xcell.shape[0], 3 ** dim
    E = np.zeros((nc, nloc, nloc))
    b = np.zeros(dim) if beta is None else np.asarray(beta, dtype=np.float64)[:dim]
    for q in range(pts.shape[0]):
        phi, gref = q2_shape(dim, pts[q])
        J = np.einsum("cad,ae->cde", xcell, gref)
        det = np.linalg.det(J)
        Jinv = np.linalg.inv(J)
        g = np.einsum("ae,ced->cad", gref, Jinv)
        w = wts[q] * det
        E += (w * kappa)[:, None, None] * np.einsum("cad,cbd->cab", g, g)
        conv = np.einsum("cbd,d->cb", g, b)
        E += w[:, None, None] * phi[None, :, None] * conv[:, None, :]
    return E


def uniform_patches(coord: np.ndarray, dim: int) -> np.ndarray:
    """Q2 elements (patches of 2^dim cells, 3^dim nodes, local order
    lexicographic) of a uniform mesh in a given node numbering."""
    n = coord.shape[0]
    N = int(round(n ** (1.0 / dim))) - 1
    c = np.rint(coord * N).astype(np.int64)
    lex = np.zeros(n, dtype=np.int64)
    for d in reversed(range(dim)):
        lex = lex * (N + 1) + c[:, d]
    inv = np.empty_like(lex)
    inv[lex] = np.arange(n)
    n1, P = N + 1, N // 2
    if dim == 3:
        k, j, i = np.meshgrid(np.arange(P), np.arange(P), np.arange(P), indexing="ij")
        base = ((2 * k * n1 + 2 * j) * n1 + 2 * i).ravel()
        loc = np.array([(a * n1 + b) * n1 + e for a in range(3) for b in range(3)
                        for e in range(3)])
    else:
        j, i = np.meshgrid(np.arange(P), np.arange(P), indexing="ij")
        base = (2 * j * n1 + 2 * i).ravel()
        loc = np.array([b * n1 + e for b in range(3) for e in range(3)])
    return inv[base[:, None] + loc[None, :]]
