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


def lps_projection(dim: int) -> np.ndarray:
    """ElementLpsIntegrator::Projection (DofHandler/elementlpsintegrator.h:
    66-110) as a matrix P (nloc x nloc, projected function i = sum_j P[i, j]
    phi_j): the middle and edge nodes keep their basis function; a corner's is
    replaced by -(1/2)^k times each node of its quarter of the patch whose k
    digits moved from the corner to the middle."""
    nloc = 3 ** dim
    P = np.eye(nloc)
    for c in range(nloc):
        dig = [(c // 3 ** d) % 3 for d in range(dim)]
        if 1 in dig:
            continue
        P[c, c] = 0.0
        for m in range(1, 1 << dim):
            j = sum((1 if (m >> d) & 1 else dig[d]) * 3 ** d for d in range(dim))
            P[c, j] = -(0.5 ** bin(m).count("1"))
    return P


def q1patch_shape(dim: int, xi: np.ndarray):
    """The Q1 functions of a patch of 2^dim cells (BaseQ12dPatch /
    BaseQ13dPatch, Discretization/Q2/baseq1patch.h: bilinear / trilinear on
    each cell, nodes 0, 1/2, 1 per direction, x fastest): values [3^dim] and
    reference gradients [3^dim, dim] at xi (not on a cell boundary)."""
    def hat(t):
        if t <= 0.5:
            return (1.0 - 2.0 * t, 2.0 * t, 0.0), (-2.0, 2.0, 0.0)
        return (0.0, 2.0 - 2.0 * t, 2.0 * t - 1.0), (0.0, -2.0, 2.0)
    nloc = 3 ** dim
    phi = np.ones(nloc)
    grad = np.ones((nloc, dim))
    hs = [hat(xi[d]) for d in range(dim)]
    for a in range(nloc):
        digits = [(a // 3 ** d) % 3 for d in range(dim)]
        for d in range(dim):
            f, df = hs[d][0][digits[d]], hs[d][1][digits[d]]
            phi[a] *= f
            for e in range(dim):
                grad[a, e] *= df if e == d else f
    return phi, grad


def gauss_points_q1patch(dim: int):
    """PatchFormula2d<4, QuadGauss4> / PatchFormula3d<8, HexGauss8>
    (Discretization/Q2/patchintegrationformula.xx:55-83): the 2-point rule in
    each cell of the patch, weights / 2^dim."""
    g = 0.5 / np.sqrt(3.0)
    p1 = np.array([0.5 * (0.5 - g), 0.5 * (0.5 + g), 0.5 + 0.5 * (0.5 - g),
                   0.5 + 0.5 * (0.5 + g)])
    grids = np.meshgrid(*([np.arange(4)] * dim), indexing="ij")
    idx = np.stack([gg.ravel() for gg in reversed(grids)], 1)
    return p1[idx], np.full(idx.shape[0], 0.25 ** dim)


def q1patch_element_matrices(dim: int, xcell: np.ndarray, kappa: np.ndarray,
                             beta=None, lps=None) -> np.ndarray:
    """q2_element_matrices for the Q1 functions of patches (CGQ1Patch /
    CGQ1Lps) with the patch formula."""
    return q2_element_matrices(dim, xcell, kappa, beta, lps, shape=q1patch_shape,
                               rule=gauss_points_q1patch)


def q2_element_matrices(dim: int, xcell: np.ndarray, kappa: np.ndarray,
                        beta=None, lps=None, shape=None, rule=None) -> np.ndarray:
    """As q1_element_matrices for Q2 elements (3^dim nodes, the isoparametric
    quadratic map) with the 3-point Gauss rule. lps = (sdelta0, xeta0) adds
    the local projection stabilisation of the convection (CGQ2Lps,
    ElementLpsIntegrator::Matrix, DofHandler/elementlpsintegrator.h:168-211):
    at each Gauss point h = |J|^(1/dim), delta = sdelta0 / (xeta0 kappa / h^2
    + (|beta| + 1e-6) / h) (LpsStabilization::ConvectionDiffusion,
    Problems/lpsstabilization.cc) and E += w |J| delta (beta . grad N_i)
    (beta . grad N_j) over the projected functions N."""
    pts, wts = (rule or gauss_points_q2)(dim)
    nc, nloc = xcell.shape[0], 3 ** dim
    E = np.zeros((nc, nloc, nloc))
    b = np.zeros(dim) if beta is None else np.asarray(beta, dtype=np.float64)[:dim]
    P = lps_projection(dim) if lps else None
    for q in range(pts.shape[0]):
        phi, gref = (shape or q2_shape)(dim, pts[q])
        J = np.einsum("cad,ae->cde", xcell, gref)
        det = np.linalg.det(J)
        Jinv = np.linalg.inv(J)
        g = np.einsum("ae,ced->cad", gref, Jinv)
        w = wts[q] * det
        E += (w * kappa)[:, None, None] * np.einsum("cad,cbd->cab", g, g)
        conv = np.einsum("cbd,d->cb", g, b)
        E += w[:, None, None] * phi[None, :, None] * conv[:, None, :]
        if P is not None:
            s0, xeta = lps
            h = np.abs(det) ** (1.0 / dim)
            nb = np.sqrt(np.sum(b * b)) + 1e-6
            delta = s0 / (xeta * kappa / (h * h) + nb / h)
            bn = np.einsum("ij,cj->ci", P, conv)          # beta . grad N_i
            E += (w * delta)[:, None, None] * bn[:, :, None] * bn[:, None, :]
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


# ------------------------------------------------------------------ hanging nodes

# Q2 interpolation weights of the node at 1/4 of a coarse edge (hnstructureq22d.cc,
# hnstructureq23d.cc:35-45: wei = 0.375, 0.75, -0.125; faces: wei[i] * wei[j])
_Q2W = (0.375, 0.75, -0.125)


def refined_elements(coord: np.ndarray, dim: int, degree: int, N: int):
    """Elements of a uniform mesh of N cells per direction in which some cells
    (Q1) or patches of 2^dim cells (Q2) were refined once, found from the node
    coordinates (every node on the 2N grid). Returns (elements [ne, nloc] in
    the node numbering of coord, parents [ne]: the element of the uniform
    coarser mesh - the N-cell mesh for Q1, the N/2-patch mesh for Q2 - each one
    lies in). Coarse elements are taken lexicographically (x fastest); a refined
    one is replaced by its 2^dim children in corner-bit order. Local node order:
    corner bits for Q1 (as q1_shape), lexicographic 3^dim for Q2 (as q2_shape)."""
    M = 2 * N
    c = np.rint(coord * M).astype(np.int64)
    lex = np.zeros(c.shape[0], dtype=np.int64)
    for d in reversed(range(dim)):
        lex = lex * (M + 1) + c[:, d]
    look = np.full((M + 1) ** dim, -1, dtype=np.int64)
    look[lex] = np.arange(c.shape[0])

    def node(p):
        k = 0
        for d in reversed(range(dim)):
            k = k * (M + 1) + int(p[d])
        return int(look[k])

    if degree == 1:
        span, nc = 2, N                      # coarse cell: 2 fine units
        offs = [[(a >> d) & 1 for d in range(dim)] for a in range(1 << dim)]
    else:
        span, nc = 4, N // 2                 # coarse patch: 4 fine units
        offs = [[(a // 3 ** d) % 3 for d in range(dim)] for a in range(3 ** dim)]
    els, par = [], []
    for k in range(nc ** dim):
        base = [((k // nc ** d) % nc) * span for d in range(dim)]
        if node([b + 1 for b in base]) >= 0:  # refined: its first inner fine node exists
            sub = span // 2
            for ch in range(1 << dim):
                b2 = [base[d] + sub * ((ch >> d) & 1) for d in range(dim)]
                step = sub // (1 if degree == 1 else 2)
                els.append([node([b2[d] + step * o[d] for d in range(dim)]) for o in offs])
                par.append(k)
        else:
            step = span // (1 if degree == 1 else 2)
            els.append([node([base[d] + step * o[d] for d in range(dim)]) for o in offs])
            par.append(k)
    el = np.array(els, dtype=np.int64)
    assert (el >= 0).all(), "node missing from the refined mesh"
    return el, np.array(par, dtype=np.int64)


def hn_maps(level, dim: int):
    """The level's hanging nodes as two dicts (edges, faces): node -> list of
    (parent, weight) in the reference's parent order (HNStructureQ12d/Q13d:
    2 edge parents 0.5, 4 face parents {0, 1, 3, 4} of the 9 with 0.25;
    HNStructureQ22d/Q23d: 3 edge parents 0.375, 0.75, -0.125, 9 face parents
    with the tensor products)."""
    q2 = level.hn_disc >= 2
    edges, faces = {}, {}
    for row in np.asarray(level.hn_edges).reshape(-1, 4):
        if q2:
            edges[int(row[0])] = [(int(row[1 + j]), _Q2W[j]) for j in range(3)]
        else:
            edges[int(row[0])] = [(int(row[1 + j]), 0.5) for j in range(2)]
    if level.hn_faces is not None:
        for row in np.asarray(level.hn_faces).reshape(-1, 10):
            if q2:
                faces[int(row[0])] = [(int(row[1 + s]), _Q2W[s // 3] * _Q2W[s % 3])
                                      for s in range(9)]
            else:
                faces[int(row[0])] = [(int(row[1 + s]), 0.25) for s in (0, 1, 3, 4)]
    return edges, faces


def condense(E: np.ndarray, cells: np.ndarray, hn):
    """Element condensation of hanging nodes (CGDisc::LocalToGlobal,
    DofHandler/cgdisc.h:354-364, with HNStructureQ12d::CondenseHanging,
    Discretization/Q1/hnstructureq12d.cc:129-158, HNStructureQ13d,
    Discretization/Q1/hnstructureq13d.cc:275-331 and 401-438,
    HNStructureQ22d, Discretization/Q2/hnstructureq22d.cc:84-110, and
    HNStructureQ23d, Discretization/Q2/hnstructureq23d.cc:161-378): edge
    hanging nodes first, then face hanging nodes, each phase over the local
    slots in ascending order. A hanging node h in slot s with parents p_j,
    weights w_j: every parent already in the element (slot t_j) takes
    column t_j += w_j column s and row t_j += w_j row s; the one parent that is
    missing takes slot s, whose column and row are scaled by its weight
    (C^T E C for u_h = sum w_j u_pj). Returns (E', indices')."""
    E = np.array(E, dtype=np.float64, copy=True)
    idx = np.array(cells, dtype=np.int64, copy=True)
    for c in range(idx.shape[0]):
        for phase in hn:
            for s in range(idx.shape[1]):
                h = int(idx[c, s])
                if h not in phase:
                    continue
                where = {int(v): t for t, v in enumerate(idx[c])}
                miss = [(p, w) for p, w in phase[h] if p not in where]
                assert len(miss) == 1, "a hanging node needs exactly one missing parent"
                for p, w in phase[h]:
                    if p in where:
                        t = where[p]
                        E[c, :, t] += w * E[c, :, s]
                        E[c, t, :] += w * E[c, s, :]
                E[c, :, s] *= miss[0][1]
                E[c, s, :] *= miss[0][1]
                idx[c, s] = miss[0][0]
    return E, idx


def assemble_hn(n, rowptr, col, cells, E, dirichlet, hanging) -> np.ndarray:
    """assemble() of condensed elements (cells: condensed indices), then the
    hanging rows' diagonal set to 1 (HNStructure::MatrixDiag, called by
    CGDisc::Matrix, DofHandler/cgdisc.h:634) before the Dirichlet rows."""
    val = assemble(n, rowptr, col, cells, E, dirichlet)
    ri = np.repeat(np.arange(n), np.diff(rowptr))
    hm = np.zeros(n, dtype=bool)
    hm[np.asarray(hanging, dtype=np.int64)] = True
    val[hm[ri] & (ri == col)] = 1.0
    return val
