"""Assembled multilevel systems: the data that crosses the drop-in boundary.

A ``Problem`` holds exactly what the reference hands its GPU backend for the
linear-solve path (Gascoigne ``cuda/cudasolver.cc:115-128, 161-298``,
``cuda/cudamgintepolatornested.cc:21-25``):

* per level (0 = coarsest, the reference's solver indexing,
  ``Solver/stdmultilevelsolver.cc:224-231``) the block-CSR matrix of
  ``SparseBlockMatrix<FMatrixBlock<B>>`` with its ``ColumnDiagStencil``
  (``LinAlg/columnstencil.h:57-60``, ``LinAlg/columndiagstencil.h:54-57``),
  blocks row-major (``LinAlg/nodematrix.h:44-48``);
* per level the strong-Dirichlet node list (``DofHandler/cgdisc.h:1162-1179``);
* per level pair the mesh-transfer maps ``c2f``/``zweier``/``vierer``/``achter``
  (``Mesh/gascoignemeshtransfer.h:48-51``);
* the finest-level right-hand side.

Two producers exist: ``load_reference_dump`` reads what the reference's own
solver assembled (written by the oracle harness), and ``structured_problem``
assembles the same operator on a lexicographically numbered uniform Q1 mesh
(the synthetic workload generator used where the reference is not present).
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np


@dataclass
class Level:
    n: int                      # block rows (nodes)
    B: int                      # block size (components per node)
    rowptr: np.ndarray          # int64 [n+1]
    col: np.ndarray             # int64 [nnzb]
    diag: np.ndarray            # int64 [n]   position of the diagonal block
    val: np.ndarray             # float64 [nnzb*B*B]
    dirichlet: np.ndarray       # int64 [ndir] Dirichlet nodes
    dircomp_mask: int = 1       # bit c: component c is Dirichlet
    coord: Optional[np.ndarray] = None  # float64 [n, dim]
    # pressure filter (PressureFilter): filtered components, per-node weights
    # (integrals of the basis functions) and the domain size; mask 0: inactive
    pf_mask: int = 0
    pf_weights: Optional[np.ndarray] = None
    pf_domain: float = 0.0
    # Vanka patches: [npatch, nodes per patch] node indices (DofHandler::
    # GetElement(2, p)); None when the level has none
    patches: Optional[np.ndarray] = None
    # hanging nodes: rows [node, 3 parents] (edges, hnq2) and [node, 9 parents]
    # (3D faces, hnq2face), and the discretisation of the HNStructure acting
    # on them: 0 Q12d, 1 Q13d, 2 Q22d, 3 Q23d
    hn_edges: Optional[np.ndarray] = None
    hn_faces: Optional[np.ndarray] = None
    hn_disc: int = 0

    @property
    def nnzb(self) -> int:
        return int(self.col.shape[0])

    @property
    def ndof(self) -> int:
        return self.n * self.B


@dataclass
class Transfer:
    """Transfer between level l (coarse) and l+1 (fine)."""
    c2f: np.ndarray             # int64 [ncoarse]
    zweier: np.ndarray          # int64 [nz, 3]  fine, 2 coarse parents
    vierer: np.ndarray          # int64 [nv, 5]
    achter: np.ndarray          # int64 [na, 9]

    @property
    def ncoarse(self) -> int:
        return int(self.c2f.shape[0])


@dataclass
class Cells:
    """Finest-level cells for the coefficient gradient: the per-cell element
    matrix of the equation is kappa_c * scale_c * kloc (the reference's
    element assembly with a per-cell coefficient, DofHandler/cgdisc.h:599-635,
    Interface/equation.h:104), so dA/dkappa_c = scale_c * kloc on the cell's
    nodes."""
    nodes: np.ndarray                   # int64 [ncells, nloc] local node order
    kloc: np.ndarray                    # float64 [nloc, nloc] unit-coefficient matrix
    mloc: Optional[np.ndarray] = None   # float64 [nloc, nloc] element mass matrix
    scale: Optional[np.ndarray] = None  # float64 [ncells], default 1

    @property
    def ncells(self) -> int:
        return int(self.nodes.shape[0])

    @property
    def nloc(self) -> int:
        return int(self.nodes.shape[1])

    def assemble(self, local: np.ndarray, n: int):
        """Sum of local[.,.] over the cells as a scipy CSR matrix of size n."""
        import scipy.sparse as sp
        nl = self.nloc
        w = np.ones(self.ncells) if self.scale is None else self.scale
        rows = np.repeat(self.nodes, nl, axis=1).ravel()
        cols = np.tile(self.nodes, (1, nl)).ravel()
        vals = (w[:, None] * local.ravel()[None, :]).ravel()
        return sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsr()


@dataclass
class Problem:
    dim: int
    levels: List[Level]
    transfers: List[Transfer]
    rhs: np.ndarray
    info: dict = field(default_factory=dict)
    cells: Optional[Cells] = None

    @property
    def nlevels(self) -> int:
        return len(self.levels)

    @property
    def finest(self) -> Level:
        return self.levels[-1]


def _i64(path):
    return np.fromfile(path, dtype=np.int64)


def load_reference_dump(d: str) -> Problem:
    """Reads the arrays the oracle harness wrote for the reference's solver."""
    summ = {}
    with open(os.path.join(d, "summary.txt")) as f:
        for line in f:
            k, *v = line.split()
            summ[k] = v
    nl = int(summ["nlevels"][0])
    levels, transfers = [], []
    dim = None
    B = int(summ.get("ncomp", ["1"])[0])
    dmask = sum(1 << int(c) for c in summ.get("dircomps", ["0"]))
    for l in range(nl):
        p = os.path.join(d, f"L{l}_")
        rowptr = _i64(p + "rowptr.i64")
        n = rowptr.shape[0] - 1
        coord = np.fromfile(p + "coord.f64")
        dim = coord.shape[0] // n
        lv = Level(n=n, B=B, rowptr=rowptr, col=_i64(p + "col.i64"),
                   diag=_i64(p + "diag.i64"), val=np.fromfile(p + "val.f64"),
                   dirichlet=_i64(p + "dirichlet.i64"), dircomp_mask=dmask,
                   coord=coord.reshape(n, dim))
        if os.path.exists(p + "pfw.f64") and f"pfdomain_L{l}" in summ:
            lv.pf_mask = 1
            lv.pf_weights = np.fromfile(p + "pfw.f64")
            lv.pf_domain = float(summ[f"pfdomain_L{l}"][0])
        if os.path.exists(p + "patches.i64"):
            pt = _i64(p + "patches.i64")
            npp = 3 ** dim
            lv.patches = pt.reshape(-1, npp)
        he = _i64(p + "hnedge.i64") if os.path.exists(p + "hnedge.i64") else None
        hf = _i64(p + "hnface.i64") if os.path.exists(p + "hnface.i64") else None
        if (he is not None and he.size) or (hf is not None and hf.size):
            lv.hn_edges = (he if he is not None else np.zeros(0, np.int64)).reshape(-1, 4)
            lv.hn_faces = (hf if hf is not None else np.zeros(0, np.int64)).reshape(-1, 10)
            q2 = summ.get("disc", ["Q1"])[0] == "Q2"
            lv.hn_disc = (2 if q2 else 0) + (1 if dim == 3 else 0)
        levels.append(lv)
    for l in range(nl - 1):
        p = os.path.join(d, f"T{l}_")
        transfers.append(Transfer(c2f=_i64(p + "c2f.i64"),
                                  zweier=_i64(p + "zweier.i64").reshape(-1, 3),
                                  vierer=_i64(p + "vierer.i64").reshape(-1, 5),
                                  achter=_i64(p + "achter.i64").reshape(-1, 9)))
    info = {k: v for k, v in summ.items()}
    return Problem(dim=dim, levels=levels, transfers=transfers,
                   rhs=np.fromfile(os.path.join(d, "rhs.f64")), info=info)


# ---------------------------------------------------------------- generator

def _q1_local_stiffness(dim: int, h: float) -> np.ndarray:
    """Q1 element stiffness of a cube of width h, unit coefficient, local node
    order lexicographic (x fastest): tensor products of the 1D mass
    [[1/3,1/6],[1/6,1/3]]*h and stiffness [[1,-1],[-1,1]]/h."""
    m = np.array([[1.0 / 3.0, 1.0 / 6.0], [1.0 / 6.0, 1.0 / 3.0]]) * h
    s = np.array([[1.0, -1.0], [-1.0, 1.0]]) / h
    if dim == 2:
        # local index = ey*2 + ex  -> kron(y, x)
        return np.kron(m, s) + np.kron(s, m)
    return (np.kron(np.kron(m, m), s) + np.kron(np.kron(m, s), m)
            + np.kron(np.kron(s, m), m))


def _q1_local_mass(dim: int, h: float) -> np.ndarray:
    """Q1 element mass matrix of a cube of width h (local order as above)."""
    m = np.array([[1.0 / 3.0, 1.0 / 6.0], [1.0 / 6.0, 1.0 / 3.0]]) * h
    return np.kron(m, m) if dim == 2 else np.kron(np.kron(m, m), m)


def _q1_local_convection(dim: int, h: float, beta) -> np.ndarray:
    """Q1 element matrix of (beta . grad u) v: entry [i, j] = integral of
    (beta . grad phi_j) phi_i, from the 1D mass m and d[i, j] = integral of
    phi_j' phi_i = [[-1/2, 1/2], [-1/2, 1/2]]."""
    m = np.array([[1.0 / 3.0, 1.0 / 6.0], [1.0 / 6.0, 1.0 / 3.0]]) * h
    d = np.array([[-0.5, 0.5], [-0.5, 0.5]])
    if dim == 2:
        return beta[0] * np.kron(m, d) + beta[1] * np.kron(d, m)
    return (beta[0] * np.kron(np.kron(m, m), d) + beta[1] * np.kron(np.kron(m, d), m)
            + beta[2] * np.kron(np.kron(d, m), m))


def cell_nodes(dim: int, N: int) -> np.ndarray:
    """Node indices of the N^dim cells (lexicographic cells and nodes, x
    fastest), local node order lexicographic: int64 [N^dim, 2^dim]."""
    n1 = N + 1
    if dim == 3:
        k, j, i = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
        base = ((k * n1 + j) * n1 + i).ravel()
        offs = np.array([(a * n1 + b) * n1 + e for a in range(2) for b in range(2)
                         for e in range(2)])
    else:
        j, i = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
        base = (j * n1 + i).ravel()
        offs = np.array([b * n1 + e for b in range(2) for e in range(2)])
    return (base[:, None] + offs[None, :]).astype(np.int64)


def kappa_pyramid(dim: int, fine: np.ndarray, levels: int) -> List[np.ndarray]:
    """Per-level cell coefficients, finest last; a coarse cell takes the mean of
    its 2^dim children summed in lexicographic child order (z, y, x)."""
    out = [fine]
    cur = fine
    for _ in range(levels - 1):
        if dim == 3:
            s = np.zeros(tuple(d // 2 for d in cur.shape))
            for a in range(2):
                for b in range(2):
                    for e in range(2):
                        s = s + cur[a::2, b::2, e::2]
            cur = s / 8.0
        else:
            s = np.zeros(tuple(d // 2 for d in cur.shape))
            for b in range(2):
                for e in range(2):
                    s = s + cur[b::2, e::2]
            cur = s / 4.0
        out.append(cur)
    return out[::-1]


def _assemble_level(dim: int, N: int, kappa: np.ndarray, beta=None) -> Level:
    """Assembles -div(kappa grad u) [+ beta . grad u] with Q1 on N^dim uniform cells of the unit
    square/cube, lexicographic node numbering, full neighbour stencil with
    columns sorted ascending, strong zero Dirichlet on the whole boundary
    (SparseBlockMatrix::dirichlet: row and column zeroed, diagonal 1,
    LinAlg/sparseblockmatrix.xx:205-218)."""
    import scipy.sparse as sp
    h = 1.0 / N
    n1 = N + 1
    K = _q1_local_stiffness(dim, h)
    nloc = 2 ** dim
    nodes = cell_nodes(dim, N)                            # [ncell, nloc]
    kap = kappa.ravel()
    rows = np.repeat(nodes, nloc, axis=1).ravel()
    cols = np.tile(nodes, (1, nloc)).ravel()
    vals = (kap[:, None] * K.ravel()[None, :])
    if beta is not None and any(beta):
        vals = vals + _q1_local_convection(dim, h, beta).ravel()[None, :]
    vals = vals.ravel()
    n = n1 ** dim
    A = sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsr()
    A.sum_duplicates()
    A.sort_indices()
    # Dirichlet: boundary nodes
    idx = np.arange(n)
    coords = [(idx // n1 ** d) % n1 for d in range(dim)]
    onb = np.zeros(n, dtype=bool)
    for c in coords:
        onb |= (c == 0) | (c == N)
    rowptr = A.indptr.astype(np.int64)
    col = A.indices.astype(np.int64)
    val = A.data.astype(np.float64).copy()
    rowidx = np.repeat(np.arange(n), np.diff(rowptr))
    zero = onb[rowidx] | onb[col]
    val[zero] = 0.0
    isdiag = rowidx == col
    val[isdiag & onb[rowidx]] = 1.0
    diag = np.nonzero(isdiag)[0].astype(np.int64)
    coord = np.stack([c * h for c in coords], axis=1).astype(np.float64)
    return Level(n=n, B=1, rowptr=rowptr, col=col, diag=diag, val=val,
                 dirichlet=np.nonzero(onb)[0].astype(np.int64), coord=coord)


def _structured_transfer(dim: int, Nc: int) -> Transfer:
    """Nested Q1 transfer maps between Nc and 2*Nc cells per dimension in
    lexicographic numbering: a fine node with m odd coordinates has 2^m coarse
    parents (c2f for m = 0, zweier/vierer/achter for m = 1, 2, 3)."""
    nf1, nc1 = 2 * Nc + 1, Nc + 1
    fidx = np.arange(nf1 ** dim)
    fc = [(fidx // nf1 ** d) % nf1 for d in range(dim)]
    odd = np.stack([c % 2 for c in fc], axis=1)
    nodd = odd.sum(axis=1)

    def cid(cs):
        r = np.zeros_like(cs[0])
        for d in reversed(range(dim)):
            r = r * nc1 + cs[d]
        return r

    c2f = np.empty(nc1 ** dim, dtype=np.int64)
    m0 = nodd == 0
    c2f[cid([c[m0] // 2 for c in fc])] = fidx[m0]
    maps = []
    for m in (1, 2, 3):
        sel = nodd == m
        f = fidx[sel]
        parents = []
        if f.size:
            lo = [c[sel] // 2 for c in fc]
            od = [o for o in odd[sel].T]
            # enumerate 2^m parent combinations over the odd coordinates
            for bits in range(2 ** dim):
                take = np.ones(f.size, dtype=bool)
                cs = []
                for d in range(dim):
                    bd = (bits >> d) & 1
                    take &= (bd == 0) | (od[d] == 1)
                    cs.append(lo[d] + bd * od[d])
                parents.append((take, cid(cs)))
            par = np.stack([p for t, p in parents if True], axis=1)
            tk = np.stack([t for t, p in parents], axis=1)
            par = par[tk].reshape(f.size, 2 ** m)
            maps.append(np.concatenate([f[:, None], par], axis=1).astype(np.int64))
        else:
            maps.append(np.zeros((0, 1 + 2 ** m), dtype=np.int64))
    return Transfer(c2f=c2f, zweier=maps[0], vierer=maps[1], achter=maps[2])


def structured_problem(dim: int, coarse: int, refine: int,
                       kappa: Optional[np.ndarray] = None,
                       rhs: Optional[np.ndarray] = None, beta=None) -> Problem:
    """The reference's multilevel system for -div(kappa grad u) = f on the unit
    square/cube built from coarse^dim cells refined `refine` times, with the
    reference's default patchdepth 1: `refine` multigrid levels, the coarsest
    having 2*coarse cells per dimension (Mesh/hierarchicalmesh.cc:126-148,
    Mesh/meshagent.cc:83). kappa: per finest cell (lexicographic, x fastest),
    default 1. rhs: per finest node (lexicographic), default 1; zeroed at
    Dirichlet nodes. beta: constant convection vector (default none; the
    operator is then symmetric). The finest level's cells (for the
    coefficient gradient and the L2 functional) come with the problem."""
    Nf = coarse << refine
    if kappa is None:
        kappa = np.ones((Nf,) * dim)
    kappa = np.asarray(kappa, dtype=np.float64).reshape((Nf,) * dim)
    nlev = refine
    kap = kappa_pyramid(dim, kappa, nlev)
    levels = []
    for l in range(nlev):
        N = (2 * coarse) << l
        levels.append(_assemble_level(dim, N, kap[l], beta))
    transfers = [_structured_transfer(dim, (2 * coarse) << l) for l in range(nlev - 1)]
    nfin = levels[-1].n
    b = np.ones(nfin) if rhs is None else np.asarray(rhs, dtype=np.float64).copy()
    b[levels[-1].dirichlet] = 0.0
    hf = 1.0 / ((2 * coarse) << (nlev - 1))
    cells = Cells(nodes=cell_nodes(dim, (2 * coarse) << (nlev - 1)),
                  kloc=_q1_local_stiffness(dim, hf), mloc=_q1_local_mass(dim, hf))
    return Problem(dim=dim, levels=levels, transfers=transfers, rhs=b,
                   info={"generator": "structured", "coarse": coarse,
                         "refine": refine,
                         "beta": None if beta is None else list(beta)},
                   cells=cells)


def cell_parents(dim: int, N: int) -> np.ndarray:
    """Parent cell on the N/2 mesh of every cell of the uniform N mesh (both
    lexicographic, x fastest)."""
    i = np.arange(N)
    h = N // 2
    if dim == 3:
        k, j, ii = np.meshgrid(i, i, i, indexing="ij")
        return (((k // 2) * h + j // 2) * h + ii // 2).ravel().astype(np.int64)
    j, ii = np.meshgrid(i, i, indexing="ij")
    return ((j // 2) * h + ii // 2).ravel().astype(np.int64)


def structured_meshes(P: Problem):
    """Per level (cells, coordinates, parents) of a structured_problem
    hierarchy for gb_level_set_mesh (lexicographic cells, local nodes
    lexicographic; parents None on level 0)."""
    out = []
    for l, L in enumerate(P.levels):
        N = int(round(L.n ** (1.0 / P.dim))) - 1
        out.append((cell_nodes(P.dim, N), L.coord, cell_parents(P.dim, N) if l else None))
    return out


def seeded_inputs(dim: int, coarse: int, refine: int, kappa_seed: int = 1001,
                  rhs_seed: int = 1002, sigma: float = 1.0):
    """Seeded synthetic coefficient and load: kappa = exp(N(0, sigma)) per finest
    cell, f ~ U[-1, 1] per finest node (numpy PCG64 default_rng)."""
    Nf = coarse << refine
    kappa = np.exp(np.random.default_rng(kappa_seed).normal(0.0, sigma, size=Nf ** dim))
    rhs = np.random.default_rng(rhs_seed).uniform(-1.0, 1.0, size=(Nf + 1) ** dim)
    return kappa, rhs


# ------------------------------------------------------------------ Stokes

def _q1_local_derivative_mass(dim: int, h: float):
    """D[i][a, b] = integral of (d phi_b / d x_i) phi_a over a cube of width h
    (local order as _q1_local_stiffness)."""
    m = np.array([[1.0 / 3.0, 1.0 / 6.0], [1.0 / 6.0, 1.0 / 3.0]]) * h
    d = np.array([[-0.5, 0.5], [-0.5, 0.5]])
    if dim == 2:
        return [np.kron(m, d), np.kron(d, m)]
    return [np.kron(np.kron(m, m), d), np.kron(np.kron(m, d), m), np.kron(np.kron(d, m), m)]


def _stokes_local(dim: int, h: float, visc: float, stab: float) -> np.ndarray:
    """Element blocks E[a, b] ((dim+1) x (dim+1)) of the Stokes system in the
    reference's NavierStokes component order (0 = p, 1..dim = velocity):
    div v tested with q, Brezzi-Pitkaranta stab h^2 grad p . grad q,
    visc grad v_i . grad w_i and -p div w."""
    K = _q1_local_stiffness(dim, h)
    D = _q1_local_derivative_mass(dim, h)
    nl, B = 2 ** dim, dim + 1
    E = np.zeros((nl, nl, B, B))
    E[:, :, 0, 0] = stab * h * h * K
    for i in range(dim):
        E[:, :, 0, i + 1] = D[i]
        E[:, :, i + 1, i + 1] = visc * K
        E[:, :, i + 1, 0] = -D[i].T
    return E


def _patches(dim: int, N: int) -> np.ndarray:
    """Patches of 2^dim cells (3^dim nodes, local order lexicographic) of the
    N^dim lexicographic mesh, patches in lexicographic order."""
    n1, P = N + 1, N // 2
    loc = np.array([(a * n1 + b) * n1 + e for a in range(3) for b in range(3)
                    for e in range(3)]) if dim == 3 else \
        np.array([b * n1 + e for b in range(3) for e in range(3)])
    if dim == 3:
        k, j, i = np.meshgrid(np.arange(P), np.arange(P), np.arange(P), indexing="ij")
        base = ((2 * k * n1 + 2 * j) * n1 + 2 * i).ravel()
    else:
        j, i = np.meshgrid(np.arange(P), np.arange(P), indexing="ij")
        base = (2 * j * n1 + 2 * i).ravel()
    return (base[:, None] + loc[None, :]).astype(np.int64)


def cell_patches(dim: int, N: int) -> np.ndarray:
    """Single-cell Vanka patches (2^dim nodes): the 4-node (2D) cell patches of
    the 12 x 12 Stokes variant, one per cell, lexicographic."""
    return cell_nodes(dim, N)


def _assemble_stokes_level(dim: int, N: int, visc: float, stab: float) -> Level:
    import scipy.sparse as sp
    h = 1.0 / N
    n1 = N + 1
    n = n1 ** dim
    B = dim + 1
    E = _stokes_local(dim, h, visc, stab)
    nodes = cell_nodes(dim, N)
    nl = nodes.shape[1]
    rows = np.repeat(nodes, nl, axis=1).ravel()
    cols = np.tile(nodes, (1, nl)).ravel()
    comp = []
    for r in range(B):
        for c in range(B):
            vals = np.tile(E[:, :, r, c].ravel(), nodes.shape[0])
            A = sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsr()
            A.sum_duplicates()
            A.sort_indices()
            comp.append(A)
    rowptr = comp[0].indptr.astype(np.int64)
    col = comp[0].indices.astype(np.int64)
    for A in comp[1:]:
        assert np.array_equal(A.indptr, comp[0].indptr)
        assert np.array_equal(A.indices, comp[0].indices)
    val = np.stack([A.data for A in comp], axis=1).reshape(-1, B, B).copy()
    idx = np.arange(n)
    coords = [(idx // n1 ** d) % n1 for d in range(dim)]
    onb = np.zeros(n, dtype=bool)
    for c in coords:
        onb |= (c == 0) | (c == N)
    rowidx = np.repeat(np.arange(n), np.diff(rowptr))
    for c in range(1, B):  # velocity: strong Dirichlet rows and columns
        val[onb[rowidx], c, :] = 0.0
        val[onb[col], :, c] = 0.0
    isdiag = rowidx == col
    for c in range(1, B):
        val[isdiag & onb[rowidx], c, c] = 1.0
    diag = np.nonzero(isdiag)[0].astype(np.int64)
    # pressure filter weights: integral of each basis function
    w = np.zeros(n)
    np.add.at(w, nodes.ravel(), h ** dim / nl)
    lv = Level(n=n, B=B, rowptr=rowptr, col=col, diag=diag, val=val.ravel(),
               dirichlet=np.nonzero(onb)[0].astype(np.int64),
               dircomp_mask=sum(1 << c for c in range(1, B)),
               coord=np.stack([c * h for c in coords], axis=1).astype(np.float64),
               pf_mask=1, pf_weights=w, pf_domain=1.0, patches=_patches(dim, N))
    return lv


def stokes_rhs(dim: int, coarse: int, refine: int, seed: int = 1002) -> np.ndarray:
    """f ~ U[-1, 1] per node and component (p, v_1..v_dim), the pressure part
    made algebraically mean-free so that the system, whose pressure is fixed
    only up to a constant, is consistent."""
    n1 = (coarse << refine) + 1
    r = np.random.default_rng(seed).uniform(-1.0, 1.0, size=(n1 ** dim, dim + 1))
    r[:, 0] -= r[:, 0].mean()
    return r.ravel()


def structured_stokes(dim: int, coarse: int, refine: int, visc: float = 1.0,
                      stab: float = 0.1, rhs: Optional[np.ndarray] = None,
                      smoother: str = "vanka", patches: str = "patch") -> Problem:
    """The reference's multilevel Stokes system (Q1/Q1, Brezzi-Pitkaranta
    pressure stabilisation, velocity Dirichlet on the whole boundary, pressure
    filter on component 0, Vanka patches of 2^dim cells) on the unit
    square/cube in lexicographic numbering: what the oracle harness assembles
    with problem=stokes, in another node order. patches="cell" puts the Vanka
    smoother on single cells instead (2^dim-node patches; the reference's
    VankaSmoother uses 2^dim-cell patches only)."""
    nlev = refine
    levels = [_assemble_stokes_level(dim, (2 * coarse) << l, visc, stab)
              for l in range(nlev)]
    if patches == "cell":  # Vanka on single cells (12 x 12 local systems in 2D)
        for l, lv in enumerate(levels):
            lv.patches = cell_patches(dim, (2 * coarse) << l)
    transfers = [_structured_transfer(dim, (2 * coarse) << l) for l in range(nlev - 1)]
    b = stokes_rhs(dim, coarse, refine) if rhs is None else np.array(rhs, dtype=np.float64)
    fin = levels[-1]
    bd = b.reshape(fin.n, fin.B)
    bd[fin.dirichlet, 1:] = 0.0
    return Problem(dim=dim, levels=levels, transfers=transfers, rhs=bd.ravel(),
                   info={"generator": "structured-stokes", "coarse": coarse,
                         "refine": refine, "smoother": smoother, "visc": visc,
                         "stab": stab, "patches": patches})


# ------------------------------------------------------------------ Q2

def _q2_1d(H: float):
    """1D quadratic Lagrange element on [0, H] (nodes 0, H/2, H): mass,
    stiffness and D[i, j] = integral of phi_j' phi_i."""
    M = np.array([[4.0, 2.0, -1.0], [2.0, 16.0, 2.0], [-1.0, 2.0, 4.0]]) * (H / 30.0)
    K = np.array([[7.0, -8.0, 1.0], [-8.0, 16.0, -8.0], [1.0, -8.0, 7.0]]) / (3.0 * H)
    D = np.array([[-3.0, 4.0, -1.0], [-4.0, 0.0, 4.0], [1.0, -4.0, 3.0]]) / 6.0
    return M, K, D


def _q2_local(dim: int, H: float, eps: float, beta) -> np.ndarray:
    """Q2 element matrix of -eps Laplace u + beta . grad u on a cube of width
    H (a patch of 2^dim cells), local nodes lexicographic (x fastest)."""
    M, K, D = _q2_1d(H)
    if dim == 2:
        A = eps * (np.kron(M, K) + np.kron(K, M))
        if beta is not None:
            A = A + beta[0] * np.kron(M, D) + beta[1] * np.kron(D, M)
        return A
    A = eps * (np.kron(np.kron(M, M), K) + np.kron(np.kron(M, K), M)
               + np.kron(np.kron(K, M), M))
    if beta is not None:
        A = A + (beta[0] * np.kron(np.kron(M, M), D) + beta[1] * np.kron(np.kron(M, D), M)
                 + beta[2] * np.kron(np.kron(D, M), M))
    return A


def _assemble_q2_level(dim: int, N: int, eps: float, beta) -> Level:
    """CGQ2 on N^dim cells: Q2 elements on the (N/2)^dim patches, strong zero
    Dirichlet on the whole boundary."""
    import scipy.sparse as sp
    h = 1.0 / N
    n1 = N + 1
    n = n1 ** dim
    E = _q2_local(dim, 2.0 * h, eps, beta)
    nodes = _patches(dim, N)
    nl = nodes.shape[1]
    rows = np.repeat(nodes, nl, axis=1).ravel()
    cols = np.tile(nodes, (1, nl)).ravel()
    vals = np.tile(E.ravel(), nodes.shape[0])
    A = sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsr()
    A.sum_duplicates()
    A.sort_indices()
    idx = np.arange(n)
    coords = [(idx // n1 ** d) % n1 for d in range(dim)]
    onb = np.zeros(n, dtype=bool)
    for c in coords:
        onb |= (c == 0) | (c == N)
    rowptr = A.indptr.astype(np.int64)
    col = A.indices.astype(np.int64)
    val = A.data.astype(np.float64).copy()
    rowidx = np.repeat(np.arange(n), np.diff(rowptr))
    val[onb[rowidx] | onb[col]] = 0.0
    isdiag = rowidx == col
    val[isdiag & onb[rowidx]] = 1.0
    return Level(n=n, B=1, rowptr=rowptr, col=col, diag=np.nonzero(isdiag)[0].astype(np.int64),
                 val=val, dirichlet=np.nonzero(onb)[0].astype(np.int64),
                 coord=np.stack([c * h for c in coords], axis=1).astype(np.float64))


def structured_q2(dim: int, coarse: int, refine: int, eps: float = 1e-2,
                  beta=(1.0, 0.5, 0.25), rhs: Optional[np.ndarray] = None,
                  seed: int = 1002) -> Problem:
    """The reference's CGQ2 system (discname CGQ2, patchdepth 1) for
    -eps Laplace u + beta . grad u = f on the unit square/cube of
    (coarse*2^refine)^dim cells, lexicographic numbering, f ~ U[-1, 1] per
    node (seeded), zero Dirichlet; the multigrid transfers are the nodal ones
    of MgInterpolatorMatrix, as the reference uses them for Q2 as well."""
    beta = None if beta is None else tuple(beta)[:dim]
    levels = [_assemble_q2_level(dim, (2 * coarse) << l, eps, beta) for l in range(refine)]
    transfers = [_structured_transfer(dim, (2 * coarse) << l) for l in range(refine - 1)]
    nf = levels[-1].n
    b = (np.random.default_rng(seed).uniform(-1.0, 1.0, size=nf) if rhs is None
         else np.array(rhs, dtype=np.float64))
    b[levels[-1].dirichlet] = 0.0
    return Problem(dim=dim, levels=levels, transfers=transfers, rhs=b,
                   info={"generator": "structured-q2", "coarse": coarse, "refine": refine,
                         "eps": eps, "beta": None if beta is None else list(beta)})


# ------------------------------------------------ Q2 with a refined ball

def structured_q2_ball(coarse: int, refine: int, eps: float = 1e-2,
                       beta=(1.0, 0.5, 0.25), radius: float = 0.25,
                       seed: int = 1002) -> Problem:
    """CGQ2 convection-diffusion on the unit cube as structured_q2, plus one
    more level on which every patch (2x2x2 cells) whose centre lies within
    `radius` of the cube's centre is refined once (its 8 cells split, giving 8
    Q2 elements of half the width). Nodes of refined patches on faces and
    edges of unrefined neighbours hang: edge nodes on the neighbour's
    quadratic edge trace (3 parents, weights 3/8, 6/8, -1/8, nearest first),
    face nodes on its face (9 parents, tensor weights) - the hnq2 / hnq2face
    maps and weights of HNStructureQ23d. The matrix is condensed
    (C^T A C with the hanging rows and columns replaced by identity) on the
    pattern of the condensed elements' couplings plus every diagonal (as
    CGDisc::Structure builds it), strong zero Dirichlet on the boundary;
    transfers to the uniform level below are the nodal c2f / zweier / vierer /
    achter maps. The refinement rule is this generator's own (whole patches by
    centre), not the reference's. info["elements"] / info["parents"]: the
    finest level's Q2 elements (27 nodes, x fastest, hanging nodes included)
    and the patch of the level below each lies in, for the device assembly."""
    import scipy.sparse as sp
    dim = 3
    base = structured_q2(dim, coarse, refine, eps=eps, beta=beta, seed=seed)
    N = (2 * coarse) << (refine - 1)          # cells per dimension, uniform level
    P = N // 2                                # patches per dimension
    h = 1.0 / N
    M2 = 2 * N                                # node grid of the refined level
    pz, py, px = np.meshgrid(np.arange(P), np.arange(P), np.arange(P), indexing="ij")
    cen = (np.stack([px, py, pz], -1) * 2 + 1) * h
    refined = np.linalg.norm(cen - 0.5, axis=-1) < radius       # [P, P, P] (z, y, x)
    # nodes: the uniform level's nodes (even) and every node of refined patches
    ev = np.arange(0, M2 + 1, 2)
    Z, Y, X = np.meshgrid(ev, ev, ev, indexing="ij")
    pts = [np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)]
    loc5 = np.stack(np.meshgrid(np.arange(5), np.arange(5), np.arange(5), indexing="ij"),
                    -1).reshape(-1, 3)[:, ::-1]                  # (x, y, z), x fastest
    rp = np.argwhere(refined)[:, ::-1]                            # (px, py, pz)
    for p in rp:
        pts.append(4 * p[None, :] + loc5)
    allp = np.unique(np.concatenate(pts), axis=0)
    key = (allp[:, 2] * (M2 + 1) + allp[:, 1]) * (M2 + 1) + allp[:, 0]
    order = np.argsort(key)
    allp, key = allp[order], key[order]
    n = allp.shape[0]

    def ids(q):  # integer points (x, y, z) -> node ids
        k = (q[..., 2] * (M2 + 1) + q[..., 1]) * (M2 + 1) + q[..., 0]
        i = np.searchsorted(key, k)
        assert np.all(key[np.minimum(i, n - 1)] == k)
        return i

    # elements: unrefined patches (spacing 2) and the 8 halves of refined ones
    loc3 = np.stack(np.meshgrid(np.arange(3), np.arange(3), np.arange(3), indexing="ij"),
                    -1).reshape(-1, 3)[:, ::-1]
    up = np.argwhere(~refined)[:, ::-1]
    el_c = ids(4 * up[:, None, :] + 2 * loc3[None, :, :])          # [nu, 27]
    sub = np.stack(np.meshgrid(np.arange(2), np.arange(2), np.arange(2), indexing="ij"),
                   -1).reshape(-1, 3)[:, ::-1]
    el_f = ids((4 * rp[:, None, None, :] + 2 * sub[None, :, None, :]
                + loc3[None, None, :, :]).reshape(-1, 27, 3))       # [nr*8, 27]
    Ec = _q2_local(dim, 2.0 * h, eps, beta)
    Ef = _q2_local(dim, h, eps, beta)
    rows = np.concatenate([np.repeat(el_c, 27, axis=1).ravel(),
                           np.repeat(el_f, 27, axis=1).ravel()])
    cols = np.concatenate([np.tile(el_c, (1, 27)).ravel(), np.tile(el_f, (1, 27)).ravel()])
    vals = np.concatenate([np.tile(Ec.ravel(), el_c.shape[0]),
                           np.tile(Ef.ravel(), el_f.shape[0])])
    A = sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsr()
    # hanging nodes: odd nodes on the closure of an unrefined patch
    odd = allp % 2 == 1
    nodd = odd.sum(1)
    # a node with one or two odd coordinates hangs when it lies on the closure
    # of an unrefined patch (whose own nodes are all even)
    kk = allp // 4
    on4 = (allp % 4 == 0).astype(np.int64)
    touches = np.zeros(n, dtype=bool)
    for bits in range(8):
        off = np.array([(bits >> d) & 1 for d in range(3)])
        k = kk - off[None, :] * on4
        ok = np.all((k >= 0) & (k < P), axis=1)
        kc = np.clip(k, 0, P - 1)
        touches |= ok & ~refined[kc[:, 2], kc[:, 1], kc[:, 0]]
    w3 = np.array([0.375, 0.75, -0.125])

    def line(c):  # the 3 coarse positions along an odd coordinate, nearest first
        lo = 4 * (c // 4)
        near = (c % 4) == 1
        return np.stack([np.where(near, lo, lo + 4), lo + 2, np.where(near, lo + 4, lo)], 1)

    sel_e = np.nonzero(touches & (nodd == 1))[0]
    q = allp[sel_e]
    d = np.argmax(odd[sel_e], axis=1)
    ln = line(q[np.arange(sel_e.size), d])
    par = np.repeat(q[:, None, :], 3, axis=1)
    par[np.arange(sel_e.size)[:, None], np.arange(3)[None, :], d[:, None]] = ln
    edges = np.concatenate([sel_e[:, None], ids(par)], 1)
    sel_f = np.nonzero(touches & (nodd == 2))[0]
    q = allp[sel_f]
    oo = odd[sel_f]
    d0 = np.argmax(oo, axis=1)
    d1 = 2 - np.argmax(oo[:, ::-1], axis=1)
    l0 = line(q[np.arange(sel_f.size), d0])
    l1 = line(q[np.arange(sel_f.size), d1])
    par = np.repeat(q[:, None, :], 9, axis=1)
    r = np.arange(sel_f.size)[:, None]
    par[r, np.arange(9)[None, :], d0[:, None]] = np.repeat(l0, 3, axis=1)
    par[r, np.arange(9)[None, :], d1[:, None]] = np.tile(l1, (1, 3))
    faces = np.concatenate([sel_f[:, None], ids(par)], 1)
    edges = np.array(edges, dtype=np.int64).reshape(-1, 4)
    faces = np.array(faces, dtype=np.int64).reshape(-1, 10)
    # condensation C^T A C, hanging rows and columns -> identity
    hang = np.concatenate([edges[:, 0], faces[:, 0]])
    free = np.ones(n, dtype=bool)
    free[hang] = False
    cr = [np.nonzero(free)[0]]
    cc = [np.nonzero(free)[0]]
    cv = [np.ones(free.sum())]
    for k in range(3):
        cr.append(edges[:, 0])
        cc.append(edges[:, 1 + k])
        cv.append(np.full(edges.shape[0], w3[k]))
    for a in range(3):
        for b in range(3):
            cr.append(faces[:, 0])
            cc.append(faces[:, 1 + 3 * a + b])
            cv.append(np.full(faces.shape[0], w3[a] * w3[b]))
    Cm = sp.coo_matrix((np.concatenate(cv), (np.concatenate(cr), np.concatenate(cc))),
                       shape=(n, n)).tocsr()
    Ac = (Cm.T @ A @ Cm).tocsr()
    Ac.sum_duplicates()
    Ac.sort_indices()
    # the pattern is the condensed elements' couplings plus every diagonal (a
    # product of nonnegative patterns: couplings whose values cancel stay)
    Cp = Cm.copy()
    Cp.data[:] = 1.0
    Ap = A.copy()
    Ap.data[:] = 1.0
    Sp = (Cp.T @ (Ap + sp.identity(n, format="csr")) @ Cp).tocsr()
    Sp = (Sp + sp.coo_matrix((np.ones(hang.size), (hang, hang)), shape=(n, n))).tocsr()
    Sp.sum_duplicates()
    Sp.sort_indices()
    ks = np.repeat(np.arange(n, dtype=np.int64), np.diff(Sp.indptr)) * n + Sp.indices
    ka = np.repeat(np.arange(n, dtype=np.int64), np.diff(Ac.indptr)) * n + Ac.indices
    at = np.searchsorted(ks, ka)
    assert np.array_equal(ks[at], ka)
    vals = np.zeros(ks.size)
    vals[at] = Ac.data
    hrow = np.zeros(n, dtype=bool)
    hrow[hang] = True
    vals[hrow[ks // n] & (ks // n == Sp.indices)] = 1.0   # hanging rows: identity
    Sp.data = vals
    Ac = Sp
    onb = np.any((allp == 0) | (allp == M2), axis=1)
    rowptr = Ac.indptr.astype(np.int64)
    col = Ac.indices.astype(np.int64)
    val = Ac.data.astype(np.float64).copy()
    ri = np.repeat(np.arange(n), np.diff(rowptr))
    val[onb[ri] | onb[col]] = 0.0
    isdiag = ri == col
    val[isdiag & onb[ri]] = 1.0
    fine = Level(n=n, B=1, rowptr=rowptr, col=col, diag=np.nonzero(isdiag)[0].astype(np.int64),
                 val=val, dirichlet=np.nonzero(onb)[0].astype(np.int64),
                 coord=allp.astype(np.float64) / M2, hn_edges=edges, hn_faces=faces,
                 hn_disc=3)
    # transfer from the uniform level (node (x, y, z) there is (2x, 2y, 2z) here)
    nc1 = N + 1
    cidx = np.arange(nc1 ** 3)
    cpos = np.stack([cidx % nc1, (cidx // nc1) % nc1, cidx // nc1 ** 2], 1)
    c2f = ids(2 * cpos)
    cid = lambda q: (q[:, 2] * nc1 + q[:, 1]) * nc1 + q[:, 0]
    maps = []
    for m in (1, 2, 3):
        sel = np.nonzero(nodd == m)[0]
        q = allp[sel]
        lo = q // 2
        o = odd[sel].astype(np.int64)
        par = []
        for bits in range(8):
            bb = np.array([(bits >> d) & 1 for d in range(3)])
            take = np.all((bb[None, :] == 0) | (o == 1), axis=1)
            par.append((take, cid(lo + bb[None, :] * o)))
        tk = np.stack([t for t, _ in par], 1)
        pp = np.stack([c for _, c in par], 1)[tk].reshape(sel.size, 2 ** m)
        maps.append(np.concatenate([sel[:, None], pp], 1).astype(np.int64))
    tr = Transfer(c2f=c2f.astype(np.int64), zweier=maps[0], vierer=maps[1], achter=maps[2])
    b = np.random.default_rng(seed).uniform(-1.0, 1.0, size=n)
    b[onb] = 0.0
    b[hang] = 0.0
    return Problem(dim=dim, levels=base.levels + [fine], transfers=base.transfers + [tr],
                   rhs=b, info={"generator": "structured-q2-ball", "coarse": coarse,
                                "refine": refine, "eps": eps, "radius": radius,
                                "hanging": int(hang.size), "refined_patches": int(rp.shape[0]),
                                "elements": np.concatenate([el_c, el_f]).astype(np.int64),
                                "parents": np.concatenate([
                                    (up[:, 2] * P + up[:, 1]) * P + up[:, 0],
                                    np.repeat((rp[:, 2] * P + rp[:, 1]) * P + rp[:, 0], 8)
                                ]).astype(np.int64)})


def q2_meshes(prob: Problem):
    """Per level (Q2 elements [ne, 3^dim], parent element on the level below
    or None) of a structured_q2 / structured_q2_ball problem, for
    gb_level_set_mesh_degree: uniform levels as lexicographic patches, a ball
    level as the generator recorded it."""
    out = []
    for l, L in enumerate(prob.levels):
        if l == prob.nlevels - 1 and "elements" in prob.info:
            out.append((prob.info["elements"], prob.info["parents"]))
            continue
        dim = prob.dim
        Np = (round(L.n ** (1.0 / dim)) - 1) // 2
        n1 = 2 * Np + 1
        g = np.meshgrid(*([np.arange(Np)] * dim), indexing="ij")
        base = 0
        for d in range(dim):                       # g[0] slowest (z), g[-1] x
            base = base * n1 + 2 * g[d].ravel()
        loc = np.zeros(1, dtype=np.int64)
        for d in range(dim):
            loc = (loc[:, None] * n1 + np.arange(3)[None, :]).ravel()
        out.append((base[:, None] + loc[None, :], cell_parents(dim, Np) if l else None))
    return out


# ------------------------------------------------------- accuracy helpers
#
# The benchmark reports each result's error against the reference's FP64
# solution of the same problem. The reference numbers its nodes
# hierarchically; these helpers map a uniform mesh's nodes to the
# lexicographic order by their coordinates and evaluate J(u) = int u^2 exactly
# for Q1 functions (the reference's Gauss rules integrate it exactly too).

def lex_index(coord: np.ndarray, N: int) -> np.ndarray:
    """Lexicographic index (x fastest) of every node of a uniform mesh of N
    cells per dimension on the unit square/cube, from its coordinates."""
    c = np.rint(np.asarray(coord) * N).astype(np.int64)
    idx = np.zeros(c.shape[0], dtype=np.int64)
    for d in reversed(range(c.shape[1])):
        idx = idx * (N + 1) + c[:, d]
    return idx


def to_lex(values: np.ndarray, coord: np.ndarray, N: int, ncomp: int = 1) -> np.ndarray:
    """A nodal vector (ncomp values per node, node-major) in the numbering of
    `coord`, reordered lexicographically."""
    v = np.asarray(values).reshape(-1, ncomp)
    out = np.empty_like(v)
    out[lex_index(coord, N)] = v
    return out.reshape(-1)


def q1_l2_squared(u_lex: np.ndarray, dim: int, N: int, ncomp: int = 1,
                  comps=(0,)) -> float:
    """int sum_{c in comps} u_c^2 over the unit square/cube for Q1 nodal
    values on the lexicographic grid: u^T M u with the consistent mass matrix,
    applied as the tensor product of 1D mass matrices (h/6 [1 4 1])."""
    h = 1.0 / N
    u = np.asarray(u_lex, dtype=np.float64).reshape(-1, ncomp)
    total = 0.0
    for c in comps:
        g = u[:, c].reshape((N + 1,) * dim)
        m = g.copy()
        for ax in range(dim):
            s = np.moveaxis(m, ax, 0)
            t = 4.0 * s
            t[1:] += s[:-1]
            t[:-1] += s[1:]
            t[0] -= 2.0 * s[0]   # boundary rows: h/6 [2 1]
            t[-1] -= 2.0 * s[-1]
            m = np.moveaxis(t * (h / 6.0), 0, ax)
        total += float(np.sum(g * m))
    return total


def q1_cell_gradient(u_lex: np.ndarray, lam_lex: np.ndarray, dim: int, N: int,
                     dirichlet_lex: np.ndarray) -> np.ndarray:
    """dJ/dkappa_c = -lambda_c^T K_c u_c per cell (K_c the unit-coefficient Q1
    stiffness of the uniform cell), with u and lambda read as zero on the
    Dirichlet nodes: the gradient the device's gb_coeff_gradient forms."""
    u = np.asarray(u_lex, dtype=np.float64).copy()
    lam = np.asarray(lam_lex, dtype=np.float64).copy()
    u[dirichlet_lex] = 0.0
    lam[dirichlet_lex] = 0.0
    cn = cell_nodes(dim, N)
    K = _q1_local_stiffness(dim, 1.0 / N)
    return -np.einsum("ca,ab,cb->c", lam[cn], K, u[cn])


def boundary_lex(dim: int, N: int) -> np.ndarray:
    """Lexicographic indices of the boundary nodes of the unit square/cube."""
    g = np.indices((N + 1,) * dim).reshape(dim, -1)
    return np.nonzero(((g == 0) | (g == N)).any(0))[0]
