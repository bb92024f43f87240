/*
 * ORACLE - TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, FP64, single-threaded restatement of the reference's CPU linear-solve
 * path (Gascoigne: StdMultiLevelSolver::Gmres + LinearMg/mgstep, damped-Jacobi
 * smoothing, MgInterpolatorMatrix transfers, strong Dirichlet zeroing, CGInfo).
 * Only the tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * it, and only as the checker. The product path never calls it.
 *
 * Parity is pinned against the reference itself: tests run this restatement and
 * the compiled reference (oracle/_ref/ref_harness, built from the reference's own
 * sources by oracle/ref/Makefile) on identical per-level matrices and transfer
 * maps dumped by that harness, and compare iteration counts and solutions.
 *
 * Every function cites the reference file:line it restates. Arithmetic order
 * follows the reference where it matters for rounding (sequential per-row
 * accumulation of FMatrixBlock::cadd, sequential dot products).
 *
 * Conventions: level 0 is the coarsest, as in the reference's solver indexing
 * (Solver/stdmultilevelsolver.cc:224-231). Vectors are node-major interleaved
 * (CompVector, Common/compvector.h:98-113): entry (node i, comp c) at i*B+c.
 * Matrix blocks are row-major B x B (NodeMatrix::value, LinAlg/nodematrix.h:44-48).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_MAXB 8

typedef struct
{
  int64_t n;              /* block rows */
  int B;                  /* block size (ncomp) */
  const int64_t* rowptr;  /* n+1 */
  const int64_t* col;     /* nnzb */
  const int64_t* diag;    /* n, position of the diagonal block in row i */
  const double* val;      /* nnzb*B*B, row-major blocks */
  int64_t ndir;           /* Dirichlet nodes */
  const int64_t* dir;     /* node indices */
  int dircomp_mask;       /* bit c set: component c is Dirichlet (all colours) */
  /* pressure filter (PressureFilter, Discretization/Q1/pressurefilter.cc:56-100,
   * weights from CGDisc::InitFilter, DofHandler/cgdisc.h:1061-1090) */
  int pf_mask;            /* bit c set: component c is filtered; 0: inactive */
  const double* pf_w;     /* n weights: integral of each basis function */
  double pf_domain;       /* domain size */
  int64_t nhanging;       /* hanging nodes (excluded from the algebraic mean) */
  /* Vanka patches: DofHandler::GetElement(2, p) (DofHandler/dofhandler.h:389-396) */
  int64_t npatch;
  int npp;                /* nodes per patch */
  const int64_t* patches; /* npatch * npp node indices */
  /* hanging nodes (HangingIndexHandler hnq2 / hnq2face, Mesh/
   * hangingindexhandler.h:40,65) and the discretisation whose HNStructure
   * acts on them: 0 Q12d, 1 Q13d, 2 Q22d, 3 Q23d */
  int hn_disc;
  int64_t nhedge;
  const int64_t* hnedge;  /* nhedge rows [node, 3 parents], ascending node */
  int64_t nhface;
  const int64_t* hnface;  /* nhface rows [node, 9 parents], ascending node */
} or_level;

/* Transfer level l (coarse) <-> l+1 (fine) in the form MgInterpolatorMatrix
 * builds it (Discretization/Q1/mginterpolatormatrix.cc:34-121): both directions
 * as CSR with columns sorted ascending (SparseStructure keeps std::set rows). */
typedef struct
{
  int64_t ncoarse, nfine;
  int64_t *r_ptr, *r_col; /* restriction: coarse row -> fine columns */
  double* r_w;
  int64_t *p_ptr, *p_col; /* prolongation: fine row -> coarse columns */
  double* p_w;
} or_transfer;

typedef struct
{
  int nlevels;
  or_level* L;            /* nlevels */
  or_transfer* T;         /* nlevels-1 */
  /* StdSolver / SolverData keys (Solver/solverdata.cc:41-55) */
  int iterpre, iterpost, iterexact;
  double omega;
  /* StdMultiLevelSolverData keys (Solver/stdmultilevelsolverdata.cc:88-100) */
  double mgomega;
  char mgtype;            /* 'V', 'W' or 'F' */
  /* work vectors per level: u, b, v of mgstep and the smoother's h */
  double **u, **b, **v;
  /* linear_smooth: 0 jacobi, 1 ilu with matrixtype vanka (VankaSmoother) */
  int smoother;
  double** vlu;           /* per level: npatch LU factors, (npp*B)^2 each */
  int** vperm;            /* per level: npatch row permutations, npp*B each */
  double* vtmp;           /* finest-size scratch for the Vanka solve */
  int* vcount;
  /* coarsest-level direct solve (StdSolver::smooth_exact with UMFPACK,
   * Solver/stdsolver.cc:1003-1025, when the level has fewer than ndirect
   * nodes, :218-222): dense LU with partial pivoting of level 0 */
  double* dlu;
  int* dperm;
  /* linear_smooth ilu with matrixtype block (smoother 2): per level the
   * factors of SparseBlockIlu in the identity order, columns ascending */
  int64_t **iptr, **icol, **idiag;
  double** ival;
} or_mg;

/* ---------------------------------------------------------------- vectors */

/* nvector::operator* (Common/nvector.h:332-343): sequential sum */
double
or_dot(int64_t n, const double* x, const double* y)
{
  double d = 0.0;
  for (int64_t i = 0; i < n; ++i)
    d += x[i] * y[i];
  return d;
}

/* nvector::norm: sqrt of the sequential sum of squares */
double
or_norm(int64_t n, const double* x)
{
  return sqrt(or_dot(n, x, x));
}

/* ------------------------------------------------------------- block ops */

/* SparseBlockMatrix<B>::vmult (LinAlg/sparseblockmatrix.xx:378-392) with
 * FMatrixBlock::cadd (LinAlg/fmatrixblock.h:110-122): y(i) += s * (A_ij x(j)),
 * blocks visited in stencil order, each block row sum formed first. */
void
or_bsr_vmult(const or_level* A, double* y, const double* x, double s)
{
  const int B = A->B;
  for (int64_t i = 0; i < A->n; ++i) {
    double* yi = y + i * B;
    for (int64_t pos = A->rowptr[i]; pos < A->rowptr[i + 1]; ++pos) {
      const double* m = A->val + pos * B * B;
      const double* xj = x + A->col[pos] * B;
      for (int r = 0; r < B; ++r) {
        double sum = 0.0;
        for (int c = 0; c < B; ++c)
          sum += m[r * B + c] * xj[c];
        yi[r] += s * sum;
      }
    }
  }
}

/* Transposed product y += s * A^T x, the operator SparseBlockMatrix::transpose
 * (LinAlg/sparseblockmatrix.xx:478-491) followed by vmult applies. */
void
or_bsr_vmult_transpose(const or_level* A, double* y, const double* x, double s)
{
  const int B = A->B;
  for (int64_t i = 0; i < A->n; ++i) {
    const double* xi = x + i * B;
    for (int64_t pos = A->rowptr[i]; pos < A->rowptr[i + 1]; ++pos) {
      const double* m = A->val + pos * B * B;
      double* yj = y + A->col[pos] * B;
      for (int c = 0; c < B; ++c) {
        double sum = 0.0;
        for (int r = 0; r < B; ++r)
          sum += m[r * B + c] * xi[r];
        yj[c] += s * sum;
      }
    }
  }
}

/* NodeMatrix::gauss_jordan (LinAlg/nodematrix.h:159-213), in place on a
 * row-major N x N block. */
void
or_gauss_jordan(int N, double* a)
{
  int p[OR_MAXB];
  double hv[OR_MAXB];
  int i, j, k, r;
  double max, hr;
#define A_(i, j) a[(i) * N + (j)]
  for (i = 0; i < N; i++)
    p[i] = i;
  for (j = 0; j < N; j++) {
    max = fabs(A_(j, j));
    r = j;
    for (i = j + 1; i < N; i++) {
      if (fabs(A_(i, j)) > max) {
        max = fabs(A_(i, j));
        r = i;
      }
    }
    if (r > j) {
      for (k = 0; k < N; k++) {
        hr = A_(j, k);
        A_(j, k) = A_(r, k);
        A_(r, k) = hr;
      }
      i = p[j];
      p[j] = p[r];
      p[r] = i;
    }
    hr = 1. / A_(j, j);
    A_(j, j) = hr;
    for (k = 0; k < N; k++) {
      if (k == j)
        continue;
      for (i = 0; i < N; i++) {
        if (i == j)
          continue;
        A_(i, k) -= A_(i, j) * A_(j, k) * hr;
      }
    }
    for (i = 0; i < N; i++) {
      A_(i, j) *= hr;
      A_(j, i) *= -hr;
    }
    A_(j, j) = hr;
  }
  for (i = 0; i < N; i++) {
    for (k = 0; k < N; k++)
      hv[p[k]] = A_(i, k);
    for (k = 0; k < N; k++)
      A_(i, k) = hv[k];
  }
#undef A_
}

/* SparseBlockMatrix::Jacobi (LinAlg/sparseblockmatrix.xx:47-56): each node's
 * diagonal block is inverted (gauss_jordan) and applied in place with
 * FMatrixBlock::vmult (LinAlg/fmatrixblock.h:192-218). */
void
or_jacobi(const or_level* A, double* h)
{
  const int B = A->B;
  double d[OR_MAXB * OR_MAXB], t[OR_MAXB];
  for (int64_t i = 0; i < A->n; ++i) {
    memcpy(d, A->val + A->diag[i] * B * B, sizeof(double) * B * B);
    or_gauss_jordan(B, d);
    double* hi = h + i * B;
    for (int c = 0; c < B; ++c)
      t[c] = hi[c];
    for (int r = 0; r < B; ++r) {
      hi[r] = 0.0;
      for (int c = 0; c < B; ++c)
        hi[r] += d[r * B + c] * t[c];
    }
  }
}

/* Inverse diagonal blocks for all nodes (the per-assembly form of the above). */
void
or_blockdiag_inverse(const or_level* A, double* out)
{
  const int B = A->B;
  for (int64_t i = 0; i < A->n; ++i) {
    memcpy(out + i * B * B, A->val + A->diag[i] * B * B, sizeof(double) * B * B);
    or_gauss_jordan(B, out + i * B * B);
  }
}

/* CGDisc::StrongDirichletVectorZero (DofHandler/cgdisc.h:1162-1179) */
void
or_dirichlet_zero(const or_level* A, double* u)
{
  for (int64_t k = 0; k < A->ndir; ++k)
    for (int c = 0; c < A->B; ++c)
      if (A->dircomp_mask & (1 << c))
        u[A->dir[k] * A->B + c] = 0.0;
}

/* PressureFilter::SubtractMean (Discretization/Q1/pressurefilter.cc:56-84)
 * via StdSolver::SubtractMean (Solver/stdsolver.cc:1736-1747): per filtered
 * component, mean = sum_j u(j,c) w_j (sequential), u(., c) -= mean / domain. */
void
or_subtract_mean(const or_level* A, double* u)
{
  const int B = A->B;
  for (int c = 0; c < B; ++c) {
    if (!(A->pf_mask & (1 << c)))
      continue;
    double mean = 0.0;
    for (int64_t j = 0; j < A->n; ++j)
      mean += u[j * B + c] * A->pf_w[j];
    const double sub = mean / A->pf_domain;
    for (int64_t j = 0; j < A->n; ++j)
      u[j * B + c] += -sub;
  }
}

/* PressureFilter::SubtractMeanAlgebraic (pressurefilter.cc:88-100) via
 * StdSolver::SubtractMeanAlgebraic (Solver/stdsolver.cc:1752-1762). */
void
or_subtract_mean_algebraic(const or_level* A, double* u)
{
  const int B = A->B;
  for (int c = 0; c < B; ++c) {
    if (!(A->pf_mask & (1 << c)))
      continue;
    double d = 0.0;
    for (int64_t j = 0; j < A->n; ++j)
      d += u[j * B + c];
    d /= (double)(A->n - A->nhanging);
    for (int64_t j = 0; j < A->n; ++j)
      u[j * B + c] += -d;
  }
}

/* VankaSmoother::copy_entries_sparseblockmatrix (LinAlg/vankasmoother.cc:
 * 65-113): the patch matrix (entries of the level matrix whose row and column
 * nodes both lie in the patch, node-major with the components inside), then
 * its LU factorisation with row partial pivoting (Eigen::PartialPivLU as the
 * oracle's Eigen shim restates it: the first row of largest |a_ik| is the
 * pivot; the column below the pivot is divided by it; the trailing block is
 * updated entry by entry, k ascending). lu is row-major m x m, m = npp*B. */
void
or_vanka_factor(const or_level* A, int64_t p, double* lu, int* perm)
{
  const int B = A->B, npp = A->npp, m = npp * B;
  const int64_t* pn = A->patches + p * npp;
  memset(lu, 0, sizeof(double) * m * m);
  for (int r = 0; r < npp; ++r) {
    const int64_t row = pn[r];
    for (int64_t pos = A->rowptr[row]; pos < A->rowptr[row + 1]; ++pos) {
      int c = -1;
      for (int q = 0; q < npp; ++q)
        if (pn[q] == A->col[pos]) {
          c = q;
          break;
        }
      if (c < 0)
        continue;
      const double* blk = A->val + pos * B * B;
      for (int cr = 0; cr < B; ++cr)
        for (int cc = 0; cc < B; ++cc)
          lu[(B * r + cr) * m + B * c + cc] = blk[cr * B + cc];
    }
  }
  for (int i = 0; i < m; ++i)
    perm[i] = i;
  for (int k = 0; k < m; ++k) {
    int piv = k;
    double best = fabs(lu[k * m + k]);
    for (int i = k + 1; i < m; ++i)
      if (fabs(lu[i * m + k]) > best) {
        best = fabs(lu[i * m + k]);
        piv = i;
      }
    if (piv != k) {
      for (int j = 0; j < m; ++j) {
        double t = lu[k * m + j];
        lu[k * m + j] = lu[piv * m + j];
        lu[piv * m + j] = t;
      }
      int t = perm[k];
      perm[k] = perm[piv];
      perm[piv] = t;
    }
    if (lu[k * m + k] != 0)
      for (int i = k + 1; i < m; ++i)
        lu[i * m + k] /= lu[k * m + k];
    for (int j = k + 1; j < m; ++j)
      for (int i = k + 1; i < m; ++i)
        lu[i * m + j] -= lu[i * m + k] * lu[k * m + j];
  }
}

/* VankaSmoother::solve (LinAlg/vankasmoother.cc:192-237) with one thread:
 * x = average over the patches containing each node of the patch solutions
 * of the local systems with right-hand side x (the residual); contributions
 * are summed in patch order. tmp: ndof scratch, count: n scratch. */
void
or_vanka_solve(const or_level* A, const double* lu, const int* perm, double* x,
               double* tmp, int* count)
{
  const int B = A->B, npp = A->npp, m = npp * B;
  double H[8 * 27], G[8 * 27];
  memcpy(tmp, x, sizeof(double) * A->n * B);
  memset(x, 0, sizeof(double) * A->n * B);
  memset(count, 0, sizeof(int) * A->n);
  for (int64_t p = 0; p < A->npatch; ++p) {
    const int64_t* pn = A->patches + p * npp;
    const double* L = lu + p * m * m;
    const int* P = perm + p * m;
    for (int r = 0; r < npp; ++r)
      for (int c = 0; c < B; ++c)
        G[B * r + c] = tmp[pn[r] * B + c];
    for (int i = 0; i < m; ++i)
      H[i] = G[P[i]];
    for (int i = 0; i < m; ++i) { /* unit lower */
      double s = H[i];
      for (int j = 0; j < i; ++j)
        s -= L[i * m + j] * H[j];
      H[i] = s;
    }
    for (int i = m - 1; i >= 0; --i) { /* upper */
      double s = H[i];
      for (int j = i + 1; j < m; ++j)
        s -= L[i * m + j] * H[j];
      H[i] = s / L[i * m + i];
    }
    for (int r = 0; r < npp; ++r) {
      count[pn[r]]++;
      for (int c = 0; c < B; ++c)
        x[pn[r] * B + c] += H[B * r + c];
    }
  }
  for (int64_t i = 0; i < A->n; ++i) {
    const double s = 1.0 / count[i];
    for (int c = 0; c < B; ++c)
      x[i * B + c] *= s;
  }
}

/* ------------------------------------------------------- hanging nodes */
/* HNStructureQ12d/Q13d/Q22d/Q23d Average, Distribute, Zero
 * (Discretization/Q1/hnstructureq12d.cc:196-243, hnstructureq13d.cc:148-188,
 *  Discretization/Q2/hnstructureq22d.cc:50-76, hnstructureq23d.cc:118-153),
 * with CompVector::equ_node/add_node's expression order
 * (Common/compvector.h:190-262). */
static const double or_q2w[3] = { 0.375, 0.75, -0.125 };

static void
or_hn_edges_average(const or_level* A, double* u)
{
  const int B = A->B;
  const int q2 = A->hn_disc >= 2;
  for (int64_t k = 0; k < A->nhedge; ++k) {
    const int64_t* e = A->hnedge + 4 * k;
    for (int c = 0; c < B; ++c) {
      const double u0 = u[e[1] * B + c], u1 = u[e[2] * B + c];
      if (q2)
        u[e[0] * B + c] = or_q2w[0] * u0 + or_q2w[1] * u1 + or_q2w[2] * u[e[3] * B + c];
      else
        u[e[0] * B + c] = 0.5 * u0 + 0.5 * u1;
    }
  }
}

static void
or_hn_faces_average(const or_level* A, double* u)
{
  const int B = A->B;
  for (int64_t k = 0; k < A->nhface; ++k) {
    const int64_t* f = A->hnface + 10 * k;
    const int64_t* p = f + 1;
    for (int c = 0; c < B; ++c) {
#define U_(j) u[p[j] * B + c]
      if (A->hn_disc == 3) {
        double w[9];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j)
            w[3 * i + j] = or_q2w[i] * or_q2w[j];
        double v = w[0] * U_(0) + w[1] * U_(1) + w[2] * U_(2);
        v += w[3] * U_(3) + w[4] * U_(4) + w[5] * U_(5);
        v += w[6] * U_(6) + w[7] * U_(7) + w[8] * U_(8);
        u[f[0] * B + c] = v;
      } else {
        u[f[0] * B + c] = 0.25 * U_(0) + 0.25 * U_(1) + 0.25 * U_(3) + 0.25 * U_(4);
      }
#undef U_
    }
  }
}

static void
or_hn_edges_distribute(const or_level* A, double* u)
{
  const int B = A->B;
  const int q2 = A->hn_disc >= 2;
  for (int64_t k = 0; k < A->nhedge; ++k) {
    const int64_t* e = A->hnedge + 4 * k;
    for (int j = 0; j < (q2 ? 3 : 2); ++j)
      for (int c = 0; c < B; ++c)
        u[e[1 + j] * B + c] += (q2 ? or_q2w[j] : 0.5) * u[e[0] * B + c];
    for (int c = 0; c < B; ++c)
      u[e[0] * B + c] = 0.0;
  }
}

static void
or_hn_faces_distribute(const or_level* A, double* u)
{
  const int B = A->B;
  for (int64_t k = 0; k < A->nhface; ++k) {
    const int64_t* f = A->hnface + 10 * k;
    if (A->hn_disc == 3) {
      for (int j = 0; j < 9; ++j)
        for (int c = 0; c < B; ++c)
          u[f[1 + j] * B + c] += (or_q2w[j / 3] * or_q2w[j % 3]) * u[f[0] * B + c];
    } else {
      static const int q1f[4] = { 0, 1, 3, 4 };
      for (int j = 0; j < 4; ++j)
        for (int c = 0; c < B; ++c)
          u[f[1 + q1f[j]] * B + c] += 0.25 * u[f[0] * B + c];
    }
    for (int c = 0; c < B; ++c)
      u[f[0] * B + c] = 0.0;
  }
}

void
or_hn_average(const or_level* A, double* u)
{
  if (A->hn_disc == 3) { /* Q23d: faces, then edges */
    or_hn_faces_average(A, u);
    or_hn_edges_average(A, u);
  } else {              /* Q12d, Q22d: edges; Q13d: edges, then faces */
    or_hn_edges_average(A, u);
    if (A->hn_disc == 1)
      or_hn_faces_average(A, u);
  }
}

void
or_hn_distribute(const or_level* A, double* u)
{
  if (A->hn_disc == 3) {
    or_hn_faces_distribute(A, u);
    or_hn_edges_distribute(A, u);
  } else {
    or_hn_edges_distribute(A, u);
    if (A->hn_disc == 1)
      or_hn_faces_distribute(A, u);
  }
}

void
or_hn_zero(const or_level* A, double* u)
{
  const int B = A->B;
  for (int64_t k = 0; k < A->nhedge; ++k)
    for (int c = 0; c < B; ++c)
      u[A->hnedge[4 * k] * B + c] = 0.0;
  if (A->hn_disc == 1 || A->hn_disc == 3)
    for (int64_t k = 0; k < A->nhface; ++k)
      for (int c = 0; c < B; ++c)
        u[A->hnface[10 * k] * B + c] = 0.0;
}

/* ---------------------------------------------------------- transfers */

static int
cmp_i64(const void* a, const void* b)
{
  int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
  return (x > y) - (x < y);
}

/* MgInterpolatorMatrix::BasicInit (Discretization/Q1/mginterpolatormatrix.cc:
 * 34-121) from the GascoigneMeshTransfer maps: c2f[coarse] = fine; zweier rows
 * [fine, 2 coarse], vierer [fine, 4 coarse], achter [fine, 8 coarse]. A fine
 * node's weight is 1/2, 1/4, 1/8 by the map it is in, else 1. */
int
or_transfer_build(or_transfer* T, int64_t ncoarse, const int64_t* c2f,
                  int64_t nz, const int64_t* zweier, int64_t nv,
                  const int64_t* vierer, int64_t na, const int64_t* achter)
{
  int64_t nfine = -1;
  for (int64_t i = 0; i < ncoarse; ++i)
    nfine = c2f[i] > nfine ? c2f[i] : nfine;
  for (int64_t i = 0; i < nz; ++i)
    nfine = zweier[3 * i] > nfine ? zweier[3 * i] : nfine;
  for (int64_t i = 0; i < nv; ++i)
    nfine = vierer[5 * i] > nfine ? vierer[5 * i] : nfine;
  for (int64_t i = 0; i < na; ++i)
    nfine = achter[9 * i] > nfine ? achter[9 * i] : nfine;
  nfine++;
  T->ncoarse = ncoarse;
  T->nfine = nfine;
  int64_t nent = ncoarse + 2 * nz + 4 * nv + 8 * na;
  double* wfine = (double*)calloc(nfine, sizeof(double));
  int64_t* cntf = (int64_t*)calloc(nfine + 1, sizeof(int64_t));
  int64_t* cntc = (int64_t*)calloc(ncoarse + 1, sizeof(int64_t));
  int64_t* pairs_f = (int64_t*)malloc(sizeof(int64_t) * nent); /* fine */
  int64_t* pairs_c = (int64_t*)malloc(sizeof(int64_t) * nent); /* coarse */
  if (!wfine || !cntf || !cntc || !pairs_f || !pairs_c)
    return -1;
  int64_t e = 0;
  for (int64_t i = 0; i < ncoarse; ++i) {
    pairs_f[e] = c2f[i];
    pairs_c[e++] = i;
    wfine[c2f[i]] = 1.0;
  }
  for (int64_t i = 0; i < nz; ++i)
    for (int q = 0; q < 2; ++q) {
      pairs_f[e] = zweier[3 * i];
      pairs_c[e++] = zweier[3 * i + 1 + q];
      wfine[zweier[3 * i]] = 0.5;
    }
  for (int64_t i = 0; i < nv; ++i)
    for (int q = 0; q < 4; ++q) {
      pairs_f[e] = vierer[5 * i];
      pairs_c[e++] = vierer[5 * i + 1 + q];
      wfine[vierer[5 * i]] = 0.25;
    }
  for (int64_t i = 0; i < na; ++i)
    for (int q = 0; q < 8; ++q) {
      pairs_f[e] = achter[9 * i];
      pairs_c[e++] = achter[9 * i + 1 + q];
      wfine[achter[9 * i]] = 0.125;
    }
  for (int64_t k = 0; k < nent; ++k) {
    cntf[pairs_f[k] + 1]++;
    cntc[pairs_c[k] + 1]++;
  }
  for (int64_t i = 0; i < nfine; ++i)
    cntf[i + 1] += cntf[i];
  for (int64_t i = 0; i < ncoarse; ++i)
    cntc[i + 1] += cntc[i];
  T->p_ptr = (int64_t*)malloc(sizeof(int64_t) * (nfine + 1));
  T->r_ptr = (int64_t*)malloc(sizeof(int64_t) * (ncoarse + 1));
  T->p_col = (int64_t*)malloc(sizeof(int64_t) * nent);
  T->r_col = (int64_t*)malloc(sizeof(int64_t) * nent);
  T->p_w = (double*)malloc(sizeof(double) * nent);
  T->r_w = (double*)malloc(sizeof(double) * nent);
  memcpy(T->p_ptr, cntf, sizeof(int64_t) * (nfine + 1));
  memcpy(T->r_ptr, cntc, sizeof(int64_t) * (ncoarse + 1));
  for (int64_t k = 0; k < nent; ++k) {
    T->p_col[cntf[pairs_f[k]]++] = pairs_c[k];
    T->r_col[cntc[pairs_c[k]]++] = pairs_f[k];
  }
  for (int64_t i = 0; i < nfine; ++i) {
    qsort(T->p_col + T->p_ptr[i], T->p_ptr[i + 1] - T->p_ptr[i],
          sizeof(int64_t), cmp_i64);
    for (int64_t k = T->p_ptr[i]; k < T->p_ptr[i + 1]; ++k)
      T->p_w[k] = wfine[i];
  }
  for (int64_t i = 0; i < ncoarse; ++i) {
    qsort(T->r_col + T->r_ptr[i], T->r_ptr[i + 1] - T->r_ptr[i],
          sizeof(int64_t), cmp_i64);
    for (int64_t k = T->r_ptr[i]; k < T->r_ptr[i + 1]; ++k)
      T->r_w[k] = wfine[T->r_col[k]];
  }
  free(wfine);
  free(cntf);
  free(cntc);
  free(pairs_f);
  free(pairs_c);
  return 0;
}

void
or_transfer_free(or_transfer* T)
{
  free(T->p_ptr);
  free(T->p_col);
  free(T->p_w);
  free(T->r_ptr);
  free(T->r_col);
  free(T->r_w);
  memset(T, 0, sizeof(*T));
}

/* MgInterpolatorMatrix::restrict_zero (mginterpolatormatrix.cc:123-133) */
void
or_restrict_zero(const or_transfer* T, int B, double* uL, const double* ul)
{
  for (int64_t i = 0; i < T->ncoarse; ++i) {
    for (int c = 0; c < B; ++c)
      uL[i * B + c] = 0.0;
    for (int64_t k = T->r_ptr[i]; k < T->r_ptr[i + 1]; ++k)
      for (int c = 0; c < B; ++c)
        uL[i * B + c] += T->r_w[k] * ul[T->r_col[k] * B + c];
  }
}

/* MgInterpolatorMatrix::prolongate_add (mginterpolatormatrix.cc:137-147) */
void
or_prolongate_add(const or_transfer* T, int B, double* ul, const double* uL)
{
  for (int64_t i = 0; i < T->nfine; ++i)
    for (int64_t k = T->p_ptr[i]; k < T->p_ptr[i + 1]; ++k)
      for (int c = 0; c < B; ++c)
        ul[i * B + c] += T->p_w[k] * uL[T->p_col[k] * B + c];
}

/* ---------------------------------------------------------- multigrid */

static int64_t
ndof(const or_mg* M, int l)
{
  return M->L[l].n * M->L[l].B;
}

/* SparseBlockIlu (LinAlg/sparseblockilu.xx): ConstructStructure with the
 * identity order (:72-135; columns of each row ascending), copy_entries
 * (:140-175), compute_ilu (:246-276) with FMatrixBlock's operator*= and
 * submult (LinAlg/fmatrixblock.h:73-93, 174-190) and gauss_jordan on the
 * diagonal blocks. */
static void
or_ilu_factor(const or_level* A, int64_t** pptr, int64_t** pcol, int64_t** pdiag,
              double** pval)
{
  const int B = A->B, B2 = B * B;
  const int64_t n = A->n, nnz = A->rowptr[n];
  int64_t* ptr = (int64_t*)malloc(sizeof(int64_t) * (n + 1));
  int64_t* col = (int64_t*)malloc(sizeof(int64_t) * (nnz > 0 ? nnz : 1));
  int64_t* diag = (int64_t*)malloc(sizeof(int64_t) * n);
  double* v = (double*)malloc(sizeof(double) * (nnz > 0 ? nnz * B2 : 1));
  double tmp[OR_MAXB * OR_MAXB];
  for (int64_t i = 0; i <= n; ++i)
    ptr[i] = A->rowptr[i];
  for (int64_t i = 0; i < n; ++i) {
    /* insertion sort of the row by column (rows are short) */
    const int64_t b = ptr[i], e = ptr[i + 1];
    for (int64_t k = b; k < e; ++k) {
      col[k] = A->col[k];
      memcpy(v + k * B2, A->val + k * B2, sizeof(double) * B2);
    }
    for (int64_t k = b + 1; k < e; ++k) {
      const int64_t c = col[k];
      double blk[OR_MAXB * OR_MAXB];
      memcpy(blk, v + k * B2, sizeof(double) * B2);
      int64_t q = k - 1;
      while (q >= b && col[q] > c) {
        col[q + 1] = col[q];
        memcpy(v + (q + 1) * B2, v + q * B2, sizeof(double) * B2);
        --q;
      }
      col[q + 1] = c;
      memcpy(v + (q + 1) * B2, blk, sizeof(double) * B2);
    }
    diag[i] = -1;
    for (int64_t k = b; k < e; ++k)
      if (col[k] == i)
        diag[i] = k;
  }
  for (int64_t i = 0; i < n; ++i) {
    for (int64_t pk = ptr[i]; pk < diag[i]; ++pk) {
      const int64_t k = col[pk];
      double* a = v + pk * B2;
      const double* dk = v + diag[k] * B2;
      memcpy(tmp, a, sizeof(double) * B2);
      for (int r = 0; r < B; ++r)
        for (int c = 0; c < B; ++c) {
          double acc = 0.0;
          for (int t = 0; t < B; ++t)
            acc += tmp[r * B + t] * dk[t * B + c];
          a[r * B + c] = acc;
        }
      for (int64_t pj = diag[k] + 1; pj < ptr[k + 1]; ++pj) {
        const int64_t j = col[pj];
        for (int64_t ph = ptr[i]; ph < ptr[i + 1]; ++ph) {
          if (col[ph] != j)
            continue;
          double* h = v + ph * B2;
          const double* cj = v + pj * B2;
          for (int r = 0; r < B; ++r)
            for (int c = 0; c < B; ++c)
              for (int t = 0; t < B; ++t)
                h[r * B + c] -= a[r * B + t] * cj[t * B + c];
          break;
        }
      }
    }
    or_gauss_jordan(B, v + diag[i] * B2);
  }
  *pptr = ptr;
  *pcol = col;
  *pdiag = diag;
  *pval = v;
}

/* SparseBlockIlu::solve with the identity order: forward (:202-214), then
 * backward with the inverted diagonal blocks (:217-231; FMatrixBlock::vmult) */
static void
or_ilu_solve(const or_mg* M, int l, double* y)
{
  const or_level* A = &M->L[l];
  const int B = A->B, B2 = B * B;
  const int64_t n = A->n;
  const int64_t *ptr = M->iptr[l], *col = M->icol[l], *diag = M->idiag[l];
  const double* v = M->ival[l];
  for (int64_t i = 1; i < n; ++i)
    for (int64_t pos = ptr[i]; pos < diag[i]; ++pos) {
      const double* m = v + pos * B2;
      for (int r = 0; r < B; ++r)
        for (int c = 0; c < B; ++c)
          y[i * B + r] -= m[r * B + c] * y[col[pos] * B + c];
    }
  for (int64_t i = n - 1; i >= 0; --i) {
    for (int64_t pos = ptr[i + 1] - 1; pos > diag[i]; --pos) {
      const double* m = v + pos * B2;
      for (int r = 0; r < B; ++r)
        for (int c = 0; c < B; ++c)
          y[i * B + r] -= m[r * B + c] * y[col[pos] * B + c];
    }
    double old[OR_MAXB];
    for (int r = 0; r < B; ++r)
      old[r] = y[i * B + r];
    const double* d = v + diag[i] * B2;
    for (int r = 0; r < B; ++r) {
      double acc = 0.0;
      for (int c = 0; c < B; ++c)
        acc += d[r * B + c] * old[c];
      y[i * B + r] = acc;
    }
  }
}

or_mg*
or_mg_create(int nlevels, or_level* L, or_transfer* T, int iterpre,
             int iterpost, int iterexact, double omega, double mgomega,
             char mgtype, int smoother)
{
  or_mg* M = (or_mg*)calloc(1, sizeof(or_mg));
  M->nlevels = nlevels;
  M->L = L;
  M->T = T;
  M->iterpre = iterpre;
  M->iterpost = iterpost;
  M->iterexact = iterexact;
  M->omega = omega;
  M->mgomega = mgomega;
  M->mgtype = mgtype;
  M->u = (double**)calloc(nlevels, sizeof(double*));
  M->b = (double**)calloc(nlevels, sizeof(double*));
  M->v = (double**)calloc(nlevels, sizeof(double*));
  for (int l = 0; l < nlevels; ++l) {
    M->u[l] = (double*)calloc(ndof(M, l), sizeof(double));
    M->b[l] = (double*)calloc(ndof(M, l), sizeof(double));
    M->v[l] = (double*)calloc(ndof(M, l), sizeof(double));
  }
  M->smoother = smoother;
  if (smoother == 1) {
    /* VankaSmoother::ConstructStructure + copy_entries (ComputeIlu,
     * Solver/stdsolver.cc:1547-1573) on every level */
    M->vlu = (double**)calloc(nlevels, sizeof(double*));
    M->vperm = (int**)calloc(nlevels, sizeof(int*));
    int64_t nmax = 0;
    for (int l = 0; l < nlevels; ++l) {
      const or_level* A = &L[l];
      const int64_t m = (int64_t)A->npp * A->B;
      if (A->npatch <= 0 || m > 8 * 27)
        return NULL;
      M->vlu[l] = (double*)malloc(sizeof(double) * A->npatch * m * m);
      M->vperm[l] = (int*)malloc(sizeof(int) * A->npatch * m);
      for (int64_t p = 0; p < A->npatch; ++p)
        or_vanka_factor(A, p, M->vlu[l] + p * m * m, M->vperm[l] + p * m);
      nmax = ndof(M, l) > nmax ? ndof(M, l) : nmax;
    }
    M->vtmp = (double*)malloc(sizeof(double) * nmax);
    M->vcount = (int*)malloc(sizeof(int) * nmax);
  }
  if (smoother == 2) {
    M->iptr = (int64_t**)calloc(nlevels, sizeof(int64_t*));
    M->icol = (int64_t**)calloc(nlevels, sizeof(int64_t*));
    M->idiag = (int64_t**)calloc(nlevels, sizeof(int64_t*));
    M->ival = (double**)calloc(nlevels, sizeof(double*));
    for (int l = 0; l < nlevels; ++l) {
      if (L[l].B > OR_MAXB)
        return NULL;
      or_ilu_factor(&L[l], &M->iptr[l], &M->icol[l], &M->idiag[l], &M->ival[l]);
      for (int64_t i = 0; i < L[l].n; ++i)
        if (M->idiag[l][i] < 0)
          return NULL;
    }
  }
  return M;
}

void
or_mg_free(or_mg* M)
{
  for (int l = 0; l < M->nlevels; ++l) {
    free(M->u[l]);
    free(M->b[l]);
    free(M->v[l]);
  }
  free(M->u);
  free(M->b);
  free(M->v);
  free(M->dlu);
  free(M->dperm);
  if (M->iptr) {
    for (int l = 0; l < M->nlevels; ++l) {
      free(M->iptr[l]);
      free(M->icol[l]);
      free(M->idiag[l]);
      free(M->ival[l]);
    }
    free(M->iptr);
    free(M->icol);
    free(M->idiag);
    free(M->ival);
  }
  if (M->vlu) {
    for (int l = 0; l < M->nlevels; ++l) {
      free(M->vlu[l]);
      free(M->vperm[l]);
    }
    free(M->vlu);
    free(M->vperm);
    free(M->vtmp);
    free(M->vcount);
  }
  free(M);
}

/* StdSolver::MatrixResidual (Solver/stdsolver.cc:783-791): y = b - A x,
 * then SubtractMeanAlgebraic (a no-op without a pressure filter) */
void
or_matrix_residual(const or_level* A, double* y, const double* x,
                   const double* b)
{
  memcpy(y, b, sizeof(double) * A->n * A->B);
  or_bsr_vmult(A, y, x, -1.0);
  or_subtract_mean_algebraic(A, y);
}

/* StdSolver::smooth (Solver/stdsolver.cc:951-986): h = y - A x (filtered);
 * h = D^-1 h (jacobi) or the Vanka solve (ilu with matrixtype vanka);
 * x += omega h; SubtractMean(x). */
void
or_smooth(const or_mg* M, int l, int niter, double* x, const double* y,
          double* h)
{
  const or_level* A = &M->L[l];
  const int64_t n = ndof(M, l);
  for (int it = 0; it < niter; ++it) {
    or_matrix_residual(A, h, x, y);
    if (M->smoother == 2)
      or_ilu_solve(M, l, h);
    else if (M->smoother == 1)
      or_vanka_solve(A, M->vlu[l], M->vperm[l], h, M->vtmp, M->vcount);
    else
      or_jacobi(A, h);
    for (int64_t i = 0; i < n; ++i)
      x[i] += M->omega * h[i];
    or_subtract_mean(A, x);
  }
}

/* The exact coarsest-level solve that StdSolver::smooth_exact runs when the
 * level is a direct level (fewer than ndirect nodes) and UMFPACK is compiled
 * in (Solver/stdsolver.cc:1003-1025, NewMesh :218-222): UmfIlu::Solve gives
 * x = A^-1 y. UMFPACK (a third-party multifrontal sparse LU, not part of the
 * reference tree) is restated as what it computes: a dense LU with partial
 * pivoting of the level's assembled matrix, then the two triangular solves.
 * Returns 0, or -1 when the level is too large (more than 8192 dofs) or a
 * pivot is at most 1e-13 times the largest entry (a singular matrix, e.g. a
 * Stokes level whose pressure is fixed only up to a constant). ndirect <= level-0 nodes turns the
 * direct solve off (the iterexact sweeps run). */
int
or_mg_set_direct(or_mg* M, int ndirect)
{
  free(M->dlu);
  free(M->dperm);
  M->dlu = NULL;
  M->dperm = NULL;
  const or_level* A = &M->L[0];
  if (A->n >= ndirect)
    return 0;
  const int B = A->B, B2 = B * B;
  const int64_t N = ndof(M, 0);
  if (N > 8192)
    return -1;
  double* a = (double*)calloc((size_t)(N * N), sizeof(double));
  int* pv = (int*)malloc(sizeof(int) * N);
  for (int64_t i = 0; i < A->n; ++i)
    for (int64_t k = A->rowptr[i]; k < A->rowptr[i + 1]; ++k)
      for (int r = 0; r < B; ++r)
        for (int q = 0; q < B; ++q)
          a[(i * B + r) * N + A->col[k] * B + q] = A->val[k * B2 + r * B + q];
  double anorm = 0.0;
  for (int64_t i = 0; i < N * N; ++i)
    anorm = fabs(a[i]) > anorm ? fabs(a[i]) : anorm;
  for (int64_t i = 0; i < N; ++i)
    pv[i] = (int)i;
  for (int64_t k = 0; k < N; ++k) {
    int64_t piv = k;
    double best = fabs(a[k * N + k]);
    for (int64_t i = k + 1; i < N; ++i)
      if (fabs(a[i * N + k]) > best) {
        best = fabs(a[i * N + k]);
        piv = i;
      }
    if (best <= 1e-13 * anorm) {
      free(a);
      free(pv);
      return -1;
    }
    if (piv != k) {
      for (int64_t j = 0; j < N; ++j) {
        const double t = a[k * N + j];
        a[k * N + j] = a[piv * N + j];
        a[piv * N + j] = t;
      }
      const int t = pv[k];
      pv[k] = pv[piv];
      pv[piv] = t;
    }
    const double d = a[k * N + k];
    for (int64_t i = k + 1; i < N; ++i) {
      const double f = a[i * N + k] / d;
      a[i * N + k] = f;
      if (f != 0.0)
        for (int64_t j = k + 1; j < N; ++j)
          a[i * N + j] -= f * a[k * N + j];
    }
  }
  M->dlu = a;
  M->dperm = pv;
  return 0;
}

/* x = A^-1 y with the factors of or_mg_set_direct */
void
or_direct_solve(const or_mg* M, double* x, const double* y)
{
  const int64_t N = ndof(M, 0);
  const double* a = M->dlu;
  for (int64_t i = 0; i < N; ++i) {
    double s = y[M->dperm[i]];
    for (int64_t q = 0; q < i; ++q)
      s -= a[i * N + q] * x[q];
    x[i] = s;
  }
  for (int64_t i = N - 1; i >= 0; --i) {
    double s = x[i];
    for (int64_t q = i + 1; q < N; ++q)
      s -= a[i * N + q] * x[q];
    x[i] = s / a[i * N + i];
  }
}

/* StdMultiLevelSolver::mgstep (Solver/stdmultilevelsolver.cc:462-531), the
 * smoothing, residual and transfer steps in the reference's order. The final
 * residual and norms only feed CGInfo and are kept for completeness. */
static void
or_mgstep(or_mg* M, double* res, double* rw, int l, int finelevel,
          int coarselevel, char* p0, char p)
{
  double** u = M->u;
  double** b = M->b;
  double** v = M->v;
  if (l == coarselevel) {
    if (p == 'F')
      *p0 = 'V';
    if (M->dlu && l == 0)
      or_direct_solve(M, u[l], b[l]); /* smooth_exact, direct level */
    else
      or_smooth(M, l, M->iterexact, u[l], b[l], v[l]); /* smooth_exact */
    if (l == finelevel) {
      or_matrix_residual(&M->L[l], v[l], u[l], b[l]);
      res[l] = or_norm(ndof(M, l), v[l]);
    }
  } else {
    or_smooth(M, l, M->iterpre, u[l], b[l], v[l]);
    or_matrix_residual(&M->L[l], v[l], u[l], b[l]);
    or_restrict_zero(&M->T[l - 1], M->L[l].B, b[l - 1], v[l]);
    or_hn_distribute(&M->L[l - 1], b[l - 1]);
    or_dirichlet_zero(&M->L[l - 1], b[l - 1]);
    memset(u[l - 1], 0, sizeof(double) * ndof(M, l - 1));
    int j = (*p0 == 'V') ? 1 : (*p0 == 'W') ? 2 : (*p0 == 'F') ? 3 : 0;
    for (int i = 0; i < j; ++i)
      or_mgstep(M, res, rw, l - 1, finelevel, coarselevel, p0, p);
    if ((l == 0) && (p == 'F'))
      *p0 = 'W';
    rw[l] = or_norm(ndof(M, l - 1), u[l - 1]);
    memset(v[l], 0, sizeof(double) * ndof(M, l));
    or_hn_average(&M->L[l - 1], u[l - 1]);
    or_prolongate_add(&M->T[l - 1], M->L[l].B, v[l], u[l - 1]);
    or_hn_zero(&M->L[l - 1], u[l - 1]);
    or_hn_zero(&M->L[l], v[l]);
    or_dirichlet_zero(&M->L[l], v[l]);
    for (int64_t i = 0; i < ndof(M, l); ++i)
      u[l][i] += M->mgomega * v[l][i];
    or_smooth(M, l, M->iterpost, u[l], b[l], v[l]);
    or_matrix_residual(&M->L[l], v[l], u[l], b[l]);
    res[l] = or_norm(ndof(M, l), v[l]);
  }
}

/* StdMultiLevelSolver::precondition -> LinearMg (Solver/stdmultilevelsolver.cc:
 * 940-952, 411-458) with prec_maxiter = 1: exactly one cycle, started from the
 * current content of x, on right-hand side y. */
void
or_precondition(or_mg* M, double* x, const double* y)
{
  const int fl = M->nlevels - 1;
  const int64_t n = ndof(M, fl);
  double res[64], rw[64];
  memcpy(M->b[fl], y, sizeof(double) * n);
  memcpy(M->u[fl], x, sizeof(double) * n);
  or_matrix_residual(&M->L[fl], M->v[fl], M->u[fl], M->b[fl]);
  res[fl] = or_norm(n, M->v[fl]);
  char p = M->mgtype;
  char p0 = (p == 'F') ? 'W' : p;
  or_mgstep(M, res, rw, fl, fl, 0, &p0, p);
  memcpy(x, M->u[fl], sizeof(double) * n);
}

/* -------------------------------------------------------------- CGInfo */

typedef struct
{
  double tol, globaltol, breaktol;
  int miniter, maxiter;
  int status; /* 0 waiting, 1 running, 2 converged, 3 too many, 4 exploded, 5 diverging */
  double firstresidual, previousresidual, residual, aimedresidual;
  int iteration;
} or_cginfo;

/* CGInfo::check (Common/cginfo.cc:201-255) */
int
or_cginfo_check(or_cginfo* I, double resi)
{
  double res = fabs(resi);
  I->residual = res;
  if (I->status != 1) {
    I->firstresidual = res;
    I->previousresidual = res;
    I->aimedresidual = res * I->tol;
    I->status = 1;
  } else {
    I->previousresidual = res;
  }
  double aim = I->aimedresidual > I->globaltol ? I->aimedresidual : I->globaltol;
  if (I->residual < aim)
    I->status = 2;
  else if (I->iteration >= I->maxiter)
    I->status = 3;
  else if (I->residual > I->breaktol)
    I->status = 4;
  /* "diverging" compares against previousresidual after it was overwritten
   * with res in the running branch, so it can only fire on the first call,
   * where the two are equal: it never fires. */
  I->iteration++;
  if (I->status == 1)
    return 0;
  if (I->iteration < I->miniter)
    return 0;
  return 1;
}

/* ---------------------------------------------------------------- GMRES */

/* GMRES::solve with left preconditioning (LinAlg/gmres.cc:159-230),
 * orthogonalization/reortho_test (:108-135), givens_rotation (:88-104),
 * solution + backward (:234-259, Common/mult.h:130-141), as called by
 * StdMultiLevelSolver::NewtonLinearSolve/Gmres (Solver/stdmultilevelsolver.cc:
 * 646-689): x is zeroed first. Returns `reached` (1 when CGInfo stopped).
 * hist (may be NULL) receives |gamma| per Arnoldi step, at most vmax entries. */
int
or_gmres_solve(or_mg* M, const double* b, double* x, int vmax, double tol,
               double globaltol, int maxiter, int* out_iters, int* out_status,
               double* out_first, double* out_last, double* hist)
{
  const int fl = M->nlevels - 1;
  const or_level* A = &M->L[fl];
  const int64_t n = ndof(M, fl);
  double** mem = (double**)calloc(vmax + 1, sizeof(double*));
  for (int i = 0; i <= vmax; ++i)
    mem[i] = (double*)calloc(n, sizeof(double));
  double* p = (double*)calloc(n, sizeof(double));
  double* H = (double*)calloc((size_t)vmax * (vmax + 1), sizeof(double));
  double* gamma = (double*)calloc(vmax + 1, sizeof(double));
  double* ci = (double*)calloc(vmax, sizeof(double));
  double* si = (double*)calloc(vmax, sizeof(double));
#define Hc(j, i) H[(size_t)(j) * (vmax + 1) + (i)] /* column j = H[j][i] */
  or_cginfo info = { tol, globaltol, 1e15, 0, maxiter, 0, 0, 1, 0, 0, 0 };
  int reached = 0, dim = 0;

  memset(x, 0, sizeof(double) * n);
  /* residualgmres (Solver/stdsolver.cc:742-754): p = b - A x, Dirichlet zero */
  memset(p, 0, sizeof(double) * n);
  or_bsr_vmult(A, p, x, 1.0);
  for (int64_t i = 0; i < n; ++i)
    p[i] = -1.0 * p[i] + 1.0 * b[i];
  or_dirichlet_zero(A, p);
  or_precondition(M, mem[0], p);
  double rho = sqrt(or_dot(n, mem[0], mem[0]));
  if (rho == 0.0) {
    reached = 1;
    goto done;
  }
  gamma[0] = rho;
  {
    double s = 1.0 / rho;
    for (int64_t i = 0; i < n; ++i)
      mem[0][i] = s * mem[0][i];
  }
  while ((dim < vmax - 1) && !reached) {
    dim++;
    int last = dim - 1;
    double* vv = mem[dim];
    memset(p, 0, sizeof(double) * n); /* vmulteq */
    or_bsr_vmult(A, p, mem[last], 1.0);
    or_precondition(M, vv, p);
    double* h = &Hc(last, 0);
    double s;
    for (int pass = 0; pass < 2; ++pass) {
      for (int i = 0; i < dim; ++i) {
        double d = or_dot(n, vv, mem[i]);
        h[i] += d;
        for (int64_t k = 0; k < n; ++k)
          vv[k] += -d * mem[i][k];
      }
      h[dim] = sqrt(or_dot(n, vv, vv));
      s = h[dim];
      double oldnorm = sqrt(or_dot(n, vv, vv));
      double newnorm = oldnorm + 1.e-3 * s;
      if (pass == 1 || oldnorm != newnorm)
        break;
    }
    {
      double inv = 1.0 / s;
      for (int64_t k = 0; k < n; ++k)
        vv[k] = inv * vv[k];
    }
    /* givens_rotation(H[last], last) */
    for (int i = 0; i < last; i++) {
      double dummy = h[i];
      h[i] = ci[i] * dummy + si[i] * h[i + 1];
      h[i + 1] = -si[i] * dummy + ci[i] * h[i + 1];
    }
    double r = 1. / sqrt(h[last] * h[last] + h[last + 1] * h[last + 1]);
    si[last] = h[last + 1] * r;
    ci[last] = h[last] * r;
    h[last] = ci[last] * h[last] + si[last] * h[last + 1];
    gamma[last + 1] = -si[last] * gamma[last];
    gamma[last] *= ci[last];
    rho = fabs(gamma[dim]);
    if (hist)
      hist[dim - 1] = rho;
    reached = or_cginfo_check(&info, rho);
  }
  /* solution: backward substitution on H1 (dim+1 x dim), x += sum h_i v_i */
  {
    double* hs = (double*)calloc(dim > 0 ? dim : 1, sizeof(double));
    for (int i = dim - 1; i >= 0; i--) {
      double s = gamma[i];
      for (int j = i + 1; j < dim; j++)
        s -= hs[j] * Hc(j, i);
      hs[i] = s / Hc(i, i);
    }
    for (int i = 0; i < dim; i++)
      for (int64_t k = 0; k < n; ++k)
        x[k] += hs[i] * mem[i][k];
    free(hs);
  }
done:
  or_subtract_mean(A, x); /* NewtonLinearSolve, Solver/stdmultilevelsolver.cc:671 */
  if (out_iters)
    *out_iters = info.iteration;
  if (out_status)
    *out_status = info.status;
  if (out_first)
    *out_first = info.firstresidual;
  if (out_last)
    *out_last = info.residual;
  for (int i = 0; i <= vmax; ++i)
    free(mem[i]);
  free(mem);
  free(p);
  free(H);
  free(gamma);
  free(ci);
  free(si);
#undef Hc
  return reached;
}
