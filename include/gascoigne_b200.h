/*
 * gascoigne_b200.h - C-ABI of the B200 (sm_100a) linear-solve path for Gascoigne.
 *
 * This is the boundary a Gascoigne host build binds in place of its cuSPARSE
 * backend (cuda/): the drop-in subclasses B200Solver : StdSolver,
 * B200MultiLevelSolver : StdMultiLevelSolver and B200MgInterpolatorNested :
 * MgInterpolatorNested forward their virtual overrides to these functions
 * (gascoignelib_b200/binding/b200solver.h). Plain pointers and sizes only.
 *
 * Conventions
 *  - Every function returns int status: GB_OK (0) or a GB_E* code; the message
 *    of the last failure is gb_last_error_string(ctx). Nothing calls exit().
 *  - Levels are indexed as the reference indexes its solvers: 0 = coarsest,
 *    nlevels-1 = finest (Solver/stdmultilevelsolver.cc:224-231).
 *  - Vectors are node-major interleaved like CompVector (Common/compvector.h:
 *    98-113); matrix blocks are row-major B x B (LinAlg/nodematrix.h:44-48).
 *  - A vector id names one vector on every level, like Gascoigne's Vector name
 *    (Interface/vectorinterface.h:40-81) with per-level GlobalVectors.
 *  - All work is enqueued on the context's CUDA stream; functions that return
 *    a host scalar or copy to host synchronise that stream.
 *  - A context is used by one host thread at a time.
 */
#ifndef GASCOIGNE_B200_H
#define GASCOIGNE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum gb_status
{
  GB_OK = 0,
  GB_EINVAL = 1,    /* bad argument or size */
  GB_ENOMEM = 2,    /* device or host allocation failed */
  GB_ECUDA = 3,     /* CUDA runtime error */
  GB_ENOTCONV = 4,  /* solver stopped without reaching the tolerance */
  GB_ESTATE = 5,    /* call out of order (e.g. no matrix on a level) */
  GB_ETIMEOUT = 6   /* a bounded device wait ran out */
};

enum gb_precision
{
  GB_FP64 = 0,      /* V-cycle values and vectors in FP64 */
  GB_FP32 = 1       /* V-cycle values and vectors in FP32, FP32 accumulation */
};

/* Solver keys, with the reference's defaults where it has them:
 * SolverData (Solver/solverdata.cc:41-55): iterpre 4, iterpost 4, iterexact 10,
 * omega 1; StdMultiLevelSolverData (Solver/stdmultilevelsolverdata.cc:88-100):
 * mgomega 1, mgtype V, gmressize 10; SolverInfos (Solver/solverinfos.cc:89-94):
 * linear_tol 1e-2, linear_globaltol 1e-12, linear_maxiter 10. */
typedef struct gb_params
{
  int iterpre, iterpost, iterexact;
  double omega;      /* Jacobi damping */
  double mgomega;    /* coarse-grid correction weight */
  char mgtype;       /* 'V', 'W' or 'F' */
  int gmressize;     /* Krylov memory: at most gmressize-1 Arnoldi steps */
  double tol;        /* linear_tol (relative) */
  double globaltol;  /* linear_globaltol (absolute) */
  int maxiter;       /* linear_maxiter */
  int smoother;      /* 0: linear_smooth jacobi (block Jacobi); 1: linear_smooth
                        ilu with matrixtype vanka (VankaSmoother); 2: linear_smooth
                        ilu with matrixtype block (SparseBlockIlu in the
                        matrix's own node order) */
  int ndirect;       /* ndirect (Solver/stdsolver.cc:92,218-222,1003-1025): when
                        level 0 has fewer nodes, smooth_exact there is an exact
                        solve (the reference's UMFPACK branch) with the FP64
                        inverse of level 0's operator; 0 keeps the iterexact
                        sweeps (the reference built without UMFPACK) */
} gb_params;

typedef struct gb_solve_info
{
  int iterations;        /* Arnoldi steps (CGInfo iteration count) */
  int status;            /* 0 waiting 1 running 2 converged 3 too many iterations
                            4 exploded */
  int restarts;          /* refinement cycles (flexible solver), 0 otherwise */
  double firstresidual;  /* CGInfo first residual */
  double residual;       /* last residual estimate */
  double true_residual;  /* ||b - A x||_2 in FP64 after the solve */
  double rhs_norm;       /* ||b||_2 */
  int kernel_launches;   /* kernels this call launched */
  double device_ms;      /* CUDA-event time of the call on the context stream */
} gb_solve_info;

typedef struct gb_ctx gb_ctx;

/* ---- context -------------------------------------------------------------
 * Replaces the handle set-up of CudaSolver::CudaSolver (cuda/cudasolver.cc:
 * 25-33) and check_cuda.h's abort-on-error (cuda/check_cuda.h:28-67). */
int gb_ctx_create(gb_ctx** ctx, int device);
int gb_ctx_destroy(gb_ctx* ctx);
const char* gb_last_error_string(const gb_ctx* ctx);
int gb_ctx_synchronize(gb_ctx* ctx);
/* Solver keys; replaces the ParamFile reads listed at gb_params. */
int gb_set_params(gb_ctx* ctx, const gb_params* p);
int gb_get_params(const gb_ctx* ctx, gb_params* p);
/* Number of multigrid levels; replaces StdMultiLevelSolver::NewSolvers
 * (Solver/stdmultilevelsolver.cc:210-234). Drops all level data. */
int gb_set_nlevels(gb_ctx* ctx, int nlevels);

/* ---- level data ----------------------------------------------------------
 * Uploads the assembled block-CSR matrix of one level: SparseBlockMatrix
 * <FMatrixBlock<B>>::mat() with its ColumnDiagStencil start/col/diag
 * (LinAlg/sparseblockmatrix.h:84, LinAlg/columnstencil.h:57-60,
 * LinAlg/columndiagstencil.h:54-57). Replaces CudaSolver::AssembleMatrix's
 * CudaCSRMatrixInterface upload and get_inverse_diagonal (cuda/cudasolver.cc:
 * 115-128, cuda/cudacsrmatrixinterface.cc:119-141,176-230). B = 1..4
 * components per node (ncomp; Stokes in 2D is B = 3). Rows keep their column
 * order; FP64 and FP32 copies are kept. */
int gb_level_set_matrix(gb_ctx* ctx, int level, int64_t n, int B,
                        const int64_t* rowptr, const int64_t* col,
                        const int64_t* diag, const double* val);
/* Strong-Dirichlet node list of a level with its component mask (bit c set:
 * component c). Replaces CudaSolver::SetProblem's Dirichlet matrix
 * (cuda/cudasolver.cc:271-297) and CGDisc::StrongDirichletVectorZero
 * (DofHandler/cgdisc.h:1162-1179). */
int gb_level_set_dirichlet(gb_ctx* ctx, int level, int64_t nnodes,
                           const int64_t* nodes, int comp_mask);
/* The same with one component mask per node: the union over the Dirichlet
 * colours of each colour's components (DirichletData::components_on_color,
 * CGDisc::StrongDirichletVectorZero loops colours, DofHandler/cgdisc.h:
 * 1162-1179). Nodes must be distinct. */
int gb_level_set_dirichlet_masks(gb_ctx* ctx, int level, int64_t nnodes,
                                 const int64_t* nodes, const int* comp_masks);
/* Mesh-transfer maps between coarse level `level` and level+1, as
 * GascoigneMeshTransfer holds them (Mesh/gascoignemeshtransfer.h:48-51):
 * c2f[ncoarse]; zweier rows [fine, c0, c1]; vierer [fine, c0..c3]; achter
 * [fine, c0..c7]. Replaces CudaMgInterpolatorNested::BasicInit
 * (cuda/cudamgintepolatornested.cc:21-25) and its R/P SimpleMatrix build. */
int gb_level_set_transfer(gb_ctx* ctx, int level, int64_t ncoarse,
                          const int64_t* c2f, int64_t nz, const int64_t* zweier,
                          int64_t nv, const int64_t* vierer, int64_t na,
                          const int64_t* achter);
int gb_level_size(const gb_ctx* ctx, int level, int64_t* n, int* B,
                  int64_t* nnzb);
/* Vanka patches of a level: npatch lists of npp node indices (npp <= 27), as
 * DofHandler::GetElement(2, p) returns them (DofHandler/dofhandler.h:389-396;
 * patchlevel 2 in VankaSmoother::ConstructStructure,
 * LinAlg/vankasmoother.cc:7-63). The patch matrices are copied from the
 * level matrix and LU-factorised (copy_entries_sparseblockmatrix, :65-113)
 * when a solve first needs them after a matrix or patch upload. */
int gb_level_set_patches(gb_ctx* ctx, int level, int64_t npatch, int npp,
                         const int64_t* patches);
/* The inverses of a level's patch matrices, FP64, [patch][j][i] (column j of
 * the inverse of patch p at (p * M + j) * M, M = npp * B), formed on the device
 * from the level's current values by the partial-pivot LU of
 * VankaSmoother::copy_entries_sparseblockmatrix and its solves
 * (LinAlg/vankasmoother.cc:65-113,192-237) when they are stale. */
int gb_level_get_vanka_inverse(gb_ctx* ctx, int level, double* host, int64_t len);
/* Hanging nodes of a level as the mesh's HangingIndexHandler holds them
 * (Mesh/hangingindexhandler.h:40,65): nedge rows [node, 3 parents] (hnq2) and,
 * in 3D, nface rows [node, 9 parents] (hnq2face), nodes ascending, and the
 * discretisation whose HNStructure acts on them (disc 0 Q12d, 1 Q13d, 2 Q22d,
 * 3 Q23d: Discretization/Q1/hnstructureq12d.cc, hnstructureq13d.cc,
 * Discretization/Q2/hnstructureq22d.cc, hnstructureq23d.cc; CGDisc::ReInit,
 * DofHandler/cgdisc.cc:24-50). Replaces CudaSolver::NewMesh's HN matrices
 * (cuda/cudasolver.cc:161-247). The cycle then applies HNDistribute after
 * each restriction, HNAverage before each prolongation and HNZero to the
 * prolonged correction (Solver/stdmultilevelsolver.cc:492-517). */
int gb_level_set_hn(gb_ctx* ctx, int level, int disc, int64_t nedge,
                    const int64_t* edges, int64_t nface, const int64_t* faces);
/* StdSolver::HNAverage / HNDistribute / HNZero (Solver/stdsolver.h:365-367),
 * CudaSolver's HN* overrides (cuda/cudasolver.cc:449-489). */
int gb_hn_average(gb_ctx* ctx, int level, int id);
int gb_hn_distribute(gb_ctx* ctx, int level, int id);
int gb_hn_zero(gb_ctx* ctx, int level, int id);
/* Pressure filter of a level (PressureFilter, Discretization/Q1/
 * pressurefilter.h:31-54; set up by StdSolver::NewMesh ->
 * CGDisc::InitFilter, Solver/stdsolver.cc:214-227, DofHandler/cgdisc.h:
 * 1061-1090): the filtered components (bit mask, 0 = off), the weights (per
 * node, the integral of its basis function), the domain size and the number of
 * hanging nodes. */
int gb_level_set_pfilter(gb_ctx* ctx, int level, int comp_mask,
                         const double* weights, double domain, int64_t nhanging);

/* ---- vectors -------------------------------------------------------------
 * Replaces CudaVectorInterface (cuda/cudavectorinterface.h:33-83) and
 * StdSolver's vector ops (Solver/stdsolver.cc:685-688,1775-1810). */
int gb_vec_create(gb_ctx* ctx, int* id);
int gb_vec_free(gb_ctx* ctx, int id);
int gb_vec_upload(gb_ctx* ctx, int level, int id, const double* host,
                  int64_t len);
int gb_vec_download(gb_ctx* ctx, int level, int id, double* host, int64_t len);
int gb_vec_zero(gb_ctx* ctx, int level, int id);                   /* Zero */
int gb_vec_equ(gb_ctx* ctx, int level, int dst, double s, int src); /* Equ */
int gb_vec_add(gb_ctx* ctx, int level, int dst, double s, int src); /* Add */
int gb_vec_norm(gb_ctx* ctx, int level, int id, double* out);       /* Norm */
int gb_vec_dot(gb_ctx* ctx, int level, int a, int b, double* out); /* ScalarProduct */

/* ---- level operators (StdSolver / CudaSolver overrides) ------------------ */
/* y += d A x: StdSolver::vmult (Solver/stdsolver.cc:757-764),
 * CudaSolver::vmult (cuda/cudasolver.cc:301-320). */
int gb_vmult(gb_ctx* ctx, int level, int y, int x, double d);
/* y = d A x: StdSolver::vmulteq (Solver/stdsolver.cc:768-778). */
int gb_vmulteq(gb_ctx* ctx, int level, int y, int x, double d);
/* y += d A^T x: the transposed operator SparseBlockMatrix::transpose builds
 * (LinAlg/sparseblockmatrix.xx:478-491), applied without transposing. */
int gb_vmult_transpose(gb_ctx* ctx, int level, int y, int x, double d);
/* y = b - A x, then SubtractMeanAlgebraic(y): StdSolver::MatrixResidual
 * (Solver/stdsolver.cc:783-791). */
int gb_matrix_residual(gb_ctx* ctx, int level, int y, int x, int b);
/* y = b - A x, Dirichlet-zeroed: StdSolver::residualgmres
 * (Solver/stdsolver.cc:742-754). */
int gb_residualgmres(gb_ctx* ctx, int level, int y, int x, int b);
/* niter damped-Jacobi sweeps x += omega D^-1 (y - A x): StdSolver::smooth with
 * linear_smooth jacobi (Solver/stdsolver.cc:951-986), CudaSolver::smooth
 * (cuda/cudasolver.cc:345-374). h is work space, as in the reference. With a
 * pressure filter each sweep filters the residual (SubtractMeanAlgebraic)
 * and x (SubtractMean), as the reference does. */
int gb_smooth_jacobi(gb_ctx* ctx, int level, int niter, int x, int y, int h);
/* The same with linear_smooth ilu on matrixtype vanka: each sweep
 * h = VankaSmoother::solve(y - A x) (LinAlg/vankasmoother.cc:192-237),
 * x += omega h. Needs the level's patches. */
int gb_smooth_vanka(gb_ctx* ctx, int level, int niter, int x, int y, int h);
/* StdSolver::smooth with the smoother of gb_params.smoother. */
int gb_smooth(gb_ctx* ctx, int level, int niter, int x, int y, int h);
/* StdSolver::SubtractMean / SubtractMeanAlgebraic (Solver/stdsolver.cc:
 * 1736-1762): remove the weighted (integral) or plain mean of every filtered
 * component; no-ops without a pressure filter. */
int gb_subtract_mean(gb_ctx* ctx, int level, int id);
int gb_subtract_mean_algebraic(gb_ctx* ctx, int level, int id);
/* u = 0 on Dirichlet dofs: StdSolver::SetBoundaryVectorZero
 * (Solver/stdsolver.cc:795-812). */
int gb_dirichlet_zero(gb_ctx* ctx, int level, int id);
/* Per-node inverse diagonal blocks (row-major B x B, FP64) as
 * SparseBlockMatrix::Jacobi forms them (LinAlg/sparseblockmatrix.xx:47-56,
 * NodeMatrix::gauss_jordan LinAlg/nodematrix.h:159-213). */
int gb_level_get_inverse_diagonal(gb_ctx* ctx, int level, double* host,
                                  int64_t len);

/* ---- transfers (MgInterpolatorInterface overrides) ------------------------
 * coarse = R fine: MgInterpolatorMatrix/Nested::restrict_zero
 * (Discretization/Q1/mginterpolatormatrix.cc:123-133,
 *  cuda/cudamgintepolatornested.cc:131-139). */
int gb_restrict_zero(gb_ctx* ctx, int level, int coarse_id, int fine_id);
/* fine += P coarse: prolongate_add (mginterpolatormatrix.cc:137-147,
 * cuda/cudamgintepolatornested.cc:160-167). */
int gb_prolongate_add(gb_ctx* ctx, int level, int fine_id, int coarse_id);

/* ---- multilevel solver (StdMultiLevelSolver / CudaMultiLevelSolver) ------- */
/* One multigrid cycle on the finest level, started from the current content
 * of x, right-hand side y: StdMultiLevelSolver::precondition -> LinearMg ->
 * mgstep with prec_maxiter 1 (Solver/stdmultilevelsolver.cc:411-531,940-952;
 * cuda/cudamultilevelsolver.cc:107-246). */
int gb_precondition(gb_ctx* ctx, int x, int y, int precision);
/* StdMultiLevelSolver::Gmres -> GMRES::solve (Solver/stdmultilevelsolver.cc:
 * 677-689, LinAlg/gmres.cc:159-230): x zeroed, left-preconditioned MGS-GMRES,
 * one cycle of at most gmressize-1 steps, CGInfo stopping rule
 * (Common/cginfo.cc:201-255). FP64 throughout (the parity variant). */
int gb_gmres(gb_ctx* ctx, int x, int b, gb_solve_info* info);
/* Flexible (right-preconditioned) GMRES in FP64 with the multigrid cycle run
 * in `precision`, restarted as iterative refinement until the true relative
 * residual ||b - A x|| / ||b|| <= tol (or maxiter Arnoldi steps). No
 * counterpart in the reference; it replaces the same Gmres call. */
int gb_fgmres(gb_ctx* ctx, int x, int b, int precision, gb_solve_info* info);
/* End-to-end call with host buffers: uploads b, solves (method 0: gb_gmres,
 * 1: gb_fgmres FP64 cycle, 2: gb_fgmres FP32 cycle), downloads x. */
int gb_solve_host(gb_ctx* ctx, int method, const double* b, double* x,
                  int64_t len, gb_solve_info* info);

/* ---- adjoint (dual) path ---------------------------------------------------
 * gb_set_operator(ctx, 1) makes every level operator A^T for all following
 * calls (vmult, residuals, smoothers, the cycle, both GMRES forms;
 * gb_vmult_transpose then applies A), 0 switches back to A. It stands in for
 * StdMultiLevelSolver::AssembleDualMatrix (Solver/stdmultilevelsolver.cc:
 * 920-926 -> Solver/stdsolver.cc:1815-1834: assemble, transpose, Dirichlet
 * rows only) without re-uploading: A^T is built once per level from the
 * uploaded matrix, keeping its sparsity pattern when that is structurally
 * symmetric (values swapped as SparseBlockMatrix::transpose,
 * LinAlg/sparseblockmatrix.xx:478-491). The transfers stay those of the
 * forward hierarchy (restriction R = P^T, prolongation P), as the reference's
 * dual solve uses them. Solutions equal the reference's dual solutions for
 * right-hand sides that are zero on Dirichlet dofs (the reference zeroes them,
 * StdSolver::SetBoundaryVectorZero). */
int gb_set_operator(gb_ctx* ctx, int transposed);
int gb_get_operator(const gb_ctx* ctx, int* transposed);
/* A^T x = b with the reference-semantics solver (as gb_gmres) or the
 * flexible solver (as gb_fgmres); the operator setting is restored after. */
int gb_adjoint_gmres(gb_ctx* ctx, int x, int b, gb_solve_info* info);
int gb_adjoint_fgmres(gb_ctx* ctx, int x, int b, int precision, gb_solve_info* info);
/* Cells of `level` for the coefficient gradient: cell c has nodes
 * cell_nodes[c*nloc .. c*nloc+nloc-1] (int64) and element matrix
 * kappa_c * cell_scale[c] * kloc (kloc: nloc x nloc doubles, row-major, row =
 * test function, column = trial function; cell_scale NULL means 1), the
 * element assembly of an equation with a per-cell coefficient
 * (DofHandler/cgdisc.h:599-635, Interface/equation.h:104,
 * Interface/application.h:69). nloc <= 32. */
int gb_level_set_cells(gb_ctx* ctx, int level, int64_t ncells, int nloc,
                       const int64_t* cell_nodes, const double* kloc,
                       const double* cell_scale);
/* grad[c] = -cell_scale[c] * lam_c^T kloc u_c over the cells of `level`, with
 * u and lam (vector ids) read as 0 on Dirichlet dofs: dJ/dkappa_c for
 * J(u(kappa)) when lam solves A^T lam = dJ/du (gb_adjoint_*), since
 * dA/dkappa_c is the cell matrix restricted to the non-Dirichlet dofs.
 * grad: host array of ncells doubles or NULL. No counterpart in the reference
 * (StdSolver::AdjointForm aborts, Solver/stdsolver.cc:1080). */
int gb_coeff_gradient(gb_ctx* ctx, int level, int u, int lam, double* grad,
                      int64_t ncells);
/* (grad may be NULL: the gradient is computed and kept on the device, nothing
 * is copied and the call does not wait for the GPU.)
 * A quadratic functional J(u) = u^T M u over the cells of gb_level_set_cells,
 * M = sum over cells of cell_scale[c] * mloc (nloc x nloc, row-major; NULL
 * scale means 1), assembled into the level matrix's sparsity pattern; with
 * the Q1 element mass matrix this is J = integral of u^2, the reference's
 * DomainFunctional for it (Interface/domainfunctional.h:42-64).
 * gb_functional computes J (J may be NULL: not read back) and g = dJ/du =
 * 2 M u with g = 0 on Dirichlet dofs, the dual right-hand side of
 * gb_adjoint_*. No counterpart in the reference's GPU backend. */
int gb_level_set_functional(gb_ctx* ctx, int level, const double* mloc,
                            const double* cell_scale);
int gb_functional(gb_ctx* ctx, int level, int u, int g, double* J);
/* Device-side assembly of the scalar Q1 equation -div(kappa grad u) +
 * beta . grad u with one coefficient kappa per cell, into the sparsity
 * pattern of the level's matrix (CGDisc::Matrix, DofHandler/cgdisc.h:599-635,
 * with ElementIntegrator::Matrix, DofHandler/elementintegrator.xx:350-395,
 * Gauss formulas QuadGauss4 / HexGauss8, DofHandler/elementintegrator.h:
 * 214-222; strong Dirichlet rows and columns as SparseBlockMatrix::dirichlet,
 * LinAlg/sparseblockmatrix.xx:207-218). No counterpart on the reference's GPU,
 * which assembles on the host and uploads (cuda/cudacsrmatrixinterface.cc:
 * 176-230).
 * gb_level_set_mesh: the level's quadrilateral (dim 2) or hexahedral (dim 3)
 * cells, cell c with nodes cell_nodes[c*2^dim + a], local node a at the
 * reference-cell corner (a & 1, a >> 1 & 1, a >> 2 & 1); node coordinates
 * coords[node*dim + d]; above level 0, parent[c] = the cell of level - 1 that
 * contains cell c (for gb_assemble_levels). The level's matrix (gb_level_set_
 * matrix, block size 1, its Dirichlet dofs and its hanging nodes,
 * gb_level_set_hn) must be set first: every pair of condensed nodes of a cell
 * must be in its pattern. Setting the matrix or the hanging nodes again drops
 * the mesh.
 * Hanging nodes: a cell lists its own nodes, hanging ones included; the
 * element matrix of a cell with hanging nodes is condensed on the device
 * (CGDisc::LocalToGlobal, DofHandler/cgdisc.h:354-364, with
 * HNStructureQ12d/Q13d/Q22d/Q23d::CondenseHanging, Discretization/Q1/
 * hnstructureq12d.cc:129-158, hnstructureq13d.cc:275-438, Discretization/Q2/
 * hnstructureq22d.cc:84-110, hnstructureq23d.cc:161-378): edge nodes, then
 * face nodes, each gives way to the one parent the cell lacks, the parents it
 * holds take the weighted row and column; the hanging rows keep a unit
 * diagonal (HNStructure::MatrixDiag, DofHandler/cgdisc.h:634). A cell that
 * lacks more than one parent of a hanging node, or none, is an error. */
int gb_level_set_mesh(gb_ctx* ctx, int level, int dim, int64_t ncells,
                      const int64_t* cell_nodes, const double* coords,
                      const int64_t* parent);
/* The same for elements of degree 1 (Q1, as gb_level_set_mesh) or 2 (CGQ2:
 * 3^dim nodes per element on a patch of 2^dim cells, local node
 * a = a_x + 3 a_y + 9 a_z at the reference coordinates (a_d / 2); integrated
 * with QuadGauss9 / HexGauss27 as LineGauss3 states its points and weights,
 * Discretization/Q1/integrationformula1d.cc:82-92; kappa per element, parents
 * = the element of level - 1 that contains it). degree = 3: the same patches
 * with the Q1 functions of their cells (CGQ1Patch / CGQ1Lps: BaseQ12dPatch /
 * BaseQ13dPatch, Discretization/Q2/baseq1patch.h; QuadGauss4 / HexGauss8 in
 * every cell, PatchFormula2d/3d, Discretization/Q2/patchintegrationformula.xx:
 * 55-83); the matrix equals the Q1 cells' up to rounding, and LPS needs it. */
int gb_level_set_mesh_degree(gb_ctx* ctx, int level, int dim, int degree,
                             int64_t ncells, const int64_t* cell_nodes,
                             const double* coords, const int64_t* parent);
/* Local projection stabilisation of the convection in the following device
 * assemblies of patch levels (degree 2: CGQ2Lps, degree 3: CGQ1Lps;
 * ElementLpsIntegrator::Matrix,
 * DofHandler/elementlpsintegrator.h:168-211, with the projection of :66-110):
 * at every Gauss point h = |J|^(1/dim) and
 * delta = sdelta0 / (xeta0 kappa / h^2 + (|beta| + 1e-6) / h) as
 * LpsStabilization::ConvectionDiffusion computes it
 * (Problems/lpsstabilization.cc, kappa the element's coefficient), and the
 * element matrix gains delta (beta . grad N_i)(beta . grad N_j) w |J| over the
 * projected functions N (a corner node's function replaced by minus its
 * patch-quarter neighbours weighted 1/2, 1/4, 1/8). sdelta0 = 0 turns it off
 * (the default); the reference's default xeta0 is 6. Only patch levels
 * (degree 2 or 3) with a nonzero beta are affected; a level of Q1 cells
 * assembled with it on is an error. */
int gb_set_assembly_lps(gb_ctx* ctx, double sdelta0, double xeta0);
/* Assembles the level's matrix (FP64 and FP32 values, block-diagonal inverse)
 * from kappa (ncells doubles; where = 0: host memory, 1: device memory,
 * copied on the context's stream (gb_ctx_get_stream), so writes to it on other
 * streams must be complete and it must stay valid until that copy ran) and
 * beta (dim doubles in host memory, NULL for none): element matrices at the
 * Gauss points, summed per matrix entry in ascending cell order, then the
 * Dirichlet rows (identity) and columns (zero). */
int gb_assemble(gb_ctx* ctx, int level, const double* kappa, int where,
                const double* beta);
/* gb_assemble on the finest level from kappa, then on each coarser level from
 * the mean of its cells' children (summed in ascending child order): the
 * coefficient of a coarse cell as the test harness's reference runs define it. */
int gb_assemble_levels(gb_ctx* ctx, const double* kappa, int where,
                       const double* beta);
/* The level's cell coefficients last used by gb_assemble(_levels) (host
 * array of ncells doubles). */
int gb_level_get_kappa(gb_ctx* ctx, int level, double* kappa);
/* The level's current FP64 matrix values in the order of the pattern given to
 * gb_level_set_matrix (nnzb * B * B doubles, host array): the uploaded values,
 * or those of the last device assembly; blocks row-major as NodeMatrix stores
 * them (LinAlg/nodematrix.h:44-48). */
int gb_level_get_values(gb_ctx* ctx, int level, double* val);
/* StdSolver::Form (Solver/stdsolver.cc:1041-1063 -> CGDisc::Form,
 * DofHandler/cgdisc.h:415-450) of the equation last assembled on the level
 * (gb_assemble: its kappa, beta and LPS): y += d * sum over cells of the
 * element residuals of x, summed per node in ascending cell order (Q1 cells:
 * matrix-free; patch elements: the element matrices times the local values).
 * On a level with hanging nodes x is HNAverage'd first and HNZero'd after, and
 * y is HNDistribute'd, as the reference's Form does (x is changed the same
 * way). Vectors are level vector ids. */
int gb_form(gb_ctx* ctx, int level, int y, int x, double d);
/* StdMultiLevelSolver::NewtonResidual (Solver/stdmultilevelsolver.cc:609-623)
 * on the finest level: y = b - Form(x), zero on the Dirichlet dofs; *norm (may
 * be NULL) = NewtonNorm(y) = max |y_i| (StdSolver::NewtonNorm,
 * Solver/stdsolver.cc:693-696). No pressure filter. */
int gb_newton_residual(gb_ctx* ctx, int y, int x, int b, double* norm);
/* Solution files of Common/backup.cc. binary = 0: WriteBackUp's text format
 * (".bup": "n ncomp", then per node the ncomp values as %.16e, then
 * "BackUpEnd"); binary = 1: WriteBackUpBinary's (".bip": "ncomp n", "[", the
 * raw doubles, "]", "BackUpEnd"). path is the whole file name (the reference
 * appends the suffix to its base name). The file must hold the level's node
 * count and block size. Reading with add = 1 adds the file's values to the
 * vector (ReadBackUp), add = 0 replaces them (ReadBackUpResize on a vector of
 * the right size, ReadBackUpBinary). */
int gb_vec_write_backup(gb_ctx* ctx, int level, int id, const char* path, int binary);
int gb_vec_read_backup(gb_ctx* ctx, int level, int id, const char* path, int binary,
                       int add);
/* The vector as the reference's VTK file (StdSolver::Visu -> CGDisc::VisuVtk,
 * DofHandler/cgdisc.h:136-158, and Visualization::vtk,
 * Discretization/Q1/vtk.cc:29-244): <name>.<step as %05d>.vtk, legacy ASCII
 * unstructured grid with the level's nodes (coords[node*dim + d]) and the
 * mesh's cells (ncells x nodes_per_cell node indices in the mesh's vertex
 * order: counterclockwise quads, hexes bottom face then top face; VTK cell
 * types 9 / 12), the given time and title in the header, and one scalar per
 * component named u000, u001, ... (the names of a problem without a
 * ComponentInformation of its own). Numbers are printed as a C++ stream prints
 * them by default (6 significant digits). On a level with hanging nodes the
 * written values are HNAverage'd; the vector itself is not changed (the
 * reference averages in place and zeroes the hanging values after). */
int gb_vec_write_vtk(gb_ctx* ctx, int level, int id, const char* name, int step, int dim,
                     int64_t ncells, int nodes_per_cell, const int64_t* cell_nodes,
                     const double* coords, double time, const char* title);
/* The context's CUDA stream (a cudaStream_t): every gb_* call enqueues its
 * work there, so callers can order their own work or record events on it. */
int gb_ctx_get_stream(const gb_ctx* ctx, void** stream);

/* ---- instrumentation ------------------------------------------------------
 * Per-kernel-class device time of the last gb_* solve call when timing is on
 * (CUDA events on the context stream); replaces GlobalTimer's vmult/smooth
 * labels (Common/stopwatch.h:143-270) for the device path. */
int gb_set_timing(gb_ctx* ctx, int on);
/* Per-kernel device times accumulated since gb_set_timing(ctx, 1), as JSON
 * {"kernel name": [launches, total ms], ...}; kernels inside a CUDA graph are
 * not timed individually (run the flexible solver with GB_GRAPH=0 for that). */
int gb_get_kernel_times(gb_ctx* ctx, char* buf, int64_t len);
int gb_get_kernel_count(const gb_ctx* ctx, int64_t* launches);
/* Times `reps` launches of the SpMV y = A x of `level` in `precision` with
 * CUDA events around each launch. flush_l2 between launches: 0 none, 1 write
 * a 256 MB buffer (leaves the L2 full of dirty lines), 2 read a 256 MB buffer
 * (leaves clean lines). Returns the average launch time (ms) and the
 * algorithmic bytes per launch. */
int gb_bench_spmv(gb_ctx* ctx, int level, int precision, int reps,
                  int flush_l2, double* ms_per_launch, double* bytes_per_launch);

/* The same for one smoothing step of a level, the kernel that dominates the
 * multigrid cycle: with gb_params.smoother 1 (Vanka) on a level with patches,
 * the patch solves with the inverted patch matrices and the averaging gather
 * (algorithmic bytes: inverses, patch lists, gathered residual, patch
 * solutions written and read, node map, u read and written); otherwise one
 * fused damped-Jacobi sweep of a scalar level (out = u + omega D^-1 (b - A u),
 * Dirichlet rows kept; the SpMV's bytes plus b, D^-1 and the new iterate). */
int gb_bench_sweep(gb_ctx* ctx, int level, int precision, int reps,
                   int flush_l2, double* ms_per_launch, double* bytes_per_launch);
/* ---- failure detection ------------------------------------------------------
 * The reference aborts on CUDA errors (cuda/check_cuda.h:28-67); this library
 * returns codes. gb_set_wait_limit bounds every device-side wait (the grid
 * barriers of the multi-CTA cycle, GB_MID=1) to wait_ns nanoseconds (default
 * 1 s): a barrier that runs out sets an error flag, the kernel finishes
 * without waiting further, and the call returns GB_ETIMEOUT with the context
 * still usable. phantoms > 0 makes every such barrier wait for that many CTAs
 * that do not exist, so that its wait runs out (for tests; 0 in normal use).
 * gb_debug_fail_alloc(k): the k-th device allocation from now on fails as an
 * out-of-memory cudaMalloc does (host-side fault injection for tests of the
 * GB_ENOMEM path; 0 turns it off). */
int gb_set_wait_limit(gb_ctx* ctx, uint64_t wait_ns, int phantoms);
int gb_debug_fail_alloc(int64_t nth);

/* The compute capability the library's kernels were compiled for, read at run
 * time from a kernel's attributes on the current device (cudaFuncGetAttributes:
 * binaryVersion, ptxVersion; 100 for sm_100a). Needs a device. */
int gb_kernel_arch(int* binary_version, int* ptx_version);

/* ---- allocation-free dot product -----------------------------------------
 * No counterpart in the reference. For callers that cannot allocate device
 * memory once they run: an application that hands all device memory to its
 * own pool allocator at start-up (a larger simulation code or framework that
 * owns the GPU), where a cudaMalloc in the middle of a solve fails or splits
 * the pool, and latency-critical loops that cannot afford the device-wide
 * synchronisation a cudaMalloc / cudaFree pair implies.
 * Computes *out = <a, b> over n doubles; a, b and out are device pointers
 * the caller owns; work is enqueued on `stream` (a cudaStream_t, NULL for the
 * default stream). It allocates nothing: its reduction scratch is a
 * file-scope device array of 4096 partial sums (32 KiB) that every GPU which
 * loads this library keeps until the process exits, so n is limited to
 * 4096 * 2048 = 8,388,608; larger n returns GB_EINVAL.
 * The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress, with that device current) and keeps it for the life
 * of the process. The kept address does not survive cudaDeviceReset: a caller
 * that resets a device must not call this function on it again in the same
 * process.
 * The function makes CUDA runtime calls, so it must not be called from a CUDA
 * host function (cudaLaunchHostFunc, stream callbacks). Calls share the
 * array, and each call clears its ticket before use: two calls that overlap
 * on the GPU (other streams, other host threads) race and give wrong sums.
 * An error that an earlier launch of the caller left pending is reported as
 * GB_ECUDA before anything is enqueued, and is not cleared. Same
 * deterministic reduction as gb_vec_dot; for n <= 606,208 the two use the
 * same partition and return the same bits. */
int gb_dot_noalloc(const double* a, const double* b, int64_t n, double* out,
                   void* stream);

#ifdef __cplusplus
}
#endif

#endif
