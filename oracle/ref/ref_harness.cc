// Oracle harness (test infrastructure, never shipped): drives the reference's own
// FP64 CPU multilevel solver on a seeded synthetic problem and writes what it did.
//
// It builds the problem through the reference's public classes only:
//   MeshAgent (Mesh/meshagent.cc:361-404) on a generated unit square/cube .inp,
//   StdMultiLevelSolver::ReInit/SetProblem/ReInitMatrix/AssembleMatrix/ComputeIlu
//   (Solver/stdmultilevelsolver.cc:152-309,762-790), and
//   StdMultiLevelSolver::NewtonLinearSolve -> Gmres -> GMRES::solve + LinearMg
//   (Solver/stdmultilevelsolver.cc:646-689, LinAlg/gmres.cc:159-230).
// The equation is -div(kappa grad u) + beta . grad u = f with kappa piecewise
// constant per cell
// (per finest cell from a file; a coarse cell takes the mean of its 2^dim
// children, summed in lexicographic child order) and a constant convection
// vector beta (key conv=bx,by[,bz]; default 0, which leaves the operator
// symmetric), assembled by the reference's
// CGDisc with its own Q1 element integrator (HexGauss8 / QuadGauss4,
// DofHandler/elementintegrator.h:215-222). Dirichlet data: u = 0 on the whole
// boundary (colour 1). The right-hand side is a nodal vector read from a file
// (lexicographic node order) and copied into the finest-level vector f, then
// zeroed at Dirichlet nodes (StdSolver::SetBoundaryVectorZero).
//
// With problem=stokes the equation is instead the Stokes system in the
// reference's NavierStokes component order (0 = p, 1..dim = velocity):
// -visc Laplace v + grad p = f, div v + stab h^2 (-Laplace p) = g (equal-order
// Q1/Q1 with Brezzi-Pitkaranta pressure stabilisation, h the cell width),
// velocity Dirichlet on the whole boundary, the pressure filter on component 0
// (pfilter=1), and the smoother smoother=vanka (matrixtype vanka, linear_smooth
// ilu: VankaSmoother, LinAlg/vankasmoother.cc), smoother=ilu (matrixtype block,
// linear_smooth ilu: SparseBlockIlu in the order of ilusort's default
// cuthillmckee, which the METIS-free build keeps as the identity) or
// smoother=jacobi (block
// Jacobi). The right-hand side file then holds ncomp values per node.
//
// disc=Q2 selects CGQ2 (Q2 elements on patches of 2^dim cells); ball=r refines,
// after the global refinements, once more every leaf cell whose centroid lies
// within distance r of the domain's centre (MeshAgent::refine_cells: whole
// patches, hanging nodes at the interface); diff=eps replaces the coefficient
// by the constant eps (needed with ball refinement, where cell widths differ);
// lps=s0 (with diff=) adds local projection stabilisation of the convection
// (CGQ2Lps, or CGQ1Lps with disc=Q1: Q1 functions on patches;
// DiffusionLpsEquation below);
// rhsres=N reads the right-hand side on the (N+1)^dim lexicographic grid
// (N = 2 * coarse * 2^refine covers the nodes of the extra refinement).
//
// Usage: ref_harness key=value ...   (see parse() for the keys)
// Output (directory out=): summary.txt, and with dump=1 raw little-endian arrays
//   L<l>_rowptr.i64 L<l>_col.i64 L<l>_diag.i64 L<l>_val.f64 L<l>_coord.f64
//   L<l>_dirichlet.i64   (level l = 0 coarsest, as the reference indexes solvers)
//   T<l>_c2f.i64 T<l>_zweier.i64 T<l>_vierer.i64 T<l>_achter.i64
//     (transfer between level l (coarse) and l+1 (fine); zweier rows are
//      [fine, coarse0, coarse1], vierer [fine, 4 coarse], achter [fine, 8 coarse])
//   rhs.f64 solution.f64 (finest level, reference node numbering)
//   L<l>_val.f64 holds nnzb*ncomp^2 values (row-major blocks); for
//   problem=stokes also L<l>_pfw.f64 (pressure-filter weights) and
//   L<l>_patches.i64 (Vanka patches, npatches x nodes_per_patch), with
//   pfdomain_L<l>, ncomp and dircomps in summary.txt; the hanging nodes of
//   every level as L<l>_hnedge.i64 (rows [node, 3 parents]) and
//   L<l>_hnface.i64 (3D, rows [node, 9 parents]) with disc in summary.txt
// and with dualrhs= (a nodal vector like rhs): dual_summary.txt,
//   dual_rhs.f64 dual_solution.f64, and with dump=1 L<l>_dualval.f64 (the
//   dual matrices' values in the stencil of L<l>_col.i64)
// backup=1: solution.bup and solution.bip (WriteBackUp, WriteBackUpBinary);
// vtk=1: solution.00000.vtk (StdSolver::Visu);
// formx=<raw f64 finest-level vector x>: form.f64 = Form(0, x, 1),
//   newton_residual.f64 = NewtonResidual(x, rhs) and newton.txt (its norm).
#include "backup.h"
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "cginfo.h"
#include "columndiagstencil.h"
#include "domainfunctional.h"
#include "equation.h"
#include "fmatrixblock.h"
#include "functionalcontainer.h"
#include "gascoignemeshtransfer.h"
#include "hierarchicalmesh2d.h"
#include "hierarchicalmesh3d.h"
#include "meshagent.h"
#include "paramfile.h"
#include "problemcontainer.h"
#include "problemdescriptorbase.h"
#include "sparseblockmatrix.h"
#include "stdmultilevelsolver.h"
#include "stdsolver.h"
#include "pressurefilter.h"
#include "lpsequation.h"
#include "lpsstabilization.h"
#include "navierstokes.h"
#include "zerodirichletdata.h"
#ifdef GB_B200_BINDING
#include "b200solver.h"
#endif

using namespace Gascoigne;

namespace {

struct Config
{
  int dim = 3;
  double lps = 0.0; // sdelta0 of the LPS convection stabilisation (disc=Q2), 0: none
  int coarse = 1; // coarse mesh cells per dimension (1 or 2)
  int refine = 3; // global refinements
  std::string kappa, rhs, dualrhs, out = ".";
  int gmressize = 21, iterpre = 2, iterpost = 2, iterexact = 10;
  double omega = 0.8, tol = 1e-8, globaltol = 1e-16, mgomega = 1.0;
  int maxiter = 100, ndirect = 1, dump = 0, repeat = 1, patchdepth = 1;
  std::string mgtype = "V";
  double conv[3] = { 0.0, 0.0, 0.0 };
  std::string problem = "diffusion", smoother = "jacobi";
  double visc = 1.0, stab = 0.1;
  int pfilter = 1;
  std::string disc = "Q1";
  double ball = 0.0, diff = -1.0;
  int rhsres = 0;
  int backup = 0;     // write the solution with WriteBackUp / WriteBackUpBinary
  int vtk = 0;        // write the solution with StdSolver::Visu (VTK)
  std::string formx;  // Form and NewtonResidual of this finest-level vector
  std::string backend = "cpu"; // cpu: StdMultiLevelSolver; b200 / b200host /
                               // b200mixed: B200MultiLevelSolver (binary built
                               // with the binding): the whole solve as one
                               // device call, the reference's GMRES over device
                               // operations, or the mixed-precision device solve
  int savesol = 0;    // write rhs.f64 and solution.f64 without the full dump
  int functional = 0; // functional_l2 in summary.txt: J(u) of L2Functional
  int flexreps = 0;   // binding binary: that many more device solves with the
                      // flexible solver, FP64 cycle (flex64_*) and FP32 cycle
                      // (mixed_*, solution_mixed.f64) in summary.txt
  int flexgmressize = 0; // binding binary: Krylov memory of the flexible solves
  int benchspmv = 0;  // binding binary: the finest level's SpMV (FP64, FP32) and
                      // FP32 Jacobi sweep timed alone (gb_bench_spmv / _sweep)
  int cpusample = 0;  // that many GMRES steps (maxiter) of the reference's CPU
                      // solver on the same mesh and right-hand side, timed
                      // (cpu_sample_* in summary.txt, solution_cpu.f64)
};

// kappa per cell, one array per resolution N = coarse * 2^l (cells per dim),
// lexicographic (x fastest).
struct KappaPyramid
{
  int dim = 3;
  std::map<int, std::vector<double>> byN;
  double at(int N, double x, double y, double z) const
  {
    auto it = byN.find(N);
    if (it == byN.end()) {
      fprintf(stderr, "ref_harness: no kappa for resolution %d\n", N);
      abort();
    }
    auto clampi = [N](double t) {
      int i = static_cast<int>(std::floor(t * N));
      return i < 0 ? 0 : (i >= N ? N - 1 : i);
    };
    long i = clampi(x), j = clampi(y), k = dim == 3 ? clampi(z) : 0;
    return it->second[(k * N + j) * N + i];
  }
};
KappaPyramid g_kappa;
double g_diff = -1.0; // constant coefficient (diff=), or -1: the kappa pyramid

class DiffusionEquation : public virtual Equation
{
  mutable double kappa_ = 1.0;
  int dim_;
  double beta_[3];

public:
  DiffusionEquation(int dim, const double* beta)
    : dim_(dim)
  {
    for (int i = 0; i < 3; ++i)
      beta_[i] = beta[i];
  }
  DiffusionEquation* createNew() const override
  {
    return new DiffusionEquation(dim_, beta_);
  }
  std::string GetName() const override { return "OracleDiffusion"; }
  int GetNcomp() const override { return 1; }
  // h = vol^(1/dim) is the cell width on these uniform meshes
  // (ElementIntegrator::Matrix, DofHandler/elementintegrator.xx:369-379).
  void point(double h, const FemFunction&, const Vertex2d& v) const override
  {
    if (g_diff >= 0.0) {
      kappa_ = g_diff;
      return;
    }
    int N = static_cast<int>(std::lround(1.0 / h));
    kappa_ = g_kappa.at(N, v.x(), v.y(), 0.0);
  }
  void point(double h, const FemFunction&, const Vertex3d& v) const override
  {
    if (g_diff >= 0.0) {
      kappa_ = g_diff;
      return;
    }
    int N = static_cast<int>(std::lround(1.0 / h));
    kappa_ = g_kappa.at(N, v.x(), v.y(), v.z());
  }
  void Form(VectorIterator b,
            const FemFunction& U,
            const TestFunction& N) const override
  {
    for (int i = 0; i < dim_; ++i)
      b[0] += kappa_ * U[0][i + 1] * N[i + 1] + beta_[i] * U[0][i + 1] * N.m();
  }
  void Matrix(EntryMatrix& A,
              const FemFunction&,
              const TestFunction& M,
              const TestFunction& N) const override
  {
    // M: trial function, N: test function (as Problems/navierstokes.h:164)
    for (int i = 0; i < dim_; ++i)
      A(0, 0) += kappa_ * M[i + 1] * N[i + 1] + beta_[i] * M[i + 1] * N.m();
  }
};

// The same equation with local projection stabilisation of the convection
// (lps=sdelta0, with diff=: discretisation CGQ2Lps or CGQ1Lps,
// ElementLpsIntegrator, DofHandler/elementlpsintegrator.h): at each Gauss point
// delta = LpsStabilization::ConvectionDiffusion's sdelta0 / (xeta0 visc / h^2 +
// |beta| / h) (Problems/lpsstabilization.cc; xeta0 = 6, |beta| + 1e-6, h = the
// patch width), and the term delta (beta . grad Np)(beta . grad Mp) of the
// projected test functions.
class DiffusionLpsEquation : public DiffusionEquation, public LpsEquation
{
  int dim_;
  double beta_[3], sdelta0_;
  mutable LpsStabilization ST_;

public:
  DiffusionLpsEquation(int dim, const double* beta, double sdelta0)
    : DiffusionEquation(dim, beta)
    , dim_(dim)
    , sdelta0_(sdelta0)
  {
    for (int i = 0; i < 3; ++i)
      beta_[i] = beta[i];
    ST_.BasicInit(1);
    ST_.sdelta0 = sdelta0;
  }
  DiffusionLpsEquation* createNew() const override
  {
    return new DiffusionLpsEquation(dim_, beta_, sdelta0_);
  }
  std::string GetName() const override { return "OracleDiffusionLps"; }
  void lpspoint(double h, const FemFunction&, const Vertex2d&) const override
  {
    ST_.ReInit(h, g_diff, beta_[0], beta_[1]);
    ST_.ConvectionDiffusion(g_diff);
  }
  void lpspoint(double h, const FemFunction&, const Vertex3d&) const override
  {
    ST_.ReInit(h, g_diff, beta_[0], beta_[1], beta_[2]);
    ST_.ConvectionDiffusion(g_diff);
  }
  void StabForm(VectorIterator b, const FemFunction&, const FemFunction& UP,
                const TestFunction& N) const override
  {
    double bu = 0.0, bn = 0.0;
    for (int i = 0; i < dim_; ++i) {
      bu += beta_[i] * UP[0][i + 1];
      bn += beta_[i] * N[i + 1];
    }
    b[0] += ST_.delta(0) * bu * bn;
  }
  void StabMatrix(EntryMatrix& A, const FemFunction&, const TestFunction& Np,
                  const TestFunction& Mp) const override
  {
    double bn = 0.0, bm = 0.0;
    for (int i = 0; i < dim_; ++i) {
      bn += beta_[i] * Np[i + 1];
      bm += beta_[i] * Mp[i + 1];
    }
    A(0, 0) += ST_.delta(0) * bn * bm;
  }
};

// Stokes, components (p, v_1, .., v_dim) as Problems/navierstokes.h:144-168
// orders them (M trial, N test function).
class StokesEquation : public virtual Equation
{
  int dim_;
  double visc_, stab_;
  mutable double h_ = 1.0;

public:
  StokesEquation(int dim, double visc, double stab)
    : dim_(dim)
    , visc_(visc)
    , stab_(stab)
  {}
  StokesEquation* createNew() const override
  {
    return new StokesEquation(dim_, visc_, stab_);
  }
  std::string GetName() const override { return "OracleStokes"; }
  int GetNcomp() const override { return dim_ + 1; }
  void point(double h, const FemFunction&, const Vertex2d&) const override { h_ = h; }
  void point(double h, const FemFunction&, const Vertex3d&) const override { h_ = h; }
  void Form(VectorIterator b, const FemFunction& U, const TestFunction& N) const override
  {
    for (int i = 0; i < dim_; ++i) {
      b[0] += U[i + 1][i + 1] * N.m() + stab_ * h_ * h_ * U[0][i + 1] * N[i + 1];
      for (int j = 0; j < dim_; ++j)
        b[i + 1] += visc_ * U[i + 1][j + 1] * N[j + 1];
      b[i + 1] -= U[0].m() * N[i + 1];
    }
  }
  void Matrix(EntryMatrix& A, const FemFunction&, const TestFunction& M,
              const TestFunction& N) const override
  {
    for (int i = 0; i < dim_; ++i) {
      A(0, i + 1) += M[i + 1] * N.m();
      A(0, 0) += stab_ * h_ * h_ * M[i + 1] * N[i + 1];
      for (int j = 0; j < dim_; ++j)
        A(i + 1, i + 1) += visc_ * M[j + 1] * N[j + 1];
      A(i + 1, 0) -= M.m() * N[i + 1];
    }
  }
};

class StokesProblem : public ProblemDescriptorBase
{
public:
  void BasicInit(const ParamFile& pf, int dim, double visc, double stab)
  {
    GetParamFile() = pf;
    GetEquationPointer() = new StokesEquation(dim, visc, stab);
    GetDirichletDataPointer() = new ZeroDirichletData(pf);
    ProblemDescriptorBase::BasicInit(pf);
  }
};

// Stokes with LPS pressure stabilisation (problem=stokeslps): the reference's
// NavierStokesLps (Problems/navierstokes.h:91-280, discretisation CGQ1Lps)
// linearised at u = 0. Its Jacobian at U = 0 is already the Stokes operator
// plus alpha (grad p - pi grad p, grad q - pi grad q) with alpha = alpha0 h^2 /
// visc (lpspoint at zero velocity); Form drops the convection term so that the
// residual of the lid data is that same linear operator's.
template<int DIM>
class StokesLpsEquation : public NavierStokesLps<DIM>
{
public:
  explicit StokesLpsEquation(const NavierStokesData& d)
    : NavierStokesLps<DIM>(d)
  {}
  StokesLpsEquation* createNew() const override
  {
    return new StokesLpsEquation(this->data);
  }
  std::string GetName() const override { return "OracleStokesLps"; }
  void Form(VectorIterator b, const FemFunction& U, const TestFunction& N) const override
  {
    for (int i = 0; i < DIM; ++i) {
      b[0] += U[i + 1][i + 1] * N.m();
      for (int j = 0; j < DIM; ++j)
        b[i + 1] += this->data.visc * U[i + 1][j + 1] * N[j + 1];
      b[i + 1] -= U[0].m() * N[i + 1];
    }
  }
};

// Lid-driven cavity data: velocity (1, 0[, 0]) on the top face (y = 1 in 2D,
// z = 1 in 3D, its edges included), 0 on the rest of the boundary.
class LidDirichletData : public DirichletData
{
public:
  explicit LidDirichletData(const ParamFile& pf)
    : DirichletData(pf)
  {}
  std::string GetName() const override { return "OracleLid"; }
  void operator()(DoubleVector& b, const Vertex2d& v, int) const override
  {
    b.zero();
    if (v.y() > 1.0 - 1e-12)
      b[1] = 1.0;
  }
  void operator()(DoubleVector& b, const Vertex3d& v, int) const override
  {
    b.zero();
    if (v.z() > 1.0 - 1e-12)
      b[1] = 1.0;
  }
};

class StokesLpsProblem : public ProblemDescriptorBase
{
public:
  void BasicInit(const ParamFile& pf, int dim, double visc, double alpha0)
  {
    GetParamFile() = pf;
    NavierStokesData d;
    d.visc = visc;
    d.alpha = alpha0;
    d.delta = 0.0;
    d.symmetrictensor = false;
    d.outflowcolor = -1;
    d.dt = 0.0;
    d.theta = 0.0;
    if (dim == 2)
      GetEquationPointer() = new StokesLpsEquation<2>(d);
    else
      GetEquationPointer() = new StokesLpsEquation<3>(d);
    GetDirichletDataPointer() = new LidDirichletData(pf);
    ProblemDescriptorBase::BasicInit(pf);
  }
};

// J(u) = int sum_c u_c^2 over the components c (the scalar unknown, or the
// velocity of a Stokes system), evaluated by the reference's own
// StdSolver::ComputeFunctional -> ComputeDomainFunctional (hanging values
// averaged first, Solver/stdsolver.cc:1186-1246).
class L2Functional : public DomainFunctional
{
  std::vector<int> comps_;

public:
  explicit L2Functional(std::vector<int> comps)
    : comps_(std::move(comps))
  {}
  std::string GetName() const override { return "OracleL2"; }
  double J(const FemFunction& U, const Vertex2d&) const override { return sq(U); }
  double J(const FemFunction& U, const Vertex3d&) const override { return sq(U); }

private:
  double sq(const FemFunction& U) const
  {
    double s = 0.0;
    for (int c : comps_)
      s += U[c].m() * U[c].m();
    return s;
  }
};

// the pressure filter's domain size is not exposed by PressureFilter, and
// StdSolver::GetPfilter is protected: read both through derived-class access
struct PressureFilterView : public PressureFilter
{
  double domain() const { return domainsize; }
};
struct SolverView : public StdSolver
{
  static const PressureFilter& pfilter(const StdSolver* s)
  {
    const PressureFilter& (StdSolver::*get)() const = &SolverView::GetPfilter;
    return (s->*get)();
  }
};

class DiffusionProblem : public ProblemDescriptorBase
{
public:
  void BasicInit(const ParamFile& pf, int dim, const double* beta, double lps)
  {
    GetParamFile() = pf;
    if (lps > 0.0)
      GetEquationPointer() = new DiffusionLpsEquation(dim, beta, lps);
    else
      GetEquationPointer() = new DiffusionEquation(dim, beta);
    GetDirichletDataPointer() = new ZeroDirichletData(pf);
    ProblemDescriptorBase::BasicInit(pf);
  }
};

Config
parse(int argc, char** argv)
{
  Config c;
  for (int a = 1; a < argc; ++a) {
    std::string s = argv[a];
    auto eq = s.find('=');
    if (eq == std::string::npos) {
      fprintf(stderr, "ref_harness: bad argument %s\n", s.c_str());
      exit(2);
    }
    std::string k = s.substr(0, eq), v = s.substr(eq + 1);
    if (k == "dim") c.dim = atoi(v.c_str());
    else if (k == "coarse") c.coarse = atoi(v.c_str());
    else if (k == "refine") c.refine = atoi(v.c_str());
    else if (k == "kappa") c.kappa = v;
    else if (k == "rhs") c.rhs = v;
    else if (k == "dualrhs") c.dualrhs = v;
    else if (k == "out") c.out = v;
    else if (k == "gmressize") c.gmressize = atoi(v.c_str());
    else if (k == "iterpre") c.iterpre = atoi(v.c_str());
    else if (k == "iterpost") c.iterpost = atoi(v.c_str());
    else if (k == "iterexact") c.iterexact = atoi(v.c_str());
    else if (k == "omega") c.omega = atof(v.c_str());
    else if (k == "tol") c.tol = atof(v.c_str());
    else if (k == "globaltol") c.globaltol = atof(v.c_str());
    else if (k == "mgomega") c.mgomega = atof(v.c_str());
    else if (k == "maxiter") c.maxiter = atoi(v.c_str());
    else if (k == "ndirect") c.ndirect = atoi(v.c_str());
    else if (k == "mgtype") c.mgtype = v;
    else if (k == "dump") c.dump = atoi(v.c_str());
    else if (k == "backup") c.backup = atoi(v.c_str());
    else if (k == "vtk") c.vtk = atoi(v.c_str());
    else if (k == "formx") c.formx = v;
    else if (k == "repeat") c.repeat = atoi(v.c_str());
    else if (k == "patchdepth") c.patchdepth = atoi(v.c_str());
    else if (k == "problem") c.problem = v;
    else if (k == "smoother") c.smoother = v;
    else if (k == "visc") c.visc = atof(v.c_str());
    else if (k == "stab") c.stab = atof(v.c_str());
    else if (k == "pfilter") c.pfilter = atoi(v.c_str());
    else if (k == "disc") c.disc = v;
    else if (k == "ball") c.ball = atof(v.c_str());
    else if (k == "diff") c.diff = atof(v.c_str());
    else if (k == "lps") c.lps = atof(v.c_str());
    else if (k == "rhsres") c.rhsres = atoi(v.c_str());
    else if (k == "backend") c.backend = v;
    else if (k == "savesol") c.savesol = atoi(v.c_str());
    else if (k == "functional") c.functional = atoi(v.c_str());
    else if (k == "flexreps") c.flexreps = atoi(v.c_str());
    else if (k == "flexgmressize") c.flexgmressize = atoi(v.c_str());
    else if (k == "benchspmv") c.benchspmv = atoi(v.c_str());
    else if (k == "cpusample") c.cpusample = atoi(v.c_str());
    else if (k == "conv") {
      std::stringstream ss(v);
      std::string t;
      for (int i = 0; i < 3 && std::getline(ss, t, ','); ++i)
        c.conv[i] = atof(t.c_str());
    }
    else {
      fprintf(stderr, "ref_harness: unknown key %s\n", k.c_str());
      exit(2);
    }
  }
  return c;
}

std::vector<double>
read_f64(const std::string& path, size_t n)
{
  std::vector<double> v(n);
  FILE* f = fopen(path.c_str(), "rb");
  if (!f || fread(v.data(), sizeof(double), n, f) != n) {
    fprintf(stderr, "ref_harness: cannot read %zu doubles from %s\n", n,
            path.c_str());
    exit(2);
  }
  fclose(f);
  return v;
}

template<class T>
void
write_raw(const std::string& path, const std::vector<T>& v)
{
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) {
    fprintf(stderr, "ref_harness: cannot write %s\n", path.c_str());
    exit(2);
  }
  if (!v.empty())
    fwrite(v.data(), sizeof(T), v.size(), f);
  fclose(f);
}

void
write_mesh(const Config& c, const std::string& path)
{
  // Unit square / cube split into coarse^dim cells, every boundary face colour 1,
  // in the reference's .inp format (evaluation/examples/Elasticity3d/box.inp).
  int m = c.coarse, np = m + 1;
  std::ofstream o(path);
  o.precision(17);
  if (c.dim == 2) {
    int nn = np * np, nc = m * m, nb = 4 * m;
    o << nn << " " << nc + nb << " 0 0 0\n";
    for (int j = 0; j < np; ++j)
      for (int i = 0; i < np; ++i)
        o << j * np + i << " " << double(i) / m << " " << double(j) / m
          << " 0\n"; // 2D vertices are read as Vertex3d
    int id = 0;
    auto N = [np](int i, int j) { return j * np + i; };
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < m; ++i)
        o << id++ << " 0 quad " << N(i, j) << " " << N(i + 1, j) << " "
          << N(i + 1, j + 1) << " " << N(i, j + 1) << "\n";
    for (int i = 0; i < m; ++i) {
      o << id++ << " 1 line " << N(i, 0) << " " << N(i + 1, 0) << "\n";
      o << id++ << " 1 line " << N(i + 1, m) << " " << N(i, m) << "\n";
      o << id++ << " 1 line " << N(0, i + 1) << " " << N(0, i) << "\n";
      o << id++ << " 1 line " << N(m, i) << " " << N(m, i + 1) << "\n";
    }
  } else {
    int nn = np * np * np, nc = m * m * m, nb = 6 * m * m;
    o << nn << " " << nc + nb << " 0 0 0\n";
    auto N = [np](int i, int j, int k) { return (k * np + j) * np + i; };
    for (int k = 0; k < np; ++k)
      for (int j = 0; j < np; ++j)
        for (int i = 0; i < np; ++i)
          o << N(i, j, k) << " " << double(i) / m << " " << double(j) / m << " "
            << double(k) / m << "\n";
    int id = 0;
    for (int k = 0; k < m; ++k)
      for (int j = 0; j < m; ++j)
        for (int i = 0; i < m; ++i)
          o << id++ << " 0 hex " << N(i, j, k) << " " << N(i + 1, j, k) << " "
            << N(i + 1, j + 1, k) << " " << N(i, j + 1, k) << " "
            << N(i, j, k + 1) << " " << N(i + 1, j, k + 1) << " "
            << N(i + 1, j + 1, k + 1) << " " << N(i, j + 1, k + 1) << "\n";
    for (int a = 0; a < m; ++a)
      for (int b = 0; b < m; ++b) {
        // z = 0, z = 1, y = 0, y = 1, x = 0, x = 1
        o << id++ << " 1 quad " << N(a, b, 0) << " " << N(a, b + 1, 0) << " "
          << N(a + 1, b + 1, 0) << " " << N(a + 1, b, 0) << "\n";
        o << id++ << " 1 quad " << N(a, b, m) << " " << N(a + 1, b, m) << " "
          << N(a + 1, b + 1, m) << " " << N(a, b + 1, m) << "\n";
        o << id++ << " 1 quad " << N(a, 0, b) << " " << N(a + 1, 0, b) << " "
          << N(a + 1, 0, b + 1) << " " << N(a, 0, b + 1) << "\n";
        o << id++ << " 1 quad " << N(a, m, b) << " " << N(a, m, b + 1) << " "
          << N(a + 1, m, b + 1) << " " << N(a + 1, m, b) << "\n";
        o << id++ << " 1 quad " << N(0, a, b) << " " << N(0, a, b + 1) << " "
          << N(0, a + 1, b + 1) << " " << N(0, a + 1, b) << "\n";
        o << id++ << " 1 quad " << N(m, a, b) << " " << N(m, a + 1, b) << " "
          << N(m, a + 1, b + 1) << " " << N(m, a, b + 1) << "\n";
      }
  }
}

void
write_param(const Config& c, const std::string& path, const std::string& grid)
{
  std::ofstream o(path);
  o.precision(17);
  o << "//Block Mesh\n"
    << "dimension " << c.dim << "\n"
    << "prerefine " << c.refine << "\n"
    << "patchdepth " << c.patchdepth << "\n"
    << "gridname " << grid << "\n\n"
    << "//Block BoundaryManager\n"
    << "dirichlet 1 1\n";
  if (c.problem == "stokes" || c.problem == "stokeslps") {
    o << "dirichletcomp 1 " << c.dim;
    for (int d = 1; d <= c.dim; ++d)
      o << " " << d;
    o << "\n\n";
  } else {
    o << "dirichletcomp 1 1 0\n\n";
  }
  o
    << "//Block MultiLevelSolver\n"
    << "linearsolve gmres\n"
    << "gmressize " << c.gmressize << "\n"
    << "mgtype " << c.mgtype << "\n"
    << "mgomega " << c.mgomega << "\n"
    << "coarselevel 0\n\n"
    << "//Block Solver\n"
    << "matrixtype " << (c.smoother == "vanka" ? "vanka" : "block") << "\n"
    << "discname "
    << (c.disc == "Q2" ? (c.lps > 0.0 ? "CGQ2Lps" : "CGQ2")
                       : (c.lps > 0.0 || c.problem == "stokeslps" ? "CGQ1Lps" : "CGQ1"))
    << "\n"
    << "ndirect " << c.ndirect << "\n"
    << "iterpre " << c.iterpre << "\n"
    << "iterpost " << c.iterpost << "\n"
    << "iterexact " << c.iterexact << "\n"
    << "linear_smooth " << (c.smoother == "vanka" || c.smoother == "ilu" ? "ilu" : "jacobi")
    << "\n"
    << "omega " << c.omega << "\n";
  if ((c.problem == "stokes" || c.problem == "stokeslps") && c.pfilter)
    o << "pfilter 1 0\n";
}

void
build_kappa(const Config& c)
{
  g_kappa.dim = c.dim;
  int Nf = c.coarse << c.refine;
  size_t ncell = 1;
  for (int d = 0; d < c.dim; ++d)
    ncell *= Nf;
  std::vector<double> fine = c.kappa.empty() ? std::vector<double>(ncell, 1.0)
                                             : read_f64(c.kappa, ncell);
  g_kappa.byN[Nf] = fine;
  for (int N = Nf / 2; N >= c.coarse; N /= 2) {
    const std::vector<double>& f = g_kappa.byN[2 * N];
    int M = 2 * N;
    std::vector<double> k(c.dim == 3 ? size_t(N) * N * N : size_t(N) * N);
    int nz = c.dim == 3 ? N : 1;
    for (int kk = 0; kk < nz; ++kk)
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
          double s = 0.0;
          int dz = c.dim == 3 ? 2 : 1;
          for (int a = 0; a < dz; ++a)
            for (int b = 0; b < 2; ++b)
              for (int e = 0; e < 2; ++e) {
                size_t idx = c.dim == 3
                               ? (size_t(2 * kk + a) * M + 2 * j + b) * M + 2 * i + e
                               : size_t(2 * j + b) * M + 2 * i + e;
                s += f[idx];
              }
          k[(size_t(kk) * N + j) * N + i] = s / (c.dim == 3 ? 8.0 : 4.0);
        }
    g_kappa.byN[N] = k;
  }
}

// Values of a SparseBlockMatrix<FMatrixBlock<NCOMP>> in stencil order,
// row-major blocks (NodeMatrix::value, LinAlg/nodematrix.h:44-48).
template<int NCOMP>
bool
block_values(const MatrixInterface& MI, std::vector<double>& val,
             const StencilInterface*& st)
{
  const auto* M = dynamic_cast<const SparseBlockMatrix<FMatrixBlock<NCOMP>>*>(&MI);
  if (!M)
    return false;
  const auto* ST = dynamic_cast<const ColumnDiagStencil*>(M->GetStencil());
  st = ST;
  val.resize(ST->nentries() * NCOMP * NCOMP);
  for (size_t p = 0; p < ST->nentries(); ++p)
    for (int r = 0; r < NCOMP; ++r)
      for (int q = 0; q < NCOMP; ++q)
        val[(p * NCOMP + r) * NCOMP + q] = (*M->mat(p))(r, q);
  return true;
}

} // namespace

int
run(int argc, char** argv)
{
  Config c = parse(argc, argv);
  std::string grid = c.out + "/oracle_mesh.inp";
  std::string pfile = c.out + "/oracle.param";
  write_mesh(c, grid);
  write_param(c, pfile, grid);
  build_kappa(c);

  ParamFile pf(pfile);
  DiffusionProblem PD;
  StokesProblem PS;
  StokesLpsProblem PL;
  const bool lid = c.problem == "stokeslps";
  const bool stokes = c.problem == "stokes" || lid;
  if (lid)
    PL.BasicInit(pf, c.dim, c.visc, c.stab);
  else if (stokes)
    PS.BasicInit(pf, c.dim, c.visc, c.stab);
  else
    PD.BasicInit(pf, c.dim, c.conv, c.lps);
  const int ncomp = stokes ? c.dim + 1 : 1;
  ProblemContainer PC;
  PC.AddProblem("diffusion", lid ? static_cast<ProblemDescriptorInterface*>(&PL)
                             : stokes ? static_cast<ProblemDescriptorInterface*>(&PS)
                                      : static_cast<ProblemDescriptorInterface*>(&PD));
  FunctionalContainer FC;

  g_diff = c.diff;
  MeshAgent MA;
  MA.BasicInit(pf);
  if (c.ball > 0.0) {
    // one more refinement of the leaf cells whose centroid is in the ball
    HierarchicalMesh* HM = MA.GetHierarchicalMesh();
    IntVector ref;
    const int nv = c.dim == 3 ? 8 : 4;
    for (int cell = 0; cell < HM->ncells(); ++cell) {
      if (HM->sleep(cell))
        continue;
      double x[3] = { 0, 0, 0 };
      for (int j = 0; j < nv; ++j) {
        const int vtx = HM->vertex_of_cell(cell, j);
        if (c.dim == 3) {
          const Vertex3d& w = dynamic_cast<HierarchicalMesh3d*>(HM)->vertex3d(vtx);
          x[0] += w.x() / nv, x[1] += w.y() / nv, x[2] += w.z() / nv;
        } else {
          const Vertex2d& w = dynamic_cast<HierarchicalMesh2d*>(HM)->vertex2d(vtx);
          x[0] += w.x() / nv, x[1] += w.y() / nv;
        }
      }
      double r2 = 0;
      for (int d = 0; d < c.dim; ++d)
        r2 += (x[d] - 0.5) * (x[d] - 0.5);
      if (r2 < c.ball * c.ball)
        ref.push_back(cell);
    }
    MA.refine_cells(ref);
  }
  std::unique_ptr<StdMultiLevelSolver> MLSp;
  if (c.backend == "cpu")
    MLSp.reset(new StdMultiLevelSolver);
#ifdef GB_B200_BINDING
  else if (c.backend == "b200" || c.backend == "b200host" || c.backend == "b200mixed") {
    auto* B = new B200MultiLevelSolver(0);
    B->SetDeviceGmres(c.backend != "b200host");
    B->SetFlexibleMemory(c.flexgmressize);
    B->SetDeviceSolver(c.backend == "b200mixed" ? B200MultiLevelSolver::kFlexible32
                                                : B200MultiLevelSolver::kReference);
    MLSp.reset(B);
  }
#endif
  else {
    fprintf(stderr, "ref_harness: backend %s is not built into this binary\n",
            c.backend.c_str());
    return 2;
  }
  StdMultiLevelSolver& MLS = *MLSp;
  MLS.BasicInit(&MA, pf, &PC, &FC);
  MLS.ReInit();
  MLS.SetProblem("diffusion");

  Matrix A("A");
  Vector u("u"), f("f");
  MLS.ReInitMatrix(A);
  MLS.ReInitVector(u);
  MLS.ReInitVector(f);

  auto t_as0 = std::chrono::steady_clock::now();
  MLS.AssembleMatrix(A, u);
  MLS.ComputeIlu(A, u);
  auto t_as1 = std::chrono::steady_clock::now();

  const int nl = MLS.nlevels();
  const int Nf = c.rhsres > 0 ? c.rhsres : (c.coarse << c.refine);
  StdSolver* S = MLS.GetSolver();
  const GascoigneMesh* Mf = S->GetMesh();
  const int nf = Mf->nnodes();
  GlobalVector& F = S->GetGV(f);
  if (lid) {
    // the right-hand side of the Newton update from the lid data u_D:
    // f = 0 - Form(u_D), Dirichlet-zeroed, algebraically mean-free
    // (StdMultiLevelSolver::NewtonResidual, Solver/stdmultilevelsolver.cc:609-623)
    Vector ud("ud"), z0("z0");
    MLS.ReInitVector(ud);
    MLS.ReInitVector(z0);
    S->Zero(ud);
    S->Zero(z0);
    S->SetBoundaryVector(ud);
    MLS.NewtonResidual(f, ud, z0);
  } else {
    size_t nlex = 1;
    for (int d = 0; d < c.dim; ++d)
      nlex *= Nf + 1;
    std::vector<double> r = c.rhs.empty() ? std::vector<double>(nlex * ncomp, 1.0)
                                          : read_f64(c.rhs, nlex * ncomp);
    for (int i = 0; i < nf; ++i) {
      long ix, iy, iz = 0;
      if (c.dim == 3) {
        const Vertex3d& v = Mf->vertex3d(i);
        ix = std::lround(v.x() * Nf);
        iy = std::lround(v.y() * Nf);
        iz = std::lround(v.z() * Nf);
      } else {
        const Vertex2d& v = Mf->vertex2d(i);
        ix = std::lround(v.x() * Nf);
        iy = std::lround(v.y() * Nf);
      }
      for (int cc = 0; cc < ncomp; ++cc)
        F(i, cc) = r[((iz * (Nf + 1) + iy) * (Nf + 1) + ix) * ncomp + cc];
    }
  }
  S->HNZero(f); // hanging dofs are constrained, not unknowns
  S->SetBoundaryVectorZero(f);

  std::vector<double> times, device_ms_all;
  CGInfo info(c.tol, c.globaltol, 0, c.maxiter, "Lin");
  for (int rep = 0; rep < std::max(1, c.repeat); ++rep) {
    info.reset();
    auto t0 = std::chrono::steady_clock::now();
    MLS.NewtonLinearSolve(A, u, f, info);
    auto t1 = std::chrono::steady_clock::now();
    times.push_back(std::chrono::duration<double>(t1 - t0).count());
#ifdef GB_B200_BINDING
    if (auto* B = dynamic_cast<B200MultiLevelSolver*>(&MLS))
      device_ms_all.push_back(B->LastSolveInfo().device_ms);
#endif
  }

  // true relative residual ||f - A u|| / ||f|| with the reference's own vmult
  Vector r("r");
  MLS.ReInitVector(r);
  S->residualgmres(A, r, u, f);
  double rnorm = S->Norm(r), fnorm = S->Norm(f);
  double Jl2 = 0.0;
  if (c.functional) {
    std::vector<int> jc;
    if (stokes)
      for (int d = 1; d <= c.dim; ++d)
        jc.push_back(d);
    else
      jc.push_back(0);
    L2Functional JF(jc);
    Vector jh("jh");
    MLS.ReInitVector(jh);
    Jl2 = S->ComputeFunctional(jh, u, &JF);
  }

  {
    std::ofstream o(c.out + "/summary.txt");

    o.precision(17);
    o << "nlevels " << nl << "\n";
    for (int l = 0; l < nl; ++l)
      o << "nnodes_L" << l << " " << MLS.GetSolver(l)->GetMesh()->nnodes()
        << "\n";
    o << "iterations " << info.control().iteration() << "\n";
    o << "status " << info.control().status() << "\n";
    o << "firstresidual " << info.control().firstresidual() << "\n";
    o << "residual " << info.control().residual() << "\n";
    o << "true_rel_residual " << rnorm / fnorm << "\n";
    if (c.functional)
      o << "functional_l2 " << Jl2 << "\n";
    o << "ncomp " << ncomp << "\n";
    o << "disc " << c.disc << "\n";
    o << "dircomps";
    if (stokes)
      for (int d = 1; d <= c.dim; ++d)
        o << " " << d;
    else
      o << " 0";
    o << "\n";
    if (stokes)
      for (int l = 0; l < nl; ++l)
        o << "pfdomain_L" << l << " "
          << static_cast<const PressureFilterView&>(SolverView::pfilter(MLS.GetSolver(l)))
               .domain()
          << "\n";
    o << "assemble_s "
      << std::chrono::duration<double>(t_as1 - t_as0).count() << "\n";
    o << "backend " << c.backend << "\n";
#ifdef GB_B200_BINDING
    if (auto* B = dynamic_cast<B200MultiLevelSolver*>(&MLS))
    {
      o << "device_ms " << B->LastSolveInfo().device_ms << "\n"
        << "device_launches " << B->LastSolveInfo().kernel_launches << "\n"
        << "device_ms_all";
      for (double t : device_ms_all)
        o << " " << t;
      o << "\n";
    }
#endif
    o << "solve_s";
    for (double t : times)
      o << " " << t;
    o << "\n";
  }

  if (c.savesol && !c.dump) {
    write_raw(c.out + "/rhs.f64", std::vector<double>(F.begin(), F.end()));
    const GlobalVector& U = S->GetGV(u);
    write_raw(c.out + "/solution.f64", std::vector<double>(U.begin(), U.end()));
    std::vector<double> xyz;
    for (int i = 0; i < nf; ++i) {
      if (c.dim == 3) {
        const Vertex3d& v = Mf->vertex3d(i);
        xyz.insert(xyz.end(), { v.x(), v.y(), v.z() });
      } else {
        const Vertex2d& v = Mf->vertex2d(i);
        xyz.insert(xyz.end(), { v.x(), v.y() });
      }
    }
    write_raw(c.out + "/coord.f64", xyz);
  }
#ifdef GB_B200_BINDING
  // more device solves of the same system with the flexible solver: FP64
  // cycle, then FP32 cycle (mixed precision)
  if (c.flexreps > 0) {
    auto* B = dynamic_cast<B200MultiLevelSolver*>(&MLS);
    if (!B)
      throw std::runtime_error("flexreps needs a b200 backend");
    std::vector<int> jc;
    if (stokes)
      for (int d = 1; d <= c.dim; ++d)
        jc.push_back(d);
    else
      jc.push_back(0);
    std::ofstream o(c.out + "/summary.txt", std::ios::app);
    o.precision(17);
    for (int kind = 1; kind <= 2; ++kind) {
      const std::string tag = kind == 1 ? "flex64" : "mixed";
      Vector um(tag + "_u");
      MLS.ReInitVector(um);
      B->SetDeviceSolver(kind == 1 ? B200MultiLevelSolver::kFlexible64
                                   : B200MultiLevelSolver::kFlexible32);
      std::vector<double> mms;
      CGInfo minfo(c.tol, c.globaltol, 0, c.maxiter, tag);
      for (int rep = 0; rep < c.flexreps; ++rep) {
        MLS.NewtonLinearSolve(A, um, f, minfo);
        mms.push_back(B->LastSolveInfo().device_ms);
      }
      const gb_solve_info li = B->LastSolveInfo();
      Vector rm(tag + "_r");
      MLS.ReInitVector(rm);
      S->residualgmres(A, rm, um, f);
      const double rmn = S->Norm(rm) / S->Norm(f);
      double Jm = 0.0;
      if (c.functional) {
        L2Functional JF(jc);
        Vector jh(tag + "_jh");
        MLS.ReInitVector(jh);
        Jm = S->ComputeFunctional(jh, um, &JF);
      }
      if (kind == 2) {
        const GlobalVector& Um = S->GetGV(um);
        write_raw(c.out + "/solution_mixed.f64", std::vector<double>(Um.begin(), Um.end()));
      }
      o << tag << "_iterations " << li.iterations << "\n"
        << tag << "_restarts " << li.restarts << "\n"
        << tag << "_launches " << li.kernel_launches << "\n"
        << tag << "_true_rel_residual " << rmn << "\n"
        << tag << "_functional_l2 " << Jm << "\n"
        << tag << "_device_ms_all";
      for (double t : mms)
        o << " " << t;
      o << "\n";
    }
    B->SetDeviceSolver(B200MultiLevelSolver::kReference);
  }
  if (c.benchspmv) {
    auto* B = dynamic_cast<B200MultiLevelSolver*>(&MLS);
    if (!B)
      throw std::runtime_error("benchspmv needs a b200 backend");
    gb_ctx* gc = B->DeviceContext();
    const int fl = nl - 1;
    double ms = 0, by = 0;
    std::ofstream o(c.out + "/summary.txt", std::ios::app);
    o.precision(17);
    for (int prec = 0; prec <= 1; ++prec) {
      if (gb_bench_spmv(gc, fl, prec, 20, 2, &ms, &by) != GB_OK)
        throw std::runtime_error(gb_last_error_string(gc));
      o << (prec ? "spmv32" : "spmv64") << "_ms " << ms << "\n"
        << (prec ? "spmv32" : "spmv64") << "_bytes " << by << "\n";
    }
    if (ncomp == 1) {
      if (gb_bench_sweep(gc, fl, 1, 20, 2, &ms, &by) != GB_OK)
        throw std::runtime_error(gb_last_error_string(gc));
      o << "sweep32_ms " << ms << "\n"
        << "sweep32_bytes " << by << "\n";
    }
  }
#endif
  // the reference's CPU solver on the same mesh, problem and right-hand side,
  // bounded to cpusample GMRES steps (maxiter), timed after its assembly
  if (c.cpusample > 0) {
    StdMultiLevelSolver C;
    C.BasicInit(&MA, pf, &PC, &FC);
    C.ReInit();
    C.SetProblem("diffusion");
    Matrix Ac("A");
    Vector uc("u"), fc("f");
    C.ReInitMatrix(Ac);
    C.ReInitVector(uc);
    C.ReInitVector(fc);
    auto a0 = std::chrono::steady_clock::now();
    C.AssembleMatrix(Ac, uc);
    C.ComputeIlu(Ac, uc);
    auto a1 = std::chrono::steady_clock::now();
    GlobalVector& Fc = C.GetSolver()->GetGV(fc);
    const GlobalVector& Fd = S->GetGV(f);
    std::copy(Fd.begin(), Fd.end(), Fc.begin());
    CGInfo cinfo(c.tol, c.globaltol, 0, std::min(c.maxiter, c.cpusample), "Cpu");
    auto t0 = std::chrono::steady_clock::now();
    C.NewtonLinearSolve(Ac, uc, fc, cinfo);
    auto t1 = std::chrono::steady_clock::now();
    const GlobalVector& Uc = C.GetSolver()->GetGV(uc);
    write_raw(c.out + "/solution_cpu.f64", std::vector<double>(Uc.begin(), Uc.end()));
    double Jc = 0.0;
    if (c.functional) {
      std::vector<int> jc;
      if (stokes)
        for (int d = 1; d <= c.dim; ++d)
          jc.push_back(d);
      else
        jc.push_back(0);
      L2Functional JF(jc);
      Vector jh("jh3");
      C.ReInitVector(jh);
      Jc = C.GetSolver()->ComputeFunctional(jh, uc, &JF);
    }
    std::ofstream o(c.out + "/summary.txt", std::ios::app);
    o.precision(17);
    o << "cpu_sample_iterations " << cinfo.control().iteration() << "\n"
      << "cpu_sample_status " << cinfo.control().status() << "\n"
      << "cpu_sample_s " << std::chrono::duration<double>(t1 - t0).count() << "\n"
      << "cpu_sample_assemble_s " << std::chrono::duration<double>(a1 - a0).count() << "\n"
      << "cpu_sample_functional_l2 " << Jc << "\n";
  }
  if (c.dump) {
    for (int l = 0; l < nl; ++l) {
      StdSolver* SL = MLS.GetSolver(l);
      const MatrixInterface& MI = SL->GetMatrix(A);
      const StencilInterface* STI = nullptr;
      std::vector<double> val;
      if (!block_values<1>(MI, val, STI) && !block_values<2>(MI, val, STI) &&
          !block_values<3>(MI, val, STI) && !block_values<4>(MI, val, STI)) {
        fprintf(stderr, "ref_harness: level %d is not a block matrix\n", l);
        return 3;
      }
      const auto* ST = dynamic_cast<const ColumnDiagStencil*>(STI);
      const int n = ST->n();
      std::vector<long> rowptr(n + 1), col(ST->nentries()), diag(n);
      for (int i = 0; i <= n; ++i)
        rowptr[i] = ST->start(i);
      for (size_t p = 0; p < ST->nentries(); ++p)
        col[p] = ST->col(p);
      for (int i = 0; i < n; ++i)
        diag[i] = ST->diag(i);
      std::string L = c.out + "/L" + std::to_string(l) + "_";
      write_raw(L + "rowptr.i64", rowptr);
      write_raw(L + "col.i64", col);
      write_raw(L + "diag.i64", diag);
      write_raw(L + "val.f64", val);
      const GascoigneMesh* ML = SL->GetMesh();
      std::vector<double> xyz;
      for (int i = 0; i < ML->nnodes(); ++i) {
        if (c.dim == 3) {
          const Vertex3d& v = ML->vertex3d(i);
          xyz.push_back(v.x());
          xyz.push_back(v.y());
          xyz.push_back(v.z());
        } else {
          const Vertex2d& v = ML->vertex2d(i);
          xyz.push_back(v.x());
          xyz.push_back(v.y());
        }
      }
      write_raw(L + "coord.f64", xyz);
      std::vector<long> dn;
      const IntVector* bv = ML->VertexOnBoundary(1);
      if (bv)
        for (int i : *bv)
          dn.push_back(i);
      write_raw(L + "dirichlet.i64", dn);
      {
        const HangingIndexHandler& HI = ML->GetHangingIndexHandler();
        std::vector<long> he, hf;
        for (const auto& e : *HI.GetStructure()) {
          he.push_back(e.first);
          for (int q : e.second)
            he.push_back(q);
        }
        for (const auto& e : *HI.GetStructureFace()) {
          hf.push_back(e.first);
          for (int q : e.second)
            hf.push_back(q);
        }
        write_raw(L + "hnedge.i64", he);
        write_raw(L + "hnface.i64", hf);
      }
      if (stokes) {
        const PressureFilter& PF = SolverView::pfilter(SL);
        std::vector<double> w(PF.begin(), PF.end());
        write_raw(L + "pfw.f64", w);
        std::vector<long> pl;
        for (int p = 0; p < ML->npatches(); ++p)
          for (int i : *ML->IndicesOfPatch(p))
            pl.push_back(i);
        write_raw(L + "patches.i64", pl);
      }
    }
    for (int l = 0; l + 1 < nl; ++l) {
      // interpolator l maps level l+1 (fine) to level l (coarse); it is built
      // from mesh transfer nlevels-l-2 (Solver/stdmultilevelsolver.cc:290-296)
      const GascoigneMeshTransfer* GT = MA.GetTransfer(nl - l - 2);
      std::string T = c.out + "/T" + std::to_string(l) + "_";
      std::vector<long> c2f(GT->GetC2f().begin(), GT->GetC2f().end());
      write_raw(T + "c2f.i64", c2f);
      std::vector<long> z, v4, a8;
      for (const auto& p : GT->GetZweier()) {
        z.push_back(p.first);
        for (int q : p.second)
          z.push_back(q);
      }
      for (const auto& p : GT->GetVierer()) {
        v4.push_back(p.first);
        for (int q : p.second)
          v4.push_back(q);
      }
      for (const auto& p : GT->GetAchter()) {
        a8.push_back(p.first);
        for (int q : p.second)
          a8.push_back(q);
      }
      write_raw(T + "zweier.i64", z);
      write_raw(T + "vierer.i64", v4);
      write_raw(T + "achter.i64", a8);
    }
    // the finest level's hanging-node operations on a test vector
    // t(i, c) = sin(1 + i * ncomp + c): HNAverage, HNDistribute, HNZero
    {
      Vector t("t");
      MLS.ReInitVector(t);
      GlobalVector& T = S->GetGV(t);
      auto fill = [&]() {
        for (int i = 0; i < nf; ++i)
          for (int cc = 0; cc < ncomp; ++cc)
            T(i, cc) = std::sin(1.0 + i * ncomp + cc);
      };
      fill();
      S->HNAverage(t);
      write_raw(c.out + "/hn_average.f64", std::vector<double>(T.begin(), T.end()));
      fill();
      S->HNDistribute(t);
      write_raw(c.out + "/hn_distribute.f64", std::vector<double>(T.begin(), T.end()));
      fill();
      S->HNZero(t);
      write_raw(c.out + "/hn_zero.f64", std::vector<double>(T.begin(), T.end()));
    }
    std::vector<double> rhs(F.begin(), F.end());
    write_raw(c.out + "/rhs.f64", rhs);
    const GlobalVector& U = S->GetGV(u);
    std::vector<double> sol(U.begin(), U.end());
    write_raw(c.out + "/solution.f64", sol);
    // Common/backup.cc: the text (.bup) and binary (.bip) solution files
    if (c.backup) {
      WriteBackUp(U, c.out + "/solution");
      WriteBackUpBinary(U, c.out + "/solution");
    }
    // StdSolver::Visu -> CGDisc::VisuVtk (DofHandler/cgdisc.h:136-158): the
    // finest level's solution as solution.00000.vtk (Visualization::vtk,
    // Discretization/Q1/vtk.cc), hanging values averaged first
    if (c.vtk)
      S->Visu(c.out + "/solution", u, 0);
    // StdSolver::Form (Solver/stdsolver.cc:1041-1063) of a given vector with
    // d = 1 on the finest level, and StdMultiLevelSolver::NewtonResidual
    // (Solver/stdmultilevelsolver.cc:609-623) y = f - Form(x), boundary zero,
    // with its norm
    if (!c.formx.empty()) {
      Vector x("fx"), y("fy");
      MLS.ReInitVector(x);
      MLS.ReInitVector(y);
      GlobalVector& X = S->GetGV(x);
      std::vector<double> xv = read_f64(c.formx, X.size());
      std::copy(xv.begin(), xv.end(), X.begin());
      S->Zero(y);
      S->Form(y, x, 1.);
      const GlobalVector& Y = S->GetGV(y);
      write_raw(c.out + "/form.f64", std::vector<double>(Y.begin(), Y.end()));
      std::copy(xv.begin(), xv.end(), X.begin()); // Form averaged/zeroed hanging values
      const double nr = MLS.NewtonResidual(y, x, f);
      write_raw(c.out + "/newton_residual.f64", std::vector<double>(Y.begin(), Y.end()));
      std::ofstream o(c.out + "/newton.txt");
      o.precision(17);
      o << "newton_norm " << nr << "\n";
    }
  }
  // Dual problem (optional): StdMultiLevelSolver::AssembleDualMatrix
  // (Solver/stdmultilevelsolver.cc:920-926, Solver/stdsolver.cc:1815-1834:
  // transpose, Dirichlet rows) and the same Gmres on it, right-hand side read
  // like rhs and zeroed at Dirichlet nodes.
  int dual_iterations = -1;
  std::string dual_status = "none";
  double dual_first = 0, dual_last = 0;
  std::vector<double> dual_times;
  Vector z("z"), g("g");
  if (!c.dualrhs.empty()) {
    MLS.ReInitVector(z);
    MLS.ReInitVector(g);
    GlobalVector& Gv = S->GetGV(g);
    size_t nlex = 1;
    for (int d = 0; d < c.dim; ++d)
      nlex *= Nf + 1;
    std::vector<double> r = read_f64(c.dualrhs, nlex);
    for (int i = 0; i < nf; ++i) {
      long ix, iy, iz = 0;
      if (c.dim == 3) {
        const Vertex3d& v = Mf->vertex3d(i);
        ix = std::lround(v.x() * Nf);
        iy = std::lround(v.y() * Nf);
        iz = std::lround(v.z() * Nf);
      } else {
        const Vertex2d& v = Mf->vertex2d(i);
        ix = std::lround(v.x() * Nf);
        iy = std::lround(v.y() * Nf);
      }
      Gv(i, 0) = r[(iz * (Nf + 1) + iy) * (Nf + 1) + ix];
    }
    S->SetBoundaryVectorZero(g);
    MLS.AssembleDualMatrix(A, u);
    if (c.dump)
      for (int l = 0; l < nl; ++l) {
        const auto* M = dynamic_cast<const SparseBlockMatrix<FMatrixBlock<1>>*>(
          &MLS.GetSolver(l)->GetMatrix(A));
        const auto* ST = dynamic_cast<const ColumnDiagStencil*>(M->GetStencil());
        std::vector<double> val(ST->nentries());
        for (size_t p = 0; p < ST->nentries(); ++p)
          val[p] = (*M->mat(p))(0, 0);
        write_raw(c.out + "/L" + std::to_string(l) + "_dualval.f64", val);
      }
    CGInfo dinfo(c.tol, c.globaltol, 0, c.maxiter, "Dual");
    for (int rep = 0; rep < std::max(1, c.repeat); ++rep) {
      dinfo.reset();
      auto t0 = std::chrono::steady_clock::now();
      MLS.NewtonLinearSolve(A, z, g, dinfo);
      auto t1 = std::chrono::steady_clock::now();
      dual_times.push_back(std::chrono::duration<double>(t1 - t0).count());
    }
    dual_iterations = dinfo.control().iteration();
    dual_status = dinfo.control().status();
    dual_first = dinfo.control().firstresidual();
    dual_last = dinfo.control().residual();
    const GlobalVector& Z = S->GetGV(z);
    std::vector<double> zz(Z.begin(), Z.end());
    write_raw(c.out + "/dual_solution.f64", zz);
    std::vector<double> gg(Gv.begin(), Gv.end());
    write_raw(c.out + "/dual_rhs.f64", gg);
    std::ofstream o(c.out + "/dual_summary.txt");
    o.precision(17);
    o << "dual_iterations " << dual_iterations << "\n";
    o << "dual_status " << dual_status << "\n";
    o << "dual_firstresidual " << dual_first << "\n";
    o << "dual_residual " << dual_last << "\n";
    o << "dual_solve_s";
    for (double t : dual_times)
      o << " " << t;
    o << "\n";
  }

  return 0;
}

int
main(int argc, char** argv)
{
  try {
    return run(argc, argv);
  } catch (const std::exception& e) {
    fprintf(stderr, "ref_harness: %s\n", e.what());
    return 4;
  }
}
