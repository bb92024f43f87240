// Reference-side binding of the B200 linear-solve path: the classes a
// Gascoigne build compiles in (against its own headers) to run its multigrid
// GMRES solve on a B200 through the C-ABI of include/gascoigne_b200.h.
//
// They plug in where the reference's cuSPARSE backend plugs in
// (cuda/cudaloop.cc:24-31, cuda/cudamultilevelsolver.cc:71-104,
// cuda/cudasolver.h:60-108, cuda/cudamgintepolatornested.h):
//   B200Loop : StdLoop                       installs B200MultiLevelSolver
//   B200MultiLevelSolver : StdMultiLevelSolver
//                                            NewSolver, NewMgInterpolator,
//                                            NewtonLinearSolve (the whole GMRES
//                                            solve as one device call),
//                                            mgstep (device transfers)
//   B200Solver : StdSolver                   uploads the assembled matrix and
//                                            the level's mesh data; vector and
//                                            level operations on the device
//   B200MgInterpolatorNested : MgInterpolatorNested
//                                            restrict_zero / prolongate_add on
//                                            device vectors
//
// Vector residency. A Gascoigne Vector is a name with one GlobalVector per
// level (Solver/ghostagent.h:41-140). The binding keeps, per (level, name),
// which copy is current: the host GlobalVector, the device vector, or both.
// A device operation uploads a stale device copy first and leaves the host
// copy stale; StdSolver::GetGV (the only way host code reaches a
// GlobalVector) is overridden to download a stale host copy first. So the
// reference's own host code (Newton loop, Form, output) and the device path
// can be mixed freely, and each vector crosses PCIe only when the other side
// needs it.
#ifndef GASCOIGNE_B200_BINDING_H
#define GASCOIGNE_B200_BINDING_H

#include <map>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "gascoigne_b200.h"
#include "mginterpolatornested.h"
#include "stdloop.h"
#include "stdmultilevelsolver.h"
#include "stdsolver.h"

namespace Gascoigne {

class B200Solver;

// State shared by the solvers and interpolators of one multilevel solver:
// the C-ABI context, the vector ids of Gascoigne's vector names and their
// residency per level.
class B200Device
{
public:
  struct Copy
  {
    bool host = true; // the GlobalVector is current
    bool dev = false; // the device vector is current
  };

  explicit B200Device(int device);
  ~B200Device();
  B200Device(const B200Device&) = delete;
  B200Device& operator=(const B200Device&) = delete;

  gb_ctx* ctx() const { return ctx_; }
  // throws std::runtime_error with the C-ABI's message when rc != GB_OK
  void check(int rc, const char* what) const;

  void reset_levels(int nlevels);
  int nlevels() const { return static_cast<int>(solvers_.size()); }
  void set_solver(int level, B200Solver* s) { solvers_.at(level) = s; }
  B200Solver* solver(int level) const { return solvers_.at(level); }

  // the C-ABI id of a vector name (one id names the vector on every level)
  int id(const std::string& name);
  Copy& copy(int level, const std::string& name) { return res_[{ level, name }]; }
  void forget(int level, const std::string& name) { res_.erase({ level, name }); }
  void forget_device(int level); // a level's device vectors are gone

  bool matrix_on_device(int level) const { return matrix_.at(level).size() > 0; }
  const std::string& matrix_name(int level) const { return matrix_.at(level); }
  void set_matrix_name(int level, const std::string& m) { matrix_.at(level) = m; }

private:
  gb_ctx* ctx_ = nullptr;
  std::vector<B200Solver*> solvers_;
  std::vector<std::string> matrix_;
  std::map<std::string, int> ids_;
  std::map<std::pair<int, std::string>, Copy> res_;
};

class B200Solver : public StdSolver
{
public:
  B200Solver(std::shared_ptr<B200Device> dev, int level);

  std::string GetName() const override { return "B200Solver"; }

  // mesh, problem and matrix: StdSolver's work, then the upload
  void NewMesh(const GascoigneMesh* mp) override;
  void SetProblem(const ProblemDescriptorInterface& PDX) override;
  void AssembleMatrix(Matrix& A, const Vector& u, double d) const override;
  void AssembleDualMatrix(Matrix& A, const Vector& gu, double d) override;

  // host access with residency
  void ReInitVector(Vector& dst, int comp) override;
  using StdSolver::ReInitVector;
  void DeleteVector(Vector& p) const override;
  GlobalVector& GetGV(Vector& u) const override;
  const GlobalVector& GetGV(const Vector& u) const override;

  // level operations on the device (StdSolver's on the host until the
  // level's matrix has been uploaded)
  void vmult(const Matrix& A, Vector& y, const Vector& x, double d) const override;
  void vmulteq(const Matrix& A, Vector& y, const Vector& x, double d) const override;
  void residualgmres(const Matrix& A, Vector& y, const Vector& x,
                     const Vector& b) const override;
  void MatrixResidual(const Matrix& A, Vector& y, const Vector& x,
                      const Vector& b) const override;
  void Zero(Vector& dst) const override;
  void Equ(Vector& dst, double s, const Vector& src) const override;
  void Add(Vector& dst, double s, const Vector& src) const override;
  double Norm(const Vector& dst) const override;
  double ScalarProduct(const Vector& y, const Vector& x) const override;
  void HNAverage(const Vector& x) const override;
  void HNZero(const Vector& x) const override;
  void HNDistribute(Vector& x) const override;
  void SetBoundaryVectorZero(Vector& gf) const override;
  void SubtractMean(Vector& x) const override;
  void SubtractMeanAlgebraic(Vector& x) const override;

  // residency helpers (also used by the multilevel solver and interpolators)
  int dev_in(const Vector& v) const;    // device copy made current, host kept
  int dev_out(Vector& v) const;         // device copy will be overwritten
  int dev_inout(const Vector& v) const; // read and written on the device
  bool on_device() const;               // this level's matrix is uploaded
  int level() const { return level_; }
  // the reference's key values this level's solver was configured with
  const std::string& matrixtype() const { return _matrixtype; }
  int ndirect_key() const { return _ndirect; }
  const SolverData& solver_data() const { return GetSolverData(); }
  // uploads Dirichlet nodes, hanging nodes, Vanka patches and the pressure
  // filter after a matrix upload (they follow the matrix's size)
  void upload_level_data() const;

protected:
  void smooth(int niter, const Matrix& A, Vector& x, const Vector& y,
              Vector& h) const override;

private:
  void upload_matrix(const Matrix& A) const;
  void require_matrix(const Matrix& A) const;
  GlobalVector& host(const Vector& v) const; // the GlobalVector, no sync
  void to_host(const Vector& v) const;

  std::shared_ptr<B200Device> D_;
  int level_;
};

// restrict_zero / prolongate_add on device vectors between level `coarse` and
// coarse + 1; the GlobalVector overloads (MgInterpolatorNested's host
// versions) stay for host callers such as SolutionTransfer.
class B200MgInterpolatorNested : public MgInterpolatorNested
{
public:
  B200MgInterpolatorNested(std::shared_ptr<B200Device> dev, int coarse);
  void BasicInit(const MeshTransferInterface* MT) override;
  using MgInterpolatorNested::prolongate_add;
  using MgInterpolatorNested::restrict_zero;
  void restrict_zero(Vector& coarse, const Vector& fine) const;
  void prolongate_add(Vector& fine, const Vector& coarse) const;
  // the maps go to the device once both levels hold their matrix
  void upload() const;

private:
  std::shared_ptr<B200Device> D_;
  int coarse_;
  mutable bool uploaded_ = false;
};

class B200MultiLevelSolver : public StdMultiLevelSolver
{
public:
  explicit B200MultiLevelSolver(int device = 0);
  std::string GetName() const override { return "B200MultiLevelSolver"; }

  void NewSolvers() override;
  StdSolver* NewSolver(int solverlevel) override;
  void NewMgInterpolator() override;

  // NewtonLinearSolve (Zero(x), Gmres, SubtractMean(x)) as one device call
  // (gb_gmres) when the configuration is one the device solver follows step
  // for step: linearsolve gmres on the finest level, the multigrid cycle down
  // to level 0, Jacobi / Vanka / block-ILU smoothing. Otherwise, or with
  // SetDeviceGmres(false), the reference's own NewtonLinearSolve, Gmres
  // (GMRES::solve) and LinearMg drive the device operations of B200Solver and
  // B200MgInterpolatorNested from the host.
  void NewtonLinearSolve(const Matrix& A, Vector& x, const Vector& b,
                         CGInfo& info) override;
  void mgstep(std::vector<double>& res, std::vector<double>& rw, int l,
              int finelevel, int coarselevel, std::string& p0, std::string p,
              const Matrix& A, Vector& u, Vector& b, Vector& v) override;

  // device GMRES (default) or the reference's host-driven GMRES over device
  // operations
  void SetDeviceGmres(bool on) { device_gmres_ = on; }
  // which device solver NewtonLinearSolve runs: kReference (gb_gmres, the
  // reference's left-preconditioned GMRES step for step), kFlexible64 or
  // kFlexible32 (gb_fgmres: FP64 flexible GMRES around an FP64 or FP32
  // multigrid cycle, restarted on the true FP64 residual until
  // ||b - A x|| <= tol ||b||; its stopping test is the true residual, so its
  // iteration counts differ from the reference's)
  enum DeviceSolver { kReference = 0, kFlexible64 = 1, kFlexible32 = 2 };
  void SetDeviceSolver(DeviceSolver s) { solver_ = s; }
  void SetMixedPrecision(bool on) { solver_ = on ? kFlexible32 : kReference; }
  // Krylov memory of the flexible solves (0: the parameter file's gmressize)
  void SetFlexibleMemory(int gmressize) { flex_m_ = gmressize; }
  // the C-ABI context (for instrumentation such as gb_bench_spmv)
  gb_ctx* DeviceContext() const { return D_->ctx(); }
  // the last device solve's record (iterations, residuals, device time)
  const gb_solve_info& LastSolveInfo() const { return last_; }

private:
  bool device_gmres_ok(std::string* why);
  void push_params(const CGInfo& info);
  void upload_transfers();

  std::shared_ptr<B200Device> D_;
  bool device_gmres_ = true;
  DeviceSolver solver_ = kReference;
  int flex_m_ = 0;
  gb_solve_info last_{};
};

class B200Loop : public StdLoop
{
public:
  void BasicInit(const ParamFile& paramfile, const ProblemContainer* PC,
                 const FunctionalContainer* FC) override;
};

} // namespace Gascoigne

#endif
