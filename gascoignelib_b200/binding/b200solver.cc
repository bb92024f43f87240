// Reference-side binding of the B200 linear-solve path (see b200solver.h).
#include "b200solver.h"

#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "cginfo.h"
#include "columndiagstencil.h"
#include "dirichletdata.h"
#include "fmatrixblock.h"
#include "gascoignemesh.h"
#include "gascoignemeshtransfer.h"
#include "pressurefilter.h"
#include "problemdescriptorinterface.h"
#include "sparseblockmatrix.h"

namespace Gascoigne {

// ------------------------------------------------------------------ device

B200Device::B200Device(int device)
{
  if (gb_ctx_create(&ctx_, device) != GB_OK || !ctx_)
    throw std::runtime_error("B200Device: gb_ctx_create failed (no usable GPU?)");
}

B200Device::~B200Device()
{
  if (ctx_)
    gb_ctx_destroy(ctx_);
}

void
B200Device::check(int rc, const char* what) const
{
  if (rc != GB_OK)
    throw std::runtime_error(std::string("B200 ") + what + ": " +
                             gb_last_error_string(ctx_));
}

void
B200Device::reset_levels(int nlevels)
{
  check(gb_set_nlevels(ctx_, nlevels), "gb_set_nlevels");
  solvers_.assign(nlevels, nullptr);
  matrix_.assign(nlevels, std::string());
  for (auto& r : res_)
    r.second.dev = false, r.second.host = true;
}

int
B200Device::id(const std::string& name)
{
  auto it = ids_.find(name);
  if (it != ids_.end())
    return it->second;
  int v = 0;
  check(gb_vec_create(ctx_, &v), "gb_vec_create");
  ids_[name] = v;
  return v;
}

void
B200Device::forget_device(int level)
{
  for (auto& r : res_)
    if (r.first.first == level && r.second.dev) {
      // a level whose matrix was replaced may change size: keep the host copy
      r.second.dev = false;
      r.second.host = true;
    }
}

// ------------------------------------------------------------------ solver

namespace {

// PressureFilter keeps its components, domain size and hanging-node count
// protected; the filter's upload reads them through this view.
struct PressureFilterView : public PressureFilter
{
  const IntVector& comps() const { return component; }
  double domain() const { return domainsize; }
  int hanging() const { return nhanging; }
};

template<int B>
bool
block_matrix(const MatrixInterface& MI, std::vector<int64_t>& rp,
             std::vector<int64_t>& cl, std::vector<int64_t>& dg,
             std::vector<double>& val, int& nb)
{
  const auto* M = dynamic_cast<const SparseBlockMatrix<FMatrixBlock<B>>*>(&MI);
  if (!M)
    return false;
  const auto* ST = dynamic_cast<const ColumnDiagStencil*>(M->GetStencil());
  if (!ST)
    throw std::runtime_error("B200Solver: matrix stencil is not a ColumnDiagStencil");
  const int64_t n = ST->n();
  rp.resize(n + 1);
  dg.resize(n);
  cl.resize(ST->nentries());
  val.resize(ST->nentries() * B * B);
  for (int64_t i = 0; i <= n; ++i)
    rp[i] = ST->start(i);
  for (int64_t i = 0; i < n; ++i)
    dg[i] = ST->diag(i);
  for (size_t p = 0; p < ST->nentries(); ++p) {
    cl[p] = ST->col(p);
    for (int r = 0; r < B; ++r)
      for (int q = 0; q < B; ++q) // NodeMatrix::value is row-major
        val[(p * B + r) * B + q] = (*M->mat(p))(r, q);
  }
  nb = B;
  return true;
}

} // namespace

B200Solver::B200Solver(std::shared_ptr<B200Device> dev, int level)
  : StdSolver()
  , D_(std::move(dev))
  , level_(level)
{}

bool
B200Solver::on_device() const
{
  return D_->matrix_on_device(level_);
}

void
B200Solver::NewMesh(const GascoigneMesh* mp)
{
  StdSolver::NewMesh(mp);
  // the level's mesh data follow the next matrix upload
  D_->set_matrix_name(level_, std::string());
  D_->forget_device(level_);
}

void
B200Solver::SetProblem(const ProblemDescriptorInterface& PDX)
{
  StdSolver::SetProblem(PDX);
  if (on_device())
    upload_level_data();
}

void
B200Solver::AssembleMatrix(Matrix& A, const Vector& u, double d) const
{
  StdSolver::AssembleMatrix(A, u, d);
  upload_matrix(A);
}

void
B200Solver::AssembleDualMatrix(Matrix& A, const Vector& gu, double d)
{
  // transpose, Dirichlet rows (Solver/stdsolver.cc:1815-1834) on the host,
  // then the dual matrix becomes the level's device operator
  StdSolver::AssembleDualMatrix(A, gu, d);
  upload_matrix(A);
}

void
B200Solver::upload_matrix(const Matrix& A) const
{
  const MatrixInterface& MI = StdSolver::GetMatrix(A);
  std::vector<int64_t> rp, cl, dg;
  std::vector<double> val;
  int B = 0;
  if (!block_matrix<1>(MI, rp, cl, dg, val, B) && !block_matrix<2>(MI, rp, cl, dg, val, B) &&
      !block_matrix<3>(MI, rp, cl, dg, val, B) && !block_matrix<4>(MI, rp, cl, dg, val, B))
    throw std::runtime_error("B200Solver: matrix " + A +
                             " is not a SparseBlockMatrix<FMatrixBlock<B>>, B = 1..4");
  const bool same_size = D_->matrix_on_device(level_);
  D_->check(gb_level_set_matrix(D_->ctx(), level_, static_cast<int64_t>(dg.size()), B,
                                rp.data(), cl.data(), dg.data(), val.data()),
            "gb_level_set_matrix");
  if (!same_size)
    D_->forget_device(level_);
  D_->set_matrix_name(level_, A);
  upload_level_data();
}

void
B200Solver::upload_level_data() const
{
  gb_ctx* c = D_->ctx();
  const GascoigneMesh* M = GetMesh();
  const ProblemDescriptorInterface* PD = GetProblemDescriptor();
  const int ncomp = PD->GetNcomp();
  // Dirichlet nodes per colour with that colour's components
  // (CGDisc::StrongDirichletVectorZero, DofHandler/cgdisc.h:1162-1179)
  std::vector<int64_t> nodes;
  std::vector<int> masks;
  if (const DirichletData* DD = PD->GetDirichletData()) {
    std::map<int64_t, int> m;
    for (int col : DD->dirichlet_colors()) {
      int mask = 0;
      for (int comp : DD->components_on_color(col))
        mask |= 1 << comp;
      if (const IntVector* bv = M->VertexOnBoundary(col))
        for (int i : *bv)
          m[i] |= mask;
    }
    for (auto& e : m)
      nodes.push_back(e.first), masks.push_back(e.second);
  }
  D_->check(gb_level_set_dirichlet_masks(c, level_, static_cast<int64_t>(nodes.size()),
                                         nodes.data(), masks.data()),
            "gb_level_set_dirichlet_masks");
  // hanging nodes (Mesh/hangingindexhandler.h:40,65) with the discretisation's
  // HNStructure: Q12d, Q13d, Q22d, Q23d (DofHandler/cgdisc.cc:24-50)
  const HangingIndexHandler& HI = M->GetHangingIndexHandler();
  std::vector<int64_t> e, f;
  for (const auto& h : *HI.GetStructure()) {
    e.push_back(h.first);
    for (int q : h.second)
      e.push_back(q);
  }
  for (const auto& h : *HI.GetStructureFace()) {
    f.push_back(h.first);
    for (int q : h.second)
      f.push_back(q);
  }
  if (!e.empty() || !f.empty()) {
    const int disc = (_discname.find("Q2") != std::string::npos ? 2 : 0) +
                     (M->dimension() == 3 ? 1 : 0);
    D_->check(gb_level_set_hn(c, level_, disc, static_cast<int64_t>(e.size() / 4), e.data(),
                              static_cast<int64_t>(f.size() / 10), f.data()),
              "gb_level_set_hn");
  }
  // Vanka patches (VankaSmoother::ConstructStructure, LinAlg/vankasmoother.cc:7-63)
  if (_matrixtype == "vanka" && M->npatches() > 0) {
    std::vector<int64_t> pl;
    int npp = 0;
    for (int p = 0; p < M->npatches(); ++p) {
      const IntVector& ip = *M->IndicesOfPatch(p);
      npp = static_cast<int>(ip.size());
      for (int i : ip)
        pl.push_back(i);
    }
    D_->check(gb_level_set_patches(c, level_, M->npatches(), npp, pl.data()),
              "gb_level_set_patches");
  }
  // pressure filter (CGDisc::InitFilter at StdSolver::NewMesh)
  const auto& PF = static_cast<const PressureFilterView&>(GetPfilter());
  if (PF.Active()) {
    int mask = 0;
    for (int comp : PF.comps())
      mask |= 1 << comp;
    std::vector<double> w(PF.begin(), PF.end());
    D_->check(gb_level_set_pfilter(c, level_, mask, w.data(), PF.domain(), PF.hanging()),
              "gb_level_set_pfilter");
  }
  (void)ncomp;
}

void
B200Solver::require_matrix(const Matrix& A) const
{
  if (D_->matrix_name(level_) != static_cast<const std::string&>(A))
    throw std::runtime_error("B200Solver: matrix " + A + " is not the one on the device (" +
                             D_->matrix_name(level_) + ") on level " +
                             std::to_string(level_));
}

// --- residency

GlobalVector&
B200Solver::host(const Vector& v) const
{
  return StdSolver::GetGV(const_cast<Vector&>(v));
}

void
B200Solver::to_host(const Vector& v) const
{
  B200Device::Copy& r = D_->copy(level_, v);
  if (r.host)
    return;
  GlobalVector& g = host(v);
  D_->check(gb_vec_download(D_->ctx(), level_, D_->id(v), g.data(),
                            static_cast<int64_t>(g.size())),
            "gb_vec_download");
  r.host = true;
}

GlobalVector&
B200Solver::GetGV(Vector& u) const
{
  to_host(u);
  D_->copy(level_, u).dev = false; // the caller may write through it
  return host(u);
}

const GlobalVector&
B200Solver::GetGV(const Vector& u) const
{
  to_host(u);
  return host(u);
}

int
B200Solver::dev_in(const Vector& v) const
{
  const int id = D_->id(v);
  B200Device::Copy& r = D_->copy(level_, v);
  if (!r.dev) {
    GlobalVector& g = host(v);
    D_->check(gb_vec_upload(D_->ctx(), level_, id, g.data(), static_cast<int64_t>(g.size())),
              "gb_vec_upload");
    r.dev = true;
  }
  return id;
}

int
B200Solver::dev_out(Vector& v) const
{
  const int id = D_->id(v);
  B200Device::Copy& r = D_->copy(level_, v);
  r.dev = true;
  r.host = false;
  return id;
}

int
B200Solver::dev_inout(const Vector& v) const
{
  const int id = dev_in(v);
  D_->copy(level_, v).host = false;
  return id;
}

void
B200Solver::ReInitVector(Vector& dst, int comp)
{
  StdSolver::ReInitVector(dst, comp);
  B200Device::Copy& r = D_->copy(level_, dst);
  r.host = true; // freshly zeroed on the host
  r.dev = false;
}

void
B200Solver::DeleteVector(Vector& p) const
{
  StdSolver::DeleteVector(p);
  D_->forget(level_, p);
}

// --- level operations

void
B200Solver::vmult(const Matrix& A, Vector& y, const Vector& x, double d) const
{
  if (!on_device())
    return StdSolver::vmult(A, y, x, d);
  require_matrix(A);
  const int ix = dev_in(x), iy = dev_inout(y);
  D_->check(gb_vmult(D_->ctx(), level_, iy, ix, d), "gb_vmult");
}

void
B200Solver::vmulteq(const Matrix& A, Vector& y, const Vector& x, double d) const
{
  if (!on_device())
    return StdSolver::vmulteq(A, y, x, d);
  require_matrix(A);
  const int ix = dev_in(x), iy = dev_out(y);
  D_->check(gb_vmulteq(D_->ctx(), level_, iy, ix, d), "gb_vmulteq");
}

void
B200Solver::residualgmres(const Matrix& A, Vector& y, const Vector& x,
                          const Vector& b) const
{
  if (!on_device())
    return StdSolver::residualgmres(A, y, x, b);
  require_matrix(A);
  const int ix = dev_in(x), ib = dev_in(b), iy = dev_out(y);
  D_->check(gb_residualgmres(D_->ctx(), level_, iy, ix, ib), "gb_residualgmres");
}

void
B200Solver::MatrixResidual(const Matrix& A, Vector& y, const Vector& x,
                           const Vector& b) const
{
  if (!on_device())
    return StdSolver::MatrixResidual(A, y, x, b);
  require_matrix(A);
  const int ix = dev_in(x), ib = dev_in(b), iy = dev_out(y);
  D_->check(gb_matrix_residual(D_->ctx(), level_, iy, ix, ib), "gb_matrix_residual");
}

void
B200Solver::smooth(int niter, const Matrix& A, Vector& x, const Vector& y, Vector& h) const
{
  if (!on_device())
    return StdSolver::smooth(niter, A, x, y, h);
  require_matrix(A);
  const std::string ls = GetSolverData().GetLinearSmooth();
  if (ls != "jacobi" && ls != "ilu")
    throw std::runtime_error("B200Solver: linear_smooth " + ls +
                             " has no device smoother (jacobi, ilu)");
  gb_params p;
  D_->check(gb_get_params(D_->ctx(), &p), "gb_get_params");
  const int want = ls == "jacobi" ? 0 : (_matrixtype == "vanka" ? 1 : 2);
  const double omega = GetSolverData().GetOmega();
  if (p.smoother != want || p.omega != omega) {
    p.smoother = want;
    p.omega = omega;
    D_->check(gb_set_params(D_->ctx(), &p), "gb_set_params");
  }
  const int iy = dev_in(y), ix = dev_inout(x), ih = dev_out(h);
  D_->check(gb_smooth(D_->ctx(), level_, niter, ix, iy, ih), "gb_smooth");
}

void
B200Solver::Zero(Vector& dst) const
{
  if (!on_device())
    return StdSolver::Zero(dst);
  D_->check(gb_vec_zero(D_->ctx(), level_, dev_out(dst)), "gb_vec_zero");
}

void
B200Solver::Equ(Vector& dst, double s, const Vector& src) const
{
  if (!on_device())
    return StdSolver::Equ(dst, s, src);
  const int is = dev_in(src);
  const int id = (&dst == &src || static_cast<const std::string&>(dst) == src)
                   ? dev_inout(dst)
                   : dev_out(dst);
  D_->check(gb_vec_equ(D_->ctx(), level_, id, s, is), "gb_vec_equ");
}

void
B200Solver::Add(Vector& dst, double s, const Vector& src) const
{
  if (!on_device())
    return StdSolver::Add(dst, s, src);
  const int is = dev_in(src), id = dev_inout(dst);
  D_->check(gb_vec_add(D_->ctx(), level_, id, s, is), "gb_vec_add");
}

double
B200Solver::Norm(const Vector& dst) const
{
  if (!on_device())
    return StdSolver::Norm(dst);
  double r = 0.0;
  D_->check(gb_vec_norm(D_->ctx(), level_, dev_in(dst), &r), "gb_vec_norm");
  return r;
}

double
B200Solver::ScalarProduct(const Vector& y, const Vector& x) const
{
  if (!on_device())
    return StdSolver::ScalarProduct(y, x);
  double r = 0.0;
  const int iy = dev_in(y), ix = dev_in(x);
  D_->check(gb_vec_dot(D_->ctx(), level_, iy, ix, &r), "gb_vec_dot");
  return r;
}

namespace {
bool
has_hanging(const GascoigneMesh* M)
{
  const HangingIndexHandler& HI = M->GetHangingIndexHandler();
  return !HI.GetStructure()->empty() || !HI.GetStructureFace()->empty();
}
} // namespace

void
B200Solver::HNAverage(const Vector& x) const
{
  if (!on_device())
    return StdSolver::HNAverage(x);
  if (has_hanging(GetMesh()))
    D_->check(gb_hn_average(D_->ctx(), level_, dev_inout(x)), "gb_hn_average");
}

void
B200Solver::HNZero(const Vector& x) const
{
  if (!on_device())
    return StdSolver::HNZero(x);
  if (has_hanging(GetMesh()))
    D_->check(gb_hn_zero(D_->ctx(), level_, dev_inout(x)), "gb_hn_zero");
}

void
B200Solver::HNDistribute(Vector& x) const
{
  if (!on_device())
    return StdSolver::HNDistribute(x);
  if (has_hanging(GetMesh()))
    D_->check(gb_hn_distribute(D_->ctx(), level_, dev_inout(x)), "gb_hn_distribute");
}

void
B200Solver::SetBoundaryVectorZero(Vector& gf) const
{
  if (!on_device())
    return StdSolver::SetBoundaryVectorZero(gf);
  D_->check(gb_dirichlet_zero(D_->ctx(), level_, dev_inout(gf)), "gb_dirichlet_zero");
}

void
B200Solver::SubtractMean(Vector& x) const
{
  if (!on_device())
    return StdSolver::SubtractMean(x);
  if (GetPfilter().Active())
    D_->check(gb_subtract_mean(D_->ctx(), level_, dev_inout(x)), "gb_subtract_mean");
}

void
B200Solver::SubtractMeanAlgebraic(Vector& x) const
{
  if (!on_device())
    return StdSolver::SubtractMeanAlgebraic(x);
  if (GetPfilter().Active())
    D_->check(gb_subtract_mean_algebraic(D_->ctx(), level_, dev_inout(x)),
              "gb_subtract_mean_algebraic");
}

// ------------------------------------------------------------ interpolator

B200MgInterpolatorNested::B200MgInterpolatorNested(std::shared_ptr<B200Device> dev,
                                                   int coarse)
  : MgInterpolatorNested()
  , D_(std::move(dev))
  , coarse_(coarse)
{}

void
B200MgInterpolatorNested::BasicInit(const MeshTransferInterface* MT)
{
  MgInterpolatorNested::BasicInit(MT);
  uploaded_ = false;
}

void
B200MgInterpolatorNested::upload() const
{
  if (uploaded_)
    return;
  auto* self = const_cast<B200MgInterpolatorNested*>(this);
  std::vector<int64_t> c2f(GetC2F().begin(), GetC2F().end()), z, v, a;
  for (const auto& p : self->GetZweier()) {
    z.push_back(p.first);
    for (int q : p.second)
      z.push_back(q);
  }
  for (const auto& p : self->GetVierer()) {
    v.push_back(p.first);
    for (int q : p.second)
      v.push_back(q);
  }
  for (const auto& p : self->GetAchter()) {
    a.push_back(p.first);
    for (int q : p.second)
      a.push_back(q);
  }
  D_->check(gb_level_set_transfer(D_->ctx(), coarse_, static_cast<int64_t>(c2f.size()),
                                  c2f.data(), static_cast<int64_t>(z.size() / 3), z.data(),
                                  static_cast<int64_t>(v.size() / 5), v.data(),
                                  static_cast<int64_t>(a.size() / 9), a.data()),
            "gb_level_set_transfer");
  uploaded_ = true;
}

void
B200MgInterpolatorNested::restrict_zero(Vector& coarse, const Vector& fine) const
{
  upload();
  const int fi = D_->solver(coarse_ + 1)->dev_in(fine);
  const int ci = D_->solver(coarse_)->dev_out(coarse);
  D_->check(gb_restrict_zero(D_->ctx(), coarse_, ci, fi), "gb_restrict_zero");
}

void
B200MgInterpolatorNested::prolongate_add(Vector& fine, const Vector& coarse) const
{
  upload();
  const int ci = D_->solver(coarse_)->dev_in(coarse);
  const int fi = D_->solver(coarse_ + 1)->dev_inout(fine);
  D_->check(gb_prolongate_add(D_->ctx(), coarse_, fi, ci), "gb_prolongate_add");
}

// --------------------------------------------------------- multilevel solver

B200MultiLevelSolver::B200MultiLevelSolver(int device)
  : StdMultiLevelSolver()
  , D_(std::make_shared<B200Device>(device))
{}

void
B200MultiLevelSolver::NewSolvers()
{
  // a different number of levels: every solver is new (their level indices
  // and the context's level data change together)
  if (static_cast<int>(GetSolverPointers().size()) != nlevels()) {
    for (auto*& s : GetSolverPointers()) {
      delete s;
      s = nullptr;
    }
    GetSolverPointers().clear();
  }
  if (D_->nlevels() != nlevels())
    D_->reset_levels(nlevels());
  StdMultiLevelSolver::NewSolvers();
  for (int l = 0; l < nlevels(); ++l)
    D_->set_solver(l, static_cast<B200Solver*>(GetSolver(l)));
}

StdSolver*
B200MultiLevelSolver::NewSolver(int solverlevel)
{
  return new B200Solver(D_, solverlevel);
}

void
B200MultiLevelSolver::NewMgInterpolator()
{
  if (DataP.LinearSolve() == "direct")
    return;
  for (auto*& I : _Interpolator) {
    delete I;
    I = nullptr;
  }
  _Interpolator.assign(nlevels() - 1, nullptr);
  // interpolator l maps level l+1 to level l, from mesh transfer
  // nlevels-l-2 (Solver/stdmultilevelsolver.cc:284-296)
  for (int l = 0; l < nlevels() - 1; ++l) {
    _Interpolator[l] = new B200MgInterpolatorNested(D_, l);
    GetSolver(l)->ConstructInterpolator(_Interpolator[l],
                                        GetMeshAgent()->GetTransfer(nlevels() - l - 2));
  }
}

void
B200MultiLevelSolver::upload_transfers()
{
  for (auto* I : _Interpolator)
    dynamic_cast<B200MgInterpolatorNested&>(*I).upload();
}

void
B200MultiLevelSolver::mgstep(std::vector<double>& res, std::vector<double>& rw, int l,
                             int finelevel, int coarselevel, std::string& p0,
                             std::string p, const Matrix& A, Vector& u, Vector& b,
                             Vector& v)
{
  // StdMultiLevelSolver::mgstep (Solver/stdmultilevelsolver.cc:462-531) with
  // the transfers on device vectors instead of GlobalVectors, as
  // CudaMultiLevelSolver::mgstep does (cuda/cudamultilevelsolver.cc:171-246)
  StdSolver* S = GetSolver(l);
  if (l == coarselevel) {
    if (p == "F")
      p0 = "V";
    S->smooth_exact(A, u, b, v);
    if (l == finelevel) {
      S->MatrixResidual(A, v, u, b);
      res[l] = S->Norm(v);
    }
    return;
  }
  StdSolver* C = GetSolver(l - 1);
  auto* I = dynamic_cast<B200MgInterpolatorNested*>(_Interpolator[l - 1]);
  S->smooth_pre(A, u, b, v);
  S->MatrixResidual(A, v, u, b);
  I->restrict_zero(b, v);
  C->HNDistribute(b);
  C->SetBoundaryVectorZero(b);
  C->Zero(u);
  const int visits = p0 == "V" ? 1 : (p0 == "W" ? 2 : (p0 == "F" ? 3 : 0));
  for (int i = 0; i < visits; ++i)
    mgstep(res, rw, l - 1, finelevel, coarselevel, p0, p, A, u, b, v);
  if (l == 0 && p == "F")
    p0 = "W";
  rw[l] = C->Norm(u);
  S->Zero(v);
  C->HNAverage(u);
  I->prolongate_add(v, u);
  C->HNZero(u);
  S->HNZero(v);
  S->SetBoundaryVectorZero(v);
  S->Add(u, DataP.MgOmega(), v);
  S->smooth_post(A, u, b, v);
  S->MatrixResidual(A, v, u, b);
  res[l] = S->Norm(v);
}

bool
B200MultiLevelSolver::device_gmres_ok(std::string* why)
{
  auto no = [why](const std::string& w) {
    if (why)
      *why = w;
    return false;
  };
  if (DataP.LinearSolve() != "gmres")
    return no("linearsolve is not gmres");
  if (ComputeLevel != FinestLevel())
    return no("ComputeLevel is not the finest level");
  // the cycle of precondition goes down to max(coarselevel, 0), or to the
  // finest direct level above it (Solver/stdmultilevelsolver.cc:411-425,940-952)
  if (DataP.CoarseLevel() != 0)
    return no("coarselevel is not 0");
  for (int l = 1; l < nlevels(); ++l)
    if (GetSolver(l)->DirectSolver())
      return no("a level above 0 is a direct level");
  const std::string ls =
    static_cast<const B200Solver*>(GetSolver())->solver_data().GetLinearSmooth();
  if (ls != "jacobi" && ls != "ilu")
    return no("linear_smooth " + ls + " has no device smoother");
  for (int l = 0; l < nlevels(); ++l)
    if (!static_cast<B200Solver*>(GetSolver(l))->on_device())
      return no("level " + std::to_string(l) + " has no matrix on the device");
  return true;
}

void
B200MultiLevelSolver::push_params(const CGInfo& info)
{
  const auto* B = static_cast<const B200Solver*>(GetSolver());
  const SolverData& SD = B->solver_data();
  gb_params p;
  D_->check(gb_get_params(D_->ctx(), &p), "gb_get_params");
  p.iterpre = SD.GetIterPre();
  p.iterpost = SD.GetIterPost();
  p.iterexact = SD.GetIterExact();
  p.omega = SD.GetOmega();
  p.mgomega = DataP.MgOmega();
  p.mgtype = DataP.MgType().empty() ? 'V' : DataP.MgType()[0];
  p.gmressize = (solver_ != kReference && flex_m_ > 0) ? flex_m_ : DataP.GmresMemSize();
  p.tol = info.user().tol();
  p.globaltol = info.user().globaltol();
  p.maxiter = info.user().maxiter();
  const std::string ls = SD.GetLinearSmooth();
  p.smoother = ls == "jacobi" ? 0 : (B->matrixtype() == "vanka" ? 1 : 2);
#ifdef __WITH_UMFPACK__
  // level 0 solved exactly (the UMFPACK branch of StdSolver::smooth_exact)
  p.ndirect = GetSolver(0)->DirectSolver() ? GetSolver(0)->GetMesh()->nnodes() + 1 : 0;
#else
  // without UMFPACK a direct level is smoothed with iterexact sweeps
  p.ndirect = 0;
#endif
  D_->check(gb_set_params(D_->ctx(), &p), "gb_set_params");
}

void
B200MultiLevelSolver::NewtonLinearSolve(const Matrix& A, Vector& x, const Vector& b,
                                        CGInfo& info)
{
  std::string why;
  if (!device_gmres_ || !device_gmres_ok(&why)) {
    // the reference's own control flow (GMRES::solve, LinearMg, mgstep) over
    // the device operations of B200Solver and B200MgInterpolatorNested
    StdMultiLevelSolver::NewtonLinearSolve(A, x, b, info);
    return;
  }
  // the whole solve on the device: Zero(x), Gmres, SubtractMean(x)
  // (Solver/stdmultilevelsolver.cc:646-673)
  info.reset();
  upload_transfers();
  push_params(info);
  auto* S = static_cast<B200Solver*>(GetSolver(ComputeLevel));
  const int ib = S->dev_in(b);
  const int ix = S->dev_out(x);
  last_ = gb_solve_info{};
  const int rc =
    solver_ == kReference
      ? gb_gmres(D_->ctx(), ix, ib, &last_)
      : gb_fgmres(D_->ctx(), ix, ib, solver_ == kFlexible32 ? GB_FP32 : GB_FP64, &last_);
  if (rc != GB_OK && rc != GB_ENOTCONV)
    D_->check(rc, solver_ == kReference ? "gb_gmres" : "gb_fgmres");
  // CGInfo as GMRES::solve leaves it (Common/cginfo.cc:201-255)
  static const char* kStatus[] = { "waiting", "running", "converged", "too many iterations",
                                   "exploded" };
  ControlData& cd = info.control();
  cd.iteration() = last_.iterations;
  cd.status() = (last_.status >= 0 && last_.status <= 4) ? kStatus[last_.status] : "running";
  cd.firstresidual() = last_.firstresidual;
  cd.residual() = last_.residual;
  cd.aimedresidual() = last_.firstresidual * info.user().tol();
}

// ------------------------------------------------------------------- loop

void
B200Loop::BasicInit(const ParamFile& paramfile, const ProblemContainer* PC,
                    const FunctionalContainer* FC)
{
  // as CudaLoop::BasicInit (cuda/cudaloop.cc:24-31)
  GetMultiLevelSolverPointer() = new B200MultiLevelSolver;
  StdLoop::BasicInit(paramfile, PC, FC);
}

} // namespace Gascoigne
