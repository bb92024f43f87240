// Internal header: the steps of the multigrid cycle (Emit) and the cycle's
// entry points, defined in gb_cycle.cu.
#pragma once
#include "gb_context.cuh"

namespace gb {
// ------------------------------------------------------------ smoothing

// ------------------------------------------------------------ cycle steps
//
// Every step of the cycle goes through Emit: it either launches the step's
// kernel on the context stream, or (rec set) appends it to the program of the
// coarse-level kernel.
// mask of the prolonged correction on a fine level: SetBoundaryVectorZero and
// HNZero (the hanging dofs), Solver/stdmultilevelsolver.cc:515-517
inline const uint8_t*
pmask_of(const Level& L)
{
  return L.has_hn() ? L.pmask.p : L.dirmask.p;
}

template<class T>
struct Emit
{
  Context& c;
  std::vector<CoarseOp>* rec = nullptr;
  int no_dense_at = -1; // level whose dense map is being built (run its steps)
  bool mid = false;     // recording the multi-CTA program (coarse root: dense op)

  CoarseOp level_op(int kind, const Level& L, void* out, const void* in,
                    const void* b, double alpha) const
  {
    CoarseOp o{};
    o.kind = kind;
    o.n = static_cast<int>(L.ndof());
    o.out = out;
    o.in = in;
    o.b = b;
    o.in_n = in ? o.n : 0;
    o.b_n = b ? o.n : 0;
    const Sell& A = opA(c, L);
    GB_REQUIRE(!A.sorted || mid, GB_EINVAL, "coarse-level program on a row-sorted matrix");
    o.sptr = A.sptr.p;
    o.col = A.pat ? nullptr : A.col.p;
    o.pid = A.pat ? A.pid.p : nullptr;
    o.ptab = A.pat ? A.ptab.p : nullptr;
    o.W = A.W;
    o.val = sell_vals<T>(A);
    o.perm = A.sorted ? A.rperm.p : nullptr;
    o.dinv = dinv_of<T>(L);
    o.mask = L.dirmask.p;
    o.alpha = alpha;
    return o;
  }
  void jacobi_zero(int l, T* u, const T* b);
  // out = two Jacobi sweeps from 0 (scalar levels)
  void jacobi_two_from_zero(int l, T* out, const T* b);
  // u = (u_zero ? 0 : u) + omega D^-1 h (block Jacobi update, h given;
  // h's filtered component read minus *hmean when set; the weighted mean of
  // the new u reduced into scal[9] when the level has one filtered component)
  void jacobi_apply(int l, const T* h, T* u, bool u_zero, const double* hmean = nullptr);
  // u = (u_zero ? 0 : u) + omega * Vanka(h) (VankaSmoother::solve + Add)
  void vanka(int l, const T* h, T* u, bool u_zero, const double* hmean = nullptr);
  // The single filtered component of a level (-1: no filter, or several
  // components, which take the unfused pf_sub path).
  static int pf_comp(const Level& L);
  // weighted mean of the updated iterate reduced by the update kernel
  void check_pf_scratch(const Level& L) const;
  PfArgs weighted_mean_args(const Level& L) const;
  // out = b - A u (MatrixResidual) with the algebraic mean of the filtered
  // component left in scal[8] for the consumers to subtract on read.
  const double* resid_mean(int l, const T* u, T* out, const T* b);
  // scal[8] = algebraic (or, weighted, the integral) mean of the filtered
  // component of x
  const double* mean_of(int l, const T* x, bool weighted);
  // x(., pc) -= *mean
  void sub_mean(int l, T* x, const double* mean);
  // HNStructure::Average / Distribute / Zero on level l
  void hn_average(int l, T* u);
  void hn_distribute(int l, T* u);
  void hn_zero(int l, T* u);
  void dirichlet_zero(int l, T* u);
  // pressure filter on x: weighted (SubtractMean) or algebraic
  // (SubtractMeanAlgebraic) mean of every filtered component removed
  void pf_sub(int l, T* x, bool weighted);
  void copy(int l, T* dst, const T* src);
  // h = ILU^-1 h in place (SparseBlockIlu::solve with the identity order: the
  // level kernels of the forward, then of the backward substitution)
  void ilu_solve(int l, T* h);
  // u = (u_zero ? 0 : u) + omega h
  void ilu_axpy(int l, T* u, const T* h, bool u_zero);
  void no_rec() const;
  using TV_of = T;
  static const T* vk_lu(const Level& L);
  static T* vk_out(const Level& L);
  void jacobi(int l, const T* u, T* out, const T* b);
  void resid(int l, const T* u, T* out, const T* b);
  // coarse (level l) = R fine, 0 on the coarse Dirichlet dofs; with smean
  // (block levels) the filtered component of fine is read minus *smean; with
  // u1 (scalar levels) the restriction also writes the coarse level's first
  // Jacobi sweep from 0, u1 = omega D^-1 coarse
  void restrict_to(int l, const T* fine, T* coarse, const double* smean = nullptr,
                   T* u1 = nullptr);
  // u = A^-1 b on level 0 (the direct coarse solve)
  void direct(int l, T* u, const T* b);
  void fill0(int l, T* u);
  // fine (level l+1) += mgomega * (dir ? 0 : P coarse)
  void prolong(int l, const T* coarse, T* fine);
};

template<>
inline const double* Emit<double>::vk_lu(const Level& L)
{
  return L.vk_inv64.p;
}
template<>
inline const float* Emit<float>::vk_lu(const Level& L)
{
  return L.vk_inv32.p;
}
template<>
inline double* Emit<double>::vk_out(const Level& L)
{
  return L.vk_out64.p;
}
template<>
inline float* Emit<float>::vk_out(const Level& L)
{
  return L.vk_out32.p;
}


// ---------------------------------------------- defined in gb_cycle.cu
// (instantiated there for double and float)

template<class T>
void smooth(Emit<T>& E, int l, int niter, T*& u, T*& tmp, const T* b, bool& u_zero);
template<class T>
void precondition_T(Context& c, MgWork<T>& W, T* x, const T* y, bool x_zero,
                    bool first_done = false);
template<class T>
T* precondition_first_sweep(Context& c, MgWork<T>& W, T* x);

} // namespace gb
