// The multigrid cycle: smoothing, mgstep, the coarse-level and mid-level
// programs, precondition.
#include "gb_cycle.cuh"

namespace gb {

// ------------------------------------------------------- Emit's steps

template<class T>
void Emit<T>::jacobi_zero(int l, T* u, const T* b)
{
  const Level& L = c.L[l];
  if (rec)
    return rec->push_back(level_op(kOpJacobiZero, L, u, nullptr, b, c.params.omega));
  if (L.B == 1)
    launch(c, k_jacobi_from_zero<T, T>, blocks_for(L.n, 256), 256, (int)L.n,
           dinv_of<T>(L), b, u, c.params.omega);
  else
    jacobi_apply(l, b, u, true);
}

template<class T>
void Emit<T>::jacobi_two_from_zero(int l, T* out, const T* b)
{
  const Level& L = c.L[l];
  no_rec();
  spmv<kJacobi2, T, T, T>(c, L, opA(c, L), b, out, b, dinv_of<T>(L), c.params.omega);
}

template<class T>
void Emit<T>::jacobi_apply(int l, const T* h, T* u, bool u_zero, const double* hmean)
{
  const Level& L = c.L[l];
  no_rec();
  PfArgs pf = weighted_mean_args(L);
  pf.hmean = hmean;
  const int nb = blocks_for(L.n, 256);
  switch (L.B) {
    case 1:
      launch(c, k_block_jacobi_apply<1, T, T>, nb, 256, (int)L.n, dinv_of<T>(L), h, u,
             c.params.omega, int(u_zero), pf);
      break;
    case 2:
      launch(c, k_block_jacobi_apply<2, T, T>, nb, 256, (int)L.n, dinv_of<T>(L), h, u,
             c.params.omega, int(u_zero), pf);
      break;
    case 3:
      launch(c, k_block_jacobi_apply<3, T, T>, nb, 256, (int)L.n, dinv_of<T>(L), h, u,
             c.params.omega, int(u_zero), pf);
      break;
    default:
      launch(c, k_block_jacobi_apply<4, T, T>, nb, 256, (int)L.n, dinv_of<T>(L), h, u,
             c.params.omega, int(u_zero), pf);
  }
}

template<class T>
void Emit<T>::vanka(int l, const T* h, T* u, bool u_zero, const double* hmean)
{
  const Level& L = c.L[l];
  no_rec();
  const T* inv = vk_lu(L);
  T* out = vk_out(L);
  const int pc = pf_comp(L);
  const int nbp = blocks_for(L.npatch, kVankaWarps);
  if (L.vk_M == 27 || L.vk_M == 9) {
    if (L.vk_M == 27)
      launch(c, k_vanka_inv_ct<27, T, T>, nbp, 32 * kVankaWarps, L.npatch, L.B,
             (const int*)L.vk_pn.p, inv, h, pc, hmean, out);
    else
      launch(c, k_vanka_inv_ct<9, T, T>, nbp, 32 * kVankaWarps, L.npatch, L.B,
             (const int*)L.vk_pn.p, inv, h, pc, hmean, out);
  } else switch ((L.vk_M + 31) / 32) {
    case 1:
      launch(c, k_vanka_inv<1, T, T>, nbp, 32 * kVankaWarps, L.npatch, L.vk_M, L.B,
             (const int*)L.vk_pn.p, inv, h, pc, hmean, out);
      break;
    case 2:
      launch(c, k_vanka_inv<2, T, T>, nbp, 32 * kVankaWarps, L.npatch, L.vk_M, L.B,
             (const int*)L.vk_pn.p, inv, h, pc, hmean, out);
      break;
    case 3:
      launch(c, k_vanka_inv<3, T, T>, nbp, 32 * kVankaWarps, L.npatch, L.vk_M, L.B,
             (const int*)L.vk_pn.p, inv, h, pc, hmean, out);
      break;
    default:
      launch(c, k_vanka_inv<4, T, T>, nbp, 32 * kVankaWarps, L.npatch, L.vk_M, L.B,
             (const int*)L.vk_pn.p, inv, h, pc, hmean, out);
  }
  const PfArgs pf = weighted_mean_args(L);
  const int nb = blocks_for(L.n, 256);
  switch (L.B) {
    case 1:
      launch(c, k_vanka_gather<1, T>, nb, 256, (int)L.n, (const int*)L.vk_nptr.p,
             (const int*)L.vk_ent.p, (const T*)out, L.vk_M, u, c.params.omega,
             int(u_zero), pf);
      break;
    case 2:
      launch(c, k_vanka_gather<2, T>, nb, 256, (int)L.n, (const int*)L.vk_nptr.p,
             (const int*)L.vk_ent.p, (const T*)out, L.vk_M, u, c.params.omega,
             int(u_zero), pf);
      break;
    case 3:
      launch(c, k_vanka_gather<3, T>, nb, 256, (int)L.n, (const int*)L.vk_nptr.p,
             (const int*)L.vk_ent.p, (const T*)out, L.vk_M, u, c.params.omega,
             int(u_zero), pf);
      break;
    default:
      launch(c, k_vanka_gather<4, T>, nb, 256, (int)L.n, (const int*)L.vk_nptr.p,
             (const int*)L.vk_ent.p, (const T*)out, L.vk_M, u, c.params.omega,
             int(u_zero), pf);
  }
}

template<class T>
int Emit<T>::pf_comp(const Level& L)
{
  if (!L.pf_mask || (L.pf_mask & (L.pf_mask - 1)))
    return -1;
  return __builtin_ctz(static_cast<unsigned>(L.pf_mask));
}

template<class T>
void Emit<T>::check_pf_scratch(const Level& L) const
{
  GB_REQUIRE(c.pfpart.p && c.pfpart.n >= static_cast<size_t>((L.n + 255) / 256 + 1) &&
               c.pfticket.p,
             GB_ESTATE, "filter scratch not allocated for this level");
}

template<class T>
PfArgs Emit<T>::weighted_mean_args(const Level& L) const
{
  PfArgs a{};
  a.pc = pf_comp(L);
  if (a.pc >= 0) {
    check_pf_scratch(L);
    a.w = L.pf_w.p;
    a.domain = L.pf_domain;
    a.partials = c.pfpart.p;
    a.ticket = c.pfticket.p;
    a.umean = c.scal.p + 9;
  }
  return a;
}

template<class T>
const double* Emit<T>::resid_mean(int l, const T* u, T* out, const T* b)
{
  const Level& L = c.L[l];
  no_rec();
  const int pc = pf_comp(L);
  const double denom = double(L.n - L.nhanging);
  const Sell& S = opA(c, L);
  if (L.B > 1) {
    check_pf_scratch(L);
    const SellView<T> A = view<T>(S, sell_vals<T>(S));
    const int nb = blocks_for(S.n, kSpmvThreads);
#define GB_RM(BB, PP)                                                                 \
launch(c, k_bspmv_resid_mean<BB, T, T, PP>, nb, kSpmvThreads, A, u, out, b, pc, denom, \
       c.pfpart.p, c.pfticket.p, c.scal.p + 8)
    if (L.B == 2) {
      if (S.pat) GB_RM(2, true); else GB_RM(2, false);
    } else if (L.B == 3) {
      if (S.pat) GB_RM(3, true); else GB_RM(3, false);
    } else {
      if (S.pat) GB_RM(4, true); else GB_RM(4, false);
    }
#undef GB_RM
    return c.scal.p + 8;
  }
  resid(l, u, out, b);
  return mean_of(l, out, false);
}

template<class T>
const double* Emit<T>::mean_of(int l, const T* x, bool weighted)
{
  const Level& L = c.L[l];
  no_rec();
  launch(c, k_comp_mean<T>, red_blocks(L.n), kRedThreads, (int)L.n, L.B, pf_comp(L), x,
         weighted ? (const double*)L.pf_w.p : nullptr,
         weighted ? L.pf_domain : double(L.n - L.nhanging), c.partials.p, c.ticket.p,
         c.scal.p + 8);
  return c.scal.p + 8;
}

template<class T>
void Emit<T>::sub_mean(int l, T* x, const double* mean)
{
  const Level& L = c.L[l];
  no_rec();
  launch(c, k_comp_sub<T>, stream_blocks(L.n), 256, (int)L.n, L.B, pf_comp(L), x, mean,
         1.0);
}

template<class T>
void Emit<T>::hn_average(int l, T* u)
{
  const Level& L = c.L[l];
  no_rec();
  for (const auto& ph : L.hn)
    launch(c, k_hn_average<T>, blocks_for(ph.nh, 128), 128, ph.nh, L.B,
           (const int*)ph.node.p, (const int*)ph.par.p, ph.nslots, ph.gsize,
           (const double*)ph.w.p, u);
}

template<class T>
void Emit<T>::hn_distribute(int l, T* u)
{
  const Level& L = c.L[l];
  no_rec();
  for (const auto& ph : L.hn) {
    launch(c, k_hn_distribute<T>, blocks_for(ph.np, 128), 128, ph.np, L.B,
           (const int*)ph.pnode.p, (const int*)ph.ptr.p, (const int*)ph.hnode.p,
           (const double*)ph.wt.p, u);
    launch(c, k_hn_zero<T>, blocks_for(ph.nh, 128), 128, ph.nh, L.B,
           (const int*)ph.node.p, u);
  }
}

template<class T>
void Emit<T>::hn_zero(int l, T* u)
{
  const Level& L = c.L[l];
  no_rec();
  if (!L.h_hnnodes.empty())
    launch(c, k_hn_zero<T>, blocks_for(L.h_hnnodes.size(), 128), 128,
           (int)L.h_hnnodes.size(), L.B, (const int*)L.hn_all.p, u);
}

template<class T>
void Emit<T>::dirichlet_zero(int l, T* u)
{
  const Level& L = c.L[l];
  no_rec();
  if (L.ndir)
    launch(c, k_dirichlet_zero<T>, blocks_for(L.ndir, 256), 256, L.ndir,
           (const int*)L.dirlist.p, u);
}

template<class T>
void Emit<T>::pf_sub(int l, T* x, bool weighted)
{
  const Level& L = c.L[l];
  no_rec();
  for (int comp = 0; comp < L.B; ++comp) {
    if (!(L.pf_mask & (1 << comp)))
      continue;
    launch(c, k_comp_sum<T>, red_blocks(L.n), kRedThreads, (int)L.n, L.B, comp,
           (const T*)x, weighted ? (const double*)L.pf_w.p : nullptr, c.partials.p,
           c.ticket.p, RedOut{ c.scal.p + 8, nullptr, nullptr, 0 });
    const double denom = weighted ? L.pf_domain : double(L.n - L.nhanging);
    launch(c, k_comp_sub<T>, stream_blocks(L.n), 256, (int)L.n, L.B, comp, x,
           (const double*)(c.scal.p + 8), denom);
  }
}

template<class T>
void Emit<T>::copy(int l, T* dst, const T* src)
{
  no_rec();
  launch(c, k_equ<T, T>, stream_blocks(c.L[l].ndof()), 256, (int64_t)c.L[l].ndof(), dst,
         1.0, src);
}

template<class T>
void Emit<T>::ilu_solve(int l, T* h)
{
  const Level& L = c.L[l];
  no_rec();
  const T* val = sizeof(T) == 8 ? reinterpret_cast<const T*>(L.ilu_v64.p)
                                : reinterpret_cast<const T*>(L.ilu_v32.p);
  const int* ptr = L.ilu_ptr.p;
  const int* col = L.ilu_col.p;
  const int* diag = L.ilu_diag.p;
  for (int up = 0; up < 2; ++up) {
    const std::vector<int>& off = up ? L.ilu_uptr : L.ilu_lptr;
    const int* lptr = up ? L.ilu_uptr_d.p : L.ilu_lptr_d.p;
    const int* rows = up ? L.ilu_urows.p : L.ilu_lrows.p;
    for (const Level::IluSeg& g : up ? L.ilu_useg : L.ilu_lseg) {
      const int cnt = off[g.lv0 + 1] - off[g.lv0];
#define GB_ILU_UP(BB, UP)                                                                \
if (g.cta)                                                                             \
  launch(c, k_ilu_levels<BB, T, UP>, 1, kIluCtaThreads, g.lv0, g.lv1, lptr, rows, ptr, \
         col, diag, val, h);                                                           \
else                                                                                   \
  launch(c, k_ilu_level<BB, T, UP>, blocks_for(cnt, 128), 128, cnt, rows + off[g.lv0], \
         ptr, col, diag, val, h)
#define GB_ILU(BB)                                                                       \
if (up) {                                                                              \
  GB_ILU_UP(BB, true);                                                                 \
} else {                                                                               \
  GB_ILU_UP(BB, false);                                                                \
}
      switch (L.B) {
        case 1: GB_ILU(1); break;
        case 2: GB_ILU(2); break;
        case 3: GB_ILU(3); break;
        default: GB_ILU(4);
      }
#undef GB_ILU
#undef GB_ILU_UP
    }
  }
}

template<class T>
void Emit<T>::ilu_axpy(int l, T* u, const T* h, bool u_zero)
{
  no_rec();
  launch(c, k_ilu_axpy<T>, blocks_for(c.L[l].ndof(), 256), 256, (int64_t)c.L[l].ndof(), u,
         c.params.omega, h, int(u_zero));
}

template<class T>
void Emit<T>::no_rec() const
{
  if (rec)
    throw Error{ GB_EINVAL, "step not available in the coarse-level program" };
}

template<class T>
void Emit<T>::jacobi(int l, const T* u, T* out, const T* b)
{
  const Level& L = c.L[l];
  if (rec)
    return rec->push_back(level_op(kOpJacobi, L, out, u, b, c.params.omega));
  spmv<kJacobi, T, T, T>(c, L, opA(c, L), u, out, b, dinv_of<T>(L), c.params.omega);
}

template<class T>
void Emit<T>::resid(int l, const T* u, T* out, const T* b)
{
  const Level& L = c.L[l];
  if (rec)
    return rec->push_back(level_op(kOpResid, L, out, u, b, 0.0));
  spmv<kResid, T, T, T>(c, L, opA(c, L), u, out, b, nullptr, 0.0);
}

template<class T>
void Emit<T>::restrict_to(int l, const T* fine, T* coarse, const double* smean, T* u1)
{
  const Transfer& Tr = c.T[l];
  if (rec) {
    CoarseOp o{};
    o.kind = kOpRestrict;
    o.n = Tr.nc;
    o.out = coarse;
    o.in = fine;
    o.in_n = Tr.nf;
    o.mask = c.L[l].dirmask.p;
    o.tptr = Tr.rptr.p;
    o.tent = Tr.rent.p;
    return rec->push_back(o);
  }
  const uint8_t* cm = c.L[l].dirmask.p;
  const int nb = blocks_for(Tr.nc, 256);
  const T* dv = u1 ? dinv_of<T>(c.L[l]) : nullptr;
  switch (c.L[l].B) {
    case 1:
      if (Tr.rmaxw <= 32)
        launch(c, k_restrict4<T>, blocks_for(int64_t(Tr.nc) * 4, 256), 256, Tr.nc,
               Tr.rptr.p, Tr.rent.p, fine, coarse, cm, dv, u1, c.params.omega);
      else
        launch(c, k_restrict<T>, nb, 256, Tr.nc, Tr.rptr.p, Tr.rent.p, fine, coarse, cm, dv,
               u1, c.params.omega);
      break;
    case 2:
      GB_REQUIRE(!u1, GB_EINVAL, "fused first sweep on a block level");
      launch(c, k_restrict_b<T, 2>, nb, 256, Tr.nc, Tr.rptr.p, Tr.rent.p, fine, coarse, cm,
             pf_comp(c.L[l + 1]), smean);
      break;
    case 3:
      launch(c, k_restrict_b<T, 3>, nb, 256, Tr.nc, Tr.rptr.p, Tr.rent.p, fine, coarse, cm,
             pf_comp(c.L[l + 1]), smean);
      break;
    default:
      launch(c, k_restrict_b<T, 4>, nb, 256, Tr.nc, Tr.rptr.p, Tr.rent.p, fine, coarse, cm,
             pf_comp(c.L[l + 1]), smean);
  }
}

template<class T>
void Emit<T>::direct(int l, T* u, const T* b)
{
  const Level& L = c.L[l];
  const double* inv = c.dir_inv[c.transposed ? 1 : 0].p;
  if (rec) {
    CoarseOp o{};
    o.kind = kOpDirect;
    o.n = static_cast<int>(L.ndof());
    o.out = u;
    o.in = b;
    o.in_n = o.n;
    o.val = inv;
    return rec->push_back(o);
  }
  launch(c, k_coarse_direct<T>, blocks_for(int64_t(L.ndof()) * 32, 256), 256,
         static_cast<int>(L.ndof()), inv, b, u);
}

template<class T>
void Emit<T>::fill0(int l, T* u)
{
  const Level& L = c.L[l];
  if (rec) {
    CoarseOp o{};
    o.kind = kOpFill0;
    o.n = static_cast<int>(L.ndof());
    o.out = u;
    return rec->push_back(o);
  }
  launch(c, k_fill<T>, stream_blocks(L.ndof()), 256, (int64_t)L.ndof(), u, T(0));
}

template<class T>
void Emit<T>::prolong(int l, const T* coarse, T* fine)
{
  const Transfer& Tr = c.T[l];
  if (rec) {
    CoarseOp o{};
    o.kind = kOpProlong;
    o.n = Tr.nf;
    o.out = fine;
    o.in = coarse;
    o.in_n = Tr.nc;
    o.mask = pmask_of(c.L[l + 1]);
    o.tptr = Tr.pptr.p;
    o.tent = Tr.pent.p;
    o.alpha = c.params.mgomega;
    return rec->push_back(o);
  }
  const uint8_t* fm = pmask_of(c.L[l + 1]);
  const double mw = c.params.mgomega;
  const int nb = blocks_for(Tr.nf, 256);
  switch (c.L[l + 1].B) {
    case 1:
      launch(c, k_prolong<1, T>, nb, 256, Tr.nf, Tr.pptr.p, Tr.pent.p, coarse, fine, fm, mw);
      break;
    case 2:
      launch(c, k_prolong_b<1, T, 2>, nb, 256, Tr.nf, Tr.pptr.p, Tr.pent.p, coarse, fine,
             fm, mw);
      break;
    case 3:
      launch(c, k_prolong_b<1, T, 3>, nb, 256, Tr.nf, Tr.pptr.p, Tr.pent.p, coarse, fine,
             fm, mw);
      break;
    default:
      launch(c, k_prolong_b<1, T, 4>, nb, 256, Tr.nf, Tr.pptr.p, Tr.pent.p, coarse, fine,
             fm, mw);
  }
}

template struct Emit<double>;
template struct Emit<float>;

// StdSolver::smooth, linear_smooth jacobi (Solver/stdsolver.cc:951-986): each
// sweep computes h = y - A x, h = D^-1 h, x += omega h; fused into one pass that
// writes the new iterate to the other buffer (u and tmp swap roles). A sweep
// from x = 0 needs no product (y - A 0 == y).
//
// With the Vanka smoother or a pressure filter a sweep is done in place:
// h = y - A x (tmp), SubtractMeanAlgebraic(h), h = Vanka(h) or D^-1 h,
// x += omega h, SubtractMean(x).
bool
fused_smoother(const Context& c, const Level& L)
{
  return c.params.smoother == 0 && !L.pf_mask;
}

template<class T>
void
smooth(Emit<T>& E, int l, int niter, T*& u, T*& tmp, const T* b, bool& u_zero)
{
  Context& c = E.c;
  const Level& L = c.L[l];
  const bool fused = fused_smoother(c, L);
  for (int it = 0; it < niter; ++it) {
    if (c.params.smoother == 2) {
      // linear_smooth ilu: h = y - A u (filtered), the ILU solve of h in
      // place, u += omega h, SubtractMean(u) (StdSolver::smooth)
      if (u_zero)
        E.copy(l, tmp, b);
      else
        E.resid(l, u, tmp, b);
      if (L.pf_mask)
        E.pf_sub(l, tmp, false);
      E.ilu_solve(l, tmp);
      E.ilu_axpy(l, u, tmp, u_zero);
      u_zero = false;
      if (L.pf_mask)
        E.pf_sub(l, u, true);
      continue;
    }
    if (fused) {
      if (u_zero && it + 1 < niter && L.B == 1 && !E.rec && c.jacobi2) {
        // the first two sweeps from u = 0 in one pass (the first iterate is
        // formed on the fly where the second reads it)
        E.jacobi_two_from_zero(l, tmp, b);
        std::swap(u, tmp);
        u_zero = false;
        ++it;
      } else if (u_zero) {
        E.jacobi_zero(l, u, b);
        u_zero = false;
      } else {
        E.jacobi(l, u, tmp, b);
        std::swap(u, tmp);
      }
      continue;
    }
    if (L.pf_mask && Emit<T>::pf_comp(L) >= 0) {
      // one filtered component: the residual kernel reduces its algebraic
      // mean, the smoother subtracts it on read and reduces the weighted mean
      // of the new iterate, which one pass then subtracts
      const T* h = b; // y - A 0
      const double* hm;
      if (!u_zero) {
        hm = E.resid_mean(l, u, tmp, b);
        h = tmp;
      } else {
        hm = E.mean_of(l, b, false);
      }
      if (c.params.smoother == 1)
        E.vanka(l, h, u, u_zero, hm);
      else
        E.jacobi_apply(l, h, u, u_zero, hm);
      u_zero = false;
      E.sub_mean(l, u, c.scal.p + 9);
      continue;
    }
    const T* h = b; // y - A 0
    if (!u_zero) {
      E.resid(l, u, tmp, b);
      h = tmp;
    } else if (L.pf_mask) {
      E.copy(l, tmp, b);
      h = tmp;
    }
    if (L.pf_mask)
      E.pf_sub(l, tmp, false);
    if (c.params.smoother == 1)
      E.vanka(l, h, u, u_zero);
    else
      E.jacobi_apply(l, h, u, u_zero);
    u_zero = false;
    if (L.pf_mask)
      E.pf_sub(l, u, true);
  }
}

template<class T>
bool mgstep(Emit<T>& E, MgWork<T>& W, int l, int finelevel, int coarselevel,
                   char& p0, char p, T*& u, T*& tmp, const T* b, bool u_zero,
                   bool first_done = false);
template<class T>
bool mgstep_down(Emit<T>& E, MgWork<T>& W, int l, int finelevel, int coarselevel,
                 char& p0, char p, T*& u, T*& tmp, const T* b, bool u_zero);

template<class T>
const CoarseProgram& coarse_program(Context& c, MgWork<T>& W, int l, int finelevel,
                                           int coarselevel, char p0, char p, T* u, T* tmp,
                                           const T* b, bool u_zero);

// Runs mgstep(l) for a level handled by the coarse-level kernel: the step is
// recorded once per entry state (cached) and launched as one single-CTA kernel.
template<class T>
bool
run_coarse(Emit<T>& E, MgWork<T>& W, int l, int finelevel, int coarselevel, char& p0,
           char p, T*& u, T*& tmp, const T* b, bool u_zero)
{
  Context& c = E.c;
  const CoarseProgram& prog =
    coarse_program<T>(c, W, l, finelevel, coarselevel, p0, p, u, tmp, b, u_zero);
  if (prog.nops > 0 && prog.ncols > 0) {
    const T* K = sizeof(T) == 8 ? reinterpret_cast<const T*>(prog.K64.p)
                                : reinterpret_cast<const T*>(prog.K32.p);
    launch(c, k_coarse_apply<T>, blocks_for(int64_t(prog.n_root) * 32, 256), 256,
           prog.n_root, prog.ncols, prog.nb, K, static_cast<const T*>(prog.b_root),
           static_cast<const T*>(prog.u_in),
           static_cast<T*>(const_cast<void*>(prog.u_out)));
  } else if (prog.nops > 0) {
    launch_smem(c, k_coarse_cycle<T>, 1, kCoarseThreads, prog.smem_bytes,
                (const CoarseOp*)prog.ops.p, prog.nops, (const CoarseBuf*)prog.bufs.p,
                prog.nbufs, (const CoarsePrefetch*)prog.pre.p, prog.npre,
                prog.vec_bytes, CoarseBatch{});
  }
  u = static_cast<T*>(const_cast<void*>(prog.u_out));
  tmp = static_cast<T*>(const_cast<void*>(prog.tmp_out));
  p0 = prog.p0_out;
  return prog.zero_out;
}

// In the multi-CTA program, the coarse sub-cycle from u = 0 becomes one
// kOpDense op with the single-CTA program's precomputed map.
template<class T>
bool
emit_dense(Emit<T>& E, MgWork<T>& W, int l, int finelevel, int coarselevel, char& p0,
           char p, T*& u, T*& tmp, const T* b)
{
  Context& c = E.c;
  const CoarseProgram& prog =
    coarse_program<T>(c, W, l, finelevel, coarselevel, p0, p, u, tmp, b, true);
  if (prog.nops > 0 && prog.ncols > 0) {
    CoarseOp o{};
    o.kind = kOpDense;
    o.n = prog.n_root;
    o.in_n = prog.ncols;
    o.in = prog.b_root;
    o.out = const_cast<void*>(prog.u_out);
    o.val = sizeof(T) == 8 ? static_cast<const void*>(prog.K64.p)
                           : static_cast<const void*>(prog.K32.p);
    E.rec->push_back(o);
    u = static_cast<T*>(const_cast<void*>(prog.u_out));
    tmp = static_cast<T*>(const_cast<void*>(prog.tmp_out));
    p0 = prog.p0_out;
    return prog.zero_out;
  }
  // no dense map (an empty sub-cycle): record its steps
  Emit<T> R{ E.c, E.rec, E.no_dense_at, false };
  return mgstep<T>(R, W, l, finelevel, coarselevel, p0, p, u, tmp, b, true);
}

// mgstep(l) from u = 0 for the level below the finest and everything under it,
// as one op program run by a persistent cooperative grid (k_mid_cycle).
// The CTAs of the cluster that runs the mid-level program: 16 (one GPC's
// worth of SMs, a non-portable size) when the device can schedule it, else 8.
template<class T>
int
cluster_size_for(Context& c)
{
  int& cached = c.cluster_size[sizeof(T) == 8 ? 0 : 1];
  if (cached > 0)
    return cached;
  auto* kern = k_mid_cycle<T, kMidClusterThreads, true>;
  int size = 8;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
      cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(16);
    cfg.blockDim = dim3(kMidClusterThreads);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 16;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg) == cudaSuccess && nclusters > 0)
      size = 16;
  }
  cudaGetLastError(); // a refused query leaves no error behind
  cached = size;
  return size;
}

template<class T>
bool
run_mid(Emit<T>& E, MgWork<T>& W, int l, int finelevel, int coarselevel, char& p0, char p,
        T*& u, T*& tmp, const T* b)
{
  Context& c = E.c;
  CoarseKey key{ int(sizeof(T)), l, (const void*)u, (const void*)tmp, (const void*)b,
                 true, p0, p, c.transposed != 0 };
  auto it = c.mid_progs.find(key);
  if (it == c.mid_progs.end()) {
    std::vector<CoarseOp> ops;
    Emit<T> R{ c, &ops, -1, true };
    T* u2 = u;
    T* t2 = tmp;
    char p02 = p0;
    const bool z = mgstep<T>(R, W, l, finelevel, coarselevel, p02, p, u2, t2, b, true);
    CoarseProgram prog;
    prog.nops = static_cast<int>(ops.size());
    GB_CUDA(prog.ops.alloc(std::max<size_t>(ops.size(), 1)));
    if (!ops.empty())
      GB_CUDA(h2d(c.stream, prog.ops.p, ops.data(), ops.size() * sizeof(CoarseOp)));
    int maxn = 1;
    for (const auto& o : ops)
      maxn = std::max(maxn, o.kind == kOpDense ? o.n * 32 : o.n);
    if (c.mid_on) {
      int& grid = c.mid_grid[sizeof(T) == 8 ? 0 : 1];
      if (grid == 0) {
        int occ = 0, nsm = 0;
        GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &occ, k_mid_cycle<T, kMidThreads, false>, kMidThreads, 0));
        GB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c.device));
        grid = std::max(1, occ) * nsm;
      }
      prog.n_root = std::min(grid, blocks_for(maxn, kMidThreads)); // launch grid
    } else {
      prog.n_root = cluster_size_for<T>(c); // one cluster
    }
    prog.u_out = z ? nullptr : u2;
    prog.tmp_out = t2;
    prog.p0_out = p02;
    prog.zero_out = z;
    prog.u_in = u2;
    it = c.mid_progs.emplace(key, std::move(prog)).first;
  }
  const CoarseProgram& prog = it->second;
  if (prog.nops > 0 && c.mid_on) {
    GB_CUDA(cudaMemsetAsync(c.midbar.p, 0, sizeof(unsigned), c.stream));
    cudaEvent_t e0;
    kt_begin(c, &e0);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(prog.n_root);
    cfg.blockDim = dim3(kMidThreads);
    cfg.stream = c.stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative; // all CTAs resident: the barrier ends
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    GB_CUDA(cudaLaunchKernelEx(&cfg, k_mid_cycle<T, kMidThreads, false>,
                               (const CoarseOp*)prog.ops.p, prog.nops, c.midbar.p,
                               c.miderr.p, c.wait_ns, c.barrier_phantoms));
    c.launches++;
    check_launch(c);
    kt_end(c, e0, reinterpret_cast<const void*>(k_mid_cycle<T, kMidThreads, false>));
  } else if (prog.nops > 0) {
    cudaEvent_t e0;
    kt_begin(c, &e0);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(prog.n_root);
    cfg.blockDim = dim3(kMidClusterThreads);
    cfg.stream = c.stream;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = prog.n_root;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = c.pdl ? 2 : 1;
    GB_CUDA(cudaLaunchKernelEx(&cfg, k_mid_cycle<T, kMidClusterThreads, true>,
                               (const CoarseOp*)prog.ops.p, prog.nops, c.midbar.p,
                               c.miderr.p, c.wait_ns, 0u));
    c.launches++;
    check_launch(c);
    kt_end(c, e0, reinterpret_cast<const void*>(k_mid_cycle<T, kMidClusterThreads, true>));
  }
  u = static_cast<T*>(const_cast<void*>(prog.u_in));
  tmp = static_cast<T*>(const_cast<void*>(prog.tmp_out));
  p0 = prog.p0_out;
  return prog.zero_out;
}

// The single-CTA program (and dense map) of mgstep(l) for a coarse level,
// recorded once per entry state.
template<class T>
const CoarseProgram&
coarse_program(Context& c, MgWork<T>& W, int l, int finelevel, int coarselevel, char p0,
               char p, T* u, T* tmp, const T* b, bool u_zero)
{
  CoarseKey key{ int(sizeof(T)), l, (const void*)u, (const void*)tmp, (const void*)b,
                 u_zero, p0, p, c.transposed != 0 };
  auto it = c.coarse_progs.find(key);
  if (it == c.coarse_progs.end()) {
    std::vector<CoarseOp> ops;
    Emit<T> R{ c, &ops };
    T* u2 = u;
    T* t2 = tmp;
    char p02 = p0;
    const bool z = mgstep<T>(R, W, l, finelevel, coarselevel, p02, p, u2, t2, b, u_zero);
    CoarseProgram prog;
    prog.nops = static_cast<int>(ops.size());
    // stage every vector in shared memory: offsets in first-use order; load
    // those read before written, store back those written
    std::vector<CoarseBuf> bufs;
    std::map<const void*, int> bidx;
    auto buf_of = [&](const void* p, int n) {
      auto it2 = bidx.find(p);
      if (it2 != bidx.end())
        return it2->second;
      CoarseBuf cb{ const_cast<void*>(p), n * int(sizeof(T)), prog.vec_bytes, 0, 0 };
      prog.vec_bytes += (cb.bytes + 15) / 16 * 16;
      bufs.push_back(cb);
      return bidx[p] = static_cast<int>(bufs.size()) - 1;
    };
    std::vector<char> written;
    auto read = [&](int bi) {
      if (bi >= static_cast<int>(written.size()))
        written.resize(bi + 1, 0);
      if (!written[bi])
        bufs[bi].load = 1;
    };
    auto write = [&](int bi) {
      if (bi >= static_cast<int>(written.size()))
        written.resize(bi + 1, 0);
      written[bi] = 1;
      bufs[bi].store = 1;
    };
    for (auto& o : ops) {
      int bi_in = o.in ? buf_of(o.in, o.in_n) : -1;
      int bi_b = o.b ? buf_of(o.b, o.b_n) : -1;
      int bi_out = buf_of(o.out, o.n);
      if (bi_in >= 0)
        read(bi_in);
      if (bi_b >= 0)
        read(bi_b);
      if (o.kind == kOpProlong)
        read(bi_out); // out += ...
      write(bi_out);
      o.in_off = bi_in >= 0 ? bufs[bi_in].off : 0;
      o.b_off = bi_b >= 0 ? bufs[bi_b].off : 0;
      o.out_off = bufs[bi_out].off;
    }
    // read-only data of the levels and transfers the program touches
    std::vector<CoarsePrefetch> pre;
    for (int lv = 0; lv <= l; ++lv) {
      const Level& L = c.L[lv];
      const Sell& A = opA(c, L);
      pre.push_back({ sell_vals<T>(A), int(A.entries * sizeof(T)) });
      pre.push_back({ A.sptr.p, int((A.nslices + 1) * sizeof(int)) });
      if (A.pat) {
        pre.push_back({ A.pid.p, int(L.n) });
        pre.push_back({ A.ptab.p, int(A.npat * A.W * sizeof(int)) });
      } else {
        pre.push_back({ A.col.p, int(A.entries * sizeof(int)) });
      }
      pre.push_back({ dinv_of<T>(L), int(L.ndof() * sizeof(T)) });
      pre.push_back({ L.dirmask.p, int(L.ndof()) });
      if (lv + 1 <= l) {
        const Transfer& Tr = c.T[lv];
        pre.push_back({ Tr.rptr.p, int(Tr.rptr.n * sizeof(int)) });
        pre.push_back({ Tr.rent.p, int(Tr.rent.n * sizeof(uint32_t)) });
        pre.push_back({ Tr.pptr.p, int(Tr.pptr.n * sizeof(int)) });
        pre.push_back({ Tr.pent.p, int(Tr.pent.n * sizeof(uint32_t)) });
      }
    }
    prog.nbufs = static_cast<int>(bufs.size());
    prog.npre = static_cast<int>(pre.size());
    prog.smem_bytes = prog.vec_bytes + prog.nops * int(sizeof(CoarseOp));
    GB_REQUIRE(prog.smem_bytes <= 200 * 1024, GB_EINVAL,
               "coarse-level program does not fit in shared memory");
    GB_CUDA(prog.ops.alloc(std::max<size_t>(ops.size(), 1)));
    GB_CUDA(prog.bufs.alloc(std::max<size_t>(bufs.size(), 1)));
    GB_CUDA(prog.pre.alloc(std::max<size_t>(pre.size(), 1)));
    if (!ops.empty())
      GB_CUDA(h2d(c.stream, prog.ops.p, ops.data(), ops.size() * sizeof(CoarseOp)));
    if (!bufs.empty())
      GB_CUDA(h2d(c.stream, prog.bufs.p, bufs.data(), bufs.size() * sizeof(CoarseBuf)));
    if (!pre.empty())
      GB_CUDA(h2d(c.stream, prog.pre.p, pre.data(), pre.size() * sizeof(CoarsePrefetch)));
    if (prog.smem_bytes > 48 * 1024)
      GB_CUDA(cudaFuncSetAttribute(k_coarse_cycle<T>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   prog.smem_bytes));
    if (c.coarse_dense && u_zero && prog.nops > 0) {
      // columns: unit entries of the root b (the sub-cycle starts from u = 0, so
      // it is linear in b alone; a non-zero start runs the op program instead)
      prog.n_root = static_cast<int>(c.L[l].ndof());
      prog.nb = prog.n_root;
      prog.ncols = prog.nb;
      prog.b_root = b;
      prog.u_in = u;
      CoarseBatch bt{};
      bt.ncols = prog.ncols;
      bt.nb = prog.nb;
      bt.n_root = prog.n_root;
      bt.b_off = bufs[bidx.at((const void*)b)].off;
      bt.u_in_off = 0;
      bt.u_out_off = bufs[bidx.at((const void*)u2)].off;
      const size_t kn = size_t(prog.n_root) * prog.ncols;
      if (sizeof(T) == 8) {
        GB_CUDA(prog.K64.alloc(kn));
        bt.K = prog.K64.p;
      } else {
        GB_CUDA(prog.K32.alloc(kn));
        bt.K = prog.K32.p;
      }
      launch_smem(c, k_coarse_cycle<T>, prog.ncols, kCoarseThreads, prog.smem_bytes,
                  (const CoarseOp*)prog.ops.p, prog.nops, (const CoarseBuf*)prog.bufs.p,
                  prog.nbufs, (const CoarsePrefetch*)prog.pre.p, prog.npre,
                  prog.vec_bytes, bt);
      GB_CUDA(cudaStreamSynchronize(c.stream));
      c.launches--; // set-up, not part of a solve
      prog.batch = bt;
      prog.tsize = int(sizeof(T));
    }
    prog.u_out = u2;
    prog.tmp_out = t2;
    prog.p0_out = p02;
    prog.zero_out = z;
    it = c.coarse_progs.emplace(key, std::move(prog)).first;
  }
  return it->second;
}

// mgstep(l) from u = 0 for a level whose sub-cycle the single-CTA program does
// not cover: the sub-cycle is linear in b, so it is applied as its matrix K
// (u_out = K b, one GEMV), built once per entry state by running the
// sub-cycle's own kernels on the unit vectors (b is saved and restored).
template<class T>
bool
run_dense(Emit<T>& E, MgWork<T>& W, int l, int finelevel, int coarselevel, char& p0,
          char p, T*& u, T*& tmp, const T* b)
{
  Context& c = E.c;
  CoarseKey key{ int(sizeof(T)), l, (const void*)u, (const void*)tmp, (const void*)b,
                 true, p0, p, c.transposed != 0 };
  auto it = c.dense_maps.find(key);
  if (it == c.dense_maps.end()) {
    const int n = static_cast<int>(c.L[l].ndof());
    CoarseProgram dm;
    dm.n_root = n;
    dm.nb = n;
    dm.ncols = n;
    dm.b_root = b;
    DeviceArray<T> bsave, Kt;
    GB_CUDA(bsave.alloc(n));
    GB_CUDA(Kt.alloc(size_t(n) * n));
    T* bw = const_cast<T*>(b);
    GB_CUDA(cudaMemcpyAsync(bsave.p, b, n * sizeof(T), cudaMemcpyDeviceToDevice, c.stream));
    const int64_t launches0 = c.launches;
    const T one = T(1);
    T* u2 = u;
    T* t2 = tmp;
    char p02 = p0;
    bool z = true;
    for (int j = 0; j < n; ++j) {
      GB_CUDA(cudaMemsetAsync(bw, 0, n * sizeof(T), c.stream));
      GB_CUDA(cudaMemcpyAsync(bw + j, &one, sizeof(T), cudaMemcpyHostToDevice, c.stream));
      Emit<T> E2{ c, nullptr, l };
      u2 = u;
      t2 = tmp;
      p02 = p0;
      z = mgstep<T>(E2, W, l, finelevel, coarselevel, p02, p, u2, t2, bw, true);
      if (z)
        E2.fill0(l, u2);
      // column j of K (row-major n x n) = the response to e_j
      GB_CUDA(cudaMemcpy2DAsync(Kt.p + j, n * sizeof(T), u2, sizeof(T), sizeof(T), n,
                                cudaMemcpyDeviceToDevice, c.stream));
      GB_CUDA(cudaStreamSynchronize(c.stream)); // `one` lives on this stack frame
    }
    GB_CUDA(cudaMemcpyAsync(bw, bsave.p, n * sizeof(T), cudaMemcpyDeviceToDevice, c.stream));
    GB_CUDA(cudaStreamSynchronize(c.stream));
    c.launches = launches0; // set-up, not part of a solve
    if (sizeof(T) == 8)
      dm.K64.p = reinterpret_cast<double*>(Kt.p), dm.K64.n = Kt.n;
    else
      dm.K32.p = reinterpret_cast<float*>(Kt.p), dm.K32.n = Kt.n;
    Kt.p = nullptr;
    Kt.n = 0;
    dm.u_in = u;
    dm.u_out = u2;
    dm.tmp_out = t2;
    dm.p0_out = p02;
    dm.zero_out = false;
    dm.nops = 1;
    it = c.dense_maps.emplace(key, std::move(dm)).first;
  }
  const CoarseProgram& dm = it->second;
  const T* K = sizeof(T) == 8 ? reinterpret_cast<const T*>(dm.K64.p)
                              : reinterpret_cast<const T*>(dm.K32.p);
  launch(c, k_coarse_apply<T>, blocks_for(int64_t(dm.n_root) * 32, 256), 256, dm.n_root,
         dm.ncols, dm.nb, K, static_cast<const T*>(dm.b_root),
         static_cast<const T*>(dm.u_in), static_cast<T*>(const_cast<void*>(dm.u_out)));
  u = static_cast<T*>(const_cast<void*>(dm.u_out));
  tmp = static_cast<T*>(const_cast<void*>(dm.tmp_out));
  p0 = dm.p0_out;
  return false;
}

// StdMultiLevelSolver::mgstep (Solver/stdmultilevelsolver.cc:462-531). Steps
// that only feed CGInfo (the norms and the final residual) are not computed:
// they do not change u. HNDistribute/HNAverage/HNZero are identities on meshes
// without hanging nodes.
// Returns true when u is still implicitly zero (no sweep has written it).
// With first_done, the restriction into b has already run this level's first
// Jacobi sweep from 0 into u (fuse_first_sweep).
template<class T>
bool
mgstep(Emit<T>& E, MgWork<T>& W, int l, int finelevel, int coarselevel, char& p0,
       char p, T*& u, T*& tmp, const T* b, bool u_zero, bool first_done)
{
  Context& c = E.c;
  const gb_params& P = c.params;
  if (first_done) {
    bool z = false;
    if (l == coarselevel) {
      if (p == 'F')
        p0 = 'V';
      smooth<T>(E, l, P.iterexact - 1, u, tmp, b, z); // smooth_exact
      return false;
    }
    smooth<T>(E, l, P.iterpre - 1, u, tmp, b, z);
    return mgstep_down<T>(E, W, l, finelevel, coarselevel, p0, p, u, tmp, b, false);
  }
  if (!E.rec && c.coarse_on && l == c.mid_level && u_zero && l != E.no_dense_at)
    return run_mid<T>(E, W, l, finelevel, coarselevel, p0, p, u, tmp, b);
  if (!E.rec && c.coarse_on && l <= c.coarse_root)
    return run_coarse<T>(E, W, l, finelevel, coarselevel, p0, p, u, tmp, b, u_zero);
  if (E.rec && E.mid && c.coarse_dense && c.coarse_on && l == c.coarse_root && u_zero)
    return emit_dense<T>(E, W, l, finelevel, coarselevel, p0, p, u, tmp, b);
  if (!E.rec && c.coarse_on && l <= c.dense_root && u_zero && l != E.no_dense_at)
    return run_dense<T>(E, W, l, finelevel, coarselevel, p0, p, u, tmp, b);
  if (l == coarselevel) {
    if (p == 'F')
      p0 = 'V';
    if (l == 0 && direct_on(c)) { // smooth_exact on a direct level
      E.direct(l, u, b);
      return false;
    }
    smooth<T>(E, l, P.iterexact, u, tmp, b, u_zero); // smooth_exact
    return u_zero;
  }
  smooth<T>(E, l, P.iterpre, u, tmp, b, u_zero);
  return mgstep_down<T>(E, W, l, finelevel, coarselevel, p0, p, u, tmp, b, u_zero);
}

// Whether the restriction into level lc (visited once, from u = 0) can also
// run lc's first smoothing sweep: the fused scalar Jacobi sweep from zero,
// u = omega D^-1 b, is elementwise in the restricted b, so the restriction
// kernel writes it beside b (restrict_store) and the launch of
// k_jacobi_from_zero goes. Not where lc's sub-cycle is a recorded program or a
// dense map, a direct solve, or has hanging nodes (HNDistribute comes between
// the restriction and the sweep).
template<class T>
bool
fuse_first_sweep(const Emit<T>& E, int lc, int coarselevel, int visits)
{
  const Context& c = E.c;
  const Level& C = c.L[lc];
  return !E.rec && visits == 1 && !c.jacobi2 && C.B == 1 && fused_smoother(c, C) &&
         !C.has_hn() &&
         !(c.coarse_on && (lc == c.mid_level || lc <= c.coarse_root || lc <= c.dense_root)) &&
         !(lc == 0 && direct_on(c)) &&
         (lc == coarselevel ? c.params.iterexact : c.params.iterpre) >= 1;
}

// The rest of mgstep on level l after its pre-smoothing: the residual and its
// restriction, the coarse visits, the prolonged correction and the
// post-smoothing.
template<class T>
bool
mgstep_down(Emit<T>& E, MgWork<T>& W, int l, int finelevel, int coarselevel, char& p0,
            char p, T*& u, T*& tmp, const T* b, bool u_zero)
{
  Context& c = E.c;
  const gb_params& P = c.params;
  const int j = (p0 == 'V') ? 1 : (p0 == 'W') ? 2 : (p0 == 'F') ? 3 : 0;
  // MatrixResidual into tmp (with SubtractMeanAlgebraic), restrict_zero +
  // SetBoundaryVectorZero on l-1
  bool fused = false;
  if (c.L[l].pf_mask && Emit<T>::pf_comp(c.L[l]) >= 0 && c.L[l].B > 1) {
    // filtered residual: its mean is subtracted as the restriction reads it
    if (u_zero) {
      E.restrict_to(l - 1, b, W.b[l - 1].p, E.mean_of(l, b, false));
    } else {
      const double* hm = E.resid_mean(l, u, tmp, b);
      E.restrict_to(l - 1, tmp, W.b[l - 1].p, hm);
    }
  } else if (c.L[l].pf_mask) {
    if (u_zero)
      E.copy(l, tmp, b);
    else
      E.resid(l, u, tmp, b);
    E.pf_sub(l, tmp, false);
    E.restrict_to(l - 1, tmp, W.b[l - 1].p);
  } else {
    fused = fuse_first_sweep<T>(E, l - 1, coarselevel, j);
    T* u1 = fused ? W.u[l - 1].p : nullptr;
    if (u_zero) {
      E.restrict_to(l - 1, b, W.b[l - 1].p, nullptr, u1); // u == 0: the residual is b
    } else {
      E.resid(l, u, tmp, b);
      E.restrict_to(l - 1, tmp, W.b[l - 1].p, nullptr, u1);
    }
  }
  if (c.L[l - 1].has_hn()) { // HNDistribute, then SetBoundaryVectorZero again
    E.hn_distribute(l - 1, W.b[l - 1].p);
    E.dirichlet_zero(l - 1, W.b[l - 1].p);
  }
  T* uc = W.u[l - 1].p;
  T* tc = W.v[l - 1].p;
  bool czero = true; // Zero(u) on l-1
  for (int i = 0; i < j; ++i)
    czero = mgstep<T>(E, W, l - 1, finelevel, coarselevel, p0, p, uc, tc,
                      W.b[l - 1].p, czero, fused && i == 0);
  if (czero) // no sweep ran on l-1: its u is the zero of Zero(u)
    E.fill0(l - 1, uc);
  if ((l == 0) && (p == 'F'))
    p0 = 'W';
  if (u_zero)
    E.fill0(l, u);
  // HNAverage(u_c); Zero(v); prolongate_add; HNZero(v); SetBoundaryVectorZero(v);
  // Add(u, mgomega, v). (HNZero(u_c) after it is dead: u_c is zeroed before
  // its next use.)
  if (c.L[l - 1].has_hn())
    E.hn_average(l - 1, uc);
  E.prolong(l - 1, uc, u);
  bool post_zero = false;
  smooth<T>(E, l, P.iterpost, u, tmp, b, post_zero);
  return false;
}

// One cycle on the finest level into x (T), rhs y (T), from x's content or 0.
// The buffer that a cycle from x = 0 (precondition_T with x_zero) runs its
// first finest-level sweep into.
template<class T>
static T*
first_sweep_buffer(Context& c, MgWork<T>& W, T* x, bool x_zero)
{
  const int fl = c.nlevels - 1;
  const gb_params& P = c.params;
  int pingpong = (x_zero ? std::max(P.iterpre - 1, 0) : P.iterpre) + P.iterpost;
  if (fl == 0)
    pingpong = x_zero ? std::max(P.iterexact - 1, 0) : P.iterexact;
  if (!fused_smoother(c, c.L[fl]))
    pingpong = 0; // sweeps in place
  return x_zero && (pingpong & 1) ? W.v[fl].p : x;
}

// Where the finest level's first sweep of a cycle from x = 0 can be written by
// the kernel that forms the cycle's right-hand side (k_load_idx): the buffer,
// or nullptr where that sweep is not the fused scalar Jacobi sweep from zero.
template<class T>
T*
precondition_first_sweep(Context& c, MgWork<T>& W, T* x)
{
  ensure_work(c);
  const int fl = c.nlevels - 1;
  Emit<T> E{ c, nullptr };
  if (fl == 0 || !fuse_first_sweep<T>(E, fl, 0, 1))
    return nullptr;
  return first_sweep_buffer<T>(c, W, x, true);
}

// One cycle into x from x's content or (x_zero) from 0; first_done: from 0,
// with the first finest-level sweep already in the buffer that
// precondition_first_sweep named.
template<class T>
void
precondition_T(Context& c, MgWork<T>& W, T* x, const T* y, bool x_zero, bool first_done)
{
  ensure_work(c);
  const int fl = c.nlevels - 1;
  if (first_done)
    x_zero = true;
  T* tmp = W.v[fl].p;
  // Pick the buffer of the first sweep so that the last write lands in x.
  T* u = first_sweep_buffer<T>(c, W, x, x_zero);
  if (u != x)
    tmp = x;
  const gb_params& P = c.params;
  char p = P.mgtype;
  char p0 = (p == 'F') ? 'W' : p;
  Emit<T> E{ c, nullptr };
  if (mgstep<T>(E, W, fl, fl, 0, p0, p, u, tmp, y, first_done ? false : x_zero, first_done))
    E.fill0(fl, u);
  if (u != x) {
    GB_CUDA(cudaMemcpyAsync(x, u, c.L[fl].ndof() * sizeof(T),
                            cudaMemcpyDeviceToDevice, c.stream));
  }
}

// ---------------------------------------------- instantiations used elsewhere

#define GB_CYCLE_INST(T)                                                                   \
  template void smooth<T>(Emit<T>&, int, int, T*&, T*&, const T*, bool&);                  \
  template void precondition_T<T>(Context&, MgWork<T>&, T*, const T*, bool, bool);         \
  template T* precondition_first_sweep<T>(Context&, MgWork<T>&, T*);
GB_CYCLE_INST(double)
GB_CYCLE_INST(float)
#undef GB_CYCLE_INST

} // namespace gb
