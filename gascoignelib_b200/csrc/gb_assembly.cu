// Device assembly (element matrices, condensation, the gather into the
// level values), the Form and Newton residual, cells and functionals, and
// the solution files: their drivers and C-ABI entry points.
#include "gb_cycle.cuh"

namespace gb {

// Element matrices and their sum into level l's values (FP64 and FP32), the
// Dirichlet rows and columns, and the block-diagonal inverse; the kappa of the
// level's cells is in L.m_kappa.
void
assemble_level(Context& c, int l, const double* beta)
{
  Level& L = c.L[l];
  const int dim = L.mesh_dim;
  const int nl = L.mesh_deg == 1 ? 1 << dim : (dim == 3 ? 27 : 9);
  const int nc = static_cast<int>(L.mesh_ncells);
  const bool pq1 = L.mesh_deg == 3; // Q1 functions on patches
  GB_CUDA(c.asm_E.n >= size_t(nc) * nl * nl ? cudaSuccess
                                             : c.asm_E.alloc(size_t(nc) * nl * nl));
  const double b0 = beta ? beta[0] : 0.0, b1 = beta ? beta[1] : 0.0;
  const double b2 = beta && dim == 3 ? beta[2] : 0.0;
  const double g = 0.5 / std::sqrt(3.0);
  const bool conv = b0 != 0.0 || b1 != 0.0 || b2 != 0.0;
  L.m_beta[0] = b0;
  L.m_beta[1] = b1;
  L.m_beta[2] = b2;
  L.m_lps_s0 = L.mesh_deg >= 2 ? c.lps_s0 : 0.0;
  L.m_lps_xeta = c.lps_xeta;
  L.m_assembled = true;
#define GB_ELEM(D, CV)                                                                   \
  launch(c, k_q1_element<D, CV>, blocks_for(nc, 128), 128, nc, (const int*)L.m_cells.p,  \
         (const double*)L.m_coords.p, (const double*)L.m_kappa.p, b0, b1, b2, g, c.asm_E.p)
#define GB_ELEM2(D, CV, LP, PQ)                                                          \
  launch(c, k_q2_element_warp<D, CV, LP, PQ>, blocks_for(int64_t(nc) * 32, 128), 128, nc, \
         (const int*)L.m_cells.p, (const double*)L.m_coords.p, (const double*)L.m_kappa.p, \
         b0, b1, b2, c.asm_E.p, c.lps_s0, c.lps_xeta, bnorm, g)
#define GB_ELEM2K(D, PQ)                                                                 \
  do {                                                                                   \
    if (lps) GB_ELEM2(D, true, true, PQ);                                                \
    else if (conv) GB_ELEM2(D, true, false, PQ);                                         \
    else GB_ELEM2(D, false, false, PQ);                                                  \
  } while (0)
  GB_REQUIRE(c.lps_s0 == 0.0 || L.mesh_deg >= 2, GB_EINVAL,
             "LPS is built for patch elements only (Q2, or Q1 on patches)");
  const bool lps = conv && c.lps_s0 > 0.0;
  const double bnorm = std::sqrt(b0 * b0 + b1 * b1 + b2 * b2) + 1e-6;
  if (L.mesh_deg >= 2) {
    if (dim == 2) {
      if (pq1) GB_ELEM2K(2, true); else GB_ELEM2K(2, false);
    } else {
      if (pq1) GB_ELEM2K(3, true); else GB_ELEM2K(3, false);
    }
  } else if (dim == 2) {
    if (conv) GB_ELEM(2, true); else GB_ELEM(2, false);
  } else {
    if (conv) GB_ELEM(3, true); else GB_ELEM(3, false);
  }
#undef GB_ELEM
#undef GB_ELEM2
#undef GB_ELEM2K
  if (L.m_nhcells > 0)
    launch(c, k_condense, blocks_for(int64_t(L.m_nhcells) * 32, 128), 128, L.m_nhcells,
           (const int*)L.m_hcells.p, (const int*)L.m_hopptr.p, (const CondOp*)L.m_hops.p, nl,
           nc, c.asm_E.p);
  const uint8_t* rmask = L.dirmask.p; // rows kept as the identity
  if (L.has_hn() && !L.h_hnnodes.empty()) {
    GB_CUDA(cudaMemcpyAsync(L.m_hmask.p, L.dirmask.p, L.n, cudaMemcpyDeviceToDevice, c.stream));
    launch(c, k_mark_nodes, blocks_for(int64_t(L.h_hnnodes.size()), 128), 128,
           (int)L.h_hnnodes.size(), (const int*)L.hn_all.p, L.m_hmask.p);
    rmask = L.m_hmask.p;
  }
  const Sell& A = L.A;
  launch(c, k_asm_gather, blocks_for(int64_t(A.nslices) * kAsmSplit * kSlice, 256), 256,
         (int)L.n,
         (const int*)A.sptr.p, (const int*)(A.sorted ? A.rperm.p : nullptr),
         (const int*)A.col.p, (const int*)L.m_cptr.p, (const int*)L.m_clist.p,
         (const double*)c.asm_E.p, rmask, (const int*)L.m_diagpos.p, A.v64.p, A.v32.p,
         L.m_dd.p);
  launch(c, k_blockdiag_inverse<1>, blocks_for(L.n, 128), 128, (int)L.n,
         (const double*)L.m_dd.p, L.dinv64.p, L.dinv32.p);
  L.h_val_stale = true;
  rows_refresh(c, A, false);
  if (L.has_AT && L.at_map.n) { // A^T: the same values, gathered in its order
    launch(c, k_gather_values, blocks_for(int64_t(L.AT.entries), 256), 256,
           (int64_t)L.AT.entries, (const int*)L.at_map.p, (const double*)A.v64.p, L.AT.v64.p,
           L.AT.v32.p);
    rows_refresh(c, L.AT, false);
  } else
    L.has_AT = false;
  L.ilu_ready = false;
  if (c.params.smoother != 0 || L.vk_ready) { // Vanka / ILU factors: full set-up again
    L.vk_ready = false;
    c.work_ready = false;
    c.version++;
  }
  c.values_dirty = true;
  if (c.transposed)
    ensure_AT(c, L); // the operator in use stays current
}

// kappa of level l's cells from level l + 1's (mean of the children)
void
coarsen_kappa(Context& c, int l)
{
  Level& C = c.L[l];
  Level& F = c.L[l + 1];
  if (C.child_n != C.mesh_ncells) {
    std::vector<int> ptr(C.mesh_ncells + 1, 0), ch(F.mesh_ncells);
    for (int64_t f = 0; f < F.mesh_ncells; ++f) {
      GB_REQUIRE(F.h_parent[f] < C.mesh_ncells, GB_EINVAL, "parent cell out of range");
      ptr[F.h_parent[f] + 1]++;
    }
    for (int64_t k = 0; k < C.mesh_ncells; ++k) {
      GB_REQUIRE(ptr[k + 1] > 0, GB_EINVAL, "a coarse cell without children");
      ptr[k + 1] += ptr[k];
    }
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    for (int64_t f = 0; f < F.mesh_ncells; ++f) // ascending children
      ch[fill[F.h_parent[f]]++] = static_cast<int>(f);
    GB_CUDA(cudaStreamSynchronize(c.stream));
    GB_CUDA(C.m_child_ptr.alloc(ptr.size()));
    GB_CUDA(C.m_child.alloc(ch.size()));
    GB_CUDA(h2d(c.stream, C.m_child_ptr.p, ptr.data(), ptr.size() * sizeof(int)));
    GB_CUDA(h2d(c.stream, C.m_child.p, ch.data(), ch.size() * sizeof(int)));
    C.child_n = C.mesh_ncells;
  }
  launch(c, k_kappa_coarsen, blocks_for(C.mesh_ncells, 256), 256, (int)C.mesh_ncells,
         (const int*)C.m_child_ptr.p, (const int*)C.m_child.p, (const double*)F.m_kappa.p,
         C.m_kappa.p);
}

// y += d * Form(x) on level l with the coefficient, convection and LPS of its
// last assembly (StdSolver::Form, Solver/stdsolver.cc:1041-1063): HNAverage(x),
// the element residuals added at the cells' own nodes in ascending cell order
// (CGDisc::Form and LocalToGlobal, DofHandler/cgdisc.h:367-380, 415-470),
// HNZero(x) and HNDistribute(y), as the reference does on a level with hanging
// nodes. Q1 cells: matrix-free residuals; patch elements (Q2, Q1 on patches,
// with LPS): the element matrices, then E x per element.
void
form_level(Context& c, int l, double* y, double* x, double d)
{
  Level& L = c.L[l];
  GB_REQUIRE(L.m_assembled, GB_ESTATE, "Form needs an assembled level (gb_assemble)");
  const int dim = L.mesh_dim;
  const int nl = L.mesh_deg == 1 ? 1 << dim : (dim == 3 ? 27 : 9);
  const int nc = static_cast<int>(L.mesh_ncells);
  const double b0 = L.m_beta[0], b1 = L.m_beta[1], b2 = L.m_beta[2];
  const bool conv = b0 != 0.0 || b1 != 0.0 || b2 != 0.0;
  const double g = 0.5 / std::sqrt(3.0);
  Emit<double> Em{ c, nullptr };
  if (L.has_hn())
    Em.hn_average(l, x);
  GB_CUDA(c.asm_R.n >= size_t(nc) * nl ? cudaSuccess : c.asm_R.alloc(size_t(nc) * nl));
  if (L.mesh_deg == 1) {
#define GB_FORM(D, CV)                                                                 \
  launch(c, k_q1_form<D, CV>, blocks_for(nc, 128), 128, nc, (const int*)L.m_cells.p,   \
         (const double*)L.m_coords.p, (const double*)L.m_kappa.p, b0, b1, b2, g,        \
         (const double*)x, c.asm_R.p)
    if (dim == 2) {
      if (conv) GB_FORM(2, true); else GB_FORM(2, false);
    } else {
      if (conv) GB_FORM(3, true); else GB_FORM(3, false);
    }
#undef GB_FORM
  } else {
    GB_CUDA(c.asm_E.n >= size_t(nc) * nl * nl ? cudaSuccess
                                               : c.asm_E.alloc(size_t(nc) * nl * nl));
    const bool pq1 = L.mesh_deg == 3, lps = conv && L.m_lps_s0 > 0.0;
    const double bnorm = std::sqrt(b0 * b0 + b1 * b1 + b2 * b2) + 1e-6;
#define GB_ELEM2(D, CV, LP, PQ)                                                          \
  launch(c, k_q2_element_warp<D, CV, LP, PQ>, blocks_for(int64_t(nc) * 32, 128), 128, nc, \
         (const int*)L.m_cells.p, (const double*)L.m_coords.p, (const double*)L.m_kappa.p, \
         b0, b1, b2, c.asm_E.p, L.m_lps_s0, L.m_lps_xeta, bnorm, g)
#define GB_ELEM2K(D, PQ)                                                                 \
  do {                                                                                   \
    if (lps) GB_ELEM2(D, true, true, PQ);                                                \
    else if (conv) GB_ELEM2(D, true, false, PQ);                                         \
    else GB_ELEM2(D, false, false, PQ);                                                  \
  } while (0)
    if (dim == 2) {
      if (pq1) GB_ELEM2K(2, true); else GB_ELEM2K(2, false);
      launch(c, k_elem_apply<9>, blocks_for(int64_t(nc) * 32, 128), 128, nc,
             (const int*)L.m_cells.p, (const double*)c.asm_E.p, (const double*)x, c.asm_R.p);
    } else {
      if (pq1) GB_ELEM2K(3, true); else GB_ELEM2K(3, false);
      launch(c, k_elem_apply<27>, blocks_for(int64_t(nc) * 32, 128), 128, nc,
             (const int*)L.m_cells.p, (const double*)c.asm_E.p, (const double*)x, c.asm_R.p);
    }
#undef GB_ELEM2
#undef GB_ELEM2K
  }
  launch(c, k_form_gather, blocks_for(L.n, 256), 256, (int)L.n, (const int*)L.m_nptr.p,
         (const int*)L.m_nlist.p, (const double*)c.asm_R.p, d, y);
  if (L.has_hn()) {
    Em.hn_zero(l, x);
    Em.hn_distribute(l, y);
  }
}

void
check_mesh(const Level& L)
{
  GB_REQUIRE(L.mesh_ncells > 0 && L.mesh_n == L.n, GB_ESTATE,
             "no mesh for this level's matrix (gb_level_set_mesh)");
}

void
load_kappa(Context& c, Level& L, const double* kappa, int where)
{
  GB_REQUIRE(kappa, GB_EINVAL, "null kappa");
  GB_REQUIRE(where == 0 || where == 1, GB_EINVAL, "kappa location must be 0 (host) or 1 (device)");
  GB_CUDA(cudaMemcpyAsync(L.m_kappa.p, kappa, L.mesh_ncells * sizeof(double),
                          where ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c.stream));
  if (!where)
    GB_CUDA(cudaStreamSynchronize(c.stream)); // the host array ends with the call
}

} // namespace gb

using namespace gb;

extern "C" {

int
gb_level_set_cells(gb_ctx* ctx, int lvl, int64_t ncells, int nloc,
                   const int64_t* cell_nodes, const double* kloc, const double* cell_scale)
{
  GB_API_BEGIN
  Level& L = level_with_matrix(*ctx, lvl);
  GB_REQUIRE(ncells >= 1 && ncells < (int64_t(1) << 31) / 32, GB_EINVAL,
             "ncells out of range");
  GB_REQUIRE(nloc >= 1 && nloc <= 32, GB_EINVAL, "nloc must be in 1..32");
  GB_REQUIRE(cell_nodes && kloc, GB_EINVAL, "null array");
  std::vector<int> cn(size_t(ncells) * nloc);
  for (int64_t c = 0; c < ncells; ++c)
    for (int i = 0; i < nloc; ++i) {
      const int64_t v = cell_nodes[c * nloc + i];
      GB_REQUIRE(v >= 0 && v < L.n, GB_EINVAL, "cell node out of range");
      cn[size_t(i) * ncells + c] = static_cast<int>(v);
    }
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  GB_CUDA(L.cells.alloc(cn.size()));
  GB_CUDA(L.kloc.alloc(size_t(nloc) * nloc));
  GB_CUDA(L.grad.alloc(ncells));
  GB_CUDA(cudaMemcpyAsync(L.cells.p, cn.data(), cn.size() * sizeof(int),
                          cudaMemcpyHostToDevice, ctx->stream));
  GB_CUDA(cudaMemcpyAsync(L.kloc.p, kloc, size_t(nloc) * nloc * sizeof(double),
                          cudaMemcpyHostToDevice, ctx->stream));
  L.has_scale = cell_scale != nullptr;
  if (cell_scale) {
    GB_CUDA(L.cscale.alloc(ncells));
    GB_CUDA(cudaMemcpyAsync(L.cscale.p, cell_scale, ncells * sizeof(double),
                            cudaMemcpyHostToDevice, ctx->stream));
  }
  GB_CUDA(cudaStreamSynchronize(ctx->stream)); // host arrays end with the call
  L.ncells = static_cast<int>(ncells);
  L.nloc = nloc;
  L.cells_n = L.n;
  GB_API_END
}

int
gb_level_set_functional(gb_ctx* ctx, int lvl, const double* mloc, const double* cell_scale)
{
  GB_API_BEGIN
  Level& L = level_with_matrix(*ctx, lvl);
  GB_REQUIRE(L.ncells > 0 && L.cells_n == L.n, GB_ESTATE,
             "no cells for this level's matrix (gb_level_set_cells)");
  GB_REQUIRE(L.B == 1, GB_EINVAL, "functional needs block size 1");
  GB_REQUIRE(mloc, GB_EINVAL, "null array");
  const int64_t n = L.n, nc = L.ncells;
  const int nl = L.nloc;
  // cell nodes back from the device layout
  std::vector<int> cn(size_t(nc) * nl);
  GB_CUDA(cudaMemcpyAsync(cn.data(), L.cells.p, cn.size() * sizeof(int),
                          cudaMemcpyDeviceToHost, ctx->stream));
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  // per row: columns sorted with their stencil positions, for the lookups
  std::vector<std::pair<int64_t, int64_t>> sc(L.h_col.size());
  for (int64_t i = 0; i < n; ++i) {
    for (int64_t k = L.h_rowptr[i]; k < L.h_rowptr[i + 1]; ++k)
      sc[k] = { L.h_col[k], k };
    std::sort(sc.begin() + L.h_rowptr[i], sc.begin() + L.h_rowptr[i + 1]);
  }
  std::vector<double> mv(L.h_col.size(), 0.0);
  for (int64_t c = 0; c < nc; ++c) {
    const double w = cell_scale ? cell_scale[c] : 1.0;
    for (int a = 0; a < nl; ++a) {
      const int64_t r = cn[size_t(a) * nc + c];
      auto b = sc.begin() + L.h_rowptr[r], e = sc.begin() + L.h_rowptr[r + 1];
      for (int q = 0; q < nl; ++q) {
        const int64_t col = cn[size_t(q) * nc + c];
        auto f = std::lower_bound(b, e, std::make_pair(col, int64_t(-1)));
        GB_REQUIRE(f != e && f->first == col, GB_EINVAL,
                   "cell matrix entry outside the level's sparsity pattern");
        mv[f->second] += w * mloc[a * nl + q];
      }
    }
  }
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  build_sell(L.M, n, L.h_rowptr.data(), L.h_col.data(), mv.data(), ctx->stream);
  L.func_n = n;
  GB_API_END
}

int
gb_level_set_mesh(gb_ctx* ctx, int lvl, int dim, int64_t ncells, const int64_t* cell_nodes,
                  const double* coords, const int64_t* parent)
{
  return gb_level_set_mesh_degree(ctx, lvl, dim, 1, ncells, cell_nodes, coords, parent);
}

int
gb_level_set_mesh_degree(gb_ctx* ctx, int lvl, int dim, int degree, int64_t ncells,
                         const int64_t* cell_nodes, const double* coords,
                         const int64_t* parent)
{
  GB_API_BEGIN
  ctx->version++;
  Level& L = level_with_matrix(*ctx, lvl);
  GB_REQUIRE(dim == 2 || dim == 3, GB_EINVAL, "dim must be 2 or 3");
  GB_REQUIRE(degree >= 1 && degree <= 3, GB_EINVAL,
             "degree must be 1 (Q1 cells), 2 (Q2 patches) or 3 (Q1 patches)");
  GB_REQUIRE(L.B == 1, GB_EINVAL, "device assembly needs block size 1");
  GB_REQUIRE(!L.has_hn() || L.h_hnidx.size() == size_t(L.n), GB_EINVAL,
             "the hanging nodes were set for another matrix size");
  const int nl = degree == 1 ? 1 << dim : (dim == 3 ? 27 : 9);
  GB_REQUIRE(ncells >= 1 && ncells * nl * nl < (int64_t(1) << 31), GB_EINVAL,
             "ncells out of range");
  GB_REQUIRE(cell_nodes && coords, GB_EINVAL, "null array");
  GB_REQUIRE(lvl == 0 || parent, GB_EINVAL, "parent cells are needed above level 0");
  const Sell& A = L.A;
  const int64_t n = L.n;
  // SELL position of row r's stencil entry k: sptr[t / 32] + (k - rowptr[r]) * 32 + t % 32
  std::vector<int> sptr(A.nslices + 1), perm(n), slot(n);
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  GB_CUDA(cudaMemcpy(sptr.data(), A.sptr.p, sptr.size() * sizeof(int), cudaMemcpyDeviceToHost));
  if (A.sorted)
    GB_CUDA(cudaMemcpy(perm.data(), A.rperm.p, n * sizeof(int), cudaMemcpyDeviceToHost));
  else
    for (int64_t t = 0; t < n; ++t)
      perm[t] = static_cast<int>(t);
  for (int64_t t = 0; t < n; ++t)
    slot[perm[t]] = static_cast<int>(t);
  auto sell_pos = [&](int64_t r, int64_t k) {
    const int64_t t = slot[r];
    return sptr[t / kSlice] + (k - L.h_rowptr[r]) * kSlice + t % kSlice;
  };
  for (int64_t k = 0; k < ncells * nl; ++k)
    GB_REQUIRE(cell_nodes[k] >= 0 && cell_nodes[k] < n, GB_EINVAL, "cell node out of range");
  // The matrix couples the condensed element indices: on a level with hanging
  // nodes every hanging node of a cell (edges, then faces, ascending slots)
  // gives way to the one parent that the cell lacks, and the cell's element
  // matrix is condensed by the steps recorded here (CondOp).
  std::vector<int64_t> ci(cell_nodes, cell_nodes + ncells * nl);
  std::vector<int> hcells, hopptr(1, 0);
  std::vector<CondOp> hops;
  if (L.has_hn()) {
    for (int64_t c = 0; c < ncells; ++c) {
      int64_t* id = ci.data() + c * nl;
      const size_t op0 = hops.size();
      for (int ph = 0; ph < 2; ++ph)
        for (int s = 0; s < nl; ++s) {
          const int hi = L.h_hnidx[id[s]];
          if (hi < 0 || L.h_hncond[hi].phase != ph)
            continue;
          const Level::HnCond& hc = L.h_hncond[hi];
          int miss = -1, at[9];
          for (int j = 0; j < hc.np; ++j) {
            at[j] = -1;
            for (int t = 0; t < nl; ++t)
              if (id[t] == hc.par[j])
                at[j] = t;
            if (at[j] < 0) {
              GB_REQUIRE(miss < 0, GB_EINVAL,
                         "a cell lacks more than one parent of its hanging node");
              miss = j;
            }
          }
          GB_REQUIRE(miss >= 0, GB_EINVAL, "a cell holds every parent of its hanging node");
          for (int j = 0; j < hc.np; ++j)
            if (at[j] >= 0)
              hops.push_back(CondOp{ s, at[j], hc.w[j] });
          hops.push_back(CondOp{ s, -1, hc.w[miss] });
          id[s] = hc.par[miss];
        }
      if (hops.size() > op0) {
        hcells.push_back(static_cast<int>(c));
        hopptr.push_back(static_cast<int>(hops.size()));
      }
    }
  }
  std::vector<std::pair<int64_t, int64_t>> sc(L.h_col.size());
  for (int64_t i = 0; i < n; ++i) {
    for (int64_t k = L.h_rowptr[i]; k < L.h_rowptr[i + 1]; ++k)
      sc[k] = { L.h_col[k], k };
    std::sort(sc.begin() + L.h_rowptr[i], sc.begin() + L.h_rowptr[i + 1]);
  }
  // positions of every (cell, a, b), then the contributions per position in
  // ascending cell order (counting sort)
  const int64_t np = ncells * nl * nl;
  std::vector<int> pos(np), cn(size_t(ncells) * nl);
  std::vector<int> cptr(A.entries + 1, 0);
  for (int64_t c = 0; c < ncells; ++c)
    for (int a = 0; a < nl; ++a) {
      const int64_t r = ci[c * nl + a];
      cn[size_t(a) * ncells + c] = static_cast<int>(cell_nodes[c * nl + a]); // geometry
      auto b0 = sc.begin() + L.h_rowptr[r], b1 = sc.begin() + L.h_rowptr[r + 1];
      for (int b = 0; b < nl; ++b) {
        const int64_t q = ci[c * nl + b];
        auto it = std::lower_bound(b0, b1, std::make_pair(q, int64_t(-1)));
        GB_REQUIRE(it != b1 && it->first == q, GB_EINVAL,
                   "a cell couples two nodes that the matrix pattern does not");
        const int e = static_cast<int>(sell_pos(r, it->second));
        pos[(c * nl + a) * nl + b] = e;
        cptr[e + 1]++;
      }
    }
  for (size_t e = 0; e < A.entries; ++e)
    cptr[e + 1] += cptr[e];
  std::vector<int> fill(cptr.begin(), cptr.end() - 1), clist(np);
  for (int64_t c = 0; c < ncells; ++c)
    for (int p = 0; p < nl * nl; ++p)
      clist[fill[pos[c * nl * nl + p]]++] = static_cast<int>(int64_t(p) * ncells + c);
  std::vector<int> dpos(n);
  for (int64_t r = 0; r < n; ++r)
    dpos[r] = static_cast<int>(sell_pos(r, L.h_diag[r]));
  std::vector<int> nptr(n + 1, 0), nlist(size_t(ncells) * nl);
  for (int64_t c = 0; c < ncells; ++c) // the cells' own nodes (Form, then HNDistribute)
    for (int a = 0; a < nl; ++a)
      nptr[cell_nodes[c * nl + a] + 1]++;
  for (int64_t r = 0; r < n; ++r)
    nptr[r + 1] += nptr[r];
  {
    std::vector<int> fill(nptr.begin(), nptr.end() - 1);
    for (int64_t c = 0; c < ncells; ++c) // ascending cells
      for (int a = 0; a < nl; ++a)
        nlist[fill[cell_nodes[c * nl + a]]++] = static_cast<int>(int64_t(a) * ncells + c);
  }
  std::vector<int64_t> par;
  if (lvl > 0) {
    par.assign(parent, parent + ncells);
    for (int64_t c = 0; c < ncells; ++c)
      GB_REQUIRE(par[c] >= 0, GB_EINVAL, "negative parent cell");
  }
  GB_CUDA(L.m_cells.alloc(cn.size()));
  GB_CUDA(L.m_coords.alloc(size_t(n) * dim));
  GB_CUDA(L.m_cptr.alloc(cptr.size()));
  GB_CUDA(L.m_clist.alloc(clist.size()));
  GB_CUDA(L.m_diagpos.alloc(n));
  GB_CUDA(L.m_kappa.alloc(ncells));
  GB_CUDA(L.m_dd.alloc(n));
  GB_CUDA(h2d(ctx->stream, L.m_cells.p, cn.data(), cn.size() * sizeof(int)));
  GB_CUDA(h2d(ctx->stream, L.m_coords.p, coords, size_t(n) * dim * sizeof(double)));
  GB_CUDA(h2d(ctx->stream, L.m_cptr.p, cptr.data(), cptr.size() * sizeof(int)));
  GB_CUDA(h2d(ctx->stream, L.m_clist.p, clist.data(), clist.size() * sizeof(int)));
  GB_CUDA(h2d(ctx->stream, L.m_diagpos.p, dpos.data(), n * sizeof(int)));
  GB_CUDA(L.m_nptr.alloc(nptr.size()));
  GB_CUDA(L.m_nlist.alloc(nlist.size()));
  GB_CUDA(h2d(ctx->stream, L.m_nptr.p, nptr.data(), nptr.size() * sizeof(int)));
  GB_CUDA(h2d(ctx->stream, L.m_nlist.p, nlist.data(), nlist.size() * sizeof(int)));
  L.m_nhcells = static_cast<int>(hcells.size());
  if (!hcells.empty()) {
    GB_CUDA(L.m_hcells.alloc(hcells.size()));
    GB_CUDA(L.m_hopptr.alloc(hopptr.size()));
    GB_CUDA(L.m_hops.alloc(hops.size()));
    GB_CUDA(h2d(ctx->stream, L.m_hcells.p, hcells.data(), hcells.size() * sizeof(int)));
    GB_CUDA(h2d(ctx->stream, L.m_hopptr.p, hopptr.data(), hopptr.size() * sizeof(int)));
    GB_CUDA(h2d(ctx->stream, L.m_hops.p, hops.data(), hops.size() * sizeof(CondOp)));
  }
  if (L.has_hn())
    GB_CUDA(L.m_hmask.alloc(n));
  L.m_assembled = false;
  L.h_parent.swap(par);
  L.mesh_dim = dim;
  L.mesh_deg = degree;
  L.mesh_ncells = ncells;
  L.mesh_n = n;
  if (L.has_AT) { // the transpose again, with its map for device refreshes
    L.has_AT = false;
    ensure_AT(*ctx, L);
  }
  if (lvl > 0)
    ctx->L[lvl - 1].child_n = -1; // its child lists follow this level's parents
  GB_API_END
}

int
gb_set_assembly_lps(gb_ctx* ctx, double sdelta0, double xeta0)
{
  GB_API_BEGIN
  GB_REQUIRE(sdelta0 >= 0.0 && std::isfinite(sdelta0), GB_EINVAL, "sdelta0 must be >= 0");
  GB_REQUIRE(xeta0 > 0.0 && std::isfinite(xeta0), GB_EINVAL, "xeta0 must be > 0");
  ctx->lps_s0 = sdelta0;
  ctx->lps_xeta = xeta0;
  GB_API_END
}

int
gb_assemble(gb_ctx* ctx, int lvl, const double* kappa, int where, const double* beta)
{
  GB_API_BEGIN
  Level& L = level_with_matrix(*ctx, lvl);
  check_mesh(L);
  load_kappa(*ctx, L, kappa, where);
  assemble_level(*ctx, lvl, beta);
  GB_API_END
}

int
gb_assemble_levels(gb_ctx* ctx, const double* kappa, int where, const double* beta)
{
  GB_API_BEGIN
  GB_REQUIRE(ctx->nlevels >= 1, GB_ESTATE, "no levels");
  for (int l = 0; l < ctx->nlevels; ++l) {
    GB_REQUIRE(ctx->L[l].has_matrix, GB_ESTATE, "every level needs a matrix");
    check_mesh(ctx->L[l]);
  }
  const int fl = ctx->nlevels - 1;
  load_kappa(*ctx, ctx->L[fl], kappa, where);
  assemble_level(*ctx, fl, beta);
  for (int l = fl - 1; l >= 0; --l) {
    coarsen_kappa(*ctx, l);
    assemble_level(*ctx, l, beta);
  }
  GB_API_END
}

int
gb_level_get_values(gb_ctx* ctx, int lvl, double* val)
{
  GB_API_BEGIN
  Level& L = level_with_matrix(*ctx, lvl);
  GB_REQUIRE(val, GB_EINVAL, "null array");
  host_values(*ctx, L);
  std::memcpy(val, L.h_val.data(), L.h_val.size() * sizeof(double));
  GB_API_END
}

int
gb_form(gb_ctx* ctx, int lvl, int y, int x, double d)
{
  GB_API_BEGIN
  Level& L = level_with_matrix(*ctx, lvl);
  check_mesh(L);
  GB_REQUIRE(y != x, GB_EINVAL, "y and x must differ");
  form_level(*ctx, lvl, vec(*ctx, lvl, y), vec(*ctx, lvl, x), d);
  GB_API_END
}

int
gb_newton_residual(gb_ctx* ctx, int y, int x, int b, double* norm)
{
  GB_API_BEGIN
  GB_REQUIRE(ctx->nlevels >= 1, GB_ESTATE, "no levels");
  const int fl = ctx->nlevels - 1;
  Level& L = level_with_matrix(*ctx, fl);
  check_mesh(L);
  GB_REQUIRE(y != x && y != b, GB_EINVAL, "y must differ from x and b");
  GB_REQUIRE(!L.pf_mask, GB_EINVAL, "Newton residual with a pressure filter");
  double* yv = vec(*ctx, fl, y);
  launch(*ctx, k_equ<double, double>, stream_blocks(L.n), 256, (int64_t)L.n, yv, 1.0,
         (const double*)vec(*ctx, fl, b));
  form_level(*ctx, fl, yv, vec(*ctx, fl, x), -1.0);
  GB_CUDA(ctx->nrm.alloc(1));
  GB_CUDA(cudaMemsetAsync(ctx->nrm.p, 0, sizeof(unsigned long long), ctx->stream));
  launch(*ctx, k_dirichlet_absmax, blocks_for(L.n, 256), 256, (int)L.n,
         (const uint8_t*)L.dirmask.p, yv, ctx->nrm.p);
  if (norm) {
    unsigned long long m = 0;
    GB_CUDA(cudaMemcpyAsync(&m, ctx->nrm.p, sizeof(m), cudaMemcpyDeviceToHost, ctx->stream));
    GB_CUDA(cudaStreamSynchronize(ctx->stream));
    double v;
    std::memcpy(&v, &m, sizeof(v));
    *norm = v;
  }
  GB_API_END
}

int
gb_vec_write_backup(gb_ctx* ctx, int lvl, int id, const char* path, int binary)
{
  GB_API_BEGIN
  Level& L = level_with_matrix(*ctx, lvl);
  GB_REQUIRE(path, GB_EINVAL, "null path");
  std::vector<double> v(L.ndof());
  GB_CUDA(cudaMemcpyAsync(v.data(), vec(*ctx, lvl, id), v.size() * sizeof(double),
                          cudaMemcpyDeviceToHost, ctx->stream));
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  FILE* f = std::fopen(path, binary ? "wb" : "w");
  GB_REQUIRE(f, GB_EINVAL, std::string("cannot open ") + path + " for writing");
  bool ok = true;
  if (binary) { // CompVector::BinWrite + "BackUpEnd"
    ok = std::fprintf(f, "%d %lld\n[", L.B, (long long)L.n) > 0 &&
         std::fwrite(v.data(), sizeof(double), v.size(), f) == v.size() &&
         std::fprintf(f, "]BackUpEnd\n") > 0;
  } else { // WriteBackUp: scientific, 16 digits, one node per line
    ok = std::fprintf(f, "%lld %d\n", (long long)L.n, L.B) > 0;
    for (int64_t i = 0; i < L.n && ok; ++i) {
      for (int c = 0; c < L.B && ok; ++c)
        ok = std::fprintf(f, "%.16e ", v[i * L.B + c]) > 0;
      ok = ok && std::fputc('\n', f) != EOF;
    }
    ok = ok && std::fprintf(f, "BackUpEnd\n") > 0;
  }
  ok = (std::fclose(f) == 0) && ok;
  GB_REQUIRE(ok, GB_EINVAL, std::string("write error on ") + path);
  GB_API_END
}

int
gb_vec_write_vtk(gb_ctx* ctx, int lvl, int id, const char* name, int step, int dim,
                 int64_t ncells, int nodes_per_cell, const int64_t* cell_nodes,
                 const double* coords, double time, const char* title)
{
  GB_API_BEGIN
  Level& L = level_with_matrix(*ctx, lvl);
  GB_REQUIRE(name && cell_nodes && coords, GB_EINVAL, "null argument");
  GB_REQUIRE(dim == 2 || dim == 3, GB_EINVAL, "dim must be 2 or 3");
  GB_REQUIRE(nodes_per_cell == (1 << dim), GB_EINVAL,
             "cells need 4 (2D) or 8 (3D) nodes");
  GB_REQUIRE(ncells >= 0 && step >= 0, GB_EINVAL, "bad cell count or step");
  for (int64_t k = 0; k < ncells * nodes_per_cell; ++k)
    GB_REQUIRE(cell_nodes[k] >= 0 && cell_nodes[k] < L.n, GB_EINVAL,
               "cell node out of range");
  // the hanging values averaged (CGDisc::VisuVtk) on a copy of the vector
  std::vector<double> v(L.ndof());
  const double* src = vec(*ctx, lvl, id);
  if (L.has_hn()) {
    DeviceArray<double> t;
    GB_CUDA(t.alloc(v.size()));
    GB_CUDA(cudaMemcpyAsync(t.p, src, v.size() * sizeof(double), cudaMemcpyDeviceToDevice,
                            ctx->stream));
    Emit<double> E{ *ctx, nullptr };
    E.hn_average(lvl, t.p);
    GB_CUDA(cudaMemcpyAsync(v.data(), t.p, v.size() * sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->stream));
    GB_CUDA(cudaStreamSynchronize(ctx->stream));
  } else {
    GB_CUDA(cudaMemcpyAsync(v.data(), src, v.size() * sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->stream));
    GB_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  // Visualization::step + compose_name: <name>.%05d, then ".vtk"
  char fn[4096];
  GB_REQUIRE(std::snprintf(fn, sizeof fn, "%s.%05d.vtk", name, step) < int(sizeof fn),
             GB_EINVAL, "file name too long");
  FILE* f = std::fopen(fn, "w");
  GB_REQUIRE(f, GB_EINVAL, std::string("cannot open ") + fn + " for writing");
  // Visualization::vtk (Discretization/Q1/vtk.cc): legacy ASCII; doubles as a
  // C++ stream prints them by default (%g, 6 digits); a vertex prints each
  // coordinate followed by a tab, 2D points add " 0"
  bool ok = std::fprintf(f, "# vtk DataFile Version 2.0 \noutput from GascoigneStd, %s\n"
                            "ASCII\nDATASET UNSTRUCTURED_GRID\nFIELD FieldData 1\n"
                            "TIME 1 1 double\n%g\n", title ? title : "", time) > 0;
  ok = ok && std::fprintf(f, "POINTS %lld DOUBLE \n", (long long)L.n) > 0;
  for (int64_t i = 0; i < L.n && ok; ++i) {
    for (int d = 0; d < dim && ok; ++d)
      ok = std::fprintf(f, "%g\t", coords[i * dim + d]) > 0;
    ok = ok && std::fputs(dim == 2 ? " 0\n" : "\n", f) >= 0;
  }
  ok = ok && std::fprintf(f, "\n\nCELLS %lld %lld\n", (long long)ncells,
                          (long long)(ncells * (nodes_per_cell + 1))) > 0;
  for (int64_t c = 0; c < ncells && ok; ++c) {
    ok = std::fprintf(f, "%d ", nodes_per_cell) > 0;
    for (int a = 0; a < nodes_per_cell && ok; ++a)
      ok = std::fprintf(f, "%lld ", (long long)cell_nodes[c * nodes_per_cell + a]) > 0;
    ok = ok && std::fputc('\n', f) != EOF;
  }
  ok = ok && std::fprintf(f, "\nCELL_TYPES %lld\n", (long long)ncells) > 0;
  for (int64_t c = 0; c < ncells && ok; ++c)
    ok = std::fputs(dim == 2 ? "9 " : "12 ", f) >= 0;
  ok = ok && std::fputc('\n', f) != EOF;
  // _vtk_pointdata: one scalar per component, u000, u001, ...
  for (int comp = 0; comp < L.B && ok; ++comp) {
    if (comp == 0)
      ok = std::fprintf(f, "POINT_DATA %lld\n", (long long)L.n) > 0;
    ok = ok && std::fprintf(f, "SCALARS u%03d DOUBLE \nLOOKUP_TABLE default\n", comp) > 0;
    for (int64_t i = 0; i < L.n && ok; ++i)
      ok = std::fprintf(f, "%g\n", v[i * L.B + comp]) > 0;
    ok = ok && std::fputs("\n\n", f) >= 0;
  }
  ok = (std::fclose(f) == 0) && ok;
  GB_REQUIRE(ok, GB_EINVAL, std::string("write error on ") + fn);
  GB_API_END
}

int
gb_vec_read_backup(gb_ctx* ctx, int lvl, int id, const char* path, int binary, int add)
{
  GB_API_BEGIN
  Level& L = level_with_matrix(*ctx, lvl);
  GB_REQUIRE(path, GB_EINVAL, "null path");
  FILE* f = std::fopen(path, binary ? "rb" : "r");
  GB_REQUIRE(f, GB_EINVAL, std::string("backup file ") + path + " not found");
  std::vector<double> v(L.ndof());
  long long n = -1;
  int comp = -1;
  bool ok;
  char tail[16] = { 0 };
  if (binary) { // "ncomp n\n[" raw values "]" then "BackUpEnd"
    char br = 0;
    ok = std::fscanf(f, "%d %lld %c", &comp, &n, &br) == 3 && br == '[' && n == L.n &&
         comp == L.B && std::fread(v.data(), sizeof(double), v.size(), f) == v.size() &&
         std::fscanf(f, " %c", &br) == 1 && br == ']';
  } else { // "n ncomp", n * ncomp numbers, "BackUpEnd"
    ok = std::fscanf(f, "%lld %d", &n, &comp) == 2 && n == L.n && comp == L.B;
    for (size_t k = 0; k < v.size() && ok; ++k)
      ok = std::fscanf(f, "%lf", &v[k]) == 1;
  }
  ok = ok && std::fscanf(f, " %15s", tail) == 1 && std::string(tail) == "BackUpEnd";
  std::fclose(f);
  GB_REQUIRE(ok, GB_EINVAL,
             std::string("backup file ") + path + " does not hold " +
               std::to_string(L.n) + " nodes of " + std::to_string(L.B) +
               " components ending in BackUpEnd");
  double* dst = vec(*ctx, lvl, id);
  if (add) { // ReadBackUp adds the file to the vector
    std::vector<double> cur(v.size());
    GB_CUDA(cudaMemcpyAsync(cur.data(), dst, v.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, ctx->stream));
    GB_CUDA(cudaStreamSynchronize(ctx->stream));
    for (size_t k = 0; k < v.size(); ++k)
      v[k] = cur[k] + v[k];
  }
  GB_CUDA(h2d(ctx->stream, dst, v.data(), v.size() * sizeof(double)));
  GB_API_END
}

int
gb_level_get_kappa(gb_ctx* ctx, int lvl, double* kappa)
{
  GB_API_BEGIN
  Level& L = level_with_matrix(*ctx, lvl);
  check_mesh(L);
  GB_REQUIRE(kappa, GB_EINVAL, "null array");
  GB_CUDA(cudaMemcpyAsync(kappa, L.m_kappa.p, L.mesh_ncells * sizeof(double),
                          cudaMemcpyDeviceToHost, ctx->stream));
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  GB_API_END
}

int
gb_functional(gb_ctx* ctx, int lvl, int u, int g, double* J)
{
  GB_API_BEGIN
  Level& L = level_with_matrix(*ctx, lvl);
  GB_REQUIRE(L.func_n == L.n, GB_ESTATE,
             "no functional for this level's matrix (gb_level_set_functional)");
  GB_REQUIRE(u != g, GB_EINVAL, "u and g must differ");
  const double* ud = vec(*ctx, lvl, u);
  double* gd = vec(*ctx, lvl, g);
  // g = 2 M u, J = u . (M u) = (u . g) / 2, then g = 0 on Dirichlet dofs
  spmv<kAx, double, double, double>(*ctx, L, L.M, ud, gd, nullptr, nullptr, 2.0);
  if (J)
    dot_dev(*ctx, L.ndof(), ud, gd, RedOut{ ctx->scal.p + 6, nullptr, nullptr, 0 });
  launch(*ctx, k_dirichlet_zero<double>, blocks_for(L.ndir, 256), 256, L.ndir,
         (const int*)L.dirlist.p, gd);
  if (J)
    *J = 0.5 * read_scalar(*ctx, ctx->scal.p + 6);
  GB_API_END
}

int
gb_ctx_get_stream(const gb_ctx* ctx, void** stream)
{
  if (!ctx || !stream)
    return GB_EINVAL;
  *stream = ctx->stream;
  return GB_OK;
}

int
gb_coeff_gradient(gb_ctx* ctx, int lvl, int u, int lam, double* grad, int64_t ncells)
{
  GB_API_BEGIN
  Level& L = level_with_matrix(*ctx, lvl);
  GB_REQUIRE(L.ncells > 0 && L.cells_n == L.n, GB_ESTATE,
             "no cells for this level's matrix (gb_level_set_cells)");
  GB_REQUIRE(L.B == 1, GB_EINVAL, "coefficient gradient needs block size 1");
  GB_REQUIRE(ncells == L.ncells, GB_EINVAL, "ncells differs from the level's cells");
  const double* ud = vec(*ctx, lvl, u);
  const double* ld = vec(*ctx, lvl, lam);
  const int nb = blocks_for(L.ncells, 256);
  const double* sc = L.has_scale ? L.cscale.p : nullptr;
  const uint8_t* mk = L.dirmask.p;
  switch (L.nloc) {
    case 4:
      launch(*ctx, k_coeff_gradient<4>, nb, 256, L.ncells, 4, (const int*)L.cells.p,
             (const double*)L.kloc.p, sc, ud, ld, mk, L.grad.p);
      break;
    case 8:
      launch(*ctx, k_coeff_gradient<8>, nb, 256, L.ncells, 8, (const int*)L.cells.p,
             (const double*)L.kloc.p, sc, ud, ld, mk, L.grad.p);
      break;
    case 9:
      launch(*ctx, k_coeff_gradient<9>, nb, 256, L.ncells, 9, (const int*)L.cells.p,
             (const double*)L.kloc.p, sc, ud, ld, mk, L.grad.p);
      break;
    case 27:
      launch(*ctx, k_coeff_gradient<27>, nb, 256, L.ncells, 27, (const int*)L.cells.p,
             (const double*)L.kloc.p, sc, ud, ld, mk, L.grad.p);
      break;
    default:
      launch(*ctx, k_coeff_gradient<0>, nb, 256, L.ncells, L.nloc, (const int*)L.cells.p,
             (const double*)L.kloc.p, sc, ud, ld, mk, L.grad.p);
  }
  if (grad) {
    GB_CUDA(cudaMemcpyAsync(grad, L.grad.p, ncells * sizeof(double),
                            cudaMemcpyDeviceToHost, ctx->stream));
    GB_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  GB_API_END
}

} // extern "C"
