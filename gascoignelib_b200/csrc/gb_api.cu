// The C-ABI (include/gascoigne_b200.h): context, parameters, levels,
// vectors, operators, smoothers, transfers, solves, diagnostics.
#include "gb_cycle.cuh"

using namespace gb;

extern "C" {

int
gb_ctx_create(gb_ctx** out, int device)
{
  if (!out)
    return GB_EINVAL;
  *out = nullptr;
  gb_ctx* ctx = new (std::nothrow) gb_ctx;
  if (!ctx)
    return GB_ENOMEM;
  try {
    ctx->device = device;
    if (const char* e = getenv("GB_COARSE_KERNEL"))
      ctx->coarse_on = atoi(e) != 0;
    if (const char* e = getenv("GB_GRAPH"))
      ctx->use_graph = atoi(e) != 0;
    if (const char* e = getenv("GB_COARSE_DENSE"))
      ctx->coarse_dense = atoi(e) != 0;
    if (const char* e = getenv("GB_MID"))
      ctx->mid_on = atoi(e) != 0;
    if (const char* e = getenv("GB_ILU_HOST"))
      ctx->ilu_host = atoi(e) != 0;
    if (const char* e = getenv("GB_RB"))
      ctx->rb_on = atoi(e) != 0;
    if (const char* e = getenv("GB_ROW_ORDER"))
      ctx->row_order = atoi(e) != 0;
    if (const char* e = getenv("GB_ILU_CTA_ROWS"))
      ctx->ilu_cta_rows = std::max(0, atoi(e));
    if (const char* e = getenv("GB_VANKA_HOST"))
      ctx->vanka_host = atoi(e) != 0;
    if (const char* e = getenv("GB_CLUSTER"))
      ctx->cluster_on = atoi(e) != 0;
    if (const char* e = getenv("GB_CLUSTER_ROWS"))
      ctx->cluster_rows = atoll(e);
    if (const char* e = getenv("GB_JACOBI2"))
      ctx->jacobi2 = atoi(e) != 0;
    if (const char* e = getenv("GB_PDL"))
      ctx->pdl = atoi(e) != 0;
    GB_CUDA(cudaSetDevice(device));
    GB_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    GB_CUDA(cudaEventCreate(&ctx->ev0));
    GB_CUDA(cudaEventCreate(&ctx->ev1));
    GB_CUDA(ctx->partials.alloc(size_t(kCgsMaxJ + 1) *
                                std::max(kMaxRedBlocks, kCgsMaxBlocks)));
    GB_CUDA(ctx->ticket.alloc(1));
    GB_CUDA(cudaMemset(ctx->ticket.p, 0, sizeof(unsigned)));
    GB_CUDA(ctx->scal.alloc(16));
    GB_CUDA(cudaMallocHost(&ctx->h_flags, 16 * sizeof(int)));
    GB_CUDA(cudaMallocHost(&ctx->h_status, sizeof(gb_ctx::SolveStatus)));
    GB_CUDA(cudaEventCreate(&ctx->evh0));
    GB_CUDA(cudaEventCreate(&ctx->evh1));
  } catch (const gb::Error& e) {
    fprintf(stderr, "gb_ctx_create: %s\n", e.msg.c_str());
    int code = e.code;
    gb_ctx_destroy(ctx);
    return code;
  }
  *out = ctx;
  return GB_OK;
}

int
gb_ctx_destroy(gb_ctx* ctx)
{
  if (!ctx)
    return GB_EINVAL;
  cudaSetDevice(ctx->device);
  if (ctx->stream)
    cudaStreamSynchronize(ctx->stream);
  if (ctx->h_flags)
    cudaFreeHost(ctx->h_flags);
  if (ctx->h_status)
    cudaFreeHost(ctx->h_status);
  if (ctx->evh0)
    cudaEventDestroy(ctx->evh0);
  if (ctx->evh1)
    cudaEventDestroy(ctx->evh1);
  if (ctx->ev0)
    cudaEventDestroy(ctx->ev0);
  if (ctx->ev1)
    cudaEventDestroy(ctx->ev1);
  cudaStream_t st = ctx->stream;
  delete ctx; // releases device arrays
  if (st)
    cudaStreamDestroy(st);
  return GB_OK;
}

const char*
gb_last_error_string(const gb_ctx* ctx)
{
  return ctx ? ctx->err.c_str() : "null context";
}

int
gb_ctx_synchronize(gb_ctx* ctx)
{
  GB_API_BEGIN
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  GB_API_END
}

int
gb_set_params(gb_ctx* ctx, const gb_params* p)
{
  GB_API_BEGIN
  ctx->version++;
  GB_REQUIRE(p, GB_EINVAL, "null params");
  GB_REQUIRE(p->iterpre >= 0 && p->iterpost >= 0 && p->iterexact >= 0, GB_EINVAL,
             "negative sweep count");
  GB_REQUIRE(p->mgtype == 'V' || p->mgtype == 'W' || p->mgtype == 'F', GB_EINVAL,
             "mgtype must be V, W or F");
  GB_REQUIRE(p->gmressize >= 2 && p->gmressize <= kMaxV, GB_EINVAL,
             "gmressize out of range [2, 128]");
  GB_REQUIRE(p->maxiter >= 1, GB_EINVAL, "maxiter must be >= 1");
  GB_REQUIRE(p->ndirect >= 0, GB_EINVAL, "ndirect must be >= 0");
  ctx->params = *p;
  ctx->work_ready = false; // recorded coarse programs depend on the keys
  GB_API_END
}

int
gb_get_params(const gb_ctx* ctx, gb_params* p)
{
  if (!ctx || !p)
    return GB_EINVAL;
  *p = ctx->params;
  return GB_OK;
}

int
gb_set_nlevels(gb_ctx* ctx, int nlevels)
{
  GB_API_BEGIN
  ctx->version++;
  GB_REQUIRE(nlevels >= 1 && nlevels <= 32, GB_EINVAL, "nlevels out of range [1, 32]");
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->nlevels = nlevels;
  ctx->L.clear();
  ctx->L.resize(nlevels);
  ctx->T.clear();
  ctx->T.resize(nlevels > 1 ? nlevels - 1 : 0);
  ctx->work_ready = false;
  for (auto& kv : ctx->vecs)
    kv.second.clear();
  GB_API_END
}

int
gb_level_set_matrix(gb_ctx* ctx, int lvl, int64_t n, int B, const int64_t* rowptr,
                    const int64_t* col, const int64_t* diag, const double* val)
{
  GB_API_BEGIN
  ctx->version++;
  Level& L = level(*ctx, lvl);
  GB_REQUIRE(B >= 1 && B <= 4, GB_EINVAL, "block size must be 1..4");
  GB_REQUIRE(B == 1 || !ctx->transposed, GB_EINVAL,
             "the transposed operator is available for block size 1 only");
  GB_REQUIRE(n >= 1 && n * B < (int64_t(1) << 29), GB_EINVAL, "n out of range");
  GB_REQUIRE(rowptr && col && diag && val, GB_EINVAL, "null array");
  GB_REQUIRE(rowptr[0] == 0, GB_EINVAL, "rowptr[0] != 0");
  for (int64_t i = 0; i < n; ++i) {
    GB_REQUIRE(rowptr[i + 1] >= rowptr[i], GB_EINVAL, "rowptr not monotone");
    GB_REQUIRE(diag[i] >= rowptr[i] && diag[i] < rowptr[i + 1] && col[diag[i]] == i,
               GB_EINVAL, "diag does not point at the diagonal block");
  }
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  const int64_t nnzb = rowptr[n];
  L.n = n;
  L.B = B;
  L.h_rowptr.assign(rowptr, rowptr + n + 1);
  L.h_col.assign(col, col + nnzb);
  L.h_diag.assign(diag, diag + n);
  L.h_val.assign(val, val + nnzb * B * B);
  build_sell(L.A, n, rowptr, col, val, ctx->stream, B, ctx->row_order);
  build_rows(*ctx, L.A, rowptr);
  L.has_AT = false;
  L.vk_ready = false;
  L.vk_struct = false;
  L.ilu_ready = false;
  L.ilu_struct = false;
  L.h_val_stale = false;
  L.mesh_ncells = 0; // the mesh maps point into the old pattern
  L.mesh_n = -1;
  if (ctx->transposed)
    ensure_AT(*ctx, L);
  // block-diagonal inverse on the device (get_inverse_diagonal / K1)
  std::vector<double> dblk(n * B * B);
  for (int64_t i = 0; i < n; ++i)
    for (int q = 0; q < B * B; ++q)
      dblk[i * B * B + q] = val[diag[i] * B * B + q];
  DeviceArray<double> dd;
  GB_CUDA(dd.alloc(dblk.size()));
  GB_CUDA(cudaMemcpyAsync(dd.p, dblk.data(), dblk.size() * sizeof(double),
                          cudaMemcpyHostToDevice, ctx->stream));
  GB_CUDA(L.dinv64.alloc(n * B * B));
  GB_CUDA(L.dinv32.alloc(n * B * B));
  switch (B) {
    case 1:
      launch(*ctx, k_blockdiag_inverse<1>, blocks_for(n, 128), 128, (int)n,
             (const double*)dd.p, L.dinv64.p, L.dinv32.p);
      break;
    case 2:
      launch(*ctx, k_blockdiag_inverse<2>, blocks_for(n, 128), 128, (int)n,
             (const double*)dd.p, L.dinv64.p, L.dinv32.p);
      break;
    case 3:
      launch(*ctx, k_blockdiag_inverse<3>, blocks_for(n, 128), 128, (int)n,
             (const double*)dd.p, L.dinv64.p, L.dinv32.p);
      break;
    default:
      launch(*ctx, k_blockdiag_inverse<4>, blocks_for(n, 128), 128, (int)n,
             (const double*)dd.p, L.dinv64.p, L.dinv32.p);
  }
  if (L.dirmask.n != static_cast<size_t>(n * B)) {
    GB_CUDA(L.dirmask.alloc(n * B));
    GB_CUDA(cudaMemsetAsync(L.dirmask.p, 0, n * B, ctx->stream));
    L.dirlist.release();
    L.ndir = 0;
  }
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  L.has_matrix = true;
  ctx->work_ready = false;
  GB_API_END
}

int
gb_level_set_dirichlet(gb_ctx* ctx, int lvl, int64_t nnodes, const int64_t* nodes,
                       int comp_mask)
{
  if (nnodes < 0)
    return gb_level_set_dirichlet_masks(ctx, lvl, nnodes, nodes, nullptr);
  std::vector<int> masks(static_cast<size_t>(nnodes), comp_mask);
  return gb_level_set_dirichlet_masks(ctx, lvl, nnodes, nodes, masks.data());
}

int
gb_level_set_dirichlet_masks(gb_ctx* ctx, int lvl, int64_t nnodes, const int64_t* nodes,
                             const int* comp_masks)
{
  GB_API_BEGIN
  ctx->version++;
  Level& L = level_with_matrix(*ctx, lvl);
  GB_REQUIRE(nnodes >= 0 && (nnodes == 0 || (nodes && comp_masks)), GB_EINVAL,
             "bad node list");
  std::vector<uint8_t> mask(L.ndof(), 0);
  std::vector<int> dofs;
  for (int64_t k = 0; k < nnodes; ++k) {
    GB_REQUIRE(nodes[k] >= 0 && nodes[k] < L.n, GB_EINVAL, "Dirichlet node out of range");
    const int comp_mask = comp_masks[k];
    for (int c = 0; c < L.B; ++c)
      if (comp_mask & (1 << c)) {
        int64_t d = nodes[k] * L.B + c;
        if (!mask[d])
          dofs.push_back(static_cast<int>(d));
        mask[d] = 1;
      }
  }
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  GB_CUDA(L.dirmask.alloc(mask.size()));
  GB_CUDA(h2d(ctx->stream, L.dirmask.p, mask.data(), mask.size()));
  GB_CUDA(L.dirlist.alloc(std::max<size_t>(dofs.size(), 1)));
  if (!dofs.empty())
    GB_CUDA(h2d(ctx->stream, L.dirlist.p, dofs.data(), dofs.size() * sizeof(int)));
  L.ndir = static_cast<int>(dofs.size());
  ctx->work_ready = false; // the prolongation mask of hanging levels includes it
  GB_API_END
}

int
gb_level_set_transfer(gb_ctx* ctx, int lvl, int64_t ncoarse, const int64_t* c2f,
                      int64_t nz, const int64_t* zweier, int64_t nv,
                      const int64_t* vierer, int64_t na, const int64_t* achter)
{
  GB_API_BEGIN
  ctx->version++;
  GB_REQUIRE(lvl >= 0 && lvl + 1 < ctx->nlevels, GB_EINVAL, "transfer level out of range");
  Level& Lc = level_with_matrix(*ctx, lvl);
  Level& Lf = level_with_matrix(*ctx, lvl + 1);
  GB_REQUIRE(ncoarse == Lc.n, GB_EINVAL, "c2f size differs from the coarse level size");
  GB_REQUIRE(Lc.B == Lf.B, GB_EINVAL, "levels of different block size");
  const int64_t nf = Lf.n;
  // (fine, coarse, weight code) pairs as MgInterpolatorMatrix::BasicInit forms them
  std::vector<int> wcode(nf, -1);
  std::vector<std::pair<int64_t, int64_t>> pairs;
  pairs.reserve(ncoarse + 2 * nz + 4 * nv + 8 * na);
  auto add = [&](int64_t f, int64_t cc, int code) {
    GB_REQUIRE(f >= 0 && f < nf, GB_EINVAL, "fine index out of range");
    GB_REQUIRE(cc >= 0 && cc < ncoarse, GB_EINVAL, "coarse index out of range");
    pairs.emplace_back(f, cc);
    wcode[f] = code;
  };
  for (int64_t i = 0; i < ncoarse; ++i)
    add(c2f[i], i, 0);
  for (int64_t i = 0; i < nz; ++i)
    for (int q = 0; q < 2; ++q)
      add(zweier[3 * i], zweier[3 * i + 1 + q], 1);
  for (int64_t i = 0; i < nv; ++i)
    for (int q = 0; q < 4; ++q)
      add(vierer[5 * i], vierer[5 * i + 1 + q], 2);
  for (int64_t i = 0; i < na; ++i)
    for (int q = 0; q < 8; ++q)
      add(achter[9 * i], achter[9 * i + 1 + q], 3);
  // fine rows (prolongation) and coarse rows (restriction), columns ascending
  std::vector<std::vector<int64_t>> prow(nf), rrow(ncoarse);
  for (auto& pr : pairs) {
    prow[pr.first].push_back(pr.second);
    rrow[pr.second].push_back(pr.first);
  }
  // SELL-32 layout of both tables (see transfer_row), columns ascending
  auto sell = [&](std::vector<std::vector<int64_t>>& rows, bool fine_rows,
                  std::vector<int>& tsp, std::vector<uint32_t>& tent) {
    const int64_t nr = static_cast<int64_t>(rows.size());
    const int64_t ns = (nr + kSlice - 1) / kSlice;
    tsp.assign(ns + 1, 0);
    for (auto& r : rows)
      std::sort(r.begin(), r.end());
    for (int64_t sl = 0; sl < ns; ++sl) {
      size_t w = 0;
      for (int64_t q = sl * kSlice; q < std::min(nr, (sl + 1) * kSlice); ++q)
        w = std::max(w, rows[q].size());
      tsp[sl + 1] = tsp[sl] + static_cast<int>(w) * kSlice;
    }
    tent.assign(tsp[ns], kPadEntry);
    for (int64_t q = 0; q < nr; ++q)
      for (size_t j = 0; j < rows[q].size(); ++j) {
        const int64_t other = rows[q][j];
        const int code = fine_rows ? wcode[q] : wcode[other];
        tent[tsp[q / kSlice] + j * kSlice + (q % kSlice)] =
          static_cast<uint32_t>(other) | (uint32_t(code) << kWShift);
      }
  };
  std::vector<int> pptr, rptr;
  std::vector<uint32_t> pent, rent;
  sell(prow, true, pptr, pent);
  sell(rrow, false, rptr, rent);
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  Transfer& T = ctx->T[lvl];
  T.nc = static_cast<int>(ncoarse);
  T.nf = static_cast<int>(nf);
  T.rmaxw = 0;
  for (size_t sl = 0; sl + 1 < rptr.size(); ++sl)
    T.rmaxw = std::max(T.rmaxw, (rptr[sl + 1] - rptr[sl]) / kSlice);
  T.nent = static_cast<int64_t>(pairs.size());
  GB_CUDA(T.pptr.alloc(pptr.size()));
  GB_CUDA(T.rptr.alloc(rptr.size()));
  GB_CUDA(T.pent.alloc(std::max<size_t>(pent.size(), 1)));
  GB_CUDA(T.rent.alloc(std::max<size_t>(rent.size(), 1)));
  GB_CUDA(h2d(ctx->stream, T.pptr.p, pptr.data(), pptr.size() * sizeof(int)));
  GB_CUDA(h2d(ctx->stream, T.rptr.p, rptr.data(), rptr.size() * sizeof(int)));
  if (!pent.empty())
    GB_CUDA(h2d(ctx->stream, T.pent.p, pent.data(), pent.size() * sizeof(uint32_t)));
  if (!rent.empty())
    GB_CUDA(h2d(ctx->stream, T.rent.p, rent.data(), rent.size() * sizeof(uint32_t)));
  T.set = true;
  ctx->work_ready = false;
  GB_API_END
}

int
gb_level_size(const gb_ctx* cctx, int lvl, int64_t* n, int* B, int64_t* nnzb)
{
  if (!cctx || lvl < 0 || lvl >= cctx->nlevels)
    return GB_EINVAL;
  const Level& L = cctx->L[lvl];
  if (n)
    *n = L.n;
  if (B)
    *B = L.B;
  if (nnzb)
    *nnzb = L.has_matrix ? L.A.nnz : 0;
  return GB_OK;
}

int
gb_vec_create(gb_ctx* ctx, int* id)
{
  GB_API_BEGIN
  GB_REQUIRE(id, GB_EINVAL, "null id");
  *id = ctx->next_id++;
  ctx->vecs[*id] = std::vector<DeviceArray<double>>();
  GB_API_END
}

int
gb_vec_free(gb_ctx* ctx, int id)
{
  GB_API_BEGIN
  auto it = ctx->vecs.find(id);
  GB_REQUIRE(it != ctx->vecs.end(), GB_EINVAL, "unknown vector id");
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->vecs.erase(it);
  GB_API_END
}

int
gb_vec_upload(gb_ctx* ctx, int lvl, int id, const double* host, int64_t len)
{
  GB_API_BEGIN
  double* d = vec(*ctx, lvl, id);
  GB_REQUIRE(host && len == ctx->L[lvl].ndof(), GB_EINVAL, "length differs from level size");
  GB_CUDA(cudaMemcpyAsync(d, host, len * sizeof(double), cudaMemcpyHostToDevice,
                          ctx->stream));
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  GB_API_END
}

int
gb_vec_download(gb_ctx* ctx, int lvl, int id, double* host, int64_t len)
{
  GB_API_BEGIN
  double* d = vec(*ctx, lvl, id);
  GB_REQUIRE(host && len == ctx->L[lvl].ndof(), GB_EINVAL, "length differs from level size");
  GB_CUDA(cudaMemcpyAsync(host, d, len * sizeof(double), cudaMemcpyDeviceToHost,
                          ctx->stream));
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  GB_API_END
}

int
gb_vec_zero(gb_ctx* ctx, int lvl, int id)
{
  GB_API_BEGIN
  double* d = vec(*ctx, lvl, id);
  GB_CUDA(cudaMemsetAsync(d, 0, ctx->L[lvl].ndof() * sizeof(double), ctx->stream));
  GB_API_END
}

int
gb_vec_equ(gb_ctx* ctx, int lvl, int dst, double s, int src)
{
  GB_API_BEGIN
  double* y = vec(*ctx, lvl, dst);
  double* x = vec(*ctx, lvl, src);
  int64_t n = ctx->L[lvl].ndof();
  launch(*ctx, k_equ<double, double>, stream_blocks(n), 256, n, y, s, (const double*)x);
  GB_API_END
}

int
gb_vec_add(gb_ctx* ctx, int lvl, int dst, double s, int src)
{
  GB_API_BEGIN
  double* y = vec(*ctx, lvl, dst);
  double* x = vec(*ctx, lvl, src);
  int64_t n = ctx->L[lvl].ndof();
  launch(*ctx, k_add, stream_blocks(n), 256, n, y, s, (const double*)x);
  GB_API_END
}

int
gb_vec_dot(gb_ctx* ctx, int lvl, int a, int b, double* out)
{
  GB_API_BEGIN
  GB_REQUIRE(out, GB_EINVAL, "null output");
  double* x = vec(*ctx, lvl, a);
  double* y = vec(*ctx, lvl, b);
  dot_dev(*ctx, ctx->L[lvl].ndof(), x, y, RedOut{ ctx->scal.p, nullptr, nullptr, 0 });
  *out = read_scalar(*ctx, ctx->scal.p);
  GB_API_END
}

int
gb_vec_norm(gb_ctx* ctx, int lvl, int id, double* out)
{
  GB_API_BEGIN
  GB_REQUIRE(out, GB_EINVAL, "null output");
  double* x = vec(*ctx, lvl, id);
  dot_dev(*ctx, ctx->L[lvl].ndof(), x, x, RedOut{ ctx->scal.p, nullptr, nullptr, 1 });
  *out = read_scalar(*ctx, ctx->scal.p);
  GB_API_END
}

int
gb_vmult(gb_ctx* ctx, int lvl, int y, int x, double d)
{
  GB_API_BEGIN
  GB_REQUIRE(y != x, GB_EINVAL, "y and x must differ");
  Level& L = level_with_matrix(*ctx, lvl);
  spmv<kAddAx, double, double, double>(*ctx, L, opA(*ctx, L), (const double*)vec(*ctx, lvl, x),
                                       vec(*ctx, lvl, y), nullptr, nullptr, d);
  GB_API_END
}

int
gb_vmulteq(gb_ctx* ctx, int lvl, int y, int x, double d)
{
  GB_API_BEGIN
  GB_REQUIRE(y != x, GB_EINVAL, "y and x must differ");
  Level& L = level_with_matrix(*ctx, lvl);
  spmv<kAx, double, double, double>(*ctx, L, opA(*ctx, L), (const double*)vec(*ctx, lvl, x),
                                    vec(*ctx, lvl, y), nullptr, nullptr, d);
  GB_API_END
}

int
gb_vmult_transpose(gb_ctx* ctx, int lvl, int y, int x, double d)
{
  GB_API_BEGIN
  GB_REQUIRE(y != x, GB_EINVAL, "y and x must differ");
  Level& L = level_with_matrix(*ctx, lvl);
  ensure_AT(*ctx, L);
  // the transpose of the current level operator
  spmv<kAddAx, double, double, double>(*ctx, L, ctx->transposed ? L.A : L.AT,
                                       (const double*)vec(*ctx, lvl, x),
                                       vec(*ctx, lvl, y), nullptr, nullptr, d);
  GB_API_END
}

int
gb_matrix_residual(gb_ctx* ctx, int lvl, int y, int x, int b)
{
  GB_API_BEGIN
  GB_REQUIRE(y != x && y != b, GB_EINVAL, "y must differ from x and b");
  Level& L = level_with_matrix(*ctx, lvl);
  double* yd = vec(*ctx, lvl, y);
  spmv<kResid, double, double, double>(*ctx, L, opA(*ctx, L), (const double*)vec(*ctx, lvl, x),
                                       yd, (const double*)vec(*ctx, lvl, b), nullptr, 0.0);
  if (L.pf_mask) { // SubtractMeanAlgebraic
    Emit<double> E{ *ctx, nullptr };
    E.pf_sub(lvl, yd, false);
  }
  GB_API_END
}

int
gb_residualgmres(gb_ctx* ctx, int lvl, int y, int x, int b)
{
  GB_API_BEGIN
  GB_REQUIRE(y != x && y != b, GB_EINVAL, "y must differ from x and b");
  Level& L = level_with_matrix(*ctx, lvl);
  spmv<kResidDir, double, double, double>(*ctx, L, opA(*ctx, L),
                                          (const double*)vec(*ctx, lvl, x),
                                          vec(*ctx, lvl, y),
                                          (const double*)vec(*ctx, lvl, b), nullptr, 0.0);
  GB_API_END
}

// StdSolver::smooth with smoother 0 (jacobi) or 1 (Vanka), FP64.
static void
smooth_api(gb_ctx* ctx, int lvl, int niter, int x, int y, int h, int smoother)
{
  GB_REQUIRE(niter >= 0, GB_EINVAL, "niter < 0");
  GB_REQUIRE(x != y && x != h && y != h, GB_EINVAL, "x, y, h must differ");
  Level& L = level_with_matrix(*ctx, lvl);
  GB_REQUIRE(smoother >= 0 && smoother <= 2, GB_EINVAL, "smoother must be 0, 1 or 2");
  if (smoother == 1) {
    GB_REQUIRE(!ctx->transposed, GB_EINVAL, "Vanka with the transposed operator");
    ensure_vanka(*ctx, L);
  }
  if (smoother == 2) {
    GB_REQUIRE(!ctx->transposed, GB_EINVAL, "ILU with the transposed operator");
    ensure_ilu(*ctx, L);
  }
  double* xd = vec(*ctx, lvl, x);
  double* hd = vec(*ctx, lvl, h);
  const double* yd = vec(*ctx, lvl, y);
  double* u = xd;
  double* t = hd;
  bool zero = false;
  const int saved = ctx->params.smoother;
  ctx->params.smoother = smoother;
  struct Restore
  {
    gb_ctx* c;
    int v;
    ~Restore() { c->params.smoother = v; }
  } restore{ ctx, saved };
  Emit<double> E{ *ctx, nullptr };
  smooth<double>(E, lvl, niter, u, t, yd, zero);
  if (u != xd)
    GB_CUDA(cudaMemcpyAsync(xd, u, ctx->L[lvl].ndof() * sizeof(double),
                            cudaMemcpyDeviceToDevice, ctx->stream));
}

int
gb_smooth_jacobi(gb_ctx* ctx, int lvl, int niter, int x, int y, int h)
{
  GB_API_BEGIN
  smooth_api(ctx, lvl, niter, x, y, h, 0);
  GB_API_END
}

int
gb_smooth_vanka(gb_ctx* ctx, int lvl, int niter, int x, int y, int h)
{
  GB_API_BEGIN
  smooth_api(ctx, lvl, niter, x, y, h, 1);
  GB_API_END
}

int
gb_smooth(gb_ctx* ctx, int lvl, int niter, int x, int y, int h)
{
  GB_API_BEGIN
  smooth_api(ctx, lvl, niter, x, y, h, ctx->params.smoother);
  GB_API_END
}

int
gb_level_set_patches(gb_ctx* ctx, int lvl, int64_t npatch, int npp, const int64_t* patches)
{
  GB_API_BEGIN
  ctx->version++;
  Level& L = level_with_matrix(*ctx, lvl);
  GB_REQUIRE(npatch >= 1 && npp >= 1 && npp <= 27 && patches, GB_EINVAL,
             "bad patch list (npp must be 1..27)");
  GB_REQUIRE(npatch * npp < (int64_t(1) << 31) && npatch < (int64_t(1) << 26), GB_EINVAL,
             "too many patches");
  for (int64_t k = 0; k < npatch * npp; ++k)
    GB_REQUIRE(patches[k] >= 0 && patches[k] < L.n, GB_EINVAL, "patch node out of range");
  for (int64_t p = 0; p < npatch; ++p)
    for (int a = 0; a < npp; ++a)
      for (int b = a + 1; b < npp; ++b)
        GB_REQUIRE(patches[p * npp + a] != patches[p * npp + b], GB_EINVAL,
                   "a node appears twice in a patch");
  L.h_patches.assign(patches, patches + npatch * npp);
  L.npatch = static_cast<int>(npatch);
  L.npp = npp;
  L.vk_ready = false;
  L.vk_struct = false;
  ctx->work_ready = false;
  GB_API_END
}

int
gb_level_set_pfilter(gb_ctx* ctx, int lvl, int comp_mask, const double* weights,
                     double domain, int64_t nhanging)
{
  GB_API_BEGIN
  ctx->version++;
  Level& L = level_with_matrix(*ctx, lvl);
  GB_REQUIRE(comp_mask >= 0 && comp_mask < (1 << L.B), GB_EINVAL, "bad component mask");
  GB_REQUIRE(comp_mask == 0 || (weights && domain > 0.0), GB_EINVAL,
             "the filter needs weights and a positive domain size");
  GB_REQUIRE(nhanging >= 0 && nhanging < L.n, GB_EINVAL, "bad hanging-node count");
  if (comp_mask) {
    GB_CUDA(cudaStreamSynchronize(ctx->stream));
    GB_CUDA(L.pf_w.alloc(L.n));
    GB_CUDA(h2d(ctx->stream, L.pf_w.p, weights, L.n * sizeof(double)));
  }
  if (comp_mask)
    ensure_pf_scratch(*ctx, L.n);
  L.pf_mask = comp_mask;
  L.pf_domain = domain;
  L.nhanging = nhanging;
  ctx->work_ready = false;
  GB_API_END
}

int
gb_level_set_hn(gb_ctx* ctx, int lvl, int disc, int64_t nedge, const int64_t* edges,
                int64_t nface, const int64_t* faces)
{
  GB_API_BEGIN
  ctx->version++;
  Level& L = level_with_matrix(*ctx, lvl);
  GB_REQUIRE(disc >= 0 && disc <= 3, GB_EINVAL, "disc must be 0 (Q12d) .. 3 (Q23d)");
  GB_REQUIRE(nedge >= 0 && nface >= 0 && (nedge == 0 || edges) && (nface == 0 || faces),
             GB_EINVAL, "bad hanging-node lists");
  const bool q2 = disc >= 2, d3 = disc == 1 || disc == 3;
  GB_REQUIRE(d3 || nface == 0, GB_EINVAL, "face hanging nodes need a 3D discretisation");
  auto check = [&](int64_t v) {
    GB_REQUIRE(v >= 0 && v < L.n, GB_EINVAL, "hanging-node index out of range");
  };
  for (int64_t k = 0; k < nedge * 4; ++k)
    check(edges[k]);
  for (int64_t k = 0; k < nface * 10; ++k)
    check(faces[k]);
  // the phases' slots and weights, as the HNStructure classes use them
  struct Spec
  {
    std::vector<int64_t> node;
    std::vector<std::vector<int64_t>> par; // per hanging node, slot order
    std::vector<double> w;
    int gsize;
  };
  const double q2w[3] = { 0.375, 0.75, -0.125 };
  Spec se, sf;
  for (int64_t k = 0; k < nedge; ++k) {
    se.node.push_back(edges[4 * k]);
    std::vector<int64_t> pp;
    for (int j = 0; j < (q2 ? 3 : 2); ++j)
      pp.push_back(edges[4 * k + 1 + j]);
    se.par.push_back(pp);
  }
  if (q2)
    se.w = { q2w[0], q2w[1], q2w[2] }, se.gsize = 3;
  else
    se.w = { 0.5, 0.5 }, se.gsize = 2;
  for (int64_t k = 0; k < nface; ++k) {
    sf.node.push_back(faces[10 * k]);
    std::vector<int64_t> pp;
    if (q2)
      for (int j = 0; j < 9; ++j)
        pp.push_back(faces[10 * k + 1 + j]);
    else
      for (int j : { 0, 1, 3, 4 })
        pp.push_back(faces[10 * k + 1 + j]);
    sf.par.push_back(pp);
  }
  if (q2) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        sf.w.push_back(q2w[i] * q2w[j]);
    sf.gsize = 3;
  } else {
    sf.w = { 0.25, 0.25, 0.25, 0.25 };
    sf.gsize = 4;
  }
  std::vector<Spec*> order;
  if (disc == 3)
    order = { &sf, &se };
  else if (disc == 1)
    order = { &se, &sf };
  else
    order = { &se };
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  L.hn.clear();
  L.h_hnnodes.clear();
  // the assembly's condensation table; a mesh set before it is dropped
  L.h_hncond.clear();
  L.h_hnidx.assign(L.n, -1);
  L.mesh_ncells = 0;
  for (int ph = 0; ph < 2; ++ph) {
    const Spec& sp = ph == 0 ? se : sf;
    for (size_t k = 0; k < sp.node.size(); ++k) {
      Level::HnCond hc;
      hc.phase = ph;
      hc.np = static_cast<int>(sp.w.size());
      for (int j = 0; j < hc.np; ++j) {
        hc.par[j] = static_cast<int>(sp.par[k][j]);
        hc.w[j] = sp.w[j];
      }
      GB_REQUIRE(L.h_hnidx[sp.node[k]] < 0, GB_EINVAL, "a node hangs twice");
      L.h_hnidx[sp.node[k]] = static_cast<int>(L.h_hncond.size());
      L.h_hncond.push_back(hc);
    }
  }
  if (L.h_hncond.empty())
    L.h_hnidx.clear();
  std::vector<uint8_t> inphase(L.n, 0);
  for (Spec* sp : order) {
    const int nh = static_cast<int>(sp->node.size());
    if (nh == 0)
      continue;
    // ascending hanging nodes (std::map order) and no chains inside a phase
    std::fill(inphase.begin(), inphase.end(), 0);
    for (int k = 0; k < nh; ++k) {
      GB_REQUIRE(k == 0 || sp->node[k] > sp->node[k - 1], GB_EINVAL,
                 "hanging nodes must be listed in ascending order");
      inphase[sp->node[k]] = 1;
    }
    for (const auto& pp : sp->par)
      for (int64_t q : pp)
        GB_REQUIRE(!inphase[q], GB_EINVAL,
                   "a hanging node is a parent of another of the same kind");
    const int ns = static_cast<int>(sp->w.size());
    std::vector<int> node(nh), par(size_t(ns) * nh);
    for (int k = 0; k < nh; ++k) {
      node[k] = static_cast<int>(sp->node[k]);
      L.h_hnnodes.push_back(node[k]);
      for (int s2 = 0; s2 < ns; ++s2)
        par[size_t(s2) * nh + k] = static_cast<int>(sp->par[k][s2]);
    }
    // distribute: per parent, (hanging node, weight) in ascending hanging order
    std::map<int, std::vector<std::pair<int, double>>> byp;
    for (int k = 0; k < nh; ++k)
      for (int s2 = 0; s2 < ns; ++s2)
        byp[static_cast<int>(sp->par[k][s2])].push_back({ node[k], sp->w[s2] });
    std::vector<int> pnode, ptr(1, 0), hnode;
    std::vector<double> wt;
    for (auto& kv : byp) {
      pnode.push_back(kv.first);
      for (auto& e : kv.second) {
        hnode.push_back(e.first);
        wt.push_back(e.second);
      }
      ptr.push_back(static_cast<int>(hnode.size()));
    }
    Level::HnPhase ph;
    ph.nh = nh;
    ph.nslots = ns;
    ph.gsize = sp->gsize;
    ph.np = static_cast<int>(pnode.size());
    GB_CUDA(ph.node.alloc(nh));
    GB_CUDA(ph.par.alloc(par.size()));
    GB_CUDA(ph.w.alloc(ns));
    GB_CUDA(ph.pnode.alloc(pnode.size()));
    GB_CUDA(ph.ptr.alloc(ptr.size()));
    GB_CUDA(ph.hnode.alloc(hnode.size()));
    GB_CUDA(ph.wt.alloc(wt.size()));
    GB_CUDA(h2d(ctx->stream, ph.node.p, node.data(), nh * sizeof(int)));
    GB_CUDA(h2d(ctx->stream, ph.par.p, par.data(), par.size() * sizeof(int)));
    GB_CUDA(h2d(ctx->stream, ph.w.p, sp->w.data(), ns * sizeof(double)));
    GB_CUDA(h2d(ctx->stream, ph.pnode.p, pnode.data(), pnode.size() * sizeof(int)));
    GB_CUDA(h2d(ctx->stream, ph.ptr.p, ptr.data(), ptr.size() * sizeof(int)));
    GB_CUDA(h2d(ctx->stream, ph.hnode.p, hnode.data(), hnode.size() * sizeof(int)));
    GB_CUDA(h2d(ctx->stream, ph.wt.p, wt.data(), wt.size() * sizeof(double)));
    L.hn.push_back(std::move(ph));
  }
  if (!L.h_hnnodes.empty()) {
    GB_CUDA(L.hn_all.alloc(L.h_hnnodes.size()));
    GB_CUDA(h2d(ctx->stream, L.hn_all.p, L.h_hnnodes.data(), L.h_hnnodes.size() * sizeof(int)));
  }
  ctx->work_ready = false;
  GB_API_END
}

int
gb_hn_average(gb_ctx* ctx, int lvl, int id)
{
  GB_API_BEGIN
  level_with_matrix(*ctx, lvl);
  Emit<double> E{ *ctx, nullptr };
  E.hn_average(lvl, vec(*ctx, lvl, id));
  GB_API_END
}

int
gb_hn_distribute(gb_ctx* ctx, int lvl, int id)
{
  GB_API_BEGIN
  level_with_matrix(*ctx, lvl);
  Emit<double> E{ *ctx, nullptr };
  E.hn_distribute(lvl, vec(*ctx, lvl, id));
  GB_API_END
}

int
gb_hn_zero(gb_ctx* ctx, int lvl, int id)
{
  GB_API_BEGIN
  level_with_matrix(*ctx, lvl);
  Emit<double> E{ *ctx, nullptr };
  E.hn_zero(lvl, vec(*ctx, lvl, id));
  GB_API_END
}

int
gb_subtract_mean(gb_ctx* ctx, int lvl, int id)
{
  GB_API_BEGIN
  Level& L = level_with_matrix(*ctx, lvl);
  Emit<double> E{ *ctx, nullptr };
  if (L.pf_mask)
    E.pf_sub(lvl, vec(*ctx, lvl, id), true);
  GB_API_END
}

int
gb_subtract_mean_algebraic(gb_ctx* ctx, int lvl, int id)
{
  GB_API_BEGIN
  Level& L = level_with_matrix(*ctx, lvl);
  Emit<double> E{ *ctx, nullptr };
  if (L.pf_mask)
    E.pf_sub(lvl, vec(*ctx, lvl, id), false);
  GB_API_END
}

int
gb_dirichlet_zero(gb_ctx* ctx, int lvl, int id)
{
  GB_API_BEGIN
  Level& L = level_with_matrix(*ctx, lvl);
  launch(*ctx, k_dirichlet_zero<double>, blocks_for(L.ndir, 256), 256, L.ndir,
         (const int*)L.dirlist.p, vec(*ctx, lvl, id));
  GB_API_END
}

int
gb_level_get_inverse_diagonal(gb_ctx* ctx, int lvl, double* host, int64_t len)
{
  GB_API_BEGIN
  Level& L = level_with_matrix(*ctx, lvl);
  GB_REQUIRE(host && len == L.n * L.B * L.B, GB_EINVAL, "length must be n*B*B");
  GB_CUDA(cudaMemcpyAsync(host, L.dinv64.p, len * sizeof(double), cudaMemcpyDeviceToHost,
                          ctx->stream));
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  GB_API_END
}

int
gb_restrict_zero(gb_ctx* ctx, int lvl, int coarse_id, int fine_id)
{
  GB_API_BEGIN
  GB_REQUIRE(lvl >= 0 && lvl + 1 < ctx->nlevels && ctx->T[lvl].set, GB_ESTATE,
             "no transfer on this level");
  Transfer& T = ctx->T[lvl];
  const int B = ctx->L[lvl].B, nb = blocks_for(T.nc, 256);
  const int* tp = T.rptr.p;
  const uint32_t* te = T.rent.p;
  const double* f = vec(*ctx, lvl + 1, fine_id);
  double* cc = vec(*ctx, lvl, coarse_id);
  const uint8_t* nm = nullptr;
  switch (B) {
    case 1:
      if (T.rmaxw <= 32)
        launch(*ctx, k_restrict4<double>, blocks_for(int64_t(T.nc) * 4, 256), 256, T.nc, tp,
               te, f, cc, nm, (const double*)nullptr, (double*)nullptr, 0.0);
      else
        launch(*ctx, k_restrict<double>, nb, 256, T.nc, tp, te, f, cc, nm,
               (const double*)nullptr, (double*)nullptr, 0.0);
      break;
    case 2:
      launch(*ctx, k_restrict_b<double, 2>, nb, 256, T.nc, tp, te, f, cc, nm, -1,
             (const double*)nullptr);
      break;
    case 3:
      launch(*ctx, k_restrict_b<double, 3>, nb, 256, T.nc, tp, te, f, cc, nm, -1,
             (const double*)nullptr);
      break;
    default:
      launch(*ctx, k_restrict_b<double, 4>, nb, 256, T.nc, tp, te, f, cc, nm, -1,
             (const double*)nullptr);
  }
  GB_API_END
}

int
gb_prolongate_add(gb_ctx* ctx, int lvl, int fine_id, int coarse_id)
{
  GB_API_BEGIN
  GB_REQUIRE(lvl >= 0 && lvl + 1 < ctx->nlevels && ctx->T[lvl].set, GB_ESTATE,
             "no transfer on this level");
  Transfer& T = ctx->T[lvl];
  const int B = ctx->L[lvl].B, nb = blocks_for(T.nf, 256);
  const int* tp = T.pptr.p;
  const uint32_t* te = T.pent.p;
  const double* cc = vec(*ctx, lvl, coarse_id);
  double* f = vec(*ctx, lvl + 1, fine_id);
  const uint8_t* nm = nullptr;
  switch (B) {
    case 1:
      launch(*ctx, k_prolong<0, double>, nb, 256, T.nf, tp, te, cc, f, nm, 1.0);
      break;
    case 2:
      launch(*ctx, k_prolong_b<0, double, 2>, nb, 256, T.nf, tp, te, cc, f, nm, 1.0);
      break;
    case 3:
      launch(*ctx, k_prolong_b<0, double, 3>, nb, 256, T.nf, tp, te, cc, f, nm, 1.0);
      break;
    default:
      launch(*ctx, k_prolong_b<0, double, 4>, nb, 256, T.nf, tp, te, cc, f, nm, 1.0);
  }
  GB_API_END
}

int
gb_precondition(gb_ctx* ctx, int x, int y, int precision)
{
  GB_API_BEGIN
  GB_REQUIRE(x != y, GB_EINVAL, "x and y must differ");
  const int fl = ctx->nlevels - 1;
  GB_REQUIRE(fl >= 0, GB_ESTATE, "no levels");
  ensure_work(*ctx);
  double* xd = vec(*ctx, fl, x);
  const double* yd = vec(*ctx, fl, y);
  const int64_t n = ctx->L[fl].ndof();
  if (precision == GB_FP32) {
    float* x32 = ctx->w32.u[fl].p;
    float* y32 = ctx->w32.b[fl].p;
    launch(*ctx, k_convert<double, float>, stream_blocks(n), 256, n, y32, yd);
    launch(*ctx, k_convert<double, float>, stream_blocks(n), 256, n, x32,
           (const double*)xd);
    precondition_T<float>(*ctx, ctx->w32, x32, y32, false);
    launch(*ctx, k_convert<float, double>, stream_blocks(n), 256, n, xd,
           (const float*)x32);
  } else {
    GB_REQUIRE(precision == GB_FP64, GB_EINVAL, "precision must be GB_FP64 or GB_FP32");
    precondition_T<double>(*ctx, ctx->w64, xd, yd, false);
  }
  GB_API_END
}

int
gb_gmres(gb_ctx* ctx, int x, int b, gb_solve_info* info)
{
  GB_API_BEGIN
  GB_REQUIRE(x != b, GB_EINVAL, "x and b must differ");
  const int fl = ctx->nlevels - 1;
  GB_REQUIRE(fl >= 0, GB_ESTATE, "no levels");
  ensure_work(*ctx);
  return gmres_left(*ctx, vec(*ctx, fl, x), vec(*ctx, fl, b), info);
  GB_API_END
}

int
gb_fgmres(gb_ctx* ctx, int x, int b, int precision, gb_solve_info* info)
{
  GB_API_BEGIN
  GB_REQUIRE(x != b, GB_EINVAL, "x and b must differ");
  GB_REQUIRE(precision == GB_FP64 || precision == GB_FP32, GB_EINVAL, "bad precision");
  const int fl = ctx->nlevels - 1;
  GB_REQUIRE(fl >= 0, GB_ESTATE, "no levels");
  ensure_work(*ctx);
  if (ctx->params.gmressize <= kCgsMaxJ)
    return fgmres_graph(*ctx, vec(*ctx, fl, x), vec(*ctx, fl, b), precision, info);
  return gmres_flexible(*ctx, vec(*ctx, fl, x), vec(*ctx, fl, b), precision, info);
  GB_API_END
}

int
gb_solve_host(gb_ctx* ctx, int method, const double* b, double* x, int64_t len,
              gb_solve_info* info)
{
  GB_API_BEGIN
  const int fl = ctx->nlevels - 1;
  GB_REQUIRE(fl >= 0, GB_ESTATE, "no levels");
  GB_REQUIRE(b && x && len == ctx->L[fl].ndof(), GB_EINVAL, "length differs from level size");
  GB_REQUIRE(method >= 0 && method <= 2, GB_EINVAL, "method must be 0, 1 or 2");
  ensure_work(*ctx);
  const int prec = method == 1 ? GB_FP64 : GB_FP32;
  const bool graph = method != 0 && ctx->use_graph && ctx->params.gmressize <= kCgsMaxJ;
  double* bd;
  double* xd;
  if (graph) {
    // the graph's own right-hand side and solution buffers: b goes straight
    // in, x straight out, with no device-side staging copies
    if (prec == GB_FP32)
      fg_buffers<float>(*ctx, prec);
    else
      fg_buffers<double>(*ctx, prec);
    bd = ctx->bg.p;
    xd = ctx->xg.p;
  } else {
    // resident work vectors of the host-buffer call (created on first use)
    static const int kB = -1, kX = -2;
    ctx->vecs[kB];
    ctx->vecs[kX];
    bd = vec(*ctx, fl, kB);
    xd = vec(*ctx, fl, kX);
  }
  GB_CUDA(cudaEventRecord(ctx->evh0, ctx->stream));
  GB_CUDA(cudaMemcpyAsync(bd, b, len * sizeof(double), cudaMemcpyHostToDevice,
                          ctx->stream));
  int rc;
  if (graph) {
    rc = fgmres_graph(*ctx, xd, bd, prec, info, false, false, x, ctx->evh1);
  } else {
    rc = method == 0 ? gmres_left(*ctx, xd, bd, info)
                     : gmres_flexible(*ctx, xd, bd, prec, info);
    GB_CUDA(cudaMemcpyAsync(x, xd, len * sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->stream));
    GB_CUDA(cudaEventRecord(ctx->evh1, ctx->stream));
  }
  GB_CUDA(cudaEventSynchronize(ctx->evh1));
  float ms = 0;
  GB_CUDA(cudaEventElapsedTime(&ms, ctx->evh0, ctx->evh1));
  if (info)
    info->device_ms = ms;
  return rc;
  GB_API_END
}

int
gb_set_operator(gb_ctx* ctx, int transposed)
{
  GB_API_BEGIN
  GB_REQUIRE(transposed == 0 || transposed == 1, GB_EINVAL, "transposed must be 0 or 1");
  if (transposed)
    for (auto& L : ctx->L)
      if (L.has_matrix) {
        GB_REQUIRE(L.B == 1, GB_EINVAL,
                   "the transposed solver operators need block size 1");
        ensure_AT(*ctx, L);
      }
  ctx->transposed = transposed;
  GB_API_END
}

int
gb_get_operator(const gb_ctx* ctx, int* transposed)
{
  if (!ctx || !transposed)
    return GB_EINVAL;
  *transposed = ctx->transposed;
  return GB_OK;
}

int
gb_adjoint_gmres(gb_ctx* ctx, int x, int b, gb_solve_info* info)
{
  GB_API_BEGIN
  return with_transposed(ctx, [&] { return gb_gmres(ctx, x, b, info); });
  GB_API_END
}

int
gb_adjoint_fgmres(gb_ctx* ctx, int x, int b, int precision, gb_solve_info* info)
{
  GB_API_BEGIN
  return with_transposed(ctx, [&] { return gb_fgmres(ctx, x, b, precision, info); });
  GB_API_END
}

int
gb_set_timing(gb_ctx* ctx, int on)
{
  GB_API_BEGIN
  kt_flush(*ctx);
  ctx->ktime = on != 0;
  ctx->kt_acc.clear();
  GB_API_END
}

int
gb_get_kernel_times(gb_ctx* ctx, char* buf, int64_t len)
{
  GB_API_BEGIN
  GB_REQUIRE(buf && len > 0, GB_EINVAL, "null buffer");
  kt_flush(*ctx);
  std::string js = "{";
  bool first = true;
  for (auto& kv : ctx->kt_acc) {
    char item[512];
    snprintf(item, sizeof(item), "%s\"%s\": [%lld, %.6f]", first ? "" : ", ",
             kv.first.c_str(), (long long)kv.second.first, kv.second.second);
    js += item;
    first = false;
  }
  js += "}";
  GB_REQUIRE(int64_t(js.size()) < len, GB_EINVAL, "buffer too small");
  memcpy(buf, js.c_str(), js.size() + 1);
  GB_API_END
}

int
gb_get_kernel_count(const gb_ctx* ctx, int64_t* launches)
{
  if (!ctx || !launches)
    return GB_EINVAL;
  *launches = ctx->launches;
  return GB_OK;
}

int
gb_bench_spmv(gb_ctx* ctx, int lvl, int precision, int reps, int flush_l2,
              double* ms_per_launch, double* bytes_per_launch)
{
  GB_API_BEGIN
  GB_REQUIRE(reps >= 1, GB_EINVAL, "reps < 1");
  Level& L = level_with_matrix(*ctx, lvl);
  ensure_work(*ctx);
  const size_t flush_bytes = size_t(256) << 20; // > 126 MB L2
  if (flush_l2 && ctx->flush.n < flush_bytes)
    GB_CUDA(ctx->flush.alloc(flush_bytes));
  cudaEvent_t a, bq;
  GB_CUDA(cudaEventCreate(&a));
  GB_CUDA(cudaEventCreate(&bq));
  double total = 0;
  if (flush_l2 == 2) // first touch, so that the read flush finds mapped pages
    GB_CUDA(cudaMemsetAsync(ctx->flush.p, 0, flush_bytes, ctx->stream));
  for (int r = 0; r < reps; ++r) {
    if (flush_l2 == 1)
      GB_CUDA(cudaMemsetAsync(ctx->flush.p, r & 0xff, flush_bytes, ctx->stream));
    else if (flush_l2 == 2)
      k_read_flush<<<4 * 148, 512, 0, ctx->stream>>>(
        reinterpret_cast<const uint4*>(ctx->flush.p), int64_t(flush_bytes / 16), nullptr);
    GB_CUDA(cudaEventRecord(a, ctx->stream));
    if (precision == GB_FP32)
      spmv<kAx, float, float, float>(*ctx, L, opA(*ctx, L), (const float*)ctx->w32.b[lvl].p,
                                     ctx->w32.u[lvl].p, nullptr, nullptr, 1.0);
    else
      spmv<kAx, double, double, double>(*ctx, L, opA(*ctx, L),
                                        (const double*)ctx->w64.b[lvl].p,
                                        ctx->w64.u[lvl].p, nullptr, nullptr, 1.0);
    GB_CUDA(cudaEventRecord(bq, ctx->stream));
    GB_CUDA(cudaEventSynchronize(bq));
    float ms = 0;
    GB_CUDA(cudaEventElapsedTime(&ms, a, bq));
    total += ms;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(bq);
  const double sv = precision == GB_FP32 ? 4.0 : 8.0;
  const double nnz = static_cast<double>(L.A.nnz), n = static_cast<double>(L.n);
  if (ms_per_launch)
    *ms_per_launch = total / reps;
  if (bytes_per_launch) // SpMV algorithmic bytes: values + indices + rowptr + x + y
    *bytes_per_launch = nnz * sv + 4.0 * nnz + 4.0 * (n + 1) + 2.0 * n * sv;
  GB_API_END
}

int
gb_bench_sweep(gb_ctx* ctx, int lvl, int precision, int reps, int flush_l2,
               double* ms_per_launch, double* bytes_per_launch)
{
  GB_API_BEGIN
  GB_REQUIRE(reps >= 1, GB_EINVAL, "reps < 1");
  Level& L = level_with_matrix(*ctx, lvl);
  const bool vk = ctx->params.smoother == 1 && L.npatch > 0;
  GB_REQUIRE(vk || L.B == 1, GB_EINVAL,
             "a sweep of the fused Jacobi kernel (B = 1) or of the Vanka smoother");
  ensure_work(*ctx);
  if (vk)
    ensure_vanka(*ctx, L);
  const int64_t n = L.ndof();
  const size_t flush_bytes = size_t(256) << 20; // > 126 MB L2
  if (flush_l2 && ctx->flush.n < flush_bytes)
    GB_CUDA(ctx->flush.alloc(flush_bytes));
  // three vectors of the level (u, b, out) in the sweep's precision
  DeviceArray<double> buf;
  GB_CUDA(buf.alloc(size_t(3) * n));
  GB_CUDA(cudaMemsetAsync(buf.p, 0, size_t(3) * n * sizeof(double), ctx->stream));
  cudaEvent_t a, bq;
  GB_CUDA(cudaEventCreate(&a));
  GB_CUDA(cudaEventCreate(&bq));
  double total = 0;
  if (flush_l2 == 2)
    GB_CUDA(cudaMemsetAsync(ctx->flush.p, 0, flush_bytes, ctx->stream));
  for (int r = 0; r < reps; ++r) {
    if (flush_l2 == 1)
      GB_CUDA(cudaMemsetAsync(ctx->flush.p, r & 0xff, flush_bytes, ctx->stream));
    else if (flush_l2 == 2)
      k_read_flush<<<4 * 148, 512, 0, ctx->stream>>>(
        reinterpret_cast<const uint4*>(ctx->flush.p), int64_t(flush_bytes / 16), nullptr);
    GB_CUDA(cudaEventRecord(a, ctx->stream));
    if (vk && precision == GB_FP32) {
      float* f = reinterpret_cast<float*>(buf.p);
      Emit<float>{ *ctx }.vanka(lvl, f + n, f, false);
    } else if (vk) {
      Emit<double>{ *ctx }.vanka(lvl, buf.p + n, buf.p, false);
    } else if (precision == GB_FP32) {
      float* f = reinterpret_cast<float*>(buf.p);
      spmv<kJacobi, float, float, float>(*ctx, L, opA(*ctx, L), (const float*)f, f + 2 * n,
                                         (const float*)(f + n), L.dinv32.p, ctx->params.omega);
    } else {
      double* f = buf.p;
      spmv<kJacobi, double, double, double>(*ctx, L, opA(*ctx, L), (const double*)f,
                                            f + 2 * n, (const double*)(f + n), L.dinv64.p,
                                            ctx->params.omega);
    }
    GB_CUDA(cudaEventRecord(bq, ctx->stream));
    GB_CUDA(cudaEventSynchronize(bq));
    float ms = 0;
    GB_CUDA(cudaEventElapsedTime(&ms, a, bq));
    total += ms;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(bq);
  const double sv = precision == GB_FP32 ? 4.0 : 8.0;
  const double nnz = static_cast<double>(L.A.nnz), nd = static_cast<double>(n);
  if (ms_per_launch)
    *ms_per_launch = total / reps;
  if (bytes_per_launch && vk) {
    // patch solves: inverses, patch lists, gathered residual, patch solutions;
    // averaging gather: patch solutions, node -> (patch, slot) map, u read and
    // written
    const double np = L.npatch, M = L.vk_M, npp = L.npp;
    *bytes_per_launch = np * M * M * sv + np * npp * 4.0 + 2.0 * np * M * sv +
                        np * M * sv + np * npp * 4.0 + 4.0 * (L.n + 1) + 2.0 * nd * sv;
  } else if (bytes_per_launch) // SpMV bytes + b + D^-1 + the new iterate
    *bytes_per_launch = nnz * sv + 4.0 * nnz + 4.0 * (nd + 1) + 4.0 * nd * sv;
  GB_API_END
}

int
gb_level_get_vanka_inverse(gb_ctx* ctx, int lvl, double* host, int64_t len)
{
  GB_API_BEGIN
  Level& L = level_with_matrix(*ctx, lvl);
  GB_REQUIRE(host, GB_EINVAL, "null output");
  ensure_vanka(*ctx, L);
  const int64_t m = int64_t(L.npatch) * L.vk_M * L.vk_M;
  GB_REQUIRE(len == m, GB_EINVAL, "length differs from npatch * M * M");
  GB_CUDA(cudaMemcpyAsync(host, L.vk_inv64.p, m * sizeof(double), cudaMemcpyDeviceToHost,
                          ctx->stream));
  GB_CUDA(cudaStreamSynchronize(ctx->stream));
  GB_API_END
}

int
gb_set_wait_limit(gb_ctx* ctx, uint64_t wait_ns, int phantoms)
{
  GB_API_BEGIN
  GB_REQUIRE(wait_ns > 0 && phantoms >= 0, GB_EINVAL, "bad wait limit");
  ctx->version++; // captured solver graphs hold the old values
  ctx->wait_ns = wait_ns;
  ctx->barrier_phantoms = static_cast<unsigned>(phantoms);
  GB_API_END
}

int
gb_debug_fail_alloc(int64_t nth)
{
  if (nth < 0)
    return GB_EINVAL;
  g_fail_alloc_countdown.store(nth);
  return GB_OK;
}

int
gb_kernel_arch(int* binary_version, int* ptx_version)
{
  if (!binary_version || !ptx_version)
    return GB_EINVAL;
  cudaFuncAttributes a{};
  if (cudaFuncGetAttributes(&a, gb::k_dot<double, double>) != cudaSuccess)
    return GB_ECUDA;
  *binary_version = a.binaryVersion;
  *ptx_version = a.ptxVersion;
  return GB_OK;
}

} // extern "C"
