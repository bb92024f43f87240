// The GMRES drivers: the reference-semantics left-preconditioned GMRES and
// the flexible GMRES with refinement, host-driven or as one CUDA graph.
#include "gb_cycle.cuh"

namespace gb {

// ------------------------------------------------------------------ GMRES

void
ensure_gmres(Context& c, int vmax, bool flexible, int prec)
{
  GB_REQUIRE(vmax >= 2 && vmax <= kMaxV, GB_EINVAL, "gmressize out of range [2, 128]");
  const size_t n = c.L[c.nlevels - 1].ndof();
  GB_CUDA(c.krylov.alloc((vmax + 1) * n));
  GB_CUDA(c.pbuf.alloc(n));
  if (!c.G.p)
    GB_CUDA(c.G.alloc(1));
  if (flexible) {
    if (prec == GB_FP32) {
      GB_CUDA(c.zb32.alloc(vmax * n));
      GB_CUDA(c.fine_rhs32.alloc(n));
    } else {
      GB_CUDA(c.zb64.alloc(vmax * n));
    }
  }
}

__global__ void
k_gmres_setup(GmresDev* G, double tol, double globaltol, int maxiter)
{
  GB_PDL_ENTRY();
  G->info.tol = tol;
  G->info.globaltol = globaltol;
  G->info.breaktol = 1e15;
  G->info.miniter = 0;
  G->info.maxiter = maxiter;
  G->info.status = 0;
  G->info.iteration = 0;
  G->info.firstresidual = 0;
  G->info.previousresidual = 1;
  G->info.residual = 0;
  G->info.aimedresidual = 0;
  G->reached = 0;
  G->need_reortho = 0;
  G->zero_rho = 0;
}

__global__ void
k_scale_gmres(int64_t n, double* __restrict__ y, const GmresDev* G)
{
  GB_PDL_ENTRY();
  if (G->need_reortho)
    return;
  const double s = G->inv;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = s * y[i];
}

// MGS of vv against V_0..V_{dim-1} into column H[last] (GMRES::orthogonalization)
void
mgs(Context& c, int64_t n, double* vv, double* V, int dim, int last)
{
  GmresDev* G = c.G.p;
  const int grid = red_blocks(n);
  // d_0 = <vv, V_0>; H[last][0] += d_0
  {
    RedOut ro{ &G->d[0], &G->H[last][0], nullptr, 0 };
    launch(c, k_mgs, grid, kRedThreads, n, vv, (const double*)nullptr,
           (const double*)nullptr, (const double*)V, c.partials.p, c.ticket.p, ro);
  }
  for (int i = 0; i < dim; ++i) {
    const double* vi = V + int64_t(i) * n;
    if (i + 1 < dim) {
      RedOut ro{ &G->d[i + 1], &G->H[last][i + 1], nullptr, 0 };
      launch(c, k_mgs, grid, kRedThreads, n, vv, vi, (const double*)&G->d[i],
             (const double*)(V + int64_t(i + 1) * n), c.partials.p, c.ticket.p, ro);
    } else {
      RedOut ro{ &G->H[last][dim], nullptr, nullptr, 1 };
      launch(c, k_mgs, grid, kRedThreads, n, vv, vi, (const double*)&G->d[i],
             (const double*)vv, c.partials.p, c.ticket.p, ro);
    }
  }
}

void
read_flags(Context& c)
{
  GB_CUDA(cudaMemcpyAsync(c.h_flags, &c.G.p->reached, 3 * sizeof(int),
                          cudaMemcpyDeviceToHost, c.stream));
  GB_CUDA(cudaStreamSynchronize(c.stream));
}

void
fill_info_enqueue(Context& c, const double* x_for_residual, const double* b)
{
  auto* st = c.h_status;
  GB_CUDA(cudaMemcpyAsync(&st->info, &c.G.p->info, sizeof(CGInfoDev), cudaMemcpyDeviceToHost,
                          c.stream));
  st->mid_err = 0;
  if (c.miderr.p)
    GB_CUDA(cudaMemcpyAsync(&st->mid_err, c.miderr.p, sizeof(int), cudaMemcpyDeviceToHost,
                            c.stream));
  // true residual ||b - A x|| and ||b|| (FP64)
  const int fl = c.nlevels - 1;
  Level& L = c.L[fl];
  spmv<kResid, double, double, double>(c, L, opA(c, L), x_for_residual, c.pbuf.p, b,
                                       nullptr, 0.0);
  dot_dev(c, L.ndof(), c.pbuf.p, c.pbuf.p, RedOut{ c.scal.p + 4, nullptr, nullptr, 1 });
  dot_dev(c, L.ndof(), b, b, RedOut{ c.scal.p + 5, nullptr, nullptr, 1 });
  GB_CUDA(cudaMemcpyAsync(&st->true_res, c.scal.p + 4, 2 * sizeof(double),
                          cudaMemcpyDeviceToHost, c.stream));
}

// After the stream has been synchronised: the staged status into info.
void
fill_info_finish(Context& c, gb_solve_info* info)
{
  auto* st = c.h_status;
  if (st->mid_err) {
    GB_CUDA(cudaMemsetAsync(c.miderr.p, 0, sizeof(int), c.stream));
    throw Error{ GB_ETIMEOUT, "a grid barrier of the multi-CTA cycle gave up waiting" };
  }
  info->iterations = st->info.iteration;
  info->status = st->info.status;
  info->firstresidual = st->info.firstresidual;
  info->residual = st->info.residual;
  info->true_residual = st->true_res;
  info->rhs_norm = st->rhs_norm;
}

// The closing status and true residual of a solve, read with one sync.
void
fill_info(Context& c, gb_solve_info* info, double* x_for_residual, const double* b)
{
  fill_info_enqueue(c, x_for_residual, b);
  GB_CUDA(cudaStreamSynchronize(c.stream));
  fill_info_finish(c, info);
}

// NewtonLinearSolve's closing SubtractMean(x) on the finest level
// (Solver/stdmultilevelsolver.cc:671); a no-op without a pressure filter.
void
final_filter(Context& c, double* x)
{
  const int fl = c.nlevels - 1;
  if (!c.L[fl].pf_mask)
    return;
  Emit<double> E{ c, nullptr };
  E.pf_sub(fl, x, true);
}

// StdMultiLevelSolver::Gmres -> GMRES::solve (left preconditioning)
int
gmres_left(Context& c, double* x, const double* b, gb_solve_info* info)
{
  ensure_work(c);
  const int vmax = c.params.gmressize;
  ensure_gmres(c, vmax, false, GB_FP64);
  const int fl = c.nlevels - 1;
  Level& L = c.L[fl];
  const int64_t n = L.ndof();
  GmresDev* G = c.G.p;
  double* V = c.krylov.p;
  const int64_t l0 = c.launches;
  GB_CUDA(cudaEventRecord(c.ev0, c.stream));

  GB_CUDA(cudaMemsetAsync(G, 0, sizeof(GmresDev), c.stream));
  launch(c, k_gmres_setup, 1, 1, G, c.params.tol, c.params.globaltol,
         c.params.maxiter);
  GB_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), c.stream)); // NewtonLinearSolve
  // residualgmres: p = b - A x, Dirichlet zero
  spmv<kResidDir, double, double, double>(c, L, opA(c, L), x, c.pbuf.p, b, nullptr, 0.0);
  precondition_T<double>(c, c.w64, V, c.pbuf.p, true);
  dot_dev(c, n, V, V, RedOut{ c.scal.p, nullptr, nullptr, 1 });
  launch(c, k_gmres_init, 1, 1, G, (const double*)c.scal.p);
  read_flags(c);
  int dim = 0;
  if (!c.h_flags[2]) { // rho != 0
    launch(c, k_scale_dev, stream_blocks(n), 256, n, V, (const double*)&G->inv);
    int reached = 0;
    while (dim < vmax - 1 && !reached) {
      dim++;
      const int last = dim - 1;
      double* vv = V + int64_t(dim) * n;
      spmv<kAx, double, double, double>(c, L, opA(c, L), V + int64_t(last) * n, c.pbuf.p,
                                        nullptr, nullptr, 1.0);
      precondition_T<double>(c, c.w64, vv, c.pbuf.p, true);
      mgs(c, n, vv, V, dim, last);
      launch(c, k_gmres_step, 1, 1, G, dim, 0, 1, 0);
      launch(c, k_scale_gmres, stream_blocks(n), 256, n, vv, (const GmresDev*)G);
      read_flags(c);
      if (c.h_flags[1]) { // REORTHO: second orthogonalization pass
        mgs(c, n, vv, V, dim, last);
        launch(c, k_gmres_step, 1, 1, G, dim, 1, 1, 0);
        launch(c, k_scale_gmres, stream_blocks(n), 256, n, vv, (const GmresDev*)G);
        read_flags(c);
      }
      reached = c.h_flags[0];
    }
    launch(c, k_gmres_backward, 1, 1, G, dim);
    launch(c, k_multi_axpy<double>, stream_blocks(n), 256, n, x, (const double*)V, n,
           (const double*)G->hs, dim);
  }
  final_filter(c, x);
  GB_CUDA(cudaEventRecord(c.ev1, c.stream));
  GB_CUDA(cudaEventSynchronize(c.ev1));
  float ms = 0;
  GB_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
  if (info) {
    fill_info(c, info, x, b);
    info->restarts = 0;
    info->kernel_launches = static_cast<int>(c.launches - l0);
    info->device_ms = ms;
    if (c.h_flags[2]) {
      info->iterations = 0;
      info->status = 2;
    }
  }
  return GB_OK;
}

// Flexible GMRES (FP64 Arnoldi, cycle in `prec`), restarted as iterative
// refinement on the true FP64 residual.
int
gmres_flexible(Context& c, double* x, const double* b, int prec, gb_solve_info* info)
{
  ensure_work(c);
  const int vmax = c.params.gmressize;
  ensure_gmres(c, vmax, true, prec);
  const int fl = c.nlevels - 1;
  Level& L = c.L[fl];
  const int64_t n = L.ndof();
  const int m = vmax - 1;
  GmresDev* G = c.G.p;
  double* V = c.krylov.p;
  const int64_t l0 = c.launches;
  GB_CUDA(cudaEventRecord(c.ev0, c.stream));

  GB_CUDA(cudaMemsetAsync(G, 0, sizeof(GmresDev), c.stream));
  launch(c, k_gmres_setup, 1, 1, G, c.params.tol, c.params.globaltol,
         c.params.maxiter);
  dot_dev(c, n, b, b, RedOut{ &G->bnorm, nullptr, nullptr, 1 });
  GB_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), c.stream));
  int total = 0, restarts = 0, converged = 0, exploded = 0;
  double bnorm = -1.0;
  for (;;) {
    // r = b - A x (Dirichlet zero) into V_0, beta = ||r||
    spmv<kResidDir, double, double, double>(c, L, opA(c, L), x, V, b, nullptr, 0.0);
    dot_dev(c, n, V, V, RedOut{ c.scal.p, nullptr, nullptr, 1 });
    launch(c, k_fgmres_restart, 1, 1, G, (const double*)c.scal.p, vmax);
    double hv[2];
    GB_CUDA(cudaMemcpyAsync(&hv[0], c.scal.p, sizeof(double), cudaMemcpyDeviceToHost,
                            c.stream));
    GB_CUDA(cudaMemcpyAsync(&hv[1], &G->bnorm, sizeof(double), cudaMemcpyDeviceToHost,
                            c.stream));
    GB_CUDA(cudaStreamSynchronize(c.stream));
    const double beta = hv[0];
    bnorm = hv[1];
    if (!std::isfinite(beta) || !std::isfinite(bnorm)) {
      exploded = 1; // a non-finite residual never counts as converged
      break;
    }
    if (beta <= c.params.tol * bnorm || beta < c.params.globaltol || beta == 0.0) {
      converged = 1;
      break;
    }
    if (total >= c.params.maxiter || restarts > 50)
      break;
    launch(c, k_scale_dev, stream_blocks(n), 256, n, V, (const double*)&G->inv);
    int steps = 0;
    const int maxsteps = std::min(m, c.params.maxiter - total);
    for (int j = 0; j < maxsteps; ++j) {
      double* vj = V + int64_t(j) * n;
      double* w = V + int64_t(j + 1) * n;
      if (prec == GB_FP32) {
        float* z = c.zb32.p + int64_t(j) * n;
        launch(c, k_convert<double, float>, stream_blocks(n), 256, n, c.fine_rhs32.p,
               (const double*)vj);
        precondition_T<float>(c, c.w32, z, c.fine_rhs32.p, true);
        spmv<kAx, double, float, double>(c, L, opA(c, L), (const float*)z, w, nullptr,
                                         nullptr, 1.0);
      } else {
        double* z = c.zb64.p + int64_t(j) * n;
        precondition_T<double>(c, c.w64, z, vj, true);
        spmv<kAx, double, double, double>(c, L, opA(c, L), (const double*)z, w, nullptr,
                                          nullptr, 1.0);
      }
      mgs(c, n, w, V, j + 1, j);
      launch(c, k_gmres_step, 1, 1, G, j + 1, 1, 2, maxsteps);
      launch(c, k_scale_gmres, stream_blocks(n), 256, n, w, (const GmresDev*)G);
      steps = j + 1;
      read_flags(c);
      if (c.h_flags[0])
        break;
    }
    launch(c, k_gmres_backward, 1, 1, G, steps);
    if (prec == GB_FP32)
      launch(c, k_multi_axpy<float>, stream_blocks(n), 256, n, x,
             (const float*)c.zb32.p, n, (const double*)G->hs, steps);
    else
      launch(c, k_multi_axpy<double>, stream_blocks(n), 256, n, x,
             (const double*)c.zb64.p, n, (const double*)G->hs, steps);
    total += steps;
    restarts++;
  }
  final_filter(c, x);
  GB_CUDA(cudaEventRecord(c.ev1, c.stream));
  GB_CUDA(cudaEventSynchronize(c.ev1));
  float ms = 0;
  GB_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
  if (info) {
    fill_info(c, info, x, b);
    info->iterations = total;
    info->status = converged ? 2 : (exploded ? 4 : 3);
    info->restarts = restarts;
    info->kernel_launches = static_cast<int>(c.launches - l0);
    info->device_ms = ms;
  }
  return converged ? GB_OK : GB_ENOTCONV;
}


// ------------------------------------------------ graph-resident flexible GMRES

template<class T>
MgWork<T>& work(Context& c);
template<>
MgWork<double>& work<double>(Context& c)
{
  return c.w64;
}
template<>
MgWork<float>& work<float>(Context& c)
{
  return c.w32;
}

std::vector<cudaGraphNode_t>
leaf_nodes(cudaGraph_t g)
{
  size_t nn = 0, ne = 0;
  GB_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  if (nn)
    GB_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
  // _v2: the graph may hold programmatic (PDL) edges
  GB_CUDA(cudaGraphGetEdges_v2(g, nullptr, nullptr, nullptr, &ne));
  std::vector<cudaGraphNode_t> from(ne), to(ne);
  std::vector<cudaGraphEdgeData> ed(ne);
  if (ne)
    GB_CUDA(cudaGraphGetEdges_v2(g, from.data(), to.data(), ed.data(), &ne));
  std::vector<cudaGraphNode_t> leaves;
  for (auto nd : nodes)
    if (std::find(from.begin(), from.end(), nd) == from.end())
      leaves.push_back(nd);
  return leaves;
}

cudaGraph_t
add_while(cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps,
          cudaGraphConditionalHandle h, cudaGraphNode_t* node)
{
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  GB_CUDA(cudaGraphAddNode(node, g, deps.empty() ? nullptr : deps.data(), deps.size(),
                           &cp));
  return cp.conditional.phGraph_out[0];
}

// Buffers of the flexible solver for cycle precision T.

template<class T>
FBufs<T>
fg_buffers(Context& c, int prec)
{
  ensure_work(c);
  const int vmax = c.params.gmressize;
  GB_REQUIRE(vmax <= kCgsMaxJ, GB_EINVAL, "flexible solver needs gmressize <= 32");
  const int64_t n = c.L[c.nlevels - 1].ndof();
  GB_CUDA(c.krylov.alloc((vmax + 1) * n));
  GB_CUDA(c.pbuf.alloc(n));
  if (!c.G.p)
    GB_CUDA(c.G.alloc(1));
  GB_CUDA(c.xg.alloc(n));
  GB_CUDA(c.bg.alloc(n));
  if (prec == GB_FP32) {
    GB_CUDA(c.zb32.alloc(vmax * n));
    GB_CUDA(c.zfix32.alloc(n));
    GB_CUDA(c.rhs32.alloc(n));
    return FBufs<T>{ reinterpret_cast<T*>(c.zb32.p), reinterpret_cast<T*>(c.zfix32.p),
                     reinterpret_cast<T*>(c.rhs32.p) };
  }
  GB_CUDA(c.zb64.alloc(vmax * n));
  GB_CUDA(c.zfix64.alloc(n));
  GB_CUDA(c.rhs64.alloc(n));
  return FBufs<T>{ reinterpret_cast<T*>(c.zb64.p), reinterpret_cast<T*>(c.zfix64.p),
                   reinterpret_cast<T*>(c.rhs64.p) };
}

// Segments of the flexible solve; the graph captures them, the eager driver
// (profiling) launches them from host loops. hOuter/hInner == 0: no graph.
template<class T>
void
fg_setup(Context& c)
{
  const int64_t n = c.L[c.nlevels - 1].ndof();
  GmresDev* G = c.G.p;
  launch(c, k_fg_setup, 1, 1, G, c.params.tol, c.params.globaltol, c.params.maxiter);
  dot_dev(c, n, c.bg.p, c.bg.p, RedOut{ &G->bnorm, nullptr, nullptr, 1 });
  launch(c, k_fill<double>, stream_blocks(n), 256, n, c.xg.p, 0.0);
}

template<class T>
void
fg_outer_pre(Context& c, cudaGraphConditionalHandle hOuter,
             cudaGraphConditionalHandle hInner, int use_cond)
{
  const int fl = c.nlevels - 1;
  Level& L = c.L[fl];
  const int64_t n = L.ndof();
  GmresDev* G = c.G.p;
  double* V = c.krylov.p;
  spmv<kResidDir, double, double, double>(c, L, opA(c, L), (const double*)c.xg.p, V, c.bg.p,
                                          nullptr, 0.0);
  dot_dev(c, n, V, V, RedOut{ &G->beta_tmp, nullptr, nullptr, 1 });
  launch(c, k_fg_restart, 1, 1, G, hOuter, hInner, c.params.gmressize - 1, 50,
         use_cond);
  launch(c, k_scale_dev, stream_blocks(n), 256, n, V, (const double*)&G->inv);
}

template<class T>
void
fg_inner(Context& c, const FBufs<T>& F, cudaGraphConditionalHandle hInner, int use_cond)
{
  const int fl = c.nlevels - 1;
  Level& L = c.L[fl];
  const int64_t n = L.ndof();
  GmresDev* G = c.G.p;
  double* V = c.krylov.p;
  // the cycle's right-hand side v_j and, where the finest smoother allows,
  // the cycle's first finest-level sweep from zero in the same pass
  T* u1 = precondition_first_sweep<T>(c, work<T>(c), F.zfix);
  launch(c, k_load_idx<T>, stream_blocks(n), 256, n, F.rhs, V, (const GmresDev*)G,
         dinv_of<T>(L), u1, c.params.omega);
  precondition_T<T>(c, work<T>(c), F.zfix, F.rhs, true, u1 != nullptr);
  spmv<kAx, double, T, double>(c, L, opA(c, L), (const T*)F.zfix, V, nullptr, nullptr, 1.0,
                               (const int*)&G->j, n, F.Z);
  // one block of kCgsThreads per 2 kCgsThreads rows, at most one wave
  const int rg = static_cast<int>(std::max<int64_t>(
    1, std::min<int64_t>((n + 2 * kCgsThreads - 1) / (2 * kCgsThreads), kCgsMaxBlocks)));
  const int m = c.params.gmressize - 1;
  launch(c, k_cgs<0>, rg, kCgsThreads, n, V, G, c.partials.p, c.ticket.p, hInner, m, 0);
  // second pass, norm, Givens update, loop test; v_{j+1} gets the second
  // pass's update and its normalisation from the next k_load_idx
  launch(c, k_cgs<1>, rg, kCgsThreads, n, V, G, c.partials.p, c.ticket.p, hInner, m,
         use_cond);
}

template<class T>
void
fg_outer_post(Context& c, const FBufs<T>& F)
{
  const int64_t n = c.L[c.nlevels - 1].ndof();
  GmresDev* G = c.G.p;
  launch(c, k_fg_backward, 1, 1, G);
  launch(c, k_fg_update<T>, stream_blocks(n), 256, n, c.xg.p, (const T*)F.Z,
         (const GmresDev*)G);
}

// Builds the one-graph solve: setup; WHILE(refine) { r = b - A x; beta; restart;
// v0 = r / beta; WHILE(arnoldi) { z = M v_j (cycle in T); v_{j+1} = A z; CGS2;
// Givens } ; y = H^-1 gamma; x += Z y }. Operates on the context's xg/bg.
template<class T>
void
build_fgraph(Context& c, int prec)
{
  const FBufs<T> F = fg_buffers<T>(c, prec);
  const int64_t n = c.L[c.nlevels - 1].ndof();
  auto& FG = c.fg[c.transposed][prec];
  if (FG.exec) {
    cudaGraphExecDestroy(FG.exec);
    FG.exec = nullptr;
  }
  if (FG.graph) {
    cudaGraphDestroy(FG.graph);
    FG.graph = nullptr;
  }
  // Record the coarse-kernel programs outside the capture (one eager cycle on
  // zeros), so that nothing is allocated or copied while capturing.
  GB_CUDA(cudaMemsetAsync(F.rhs, 0, n * sizeof(T), c.stream));
  precondition_T<T>(c, work<T>(c), F.zfix, F.rhs, true);
  GB_CUDA(cudaStreamSynchronize(c.stream));
  const cudaStreamCaptureMode mode = cudaStreamCaptureModeRelaxed;
  cudaGraph_t top;
  GB_CUDA(cudaGraphCreate(&top, 0));
  FG.graph = top;
  // each conditional handle belongs to the graph that holds its node
  cudaGraphConditionalHandle hOuter, hInner;
  GB_CUDA(cudaGraphConditionalHandleCreate(&hOuter, top, 1, cudaGraphCondAssignDefault));
  const int64_t k_start = c.launches;
  GB_CUDA(cudaStreamBeginCaptureToGraph(c.stream, top, nullptr, nullptr, 0, mode));
  fg_setup<T>(c);
  GB_CUDA(cudaStreamEndCapture(c.stream, &top));
  FG.setup_k = static_cast<int>(c.launches - k_start);
  cudaGraphNode_t outerNode, innerNode;
  cudaGraph_t outerBody = add_while(top, leaf_nodes(top), hOuter, &outerNode);
  GB_CUDA(cudaGraphConditionalHandleCreate(&hInner, outerBody, 0,
                                           cudaGraphCondAssignDefault));
  const int64_t k0 = c.launches;
  GB_CUDA(cudaStreamBeginCaptureToGraph(c.stream, outerBody, nullptr, nullptr, 0, mode));
  fg_outer_pre<T>(c, hOuter, hInner, 1);
  GB_CUDA(cudaStreamEndCapture(c.stream, &outerBody));
  cudaGraph_t innerBody = add_while(outerBody, leaf_nodes(outerBody), hInner, &innerNode);
  const int64_t k1 = c.launches;
  GB_CUDA(cudaStreamBeginCaptureToGraph(c.stream, innerBody, nullptr, nullptr, 0, mode));
  fg_inner<T>(c, F, hInner, 1);
  GB_CUDA(cudaStreamEndCapture(c.stream, &innerBody));
  FG.inner_k = static_cast<int>(c.launches - k1);
  const int64_t k2 = c.launches;
  GB_CUDA(cudaStreamBeginCaptureToGraph(c.stream, outerBody, &innerNode, nullptr, 1, mode));
  fg_outer_post<T>(c, F);
  GB_CUDA(cudaStreamEndCapture(c.stream, &outerBody));
  FG.outer_k = static_cast<int>(k1 - k0) + static_cast<int>(c.launches - k2);
  c.launches = k_start; // capture executes nothing; executions are counted per solve
  GB_CUDA(cudaGraphInstantiate(&FG.exec, top, 0));
  FG.version = c.version;
}

// The same solve driven from the host (no graph, no conditional nodes): used
// when GB_GRAPH=0, e.g. for per-kernel profiling, which cannot see inside
// conditional graph nodes.
template<class T>
void
fgmres_eager(Context& c, int prec)
{
  const FBufs<T> F = fg_buffers<T>(c, prec);
  GmresDev* G = c.G.p;
  fg_setup<T>(c);
  for (;;) {
    fg_outer_pre<T>(c, 0, 0, 0);
    int st = 0;
    GB_CUDA(cudaMemcpyAsync(&st, &G->stop, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    GB_CUDA(cudaStreamSynchronize(c.stream));
    if (!st) {
      for (;;) {
        fg_inner<T>(c, F, 0, 0);
        int reached = 0;
        GB_CUDA(cudaMemcpyAsync(&reached, &G->reached, sizeof(int),
                                cudaMemcpyDeviceToHost, c.stream));
        GB_CUDA(cudaStreamSynchronize(c.stream));
        if (reached)
          break;
      }
    }
    fg_outer_post<T>(c, F);
    if (st)
      break;
  }
}

// Runs the graph on b (device), result into x (device); info as gb_fgmres.
int
fgmres_graph(Context& c, double* x, const double* b, int prec, gb_solve_info* info,
             bool copy_in, bool copy_out, double* host_x, cudaEvent_t after_copy)
{
  auto& F = c.fg[c.transposed][prec];
  if (c.use_graph && (!F.exec || F.version != c.version)) {
    if (prec == GB_FP32)
      build_fgraph<float>(c, prec);
    else
      build_fgraph<double>(c, prec);
  }
  if (!c.use_graph) {
    if (prec == GB_FP32)
      fg_buffers<float>(c, prec);
    else
      fg_buffers<double>(c, prec);
  }
  const int64_t n = c.L[c.nlevels - 1].ndof();
  if (copy_in && b != c.bg.p)
    GB_CUDA(cudaMemcpyAsync(c.bg.p, b, n * sizeof(double), cudaMemcpyDeviceToDevice,
                            c.stream));
  const int64_t l_before = c.launches;
  GB_CUDA(cudaEventRecord(c.ev0, c.stream));
  if (c.use_graph) {
    GB_CUDA(cudaGraphLaunch(F.exec, c.stream));
  } else if (prec == GB_FP32) {
    fgmres_eager<float>(c, prec);
  } else {
    fgmres_eager<double>(c, prec);
  }
  const int64_t l_filter = c.launches;
  final_filter(c, c.xg.p);
  const int64_t filter_k = c.launches - l_filter;
  const int64_t l_solved = c.launches; // the status read below launches more
  GB_CUDA(cudaEventRecord(c.ev1, c.stream));
  if (copy_out && x != c.xg.p)
    GB_CUDA(cudaMemcpyAsync(x, c.xg.p, n * sizeof(double), cudaMemcpyDeviceToDevice,
                            c.stream));
  // a host-buffer caller's solution goes out before the status read, inside
  // its timing window
  if (host_x)
    GB_CUDA(cudaMemcpyAsync(host_x, c.xg.p, n * sizeof(double), cudaMemcpyDeviceToHost,
                            c.stream));
  if (after_copy)
    GB_CUDA(cudaEventRecord(after_copy, c.stream));
  auto* st = c.h_status;
  GB_CUDA(cudaMemcpyAsync(&st->total, &c.G.p->total, 2 * sizeof(int), cudaMemcpyDeviceToHost,
                          c.stream));
  GB_CUDA(cudaMemcpyAsync(&st->converged, &c.G.p->converged, sizeof(int),
                          cudaMemcpyDeviceToHost, c.stream));
  if (info)
    fill_info_enqueue(c, c.xg.p, c.bg.p);
  GB_CUDA(cudaStreamSynchronize(c.stream));
  float ms = 0;
  GB_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
  const int total = st->total, restarts = st->restarts, conv = st->converged;
  int64_t kernels = l_solved - l_before;
  if (c.use_graph) {
    kernels = F.setup_k + int64_t(restarts + 1) * F.outer_k + int64_t(total) * F.inner_k;
    c.launches += kernels;
    kernels += filter_k;
  }
  if (info) {
    fill_info_finish(c, info);
    info->iterations = total;
    info->restarts = restarts;
    info->status = conv ? 2 : (info->status == 4 ? 4 : 3); // 4: non-finite residual
    info->kernel_launches = static_cast<int>(kernels);
    info->device_ms = ms;
  }
  return conv ? GB_OK : GB_ENOTCONV;
}

template FBufs<double> fg_buffers<double>(Context&, int);
template FBufs<float> fg_buffers<float>(Context&, int);

} // namespace gb
