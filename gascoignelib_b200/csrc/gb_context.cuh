// Internal header of the host library: device memory, the level and
// context types, launch helpers and the SpMV dispatch shared by the
// translation units (gb_setup.cu: matrix layouts and level set-up;
// gb_cycle.cu: the multigrid cycle; gb_gmres.cu: the GMRES drivers;
// gb_api.cu, gb_assembly.cu, gb_noalloc.cu: the C-ABI).
//
// The classes here mirror the reference's call surface for this path:
//   Level      ~ StdSolver / CudaSolver per level (vmult, MatrixResidual, smooth,
//                SetBoundaryVectorZero, vector ops)   Solver/stdsolver.cc,
//                cuda/cudasolver.cc
//   Transfer   ~ MgInterpolatorMatrix / CudaMgInterpolatorNested
//                (restrict_zero, prolongate_add)      Discretization/Q1/
//                mginterpolatormatrix.cc, cuda/cudamgintepolatornested.cc
//   Context    ~ StdMultiLevelSolver / CudaMultiLevelSolver (LinearMg, mgstep,
//                precondition, Gmres)                 Solver/stdmultilevelsolver.cc
// Device vectors stay resident for the whole solve; nothing is copied between
// host and device inside a solve except 8-byte status words.
#pragma once
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <string>
#include <vector>

#include "../../include/gascoigne_b200.h"
#include "gb_kernels.cuh"
#include "gb_block.cuh"
#include "gb_assembly.cuh"

namespace gb {

// ------------------------------------------------------------------ memory

// Host-side fault injection for the tests of the out-of-memory path
// (gb_debug_fail_alloc): when set to k > 0, the k-th device allocation from
// then on fails as cudaMalloc does when the device is out of memory.
extern std::atomic<long long> g_fail_alloc_countdown;

inline cudaError_t
device_malloc(void** p, size_t bytes)
{
  long long k = g_fail_alloc_countdown.load();
  while (k > 0 && !g_fail_alloc_countdown.compare_exchange_weak(k, k - 1)) {
  }
  if (k == 1) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}

template<class T>
struct DeviceArray
{
  T* p = nullptr;
  size_t n = 0;
  DeviceArray() = default;
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  DeviceArray(DeviceArray&& o) noexcept
    : p(o.p)
    , n(o.n)
  {
    o.p = nullptr;
    o.n = 0;
  }
  DeviceArray& operator=(DeviceArray&& o) noexcept
  {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DeviceArray() { release(); }
  void release()
  {
    if (p)
      cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count)
  {
    if (count == n && p)
      return cudaSuccess;
    release();
    if (count == 0)
      return cudaSuccess;
    cudaError_t e = device_malloc(reinterpret_cast<void**>(&p), count * sizeof(T));
    if (e == cudaSuccess)
      n = count;
    else
      p = nullptr;
    return e;
  }
};

struct Error
{
  int code;
  std::string msg;
};

#define GB_CUDA(call)                                                          \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess)                                                     \
      throw ::gb::Error{ (e_ == cudaErrorMemoryAllocation) ? GB_ENOMEM         \
                                                           : GB_ECUDA,         \
                         std::string(#call) + ": " + cudaGetErrorString(e_) }; \
  } while (0)

#define GB_REQUIRE(cond, code, msg)                                            \
  do {                                                                         \
    if (!(cond))                                                               \
      throw ::gb::Error{ code, msg };                                          \
  } while (0)

// --------------------------------------------------------------- matrices

// SELL-32: slice s holds rows 32s..32s+31, column-major (entry j of lane l at
// sptr[s] + 32 j + l); slice width = longest row of the slice; padding uses
// column = own row (or 0 past n) and value 0. Block rows (B > 1) keep one
// column per block; value q of the block is at (sptr[s] + 32 j) * B*B + 32 q + l.
struct Sell
{
  int n = 0, nslices = 0, B = 1; // n block rows of B x B blocks
  int64_t entries = 0, nnz = 0;
  DeviceArray<int> sptr, col;
  DeviceArray<double> v64;
  DeviceArray<float> v32;
  // pattern-compressed form: row r's columns are r + ptab[pid[r]*W + j]
  bool pat = false;
  int npat = 0, W = 0;
  DeviceArray<uint8_t> pid;
  DeviceArray<int> ptab;
  // slot -> row when the rows are ordered by length in windows (SELL-C-sigma)
  bool sorted = false;
  DeviceArray<int> rperm;
  // without patterns: 16-bit offsets col - row beside col when they all fit
  // (the scalar SpMV reads these; the op programs read col)
  bool off16 = false;
  DeviceArray<int16_t> c16;
  // host copies of the layout: slice starts and slot -> row (device-side
  // gathers built on the host, e.g. the Vanka patch matrices, address these)
  std::vector<int> h_sptr, h_perm;
  // row-major FP32 copy for the row-block SpMV (GB_RB=1, large B = 1 levels):
  // row r's entries at r * Wr + j, columns from the patterns (rows of Wr
  // offsets) or from rcol; rslot = row -> slot when the slots are sorted
  bool rb = false;
  int Wr = 0;
  DeviceArray<float> r32;
  DeviceArray<int> rcol, rslot;
};

// Host-to-device copy ordered on `st` (the context's stream) and complete on
// return. A plain cudaMemcpy from pageable host memory can return before its
// DMA has reached the device, and kernels on a non-blocking stream do not wait
// for the legacy stream it runs on.
inline cudaError_t
h2d(cudaStream_t st, void* dst, const void* src, size_t bytes)
{
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(st);
  return e;
}

template<class TV>
inline SellView<TV>
view(const Sell& S, const TV* val)
{
  return SellView<TV>{ S.n, S.sptr.p, S.pat ? nullptr : S.col.p,
                       S.pat ? S.pid.p : nullptr, S.pat ? S.ptab.p : nullptr,
                       S.W, val, S.sorted ? S.rperm.p : nullptr,
                       !S.pat && S.off16 ? S.c16.p : nullptr };
}

template<class T>
const T* sell_vals(const Sell& S);
template<>
inline const double* sell_vals<double>(const Sell& S)
{
  return S.v64.p;
}
template<>
inline const float* sell_vals<float>(const Sell& S)
{
  return S.v32.p;
}

struct Level
{
  int64_t n = 0;
  int B = 1;
  bool has_matrix = false;
  std::vector<int64_t> h_rowptr, h_col, h_diag;
  std::vector<double> h_val;
  Sell A, AT;
  bool has_AT = false;
  DeviceArray<double> dinv64;
  DeviceArray<float> dinv32;
  DeviceArray<uint8_t> dirmask;
  DeviceArray<int> dirlist;
  int ndir = 0;
  // cells for the coefficient gradient (gb_level_set_cells)
  int ncells = 0, nloc = 0;
  int64_t cells_n = -1; // level size the cell node indices were checked against
  DeviceArray<int> cells; // node-major: entry i of cell c at i * ncells + c
  DeviceArray<double> kloc, cscale, grad;
  bool has_scale = false;
  // quadratic functional J(u) = u^T M u over the cells (gb_level_set_functional)
  Sell M;
  int64_t func_n = -1;
  // pressure filter (gb_level_set_pfilter): filtered components, weights
  int pf_mask = 0;
  DeviceArray<double> pf_w;
  double pf_domain = 0.0;
  int64_t nhanging = 0;
  // Vanka patches (gb_level_set_patches) and their factorisations
  std::vector<int64_t> h_patches;
  int npatch = 0, npp = 0, vk_M = 0;
  bool vk_ready = false;
  bool vk_struct = false; // patch lists, node map and gather offsets built
  DeviceArray<int> vk_pn, vk_nptr, vk_ent, vk_map;
  DeviceArray<double> vk_inv64, vk_out64; // inverses [patch][j][i], solutions
  DeviceArray<float> vk_inv32, vk_out32;
  // hanging nodes (gb_level_set_hn): phases in the discretisation's order
  struct HnPhase
  {
    int nh = 0, nslots = 0, gsize = 0, np = 0;
    DeviceArray<int> node, par, pnode, ptr, hnode;
    DeviceArray<double> w, wt;
  };
  std::vector<HnPhase> hn;
  std::vector<int> h_hnnodes;  // all hanging nodes
  DeviceArray<int> hn_all;
  DeviceArray<uint8_t> pmask;  // Dirichlet | hanging dofs (prolongation mask)
  // Q1 mesh for the device assembly (gb_level_set_mesh): cells [a][c], node
  // coordinates, per SELL entry the element-matrix entries summed into it
  // (ascending cells), the diagonal's SELL position per row, this level's
  // cell coefficients, and the parent cell (level - 1) of every cell
  int mesh_dim = 0, mesh_deg = 1;
  int64_t mesh_ncells = 0, mesh_n = -1;
  DeviceArray<int> m_cells, m_cptr, m_clist, m_diagpos, m_child_ptr, m_child;
  DeviceArray<int> m_nptr, m_nlist; // per node its (cell, local index) pairs
  double m_beta[3] = { 0.0, 0.0, 0.0 }; // convection of the last assembly
  double m_lps_s0 = 0.0, m_lps_xeta = 6.0; // its LPS (sdelta0 0: none)
  bool m_assembled = false;
  DeviceArray<double> m_coords, m_kappa, m_dd;
  // hanging nodes in the device assembly: per hanging node (h_hnidx[node],
  // -1 elsewhere) its phase (0 edges, 1 faces), parents and weights in the
  // HNStructure's parent order; the cells with a hanging node, their
  // condensation steps (m_hopptr per cell), and the Dirichlet-or-hanging mask
  struct HnCond
  {
    int phase = 0, np = 0;
    int par[9];
    double w[9];
  };
  std::vector<HnCond> h_hncond;
  std::vector<int> h_hnidx;
  int m_nhcells = 0;
  DeviceArray<int> m_hcells, m_hopptr;
  DeviceArray<CondOp> m_hops;
  DeviceArray<uint8_t> m_hmask;
  std::vector<int64_t> h_parent;
  int64_t child_n = -1; // coarse cells the child lists were built for
  // block ILU (smoother 2, SparseBlockIlu): the factors in the matrix's row
  // order with ascending columns, the diagonal blocks inverted, and the rows
  // grouped in dependency levels for the two substitutions
  bool ilu_ready = false;
  DeviceArray<int> ilu_ptr, ilu_col, ilu_diag, ilu_lrows, ilu_urows, ilu_map;
  bool ilu_struct = false; // the sorted layout, levels and gather map built
  DeviceArray<double> ilu_v64;
  DeviceArray<float> ilu_v32;
  std::vector<int> ilu_lptr, ilu_uptr; // level offsets into ilu_lrows / ilu_urows
  DeviceArray<int> ilu_lptr_d, ilu_uptr_d;
  // the launches of the two substitutions: [lv0, lv1) in one CTA, or one wide level
  struct IluSeg
  {
    int lv0, lv1;
    bool cta;
  };
  std::vector<IluSeg> ilu_lseg, ilu_useg;
  // values assembled on the device since the host copy was made
  bool h_val_stale = false;
  // per A^T SELL entry the A SELL entry it copies (-1: padding), block size 1:
  // the transpose's values follow a device assembly without the host
  DeviceArray<int> at_map;
  bool has_hn() const { return !hn.empty(); }
  int64_t ndof() const { return n * B; }
};

struct Transfer
{
  bool set = false;
  int nc = 0, nf = 0;
  int rmaxw = 0; // widest restriction row (k_restrict4 takes rows of <= 32)
  int64_t nent = 0;
  DeviceArray<int> rptr, pptr;
  DeviceArray<uint32_t> rent, pent;
};

struct CoarseKey
{
  int tsize, level;
  const void *u, *tmp, *b;
  bool zero;
  char p0, p;
  bool tr;
  bool operator<(const CoarseKey& o) const
  {
    return std::tie(tsize, level, u, tmp, b, zero, p0, p, tr) <
           std::tie(o.tsize, o.level, o.u, o.tmp, o.b, o.zero, o.p0, o.p, o.tr);
  }
};

struct CoarseProgram
{
  DeviceArray<CoarseOp> ops;
  DeviceArray<CoarseBuf> bufs;
  DeviceArray<CoarsePrefetch> pre;
  int nops = 0, nbufs = 0, npre = 0, vec_bytes = 0, smem_bytes = 0;
  // precomputed linear map u_out = K [b; u_start] (dense mode)
  DeviceArray<double> K64;
  DeviceArray<float> K32;
  int ncols = 0, nb = 0, n_root = 0;
  const void* b_root = nullptr;
  const void* u_in = nullptr;
  const void* u_out = nullptr;
  const void* tmp_out = nullptr;
  char p0_out = 'V';
  bool zero_out = false;
  // the batch launch that formed K, kept to form it again in place after the
  // matrix values change (a device assembly)
  CoarseBatch batch{};
  int tsize = 0;
};

template<class T>
struct MgWork
{
  std::vector<DeviceArray<T>> u, b, v; // per level (finest: v only used)
};

} // namespace gb

struct gb_ctx
{
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  gb_params params{ 4, 4, 10, 1.0, 1.0, 'V', 10, 1e-2, 1e-12, 10, 0, 0 };
  int nlevels = 0;
  std::vector<gb::Level> L;
  std::vector<gb::Transfer> T;
  std::map<int, std::vector<gb::DeviceArray<double>>> vecs;
  int next_id = 1;
  gb::MgWork<double> w64;
  gb::MgWork<float> w32;
  bool work_ready = false;
  gb::DeviceArray<double> partials;
  gb::DeviceArray<double> pfpart;    // per-block sums of the fused filter reductions
  gb::DeviceArray<unsigned> pfticket;
  gb::DeviceArray<unsigned> ticket;
  gb::DeviceArray<double> scal; // general device scalars
  gb::DeviceArray<gb::GmresDev> G;
  gb::DeviceArray<double> krylov, zb64, pbuf, fine32_rhs_dummy;
  gb::DeviceArray<float> zb32, fine_rhs32;
  int* h_flags = nullptr; // pinned
  // pinned staging of a solve's closing status read (one transfer, one sync)
  struct SolveStatus
  {
    gb::CGInfoDev info;
    double true_res, rhs_norm;
    int total, restarts, converged, mid_err;
  };
  SolveStatus* h_status = nullptr;
  cudaEvent_t evh0 = nullptr, evh1 = nullptr; // gb_solve_host's window
  int64_t launches = 0;
  gb::DeviceArray<unsigned char> flush;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // graph-resident flexible GMRES, one per cycle precision
  int64_t version = 0; // bumped by every change of levels, transfers or keys
  struct FGraph
  {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t version = -1;
    int setup_k = 0, outer_k = 0, inner_k = 0;
  } fg[2][2]; // [operator transposed][cycle precision]
  // level operators: A (0) or A^T (1) for every solver step (gb_set_operator)
  int transposed = 0;
  // coarse-level kernel: levels 0..coarse_root, programs per entry state
  bool coarse_on = true;
  bool coarse_dense = true; // apply the coarse sub-cycle as its precomputed map
  bool use_graph = true; // flexible solver as one CUDA graph (GB_GRAPH=0: host loops)
  bool pdl = true;       // programmatic dependent launch between kernels
  // first two sweeps from zero in one pass (GB_JACOBI2=1); off by default:
  // the saved launch costs more in the second sweep's extra gathers (C2: mixed
  // 1.680 vs 1.670 ms, FP64 1.91 vs 1.86 ms)
  bool jacobi2 = false;
  // per-kernel timing
  bool ktime = false;
  struct KtPending
  {
    const void* func;
    cudaEvent_t e0, e1;
  };
  std::vector<cudaEvent_t> kt_pool;
  std::vector<KtPending> kt_pending;
  std::map<std::string, std::pair<int64_t, double>> kt_acc;
  int coarse_root = -1;
  std::map<gb::CoarseKey, gb::CoarseProgram> coarse_progs;
  // coarsest-level direct solve (gb_params.ndirect): the FP64 inverse of level
  // 0's operator, per orientation (A, A^T)
  gb::DeviceArray<double> dir_inv[2];
  bool dir_ready[2] = { false, false };
  // dense maps of coarse sub-cycles that the single-CTA program does not cover
  // (block systems, Vanka, pressure filter): levels 0..dense_root
  int dense_root = -1;
  std::map<gb::CoarseKey, gb::CoarseProgram> dense_maps;
  // multi-CTA program for the levels below the finest (mid_level and down)
  // GB_MID=1: the levels below the finest as one cooperative persistent grid
  // with grid barriers between the ops. Off by default: on C2 it measured
  // slower than the per-level kernels with programmatic dependent launch
  // (mixed solve 1.97 vs 1.69 ms): each op there is itself latency-bound
  // (1-2 rows per thread) and a grid barrier costs about as much as a launch.
  bool mid_on = false;
  // GB_VANKA_HOST=1: Vanka patch inverses formed on the host (the default is
  // the device kernel k_vanka_factor, which gives the same bits)
  bool vanka_host = false;
  bool ilu_host = false; // GB_ILU_HOST=1: block ILU factors formed on the host
  bool rb_on = false;    // GB_RB=1: row-block copies and SpMV on the large FP32 levels
  // the slots of scalar levels above 1024 rows without column patterns
  // ordered by each row's smallest column before the windows are sorted by
  // length (GB_ROW_ORDER=0: not)
  bool row_order = true;
  // widest substitution level run inside a single-CTA launch
  // (GB_ILU_CTA_ROWS; 0: one launch per level)
  int ilu_cta_rows = gb::kIluCtaDefaultRows;
  // GB_CLUSTER=1: the levels of at most cluster_rows dofs below the finest
  // (and above the single-CTA coarse levels) as one op program run by one
  // thread-block cluster of 16 CTAs with the hardware cluster barrier between
  // ops (GB_CLUSTER_ROWS: the bound). Off by default: on C2 it measured slower
  // than the per-level kernels with programmatic dependent launch (mixed solve
  // 1.88 ms with the 17^3 level and below, 2.85 ms with the 33^3 level and
  // below, against 1.60 ms): 16 SMs run each op of a level of 5,000 to 36,000
  // rows at L2 latency, row after row, slower than a whole-GPU launch does.
  bool cluster_on = false;
  int64_t cluster_rows = 8192;
  int cluster_size[2] = { 0, 0 }; // CTAs of the cluster per cycle type (0: not queried)
  // bound of every device-side wait (grid barriers), and the phantom
  // arrivals a test adds so that a wait runs out (gb_set_wait_limit)
  unsigned long long wait_ns = 1000000000ull;
  unsigned barrier_phantoms = 0;
  int mid_level = -1;
  std::map<gb::CoarseKey, gb::CoarseProgram> mid_progs;
  gb::DeviceArray<unsigned> midbar;
  gb::DeviceArray<int> miderr;
  int mid_grid[2] = { 0, 0 }; // per precision (FP64, FP32)
  gb::DeviceArray<double> xg, bg, rhs64, zfix64;
  gb::DeviceArray<double> asm_E; // element matrices of the level being assembled
  gb::DeviceArray<double> asm_R; // element residuals (Form of patch elements)
  double lps_s0 = 0.0, lps_xeta = 6.0; // LPS of the convection in Q2 assemblies (0: off)
  gb::DeviceArray<unsigned long long> nrm; // largest |y| of gb_newton_residual
  // matrix values changed on the device since the solver's set-up (dense
  // coarse maps, direct inverse): refreshed in place at the next solve
  bool values_dirty = false;
  gb::DeviceArray<float> rhs32, zfix32;
  ~gb_ctx()
  {
    for (auto e : kt_pool)
      cudaEventDestroy(e);
    for (auto& p : kt_pending) {
      cudaEventDestroy(p.e0);
      cudaEventDestroy(p.e1);
    }
    for (auto& row : fg)
      for (auto& g : row) {
        if (g.exec)
          cudaGraphExecDestroy(g.exec);
        if (g.graph)
          cudaGraphDestroy(g.graph);
      }
  }
};

namespace gb {
using Context = gb_ctx;

inline void
check_launch(Context& c)
{
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    throw Error{ GB_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e) };
}

// Per-kernel device timing (gb_set_timing): an event pair around each launch
// outside graph capture, resolved by kt_flush.
inline void
kt_begin(Context& c, cudaEvent_t* e0)
{
  *e0 = nullptr;
  if (!c.ktime)
    return;
  cudaStreamCaptureStatus cs;
  if (cudaStreamIsCapturing(c.stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
    return;
  if (c.kt_pool.empty()) {
    cudaEvent_t e;
    GB_CUDA(cudaEventCreate(&e));
    c.kt_pool.push_back(e);
  }
  *e0 = c.kt_pool.back();
  c.kt_pool.pop_back();
  GB_CUDA(cudaEventRecord(*e0, c.stream));
}

inline void
kt_end(Context& c, cudaEvent_t e0, const void* func)
{
  if (!e0)
    return;
  if (c.kt_pool.empty()) {
    cudaEvent_t e;
    GB_CUDA(cudaEventCreate(&e));
    c.kt_pool.push_back(e);
  }
  cudaEvent_t e1 = c.kt_pool.back();
  c.kt_pool.pop_back();
  GB_CUDA(cudaEventRecord(e1, c.stream));
  c.kt_pending.push_back({ func, e0, e1 });
}

inline void
kt_flush(Context& c)
{
  if (c.kt_pending.empty())
    return;
  GB_CUDA(cudaStreamSynchronize(c.stream));
  for (auto& p : c.kt_pending) {
    float ms = 0;
    GB_CUDA(cudaEventElapsedTime(&ms, p.e0, p.e1));
    const char* name = nullptr;
    if (cudaFuncGetName(&name, p.func) != cudaSuccess || !name)
      name = "?";
    auto& a = c.kt_acc[name];
    a.first += 1;
    a.second += ms;
    c.kt_pool.push_back(p.e0);
    c.kt_pool.push_back(p.e1);
  }
  c.kt_pending.clear();
}

// Launches on the context stream; with programmatic dependent launch unless
// GB_PDL=0 (every kernel begins with GB_PDL_ENTRY).
template<class... KArgs, class... Args>
inline void
launch_smem(Context& c, void (*kern)(KArgs...), int grid, int block, int smem,
            Args... args)
{
  if (grid <= 0)
    return;
  cudaEvent_t e0;
  kt_begin(c, &e0);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c.stream;
  cudaLaunchAttribute attr[1];
  int na = 0;
  if (c.pdl) {
    attr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[na].val.programmaticStreamSerializationAllowed = 1;
    ++na;
  }
  cfg.attrs = attr;
  cfg.numAttrs = na;
  GB_CUDA(cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...));
  c.launches++;
  check_launch(c);
  kt_end(c, e0, reinterpret_cast<const void*>(kern));
}

template<class... KArgs, class... Args>
inline void
launch(Context& c, void (*kern)(KArgs...), int grid, int block, Args... args)
{
  launch_smem(c, kern, grid, block, 0, args...);
}

inline int
blocks_for(int64_t n, int threads)
{
  return static_cast<int>((n + threads - 1) / threads);
}

inline int
red_blocks(int64_t n)
{
  int64_t b = (n + kRedThreads * 8 - 1) / (kRedThreads * 8);
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(b, kMaxRedBlocks)));
}

inline int
stream_blocks(int64_t n)
{
  int64_t b = (n + 255) / 256;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(b, 148 * 16)));
}

inline Level&
level(Context& c, int l)
{
  GB_REQUIRE(l >= 0 && l < c.nlevels, GB_EINVAL, "level out of range");
  return c.L[l];
}

inline Level&
level_with_matrix(Context& c, int l)
{
  Level& L = level(c, l);
  GB_REQUIRE(L.has_matrix, GB_ESTATE, "no matrix on this level");
  return L;
}

inline double*
vec(Context& c, int l, int id)
{
  auto it = c.vecs.find(id);
  GB_REQUIRE(it != c.vecs.end(), GB_EINVAL, "unknown vector id");
  Level& L = level_with_matrix(c, l);
  auto& lv = it->second;
  if (lv.size() < static_cast<size_t>(c.nlevels))
    lv.resize(c.nlevels);
  if (lv[l].n != static_cast<size_t>(L.ndof())) {
    GB_CUDA(lv[l].alloc(L.ndof()));
    GB_CUDA(cudaMemsetAsync(lv[l].p, 0, L.ndof() * sizeof(double), c.stream));
  }
  return lv[l].p;
}

// --------------------------------------------------------------- reductions

inline void
dot_dev(Context& c, int64_t n, const double* a, const double* b, RedOut ro)
{
  launch(c, k_dot<double, double>, red_blocks(n), kRedThreads, n, a, b,
         c.partials.p, c.ticket.p, ro);
}

inline double
read_scalar(Context& c, const double* dptr)
{
  double h = 0;
  GB_CUDA(cudaMemcpyAsync(&h, dptr, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  GB_CUDA(cudaStreamSynchronize(c.stream));
  return h;
}

// The row-block copy is kept for B = 1 levels of at least kRbMinRows rows
// whose padding to Wr entries per row (a multiple of 4) adds at most a
// quarter to the stored entries; other levels use the SELL kernel only.
constexpr int64_t kRbMinRows = 16384;
constexpr int kRbLanes = 4; // lanes per row (2, 4 and 8 measured; 2 and 4 fastest)


// ---------------------------------------------- defined in gb_setup.cu

void build_patterns(Sell& S, int64_t n, const int64_t* rowptr, const int64_t* col,
                    cudaStream_t st);
void build_sell(Sell& S, int64_t n, const int64_t* rowptr, const int64_t* col,
                const double* val, cudaStream_t st, int B = 1, bool locality = false);
void rows_refresh(Context& c, const Sell& S, bool columns);
void build_rows(Context& c, Sell& S, const int64_t* rowptr);
void host_values(Context& c, Level& L);
void ensure_AT(Context& c, Level& L);
void ensure_pf_scratch(Context& c, int64_t n);
bool direct_on(const Context& c);
void ensure_vanka(Context& c, Level& L);
void ensure_ilu(Context& c, Level& L);
void ensure_work(Context& c);

template<int MODE, int B, class TV, class TX, class TO>
inline void
bspmv(Context& c, const Level& L, const Sell& S, const TX* x, TO* y, const TO* b,
      const TV* dinv, double alpha, const int* yidx, int64_t ystride, TX* xcopy)
{
  const SellView<TV> A = view<TV>(S, sell_vals<TV>(S));
  if (S.pat)
    launch(c, k_bspmv<MODE, B, TV, TX, TO, true>, blocks_for(S.n, kSpmvThreads),
           kSpmvThreads, A, x, y, b, dinv, (const uint8_t*)L.dirmask.p, alpha, yidx,
           ystride, xcopy);
  else
    launch(c, k_bspmv<MODE, B, TV, TX, TO, false>, blocks_for(S.n, kSpmvThreads),
           kSpmvThreads, A, x, y, b, dinv, (const uint8_t*)L.dirmask.p, alpha, yidx,
           ystride, xcopy);
}

template<int MODE, class TV, class TX, class TO>
inline void
spmv(Context& c, const Level& L, const Sell& S, const TX* x, TO* y, const TO* b,
     const TV* dinv, double alpha, const int* yidx = nullptr, int64_t ystride = 0,
     TX* xcopy = nullptr)
{
  switch (S.B) {
    case 1:
      break;
    case 2:
      return bspmv<MODE, 2>(c, L, S, x, y, b, dinv, alpha, yidx, ystride, xcopy);
    case 3:
      return bspmv<MODE, 3>(c, L, S, x, y, b, dinv, alpha, yidx, ystride, xcopy);
    case 4:
      return bspmv<MODE, 4>(c, L, S, x, y, b, dinv, alpha, yidx, ystride, xcopy);
    default:
      throw Error{ GB_EINVAL, "block size must be 1..4" };
  }
  if constexpr (std::is_same<TV, float>::value && std::is_same<TX, float>::value &&
                std::is_same<TO, float>::value &&
                (MODE == kResid || MODE == kResidDir || MODE == kJacobi)) {
    if (S.rb && !yidx) {
      const int nb = blocks_for(int64_t(S.n) * kRbLanes, 256);
      const float a = static_cast<float>(alpha);
      const uint8_t* dm = L.dirmask.p;
      if (S.pat)
        launch(c, k_spmv_rb<MODE, kRbLanes, true>, nb, 256, S.n, S.Wr, (const float*)S.r32.p,
               (const int*)S.ptab.p, (const uint8_t*)S.pid.p, x, y, b, dinv, dm, a);
      else
        launch(c, k_spmv_rb<MODE, kRbLanes, false>, nb, 256, S.n, S.Wr, (const float*)S.r32.p,
               (const int*)S.rcol.p, (const uint8_t*)nullptr, x, y, b, dinv, dm, a);
      return;
    }
  }
  const SellView<TV> A = view<TV>(S, sell_vals<TV>(S));
  const int nb = blocks_for(S.n, kSpmvThreads);
  const uint8_t* dm = L.dirmask.p;
  // FP32 values only: measured on C2, the FP32 cycle gains (1.550 -> 1.544 ms)
  // where the FP64 one, already at 64 registers for its smoother, loses
  const bool small = sizeof(TV) == 4 && S.n < kSpmvSmallRows;
  if (S.pat && small)
    launch(c, k_spmv<MODE, TV, TX, TO, kColPat, true>, nb, kSpmvThreads, A, x, y, b, dinv,
           dm, alpha, yidx, ystride, xcopy);
  else if (S.pat)
    launch(c, k_spmv<MODE, TV, TX, TO, kColPat>, nb, kSpmvThreads, A, x, y, b, dinv, dm,
           alpha, yidx, ystride, xcopy);
  else if (A.c16 && small)
    launch(c, k_spmv<MODE, TV, TX, TO, kColOff16, true>, nb, kSpmvThreads, A, x, y, b, dinv,
           dm, alpha, yidx, ystride, xcopy);
  else if (A.c16)
    launch(c, k_spmv<MODE, TV, TX, TO, kColOff16>, nb, kSpmvThreads, A, x, y, b, dinv, dm,
           alpha, yidx, ystride, xcopy);
  else if (small)
    launch(c, k_spmv<MODE, TV, TX, TO, kColIdx, true>, nb, kSpmvThreads, A, x, y, b, dinv,
           dm, alpha, yidx, ystride, xcopy);
  else
    launch(c, k_spmv<MODE, TV, TX, TO, kColIdx>, nb, kSpmvThreads, A, x, y, b, dinv, dm,
           alpha, yidx, ystride, xcopy);
}

template<class T>
const T* dinv_of(const Level& L);
template<>
inline const double* dinv_of<double>(const Level& L)
{
  return L.dinv64.p;
}
template<>
inline const float* dinv_of<float>(const Level& L)
{
  return L.dinv32.p;
}

// The operator of every solver step on level L: A, or A^T after
// gb_set_operator(ctx, 1) (the dual matrix of StdSolver::AssembleDualMatrix,
// Solver/stdsolver.cc:1815-1834).
inline const Sell&
opA(const Context& c, const Level& L)
{
  return c.transposed ? L.AT : L.A;
}

// ---------------------------------------------- defined in gb_gmres.cu

int gmres_left(Context& c, double* x, const double* b, gb_solve_info* info);
int gmres_flexible(Context& c, double* x, const double* b, int prec, gb_solve_info* info);
// Runs the graph on b (device), result into x (device); info as gb_fgmres.
int fgmres_graph(Context& c, double* x, const double* b, int prec, gb_solve_info* info,
                 bool copy_in = true, bool copy_out = true, double* host_x = nullptr,
                 cudaEvent_t after_copy = nullptr);
// the flexible solver's per-precision buffers (instantiated for double and float)
template<class T>
struct FBufs
{
  T* Z;
  T* zfix;
  T* rhs;
};
template<class T>
FBufs<T> fg_buffers(Context& c, int prec);



// Runs f with the transposed level operators, restoring the setting after.
template<class F>
int
with_transposed(gb_ctx* ctx, F f)
{
  const int saved = ctx->transposed;
  if (!saved) {
    for (auto& L : ctx->L)
      if (L.has_matrix) {
        GB_REQUIRE(L.B == 1, GB_EINVAL,
                   "the transposed solver operators need block size 1");
        gb::ensure_AT(*ctx, L);
      }
    ctx->transposed = 1;
  }
  struct Restore
  {
    gb_ctx* c;
    int v;
    ~Restore() { c->transposed = v; }
  } restore{ ctx, saved };
  return f();
}

#define GB_API_BEGIN                                                           \
  if (!ctx)                                                                    \
    return GB_EINVAL;                                                          \
  try {
#define GB_API_END                                                             \
  }                                                                            \
  catch (const gb::Error& e)                                                   \
  {                                                                            \
    ctx->err = e.msg;                                                          \
    return e.code;                                                             \
  }                                                                            \
  catch (const std::bad_alloc&)                                                \
  {                                                                            \
    ctx->err = "host allocation failed";                                       \
    return GB_ENOMEM;                                                          \
  }                                                                            \
  return GB_OK;

} // namespace gb
