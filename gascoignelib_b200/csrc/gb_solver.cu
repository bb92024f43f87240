// Host orchestration of the B200 linear-solve path and its C-ABI.
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
static std::atomic<long long> g_fail_alloc_countdown{ 0 };

static cudaError_t
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
static cudaError_t
h2d(cudaStream_t st, void* dst, const void* src, size_t bytes)
{
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(st);
  return e;
}

template<class TV>
static SellView<TV>
view(const Sell& S, const TV* val)
{
  return SellView<TV>{ S.n, S.sptr.p, S.pat ? nullptr : S.col.p,
                       S.pat ? S.pid.p : nullptr, S.pat ? S.ptab.p : nullptr,
                       S.W, val, S.sorted ? S.rperm.p : nullptr,
                       !S.pat && S.off16 ? S.c16.p : nullptr };
}

// Rows whose column lists, relative to the row, coincide share one pattern. A
// level uses the compressed form when it has at most 256 patterns.
static void
build_patterns(Sell& S, int64_t n, const int64_t* rowptr, const int64_t* col,
               cudaStream_t st)
{
  S.pat = false;
  int64_t W = 0;
  for (int64_t r = 0; r < n; ++r)
    W = std::max<int64_t>(W, rowptr[r + 1] - rowptr[r]);
  std::map<std::vector<int>, int> dict;
  std::vector<uint8_t> pid(n);
  std::vector<int> key;
  for (int64_t r = 0; r < n; ++r) {
    key.clear();
    for (int64_t k = rowptr[r]; k < rowptr[r + 1]; ++k) {
      int64_t d = col[k] - r;
      if (d < INT32_MIN || d > INT32_MAX)
        return;
      key.push_back(static_cast<int>(d));
    }
    auto it = dict.find(key);
    if (it == dict.end()) {
      if (dict.size() >= 256)
        return;
      it = dict.emplace(key, static_cast<int>(dict.size())).first;
    }
    pid[r] = static_cast<uint8_t>(it->second);
  }
  W = (W + 3) / 4 * 4; // rows of 16 bytes: the row-block SpMV loads 4 offsets at once
  std::vector<int> tab(dict.size() * W, 0);
  for (auto& kv : dict)
    for (size_t j = 0; j < kv.first.size(); ++j)
      tab[kv.second * W + j] = kv.first[j];
  GB_CUDA(S.pid.alloc(n));
  GB_CUDA(S.ptab.alloc(std::max<size_t>(tab.size(), 1)));
  GB_CUDA(cudaMemcpyAsync(S.pid.p, pid.data(), n, cudaMemcpyHostToDevice, st));
  GB_CUDA(cudaMemcpyAsync(S.ptab.p, tab.data(), tab.size() * sizeof(int),
                          cudaMemcpyHostToDevice, st));
  GB_CUDA(cudaStreamSynchronize(st));
  S.npat = static_cast<int>(dict.size());
  S.W = static_cast<int>(W);
  S.pat = true;
}

static void
build_sell(Sell& S, int64_t n, const int64_t* rowptr, const int64_t* col,
           const double* val, cudaStream_t st, int B = 1)
{
  const int B2 = B * B;
  S.B = B;
  S.n = static_cast<int>(n);
  S.nslices = static_cast<int>((n + kSlice - 1) / kSlice);
  S.nnz = rowptr[n];
  // Slot order: rows sorted by length (descending, stable) inside windows of
  // kSortWindow rows when that saves more than a tenth of the padded slots
  // (levels above the single-CTA coarse size only).
  constexpr int64_t kSortWindow = 256;
  std::vector<int> perm(n);
  for (int64_t r = 0; r < n; ++r)
    perm[r] = static_cast<int>(r);
  auto padded = [&](const std::vector<int>& pm) {
    int64_t tot = 0;
    for (int64_t s0 = 0; s0 < n; s0 += kSlice) {
      int64_t w = 0;
      for (int64_t t = s0; t < std::min<int64_t>(n, s0 + kSlice); ++t)
        w = std::max<int64_t>(w, rowptr[pm[t] + 1] - rowptr[pm[t]]);
      tot += w * kSlice;
    }
    return tot;
  };
  S.sorted = false;
  if (n > 1024) {
    std::vector<int> sp(perm);
    for (int64_t w0 = 0; w0 < n; w0 += kSortWindow)
      std::stable_sort(sp.begin() + w0, sp.begin() + std::min<int64_t>(n, w0 + kSortWindow),
                       [&](int a, int b) {
                         return rowptr[a + 1] - rowptr[a] > rowptr[b + 1] - rowptr[b];
                       });
    if (padded(sp) * 10 < padded(perm) * 9) {
      perm.swap(sp);
      S.sorted = true;
    }
  }
  std::vector<int> sptr(S.nslices + 1, 0);
  for (int s = 0; s < S.nslices; ++s) {
    int64_t w = 0;
    for (int l = 0; l < kSlice; ++l) {
      int64_t t = int64_t(s) * kSlice + l;
      if (t < n)
        w = std::max<int64_t>(w, rowptr[perm[t] + 1] - rowptr[perm[t]]);
    }
    int64_t next = int64_t(sptr[s]) + w * kSlice;
    GB_REQUIRE(next < (int64_t(1) << 31), GB_EINVAL,
               "matrix too large for 32-bit SELL offsets");
    sptr[s + 1] = static_cast<int>(next);
  }
  S.entries = sptr[S.nslices];
  std::vector<int> c(S.entries);
  std::vector<double> v(S.entries * B2, 0.0);
  std::vector<float> v32(S.entries * B2, 0.0f);
  for (int s = 0; s < S.nslices; ++s) {
    int w = (sptr[s + 1] - sptr[s]) / kSlice;
    for (int l = 0; l < kSlice; ++l) {
      const int64_t t = int64_t(s) * kSlice + l;
      const int64_t r = t < n ? perm[t] : t;
      int64_t len = t < n ? rowptr[r + 1] - rowptr[r] : 0;
      for (int j = 0; j < w; ++j) {
        int64_t e = sptr[s] + int64_t(j) * kSlice + l;
        if (j < len) {
          int64_t cc = col[rowptr[r] + j];
          GB_REQUIRE(cc >= 0 && cc < n, GB_EINVAL, "column index out of range");
          c[e] = static_cast<int>(cc);
          for (int q = 0; q < B2; ++q) {
            const int64_t ev = (sptr[s] + int64_t(j) * kSlice) * B2 + int64_t(q) * kSlice + l;
            v[ev] = val[(rowptr[r] + j) * B2 + q];
            v32[ev] = static_cast<float>(v[ev]);
          }
        } else {
          c[e] = r < n ? static_cast<int>(r) : 0;
        }
      }
    }
  }
  GB_CUDA(S.sptr.alloc(sptr.size()));
  GB_CUDA(S.col.alloc(std::max<size_t>(c.size(), 1)));
  GB_CUDA(S.v64.alloc(std::max<size_t>(v.size(), 1)));
  GB_CUDA(S.v32.alloc(std::max<size_t>(v32.size(), 1)));
  GB_CUDA(cudaMemcpyAsync(S.sptr.p, sptr.data(), sptr.size() * sizeof(int),
                          cudaMemcpyHostToDevice, st));
  if (S.entries) {
    GB_CUDA(cudaMemcpyAsync(S.col.p, c.data(), c.size() * sizeof(int),
                            cudaMemcpyHostToDevice, st));
    GB_CUDA(cudaMemcpyAsync(S.v64.p, v.data(), v.size() * sizeof(double),
                            cudaMemcpyHostToDevice, st));
    GB_CUDA(cudaMemcpyAsync(S.v32.p, v32.data(), v32.size() * sizeof(float),
                            cudaMemcpyHostToDevice, st));
  }
  if (S.sorted) {
    GB_CUDA(S.rperm.alloc(n));
    GB_CUDA(cudaMemcpyAsync(S.rperm.p, perm.data(), n * sizeof(int), cudaMemcpyHostToDevice,
                            st));
  }
  // host vectors must outlive the async copies
  GB_CUDA(cudaStreamSynchronize(st));
  S.h_sptr = sptr;
  S.h_perm = perm;
  build_patterns(S, n, rowptr, col, st);
  S.off16 = false;
  if (!S.pat && S.entries) {
    std::vector<int16_t> h(S.entries, 0);
    bool fits = true;
    for (int s = 0; s < S.nslices && fits; ++s) {
      const int w = (sptr[s + 1] - sptr[s]) / kSlice;
      for (int l = 0; l < kSlice && fits; ++l) {
        const int64_t t = int64_t(s) * kSlice + l;
        if (t >= n)
          continue; // padding lanes exit before reading
        const int64_t r = perm[t];
        for (int j = 0; j < w; ++j) {
          const int64_t e = sptr[s] + int64_t(j) * kSlice + l;
          const int64_t d = int64_t(c[e]) - r;
          if (d < -32768 || d > 32767) {
            fits = false;
            break;
          }
          h[e] = static_cast<int16_t>(d);
        }
      }
    }
    if (fits) {
      GB_CUDA(S.c16.alloc(h.size()));
      GB_CUDA(h2d(st, S.c16.p, h.data(), h.size() * sizeof(int16_t)));
      S.off16 = true;
    }
  }
}

template<class T>
static const T* sell_vals(const Sell& S);
template<>
const double* sell_vals<double>(const Sell& S)
{
  return S.v64.p;
}
template<>
const float* sell_vals<float>(const Sell& S)
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

static void
check_launch(Context& c)
{
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    throw Error{ GB_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e) };
}

// Per-kernel device timing (gb_set_timing): an event pair around each launch
// outside graph capture, resolved by kt_flush.
static void
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

static void
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

static void
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
static void
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
static void
launch(Context& c, void (*kern)(KArgs...), int grid, int block, Args... args)
{
  launch_smem(c, kern, grid, block, 0, args...);
}

static int
blocks_for(int64_t n, int threads)
{
  return static_cast<int>((n + threads - 1) / threads);
}

static int
red_blocks(int64_t n)
{
  int64_t b = (n + kRedThreads * 8 - 1) / (kRedThreads * 8);
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(b, kMaxRedBlocks)));
}

static int
stream_blocks(int64_t n)
{
  int64_t b = (n + 255) / 256;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(b, 148 * 16)));
}

static Level&
level(Context& c, int l)
{
  GB_REQUIRE(l >= 0 && l < c.nlevels, GB_EINVAL, "level out of range");
  return c.L[l];
}

static Level&
level_with_matrix(Context& c, int l)
{
  Level& L = level(c, l);
  GB_REQUIRE(L.has_matrix, GB_ESTATE, "no matrix on this level");
  return L;
}

static double*
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

static void
dot_dev(Context& c, int64_t n, const double* a, const double* b, RedOut ro)
{
  launch(c, k_dot<double, double>, red_blocks(n), kRedThreads, n, a, b,
         c.partials.p, c.ticket.p, ro);
}

static double
read_scalar(Context& c, const double* dptr)
{
  double h = 0;
  GB_CUDA(cudaMemcpyAsync(&h, dptr, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  GB_CUDA(cudaStreamSynchronize(c.stream));
  return h;
}

// ----------------------------------------------------------------- SpMV

// The row-major FP32 values of S for the row-block SpMV, from its SELL
// values (again after every change of those on the device); with
// `columns`, also the columns of a level without patterns.
static void
rows_refresh(Context& c, const Sell& S, bool columns)
{
  if (!S.rb)
    return;
  const int64_t total = int64_t(S.n) * S.Wr;
  launch(c, k_sell_to_rows, static_cast<int>(std::min<int64_t>((total + 255) / 256, 148 * 16)),
         256, S.n, S.Wr, (const int*)S.sptr.p, (const int*)(S.sorted ? S.rslot.p : nullptr),
         (const float*)S.v32.p, (const int*)S.col.p, S.r32.p,
         columns && !S.pat ? S.rcol.p : (int*)nullptr);
}

// The row-block copy is kept for B = 1 levels of at least kRbMinRows rows
// whose padding to Wr entries per row (a multiple of 4) adds at most a
// quarter to the stored entries; other levels use the SELL kernel only.
constexpr int64_t kRbMinRows = 16384;
constexpr int kRbLanes = 4; // lanes per row (2, 4 and 8 measured; 2 and 4 fastest)

static void
build_rows(Context& c, Sell& S, const int64_t* rowptr)
{
  S.rb = false;
  const int64_t n = S.n;
  if (S.B != 1 || n < kRbMinRows || !c.rb_on)
    return;
  int64_t W = 0;
  for (int64_t r = 0; r < n; ++r)
    W = std::max<int64_t>(W, rowptr[r + 1] - rowptr[r]);
  const int64_t Wr = S.pat ? S.W : (W + 3) / 4 * 4;
  if (Wr * n * 4 > S.nnz * 5 || Wr * n >= (int64_t(1) << 31))
    return;
  GB_CUDA(S.r32.alloc(size_t(n * Wr)));
  if (!S.pat)
    GB_CUDA(S.rcol.alloc(size_t(n * Wr)));
  if (S.sorted) {
    std::vector<int> slot(n);
    for (int64_t t = 0; t < n; ++t)
      slot[S.h_perm[t]] = static_cast<int>(t);
    GB_CUDA(S.rslot.alloc(n));
    GB_CUDA(h2d(c.stream, S.rslot.p, slot.data(), n * sizeof(int)));
  }
  S.Wr = static_cast<int>(Wr);
  S.rb = true;
  rows_refresh(c, S, true);
}

template<int MODE, int B, class TV, class TX, class TO>
static void
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
static void
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
static const T* dinv_of(const Level& L);
template<>
const double* dinv_of<double>(const Level& L)
{
  return L.dinv64.p;
}
template<>
const float* dinv_of<float>(const Level& L)
{
  return L.dinv32.p;
}

// The operator of every solver step on level L: A, or A^T after
// gb_set_operator(ctx, 1) (the dual matrix of StdSolver::AssembleDualMatrix,
// Solver/stdsolver.cc:1815-1834).
static const Sell&
opA(const Context& c, const Level& L)
{
  return c.transposed ? L.AT : L.A;
}

// A^T of the uploaded (Dirichlet-modified) level matrix. A structurally
// symmetric matrix keeps its own sparsity pattern and row order, with the
// values swapped in place as SparseBlockMatrix::transpose does
// (LinAlg/sparseblockmatrix.xx:478-491); otherwise rows of A^T list the
// columns of A in ascending order. Strong Dirichlet rows and columns of the
// uploaded matrix are both identity, so A^T is the reference's dual matrix
// (transpose, then DirichletMatrixOnlyRow) wherever it meets a vector that is
// zero on the Dirichlet dofs, which every vector of the dual solve is.
// The host copy of a level's values after a device assembly (gb_assemble),
// for the set-up steps that read it (transpose, Vanka factors, direct coarse
// inverse): the FP64 SELL values read back and put in stencil order.
static void
host_values(Context& c, Level& L)
{
  if (!L.h_val_stale)
    return;
  const Sell& A = L.A;
  std::vector<double> v(A.entries);
  std::vector<int> sptr(A.nslices + 1), perm;
  GB_CUDA(cudaStreamSynchronize(c.stream));
  GB_CUDA(cudaMemcpy(v.data(), A.v64.p, v.size() * sizeof(double), cudaMemcpyDeviceToHost));
  GB_CUDA(cudaMemcpy(sptr.data(), A.sptr.p, sptr.size() * sizeof(int), cudaMemcpyDeviceToHost));
  if (A.sorted) {
    perm.resize(L.n);
    GB_CUDA(cudaMemcpy(perm.data(), A.rperm.p, L.n * sizeof(int), cudaMemcpyDeviceToHost));
  }
  for (int64_t t = 0; t < L.n; ++t) {
    const int64_t r = A.sorted ? perm[t] : t;
    const int64_t s0 = sptr[t / kSlice] + t % kSlice;
    for (int64_t k = L.h_rowptr[r]; k < L.h_rowptr[r + 1]; ++k)
      L.h_val[k] = v[s0 + (k - L.h_rowptr[r]) * kSlice];
  }
  L.h_val_stale = false;
}

// SELL position of every stored entry k (CSR order of rowptr) of S.
static std::vector<int>
sell_positions(Context& c, const Sell& S, const int64_t* rowptr, int64_t n)
{
  std::vector<int> sptr(S.nslices + 1), perm(n), slot(n), pos(rowptr[n]);
  GB_CUDA(cudaStreamSynchronize(c.stream));
  GB_CUDA(cudaMemcpy(sptr.data(), S.sptr.p, sptr.size() * sizeof(int), cudaMemcpyDeviceToHost));
  if (S.sorted)
    GB_CUDA(cudaMemcpy(perm.data(), S.rperm.p, n * sizeof(int), cudaMemcpyDeviceToHost));
  else
    for (int64_t t = 0; t < n; ++t)
      perm[t] = static_cast<int>(t);
  for (int64_t t = 0; t < n; ++t)
    slot[perm[t]] = static_cast<int>(t);
  for (int64_t r = 0; r < n; ++r) {
    const int64_t t = slot[r];
    for (int64_t k = rowptr[r]; k < rowptr[r + 1]; ++k)
      pos[k] = static_cast<int>(sptr[t / kSlice] + (k - rowptr[r]) * kSlice + t % kSlice);
  }
  return pos;
}

static void
ensure_AT(Context& c, Level& L)
{
  if (L.has_AT)
    return;
  host_values(c, L);
  const int B = L.B, B2 = B * B;
  const int64_t n = L.n, nnz = L.h_rowptr[n];
  std::vector<int64_t> tp(n + 1, 0), tc(nnz);
  std::vector<double> tv(nnz * B2);
  std::vector<int64_t> srcidx(nnz);
  // block (j, i) of A, transposed, as block (i, j) of A^T
  auto put = [&](int64_t dst, int64_t src) {
    srcidx[dst] = src;
    for (int r = 0; r < B; ++r)
      for (int q = 0; q < B; ++q)
        tv[dst * B2 + r * B + q] = L.h_val[src * B2 + q * B + r];
  };
  bool symmetric = true;
  for (int64_t i = 0; i < n && symmetric; ++i)
    for (int64_t k = L.h_rowptr[i]; k < L.h_rowptr[i + 1]; ++k) {
      const int64_t j = L.h_col[k];
      const int64_t* b = L.h_col.data() + L.h_rowptr[j];
      const int64_t* e = L.h_col.data() + L.h_rowptr[j + 1];
      const int64_t* f = std::find(b, e, i);
      if (f == e) {
        symmetric = false;
        break;
      }
      put(k, L.h_rowptr[j] + (f - b));
    }
  if (symmetric) {
    tp = L.h_rowptr;
    tc = L.h_col;
  } else {
    for (int64_t k = 0; k < nnz; ++k)
      tp[L.h_col[k] + 1]++;
    for (int64_t i = 0; i < n; ++i)
      tp[i + 1] += tp[i];
    std::vector<int64_t> pos(tp.begin(), tp.end() - 1);
    for (int64_t i = 0; i < n; ++i)
      for (int64_t k = L.h_rowptr[i]; k < L.h_rowptr[i + 1]; ++k) {
        int64_t q = pos[L.h_col[k]]++;
        tc[q] = i;
        put(q, k);
      }
  }
  GB_CUDA(cudaStreamSynchronize(c.stream));
  build_sell(L.AT, n, tp.data(), tc.data(), tv.data(), c.stream, B);
  build_rows(c, L.AT, tp.data());
  L.has_AT = true;
  if (B == 1 && L.mesh_ncells > 0) { // device-assembled level: keep A^T current on the GPU
    const std::vector<int> pa = sell_positions(c, L.A, L.h_rowptr.data(), n);
    const std::vector<int> pt = sell_positions(c, L.AT, tp.data(), n);
    std::vector<int> map(L.AT.entries, -1);
    for (int64_t q = 0; q < nnz; ++q)
      map[pt[q]] = pa[srcidx[q]];
    GB_CUDA(L.at_map.alloc(map.size()));
    GB_CUDA(h2d(c.stream, L.at_map.p, map.data(), map.size() * sizeof(int)));
  } else {
    L.at_map.release();
  }
}

// ---------------------------------------------------------- level set-up

// Per-block sums of the filter reductions fused into the residual and update
// kernels (grid of blocks_for(n, 256) blocks on a level of n nodes).
static void
ensure_pf_scratch(Context& c, int64_t n)
{
  const size_t need = static_cast<size_t>((n + 255) / 256 + 1);
  if (c.pfpart.n < need)
    GB_CUDA(c.pfpart.alloc(need));
  if (c.pfticket.n < 1) {
    GB_CUDA(c.pfticket.alloc(1));
    GB_CUDA(cudaMemsetAsync(c.pfticket.p, 0, sizeof(unsigned), c.stream));
  }
}

// VankaSmoother::ConstructStructure + copy_entries (LinAlg/vankasmoother.cc:
// 7-113) for one level: each patch's matrix (the level matrix's entries whose
// row and column nodes both lie in the patch; node-major, components inside)
// factorised on the host with row partial pivoting in the reference's
// operation order (first row of largest |a_ik| as pivot, column divided by the
// pivot, trailing entries updated k by k). The device applies the inverse,
// formed from these factors column by column (the LU solves of the unit
// vectors), so a local solve is a dense product without dependency chains; it
// agrees with the reference's LU solves to rounding. Uploaded in FP64 and FP32,
// transposed per patch, with the patch node lists and, per node, the (patch,
// local node) pairs in ascending patch order for the averaging gather.
static void
ensure_vanka_host(Context& c, Level& L);

// The patch structure of a level (once per matrix structure and patch list):
// patch node lists, the node -> (patch, slot) map of the averaging gather, and
// per node pair of a patch the offset of its block in the SELL values (-1
// where the matrix has no block), with the factor and solution buffers.
static void
vanka_structure(Context& c, Level& L)
{
  const int B = L.B, npp = L.npp, M = npp * B, B2 = B * B;
  const int64_t np = L.npatch;
  std::vector<int> pn(size_t(np) * npp), map(size_t(np) * npp * npp, -1);
  std::vector<int> slot_of(L.n);
  const Sell& S = L.A;
  for (int64_t t = 0; t < L.n; ++t)
    slot_of[S.h_perm[t]] = static_cast<int>(t);
  for (int64_t p = 0; p < np; ++p) {
    const int64_t* nodes = L.h_patches.data() + p * npp;
    for (int r = 0; r < npp; ++r) {
      const int64_t row = nodes[r];
      const int t = slot_of[row], sl = t / kSlice, lane = t % kSlice;
      for (int64_t pos = L.h_rowptr[row]; pos < L.h_rowptr[row + 1]; ++pos) {
        int q = -1;
        for (int k = 0; k < npp; ++k)
          if (nodes[k] == L.h_col[pos]) {
            q = k;
            break;
          }
        if (q < 0)
          continue;
        const int64_t j = pos - L.h_rowptr[row];
        const int64_t base = (int64_t(S.h_sptr[sl]) + j * kSlice) * B2 + lane;
        GB_REQUIRE(base < (int64_t(1) << 31), GB_EINVAL, "Vanka gather offset too large");
        map[(size_t(p) * npp + r) * npp + q] = static_cast<int>(base);
      }
      pn[size_t(r) * np + p] = static_cast<int>(row);
    }
  }
  // node -> (patch, local node), patches ascending
  std::vector<int> nptr(L.n + 1, 0), ent(size_t(np) * npp);
  for (size_t k = 0; k < L.h_patches.size(); ++k)
    nptr[L.h_patches[k] + 1]++;
  for (int64_t i = 0; i < L.n; ++i) {
    GB_REQUIRE(nptr[i + 1] > 0, GB_EINVAL, "a node lies in no Vanka patch");
    nptr[i + 1] += nptr[i];
  }
  std::vector<int> fill(nptr.begin(), nptr.end() - 1);
  for (int64_t p = 0; p < np; ++p)
    for (int r = 0; r < npp; ++r)
      ent[fill[L.h_patches[p * npp + r]]++] = static_cast<int>(p * 32 + r);
  GB_CUDA(cudaStreamSynchronize(c.stream));
  GB_CUDA(L.vk_inv64.alloc(size_t(np) * M * M));
  GB_CUDA(L.vk_inv32.alloc(size_t(np) * M * M));
  GB_CUDA(L.vk_pn.alloc(pn.size()));
  GB_CUDA(L.vk_map.alloc(map.size()));
  GB_CUDA(L.vk_nptr.alloc(nptr.size()));
  GB_CUDA(L.vk_ent.alloc(ent.size()));
  GB_CUDA(L.vk_out64.alloc(size_t(np) * M));
  GB_CUDA(L.vk_out32.alloc(size_t(np) * M));
  GB_CUDA(h2d(c.stream, L.vk_pn.p, pn.data(), pn.size() * sizeof(int)));
  GB_CUDA(h2d(c.stream, L.vk_map.p, map.data(), map.size() * sizeof(int)));
  GB_CUDA(h2d(c.stream, L.vk_nptr.p, nptr.data(), nptr.size() * sizeof(int)));
  GB_CUDA(h2d(c.stream, L.vk_ent.p, ent.data(), ent.size() * sizeof(int)));
  L.vk_M = M;
  L.vk_struct = true;
}

// The patches' inverses from the level's current values, on the device
// (k_vanka_factor); GB_VANKA_HOST=1 forms them on the host instead (the same
// arithmetic, for comparison).
static void
ensure_vanka(Context& c, Level& L)
{
  if (L.vk_ready)
    return;
  GB_REQUIRE(L.npatch > 0, GB_ESTATE, "Vanka needs the patches of every level "
                                      "(gb_level_set_patches)");
  const int M = L.npp * L.B;
  GB_REQUIRE(M <= kVankaMaxM && L.npp <= 32, GB_EINVAL, "Vanka patch too large");
  if (c.vanka_host)
    return ensure_vanka_host(c, L);
  if (!L.vk_struct)
    vanka_structure(c, L);
  const int smem = M * (M + 1) * int(sizeof(double)) + M * int(sizeof(int));
  GB_CUDA(cudaFuncSetAttribute(k_vanka_factor, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               smem));
  const int threads = std::min(kVankaFactorThreads, std::max(32, (M + 31) / 32 * 32));
  launch_smem(c, k_vanka_factor, L.npatch, threads, smem, L.npatch, L.npp, L.B, M,
              (const int*)L.vk_map.p, (const double*)L.A.v64.p, L.vk_inv64.p, L.vk_inv32.p);
  L.vk_ready = true;
}

static void
ensure_vanka_host(Context& c, Level& L)
{
  if (L.vk_ready)
    return;
  host_values(c, L);
  GB_REQUIRE(L.npatch > 0, GB_ESTATE, "Vanka needs the patches of every level "
                                      "(gb_level_set_patches)");
  const int B = L.B, npp = L.npp, M = npp * B, B2 = B * B;
  GB_REQUIRE(M <= kVankaMaxM && npp <= 32, GB_EINVAL, "Vanka patch too large");
  const int64_t np = L.npatch;
  std::vector<double> inv(size_t(np) * M * M);
  std::vector<int> pn(size_t(np) * npp);
  std::vector<double> a(size_t(M) * M), x(M);
  std::vector<int> pv(M);
  for (int64_t p = 0; p < np; ++p) {
    const int64_t* nodes = L.h_patches.data() + p * npp;
    std::fill(a.begin(), a.end(), 0.0);
    for (int r = 0; r < npp; ++r) {
      const int64_t row = nodes[r];
      for (int64_t pos = L.h_rowptr[row]; pos < L.h_rowptr[row + 1]; ++pos) {
        int cl = -1;
        for (int q = 0; q < npp; ++q)
          if (nodes[q] == L.h_col[pos]) {
            cl = q;
            break;
          }
        if (cl < 0)
          continue;
        for (int cr = 0; cr < B; ++cr)
          for (int cc = 0; cc < B; ++cc)
            a[size_t(B * r + cr) * M + B * cl + cc] = L.h_val[pos * B2 + cr * B + cc];
      }
    }
    for (int i = 0; i < M; ++i)
      pv[i] = i;
    for (int k = 0; k < M; ++k) {
      int piv = k;
      double best = std::fabs(a[size_t(k) * M + k]);
      for (int i = k + 1; i < M; ++i)
        if (std::fabs(a[size_t(i) * M + k]) > best) {
          best = std::fabs(a[size_t(i) * M + k]);
          piv = i;
        }
      if (piv != k) {
        for (int j = 0; j < M; ++j)
          std::swap(a[size_t(k) * M + j], a[size_t(piv) * M + j]);
        std::swap(pv[k], pv[piv]);
      }
      if (a[size_t(k) * M + k] != 0)
        for (int i = k + 1; i < M; ++i)
          a[size_t(i) * M + k] /= a[size_t(k) * M + k];
      for (int j = k + 1; j < M; ++j)
        for (int i = k + 1; i < M; ++i)
          a[size_t(i) * M + j] -= a[size_t(i) * M + k] * a[size_t(k) * M + j];
    }
    for (int j = 0; j < M; ++j) { // column j of the inverse: LU x = P e_j
      for (int i = 0; i < M; ++i)
        x[i] = pv[i] == j ? 1.0 : 0.0;
      for (int i = 1; i < M; ++i) {
        double sacc = x[i];
        for (int q = 0; q < i; ++q)
          sacc -= a[size_t(i) * M + q] * x[q];
        x[i] = sacc;
      }
      for (int i = M - 1; i >= 0; --i) {
        double sacc = x[i];
        for (int q = i + 1; q < M; ++q)
          sacc -= a[size_t(i) * M + q] * x[q];
        x[i] = sacc / a[size_t(i) * M + i];
      }
      for (int i = 0; i < M; ++i)
        inv[size_t(p) * M * M + size_t(j) * M + i] = x[i];
    }
    for (int r = 0; r < npp; ++r)
      pn[size_t(r) * np + p] = static_cast<int>(nodes[r]);
  }
  // node -> (patch, local node), patches ascending
  std::vector<int> nptr(L.n + 1, 0), ent(size_t(np) * npp);
  for (size_t k = 0; k < L.h_patches.size(); ++k)
    nptr[L.h_patches[k] + 1]++;
  for (int64_t i = 0; i < L.n; ++i) {
    GB_REQUIRE(nptr[i + 1] > 0, GB_EINVAL, "a node lies in no Vanka patch");
    nptr[i + 1] += nptr[i];
  }
  std::vector<int> fill(nptr.begin(), nptr.end() - 1);
  for (int64_t p = 0; p < np; ++p)
    for (int r = 0; r < npp; ++r)
      ent[fill[L.h_patches[p * npp + r]]++] = static_cast<int>(p * 32 + r);
  std::vector<float> inv32(inv.begin(), inv.end());
  GB_CUDA(cudaStreamSynchronize(c.stream));
  GB_CUDA(L.vk_inv64.alloc(inv.size()));
  GB_CUDA(L.vk_inv32.alloc(inv.size()));
  GB_CUDA(L.vk_pn.alloc(pn.size()));
  GB_CUDA(L.vk_nptr.alloc(nptr.size()));
  GB_CUDA(L.vk_ent.alloc(ent.size()));
  GB_CUDA(L.vk_out64.alloc(size_t(np) * M));
  GB_CUDA(L.vk_out32.alloc(size_t(np) * M));
  GB_CUDA(h2d(c.stream, L.vk_inv64.p, inv.data(), inv.size() * sizeof(double)));
  GB_CUDA(h2d(c.stream, L.vk_inv32.p, inv32.data(), inv32.size() * sizeof(float)));
  GB_CUDA(h2d(c.stream, L.vk_pn.p, pn.data(), pn.size() * sizeof(int)));
  GB_CUDA(h2d(c.stream, L.vk_nptr.p, nptr.data(), nptr.size() * sizeof(int)));
  GB_CUDA(h2d(c.stream, L.vk_ent.p, ent.data(), ent.size() * sizeof(int)));
  L.vk_M = M;
  L.vk_ready = true;
  L.vk_struct = false; // the device path rebuilds its gather map
}

// The exact coarsest-level solve of StdSolver::smooth_exact on a direct level
// (UmfIlu::Solve when the level has fewer than ndirect nodes, Solver/
// stdsolver.cc:1003-1025 and :218-222): the inverse of level 0's operator (A or
// its transpose), formed once per assembly in FP64 by Gauss-Jordan elimination
// with partial pivoting on the host and applied as one GEMV per coarse solve.
static bool
direct_on(const Context& c)
{
  return c.params.ndirect > 0 && c.nlevels > 0 && c.L[0].n < c.params.ndirect;
}

static void
ensure_direct(Context& c)
{
  const int t = c.transposed ? 1 : 0;
  if (!direct_on(c) || c.dir_ready[t])
    return;
  Level& L = c.L[0];
  host_values(c, L);
  const int B = L.B, B2 = B * B;
  const int64_t N = L.ndof();
  GB_REQUIRE(N <= 8192, GB_EINVAL, "direct coarse solve: level 0 has more than 8192 dofs");
  // augmented [A | I] reduced to [I | A^-1], rows swapped for the pivots
  std::vector<double> a(size_t(N) * N, 0.0), inv(size_t(N) * N, 0.0);
  for (int64_t i = 0; i < L.n; ++i)
    for (int64_t k = L.h_rowptr[i]; k < L.h_rowptr[i + 1]; ++k)
      for (int r = 0; r < B; ++r)
        for (int q = 0; q < B; ++q)
          a[size_t(i * B + r) * N + L.h_col[k] * B + q] = L.h_val[k * B2 + r * B + q];
  double anorm = 0.0;
  for (double v : a)
    anorm = std::max(anorm, std::fabs(v));
  for (int64_t i = 0; i < N; ++i)
    inv[size_t(i) * N + i] = 1.0;
  for (int64_t k = 0; k < N; ++k) {
    int64_t piv = k;
    double best = std::fabs(a[size_t(k) * N + k]);
    for (int64_t i = k + 1; i < N; ++i)
      if (std::fabs(a[size_t(i) * N + k]) > best) {
        best = std::fabs(a[size_t(i) * N + k]);
        piv = i;
      }
    // a pivot at roundoff level: singular (e.g. a Stokes level whose pressure
    // is fixed only up to a constant)
    GB_REQUIRE(best > 1e-13 * anorm, GB_EINVAL,
               "direct coarse solve: level 0 matrix is singular");
    if (piv != k) {
      std::swap_ranges(a.begin() + size_t(k) * N, a.begin() + size_t(k + 1) * N,
                       a.begin() + size_t(piv) * N);
      std::swap_ranges(inv.begin() + size_t(k) * N, inv.begin() + size_t(k + 1) * N,
                       inv.begin() + size_t(piv) * N);
    }
    const double d = 1.0 / a[size_t(k) * N + k];
    double* ak = a.data() + size_t(k) * N;
    double* ik = inv.data() + size_t(k) * N;
    for (int64_t j = 0; j < N; ++j) {
      ak[j] *= d;
      ik[j] *= d;
    }
    for (int64_t i = 0; i < N; ++i) {
      if (i == k)
        continue;
      double* ai = a.data() + size_t(i) * N;
      const double f = ai[k];
      if (f == 0.0)
        continue;
      double* ii = inv.data() + size_t(i) * N;
      for (int64_t j = k; j < N; ++j)
        ai[j] -= f * ak[j];
      for (int64_t j = 0; j < N; ++j)
        ii[j] -= f * ik[j];
    }
  }
  if (t) { // (A^T)^-1 = (A^-1)^T
    for (int64_t i = 0; i < N; ++i)
      for (int64_t j = i + 1; j < N; ++j)
        std::swap(inv[size_t(i) * N + j], inv[size_t(j) * N + i]);
  }
  GB_CUDA(cudaStreamSynchronize(c.stream));
  GB_CUDA(c.dir_inv[t].alloc(size_t(N) * N));
  GB_CUDA(h2d(c.stream, c.dir_inv[t].p, inv.data(), inv.size() * sizeof(double)));
  c.dir_ready[t] = true;
}

// SparseBlockIlu on the host (ConstructStructure with the identity order,
// copy_entries, compute_ilu: LinAlg/sparseblockilu.xx:72-135, 140-175,
// 246-276), the block products in FMatrixBlock's order (operator*=,
// LinAlg/fmatrixblock.h:174-190; submult, :73-93) and the diagonal blocks by
// gauss_jordan; then the dependency levels of both triangular solves.
template<int B>
static void
ilu_factor(std::vector<int>& ptr, std::vector<int>& col, std::vector<int>& diag,
           std::vector<double>& v, int64_t n)
{
  constexpr int B2 = B * B;
  double tmp[B2];
  for (int64_t i = 0; i < n; ++i) {
    for (int pk = ptr[i]; pk < diag[i]; ++pk) {
      const int k = col[pk];
      double* a = v.data() + size_t(pk) * B2;
      const double* dk = v.data() + size_t(diag[k]) * B2;
      for (int q = 0; q < B2; ++q)
        tmp[q] = a[q];
      for (int r = 0; r < B; ++r) // a(i,k) *= a(k,k)
        for (int cc = 0; cc < B; ++cc) {
          double acc = 0.0;
          for (int t = 0; t < B; ++t)
            acc = rn_add(acc, rn_mul(tmp[r * B + t], dk[t * B + cc]));
          a[r * B + cc] = acc;
        }
      for (int pj = diag[k] + 1; pj < ptr[k + 1]; ++pj) {
        const int j = col[pj];
        for (int ph = ptr[i]; ph < ptr[i + 1]; ++ph) {
          if (col[ph] != j)
            continue;
          double* h = v.data() + size_t(ph) * B2;
          const double* cj = v.data() + size_t(pj) * B2;
          for (int r = 0; r < B; ++r) // a(i,j) -= a(i,k) a(k,j)
            for (int cc = 0; cc < B; ++cc)
              for (int t = 0; t < B; ++t)
                h[r * B + cc] = rn_sub(h[r * B + cc], rn_mul(a[r * B + t], cj[t * B + cc]));
          break;
        }
      }
    }
    gauss_jordan<B>(v.data() + size_t(diag[i]) * B2);
  }
}

// The ILU's row-sorted layout, dependency levels and gather map (once per
// matrix structure): columns ascending per row (SparseBlockIlu's order), the
// forward and backward levels of the substitutions (the forward ones are also
// the factorisation's), and per entry the offset of its block in the SELL
// values.
// The dependency levels of both substitutions on the device and as launches:
// a run of consecutive levels of at most ilu_cta_rows rows each goes to one
// single-CTA launch (k_ilu_levels, a block barrier between levels instead of
// a launch), a wider level to a launch of its own (k_ilu_level).
static void
ilu_levels_upload(Context& c, Level& L)
{
  auto segments = [&](const std::vector<int>& off) {
    std::vector<Level::IluSeg> seg;
    const int nlev = static_cast<int>(off.size()) - 1;
    for (int lv = 0; lv < nlev;) {
      if (off[lv + 1] - off[lv] > c.ilu_cta_rows) {
        seg.push_back({ lv, lv + 1, false });
        ++lv;
        continue;
      }
      int e = lv;
      while (e < nlev && off[e + 1] - off[e] <= c.ilu_cta_rows)
        ++e;
      seg.push_back({ lv, e, true });
      lv = e;
    }
    return seg;
  };
  L.ilu_lseg = segments(L.ilu_lptr);
  L.ilu_useg = segments(L.ilu_uptr);
  GB_CUDA(L.ilu_lptr_d.alloc(L.ilu_lptr.size()));
  GB_CUDA(L.ilu_uptr_d.alloc(L.ilu_uptr.size()));
  GB_CUDA(h2d(c.stream, L.ilu_lptr_d.p, L.ilu_lptr.data(), L.ilu_lptr.size() * sizeof(int)));
  GB_CUDA(h2d(c.stream, L.ilu_uptr_d.p, L.ilu_uptr.data(), L.ilu_uptr.size() * sizeof(int)));
}

static void
ilu_structure(Context& c, Level& L)
{
  const int B = L.B, B2 = B * B;
  const int64_t n = L.n, nnz = L.h_rowptr[n];
  std::vector<int> ptr(n + 1), col(nnz), diag(n, -1), map(nnz);
  std::vector<int> slot_of(n);
  const Sell& S = L.A;
  for (int64_t t = 0; t < n; ++t)
    slot_of[S.h_perm[t]] = static_cast<int>(t);
  std::vector<int64_t> idx;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t b = L.h_rowptr[i], e = L.h_rowptr[i + 1];
    ptr[i] = static_cast<int>(b);
    idx.resize(e - b);
    for (int64_t k = b; k < e; ++k)
      idx[k - b] = k;
    std::stable_sort(idx.begin(), idx.end(),
                     [&](int64_t x, int64_t y) { return L.h_col[x] < L.h_col[y]; });
    const int t = slot_of[i], sl = t / kSlice, lane = t % kSlice;
    for (int64_t q = 0; q < e - b; ++q) {
      col[b + q] = static_cast<int>(L.h_col[idx[q]]);
      if (col[b + q] == i)
        diag[i] = static_cast<int>(b + q);
      const int64_t j = idx[q] - b; // the entry's place in the row: its SELL column
      const int64_t base = (int64_t(S.h_sptr[sl]) + j * kSlice) * B2 + lane;
      GB_REQUIRE(base < (int64_t(1) << 31), GB_EINVAL, "ILU gather offset too large");
      map[b + q] = static_cast<int>(base);
    }
    GB_REQUIRE(diag[i] >= 0, GB_EINVAL, "ILU: a row without its diagonal");
  }
  ptr[n] = static_cast<int>(nnz);
  std::vector<int> lev(n, 0);
  int nl = 0;
  for (int64_t i = 0; i < n; ++i) {
    int m = 0;
    for (int p = ptr[i]; p < diag[i]; ++p)
      m = std::max(m, lev[col[p]] + 1);
    lev[i] = m;
    nl = std::max(nl, m + 1);
  }
  auto group = [&](const std::vector<int>& lv, int nlev, std::vector<int>& off,
                   std::vector<int>& rows) {
    off.assign(nlev + 1, 0);
    for (int64_t i = 0; i < n; ++i)
      off[lv[i] + 1]++;
    for (int q = 0; q < nlev; ++q)
      off[q + 1] += off[q];
    rows.resize(n);
    std::vector<int> fill(off.begin(), off.end() - 1);
    for (int64_t i = 0; i < n; ++i)
      rows[fill[lv[i]]++] = static_cast<int>(i);
  };
  std::vector<int> lrows, urows;
  group(lev, nl, L.ilu_lptr, lrows);
  int nu = 0;
  for (int64_t i = n - 1; i >= 0; --i) {
    int m = 0;
    for (int p = diag[i] + 1; p < ptr[i + 1]; ++p)
      m = std::max(m, lev[col[p]] + 1);
    lev[i] = m;
    nu = std::max(nu, m + 1);
  }
  group(lev, nu, L.ilu_uptr, urows);
  GB_CUDA(L.ilu_ptr.alloc(ptr.size()));
  GB_CUDA(L.ilu_col.alloc(std::max<size_t>(col.size(), 1)));
  GB_CUDA(L.ilu_diag.alloc(n));
  GB_CUDA(L.ilu_lrows.alloc(n));
  GB_CUDA(L.ilu_urows.alloc(n));
  GB_CUDA(L.ilu_map.alloc(std::max<size_t>(map.size(), 1)));
  GB_CUDA(L.ilu_v64.alloc(std::max<size_t>(size_t(nnz) * B2, 1)));
  GB_CUDA(L.ilu_v32.alloc(std::max<size_t>(size_t(nnz) * B2, 1)));
  GB_CUDA(h2d(c.stream, L.ilu_ptr.p, ptr.data(), ptr.size() * sizeof(int)));
  GB_CUDA(h2d(c.stream, L.ilu_col.p, col.data(), col.size() * sizeof(int)));
  GB_CUDA(h2d(c.stream, L.ilu_diag.p, diag.data(), n * sizeof(int)));
  GB_CUDA(h2d(c.stream, L.ilu_lrows.p, lrows.data(), n * sizeof(int)));
  GB_CUDA(h2d(c.stream, L.ilu_urows.p, urows.data(), n * sizeof(int)));
  GB_CUDA(h2d(c.stream, L.ilu_map.p, map.data(), map.size() * sizeof(int)));
  ilu_levels_upload(c, L);
  L.ilu_struct = true;
}

static void ensure_ilu_host(Context& c, Level& L);

// The block ILU factors from the level's current values, on the device: the
// values gathered into the row-sorted layout, then one k_ilu_factor launch per
// dependency level, then the FP32 copy. GB_ILU_HOST=1 factors on the host
// instead (the same arithmetic, for comparison).
static void
ensure_ilu(Context& c, Level& L)
{
  if (L.ilu_ready)
    return;
  if (c.ilu_host)
    return ensure_ilu_host(c, L);
  if (!L.ilu_struct)
    ilu_structure(c, L);
  const int B = L.B, B2 = B * B;
  const int64_t nnz = L.h_rowptr[L.n];
  launch(c, k_ilu_gather, stream_blocks(nnz), 256, nnz, B2, (const int*)L.ilu_map.p,
         (const double*)L.A.v64.p, L.ilu_v64.p);
  for (size_t q = 0; q + 1 < L.ilu_lptr.size(); ++q) {
    const int nr = L.ilu_lptr[q + 1] - L.ilu_lptr[q];
    const int* rows = L.ilu_lrows.p + L.ilu_lptr[q];
    const int nb = blocks_for(nr, 128);
    switch (B) {
      case 1:
        launch(c, k_ilu_factor<1>, nb, 128, nr, rows, (const int*)L.ilu_ptr.p,
               (const int*)L.ilu_col.p, (const int*)L.ilu_diag.p, L.ilu_v64.p);
        break;
      case 2:
        launch(c, k_ilu_factor<2>, nb, 128, nr, rows, (const int*)L.ilu_ptr.p,
               (const int*)L.ilu_col.p, (const int*)L.ilu_diag.p, L.ilu_v64.p);
        break;
      case 3:
        launch(c, k_ilu_factor<3>, nb, 128, nr, rows, (const int*)L.ilu_ptr.p,
               (const int*)L.ilu_col.p, (const int*)L.ilu_diag.p, L.ilu_v64.p);
        break;
      default:
        launch(c, k_ilu_factor<4>, nb, 128, nr, rows, (const int*)L.ilu_ptr.p,
               (const int*)L.ilu_col.p, (const int*)L.ilu_diag.p, L.ilu_v64.p);
    }
  }
  launch(c, k_to_float, stream_blocks(nnz * B2), 256, nnz * B2, (const double*)L.ilu_v64.p,
         L.ilu_v32.p);
  L.ilu_ready = true;
}

static void
ensure_ilu_host(Context& c, Level& L)
{
  if (L.ilu_ready)
    return;
  host_values(c, L);
  const int B = L.B, B2 = B * B;
  const int64_t n = L.n, nnz = L.h_rowptr[n];
  std::vector<int> ptr(n + 1), col(nnz), diag(n, -1);
  std::vector<double> v(size_t(nnz) * B2);
  std::vector<int64_t> idx;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t b = L.h_rowptr[i], e = L.h_rowptr[i + 1];
    ptr[i] = static_cast<int>(b);
    idx.resize(e - b);
    for (int64_t k = b; k < e; ++k)
      idx[k - b] = k;
    std::stable_sort(idx.begin(), idx.end(),
                     [&](int64_t x, int64_t y) { return L.h_col[x] < L.h_col[y]; });
    for (int64_t q = 0; q < e - b; ++q) {
      col[b + q] = static_cast<int>(L.h_col[idx[q]]);
      if (col[b + q] == i)
        diag[i] = static_cast<int>(b + q);
      std::memcpy(v.data() + size_t(b + q) * B2, L.h_val.data() + size_t(idx[q]) * B2,
                  B2 * sizeof(double));
    }
    GB_REQUIRE(diag[i] >= 0, GB_EINVAL, "ILU: a row without its diagonal");
  }
  ptr[n] = static_cast<int>(nnz);
  switch (B) {
    case 1: ilu_factor<1>(ptr, col, diag, v, n); break;
    case 2: ilu_factor<2>(ptr, col, diag, v, n); break;
    case 3: ilu_factor<3>(ptr, col, diag, v, n); break;
    default: ilu_factor<4>(ptr, col, diag, v, n);
  }
  // levels: a row waits for the rows it reads (lower part forward, upper part
  // backward); rows of one level ascending
  std::vector<int> lev(n, 0);
  int nl = 0;
  for (int64_t i = 0; i < n; ++i) {
    int m = 0;
    for (int p = ptr[i]; p < diag[i]; ++p)
      m = std::max(m, lev[col[p]] + 1);
    lev[i] = m;
    nl = std::max(nl, m + 1);
  }
  auto group = [&](const std::vector<int>& lv, int nlev, std::vector<int>& off,
                   std::vector<int>& rows) {
    off.assign(nlev + 1, 0);
    for (int64_t i = 0; i < n; ++i)
      off[lv[i] + 1]++;
    for (int q = 0; q < nlev; ++q)
      off[q + 1] += off[q];
    rows.resize(n);
    std::vector<int> fill(off.begin(), off.end() - 1);
    for (int64_t i = 0; i < n; ++i)
      rows[fill[lv[i]]++] = static_cast<int>(i);
  };
  std::vector<int> lrows, urows;
  group(lev, nl, L.ilu_lptr, lrows);
  int nu = 0;
  for (int64_t i = n - 1; i >= 0; --i) {
    int m = 0;
    for (int p = diag[i] + 1; p < ptr[i + 1]; ++p)
      m = std::max(m, lev[col[p]] + 1);
    lev[i] = m;
    nu = std::max(nu, m + 1);
  }
  group(lev, nu, L.ilu_uptr, urows);
  std::vector<float> v32(v.size());
  for (size_t q = 0; q < v.size(); ++q)
    v32[q] = static_cast<float>(v[q]);
  GB_CUDA(L.ilu_ptr.alloc(ptr.size()));
  GB_CUDA(L.ilu_col.alloc(std::max<size_t>(col.size(), 1)));
  GB_CUDA(L.ilu_diag.alloc(n));
  GB_CUDA(L.ilu_lrows.alloc(n));
  GB_CUDA(L.ilu_urows.alloc(n));
  GB_CUDA(L.ilu_v64.alloc(std::max<size_t>(v.size(), 1)));
  GB_CUDA(L.ilu_v32.alloc(std::max<size_t>(v32.size(), 1)));
  GB_CUDA(h2d(c.stream, L.ilu_ptr.p, ptr.data(), ptr.size() * sizeof(int)));
  GB_CUDA(h2d(c.stream, L.ilu_col.p, col.data(), col.size() * sizeof(int)));
  GB_CUDA(h2d(c.stream, L.ilu_diag.p, diag.data(), n * sizeof(int)));
  GB_CUDA(h2d(c.stream, L.ilu_lrows.p, lrows.data(), n * sizeof(int)));
  GB_CUDA(h2d(c.stream, L.ilu_urows.p, urows.data(), n * sizeof(int)));
  GB_CUDA(h2d(c.stream, L.ilu_v64.p, v.data(), v.size() * sizeof(double)));
  GB_CUDA(h2d(c.stream, L.ilu_v32.p, v32.data(), v32.size() * sizeof(float)));
  ilu_levels_upload(c, L);
  L.ilu_ready = true;
  L.ilu_struct = false; // the device path rebuilds its gather map
}

// After a device assembly: the dense maps of the single-CTA coarse programs
// formed again into their own buffers (the captured solver graphs keep
// pointing at them), generic dense maps dropped (rebuilt at first use, with
// the graphs), the direct coarse inverse formed again at its next use.
static void
refresh_values(Context& c)
{
  const int64_t launches0 = c.launches;
  for (auto& kv : c.coarse_progs) {
    CoarseProgram& p = kv.second;
    if (p.ncols == 0 || p.tsize == 0)
      continue;
    if (kv.first.tr)
      for (int l = 0; l <= kv.first.level; ++l)
        ensure_AT(c, c.L[l]);
    if (p.tsize == 8)
      launch_smem(c, k_coarse_cycle<double>, p.ncols, kCoarseThreads, p.smem_bytes,
                  (const CoarseOp*)p.ops.p, p.nops, (const CoarseBuf*)p.bufs.p, p.nbufs,
                  (const CoarsePrefetch*)p.pre.p, p.npre, p.vec_bytes, p.batch);
    else
      launch_smem(c, k_coarse_cycle<float>, p.ncols, kCoarseThreads, p.smem_bytes,
                  (const CoarseOp*)p.ops.p, p.nops, (const CoarseBuf*)p.bufs.p, p.nbufs,
                  (const CoarsePrefetch*)p.pre.p, p.npre, p.vec_bytes, p.batch);
  }
  GB_CUDA(cudaStreamSynchronize(c.stream));
  c.launches = launches0; // set-up, not part of a solve
  if (!c.dense_maps.empty()) {
    c.dense_maps.clear();
    c.version++;
  }
  c.dir_ready[0] = c.dir_ready[1] = false;
  c.values_dirty = false;
}

static void
ensure_work(Context& c)
{
  if (c.work_ready) {
    if (c.values_dirty)
      refresh_values(c);
    ensure_direct(c); // the other orientation after gb_set_operator
    return;
  }
  for (int l = 0; l < c.nlevels; ++l) {
    GB_REQUIRE(c.L[l].has_matrix, GB_ESTATE, "every level needs a matrix");
    if (l + 1 < c.nlevels) {
      GB_REQUIRE(c.T[l].set, GB_ESTATE, "every level pair needs a transfer");
      GB_REQUIRE(c.T[l].nc == c.L[l].n && c.T[l].nf == c.L[l + 1].n, GB_ESTATE,
                 "transfer sizes differ from the level sizes");
    }
  }
  c.w64.u.resize(c.nlevels);
  c.w64.b.resize(c.nlevels);
  c.w64.v.resize(c.nlevels);
  c.w32.u.resize(c.nlevels);
  c.w32.b.resize(c.nlevels);
  c.w32.v.resize(c.nlevels);
  for (int l = 0; l < c.nlevels; ++l) {
    size_t nd = c.L[l].ndof();
    GB_CUDA(c.w64.u[l].alloc(nd));
    GB_CUDA(c.w64.b[l].alloc(nd));
    GB_CUDA(c.w64.v[l].alloc(nd));
    GB_CUDA(c.w32.u[l].alloc(nd));
    GB_CUDA(c.w32.b[l].alloc(nd));
    GB_CUDA(c.w32.v[l].alloc(nd));
  }
  if (c.transposed)
    for (int l = 0; l < c.nlevels; ++l)
      ensure_AT(c, c.L[l]);
  GB_REQUIRE(c.params.smoother >= 0 && c.params.smoother <= 2, GB_EINVAL,
             "smoother must be 0 (jacobi), 1 (vanka) or 2 (ilu)");
  if (c.params.smoother == 1) {
    GB_REQUIRE(!c.transposed, GB_EINVAL, "Vanka with the transposed operator");
    for (int l = 0; l < c.nlevels; ++l)
      ensure_vanka(c, c.L[l]);
  }
  if (c.params.smoother == 2) {
    GB_REQUIRE(!c.transposed, GB_EINVAL, "ILU with the transposed operator");
    for (int l = 0; l < c.nlevels; ++l)
      ensure_ilu(c, c.L[l]);
  }
  for (int l = 0; l < c.nlevels; ++l)
    ensure_pf_scratch(c, c.L[l].n);
  for (int l = 0; l < c.nlevels; ++l) {
    Level& L = c.L[l];
    if (!L.has_hn())
      continue;
    std::vector<uint8_t> m(L.ndof(), 0);
    GB_CUDA(cudaMemcpy(m.data(), L.dirmask.p, m.size(), cudaMemcpyDeviceToHost));
    for (int h : L.h_hnnodes)
      for (int cc = 0; cc < L.B; ++cc)
        m[int64_t(h) * L.B + cc] = 1;
    GB_CUDA(L.pmask.alloc(m.size()));
    GB_CUDA(h2d(c.stream, L.pmask.p, m.data(), m.size()));
  }
  // the single-CTA coarse-level program covers scalar Jacobi cycles without
  // hanging-node steps
  bool simple = c.params.smoother == 0;
  for (int l = 0; l < c.nlevels; ++l)
    simple = simple && c.L[l].B == 1 && !c.L[l].pf_mask &&
             (l == c.nlevels - 1 || !c.L[l].has_hn());
  c.coarse_root = -1;
  for (int l = 0; l < c.nlevels && simple; ++l) {
    if (c.L[l].ndof() > kCoarseMaxRows)
      break;
    c.coarse_root = l;
  }
  c.dense_root = -1;
  for (int l = 0; l < c.nlevels && !simple && c.coarse_dense; ++l) {
    if (c.L[l].ndof() > kCoarseMaxRows)
      break;
    c.dense_root = l;
  }
  c.mid_level = -1;
  if (simple && c.mid_on && c.coarse_on && c.nlevels >= 2 && c.nlevels - 2 > c.coarse_root)
    c.mid_level = c.nlevels - 2;
  else if (simple && c.cluster_on && c.coarse_on && c.nlevels >= 2) {
    // the highest level below the finest that the cluster program takes
    for (int l = c.nlevels - 2; l > c.coarse_root; --l)
      if (c.L[l].ndof() <= c.cluster_rows) {
        c.mid_level = l;
        break;
      }
  }
  if (c.midbar.n < 1) {
    GB_CUDA(c.midbar.alloc(1));
    GB_CUDA(c.miderr.alloc(1));
    GB_CUDA(cudaMemsetAsync(c.miderr.p, 0, sizeof(int), c.stream));
  }
  c.coarse_progs.clear();
  c.dense_maps.clear();
  c.mid_progs.clear();
  c.dir_ready[0] = c.dir_ready[1] = false;
  c.values_dirty = false;
  ensure_direct(c);
  c.work_ready = true;
}

// ------------------------------------------------------------ smoothing

// ------------------------------------------------------------ cycle steps
//
// Every step of the cycle goes through Emit: it either launches the step's
// kernel on the context stream, or (rec set) appends it to the program of the
// coarse-level kernel.
// mask of the prolonged correction on a fine level: SetBoundaryVectorZero and
// HNZero (the hanging dofs), Solver/stdmultilevelsolver.cc:515-517
static const uint8_t*
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
  void jacobi_zero(int l, T* u, const T* b)
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
  // out = two Jacobi sweeps from 0 (scalar levels)
  void jacobi_two_from_zero(int l, T* out, const T* b)
  {
    const Level& L = c.L[l];
    no_rec();
    spmv<kJacobi2, T, T, T>(c, L, opA(c, L), b, out, b, dinv_of<T>(L), c.params.omega);
  }
  // u = (u_zero ? 0 : u) + omega D^-1 h (block Jacobi update, h given;
  // h's filtered component read minus *hmean when set; the weighted mean of
  // the new u reduced into scal[9] when the level has one filtered component)
  void jacobi_apply(int l, const T* h, T* u, bool u_zero, const double* hmean = nullptr)
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
  // u = (u_zero ? 0 : u) + omega * Vanka(h) (VankaSmoother::solve + Add)
  void vanka(int l, const T* h, T* u, bool u_zero, const double* hmean = nullptr)
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
  // The single filtered component of a level (-1: no filter, or several
  // components, which take the unfused pf_sub path).
  static int pf_comp(const Level& L)
  {
    if (!L.pf_mask || (L.pf_mask & (L.pf_mask - 1)))
      return -1;
    return __builtin_ctz(static_cast<unsigned>(L.pf_mask));
  }
  // weighted mean of the updated iterate reduced by the update kernel
  void check_pf_scratch(const Level& L) const
  {
    GB_REQUIRE(c.pfpart.p && c.pfpart.n >= static_cast<size_t>((L.n + 255) / 256 + 1) &&
                 c.pfticket.p,
               GB_ESTATE, "filter scratch not allocated for this level");
  }
  PfArgs weighted_mean_args(const Level& L) const
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
  // out = b - A u (MatrixResidual) with the algebraic mean of the filtered
  // component left in scal[8] for the consumers to subtract on read.
  const double* resid_mean(int l, const T* u, T* out, const T* b)
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
  // scal[8] = algebraic (or, weighted, the integral) mean of the filtered
  // component of x
  const double* mean_of(int l, const T* x, bool weighted)
  {
    const Level& L = c.L[l];
    no_rec();
    launch(c, k_comp_mean<T>, red_blocks(L.n), kRedThreads, (int)L.n, L.B, pf_comp(L), x,
           weighted ? (const double*)L.pf_w.p : nullptr,
           weighted ? L.pf_domain : double(L.n - L.nhanging), c.partials.p, c.ticket.p,
           c.scal.p + 8);
    return c.scal.p + 8;
  }
  // x(., pc) -= *mean
  void sub_mean(int l, T* x, const double* mean)
  {
    const Level& L = c.L[l];
    no_rec();
    launch(c, k_comp_sub<T>, stream_blocks(L.n), 256, (int)L.n, L.B, pf_comp(L), x, mean,
           1.0);
  }
  // HNStructure::Average / Distribute / Zero on level l
  void hn_average(int l, T* u)
  {
    const Level& L = c.L[l];
    no_rec();
    for (const auto& ph : L.hn)
      launch(c, k_hn_average<T>, blocks_for(ph.nh, 128), 128, ph.nh, L.B,
             (const int*)ph.node.p, (const int*)ph.par.p, ph.nslots, ph.gsize,
             (const double*)ph.w.p, u);
  }
  void hn_distribute(int l, T* u)
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
  void hn_zero(int l, T* u)
  {
    const Level& L = c.L[l];
    no_rec();
    if (!L.h_hnnodes.empty())
      launch(c, k_hn_zero<T>, blocks_for(L.h_hnnodes.size(), 128), 128,
             (int)L.h_hnnodes.size(), L.B, (const int*)L.hn_all.p, u);
  }
  void dirichlet_zero(int l, T* u)
  {
    const Level& L = c.L[l];
    no_rec();
    if (L.ndir)
      launch(c, k_dirichlet_zero<T>, blocks_for(L.ndir, 256), 256, L.ndir,
             (const int*)L.dirlist.p, u);
  }
  // pressure filter on x: weighted (SubtractMean) or algebraic
  // (SubtractMeanAlgebraic) mean of every filtered component removed
  void pf_sub(int l, T* x, bool weighted)
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
  void copy(int l, T* dst, const T* src)
  {
    no_rec();
    launch(c, k_equ<T, T>, stream_blocks(c.L[l].ndof()), 256, (int64_t)c.L[l].ndof(), dst,
           1.0, src);
  }
  // h = ILU^-1 h in place (SparseBlockIlu::solve with the identity order: the
  // level kernels of the forward, then of the backward substitution)
  void ilu_solve(int l, T* h)
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
  // u = (u_zero ? 0 : u) + omega h
  void ilu_axpy(int l, T* u, const T* h, bool u_zero)
  {
    no_rec();
    launch(c, k_ilu_axpy<T>, blocks_for(c.L[l].ndof(), 256), 256, (int64_t)c.L[l].ndof(), u,
           c.params.omega, h, int(u_zero));
  }
  void no_rec() const
  {
    if (rec)
      throw Error{ GB_EINVAL, "step not available in the coarse-level program" };
  }
  using TV_of = T;
  static const T* vk_lu(const Level& L);
  static T* vk_out(const Level& L);
  void jacobi(int l, const T* u, T* out, const T* b)
  {
    const Level& L = c.L[l];
    if (rec)
      return rec->push_back(level_op(kOpJacobi, L, out, u, b, c.params.omega));
    spmv<kJacobi, T, T, T>(c, L, opA(c, L), u, out, b, dinv_of<T>(L), c.params.omega);
  }
  void resid(int l, const T* u, T* out, const T* b)
  {
    const Level& L = c.L[l];
    if (rec)
      return rec->push_back(level_op(kOpResid, L, out, u, b, 0.0));
    spmv<kResid, T, T, T>(c, L, opA(c, L), u, out, b, nullptr, 0.0);
  }
  // coarse (level l) = R fine, 0 on the coarse Dirichlet dofs; with smean
  // (block levels) the filtered component of fine is read minus *smean
  void restrict_to(int l, const T* fine, T* coarse, const double* smean = nullptr)
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
    switch (c.L[l].B) {
      case 1:
        if (Tr.rmaxw <= 32)
          launch(c, k_restrict4<T>, blocks_for(int64_t(Tr.nc) * 4, 256), 256, Tr.nc,
                 Tr.rptr.p, Tr.rent.p, fine, coarse, cm);
        else
          launch(c, k_restrict<T>, nb, 256, Tr.nc, Tr.rptr.p, Tr.rent.p, fine, coarse, cm);
        break;
      case 2:
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
  // u = A^-1 b on level 0 (the direct coarse solve)
  void direct(int l, T* u, const T* b)
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
  void fill0(int l, T* u)
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
  // fine (level l+1) += mgomega * (dir ? 0 : P coarse)
  void prolong(int l, const T* coarse, T* fine)
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
};

template<>
const double* Emit<double>::vk_lu(const Level& L)
{
  return L.vk_inv64.p;
}
template<>
const float* Emit<float>::vk_lu(const Level& L)
{
  return L.vk_inv32.p;
}
template<>
double* Emit<double>::vk_out(const Level& L)
{
  return L.vk_out64.p;
}
template<>
float* Emit<float>::vk_out(const Level& L)
{
  return L.vk_out32.p;
}

// StdSolver::smooth, linear_smooth jacobi (Solver/stdsolver.cc:951-986): each
// sweep computes h = y - A x, h = D^-1 h, x += omega h; fused into one pass that
// writes the new iterate to the other buffer (u and tmp swap roles). A sweep
// from x = 0 needs no product (y - A 0 == y).
//
// With the Vanka smoother or a pressure filter a sweep is done in place:
// h = y - A x (tmp), SubtractMeanAlgebraic(h), h = Vanka(h) or D^-1 h,
// x += omega h, SubtractMean(x).
static bool
fused_smoother(const Context& c, const Level& L)
{
  return c.params.smoother == 0 && !L.pf_mask;
}

template<class T>
static void
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
static bool mgstep(Emit<T>& E, MgWork<T>& W, int l, int finelevel, int coarselevel,
                   char& p0, char p, T*& u, T*& tmp, const T* b, bool u_zero);

template<class T>
static const CoarseProgram& coarse_program(Context& c, MgWork<T>& W, int l, int finelevel,
                                           int coarselevel, char p0, char p, T* u, T* tmp,
                                           const T* b, bool u_zero);

// Runs mgstep(l) for a level handled by the coarse-level kernel: the step is
// recorded once per entry state (cached) and launched as one single-CTA kernel.
template<class T>
static bool
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
static bool
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
static int
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
static bool
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
static const CoarseProgram&
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
static bool
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
template<class T>
static bool
mgstep(Emit<T>& E, MgWork<T>& W, int l, int finelevel, int coarselevel, char& p0,
       char p, T*& u, T*& tmp, const T* b, bool u_zero)
{
  Context& c = E.c;
  if (!E.rec && c.coarse_on && l == c.mid_level && u_zero && l != E.no_dense_at)
    return run_mid<T>(E, W, l, finelevel, coarselevel, p0, p, u, tmp, b);
  if (!E.rec && c.coarse_on && l <= c.coarse_root)
    return run_coarse<T>(E, W, l, finelevel, coarselevel, p0, p, u, tmp, b, u_zero);
  if (E.rec && E.mid && c.coarse_dense && c.coarse_on && l == c.coarse_root && u_zero)
    return emit_dense<T>(E, W, l, finelevel, coarselevel, p0, p, u, tmp, b);
  if (!E.rec && c.coarse_on && l <= c.dense_root && u_zero && l != E.no_dense_at)
    return run_dense<T>(E, W, l, finelevel, coarselevel, p0, p, u, tmp, b);
  const gb_params& P = c.params;
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
  // MatrixResidual into tmp (with SubtractMeanAlgebraic), restrict_zero +
  // SetBoundaryVectorZero on l-1
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
  } else if (u_zero) {
    E.restrict_to(l - 1, b, W.b[l - 1].p); // u == 0: the residual is b
  } else {
    E.resid(l, u, tmp, b);
    E.restrict_to(l - 1, tmp, W.b[l - 1].p);
  }
  if (c.L[l - 1].has_hn()) { // HNDistribute, then SetBoundaryVectorZero again
    E.hn_distribute(l - 1, W.b[l - 1].p);
    E.dirichlet_zero(l - 1, W.b[l - 1].p);
  }
  int j = (p0 == 'V') ? 1 : (p0 == 'W') ? 2 : (p0 == 'F') ? 3 : 0;
  T* uc = W.u[l - 1].p;
  T* tc = W.v[l - 1].p;
  bool czero = true; // Zero(u) on l-1
  for (int i = 0; i < j; ++i)
    czero = mgstep<T>(E, W, l - 1, finelevel, coarselevel, p0, p, uc, tc,
                      W.b[l - 1].p, czero);
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
template<class T>
static void
precondition_T(Context& c, MgWork<T>& W, T* x, const T* y, bool x_zero)
{
  ensure_work(c);
  const int fl = c.nlevels - 1;
  T* u = x;
  T* tmp = W.v[fl].p;
  // Pick the buffer of the first sweep so that the last write lands in x.
  const gb_params& P = c.params;
  int pingpong = (x_zero ? std::max(P.iterpre - 1, 0) : P.iterpre) + P.iterpost;
  if (fl == 0)
    pingpong = x_zero ? std::max(P.iterexact - 1, 0) : P.iterexact;
  if (!fused_smoother(c, c.L[fl]))
    pingpong = 0; // sweeps in place
  if (x_zero && (pingpong & 1))
    std::swap(u, tmp);
  char p = P.mgtype;
  char p0 = (p == 'F') ? 'W' : p;
  Emit<T> E{ c, nullptr };
  if (mgstep<T>(E, W, fl, fl, 0, p0, p, u, tmp, y, x_zero))
    E.fill0(fl, u);
  if (u != x) {
    GB_CUDA(cudaMemcpyAsync(x, u, c.L[fl].ndof() * sizeof(T),
                            cudaMemcpyDeviceToDevice, c.stream));
  }
}

// ------------------------------------------------------------------ GMRES

static void
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
static void
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

static void
read_flags(Context& c)
{
  GB_CUDA(cudaMemcpyAsync(c.h_flags, &c.G.p->reached, 3 * sizeof(int),
                          cudaMemcpyDeviceToHost, c.stream));
  GB_CUDA(cudaStreamSynchronize(c.stream));
}

static void
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
static void
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
static void
fill_info(Context& c, gb_solve_info* info, double* x_for_residual, const double* b)
{
  fill_info_enqueue(c, x_for_residual, b);
  GB_CUDA(cudaStreamSynchronize(c.stream));
  fill_info_finish(c, info);
}

// NewtonLinearSolve's closing SubtractMean(x) on the finest level
// (Solver/stdmultilevelsolver.cc:671); a no-op without a pressure filter.
static void
final_filter(Context& c, double* x)
{
  const int fl = c.nlevels - 1;
  if (!c.L[fl].pf_mask)
    return;
  Emit<double> E{ c, nullptr };
  E.pf_sub(fl, x, true);
}

// StdMultiLevelSolver::Gmres -> GMRES::solve (left preconditioning)
static int
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
static int
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
static MgWork<T>& work(Context& c);
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

static std::vector<cudaGraphNode_t>
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

static cudaGraph_t
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
struct FBufs
{
  T* Z;
  T* zfix;
  T* rhs;
};

template<class T>
static FBufs<T>
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
static void
fg_setup(Context& c)
{
  const int64_t n = c.L[c.nlevels - 1].ndof();
  GmresDev* G = c.G.p;
  launch(c, k_fg_setup, 1, 1, G, c.params.tol, c.params.globaltol, c.params.maxiter);
  dot_dev(c, n, c.bg.p, c.bg.p, RedOut{ &G->bnorm, nullptr, nullptr, 1 });
  launch(c, k_fill<double>, stream_blocks(n), 256, n, c.xg.p, 0.0);
}

template<class T>
static void
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
static void
fg_inner(Context& c, const FBufs<T>& F, cudaGraphConditionalHandle hInner, int use_cond)
{
  const int fl = c.nlevels - 1;
  Level& L = c.L[fl];
  const int64_t n = L.ndof();
  GmresDev* G = c.G.p;
  double* V = c.krylov.p;
  launch(c, k_load_idx<T>, stream_blocks(n), 256, n, F.rhs, V, (const GmresDev*)G);
  precondition_T<T>(c, work<T>(c), F.zfix, F.rhs, true);
  spmv<kAx, double, T, double>(c, L, opA(c, L), (const T*)F.zfix, V, nullptr, nullptr, 1.0,
                               (const int*)&G->j, n, F.Z);
  // one block of kCgsThreads per 2 kCgsThreads rows, at most four per SM
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
static void
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
static void
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
static void
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
static int
fgmres_graph(Context& c, double* x, const double* b, int prec, gb_solve_info* info,
             bool copy_in = true, bool copy_out = true, double* host_x = nullptr,
             cudaEvent_t after_copy = nullptr)
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

} // namespace gb

// ==================================================================== C-ABI

using namespace gb;

// Runs f with the transposed level operators, restoring the setting after.
template<class F>
static int
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

namespace gb {

// Element matrices and their sum into level l's values (FP64 and FP32), the
// Dirichlet rows and columns, and the block-diagonal inverse; the kappa of the
// level's cells is in L.m_kappa.
static void
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
static void
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
static void
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

static void
check_mesh(const Level& L)
{
  GB_REQUIRE(L.mesh_ncells > 0 && L.mesh_n == L.n, GB_ESTATE,
             "no mesh for this level's matrix (gb_level_set_mesh)");
}

static void
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
  build_sell(L.A, n, rowptr, col, val, ctx->stream, B);
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
               te, f, cc, nm);
      else
        launch(*ctx, k_restrict<double>, nb, 256, T.nc, tp, te, f, cc, nm);
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

// ------------------------------------------------- allocation-free dot product
//
// Scratch of gb_dot_noalloc: one FP64 partial per block plus the last-block
// ticket, in file-scope device arrays. Host code may not pass these names to a
// kernel (on the host they are stand-ins, not device addresses); their device
// addresses are looked up once per device with cudaGetSymbolAddress.

namespace gb {
constexpr int kNoAllocBlocks = 4096;
constexpr int64_t kNoAllocMaxN = int64_t(kNoAllocBlocks) * kRedThreads * 8;
static __device__ __align__(256) double g_noalloc_partials[kNoAllocBlocks];
static __device__ __align__(256) unsigned g_noalloc_ticket[64];
struct NoAllocAddr
{
  double* partials = nullptr;
  unsigned* ticket = nullptr;
};
constexpr int kNoAllocMaxDevices = 64;
static NoAllocAddr g_noalloc_addr[kNoAllocMaxDevices];
static std::mutex g_noalloc_mutex;
} // namespace gb

int
gb_dot_noalloc(const double* a, const double* b, int64_t n, double* out, void* stream)
{
  using namespace gb;
  if (!a || !b || !out || n < 0) {
    fprintf(stderr, "gb_dot_noalloc: null pointer or negative length\n");
    return GB_EINVAL;
  }
  if (n > kNoAllocMaxN) {
    fprintf(stderr,
            "gb_dot_noalloc: n = %lld exceeds the maximum %lld (scratch of %d "
            "partial sums); use gb_vec_dot\n",
            (long long)n, (long long)kNoAllocMaxN, kNoAllocBlocks);
    return GB_EINVAL;
  }
  // an error the caller's own earlier work left pending is reported, not
  // consumed: cudaGetLastError after our launch would otherwise clear it
  if (cudaPeekAtLastError() != cudaSuccess) {
    fprintf(stderr, "gb_dot_noalloc: a CUDA error is already pending\n");
    return GB_ECUDA;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices)
    return GB_ECUDA;
  // the address is looked up once per device ordinal and kept for the life of
  // the process (it does not survive cudaDeviceReset of that device)
  NoAllocAddr addr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mutex);
    if (!g_noalloc_addr[dev].partials) {
      void* pp = nullptr;
      void* tp = nullptr;
      if (cudaGetSymbolAddress(&pp, g_noalloc_partials) != cudaSuccess ||
          cudaGetSymbolAddress(&tp, g_noalloc_ticket) != cudaSuccess || !pp || !tp) {
        fprintf(stderr, "gb_dot_noalloc: cudaGetSymbolAddress failed\n");
        return GB_ECUDA;
      }
      g_noalloc_addr[dev].partials = static_cast<double*>(pp);
      g_noalloc_addr[dev].ticket = static_cast<unsigned*>(tp);
    }
    addr = g_noalloc_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the ticket must start at 0 (an earlier failed call may have left it set)
  if (cudaMemsetAsync(addr.ticket, 0, sizeof(unsigned), st) != cudaSuccess)
    return GB_ECUDA;
  const int grid = static_cast<int>(
    std::max<int64_t>(1, (n + int64_t(kRedThreads) * 8 - 1) / (int64_t(kRedThreads) * 8)));
  k_dot<double, double><<<grid, kRedThreads, 0, st>>>(
    n, a, b, addr.partials, addr.ticket, RedOut{ out, nullptr, nullptr, 0 });
  if (cudaGetLastError() != cudaSuccess)
    return GB_ECUDA;
  return GB_OK;
}

} // extern "C"
