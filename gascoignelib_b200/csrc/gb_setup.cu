// Matrix layouts on the device (SELL-32, patterns, row-block copies), the
// transpose, and the per-level set-up: transfers, Vanka and block-ILU
// factorisations, the direct coarse inverse.
#include "gb_context.cuh"

namespace gb {

std::atomic<long long> g_fail_alloc_countdown{ 0 };

// Rows whose column lists, relative to the row, coincide share one pattern. A
// level uses the compressed form when it has at most 256 patterns.
void
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

void
build_sell(Sell& S, int64_t n, const int64_t* rowptr, const int64_t* col,
           const double* val, cudaStream_t st, int B, bool locality)
{
  const int B2 = B * B;
  S.B = B;
  S.n = static_cast<int>(n);
  S.nslices = static_cast<int>((n + kSlice - 1) / kSlice);
  S.nnz = rowptr[n];
  // the column patterns (per row, independent of the slot order)
  build_patterns(S, n, rowptr, col, st);
  // Slot order: on levels without column patterns (locality), rows in the
  // order of their smallest column; then rows sorted by length (descending,
  // stable) inside windows of sort_window rows when that saves more than a
  // tenth of the padded slots (levels above the single-CTA coarse size only):
  // 1024 rows on the locality-ordered levels (C4: mixed solve 154.4 ms against
  // 156.0 with 256 and 170.6 with 64), 256 elsewhere.
  int64_t sort_window = 256;
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
  if (locality && !S.pat && B == 1 && n > 1024) {
    // slots in the order of each row's smallest column: on a hierarchically
    // numbered mesh (the reference's refined meshes: no column patterns) the
    // rows of one neighbourhood share their smallest (coarsest) column, so the
    // 32 rows of a slice gather nearby x values. Each row keeps its entries
    // and their order, so every row's result is unchanged. Measured on C4 (the
    // reference's ball-refined Q2 mesh): FP32 sweep 182 -> 148 us, FP64 SpMV
    // 203 -> 174 us, mixed solve 170.8 -> 155.8 ms. Block levels (B > 1)
    // keep the mesh's order: on C3 (2D Q1/Q1 Stokes, B = 3) this order made
    // the FP64 solve slower (16.5 -> 18.0 ms).
    std::vector<int64_t> key(n);
    for (int64_t r = 0; r < n; ++r) {
      int64_t m = r;
      for (int64_t k = rowptr[r]; k < rowptr[r + 1]; ++k)
        m = std::min(m, col[k]);
      key[r] = m;
    }
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return key[a] < key[b]; });
    for (int64_t t = 0; t < n && !S.sorted; ++t)
      S.sorted = perm[t] != t;
    sort_window = 1024;
  }
  if (n > 1024) {
    std::vector<int> sp(perm);
    for (int64_t w0 = 0; w0 < n; w0 += sort_window)
      std::stable_sort(sp.begin() + w0, sp.begin() + std::min<int64_t>(n, w0 + sort_window),
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

// The row-major FP32 values of S for the row-block SpMV, from its SELL
// values (again after every change of those on the device); with
// `columns`, also the columns of a level without patterns.
void
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

void
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

// The host copy of a level's values after a device assembly (gb_assemble),
// for the set-up steps that read it (transpose, Vanka factors, direct coarse
// inverse): the FP64 SELL values read back and put in stencil order.
void
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
std::vector<int>
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

// A^T of the uploaded (Dirichlet-modified) level matrix. A structurally
// symmetric matrix keeps its own sparsity pattern and row order, with the
// values swapped in place as SparseBlockMatrix::transpose does
// (LinAlg/sparseblockmatrix.xx:478-491); otherwise rows of A^T list the
// columns of A in ascending order. Strong Dirichlet rows and columns of the
// uploaded matrix are both identity, so A^T is the reference's dual matrix
// (transpose, then DirichletMatrixOnlyRow) wherever it meets a vector that is
// zero on the Dirichlet dofs, which every vector of the dual solve is.
void
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
  build_sell(L.AT, n, tp.data(), tc.data(), tv.data(), c.stream, B, c.row_order);
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
void
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
void
ensure_vanka_host(Context& c, Level& L);

// The patch structure of a level (once per matrix structure and patch list):
// patch node lists, the node -> (patch, slot) map of the averaging gather, and
// per node pair of a patch the offset of its block in the SELL values (-1
// where the matrix has no block), with the factor and solution buffers.
void
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
void
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

void
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
bool
direct_on(const Context& c)
{
  return c.params.ndirect > 0 && c.nlevels > 0 && c.L[0].n < c.params.ndirect;
}

void
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
void
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
void
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

void
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

void ensure_ilu_host(Context& c, Level& L);

// The block ILU factors from the level's current values, on the device: the
// values gathered into the row-sorted layout, then one k_ilu_factor launch per
// dependency level, then the FP32 copy. GB_ILU_HOST=1 factors on the host
// instead (the same arithmetic, for comparison).
void
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

void
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
void
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

void
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

} // namespace gb
