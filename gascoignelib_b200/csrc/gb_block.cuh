// Block-system kernels (ncomp = B > 1 components per node, Stokes-type
// systems), the pressure filter and the Vanka smoother. Included by
// gb_solver.cu after gb_kernels.cuh.
#pragma once
#include "gb_kernels.cuh"

namespace gb {

// Block SpMV over SELL-32 block rows: one thread per node; block entry j of
// lane l holds its B*B values component-major inside the slice, value q at
// val[(sptr[s] + 32 j) * B*B + 32 q + l] (coalesced per q). Per block the row
// sums are formed first and then added (FMatrixBlock::cadd,
// LinAlg/fmatrixblock.h:110-122; SparseBlockMatrix::vmult,
// LinAlg/sparseblockmatrix.xx:378-392). Modes as k_spmv; kJacobi applies the
// node's inverse diagonal block (FMatrixBlock::vmult order).
template<int MODE, int B, class TV, class TX, class TO, bool PAT>
__global__ void __launch_bounds__(kSpmvThreads)
k_bspmv(SellView<TV> A, const TX* __restrict__ x, TO* __restrict__ y,
        const TO* __restrict__ b, const TV* __restrict__ dinv,
        const uint8_t* __restrict__ dirmask, double alpha_,
        const int* __restrict__ yidx, int64_t ystride, TX* __restrict__ xcopy)
{
  GB_PDL_ENTRY();
  using TA = typename Acc<TV, TO>::type;
  constexpr int B2 = B * B;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= A.n)
    return;
  const int s = row >> 5, lane = row & 31;
  const int beg = A.sptr[s];
  const int w = (A.sptr[s + 1] - beg) >> 5;
  const TV* vp = A.val + int64_t(beg) * B2 + lane;
  const int* cp = PAT ? (A.ptab + int(A.pid[row]) * A.W) : (A.col + beg + lane);
  constexpr bool NEG = (MODE == kResid || MODE == kResidDir || MODE == kJacobi);
  TA acc[B];
#pragma unroll
  for (int r = 0; r < B; ++r)
    acc[r] = NEG ? static_cast<TA>(b[int64_t(row) * B + r]) : TA(0);
#pragma unroll 2
  for (int j = 0; j < w; ++j) {
    const int c = PAT ? row + ldg(cp + j) : ldg(cp + j * kSlice);
    TA xv[B], m[B2];
#pragma unroll
    for (int k = 0; k < B; ++k)
      xv[k] = static_cast<TA>(ldg(x + int64_t(c) * B + k));
#pragma unroll
    for (int q = 0; q < B2; ++q)
      m[q] = static_cast<TA>(ldg(vp + int64_t(j) * kSlice * B2 + q * kSlice));
#pragma unroll
    for (int r = 0; r < B; ++r) {
      TA sum = TA(0);
#pragma unroll
      for (int k = 0; k < B; ++k)
        sum = fma(m[r * B + k], xv[k], sum);
      acc[r] = NEG ? acc[r] - sum : acc[r] + sum;
    }
  }
  const TA alpha = static_cast<TA>(alpha_);
  const int64_t o = int64_t(row) * B;
  if (yidx) { // device-indexed output, as k_spmv
    const int64_t jj = *yidx;
#pragma unroll
    for (int r = 0; r < B; ++r)
      xcopy[jj * ystride + o + r] = x[o + r];
    y += (jj + 1) * ystride;
  }
  if (MODE == kJacobi) {
#pragma unroll
    for (int r = 0; r < B; ++r) {
      TA h = TA(0);
#pragma unroll
      for (int k = 0; k < B; ++k)
        h = fma(static_cast<TA>(dinv[o * B + r * B + k]), acc[k], h);
      y[o + r] = static_cast<TO>(static_cast<TA>(x[o + r]) + alpha * h);
    }
    return;
  }
#pragma unroll
  for (int r = 0; r < B; ++r) {
    if (MODE == kAx)
      y[o + r] = static_cast<TO>(alpha * acc[r]);
    else if (MODE == kAddAx)
      y[o + r] = static_cast<TO>(static_cast<TA>(y[o + r]) + alpha * acc[r]);
    else if (MODE == kResid)
      y[o + r] = static_cast<TO>(acc[r]);
    else
      y[o + r] = dirmask[o + r] ? TO(0) : static_cast<TO>(acc[r]);
  }
}

// u = (u_zero ? 0 : u) + omega * (D^-1 h) per node: SparseBlockMatrix::Jacobi
// (LinAlg/sparseblockmatrix.xx:47-56) followed by Add(x, omega, h).
template<int B, class TV, class T>
__global__ void
k_block_jacobi_apply(int n, const TV* __restrict__ dinv, const T* __restrict__ h,
                     T* __restrict__ u, double omega, int u_zero)
{
  GB_PDL_ENTRY();
  using TA = typename Acc<TV, T>::type;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const int64_t o = int64_t(i) * B;
  TA t[B];
#pragma unroll
  for (int k = 0; k < B; ++k)
    t[k] = static_cast<TA>(h[o + k]);
#pragma unroll
  for (int r = 0; r < B; ++r) {
    TA v = TA(0);
#pragma unroll
    for (int k = 0; k < B; ++k)
      v = fma(static_cast<TA>(dinv[o * B + r * B + k]), t[k], v);
    const TA base = u_zero ? TA(0) : static_cast<TA>(u[o + r]);
    u[o + r] = static_cast<T>(base + static_cast<TA>(omega) * v);
  }
}

// Block transfers: the scalar tables applied to each of the B components.
// acc holds the starting values (0, or the target for an in-place add: the
// weights are powers of two, so each fused add rounds like the reference's
// y += w x).
template<class T, int B>
__device__ __forceinline__ void
transfer_row_b(const int* __restrict__ tsp, const uint32_t* __restrict__ tent,
               const T* __restrict__ src, int i, T (&acc)[B])
{
  const int beg = __ldg(tsp + (i >> 5));
  const int w = (__ldg(tsp + (i >> 5) + 1) - beg) >> 5;
  const uint32_t* ep = tent + beg + (i & 31);
  for (int j = 0; j < w; ++j) {
    const uint32_t e = __ldg(ep + j * kSlice);
    const T wgt = wcode<T>(e);
    const T* sp = src + int64_t(e & kIdxMask) * B;
#pragma unroll
    for (int c = 0; c < B; ++c)
      acc[c] = fma(wgt, __ldg(sp + c), acc[c]);
  }
}

template<class T, int B>
__global__ void
k_restrict_b(int nc, const int* __restrict__ tsp, const uint32_t* __restrict__ tent,
             const T* __restrict__ fine, T* __restrict__ coarse,
             const uint8_t* __restrict__ cdir)
{
  GB_PDL_ENTRY();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nc)
    return;
  T acc[B];
#pragma unroll
  for (int c = 0; c < B; ++c)
    acc[c] = T(0);
  transfer_row_b<T, B>(tsp, tent, fine, i, acc);
#pragma unroll
  for (int c = 0; c < B; ++c) {
    const int64_t d = int64_t(i) * B + c;
    coarse[d] = (cdir && cdir[d]) ? T(0) : acc[c];
  }
}

template<int MODE, class T, int B>
__global__ void
k_prolong_b(int nf, const int* __restrict__ tsp, const uint32_t* __restrict__ tent,
            const T* __restrict__ coarse, T* __restrict__ fine,
            const uint8_t* __restrict__ fdir, double mgomega)
{
  GB_PDL_ENTRY();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nf)
    return;
  T acc[B];
#pragma unroll
  for (int c = 0; c < B; ++c)
    acc[c] = MODE == 0 ? fine[int64_t(i) * B + c] : T(0);
  transfer_row_b<T, B>(tsp, tent, coarse, i, acc);
#pragma unroll
  for (int c = 0; c < B; ++c) {
    const int64_t d = int64_t(i) * B + c;
    if (MODE == 0) {
      fine[d] = acc[c];
    } else {
      const T a = (fdir && fdir[d]) ? T(0) : acc[c];
      fine[d] = fine[d] + static_cast<T>(mgomega) * a;
    }
  }
}

// ------------------------------------------------------ pressure filter
//
// PressureFilter::IntegrateVector / SubtractMeanAlgebraic's sum
// (Discretization/Q1/pressurefilter.cc:56-100): sum over nodes of
// x(j, c) * w_j (w null: plain sum), deterministic FP64 reduction.
template<class T>
__global__ void __launch_bounds__(kRedThreads)
k_comp_sum(int n, int B, int c, const T* __restrict__ x, const double* __restrict__ w,
           double* partials, unsigned* ticket, RedOut ro)
{
  GB_PDL_ENTRY();
  __shared__ double sh[32];
  double v = 0.0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const double xv = static_cast<double>(x[int64_t(j) * B + c]);
    v = w ? fma(xv, w[j], v) : v + xv;
  }
  v = block_sum(v, sh);
  red_finish(partials, ticket, v, ro, sh);
}

// x(., c) += -(sum / denom): CompAdd(comp, -mean / domainsize) or
// CompAdd(comp, -sum / (n - nhanging)).
template<class T>
__global__ void
k_comp_sub(int n, int B, int c, T* __restrict__ x, const double* __restrict__ sum,
           double denom)
{
  GB_PDL_ENTRY();
  const double sub = sum[0] / denom;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    x[int64_t(j) * B + c] = static_cast<T>(static_cast<double>(x[int64_t(j) * B + c]) - sub);
}

// ------------------------------------------------------------------ Vanka
//
// VankaSmoother::solve (LinAlg/vankasmoother.cc:192-237) in two kernels: the
// local solves (one per patch, writing the patch solutions), then a gather per
// node that sums the solutions of the patches containing it in ascending
// patch order (the reference's order on one thread), scales by 1/count and
// adds omega times it to u (StdSolver::smooth's Add).
//
// Thread per patch (M = patch nodes * B <= 32): LU factors, pivots and
// solutions stored entry-major ([entry][patch]) so that a warp's loads are
// contiguous. The right-hand side is gathered through the row permutation,
// then unit-lower forward and upper backward substitution, rows in order and
// each row's sum in ascending column order (the triangular solves of the LU).
template<int M, int B, class TL, class T>
__global__ void __launch_bounds__(128)
k_vanka_local(int npatch, const int* __restrict__ pn, const TL* __restrict__ lu,
              const uint8_t* __restrict__ perm, const T* __restrict__ h,
              T* __restrict__ hout)
{
  GB_PDL_ENTRY();
  using TA = typename Acc<TL, T>::type;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npatch)
    return;
  const int64_t np = npatch;
  TA H[M];
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const int P = __ldg(perm + i * np + p);
    const int node = __ldg(pn + (P / B) * np + p);
    H[i] = static_cast<TA>(__ldg(h + int64_t(node) * B + (P % B)));
  }
#pragma unroll
  for (int i = 1; i < M; ++i) {
    TA s = H[i];
#pragma unroll
    for (int j = 0; j < i; ++j)
      s -= static_cast<TA>(__ldg(lu + (i * M + j) * np + p)) * H[j];
    H[i] = s;
  }
#pragma unroll
  for (int i = M - 1; i >= 0; --i) {
    TA s = H[i];
#pragma unroll
    for (int j = i + 1; j < M; ++j)
      s -= static_cast<TA>(__ldg(lu + (i * M + j) * np + p)) * H[j];
    H[i] = s / static_cast<TA>(__ldg(lu + (i * M + i) * np + p));
  }
#pragma unroll
  for (int i = 0; i < M; ++i)
    hout[i * np + p] = static_cast<T>(H[i]);
}

// Warp per patch (any M <= kVankaMaxM): factors patch-major ([patch][M*M]),
// solutions patch-major ([patch][M]); each row's sum is split over the lanes
// and reduced by shuffles.
constexpr int kVankaMaxM = 128;
constexpr int kVankaWarps = 4;

template<class TL, class T>
__global__ void __launch_bounds__(32 * kVankaWarps)
k_vanka_local_warp(int npatch, int M, int B, const int* __restrict__ pn,
                   const TL* __restrict__ lu, const uint8_t* __restrict__ perm,
                   const T* __restrict__ h, T* __restrict__ hout)
{
  GB_PDL_ENTRY();
  __shared__ double sH[kVankaWarps][kVankaMaxM];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = blockIdx.x * kVankaWarps + wid;
  if (p >= npatch)
    return;
  const int64_t np = npatch;
  double* H = sH[wid];
  const TL* L = lu + int64_t(p) * M * M;
  for (int i = lane; i < M; i += 32) {
    const int P = perm[int64_t(p) * M + i];
    const int node = pn[(P / B) * np + p];
    H[i] = static_cast<double>(h[int64_t(node) * B + (P % B)]);
  }
  __syncwarp();
  for (int i = 1; i < M; ++i) {
    double s = 0.0;
    for (int j = lane; j < i; j += 32)
      s = fma(static_cast<double>(L[i * M + j]), H[j], s);
    for (int o = 16; o > 0; o >>= 1)
      s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0)
      H[i] -= s;
    __syncwarp();
  }
  for (int i = M - 1; i >= 0; --i) {
    double s = 0.0;
    for (int j = i + 1 + lane; j < M; j += 32)
      s = fma(static_cast<double>(L[i * M + j]), H[j], s);
    for (int o = 16; o > 0; o >>= 1)
      s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0)
      H[i] = (H[i] - s) / static_cast<double>(L[i * M + i]);
    __syncwarp();
  }
  for (int i = lane; i < M; i += 32)
    hout[int64_t(p) * M + i] = static_cast<T>(H[i]);
}

// u(i, c) = (u_zero ? 0 : u(i, c)) + omega * ((sum over the node's patches of
// their solution at (i, c)) * (1 / count)). ent packs (patch, local node):
// patch * 32 + r (npp <= 27). Solution (patch p, local dof q) at
// hout[q * s1 + p * s2].
template<int B, class T>
__global__ void
k_vanka_gather(int n, const int* __restrict__ nptr, const int* __restrict__ ent,
               const T* __restrict__ hout, int64_t s1, int64_t s2, T* __restrict__ u,
               double omega, int u_zero)
{
  GB_PDL_ENTRY();
  using TA = typename Acc<T, T>::type;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const int k0 = __ldg(nptr + i), k1 = __ldg(nptr + i + 1);
  TA acc[B];
#pragma unroll
  for (int c = 0; c < B; ++c)
    acc[c] = TA(0);
  for (int k = k0; k < k1; ++k) {
    const int e = __ldg(ent + k);
    const int64_t p = e >> 5, r = e & 31;
#pragma unroll
    for (int c = 0; c < B; ++c)
      acc[c] += static_cast<TA>(hout[(r * B + c) * s1 + p * s2]);
  }
  const TA sc = TA(1) / static_cast<TA>(k1 - k0);
#pragma unroll
  for (int c = 0; c < B; ++c) {
    const int64_t d = int64_t(i) * B + c;
    const TA base = u_zero ? TA(0) : static_cast<TA>(u[d]);
    u[d] = static_cast<T>(base + static_cast<TA>(omega) * (acc[c] * sc));
  }
}

} // namespace gb
