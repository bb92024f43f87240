// Block-system kernels (ncomp = B > 1 components per node, Stokes-type
// systems), the pressure filter, the Vanka smoother and the block ILU.
// Included by gb_context.cuh after gb_kernels.cuh.
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
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= A.n)
    return;
  const int row = A.perm ? __ldg(A.perm + slot) : slot;
  const int s = slot >> 5, lane = slot & 31;
  const int beg = A.sptr[s];
  const int w = (A.sptr[s + 1] - beg) >> 5;
  const TV* vp = A.val + int64_t(beg) * B2 + lane;
  const int* cp = PAT ? (A.ptab + int(A.pid[row]) * A.W) : (A.col + beg + lane);
  constexpr bool NEG = (MODE == kResid || MODE == kResidDir || MODE == kJacobi);
  TA acc[B];
#pragma unroll
  for (int r = 0; r < B; ++r)
    acc[r] = NEG ? static_cast<TA>(b[int64_t(row) * B + r]) : TA(0);
#pragma unroll 4
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

// y = b - A x on block rows with the pressure filter's plain mean of
// component pc of y (StdSolver::MatrixResidual with SubtractMeanAlgebraic):
// the last block writes sum / denom to *mean; consumers subtract it on read.
template<int B, class TV, class T, bool PAT>
__global__ void __launch_bounds__(kSpmvThreads)
k_bspmv_resid_mean(SellView<TV> A, const T* __restrict__ x, T* __restrict__ y,
                   const T* __restrict__ b, int pc, double denom, double* partials,
                   unsigned* ticket, double* mean)
{
  GB_PDL_ENTRY();
  using TA = typename Acc<TV, T>::type;
  constexpr int B2 = B * B;
  __shared__ double sh[32];
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (slot < A.n) {
    const int row = A.perm ? __ldg(A.perm + slot) : slot;
    const int s = slot >> 5, lane = slot & 31;
    const int beg = A.sptr[s];
    const int w = (A.sptr[s + 1] - beg) >> 5;
    const TV* vp = A.val + int64_t(beg) * B2 + lane;
    const int* cp = PAT ? (A.ptab + int(A.pid[row]) * A.W) : (A.col + beg + lane);
    TA acc[B];
#pragma unroll
    for (int r = 0; r < B; ++r)
      acc[r] = static_cast<TA>(b[int64_t(row) * B + r]);
#pragma unroll 4
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
        acc[r] = acc[r] - sum;
      }
    }
#pragma unroll
    for (int r = 0; r < B; ++r) {
      const T o = static_cast<T>(acc[r]);
      y[int64_t(row) * B + r] = o;
      if (r == pc)
        v = static_cast<double>(o);
    }
  }
  v = block_sum(v, sh);
  red_finish(partials, ticket, v, RedOut{ mean, nullptr, nullptr, 0, denom }, sh);
}

// Plain or weighted mean of component pc (no subtraction): *mean =
// (sum_j x(j, pc) [* w_j]) / denom.
template<class T>
__global__ void __launch_bounds__(kRedThreads)
k_comp_mean(int n, int B, int pc, const T* __restrict__ x, const double* __restrict__ w,
            double denom, double* partials, unsigned* ticket, double* mean)
{
  GB_PDL_ENTRY();
  __shared__ double sh[32];
  double v = 0.0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const double xv = static_cast<double>(x[int64_t(j) * B + pc]);
    v = w ? fma(xv, w[j], v) : v + xv;
  }
  v = block_sum(v, sh);
  red_finish(partials, ticket, v, RedOut{ mean, nullptr, nullptr, 0, denom }, sh);
}

// u = (u_zero ? 0 : u) + omega * (D^-1 h) per node: SparseBlockMatrix::Jacobi
// (LinAlg/sparseblockmatrix.xx:47-56) followed by Add(x, omega, h).
// Pressure filter around it (pc >= 0): h's component pc is read minus *hmean
// (its algebraic mean, when hmean is set), and the weighted mean of the new
// u's component pc is reduced into *umean (sum of u(j, pc) w_j / domain) when
// w is set.
struct PfArgs
{
  int pc;              // filtered component, -1: none
  const double* hmean; // subtract from h(., pc) on read, or null
  const double* w;     // weights for the mean of the result, or null
  double domain;
  double* partials;
  unsigned* ticket;
  double* umean;
};

template<int B, class TV, class T>
__global__ void __launch_bounds__(256)
k_block_jacobi_apply(int n, const TV* __restrict__ dinv, const T* __restrict__ h,
                     T* __restrict__ u, double omega, int u_zero, PfArgs pf)
{
  GB_PDL_ENTRY();
  using TA = typename Acc<TV, T>::type;
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double wv = 0.0;
  if (i < n) {
    const int64_t o = int64_t(i) * B;
    const double hm = pf.hmean ? *pf.hmean : 0.0;
    TA t[B];
#pragma unroll
    for (int k = 0; k < B; ++k)
      t[k] = (pf.hmean && k == pf.pc)
               ? static_cast<TA>(static_cast<double>(h[o + k]) - hm)
               : static_cast<TA>(h[o + k]);
#pragma unroll
    for (int r = 0; r < B; ++r) {
      TA v = TA(0);
#pragma unroll
      for (int k = 0; k < B; ++k)
        v = fma(static_cast<TA>(dinv[o * B + r * B + k]), t[k], v);
      const TA base = u_zero ? TA(0) : static_cast<TA>(u[o + r]);
      const T un = static_cast<T>(base + static_cast<TA>(omega) * v);
      u[o + r] = un;
      if (pf.w && r == pf.pc)
        wv = static_cast<double>(un) * pf.w[i];
    }
  }
  if (pf.w) {
    wv = block_sum(wv, sh);
    red_finish(pf.partials, pf.ticket, wv, RedOut{ pf.umean, nullptr, nullptr, 0, pf.domain },
               sh);
  }
}

// Block transfers: the scalar tables applied to each of the B components.
// acc holds the starting values (0, or the target for an in-place add: the
// weights are powers of two, so each fused add rounds like the reference's
// y += w x).
template<class T, int B>
__device__ __forceinline__ void
transfer_row_b(const int* __restrict__ tsp, const uint32_t* __restrict__ tent,
               const T* __restrict__ src, int i, T (&acc)[B], int pc = -1,
               double smean = 0.0)
{
  const int beg = __ldg(tsp + (i >> 5));
  const int w = (__ldg(tsp + (i >> 5) + 1) - beg) >> 5;
  const uint32_t* ep = tent + beg + (i & 31);
  for (int j = 0; j < w; ++j) {
    const uint32_t e = __ldg(ep + j * kSlice);
    const T wgt = wcode<T>(e);
    const T* sp = src + int64_t(e & kIdxMask) * B;
#pragma unroll
    for (int c = 0; c < B; ++c) {
      const T sv = c == pc ? static_cast<T>(static_cast<double>(__ldg(sp + c)) - smean)
                           : __ldg(sp + c);
      acc[c] = fma(wgt, sv, acc[c]);
    }
  }
}

// fine's component pc is read minus *smean when smean is set (the filtered
// residual of MatrixResidual, restricted).
template<class T, int B>
__global__ void
k_restrict_b(int nc, const int* __restrict__ tsp, const uint32_t* __restrict__ tent,
             const T* __restrict__ fine, T* __restrict__ coarse,
             const uint8_t* __restrict__ cdir, int pc = -1,
             const double* __restrict__ smean = nullptr)
{
  GB_PDL_ENTRY();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nc)
    return;
  T acc[B];
#pragma unroll
  for (int c = 0; c < B; ++c)
    acc[c] = T(0);
  transfer_row_b<T, B>(tsp, tent, fine, i, acc, smean ? pc : -1, smean ? *smean : 0.0);
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
// The local solves apply each patch's inverse (formed once per assembly from
// its LU factors): one warp per patch, lane i computing rows i, i+32, ..;
// the inverse is stored transposed per patch ([patch][j][i]) so that for each
// column j the warp's loads are contiguous; the patch's right-hand side
// (component pc read minus *hmean when set) is staged in shared memory.
constexpr int kVankaMaxM = 128;
constexpr int kVankaWarps = 4;

// Per assembly, the patches' local matrices and their inverses on the device
// (VankaSmoother::copy_entries_sparseblockmatrix, LinAlg/vankasmoother.cc:
// 65-113, then the LU solves of VankaSmoother::solve, :192-237, applied to the
// unit vectors). One CTA per patch, the M x M matrix in shared memory:
//  - gather: entry (B r + cr, B q + cc) from the level's FP64 SELL values at
//    map[p][r][q] + 32 (cr B + cc) (a host-built offset per node pair of the
//    patch, -1 where the matrix holds no block), zero elsewhere;
//  - LU with partial pivoting in the order of the partial-pivot LU the
//    reference calls (pivot = the first row of largest |a_ik|, rows swapped,
//    column scaled by the pivot when it is nonzero, rank-1 update of the
//    trailing block), each product and difference rounded separately;
//  - column j of the inverse (thread j): forward substitution with the unit
//    lower factor on P e_j, backward with the upper, the same operation order;
//    stored transposed ([patch][j][i]), FP64 and FP32.
// The result equals the host factorisation of the same arithmetic bit for bit.
constexpr int kVankaFactorThreads = 128;

static __global__ void __launch_bounds__(kVankaFactorThreads)
k_vanka_factor(int npatch, int npp, int B, int M, const int* __restrict__ map,
               const double* __restrict__ val, double* __restrict__ inv64,
               float* __restrict__ inv32)
{
  GB_PDL_ENTRY();
  extern __shared__ double sm_vf[];
  const int ld = M + 1;
  double* A = sm_vf;                                   // [M][M + 1]
  int* pv = reinterpret_cast<int*>(A + M * ld);        // [M]
  __shared__ int s_piv;
  const int p = blockIdx.x;
  if (p >= npatch)
    return; // whole CTA
  const int t = threadIdx.x, nt = blockDim.x;
  for (int e = t; e < M * M; e += nt) {
    const int i = e / M, jc = e - i * M;
    const int r = i / B, cr = i - r * B, q = jc / B, cc = jc - q * B;
    const int base = __ldg(map + (int64_t(p) * npp + r) * npp + q);
    A[i * ld + jc] = base < 0 ? 0.0 : __ldg(val + int64_t(base) + int64_t(kSlice) * (cr * B + cc));
  }
  for (int i = t; i < M; i += nt)
    pv[i] = i;
  __syncthreads();
  for (int k = 0; k < M; ++k) {
    if (t == 0) {
      int piv = k;
      double best = fabs(A[k * ld + k]);
      for (int i = k + 1; i < M; ++i) {
        const double v = fabs(A[i * ld + k]);
        if (v > best) {
          best = v;
          piv = i;
        }
      }
      s_piv = piv;
      if (piv != k) {
        const int tmp = pv[k];
        pv[k] = pv[piv];
        pv[piv] = tmp;
      }
    }
    __syncthreads();
    const int piv = s_piv;
    if (piv != k)
      for (int j = t; j < M; j += nt) {
        const double tmp = A[k * ld + j];
        A[k * ld + j] = A[piv * ld + j];
        A[piv * ld + j] = tmp;
      }
    __syncthreads();
    const double akk = A[k * ld + k];
    if (akk != 0.0)
      for (int i = k + 1 + t; i < M; i += nt)
        A[i * ld + k] = __ddiv_rn(A[i * ld + k], akk);
    __syncthreads();
    const int rem = M - k - 1;
    for (int e = t; e < rem * rem; e += nt) {
      const int i = k + 1 + e / rem, j = k + 1 + e % rem;
      A[i * ld + j] = __dsub_rn(A[i * ld + j], __dmul_rn(A[i * ld + k], A[k * ld + j]));
    }
    __syncthreads();
  }
  for (int j = t; j < M; j += nt) {
    double* x = inv64 + (int64_t(p) * M + j) * M; // the column, built in place
    for (int i = 0; i < M; ++i)
      x[i] = pv[i] == j ? 1.0 : 0.0;
    for (int i = 1; i < M; ++i) {
      double sacc = x[i];
      for (int q = 0; q < i; ++q)
        sacc = __dsub_rn(sacc, __dmul_rn(A[i * ld + q], x[q]));
      x[i] = sacc;
    }
    for (int i = M - 1; i >= 0; --i) {
      double sacc = x[i];
      for (int q = i + 1; q < M; ++q)
        sacc = __dsub_rn(sacc, __dmul_rn(A[i * ld + q], x[q]));
      x[i] = __ddiv_rn(sacc, A[i * ld + i]);
    }
    float* y = inv32 + (int64_t(p) * M + j) * M;
    for (int i = 0; i < M; ++i)
      y[i] = static_cast<float>(x[i]);
  }
}

template<int R, class TL, class T>
__global__ void __launch_bounds__(32 * kVankaWarps)
k_vanka_inv(int npatch, int M, int B, const int* __restrict__ pn,
            const TL* __restrict__ inv, const T* __restrict__ h, int pc,
            const double* __restrict__ hmean, T* __restrict__ hout)
{
  GB_PDL_ENTRY();
  using TA = typename Acc<TL, T>::type;
  __shared__ TA sH[kVankaWarps][kVankaMaxM];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = blockIdx.x * kVankaWarps + wid;
  if (p >= npatch)
    return; // whole warp
  const int64_t np = npatch;
  TA* H = sH[wid];
  const double hm = hmean ? *hmean : 0.0;
  for (int i = lane; i < M; i += 32) {
    const int r = i / B, c = i - r * B;
    const int node = __ldg(pn + r * np + p);
    const T hv = __ldg(h + int64_t(node) * B + c);
    H[i] = (hmean && c == pc) ? static_cast<TA>(static_cast<double>(hv) - hm)
                              : static_cast<TA>(hv);
  }
  __syncwarp();
  const TL* ip = inv + int64_t(p) * M * M + lane;
  TA acc[R];
#pragma unroll
  for (int k = 0; k < R; ++k)
    acc[k] = TA(0);
#pragma unroll 3
  for (int j = 0; j < M; ++j) {
    const TA hj = H[j];
#pragma unroll
    for (int k = 0; k < R; ++k)
      if (lane + 32 * k < M)
        acc[k] = fma(static_cast<TA>(__ldg(ip + j * M + 32 * k)), hj, acc[k]);
  }
#pragma unroll
  for (int k = 0; k < R; ++k)
    if (lane + 32 * k < M)
      hout[int64_t(p) * M + lane + 32 * k] = static_cast<T>(acc[k]);
}

// The same for a patch size known at compile time (M <= 32: one row per lane):
// every load of the warp's 27 (or 9) inverse columns is issued up front.
template<int M, class TL, class T>
__global__ void __launch_bounds__(32 * kVankaWarps)
k_vanka_inv_ct(int npatch, int B, const int* __restrict__ pn, const TL* __restrict__ inv,
               const T* __restrict__ h, int pc, const double* __restrict__ hmean,
               T* __restrict__ hout)
{
  GB_PDL_ENTRY();
  static_assert(M <= 32, "one row per lane");
  using TA = typename Acc<TL, T>::type;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = blockIdx.x * kVankaWarps + wid;
  if (p >= npatch)
    return; // whole warp
  const int64_t np = npatch;
  const bool act = lane < M;
  // this lane's row of the inverse (column j at ip[j * M]) and its residual entry
  const TL* ip = inv + int64_t(p) * M * M + (act ? lane : 0);
  TL a[M];
#pragma unroll
  for (int j = 0; j < M; ++j)
    a[j] = __ldg(ip + j * M);
  TA hv = TA(0);
  if (act) {
    const int r = lane / B, c = lane - r * B;
    const int node = __ldg(pn + r * np + p);
    const T x = __ldg(h + int64_t(node) * B + c);
    hv = (hmean && c == pc) ? static_cast<TA>(static_cast<double>(x) - *hmean)
                            : static_cast<TA>(x);
  }
  TA acc = TA(0);
#pragma unroll
  for (int j = 0; j < M; ++j)
    acc = fma(static_cast<TA>(a[j]), __shfl_sync(0xffffffffu, hv, j), acc);
  if (act)
    hout[int64_t(p) * M + lane] = static_cast<T>(acc);
}

// u(i, c) = (u_zero ? 0 : u(i, c)) + omega * ((sum over the node's patches of
// their solution at (i, c)) * (1 / count)). ent packs (patch, local node):
// patch * 32 + r (npp <= 27). Solution (patch p, local dof q) at
// hout[q * s1 + p * s2].
template<int B, class T>
__global__ void __launch_bounds__(256)
k_vanka_gather(int n, const int* __restrict__ nptr, const int* __restrict__ ent,
               const T* __restrict__ hout, int M, T* __restrict__ u, double omega,
               int u_zero, PfArgs pf)
{
  GB_PDL_ENTRY();
  using TA = typename Acc<T, T>::type;
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double wv = 0.0;
  if (i < n) {
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
        acc[c] += static_cast<TA>(hout[p * M + r * B + c]);
    }
    const TA sc = TA(1) / static_cast<TA>(k1 - k0);
#pragma unroll
    for (int c = 0; c < B; ++c) {
      const int64_t d = int64_t(i) * B + c;
      const TA base = u_zero ? TA(0) : static_cast<TA>(u[d]);
      const T un = static_cast<T>(base + static_cast<TA>(omega) * (acc[c] * sc));
      u[d] = un;
      if (pf.w && c == pf.pc)
        wv = static_cast<double>(un) * pf.w[i];
    }
  }
  if (pf.w) {
    wv = block_sum(wv, sh);
    red_finish(pf.partials, pf.ticket, wv, RedOut{ pf.umean, nullptr, nullptr, 0, pf.domain },
               sh);
  }
}

} // namespace gb

namespace gb {

// ------------------------------------------------------------ hanging nodes
//
// HNStructureQ12d/Q13d/Q22d/Q23d (Discretization/Q1/hnstructureq12d.cc,
// hnstructureq13d.cc, Discretization/Q2/hnstructureq22d.cc,
// hnstructureq23d.cc) act in phases (edges, faces, in the discretisation's
// order); within a phase no hanging node is a parent of another. Products and
// sums are rounded separately (no fused multiply-add) and associated as
// CompVector::equ_node/add_node write them, so the FP64 results are the
// reference's bit for bit.
__device__ __forceinline__ double hn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double hn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float hn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float hn_add(float a, float b) { return __fadd_rn(a, b); }

// u(h) = sum over groups (left to right inside a group, groups added in
// turn); parents slot-major: par[s * nh + k], weights w[s].
template<class T>
__global__ void
k_hn_average(int nh, int B, const int* __restrict__ node, const int* __restrict__ par,
             int nslots, int gsize, const double* __restrict__ w, T* __restrict__ u)
{
  GB_PDL_ENTRY();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nh)
    return;
  for (int c = 0; c < B; ++c) {
    T acc = T(0);
    for (int g = 0; g < nslots; g += gsize) {
      T sg = hn_mul(static_cast<T>(w[g]), u[int64_t(par[g * nh + k]) * B + c]);
      for (int s = g + 1; s < g + gsize; ++s)
        sg = hn_add(sg, hn_mul(static_cast<T>(w[s]), u[int64_t(par[s * nh + k]) * B + c]));
      acc = g == 0 ? sg : hn_add(acc, sg);
    }
    u[int64_t(node[k]) * B + c] = acc;
  }
}

// parents += w * u(h) in ascending hanging-node order (one thread per parent:
// its contributions in the reference's sequence)
template<class T>
__global__ void
k_hn_distribute(int np, int B, const int* __restrict__ pnode, const int* __restrict__ ptr,
                const int* __restrict__ hnode, const double* __restrict__ wt,
                T* __restrict__ u)
{
  GB_PDL_ENTRY();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= np)
    return;
  const int64_t p = pnode[k];
  for (int c = 0; c < B; ++c) {
    T acc = u[p * B + c];
    for (int e = ptr[k]; e < ptr[k + 1]; ++e)
      acc = hn_add(acc, hn_mul(static_cast<T>(wt[e]), u[int64_t(hnode[e]) * B + c]));
    u[p * B + c] = acc;
  }
}

template<class T>
__global__ void
k_hn_zero(int nh, int B, const int* __restrict__ node, T* __restrict__ u)
{
  GB_PDL_ENTRY();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nh)
    return;
  for (int c = 0; c < B; ++c)
    u[int64_t(node[k]) * B + c] = T(0);
}

// --------------------------------------------------------- block ILU

template<class T>
__device__ __forceinline__ T ilu_mul(T a, T b);
template<>
__device__ __forceinline__ double ilu_mul(double a, double b) { return __dmul_rn(a, b); }
template<>
__device__ __forceinline__ float ilu_mul(float a, float b) { return __fmul_rn(a, b); }
template<class T>
__device__ __forceinline__ T ilu_sub(T a, T b);
template<>
__device__ __forceinline__ double ilu_sub(double a, double b) { return __dsub_rn(a, b); }
template<>
__device__ __forceinline__ float ilu_sub(float a, float b) { return __fsub_rn(a, b); }
template<class T>
__device__ __forceinline__ T ilu_add(T a, T b);
template<>
__device__ __forceinline__ double ilu_add(double a, double b) { return __dadd_rn(a, b); }
template<>
__device__ __forceinline__ float ilu_add(float a, float b) { return __fadd_rn(a, b); }

// SparseBlockIlu::compute_ilu (LinAlg/sparseblockilu.xx:246-275) on the
// device, one dependency level per launch, one thread per row: a row waits
// only for the rows of its lower part (earlier levels), exactly as in the
// forward substitution. Each row runs the host factorisation's steps in its
// order: for every lower entry k ascending, a(i,k) times the inverted
// diagonal block of row k, then a(i,j) -= a(i,k) a(k,j) over row k's upper
// entries (the target found by a search of row i), and finally the
// Gauss-Jordan inverse of the diagonal block; products and sums rounded
// separately, as on the host: the factors are the host's bit for bit.
template<int B>
__global__ void __launch_bounds__(128)
k_ilu_factor(int nr, const int* __restrict__ rows, const int* __restrict__ ptr,
             const int* __restrict__ col, const int* __restrict__ diag,
             double* __restrict__ v)
{
  GB_PDL_ENTRY();
  constexpr int B2 = B * B;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nr)
    return;
  const int i = rows[t];
  const int pb = ptr[i], pe = ptr[i + 1], pd = diag[i];
  double tmp[B2];
  for (int pk = pb; pk < pd; ++pk) {
    const int k = col[pk];
    double* a = v + int64_t(pk) * B2;
    const double* dk = v + int64_t(diag[k]) * B2;
#pragma unroll
    for (int q = 0; q < B2; ++q)
      tmp[q] = a[q];
#pragma unroll
    for (int r = 0; r < B; ++r)
#pragma unroll
      for (int cc = 0; cc < B; ++cc) {
        double acc = 0.0;
#pragma unroll
        for (int u = 0; u < B; ++u)
          acc = rn_add(acc, rn_mul(tmp[r * B + u], dk[u * B + cc]));
        a[r * B + cc] = acc;
      }
    const int ke = ptr[k + 1];
    for (int pj = diag[k] + 1; pj < ke; ++pj) {
      const int j = col[pj];
      for (int ph = pb; ph < pe; ++ph) {
        if (col[ph] != j)
          continue;
        double* h = v + int64_t(ph) * B2;
        const double* cj = v + int64_t(pj) * B2;
#pragma unroll
        for (int r = 0; r < B; ++r)
#pragma unroll
          for (int cc = 0; cc < B; ++cc)
#pragma unroll
            for (int u = 0; u < B; ++u)
              h[r * B + cc] = rn_sub(h[r * B + cc], rn_mul(a[r * B + u], cj[u * B + cc]));
        break;
      }
    }
  }
  gauss_jordan<B>(v + int64_t(pd) * B2);
}

// The ILU's values in its row-sorted layout from the level's SELL values:
// entry e, component q at val[map[e] + 32 q].
static __global__ void
k_ilu_gather(int64_t nnz, int B2, const int* __restrict__ map,
             const double* __restrict__ val, double* __restrict__ v)
{
  GB_PDL_ENTRY();
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < nnz;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t base = map[e];
    for (int q = 0; q < B2; ++q)
      v[e * B2 + q] = __ldg(val + base + int64_t(kSlice) * q);
  }
}

static __global__ void
k_to_float(int64_t n, const double* __restrict__ a, float* __restrict__ b)
{
  GB_PDL_ENTRY();
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    b[i] = static_cast<float>(a[i]);
}

// FP64 rows one entry at a time: groups of 4 FP64 entries measured slower
// (C2 ILU solve 240 against 168 ms with a launch per level), FP32 groups of 8
// faster (123.9 against 133.7 ms)
#ifndef GB_ILU_GROUP_F64
#define GB_ILU_GROUP_F64 1
#endif

// One row of a substitution. Forward, with the unit lower factor
// (SparseBlockIlu::forward, LinAlg/sparseblockilu.xx:202-214): y_i -= L_ik y_k
// over the row's lower blocks in stored (ascending column) order, block
// entries as FMatrixBlock::subtract (LinAlg/fmatrixblock.h:136-145).
// Backward (SparseBlockIlu::backward, LinAlg/sparseblockilu.xx:217-231):
// y_i -= U_ik y_k over the upper blocks in descending order, then
// y_i = D_i^-1 y_i with the inverted diagonal block (FMatrixBlock::vmult,
// LinAlg/fmatrixblock.h:194-217). The entries are taken G at a time: their
// columns, then their y blocks and values are loaded together before the
// subtractions run in the reference's order, so a row waits for about two
// memory round trips per G entries instead of one per entry. The rows of one
// dependency level depend only on rows of earlier levels, so running the
// levels in order gives the sequential sweep bit for bit.
template<int B, class T, bool UP>
__device__ __forceinline__ void
ilu_row(int i, const int* __restrict__ ptr, const int* __restrict__ col,
        const int* __restrict__ diag, const T* __restrict__ val, T* __restrict__ y)
{
  constexpr int B2 = B * B;
  // the G value blocks of a group take at most 32 registers; FP64 rows take
  // GB_ILU_GROUP_F64 entries at a time at most
  constexpr int G0 = 32 / (B2 * int(sizeof(T) / 4));
  constexpr int GM = sizeof(T) == 8 ? GB_ILU_GROUP_F64 : 8;
  constexpr int G = G0 < 1 ? 1 : (G0 > GM ? GM : G0);
  T yi[B];
#pragma unroll
  for (int r = 0; r < B; ++r)
    yi[r] = y[int64_t(i) * B + r];
  const int d = __ldg(diag + i);
  const int first = UP ? __ldg(ptr + i + 1) - 1 : __ldg(ptr + i);
  const int cnt = UP ? first - d : d - first;
  for (int q0 = 0; q0 < cnt; q0 += G) {
    int pos[G];
    int64_t k[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      pos[g] = UP ? first - (q0 + g) : first + (q0 + g);
      k[g] = q0 + g < cnt ? __ldg(col + pos[g]) : i; // past the end: a harmless load of y_i
    }
    T yk[G][B], m[G][B2];
#pragma unroll
    for (int g = 0; g < G; ++g) {
#pragma unroll
      for (int c = 0; c < B; ++c)
        yk[g][c] = y[k[g] * B + c];
#pragma unroll
      for (int q = 0; q < B2; ++q)
        m[g][q] = q0 + g < cnt ? __ldg(val + int64_t(pos[g]) * B2 + q) : T(0);
    }
#pragma unroll
    for (int g = 0; g < G; ++g)
      if (q0 + g < cnt) {
#pragma unroll
        for (int r = 0; r < B; ++r)
#pragma unroll
          for (int c = 0; c < B; ++c)
            yi[r] = ilu_sub(yi[r], ilu_mul(m[g][r * B + c], yk[g][c]));
      }
  }
  if (!UP) {
#pragma unroll
    for (int r = 0; r < B; ++r)
      y[int64_t(i) * B + r] = yi[r];
    return;
  }
  const T* D = val + int64_t(d) * B2;
#pragma unroll
  for (int r = 0; r < B; ++r) {
    T acc = ilu_mul(__ldg(D + r * B), yi[0]);
#pragma unroll
    for (int c = 1; c < B; ++c)
      acc = ilu_add(acc, ilu_mul(__ldg(D + r * B + c), yi[c]));
    y[int64_t(i) * B + r] = acc;
  }
}

// One wide dependency level of a substitution, one thread per row.
template<int B, class T, bool UP>
__global__ void
k_ilu_level(int nr, const int* __restrict__ rows, const int* __restrict__ ptr,
            const int* __restrict__ col, const int* __restrict__ diag,
            const T* __restrict__ val, T* __restrict__ y)
{
  GB_PDL_ENTRY();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nr)
    return;
  ilu_row<B, T, UP>(__ldg(rows + t), ptr, col, diag, val, y);
}

__device__ __forceinline__ void
prefetch_l1(const void* p)
{
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// The consecutive narrow levels lv0..lv1-1 of a substitution in one CTA: the
// levels run in order with a block barrier between them, which makes the rows
// one level wrote visible to the threads of the next (y is read by coherent
// loads). Per level a thread takes rows t, t + 1024, ... of the level. Before
// the barrier it fetches the first row of its next level, that row's entry
// range and the cache lines of the row's columns and values into L1, so that
// after the barrier only the loads of y wait on the previous level. The rows
// run the same arithmetic in the same order as k_ilu_level's.
template<int B, class T, bool UP>
__global__ void __launch_bounds__(kIluCtaThreads, 1)
k_ilu_levels(int lv0, int lv1, const int* __restrict__ lptr, const int* __restrict__ rows,
             const int* __restrict__ ptr, const int* __restrict__ col,
             const int* __restrict__ diag, const T* __restrict__ val, T* __restrict__ y)
{
  GB_PDL_ENTRY();
  int o0 = __ldg(lptr + lv0), o1 = __ldg(lptr + lv0 + 1);
  for (int lv = lv0; lv < lv1; ++lv) {
    for (int t = o0 + threadIdx.x; t < o1; t += kIluCtaThreads)
      ilu_row<B, T, UP>(__ldg(rows + t), ptr, col, diag, val, y);
    int o2 = o1;
    if (lv + 1 < lv1) {
      o2 = __ldg(lptr + lv + 2);
      const int t = o1 + threadIdx.x;
      if (t < o2) {
        const int i = __ldg(rows + t);
        const int pb = __ldg(ptr + i), pe = __ldg(ptr + i + 1) - 1;
        prefetch_l1(col + pb);
        prefetch_l1(col + pe);
        prefetch_l1(val + int64_t(pb) * B * B);
        prefetch_l1(val + (int64_t(pb + pe) / 2) * B * B);
        prefetch_l1(val + (int64_t(pe) + 1) * B * B - 1);
      }
    }
    __syncthreads();
    o0 = o1;
    o1 = o2;
  }
}

// u = (u_zero ? 0 : u) + omega h (StdSolver::Add after the ILU solve, unfused)
template<class T>
__global__ void
k_ilu_axpy(int64_t n, T* __restrict__ u, double omega, const T* __restrict__ h, int u_zero)
{
  GB_PDL_ENTRY();
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n)
    return;
  const T w = ilu_mul(static_cast<T>(omega), h[i]);
  u[i] = u_zero ? w : ilu_add(u[i], w);
}

} // namespace gb
