// Device kernels of the B200 linear-solve path (sm_100a). All kernels are
// HBM/L2-bandwidth or latency bound: sparse matrix-vector products, pointwise
// smoother updates, gather-form transfers and deterministic reductions. None is a
// dense contraction large enough for the tensor cores.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gb {

constexpr int kSlice = 32;          // SELL slice height = warp size
constexpr int kSpmvThreads = 256;   // 8 warps = 8 slices per CTA
constexpr int kRedThreads = 256;
constexpr int kMaxRedBlocks = 2 * 148;
constexpr int kMaxV = 128;          // largest gmressize supported

// SpMV epilogue modes
enum SpmvMode
{
  kAx = 0,       // y = alpha * (A x)
  kAddAx = 1,    // y = y + alpha * (A x)
  kResid = 2,    // y = b - A x
  kResidDir = 3, // y = b - A x, then 0 on Dirichlet dofs
  kJacobi = 4    // y = x + alpha * dinv * (b - A x)     (y != x)
};

// Accumulator type: FP64 when matrix or output is FP64, FP32 only when
// everything is FP32 (the FP32 V-cycle with FP32 accumulation).
template<class TV, class TO>
struct Acc
{
  using type = double;
};
template<>
struct Acc<float, float>
{
  using type = float;
};

template<class T>
__device__ __forceinline__ T ldg(const T* p)
{
  return __ldg(p);
}

// Device view of one SELL-32 matrix. Slice s holds rows 32s..32s+31,
// column-major: entry j of lane l at sptr[s] + 32 j + l. Column indices are
// either explicit (col) or, when the rows of the level share few column-offset
// patterns, implicit: row + ptab[pid[row] * W + j] (pattern-compressed SELL).
template<class TV>
struct SellView
{
  int n;
  const int* sptr;
  const int* col;      // explicit columns, or null
  const uint8_t* pid;  // pattern id per row, or null
  const int* ptab;     // [npatterns][W] offsets col - row (0-padded)
  int W;
  const TV* val;
};

// y = f(A x) for one row per thread, columns in the reference's stored order.
// Loads are issued in predicated chunks of kChunk entries so that a thread keeps
// kChunk value loads and kChunk gathers of x in flight.
// Optional device-indexed output (flexible GMRES, graph-resident): when yidx is
// set, y += (*yidx + 1) * ystride and x[row] is also copied to
// xcopy + (*yidx) * ystride.
constexpr int kChunk = 16;

template<int MODE, class TV, class TX, class TO, bool PAT>
__global__ void __launch_bounds__(kSpmvThreads)
k_spmv(SellView<TV> A, const TX* __restrict__ x, TO* __restrict__ y,
       const TO* __restrict__ b, const TV* __restrict__ dinv,
       const uint8_t* __restrict__ dirmask, double alpha_,
       const int* __restrict__ yidx, int64_t ystride, TX* __restrict__ xcopy)
{
  using TA = typename Acc<TV, TO>::type;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= A.n)
    return;
  const int s = row >> 5, lane = row & 31;
  const int beg = A.sptr[s];
  const int w = (A.sptr[s + 1] - beg) >> 5;
  const TV* vp = A.val + beg + lane;
  const int* cp = PAT ? (A.ptab + int(A.pid[row]) * A.W) : (A.col + beg + lane);
  const TA alpha = static_cast<TA>(alpha_);
  constexpr bool NEG = (MODE == kResid || MODE == kResidDir || MODE == kJacobi);
  TA acc = NEG ? static_cast<TA>(b[row]) : TA(0);
  for (int j0 = 0; j0 < w; j0 += kChunk) {
    TA av[kChunk], xv[kChunk];
#pragma unroll
    for (int q = 0; q < kChunk; ++q) {
      const int j = j0 + q;
      if (j < w) {
        const int c = PAT ? row + ldg(cp + j) : ldg(cp + j * kSlice);
        av[q] = static_cast<TA>(ldg(vp + j * kSlice));
        xv[q] = static_cast<TA>(ldg(x + c));
      } else {
        av[q] = TA(0);
        xv[q] = TA(0);
      }
    }
#pragma unroll
    for (int q = 0; q < kChunk; ++q)
      acc = NEG ? fma(-av[q], xv[q], acc) : fma(av[q], xv[q], acc);
  }
  if (yidx) {
    const int64_t jj = *yidx;
    xcopy[jj * ystride + row] = x[row];
    y += (jj + 1) * ystride;
  }
  if (MODE == kAx) {
    y[row] = static_cast<TO>(alpha * acc);
  } else if (MODE == kAddAx) {
    y[row] = static_cast<TO>(static_cast<TA>(y[row]) + alpha * acc);
  } else if (MODE == kResid) {
    y[row] = static_cast<TO>(acc);
  } else if (MODE == kResidDir) {
    y[row] = dirmask[row] ? TO(0) : static_cast<TO>(acc);
  } else { // kJacobi: reference order h = d*h; x = x + omega*h
    const TA h = static_cast<TA>(dinv[row]) * acc;
    y[row] = static_cast<TO>(static_cast<TA>(x[row]) + alpha * h);
  }
}

// First Jacobi sweep from x = 0: x = omega * (dinv * b); b - A*0 == b exactly.
template<class TV, class T>
__global__ void
k_jacobi_from_zero(int n, const TV* __restrict__ dinv, const T* __restrict__ b,
                   T* __restrict__ x, double omega)
{
  using TA = typename Acc<TV, T>::type;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    x[i] = static_cast<T>(static_cast<TA>(omega) *
                          (static_cast<TA>(dinv[i]) * static_cast<TA>(b[i])));
}

// Transfer weights are exact powers of two: packed entry = index | code << 29,
// weight = 2^-code (1, 1/2, 1/4, 1/8).
constexpr int kWShift = 29;
constexpr uint32_t kIdxMask = (1u << kWShift) - 1u;

template<class T>
__device__ __forceinline__ T wcode(uint32_t e)
{
  const uint32_t c = e >> kWShift;
  return c == 0 ? T(1) : c == 1 ? T(0.5) : c == 2 ? T(0.25) : T(0.125);
}

// coarse = R fine (gather over the coarse row, ascending fine index, as
// MgInterpolatorMatrix::restrict_zero), then 0 on coarse Dirichlet dofs.
template<class T>
__global__ void
k_restrict(int nc, const int* __restrict__ rptr, const uint32_t* __restrict__ rent,
           const T* __restrict__ fine, T* __restrict__ coarse,
           const uint8_t* __restrict__ cdir)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nc)
    return;
  T acc = T(0);
  for (int k = rptr[i]; k < rptr[i + 1]; ++k) {
    uint32_t e = rent[k];
    acc = fma(wcode<T>(e), ldg(fine + (e & kIdxMask)), acc);
  }
  coarse[i] = (cdir && cdir[i]) ? T(0) : acc;
}

// Plain restriction without the Dirichlet step (gb_restrict_zero).
// fine += P coarse (gather over the fine row's parents, ascending), optionally
// masked by the fine Dirichlet dofs and scaled: MODE 0: fine += P c;
// MODE 1 (coarse-grid correction): u += mgomega * (dir ? 0 : P c).
template<int MODE, class T>
__global__ void
k_prolong(int nf, const int* __restrict__ pptr, const uint32_t* __restrict__ pent,
          const T* __restrict__ coarse, T* __restrict__ fine,
          const uint8_t* __restrict__ fdir, double mgomega)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nf)
    return;
  T acc = T(0);
  for (int k = pptr[i]; k < pptr[i + 1]; ++k) {
    uint32_t e = pent[k];
    acc = fma(wcode<T>(e), ldg(coarse + (e & kIdxMask)), acc);
  }
  if (MODE == 0) {
    fine[i] = fine[i] + acc;
  } else {
    if (fdir && fdir[i])
      acc = T(0);
    fine[i] = fine[i] + static_cast<T>(mgomega) * acc;
  }
}

// ------------------------------------------------------------- vectors

template<class T>
__global__ void
k_fill(int64_t n, T* __restrict__ y, T v)
{
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = v;
}

// y = s * x   (Equ)
template<class TI, class TO>
__global__ void
k_equ(int64_t n, TO* __restrict__ y, double s, const TI* __restrict__ x)
{
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = static_cast<TO>(s * static_cast<double>(x[i]));
}

// y = (TO) x   (precision conversion)
template<class TI, class TO>
__global__ void
k_convert(int64_t n, TO* __restrict__ y, const TI* __restrict__ x)
{
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = static_cast<TO>(x[i]);
}

// y += s * x   (Add)
__global__ void
k_add(int64_t n, double* __restrict__ y, double s, const double* __restrict__ x)
{
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = fma(s, x[i], y[i]);
}

// y *= *scale (device scalar): Equ(v, 1/s, v) with the reciprocal formed first
__global__ void
k_scale_dev(int64_t n, double* __restrict__ y, const double* __restrict__ scale)
{
  const double s = *scale;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = s * y[i];
}

// y(dir dofs) = 0
template<class T>
__global__ void
k_dirichlet_zero(int nd, const int* __restrict__ dofs, T* __restrict__ y)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nd)
    y[dofs[i]] = T(0);
}

// x += sum_i coef[i] * V_i, i = 0..k-1 in order (GMRES::solution); V_i at
// base + i*stride; coefficients on the device; TV: FP64 basis or FP32 (Z).
template<class TV>
__global__ void
k_multi_axpy(int64_t n, double* __restrict__ x, const TV* __restrict__ base,
             int64_t stride, const double* __restrict__ coef, int k)
{
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double acc = x[i];
    for (int q = 0; q < k; ++q)
      acc = fma(coef[q], static_cast<double>(base[q * stride + i]), acc);
    x[i] = acc;
  }
}

// ----------------------------------------------------------- reductions
//
// Deterministic: each block sums a fixed grid-stride subset in order, reduces
// in a fixed tree, writes one partial; the last block to finish (atomic ticket)
// sums the partials in a fixed order. Same grid for the same n => same bits.

__device__ __forceinline__ double
block_sum(double v, double* sh)
{
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
    sh[wid] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  v = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
  if (wid == 0)
    for (int o = 16; o > 0; o >>= 1)
      v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  return v; // valid in thread 0
}

// What the last block does with the reduced value r.
struct RedOut
{
  double* out;      // out[0] = op(r)            (may be null)
  double* accum;    // accum[0] += op(r)         (may be null)
  double* recip;    // recip[0] = 1 / op(r)      (may be null)
  int sqrt_result;  // op = sqrt when set
};

__device__ __forceinline__ void
red_finish(double* partials, unsigned* ticket, double bsum, RedOut ro, double* sh)
{
  __shared__ bool am_last;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = bsum;
    __threadfence();
    unsigned t = atomicAdd(ticket, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last)
    return;
  __threadfence();
  double v = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x)
    v += __ldcg(partials + i);
  v = block_sum(v, sh);
  if (threadIdx.x == 0) {
    double r = ro.sqrt_result ? sqrt(v) : v;
    if (ro.out)
      ro.out[0] = r;
    if (ro.accum)
      ro.accum[0] += r;
    if (ro.recip)
      ro.recip[0] = 1.0 / r;
    *ticket = 0u;
  }
}

// r = <a, b> (TA, TB may be float or double; accumulation in FP64)
template<class TA, class TB>
__global__ void __launch_bounds__(kRedThreads)
k_dot(int64_t n, const TA* __restrict__ a, const TB* __restrict__ b,
      double* partials, unsigned* ticket, RedOut ro)
{
  __shared__ double sh[32];
  double v = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    v = fma(static_cast<double>(a[i]), static_cast<double>(b[i]), v);
  v = block_sum(v, sh);
  red_finish(partials, ticket, v, ro, sh);
}

// Modified Gram-Schmidt step (GMRES::orthogonalization, LinAlg/gmres.cc:
// 108-118), fused: vv -= d * vi (if vi), then partial <vv, vnext>.
__global__ void __launch_bounds__(kRedThreads)
k_mgs(int64_t n, double* __restrict__ vv, const double* __restrict__ vi,
      const double* __restrict__ dcoef, const double* __restrict__ vnext,
      double* partials, unsigned* ticket, RedOut ro)
{
  __shared__ double sh[32];
  const double d = vi ? *dcoef : 0.0;
  double v = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double t = vv[i];
    if (vi) {
      t = fma(-d, vi[i], t);
      vv[i] = t;
    }
    const double q = (vnext == vv) ? t : vnext[i];
    v = fma(t, q, v);
  }
  v = block_sum(v, sh);
  red_finish(partials, ticket, v, ro, sh);
}

// ------------------------------------------------------------- inverse

// Block-diagonal inverse by NodeMatrix::gauss_jordan (LinAlg/nodematrix.h:
// 159-213), same pivot order; one thread per node, the block in registers.
template<int B>
__global__ void
k_blockdiag_inverse(int n, const double* __restrict__ dblocks, double* __restrict__ dinv64,
                    float* __restrict__ dinv32)
{
  int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= n)
    return;
  double a[B * B];
  int p[B];
#pragma unroll
  for (int q = 0; q < B * B; ++q)
    a[q] = dblocks[(int64_t)node * B * B + q];
#define A_(i, j) a[(i) * B + (j)]
  for (int i = 0; i < B; i++)
    p[i] = i;
  for (int j = 0; j < B; j++) {
    double mx = fabs(A_(j, j));
    int r = j;
    for (int i = j + 1; i < B; i++)
      if (fabs(A_(i, j)) > mx) {
        mx = fabs(A_(i, j));
        r = i;
      }
    if (r > j) {
      for (int k = 0; k < B; k++) {
        double hr = A_(j, k);
        A_(j, k) = A_(r, k);
        A_(r, k) = hr;
      }
      int t = p[j];
      p[j] = p[r];
      p[r] = t;
    }
    double hr = 1. / A_(j, j);
    A_(j, j) = hr;
    for (int k = 0; k < B; k++) {
      if (k == j)
        continue;
      for (int i = 0; i < B; i++) {
        if (i == j)
          continue;
        A_(i, k) -= A_(i, j) * A_(j, k) * hr;
      }
    }
    for (int i = 0; i < B; i++) {
      A_(i, j) *= hr;
      A_(j, i) *= -hr;
    }
    A_(j, j) = hr;
  }
  for (int i = 0; i < B; i++) {
    double hv[B];
    for (int k = 0; k < B; k++)
      hv[p[k]] = A_(i, k);
    for (int k = 0; k < B; k++)
      A_(i, k) = hv[k];
  }
#undef A_
#pragma unroll
  for (int q = 0; q < B * B; ++q) {
    dinv64[(int64_t)node * B * B + q] = a[q];
    dinv32[(int64_t)node * B * B + q] = static_cast<float>(a[q]);
  }
}

// ---------------------------------------------------------- GMRES scalars

struct CGInfoDev
{
  double tol, globaltol, breaktol;
  int miniter, maxiter;
  int status; // 0 waiting 1 running 2 converged 3 too many 4 exploded
  double firstresidual, previousresidual, residual, aimedresidual;
  int iteration;
};

struct GmresDev
{
  double H[kMaxV][kMaxV + 1]; // H[col][row], as GMRES::H
  double gamma[kMaxV + 1], ci[kMaxV], si[kMaxV];
  double d[kMaxV + 1];        // MGS coefficients of the current pass
  double s;                   // ||vv|| of the current step
  double inv;                 // 1 / s (or 1 / rho for v0)
  double hs[kMaxV];           // back-substitution result
  double hist[kMaxV];         // |gamma| per step
  double bnorm, beta, xnorm;
  CGInfoDev info;
  int reached, need_reortho, zero_rho, pad;
  // graph-resident flexible GMRES
  double d2[kMaxV + 1];       // second CGS pass coefficients
  double beta_tmp;            // ||r|| of the current restart
  int j;                      // Arnoldi step of the current cycle
  int total;                  // Arnoldi steps over all cycles
  int restarts;               // refinement cycles started
  int stop, converged, pad2;
};

// CGInfo::check (Common/cginfo.cc:201-255); "diverging" cannot fire there.
__device__ inline int
cginfo_check(CGInfoDev& I, double resi)
{
  double res = fabs(resi);
  I.residual = res;
  if (I.status != 1) {
    I.firstresidual = res;
    I.previousresidual = res;
    I.aimedresidual = res * I.tol;
    I.status = 1;
  } else {
    I.previousresidual = res;
  }
  double aim = fmax(I.aimedresidual, I.globaltol);
  if (I.residual < aim)
    I.status = 2;
  else if (I.iteration >= I.maxiter)
    I.status = 3;
  else if (I.residual > I.breaktol)
    I.status = 4;
  I.iteration++;
  if (I.status == 1)
    return 0;
  if (I.iteration < I.miniter)
    return 0;
  return 1;
}

// gamma[0] = rho, inv = 1/rho (GMRES::solve, LinAlg/gmres.cc:182-192)
__global__ void
k_gmres_init(GmresDev* G, const double* rho_p)
{
  double rho = *rho_p;
  G->gamma[0] = rho;
  G->zero_rho = (rho == 0.0);
  G->inv = 1.0 / rho;
  G->reached = G->zero_rho;
}

// After the MGS pass of step `dim` (last = dim-1): reortho test
// (LinAlg/gmres.cc:122-135), 1/s, givens_rotation (:88-104), CGInfo check.
// mode 1 = left-preconditioned (CGInfo rule); mode 2 = flexible (stop when
// |gamma| <= tol * bnorm or maxsteps).
__global__ void
k_gmres_step(GmresDev* G, int dim, int second_pass, int mode, int maxsteps)
{
  const int last = dim - 1;
  double* h = G->H[last];
  const double s = h[dim];
  G->s = s;
  if (!second_pass && mode == 1) {
    double oldnorm = s;
    double newnorm = oldnorm + 1.e-3 * s;
    if (oldnorm == newnorm) {
      G->need_reortho = 1;
      return;
    }
  }
  G->need_reortho = 0;
  G->inv = 1.0 / s;
  for (int i = 0; i < last; i++) {
    double dummy = h[i];
    h[i] = G->ci[i] * dummy + G->si[i] * h[i + 1];
    h[i + 1] = -G->si[i] * dummy + G->ci[i] * h[i + 1];
  }
  double r = 1. / sqrt(h[last] * h[last] + h[last + 1] * h[last + 1]);
  G->si[last] = h[last + 1] * r;
  G->ci[last] = h[last] * r;
  h[last] = G->ci[last] * h[last] + G->si[last] * h[last + 1];
  G->gamma[last + 1] = -G->si[last] * G->gamma[last];
  G->gamma[last] *= G->ci[last];
  double rho = fabs(G->gamma[dim]);
  G->hist[dim - 1] = rho;
  if (mode == 1) {
    G->reached = cginfo_check(G->info, rho);
  } else {
    G->info.residual = rho;
    G->info.iteration++;
    int conv = rho <= G->info.tol * G->bnorm || rho < G->info.globaltol;
    G->reached = conv || dim >= maxsteps || !(rho == rho);
  }
}

// GMRES::solution's backward (Common/mult.h:130-141) on H1(i,j) = H[j][i].
__global__ void
k_gmres_backward(GmresDev* G, int dim)
{
  for (int i = dim - 1; i >= 0; i--) {
    double s = G->gamma[i];
    for (int j = i + 1; j < dim; j++)
      s -= G->hs[j] * G->H[j][i];
    G->hs[i] = s / G->H[i][i];
  }
}

// Flexible GMRES restart: gamma[0] = beta, inv = 1/beta, reset the Hessenberg.
__global__ void
k_fgmres_restart(GmresDev* G, const double* beta_p, int vmax)
{
  double beta = *beta_p;
  G->beta = beta;
  for (int j = 0; j < vmax && j < kMaxV; ++j) {
    for (int i = 0; i <= vmax && i <= kMaxV; ++i)
      G->H[j][i] = 0.0;
    G->ci[j] = 0.0;
    G->si[j] = 0.0;
  }
  for (int i = 0; i <= vmax && i <= kMaxV; ++i)
    G->gamma[i] = 0.0;
  G->gamma[0] = beta;
  G->inv = 1.0 / beta;
  G->zero_rho = (beta == 0.0);
  G->reached = 0;
}

// ------------------------------------------- graph-resident flexible GMRES
//
// The whole flexible GMRES solve is one CUDA graph: a conditional WHILE node runs
// the refinement cycles, a nested one the Arnoldi steps. Loop indices live in
// GmresDev; kernels read them, so the graph needs no host round trip.

constexpr int kCgsMaxJ = 32; // graph path: gmressize <= 33

__global__ void
k_fg_setup(GmresDev* G, double tol, double globaltol, int maxiter)
{
  G->info.tol = tol;
  G->info.globaltol = globaltol;
  G->info.maxiter = maxiter;
  G->info.status = 1;
  G->info.iteration = 0;
  G->info.residual = 0;
  G->total = 0;
  G->restarts = 0;
  G->j = 0;
  G->stop = 0;
  G->converged = 0;
}

// Refinement cycle start: beta = ||b - A x|| (in beta_tmp). Stops both loops
// when converged, out of iterations or non-finite; otherwise resets the
// Hessenberg system of the cycle.
__global__ void
k_fg_restart(GmresDev* G, cudaGraphConditionalHandle outer,
             cudaGraphConditionalHandle inner, int m, int maxrestarts)
{
  const double beta = G->beta_tmp;
  const double aim = fmax(G->info.tol * G->bnorm, G->info.globaltol);
  const int conv = (beta <= aim) || beta == 0.0;
  const int stop = conv || G->total >= G->info.maxiter ||
                   G->restarts >= maxrestarts || !(beta == beta);
  G->converged = conv;
  G->j = 0;
  if (G->restarts == 0)
    G->info.firstresidual = beta;
  G->info.residual = beta;
  if (stop) {
    G->stop = 1;
    G->inv = 0.0;
    G->info.status = conv ? 2 : 3;
    cudaGraphSetConditional(outer, 0);
    cudaGraphSetConditional(inner, 0);
    return;
  }
  for (int c = 0; c < m; ++c) {
    for (int r = 0; r <= m; ++r)
      G->H[c][r] = 0.0;
    G->ci[c] = 0.0;
    G->si[c] = 0.0;
  }
  for (int r = 0; r <= m; ++r)
    G->gamma[r] = 0.0;
  G->gamma[0] = beta;
  G->beta = beta;
  G->inv = 1.0 / beta;
  G->restarts += 1;
  cudaGraphSetConditional(inner, 1);
}

// y = (TO) V[(*jp) * n + i]   (Arnoldi vector j into the cycle's right-hand side)
template<class TO>
__global__ void
k_load_idx(int64_t n, TO* __restrict__ y, const double* __restrict__ V,
           const int* __restrict__ jp)
{
  const double* v = V + int64_t(*jp) * n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = static_cast<TO>(v[i]);
}

// V[(*jp) * n + i] *= *s
__global__ void
k_scale_idx(int64_t n, double* __restrict__ V, const int* __restrict__ jp,
            const double* __restrict__ sp)
{
  double* v = V + int64_t(*jp) * n;
  const double s = *sp;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    v[i] = s * v[i];
}

// Classical Gram-Schmidt, twice (CGS2), on w = V_{j+1} against V_0..V_j, j = G->j:
//  MODE 0: c1[i] = <w, V_i>;                         H[j][i]  = c1[i]
//  MODE 1: w -= sum_i c1[i] V_i; c2[i] = <w, V_i>;   H[j][i] += c2[i]
//  MODE 2: w -= sum_i c2[i] V_i; s = ||w||;          H[j][j+1] = s
// Each pass reads the j+1 basis vectors once; accumulators stay in registers;
// reductions are deterministic (fixed grid, fixed order).
template<int MODE>
__global__ void __launch_bounds__(kRedThreads)
k_cgs(int64_t n, double* __restrict__ V, GmresDev* G, double* partials,
      unsigned* ticket)
{
  __shared__ double s_coef[kCgsMaxJ];
  __shared__ double s_red[kRedThreads / 32][kCgsMaxJ];
  __shared__ bool am_last;
  const int j = G->j;
  const int nv = j + 1;
  double* w = V + int64_t(j + 1) * n;
  if (MODE >= 1 && threadIdx.x < kCgsMaxJ)
    s_coef[threadIdx.x] = (threadIdx.x < nv) ? (MODE == 1 ? G->d[threadIdx.x]
                                                          : G->d2[threadIdx.x])
                                             : 0.0;
  __syncthreads();
  double acc[kCgsMaxJ];
#pragma unroll
  for (int i = 0; i < kCgsMaxJ; ++i)
    acc[i] = 0.0;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
       r += (int64_t)gridDim.x * blockDim.x) {
    double t = w[r];
    if (MODE >= 1) {
#pragma unroll
      for (int i = 0; i < kCgsMaxJ; ++i)
        if (i < nv)
          t = fma(-s_coef[i], V[int64_t(i) * n + r], t);
      w[r] = t;
    }
    if (MODE <= 1) {
#pragma unroll
      for (int i = 0; i < kCgsMaxJ; ++i)
        if (i < nv)
          acc[i] = fma(t, V[int64_t(i) * n + r], acc[i]);
    } else {
      acc[0] = fma(t, t, acc[0]);
    }
  }
  const int nred = (MODE == 2) ? 1 : nv;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < kCgsMaxJ; ++i) {
    if (i < nred) {
      double v = acc[i];
      for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0)
        s_red[wid][i] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x < nred) {
    double v = 0.0;
    for (int q = 0; q < kRedThreads / 32; ++q)
      v += s_red[q][threadIdx.x];
    partials[int64_t(threadIdx.x) * gridDim.x + blockIdx.x] = v;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0)
    am_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!am_last)
    return;
  __threadfence();
  if (threadIdx.x < nred) {
    double v = 0.0;
    for (int q = 0; q < (int)gridDim.x; ++q)
      v += __ldcg(partials + int64_t(threadIdx.x) * gridDim.x + q);
    const int i = threadIdx.x;
    if (MODE == 0) {
      G->d[i] = v;
      G->H[j][i] = v;
    } else if (MODE == 1) {
      G->d2[i] = v;
      G->H[j][i] += v;
    } else {
      const double sv = sqrt(v);
      G->H[j][j + 1] = sv;
      G->s = sv;
    }
  }
  if (threadIdx.x == 0)
    *ticket = 0u;
}

// Givens update of column j (LinAlg/gmres.cc:88-104 applied to the flexible
// Hessenberg), residual estimate |gamma[j+1]| = ||b - A x_j|| in exact
// arithmetic, then j += 1 and the inner loop condition.
__global__ void
k_fg_step(GmresDev* G, cudaGraphConditionalHandle inner, int m)
{
  const int last = G->j, dim = last + 1;
  double* h = G->H[last];
  const double s = h[dim];
  G->inv = 1.0 / s;
  for (int i = 0; i < last; i++) {
    double dummy = h[i];
    h[i] = G->ci[i] * dummy + G->si[i] * h[i + 1];
    h[i + 1] = -G->si[i] * dummy + G->ci[i] * h[i + 1];
  }
  double r = 1. / sqrt(h[last] * h[last] + h[last + 1] * h[last + 1]);
  G->si[last] = h[last + 1] * r;
  G->ci[last] = h[last] * r;
  h[last] = G->ci[last] * h[last] + G->si[last] * h[last + 1];
  G->gamma[last + 1] = -G->si[last] * G->gamma[last];
  G->gamma[last] *= G->ci[last];
  const double rho = fabs(G->gamma[dim]);
  if (G->total < kMaxV)
    G->hist[G->total] = rho;
  G->info.residual = rho;
  G->info.iteration += 1;
  G->total += 1;
  G->j = dim;
  const double aim = fmax(G->info.tol * G->bnorm, G->info.globaltol);
  const int reached = (rho <= aim) || dim >= m || G->total >= G->info.maxiter ||
                      !(rho == rho);
  cudaGraphSetConditional(inner, reached ? 0 : 1);
}

// hs = H^-1 gamma on the first G->j columns (Common/mult.h:130-141)
__global__ void
k_fg_backward(GmresDev* G)
{
  const int dim = G->j;
  for (int i = dim - 1; i >= 0; i--) {
    double s = G->gamma[i];
    for (int jj = i + 1; jj < dim; jj++)
      s -= G->hs[jj] * G->H[jj][i];
    G->hs[i] = s / G->H[i][i];
  }
}

// x += sum_{q < G->j} hs[q] Z_q
template<class TZ>
__global__ void
k_fg_update(int64_t n, double* __restrict__ x, const TZ* __restrict__ Z,
            const GmresDev* __restrict__ G)
{
  const int k = G->j;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double acc = x[i];
    for (int q = 0; q < k; ++q)
      acc = fma(G->hs[q], static_cast<double>(Z[int64_t(q) * n + i]), acc);
    x[i] = acc;
  }
}

} // namespace gb
