// Device-side matrix assembly of the scalar Q1 equation
// -div(kappa grad u) + beta . grad u on quadrilateral / hexahedral cells with
// one coefficient kappa per cell: element matrices, their summation into the
// level's SELL-32 values, the strong Dirichlet rows and columns, and the
// coarsening of kappa to the next coarser level. Included by gb_context.cuh
// after gb_block.cuh.
#pragma once
#include "gb_kernels.cuh"

namespace gb {

// Element matrices of the cells, one thread per cell (CGDisc::Matrix,
// DofHandler/cgdisc.h:599-635, with ElementIntegrator::Matrix,
// DofHandler/elementintegrator.xx:350-395, and the matrix formula QuadGauss4 /
// HexGauss8 of ElementIntegratorQ12d / Q13d): at the 2^DIM Gauss points
// 1/2 -+ g of the unit cell the multilinear map's Jacobian J, the physical
// gradients of the Q1 basis, and
//   E[a][b] += w |J| (kappa grad phi_b . grad phi_a + (beta . grad phi_b) phi_a)
// (row a: test function, column b: trial function; CONV: beta is not zero).
// Local node a has the
// corner bits (a & 1, a >> 1 & 1, a >> 2 & 1). cells: node of local a of cell
// c at cells[a * ncells + c]; coords: node-major, DIM per node. E: entry (a, b)
// of cell c at E[(a * NL + b) * ncells + c] (coalesced per entry).
template<int DIM, bool CONV>
__global__ void __launch_bounds__(128)
k_q1_element(int ncells, const int* __restrict__ cells, const double* __restrict__ coords,
             const double* __restrict__ kappa, double b0, double b1, double b2, double g,
             double* __restrict__ E)
{
  GB_PDL_ENTRY();
  constexpr int NL = 1 << DIM;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells)
    return;
  double X[NL][DIM];
#pragma unroll
  for (int a = 0; a < NL; ++a) {
    const int64_t node = __ldg(cells + int64_t(a) * ncells + c);
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      X[a][d] = __ldg(coords + node * DIM + d);
  }
  const double kap = __ldg(kappa + c);
  const double beta[3] = { b0, b1, b2 };
  const double gp[2] = { 0.5 - g, 0.5 + g };
  constexpr double wq = DIM == 3 ? 0.125 : 0.25;
  double e[NL * NL];
#pragma unroll
  for (int p = 0; p < NL * NL; ++p)
    e[p] = 0.0;
#pragma unroll 1
  for (int q = 0; q < NL; ++q) {
    double xi[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      xi[d] = gp[(q >> d) & 1];
    // reference values and gradients of the basis
    double phi[NL], gr[NL][DIM];
#pragma unroll
    for (int a = 0; a < NL; ++a) {
      phi[a] = 1.0;
#pragma unroll
      for (int k = 0; k < DIM; ++k)
        gr[a][k] = 1.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        const bool bit = (a >> d) & 1;
        const double f = bit ? xi[d] : 1.0 - xi[d];
        phi[a] *= f;
#pragma unroll
        for (int k = 0; k < DIM; ++k)
          gr[a][k] *= k == d ? (bit ? 1.0 : -1.0) : f;
      }
    }
    // J[d][k] = d x_d / d xi_k, its determinant and inverse
    double J[DIM][DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
#pragma unroll
      for (int k = 0; k < DIM; ++k) {
        double s = 0.0;
#pragma unroll
        for (int a = 0; a < NL; ++a)
          s = fma(X[a][d], gr[a][k], s);
        J[d][k] = s;
      }
    double det, Ji[DIM][DIM]; // Ji[k][d] = d xi_k / d x_d (cofactors / det)
    if (DIM == 2) {
      det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
      const double r = 1.0 / det;
      Ji[0][0] = J[1][1] * r;
      Ji[0][1] = -J[0][1] * r;
      Ji[1][0] = -J[1][0] * r;
      Ji[1][1] = J[0][0] * r;
    } else {
      const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
      const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
      const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
      det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
      const double r = 1.0 / det;
      Ji[0][0] = c00 * r;
      Ji[1][0] = c01 * r;
      Ji[2][0] = c02 * r;
      Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * r;
      Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * r;
      Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * r;
      Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * r;
      Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * r;
      Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * r;
    }
    const double w = wq * fabs(det);
    // physical gradients and beta . grad phi
    double gx[NL][DIM], bg[NL];
#pragma unroll
    for (int a = 0; a < NL; ++a) {
      double s = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        double t = 0.0;
#pragma unroll
        for (int k = 0; k < DIM; ++k)
          t = fma(gr[a][k], Ji[k][d], t);
        gx[a][d] = t;
        s = fma(beta[d], t, s);
      }
      bg[a] = s;
    }
    // the diffusion part is symmetric: each product once, added to both
    const double wk = w * kap;
#pragma unroll
    for (int a = 0; a < NL; ++a)
#pragma unroll
      for (int b = a; b < NL; ++b) {
        double dg = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d)
          dg = fma(gx[b][d], gx[a][d], dg);
        e[a * NL + b] = fma(wk, dg, e[a * NL + b]);
        if (b != a)
          e[b * NL + a] = fma(wk, dg, e[b * NL + a]);
      }
    if (CONV) {
#pragma unroll
      for (int a = 0; a < NL; ++a) {
        const double wp = w * phi[a];
#pragma unroll
        for (int b = 0; b < NL; ++b)
          e[a * NL + b] = fma(wp, bg[b], e[a * NL + b]);
      }
    }
  }
#pragma unroll
  for (int p = 0; p < NL * NL; ++p)
    E[int64_t(p) * ncells + c] = e[p];
}

__device__ __forceinline__ void
q2_basis_1d(double t, double* L, double* dL)
{
  L[0] = 2.0 * (t - 0.5) * (t - 1.0);
  L[1] = -4.0 * t * (t - 1.0);
  L[2] = 2.0 * t * (t - 0.5);
  dL[0] = 4.0 * t - 3.0;
  dL[1] = -8.0 * t + 4.0;
  dL[2] = 4.0 * t - 1.0;
}

// The piecewise linear basis of a patch of two cells in one direction (nodes 0,
// 1/2, 1) at Gauss point qd of the 4 of the patch: LineGauss2 (1/2 -+ g) in cell
// qd / 2, mapped to it (PatchFormula2d/3d,
// Discretization/Q2/patchintegrationformula.xx:55-83; BaseQ12dPatch,
// Discretization/Q2/baseq1patch.h: the cell's Q1 functions, derivatives times 2).
__device__ __forceinline__ void
q1patch_basis_1d(int qd, double g, double* L, double* dL)
{
  const int k = qd >> 1;                    // the cell
  const double s = (qd & 1) ? 0.5 + g : 0.5 - g;
  L[0] = L[1] = L[2] = 0.0;
  dL[0] = dL[1] = dL[2] = 0.0;
  L[k] = 1.0 - s;
  L[k + 1] = s;
  dL[k] = -2.0;
  dL[k + 1] = 2.0;
}

// Q2 element matrices (CGQ2: 3^DIM-node elements on patches of 2^DIM cells,
// the isoparametric quadratic map, the matrix formula QuadGauss9 / HexGauss27
// with LineGauss3's points and 12-digit weights as the reference states them,
// Discretization/Q1/integrationformula1d.cc:82-92): row a of
//   w |J| (kappa grad phi_b . grad phi_a + (beta . grad phi_b) phi_a),
// local node a = sum_d a_d 3^d (x fastest), basis nodes 0, 1/2, 1 per axis.
// One warp per element: lane b (< 3^DIM) holds
// node b. At each Gauss point the lanes form their terms of J and sum them
// with a butterfly of shuffles (the same sum, in the same order, on every
// lane), then each lane computes its own physical gradient once and hands it
// to the other lanes by shuffles; lane a accumulates row a. Per element and
// point this forms each basis gradient once instead of once per row.
// LPS (with CONV): the local projection stabilisation of the convection
// (CGQ2Lps, ElementLpsIntegrator::Matrix, DofHandler/elementlpsintegrator.h:
// 168-211): at each Gauss point h = |J|^(1/DIM), delta = s0 / (xeta kappa /
// h^2 + bnorm / h) (LpsStabilization::ConvectionDiffusion,
// Problems/lpsstabilization.cc), and E(a, b) += delta (beta . grad N_a)
// (w |J| beta . grad N_b) with the projected functions N of
// ElementLpsIntegrator::Projection (:66-110): a corner node's function is
// -(1/2)^k times each node of its quarter of the patch that has k digits
// moved to the middle, the other nodes keep theirs.
// PQ1: the patch's Q1 functions instead (CGQ1Lps / CGQ1Patch: BaseQ12dPatch /
// BaseQ13dPatch, bilinear / trilinear on each cell of the patch) with the
// patch formula of QuadGauss4 / HexGauss8 in every cell (4 points per
// direction, weight 1/4 each); g = 1/(2 sqrt 3).
template<int DIM, bool CONV, bool LPS = false, bool PQ1 = false>
__global__ void __launch_bounds__(128)
k_q2_element_warp(int ncells, const int* __restrict__ cells,
                  const double* __restrict__ coords, const double* __restrict__ kappa,
                  double b0, double b1, double b2, double* __restrict__ E,
                  double s0 = 0.0, double xeta = 0.0, double bnorm = 0.0, double g = 0.0)
{
  GB_PDL_ENTRY();
  constexpr int NL = DIM == 3 ? 27 : 9;
  const int64_t wid = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= ncells) // whole warps leave together
    return;
  const int c = static_cast<int>(wid);
  const bool act = lane < NL;
  const double P3[3] = { 0.11270166537925831148, 0.5, 0.88729833462074168852 };
  const double W3[3] = { 0.277777777778, 0.444444444444, 0.277777777778 };
  const double beta[3] = { b0, b1, b2 };
  const double kap = __ldg(kappa + c);
  int ld[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d)
    ld[d] = (lane / (d == 0 ? 1 : d == 1 ? 3 : 9)) % 3;
  double X[DIM];
  {
    const int64_t node = act ? __ldg(cells + int64_t(lane) * ncells + c) : 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      X[d] = act ? __ldg(coords + node * DIM + d) : 0.0;
  }
  double e[NL];
#pragma unroll
  for (int b = 0; b < NL; ++b)
    e[b] = 0.0;
  constexpr int NQ = PQ1 ? 4 : 3;            // Gauss points per direction
  constexpr int NQT = DIM == 3 ? NQ * NQ * NQ : NQ * NQ;
#pragma unroll 1
  for (int q = 0; q < NQT; ++q) {
    double L[DIM][3], dL[DIM][3], wq = 1.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const int qd = (q / (d == 0 ? 1 : d == 1 ? NQ : NQ * NQ)) % NQ;
      if (PQ1) {
        q1patch_basis_1d(qd, g, L[d], dL[d]);
        wq *= 0.25;
      } else {
        q2_basis_1d(P3[qd], L[d], dL[d]);
        wq *= W3[qd];
      }
    }
    // this lane's basis function: value and reference gradient
    double phi = 1.0, gr[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      phi *= L[d][ld[d]];
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      double g = 1.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        g *= d == k ? dL[d][ld[d]] : L[d][ld[d]];
      gr[k] = act ? g : 0.0;
    }
    // J[d][k] = sum over nodes of X[d] gr[k]
    double J[DIM][DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
#pragma unroll
      for (int k = 0; k < DIM; ++k) {
        double v = X[d] * gr[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
          v += __shfl_xor_sync(0xffffffffu, v, o);
        J[d][k] = v;
      }
    double det, Ji[DIM][DIM];
    if (DIM == 2) {
      det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
      const double r = 1.0 / det;
      Ji[0][0] = J[1][1] * r;
      Ji[0][1] = -J[0][1] * r;
      Ji[1][0] = -J[1][0] * r;
      Ji[1][1] = J[0][0] * r;
    } else {
      const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
      const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
      const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
      det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
      const double r = 1.0 / det;
      Ji[0][0] = c00 * r;
      Ji[1][0] = c01 * r;
      Ji[2][0] = c02 * r;
      Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * r;
      Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * r;
      Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * r;
      Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * r;
      Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * r;
      Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * r;
    }
    const double w = wq * fabs(det);
    double gx[DIM], bg = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      double t = 0.0;
#pragma unroll
      for (int k = 0; k < DIM; ++k)
        t = fma(gr[k], Ji[k][d], t);
      gx[d] = t;
      if (CONV)
        bg = fma(beta[d], t, bg);
    }
    const double wk = w * kap, wp = w * phi;
    double bn = 0.0, dl = 0.0; // beta . grad N of this lane's projected function
    if (LPS) {
      bool corner = true;
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        corner = corner && ld[d] != 1;
      bn = corner ? 0.0 : bg;
#pragma unroll
      for (int m = 1; m < (1 << DIM); ++m) {
        int src = lane;
        double wt = -1.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d)
          if ((m >> d) & 1) {
            src += (1 - ld[d]) * (d == 0 ? 1 : d == 1 ? 3 : 9);
            wt *= 0.5;
          }
        const double v = __shfl_sync(0xffffffffu, bg, act ? src : lane);
        if (corner)
          bn = fma(wt, v, bn);
      }
      const double h = pow(fabs(det), 1.0 / DIM);
      dl = s0 / (xeta * kap / (h * h) + bnorm / h);
    }
#pragma unroll
    for (int b = 0; b < NL; ++b) {
      double dg = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        dg = fma(__shfl_sync(0xffffffffu, gx[d], b), gx[d], dg);
      e[b] = fma(wk, dg, e[b]);
      if (CONV)
        e[b] = fma(wp, __shfl_sync(0xffffffffu, bg, b), e[b]);
      if (LPS)
        e[b] = fma(dl * bn, w * __shfl_sync(0xffffffffu, bn, b), e[b]);
    }
  }
  if (act) {
#pragma unroll
    for (int b = 0; b < NL; ++b)
      E[(int64_t(lane) * NL + b) * ncells + c] = e[b];
  }
}

// One step of the hanging-node condensation of an element matrix: with t >= 0
// column t += w column s, then row t += w row s (a parent of the hanging node
// in slot s that the element holds in slot t); with t < 0 column s and row s
// scaled by w (the one parent the element lacks, which takes slot s).
struct CondOp
{
  int s, t;
  double w;
};

// The element matrices of the cells with hanging nodes condensed in place
// (CGDisc::LocalToGlobal, DofHandler/cgdisc.h:354-364, with the
// HNStructure::CondenseHanging of the discretisation: Q1 2D/3D,
// Discretization/Q1/hnstructureq12d.cc:129-158, hnstructureq13d.cc:275-438;
// Q2 2D/3D, Discretization/Q2/hnstructureq22d.cc:84-110,
// hnstructureq23d.cc:161-378). The host orders each cell's steps (edges,
// then faces, ascending slots). One warp per cell, lane i holding row /
// column i; a product and a sum per entry, rounded separately.
static __global__ void __launch_bounds__(128)
k_condense(int nh, const int* __restrict__ hcells, const int* __restrict__ opptr,
           const CondOp* __restrict__ ops, int nl, int ncells, double* __restrict__ E)
{
  GB_PDL_ENTRY();
  const int64_t wid = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= nh) // whole warps leave together
    return;
  const int64_t c = __ldg(hcells + wid), nc = ncells;
  const bool act = lane < nl;
  const int k1 = __ldg(opptr + wid + 1);
  for (int k = __ldg(opptr + wid); k < k1; ++k) {
    const CondOp op = ops[k];
    if (act) { // column step: entry (lane, .)
      double* es = E + (int64_t(lane) * nl + op.s) * nc + c;
      if (op.t >= 0) {
        double* et = E + (int64_t(lane) * nl + op.t) * nc + c;
        *et = __dadd_rn(*et, __dmul_rn(op.w, *es));
      } else {
        *es = __dmul_rn(*es, op.w);
      }
    }
    __syncwarp();
    if (act) { // row step: entry (., lane)
      double* es = E + (int64_t(op.s) * nl + lane) * nc + c;
      if (op.t >= 0) {
        double* et = E + (int64_t(op.t) * nl + lane) * nc + c;
        *et = __dadd_rn(*et, __dmul_rn(op.w, *es));
      } else {
        *es = __dmul_rn(*es, op.w);
      }
    }
    __syncwarp();
  }
}

// mask[list[k]] = 1 for k < nl (the hanging nodes into the assembly's
// Dirichlet-or-hanging row mask)
static __global__ void
k_mark_nodes(int nl, const int* __restrict__ list, uint8_t* __restrict__ mask)
{
  GB_PDL_ENTRY();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nl)
    mask[__ldg(list + k)] = 1;
}

// The level's SELL values from the element matrices (LocalToGlobal +
// MatrixInterface::entry, DofHandler/cgdisc.h:353-366): entry e sums
// E[clist[k]] for k in [cptr[e], cptr[e+1]), the contributions in ascending
// cell order (the reference's cell loop). Then the strong Dirichlet condition
// (SparseBlockMatrix::dirichlet, LinAlg/sparseblockmatrix.xx:207-218): a
// Dirichlet row keeps only its diagonal, set to 1, and a Dirichlet column is
// zero elsewhere. On a level with hanging nodes the mask also holds the
// hanging rows, whose only entry is the diagonal, set to 1 like a Dirichlet
// row (HNStructure::MatrixDiag, DofHandler/cgdisc.h:634). Writes the FP64 and
// FP32 values and the diagonal (dd) for the
// block-diagonal inverse. kAsmSplit warps per slice: warp g of slice s takes
// the entries j = g, g + kAsmSplit, .. of the slice's 32 rows (lane = row), so
// that a row's entries are summed by several threads at once.
constexpr int kAsmSplit = 4;

static __global__ void __launch_bounds__(256)
k_asm_gather(int n, const int* __restrict__ sptr, const int* __restrict__ perm,
             const int* __restrict__ col, const int* __restrict__ cptr,
             const int* __restrict__ clist, const double* __restrict__ E,
             const uint8_t* __restrict__ dirmask, const int* __restrict__ diagpos,
             double* __restrict__ v64, float* __restrict__ v32, double* __restrict__ dd)
{
  GB_PDL_ENTRY();
  const int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  const int lane = static_cast<int>(t & 31);
  const int64_t wq = t >> 5;
  const int s = static_cast<int>(wq / kAsmSplit), g = static_cast<int>(wq % kAsmSplit);
  const int slot = s * kSlice + lane;
  if (slot >= n)
    return;
  const int row = perm ? __ldg(perm + slot) : slot;
  const int beg = __ldg(sptr + s);
  const int w = (__ldg(sptr + s + 1) - beg) >> 5;
  const bool drow = __ldg(dirmask + row) != 0;
  const int dpos = __ldg(diagpos + row);
  for (int j = g; j < w; j += kAsmSplit) {
    const int e = beg + j * kSlice + lane;
    double v = 0.0;
    if (drow) {
      v = e == dpos ? 1.0 : 0.0;
    } else if (!__ldg(dirmask + __ldg(col + e))) {
      // the entry's contributions in groups of 8: their indices, then their
      // values, are loaded together; summed in ascending order
      const int k1 = __ldg(cptr + e + 1);
      for (int k0 = __ldg(cptr + e); k0 < k1; k0 += 8) {
        int idx[8];
#pragma unroll
        for (int q = 0; q < 8; ++q)
          idx[q] = k0 + q < k1 ? __ldg(clist + k0 + q) : -1;
        double ev[8];
#pragma unroll
        for (int q = 0; q < 8; ++q)
          ev[q] = idx[q] >= 0 ? __ldg(E + idx[q]) : 0.0;
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (idx[q] >= 0)
            v += ev[q];
      }
    }
    v64[e] = v;
    v32[e] = static_cast<float>(v);
    if (e == dpos)
      dd[row] = v;
  }
}

// kappa of each coarse cell: the sum of its children's values in ascending
// order divided by their number (the harness's coefficient pyramid; a
// per-cell coefficient of the coarser mesh, Application::SetCellData).
static __global__ void
k_kappa_coarsen(int nc, const int* __restrict__ cptr, const int* __restrict__ child,
                const double* __restrict__ kf, double* __restrict__ kc)
{
  GB_PDL_ENTRY();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc)
    return;
  const int k0 = __ldg(cptr + c), k1 = __ldg(cptr + c + 1);
  double s = 0.0;
  for (int k = k0; k < k1; ++k)
    s += __ldg(kf + __ldg(child + k));
  kc[c] = s / double(k1 - k0);
}

// v[e] = src[map[e]] (0 where map[e] < 0), FP64 and FP32: the transpose's
// values from the matrix's after a device assembly.
static __global__ void
k_gather_values(int64_t ne, const int* __restrict__ map, const double* __restrict__ src,
                double* __restrict__ v64, float* __restrict__ v32)
{
  GB_PDL_ENTRY();
  const int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (e >= ne)
    return;
  const int m = __ldg(map + e);
  const double v = m >= 0 ? __ldg(src + m) : 0.0;
  v64[e] = v;
  v32[e] = static_cast<float>(v);
}

// Element residuals of the same equation for a given vector x, one thread per
// cell (CGDisc::Form, DofHandler/cgdisc.h:415-450, with the element
// integrator's Form at the Gauss points of the matrix formula): with grad u =
// sum_b x_b grad phi_b,
//   F[a] += w |J| (kappa grad u . grad phi_a + (beta . grad u) phi_a),
// written F[a * ncells + c].
template<int DIM, bool CONV>
__global__ void __launch_bounds__(128)
k_q1_form(int ncells, const int* __restrict__ cells, const double* __restrict__ coords,
          const double* __restrict__ kappa, double b0, double b1, double b2, double g,
          const double* __restrict__ x, double* __restrict__ F)
{
  GB_PDL_ENTRY();
  constexpr int NL = 1 << DIM;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells)
    return;
  double X[NL][DIM], u[NL];
#pragma unroll
  for (int a = 0; a < NL; ++a) {
    const int64_t node = __ldg(cells + int64_t(a) * ncells + c);
    u[a] = __ldg(x + node);
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      X[a][d] = __ldg(coords + node * DIM + d);
  }
  const double kap = __ldg(kappa + c);
  const double beta[3] = { b0, b1, b2 };
  const double gp[2] = { 0.5 - g, 0.5 + g };
  constexpr double wq = DIM == 3 ? 0.125 : 0.25;
  double f[NL];
#pragma unroll
  for (int a = 0; a < NL; ++a)
    f[a] = 0.0;
#pragma unroll 1
  for (int q = 0; q < NL; ++q) {
    double xi[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      xi[d] = gp[(q >> d) & 1];
    double phi[NL], gr[NL][DIM];
#pragma unroll
    for (int a = 0; a < NL; ++a) {
      phi[a] = 1.0;
#pragma unroll
      for (int k = 0; k < DIM; ++k)
        gr[a][k] = 1.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        const bool bit = (a >> d) & 1;
        const double fd = bit ? xi[d] : 1.0 - xi[d];
        phi[a] *= fd;
#pragma unroll
        for (int k = 0; k < DIM; ++k)
          gr[a][k] *= k == d ? (bit ? 1.0 : -1.0) : fd;
      }
    }
    double J[DIM][DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
#pragma unroll
      for (int k = 0; k < DIM; ++k) {
        double s = 0.0;
#pragma unroll
        for (int a = 0; a < NL; ++a)
          s = fma(X[a][d], gr[a][k], s);
        J[d][k] = s;
      }
    double det, Ji[DIM][DIM];
    if (DIM == 2) {
      det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
      const double r = 1.0 / det;
      Ji[0][0] = J[1][1] * r;
      Ji[0][1] = -J[0][1] * r;
      Ji[1][0] = -J[1][0] * r;
      Ji[1][1] = J[0][0] * r;
    } else {
      const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
      const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
      const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
      det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
      const double r = 1.0 / det;
      Ji[0][0] = c00 * r;
      Ji[1][0] = c01 * r;
      Ji[2][0] = c02 * r;
      Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * r;
      Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * r;
      Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * r;
      Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * r;
      Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * r;
      Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * r;
    }
    const double w = wq * fabs(det);
    double gx[NL][DIM], gu[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      gu[d] = 0.0;
#pragma unroll
    for (int a = 0; a < NL; ++a)
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        double t = 0.0;
#pragma unroll
        for (int k = 0; k < DIM; ++k)
          t = fma(gr[a][k], Ji[k][d], t);
        gx[a][d] = t;
        gu[d] = fma(u[a], t, gu[d]);
      }
    double bu = 0.0;
    if (CONV) {
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        bu = fma(beta[d], gu[d], bu);
    }
    const double wk = w * kap;
#pragma unroll
    for (int a = 0; a < NL; ++a) {
      double dg = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        dg = fma(gu[d], gx[a][d], dg);
      f[a] = fma(wk, dg, f[a]);
      if (CONV)
        f[a] = fma(w * phi[a], bu, f[a]);
    }
  }
#pragma unroll
  for (int a = 0; a < NL; ++a)
    F[int64_t(a) * ncells + c] = f[a];
}

// The element residuals R = E x of elements given by their matrices (entry-major
// E, as the element kernels write them): one warp per element, lane a holding
// node a's value of x and forming row a (the equation is linear in u, so its
// element form is its element matrix times the local values).
template<int NL>
__global__ void __launch_bounds__(128)
k_elem_apply(int ncells, const int* __restrict__ cells, const double* __restrict__ E,
             const double* __restrict__ x, double* __restrict__ R)
{
  GB_PDL_ENTRY();
  const int64_t wid = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= ncells) // whole warps leave together
    return;
  const int64_t c = wid, nc = ncells;
  const bool act = lane < NL;
  const double xb = act ? __ldg(x + __ldg(cells + int64_t(lane) * nc + c)) : 0.0;
  double acc = 0.0;
#pragma unroll
  for (int b = 0; b < NL; ++b) {
    const double v = __shfl_sync(0xffffffffu, xb, b);
    if (act)
      acc = fma(__ldg(E + (int64_t(lane) * NL + b) * nc + c), v, acc);
  }
  if (act)
    R[int64_t(lane) * nc + c] = acc;
}

// y[r] += d * (the element residuals of the cells of node r, in ascending cell
// order: LocalToGlobal, DofHandler/cgdisc.h:367-380); nodes whose entries in
// nptr are empty keep y.
static __global__ void
k_form_gather(int n, const int* __restrict__ nptr, const int* __restrict__ nlist,
              const double* __restrict__ F, double d, double* __restrict__ y)
{
  GB_PDL_ENTRY();
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n)
    return;
  double acc = y[r];
  const int k1 = __ldg(nptr + r + 1);
  for (int k = __ldg(nptr + r); k < k1; ++k)
    acc += d * __ldg(F + __ldg(nlist + k));
  y[r] = acc;
}

// y = 0 on the Dirichlet dofs, and the largest |y| into *m (the bit pattern of
// a non-negative double orders like the number: atomicMax on it is exact and
// independent of the order)
static __global__ void
k_dirichlet_absmax(int n, const uint8_t* __restrict__ dirmask, double* __restrict__ y,
                   unsigned long long* m)
{
  GB_PDL_ENTRY();
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (r < n) {
    if (__ldg(dirmask + r))
      y[r] = 0.0;
    else
      v = fabs(y[r]);
  }
  for (int o = 16; o > 0; o >>= 1)
    v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0 && v > 0.0)
    atomicMax(m, static_cast<unsigned long long>(__double_as_longlong(v)));
}

} // namespace gb
