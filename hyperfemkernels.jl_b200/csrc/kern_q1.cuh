// Matrix-free product J(u) dx of Q1 hexahedra (8 nodes, 2 x 2 x 2 Gauss points), the recompute
// formulation (tangent re-evaluated from the stored F), warp-synchronous: 8 lanes per cell, one per
// Gauss point, 4 cells per warp, no shared memory and no barrier.
//
// Lane q of a cell gathers the 3 components of node q (its ldofs q, 8 + q, 16 + q), and the cell's
// 24 values reach every lane of the cell by shuffles. Each lane evaluates the reference gradient at
// its point with the 1D tables (tensor structure inside the thread), the law's tangent action and
// its 24 nodal contributions; the contributions are summed over the cell's 8 points by a
// reduce-scatter of 21 shuffles (halves exchanged with the lanes 4, 2 and 1 apart) that leaves lane
// q exactly the sums of node q, the 3 entries whose ids it gathered, which it adds into y.
//
// Reference: apply_cells! (src/matrixfree.jl:341-396) with tp_interpolate! / tp_contract!
// (src/tensorproduct.jl:125-224) for 2 nodes and 2 points per direction; the same pointwise code as
// the other products (law_dstress_F, pull_back).
#pragma once
#include "hfk_internal.h"
#include "pointwise.cuh"

namespace hfk {

constexpr int Q1_THREADS = 256;  // 32 cells per CTA

template <typename R>
__global__ void __launch_bounds__(Q1_THREADS, 2) q1_jv_kernel(CellData cd, Tab1D<R> tab, CellIO<R> io) {
  const int lane = threadIdx.x & 31, q = lane & 7, base = lane & ~7;
  const int li = (blockIdx.x * (Q1_THREADS / 32) + (threadIdx.x >> 5)) * 4 + (lane >> 3);
  const bool valid = li < cd.ncells_list;
  const int cell = valid ? (cd.cells ? cd.cells[li] : li) : 0;
  const bool active = valid && !cd.skipped(cell);
  if (__all_sync(0xffffffffu, !active)) return;
  // this lane's node: its three components' ids and increments
  int32_t id[3];
  R xv[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    id[c] = active ? cd.ids[(size_t)cell * 24 + c * 8 + q] : 0;
    xv[c] = id[c] > 0 ? io.dx[id[c] - 1] : R(0);
  }
  // this point's 1D values: q = q1 + 2 q2 + 4 q3, node n = n1 + 2 n2 + 4 n3 (tensor orders)
  const int q1 = q & 1, q2 = (q >> 1) & 1, q3 = q >> 2;
  const R nx[2] = {tab.N1[2 * q1], tab.N1[2 * q1 + 1]}, dx1[2] = {tab.dN1[2 * q1], tab.dN1[2 * q1 + 1]};
  const R ny[2] = {tab.N1[2 * q2], tab.N1[2 * q2 + 1]}, dy1[2] = {tab.dN1[2 * q2], tab.dN1[2 * q2 + 1]};
  const R nz[2] = {tab.N1[2 * q3], tab.N1[2 * q3 + 1]}, dz1[2] = {tab.dN1[2 * q3], tab.dN1[2 * q3 + 1]};
  // reference gradient G[c][K] of the increment at this point, from the cell's 24 values
  R G[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    R x[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) x[n] = __shfl_sync(0xffffffffu, xv[c], base | n);
    R a0[4], a1[4];  // x-contractions over n1, indexed n2 + 2 n3: with the derivative, with the basis
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      a0[m] = dx1[0] * x[2 * m] + dx1[1] * x[2 * m + 1];
      a1[m] = nx[0] * x[2 * m] + nx[1] * x[2 * m + 1];
    }
    R b0[2], b1[2], b2[2];  // then over n2, indexed n3
#pragma unroll
    for (int n3 = 0; n3 < 2; ++n3) {
      b0[n3] = ny[0] * a0[2 * n3] + ny[1] * a0[2 * n3 + 1];
      b1[n3] = dy1[0] * a1[2 * n3] + dy1[1] * a1[2 * n3 + 1];
      b2[n3] = ny[0] * a1[2 * n3] + ny[1] * a1[2 * n3 + 1];
    }
    G[c][0] = nz[0] * b0[0] + nz[1] * b0[1];
    G[c][1] = nz[0] * b1[0] + nz[1] * b1[1];
    G[c][2] = dz1[0] * b2[0] + dz1[1] * b2[1];
  }
  // geometry at the point
  R iJ[9], dV;
  if (cd.affine[cell]) {
    const double* gc = cd.geo + (size_t)cell * 10;
#pragma unroll
    for (int i = 0; i < 9; ++i) iJ[i] = (R)__ldg(gc + i);
    dV = (R)(cd.w[q] * __ldg(gc + 9));
  } else {
    double Jt[9], iJd[9];
    point_jacobian_dev(cd, cell, q, Jt);
    const double det = det3(Jt);
    inv3(Jt, det, iJd);
#pragma unroll
    for (int i = 0; i < 9; ++i) iJ[i] = (R)iJd[i];
    dV = (R)(cd.w[q] * fabs(det));
  }
  R H[9], Fm[9], dP[9], out[3][3];
  phys_grad<R, 3>(iJ, G, 0, H);
#pragma unroll
  for (int i = 0; i < 9; ++i) Fm[i] = io.Fq[((size_t)cell * 9 + i) * 8 + q];
  law_dstress_F<R>(cd.law, (R)cd.lam_of(cell), (R)cd.mu_of(cell), Fm, H, dP);
  pull_back<R>(iJ, dP, dV, out);
  // this point's contributions to the 24 nodal entries: y[c][n] = sum_K out[c][K] dN[n, K, q]
  // = dx1[n1] (out0 ny nz) + nx[n1] (out1 dy1 nz + out2 ny dz1)
  R y[3][8];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int n3 = 0; n3 < 2; ++n3)
#pragma unroll
      for (int n2 = 0; n2 < 2; ++n2) {
        const R a = out[c][0] * ny[n2] * nz[n3];
        const R b = out[c][1] * dy1[n2] * nz[n3] + out[c][2] * ny[n2] * dz1[n3];
#pragma unroll
        for (int n1 = 0; n1 < 2; ++n1) y[c][n1 + 2 * n2 + 4 * n3] = dx1[n1] * a + nx[n1] * b;
      }
  // reduce-scatter over the cell's 8 lanes. Before the exchange with the lanes m apart (m = 4, 2,
  // 1) slots 0 .. 2m - 1 are live, slot s holding a partial sum of node s | (q & ~(2m - 1) & 7); the
  // lane keeps the half of each pair (s, s + m) whose bit m matches its own and adds its partner's
  // copy, into slot s. After m = 1, slot 0 holds node q summed over the cell's 8 points.
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int m = 4; m >= 1; m >>= 1) {
      const bool hi = (q & m) != 0;
#pragma unroll
      for (int s = 0; s < m; ++s) {
        const R send = hi ? y[c][s] : y[c][s + m];
        const R keep = hi ? y[c][s + m] : y[c][s];
        y[c][s] = keep + __shfl_xor_sync(0xffffffffu, send, m);
      }
    }
  }
  if (!active) return;
#pragma unroll
  for (int c = 0; c < 3; ++c)
    if (id[c] > 0) {
      if (io.atomic) atomicAdd(&io.y[id[c] - 1], y[c][0]);
      else io.y[id[c] - 1] += y[c][0];
    }
}

}  // namespace hfk
