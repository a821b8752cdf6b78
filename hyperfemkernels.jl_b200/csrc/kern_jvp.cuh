// Point-parallel variant of the matrix-free product J(u) dx with the tangent re-evaluated from the
// stored F (the same arithmetic as cell_kernel<MODE_JV>, another mapping of threads to work).
//
// A CTA of NT threads holds C = NT / P^3 cells (NT = 32 ceil(P^3 / 32): one cell per CTA, or 256:
// several, so that the barriers of one CTA stall fewer warps). Every phase spreads its tasks
// over all threads of the CTA: the tensor lines of each sum-factorisation sweep (3 fields or
// components x Q^2, P Q or P^2 lines per cell) and, in the pointwise phase, one quadrature point
// per thread (27 per Q2 cell). No thread holds a column of the y-sweep in registers across several
// points, so a thread needs far fewer registers than a lane of the line-mapped kernel and an SM
// keeps more warps resident; the price is a barrier per phase and more shared-memory traffic (each
// point reads its 9Q y-sweep values itself). Shared memory per cell: two regions that the phases
// use in turn (region 1: local values + x-sweep | point coefficients | y-contraction; region 2:
// y-sweep | z-contraction), the cell's dof ids and its scalars (inverse Jacobian, determinant,
// lambda, mu, a validity flag). A thread's F values are loaded at entry, so that their latency
// passes during the gather and the interpolation sweeps.
//
// Reference: tp_interpolate!/tp_contract! (src/tensorproduct.jl:125-224), apply_cells!
// (src/matrixfree.jl:341-396); the pointwise tangent action is law_dstress_F.
#pragma once
#include "hfk_internal.h"
#include "pointwise.cuh"

namespace hfk {

constexpr int JVP_WIDE = 256;  // threads of the several-cells CTA

template <int Q, int P, int NT>
struct JvpShape {
  static constexpr int NN = Q * Q * Q, NP = P * P * P, PP = P * P, PQQ = P * Q * Q;
  static constexpr int C = NT / NP;  // cells per CTA
  static_assert(C >= 1, "a cell's points must fit in one CTA");
  static constexpr int R1 = cmax(3 * NN + 6 * PQQ, 9 * NP);  // xl + xs | coefficients | y-contraction
  static constexpr int R2 = 9 * Q * PP;                      // y-sweep | z-contraction
  static constexpr int VALS = R1 + R2;
  static constexpr int NSC = 12;  // per-cell scalars: iJ[9], det, lambda, mu
};

// threads of the one-cell CTA
template <int P>
constexpr int jvp_narrow() {
  return (P * P * P + 31) / 32 * 32;
}

// resident CTAs per SM the register allocation targets: 24 warps per SM (80 registers a thread)
template <int NT>
constexpr int jvp_min_blocks() {
  return 24 * 32 / NT > 32 ? 32 : (24 * 32 / NT < 1 ? 1 : 24 * 32 / NT);
}

template <int Q, int P, typename R, int NT>
__host__ __device__ constexpr size_t jvp_smem_bytes() {
  using S = JvpShape<Q, P, NT>;
  return (size_t)S::C * (S::NSC * sizeof(double) + S::VALS * sizeof(R) + 3 * S::NN * sizeof(int32_t) + sizeof(int32_t) * 2);
}

template <int Q, int P, typename R, int NT>
__global__ void __launch_bounds__(NT, jvp_min_blocks<NT>()) jvp_kernel(CellData cd, Tab1D<R> tab, CellIO<R> io) {
  using S = JvpShape<Q, P, NT>;
  constexpr int NN = S::NN, NP = S::NP, PP = S::PP, PQQ = S::PQQ, C = S::C, NDL = 3 * NN;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* scal = reinterpret_cast<double*>(smem_raw);                 // [C][NSC]
  R* vals = reinterpret_cast<R*>(scal + C * S::NSC);                  // [C][VALS]
  int32_t* sid = reinterpret_cast<int32_t*>(vals + C * S::VALS);      // [C][NDL]
  int32_t* scell = sid + C * NDL;                                     // [C]: cell, or -1 (no work)
  int32_t* saff = scell + C;                                          // [C]: affine
  const int tid = threadIdx.x;
  const int base = blockIdx.x * C;
  // this thread's point (C NP <= NT: at most one) and its stored F, requested now
  R Fm[9];
  {
    const int lc = tid / NP, q = tid - lc * NP;
    const int li = base + lc;
    if (tid < C * NP && li < cd.ncells_list) {
      const int cell = cd.cells ? cd.cells[li] : li;
#pragma unroll
      for (int i = 0; i < 9; ++i) Fm[i] = io.Fq[((size_t)cell * 9 + i) * NP + q];
    } else {
#pragma unroll
      for (int i = 0; i < 9; ++i) Fm[i] = (i % 4) == 0 ? R(1) : R(0);
    }
  }

  // ---- cells of the CTA and their scalars --------------------------------------------------
  if (tid < C) {
    const int li = base + tid;
    int cell = -1;
    if (li < cd.ncells_list) {
      cell = cd.cells ? cd.cells[li] : li;
      if (cd.skipped(cell)) cell = -1;
    }
    scell[tid] = cell;
    double* sc = scal + tid * S::NSC;
    int aff = 1;
    if (cell >= 0) {
      aff = cd.affine[cell];
      if (aff) {
#pragma unroll
        for (int i = 0; i < 10; ++i) sc[i] = cd.geo[(size_t)cell * 10 + i];
      }
      sc[10] = cd.lam_of(cell);
      sc[11] = cd.mu_of(cell);
    } else {
#pragma unroll
      for (int i = 0; i < 12; ++i) sc[i] = 0.0;
    }
    saff[tid] = aff;
  }
  __syncthreads();
  {
    // a CTA without an active cell (a batch's converged problems, skipped) returns at once
    bool none = true;
    for (int lc = 0; lc < C; ++lc) none = none && scell[lc] < 0;
    if (none) return;
  }

  // ---- gather (increments are zero at Dirichlet dofs) ------------------------------------------
  for (int e = tid; e < C * NDL; e += NT) {
    const int lc = e / NDL, j = e - lc * NDL;
    const int cell = scell[lc];
    const int32_t id = cell >= 0 ? cd.ids[(size_t)cell * NDL + j] : 0;
    sid[e] = id;
    vals[lc * S::VALS + j] = id > 0 ? io.dx[id - 1] : R(0);
  }
  __syncthreads();

  // ---- interpolation, x lines (f, j, k): N and dN sweeps ---------------------------------------
  for (int e = tid; e < C * 3 * Q * Q; e += NT) {
    const int lc = e / (3 * Q * Q), r = e - lc * 3 * Q * Q;
    const int f = r / (Q * Q), jk = r - f * Q * Q;
    const R* xl = vals + lc * S::VALS + f * NN + Q * jk;
    R* xs = vals + lc * S::VALS + 3 * NN + f * 2 * PQQ + P * jk;
    R v[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) v[i] = xl[i];
#pragma unroll
    for (int a = 0; a < P; ++a) {
      R s = 0, ds = 0;
#pragma unroll
      for (int i = 0; i < Q; ++i) {
        s += tab.N1[a * Q + i] * v[i];
        ds += tab.dN1[a * Q + i] * v[i];
      }
      xs[a] = s;
      xs[PQQ + a] = ds;
    }
  }
  __syncthreads();

  // ---- interpolation, y lines (f, a, k): C = N.(N u), D = dN.(N u), E = N.(dN u) -------------
  for (int e = tid; e < C * 3 * P * Q; e += NT) {
    const int lc = e / (3 * P * Q), r = e - lc * 3 * P * Q;
    const int f = r / (P * Q), ak = r - f * P * Q, a = ak % P, k = ak / P;
    const R* xs = vals + lc * S::VALS + 3 * NN + f * 2 * PQQ + a + P * Q * k;
    R* yr = vals + lc * S::VALS + S::R1;
    R va[Q], vb[Q];
#pragma unroll
    for (int j = 0; j < Q; ++j) {
      va[j] = xs[P * j];
      vb[j] = xs[PQQ + P * j];
    }
#pragma unroll
    for (int b = 0; b < P; ++b) {
      R c0 = 0, d0 = 0, e0 = 0;
#pragma unroll
      for (int j = 0; j < Q; ++j) {
        c0 += tab.N1[b * Q + j] * va[j];
        d0 += tab.dN1[b * Q + j] * va[j];
        e0 += tab.N1[b * Q + j] * vb[j];
      }
      const int ab = a + P * b;
      yr[((f * 3 + 0) * Q + k) * PP + ab] = c0;
      yr[((f * 3 + 1) * Q + k) * PP + ab] = d0;
      yr[((f * 3 + 2) * Q + k) * PP + ab] = e0;
    }
  }
  __syncthreads();

  // ---- pointwise: one point per thread --------------------------------------------------------
  if (tid < C * NP) {
    const int lc = tid / NP, q = tid - lc * NP;
    const int ab = q % PP, c = q / PP;
    const int cell = scell[lc];
    const R* yr = vals + lc * S::VALS + S::R1;
    R G[3][3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      R g1 = 0, g2 = 0, g3 = 0;
#pragma unroll
      for (int k = 0; k < Q; ++k) {
        const R n = tab.N1[c * Q + k], dn = tab.dN1[c * Q + k];
        g1 += n * yr[((f * 3 + 2) * Q + k) * PP + ab];
        g2 += n * yr[((f * 3 + 1) * Q + k) * PP + ab];
        g3 += dn * yr[((f * 3 + 0) * Q + k) * PP + ab];
      }
      G[f][0] = g1;
      G[f][1] = g2;
      G[f][2] = g3;
    }
    const double* sc = scal + lc * S::NSC;
    R iJ[9], dV;
    if (saff[lc]) {
#pragma unroll
      for (int i = 0; i < 9; ++i) iJ[i] = (R)sc[i];
      dV = (R)(cd.w[q] * sc[9]);
    } else {
      double Jt[9], iJd[9];
      point_jacobian_dev(cd, cell, q, Jt);
      const double det = det3(Jt);
      inv3(Jt, det, iJd);
#pragma unroll
      for (int i = 0; i < 9; ++i) iJ[i] = (R)iJd[i];
      dV = (R)(cd.w[q] * fabs(det));
    }
    R H[9];
    phys_grad<R, 3>(iJ, G, 0, H);
    R dP[9];
    law_dstress_F<R>(cd.law, (R)sc[10], (R)sc[11], Fm, H, dP);
    R out[3][3];
    pull_back<R>(iJ, dP, dV, out);
    R* pc = vals + lc * S::VALS;  // region 1: [cc][K][c][ab]
#pragma unroll
    for (int cc = 0; cc < 3; ++cc)
#pragma unroll
      for (int K = 0; K < 3; ++K) pc[((cc * 3 + K) * P + c) * PP + ab] = out[cc][K];
  }
  __syncthreads();

  // ---- contraction, z lines (cc, a, b) -> rows (cc, 0..2, k) of region 2 ----------------------
  for (int e = tid; e < C * 3 * PP; e += NT) {
    const int lc = e / (3 * PP), r = e - lc * 3 * PP;
    const int cc = r / PP, ab = r - cc * PP;
    const R* pc = vals + lc * S::VALS;
    R* zc = vals + lc * S::VALS + S::R1;
    R rv[3][P];
#pragma unroll
    for (int K = 0; K < 3; ++K)
#pragma unroll
      for (int c = 0; c < P; ++c) rv[K][c] = pc[((cc * 3 + K) * P + c) * PP + ab];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      R t0 = 0, t1 = 0, t2 = 0;
#pragma unroll
      for (int c = 0; c < P; ++c) {
        const R n = tab.N1[c * Q + k], dn = tab.dN1[c * Q + k];
        t0 += dn * rv[2][c];
        t1 += n * rv[0][c];
        t2 += n * rv[1][c];
      }
      zc[((cc * 3 + 0) * Q + k) * PP + ab] = t0;
      zc[((cc * 3 + 1) * Q + k) * PP + ab] = t1;
      zc[((cc * 3 + 2) * Q + k) * PP + ab] = t2;
    }
  }
  __syncthreads();

  // ---- contraction, y lines (cc, a, k) -> region 1 -------------------------------------------
  for (int e = tid; e < C * 3 * P * Q; e += NT) {
    const int lc = e / (3 * P * Q), r = e - lc * 3 * P * Q;
    const int cc = r / (P * Q), ak = r - cc * P * Q, a = ak % P, k = ak / P;
    const R* zc = vals + lc * S::VALS + S::R1;
    R* y2 = vals + lc * S::VALS;
    R v0[P], v1[P], v2[P];
#pragma unroll
    for (int b = 0; b < P; ++b) {
      v0[b] = zc[((cc * 3 + 0) * Q + k) * PP + a + P * b];
      v1[b] = zc[((cc * 3 + 1) * Q + k) * PP + a + P * b];
      v2[b] = zc[((cc * 3 + 2) * Q + k) * PP + a + P * b];
    }
#pragma unroll
    for (int j = 0; j < Q; ++j) {
      R s0 = 0, s1 = 0;
#pragma unroll
      for (int b = 0; b < P; ++b) {
        s0 += tab.N1[b * Q + j] * v0[b] + tab.dN1[b * Q + j] * v2[b];
        s1 += tab.N1[b * Q + j] * v1[b];
      }
      y2[(cc * 2 + 0) * PQQ + a + P * (j + Q * k)] = s0;
      y2[(cc * 2 + 1) * PQQ + a + P * (j + Q * k)] = s1;
    }
  }
  __syncthreads();

  // ---- contraction, x lines (cc, j, k) and the scatter of the free test rows --------------------
  for (int e = tid; e < C * 3 * Q * Q; e += NT) {
    const int lc = e / (3 * Q * Q), r = e - lc * 3 * Q * Q;
    if (scell[lc] < 0) continue;
    const int cc = r / (Q * Q), jk = r - cc * Q * Q;
    const R* y2 = vals + lc * S::VALS;
    R v0[P], v1[P];
#pragma unroll
    for (int a = 0; a < P; ++a) {
      v0[a] = y2[(cc * 2 + 0) * PQQ + a + P * jk];
      v1[a] = y2[(cc * 2 + 1) * PQQ + a + P * jk];
    }
    const int32_t* ids = sid + lc * NDL + cc * NN + Q * jk;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      R s = 0;
#pragma unroll
      for (int a = 0; a < P; ++a) s += tab.N1[a * Q + i] * v0[a] + tab.dN1[a * Q + i] * v1[a];
      const int32_t id = ids[i];
      if (id > 0) {
        if (io.atomic) atomicAdd(&io.y[id - 1], s);
        else io.y[id - 1] += s;
      }
    }
  }
}

}  // namespace hfk
