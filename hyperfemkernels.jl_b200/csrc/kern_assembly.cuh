// Fused element Jacobian + scatter into the CSC nonzeros.
//
// One CTA per cell (all cells in one launch, or the cells of one colour per launch). Per point the
// tangent is pulled back to the reference gradients once, Dh_q[(c,K),(k,K')] = dV sum_{J,L} iJt[J,K] T[(c,J),(k,L)] iJt[L,K'], so the element matrix
//   K[(n,c),(m,k)] = sum_q sum_{K,K'} dN^[n,K,q] Dh_q[(c,K),(k,K')] dN^[m,K',q]
// only reads the reference tables (shared by all cells). For 27-node cells it is formed as the
// reference forms it (element_jacobian_mm!, src/assembly.jl:1316-1342): per test component c,
// G_c[(q,K),(m,k)] = sum_K' Dh[(c,K),(k,K')] dN^[m,K',q], then K_c = A^T G_c with A = dN^ as an
// (np*3) x nn matrix, register-tiled. The entries are added at their precomputed positions
// (scatter_jacobian!, src/assembly.jl:1402-1408) by reductions.
#pragma once
#include "hfk_internal.h"
#include "pointwise.cuh"

namespace hfk {

struct AsmIO {
  const double* u;
  const double* dvals;
  const double* dNt;      // (nn, 3, np) tensor order
  const int32_t* nzpos;   // (ndl*ndl, ncells) 1-based
  double* nzval;
  int np;
};

// Phase 1 (shared by both variants): per point, physical gradient of u, geometry, pulled-back
// tangent Dh[q][(c*3+K) + 9*(k*3+K')] in shared memory.
template <int NN>
__device__ void asm_point_phase(const CellData& cd, const AsmIO& io, int cell, const double* A, const double* xl,
                                double* Hs, double* iJs, double* dVs, double* Dh) {
  const int np = io.np;
  // per point: H, iJt, dV
  for (int q = threadIdx.x; q < np; q += blockDim.x) {
    double G[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int n = 0; n < NN; ++n) {
      const double a0 = A[n + NN * (0 + 3 * q)], a1 = A[n + NN * (1 + 3 * q)], a2 = A[n + NN * (2 + 3 * q)];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double x = xl[c * NN + n];
        G[c][0] += x * a0;
        G[c][1] += x * a1;
        G[c][2] += x * a2;
      }
    }
    double Jt[9], iJ[9], det;
    if (cd.affine[cell]) {
      for (int i = 0; i < 9; ++i) iJ[i] = cd.geo[(size_t)cell * 10 + i];
      det = cd.geo[(size_t)cell * 10 + 9];
    } else {
      point_jacobian_dev(cd, cell, q, Jt);
      det = det3(Jt);
      inv3(Jt, det, iJ);
      det = fabs(det);
    }
    for (int c = 0; c < 3; ++c)
      for (int J = 0; J < 3; ++J) Hs[q * 9 + c + 3 * J] = iJ[J] * G[c][0] + iJ[J + 3] * G[c][1] + iJ[J + 6] * G[c][2];
    for (int i = 0; i < 9; ++i) iJs[q * 9 + i] = iJ[i];
    dVs[q] = cd.w[q] * det;
  }
  __syncthreads();
  // per (point, c, k): the 3x3 block of Dh
  for (int e = threadIdx.x; e < np * 9; e += blockDim.x) {
    const int q = e / 9, ck = e % 9, c = ck / 3, k = ck % 3;
    double Tb[9];  // T[(c,J),(k,L)] at Tb[J + 3 L]
    law_tangent_block(cd.law, cd.lam_of(cell), cd.mu_of(cell), Hs + q * 9, c, k, Tb);
    const double* iJ = iJs + q * 9;
    const double dV = dVs[q];
    // X[J][K'] = sum_L T[(c,J),(k,L)] iJ[L + 3K']
    double X[3][3];
    for (int J = 0; J < 3; ++J)
      for (int Kp = 0; Kp < 3; ++Kp) {
        double s = 0;
        for (int L = 0; L < 3; ++L) s += Tb[J + 3 * L] * iJ[L + 3 * Kp];
        X[J][Kp] = s;
      }
    for (int K = 0; K < 3; ++K)
      for (int Kp = 0; Kp < 3; ++Kp) {
        double s = 0;
        for (int J = 0; J < 3; ++J) s += iJ[J + 3 * K] * X[J][Kp];
        Dh[q * 81 + (c * 3 + K) + 9 * (k * 3 + Kp)] = dV * s;
      }
  }
  __syncthreads();
}

// One element-matrix entry added at its precomputed position (scatter_jacobian!,
// src/assembly.jl:1402-1408). The add is a reduction whose result is not read: the thread does not
// wait for the nonzero to arrive from memory, as a load-add-store would. Launched colour by colour,
// no two adds of a launch meet the same nonzero (cells of one colour share no free test dof, the
// entries of one cell have distinct positions), so the colours add in a fixed order and the sums
// are deterministic; launched over all cells at once, neighbouring cells' adds meet in L2.
__device__ __forceinline__ void scatter_add(double* nzval, int32_t p, double v) {
  if (p > 0) atomicAdd(nzval + (p - 1), v);
}

// 27-node cells (Q2): G_c in shared memory, 3x3 register tiles of K_c
template <int NN>
__global__ void __launch_bounds__(256) jacobian_kernel_g(CellData cd, AsmIO io) {
  constexpr int NDL = 3 * NN;
  extern __shared__ __align__(16) double sm[];
  const int np = io.np;
  double* A = sm;                       // NN*3*np
  double* xl = A + NN * 3 * np;         // NDL
  double* Hs = xl + NDL;                // 9 np
  double* iJs = Hs + 9 * np;            // 9 np
  double* dVs = iJs + 9 * np;           // np
  double* Dh = dVs + np;                // 81 np
  double* G = Dh + 81 * np;             // (3 np) x NDL
  const int li = blockIdx.x;
  if (li >= cd.ncells_list) return;
  const int cell = cd.cells ? cd.cells[li] : li;
  const int32_t* gid = cd.ids + (size_t)cell * NDL;
  for (int i = threadIdx.x; i < NN * 3 * np; i += blockDim.x) A[i] = io.dNt[i];
  for (int j = threadIdx.x; j < NDL; j += blockDim.x) {
    const int32_t id = gid[j];
    xl[j] = id > 0 ? io.u[id - 1] : (id < 0 ? io.dvals[-id - 1] : 0.0);
  }
  __syncthreads();
  asm_point_phase<NN>(cd, io, cell, A, xl, Hs, iJs, dVs, Dh);
  const int32_t* pos = io.nzpos + (size_t)NDL * NDL * cell;
  const int R = 3 * np;
  for (int c = 0; c < 3; ++c) {
    // G_c[r = q*3 + K][mk = k*NN + m] = sum_K' Dh_q[(c,K),(k,K')] dN^[m,K',q]
    for (int e = threadIdx.x; e < R * NDL; e += blockDim.x) {
      const int r = e / NDL, mk = e % NDL;
      const int q = r / 3, K = r % 3, k = mk / NN, m = mk % NN;
      const double* D = Dh + q * 81 + (c * 3 + K) + 9 * (k * 3);
      G[e] = D[0] * A[m + NN * (0 + 3 * q)] + D[9] * A[m + NN * (1 + 3 * q)] + D[18] * A[m + NN * (2 + 3 * q)];
    }
    __syncthreads();
    // K_c[n][mk] = sum_r A[n + NN*r] G[r][mk]; tiles of 3 rows x 3 columns
    constexpr int TN = NN / 3, TM = NDL / 3;
    for (int tile = threadIdx.x; tile < TN * TM; tile += blockDim.x) {
      const int n0 = (tile % TN) * 3, mk0 = (tile / TN) * 3;
      int32_t pp[3][3];  // positions loaded first: their latency overlaps the products
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) pp[i][j] = __ldg(pos + (c * NN + n0 + i) + NDL * (mk0 + j));
      double acc[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int r = 0; r < R; ++r) {
        const double a0 = A[n0 + NN * r], a1 = A[n0 + 1 + NN * r], a2 = A[n0 + 2 + NN * r];
        const double g0 = G[r * NDL + mk0], g1 = G[r * NDL + mk0 + 1], g2 = G[r * NDL + mk0 + 2];
        acc[0][0] += a0 * g0; acc[0][1] += a0 * g1; acc[0][2] += a0 * g2;
        acc[1][0] += a1 * g0; acc[1][1] += a1 * g1; acc[1][2] += a1 * g2;
        acc[2][0] += a2 * g0; acc[2][1] += a2 * g1; acc[2][2] += a2 * g2;
      }
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) scatter_add(io.nzval, pp[i][j], acc[i][j]);
    }
    __syncthreads();
  }
}

// Small cells (Q1, any number of points): one thread per element entry
template <int NN>
__global__ void __launch_bounds__(256) jacobian_kernel_direct(CellData cd, AsmIO io) {
  constexpr int NDL = 3 * NN;
  extern __shared__ __align__(16) double sm[];
  const int np = io.np;
  double* A = sm;
  double* xl = A + NN * 3 * np;
  double* Hs = xl + NDL;
  double* iJs = Hs + 9 * np;
  double* dVs = iJs + 9 * np;
  double* Dh = dVs + np;
  const int li = blockIdx.x;
  if (li >= cd.ncells_list) return;
  const int cell = cd.cells ? cd.cells[li] : li;
  const int32_t* gid = cd.ids + (size_t)cell * NDL;
  for (int i = threadIdx.x; i < NN * 3 * np; i += blockDim.x) A[i] = io.dNt[i];
  for (int j = threadIdx.x; j < NDL; j += blockDim.x) {
    const int32_t id = gid[j];
    xl[j] = id > 0 ? io.u[id - 1] : (id < 0 ? io.dvals[-id - 1] : 0.0);
  }
  __syncthreads();
  asm_point_phase<NN>(cd, io, cell, A, xl, Hs, iJs, dVs, Dh);
  const int32_t* pos = io.nzpos + (size_t)NDL * NDL * cell;
  for (int e = threadIdx.x; e < NDL * NDL; e += blockDim.x) {
    const int ii = e % NDL, jj = e / NDL;
    const int c = ii / NN, n = ii % NN, k = jj / NN, m = jj % NN;
    const int32_t pe = __ldg(pos + ii + NDL * jj);  // loaded first: its latency overlaps the sum
    double acc = 0;
    for (int q = 0; q < np; ++q) {
      const double* D = Dh + q * 81;
      double an[3], am[3];
      for (int K = 0; K < 3; ++K) {
        an[K] = A[n + NN * (K + 3 * q)];
        am[K] = A[m + NN * (K + 3 * q)];
      }
      for (int K = 0; K < 3; ++K) {
        const double* Dk = D + (c * 3 + K) + 9 * (k * 3);
        acc += an[K] * (Dk[0] * am[0] + Dk[9] * am[1] + Dk[18] * am[2]);
      }
    }
    scatter_add(io.nzval, pe, acc);
  }
}

inline size_t asm_smem_bytes(int nn, int np, bool with_g) {
  size_t v = (size_t)nn * 3 * np + 3 * nn + 9 * np + 9 * np + np + 81 * np;
  if (with_g) v += (size_t)3 * np * 3 * nn;
  return v * sizeof(double);
}

}  // namespace hfk
