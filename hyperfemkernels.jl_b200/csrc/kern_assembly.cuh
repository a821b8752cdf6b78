// Fused element Jacobian + scatter into the CSC nonzeros.
//
// One CTA per cell (all cells in one launch, or the cells of one colour per launch). Per point the
// tangent is pulled back to the reference gradients once, Dh_q[(c,K),(k,K')] = dV sum_{J,L} iJt[J,K] T[(c,J),(k,L)] iJt[L,K'], so the element matrix
//   K[(n,c),(m,k)] = sum_q sum_{K,K'} dN^[n,K,q] Dh_q[(c,K),(k,K')] dN^[m,K',q]
// only reads the reference tables (shared by all cells). For 27-node cells it is formed as the
// reference forms it (element_jacobian_mm!, src/assembly.jl:1316-1342): per test component c,
// G_c[(q,K),(m,k)] = sum_K' Dh[(c,K),(k,K')] dN^[m,K',q], then K_c = A^T G_c with A = dN^ as an
// (np*3) x nn matrix, on the FP64 tensor cores (mma.sync m8n8k4). The entries are added at their
// precomputed positions (scatter_jacobian!, src/assembly.jl:1402-1408) by reductions.
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
  int ldg;                // shared row stride of G_c[r][mk] (27-node cells, >= 3 nn)
};

// Row stride of G_c in the 27-node kernel when it fits: at least the 88 columns of the padded
// product, with zeros past column 81, and 4 modulo 16 doubles, so that the 4 x 8 elements of a B
// fragment (k rows apart by the stride, columns adjacent) fall on distinct 8-byte bank pairs within
// each half-warp and two per pair over the warp: two wavefronts, the minimum for 32 doubles
constexpr int ASM_LDG_PADDED = 100;

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

// FP64 tensor-core product of an 8x4 and a 4x8 tile (mma.sync m8n8k4, PTX ISA "Matrix Fragments for
// mma.m8n8k4 with .f64"): lane l holds a = A[l/4][l%4], b = B[l%4][l/4] and the accumulators
// d[i] = D[l/4][2(l%4) + i].
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// One test component c of the 27-node kernel (below): G_c in shared memory, then K_c = A^T G_c on the
// FP64 tensor cores and the scatter. C is a template parameter so that the first column tile
// (TMIN, under SYM) is a constant: the tile loops and their bounds resolve at compile time.
template <int NN, bool PADDED, bool SYM, int C>
__device__ __forceinline__ void asm_component(const AsmIO& io, const int32_t* pos, const double* A, const double* Dh,
                                              double* G) {
  constexpr int NDL = 3 * NN;
  constexpr int MT = (NN + 7) / 8, NT = (NDL + 7) / 8;  // 8-row bands of K_c, 8-column tiles
  constexpr int MK0 = SYM ? C * NN : 0;                 // first column of K_c that is formed
  constexpr int TMIN = MK0 / 8;                         // first column tile that reaches it
  constexpr int TPW = (NT - TMIN + 1) / 2;              // column tiles per warp (two warps per band)
  constexpr int RG = 256 / NDL;                         // thread groups of G_c's construction
  const int np = io.np, ldg = io.ldg;
  const int R = 3 * np, ksteps = (R + 3) / 4;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int band = warp % MT, tile0 = warp / MT;
  const int fr = lane >> 2, fc = lane & 3;  // fragment row / column of this lane
  // G_c[r = q*3 + K][mk = k*NN + m] = sum_K' Dh_q[(c,K),(k,K')] dN^[m,K',q]: thread (g, mk) fills
  // column mk for the points q = g, g + RG, ...; a point's three values of A serve its three rows.
  // Only the columns of the tiles the products read are formed (from the first tile's start; the
  // few of its columns below MK0 are computed, but their entries are not scattered).
  if (threadIdx.x < RG * NDL) {
    const int g = threadIdx.x / NDL, mk = threadIdx.x - g * NDL;
    const int k = mk / NN, m = mk - k * NN;
    if (mk >= TMIN * 8)
      for (int q = g; q < np; q += RG) {
        const double a0 = A[m + NN * (3 * q)], a1 = A[m + NN * (3 * q + 1)], a2 = A[m + NN * (3 * q + 2)];
        const double* D = Dh + q * 81 + C * 3 + 27 * k;
#pragma unroll
        for (int K = 0; K < 3; ++K) G[(3 * q + K) * ldg + mk] = D[K] * a0 + D[K + 9] * a1 + D[K + 18] * a2;
      }
  }
  __syncthreads();
  // this lane's output entries: rows n = band*8 + fr, columns mk = tile*8 + 2 fc + i; positions
  // loaded first (their latency overlaps the products); under SYM also the transposed entry's
  const int n = band * 8 + fr;
  int32_t pp[TPW][2], pt[TPW][2];
  double acc[2][TPW][2];  // even and odd k-steps: two independent chains of tensor-core steps
#pragma unroll
  for (int j = 0; j < TPW; ++j) {
    const int tile = TMIN + tile0 + 2 * j;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int mk = tile * 8 + 2 * fc + i;
      const bool own = tile < NT && n < NN && mk < NDL && mk >= MK0;
      pp[j][i] = own ? __ldg(pos + (C * NN + n) + NDL * mk) : 0;
      pt[j][i] = (SYM && own && mk >= MK0 + NN) ? __ldg(pos + mk + NDL * (C * NN + n)) : 0;
      acc[0][j][i] = acc[1][j][i] = 0.0;
    }
  }
  // fragment elements past the matrices' edges are zeros: a lane whose element lies outside
  // loads a valid address and selects zero, so the warp stays converged for mma.sync
  const bool na = n < NN;
  auto kstep = [&](int ks, double (&ac)[TPW][2]) {
    const int r = ks * 4 + fc;  // k index of this lane's A^T and B fragment elements
    const bool ra = na && r < R;
    double a = A[ra ? n + NN * r : 0];
    a = ra ? a : 0.0;
    const double* Gr = G + r * ldg + fr;
#pragma unroll
    for (int j = 0; j < TPW; ++j) {
      const int tile = TMIN + tile0 + 2 * j;
      if (tile < NT) {  // uniform over the warp
        double b;
        if (PADDED) {
          b = Gr[tile * 8];
        } else {
          const bool rb = r < R && tile * 8 + fr < NDL;
          b = G[rb ? r * ldg + tile * 8 + fr : 0];
          b = rb ? b : 0.0;
        }
        dmma_8x8x4(ac[j][0], ac[j][1], a, b);
      }
    }
  };
  for (int ks = 0; ks < ksteps; ks += 2) {
    kstep(ks, acc[0]);
    if (ks + 1 < ksteps) kstep(ks + 1, acc[1]);  // uniform over the block
  }
#pragma unroll
  for (int j = 0; j < TPW; ++j)
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const double v = acc[0][j][i] + acc[1][j][i];
      scatter_add(io.nzval, pp[j][i], v);
      if (SYM) scatter_add(io.nzval, pt[j][i], v);
    }
  __syncthreads();
}

// 27-node cells (Q2): G_c in shared memory, K_c = A^T G_c on the FP64 tensor cores. Eight warps:
// warp w takes the 8-row band w % 4 of K_c (rows n, 27 padded to 32) and every other 8-column tile
// (columns mk, 81 padded to 88) from w / 4; the k dimension (r = 3 np) runs in steps of 4, padded
// with zeros. A warp loads one fragment of A^T per k-step and reuses it for its five or six tiles.
// PADDED: G_c has the row stride ASM_LDG_PADDED and zeros past its last row and column, so the B
// fragments load without bounds selects; otherwise (large np) the stride is 81 and they select.
// SYM: the tangent has the major symmetry T[(c,J),(k,L)] = T[(k,L),(c,J)] (every hyperelastic law:
// SVK, linear elasticity), so K[(n,c),(m,k)] = K[(m,k),(n,c)]: only the blocks k >= c are formed
// (the column tiles that reach columns k*NN + m >= c*NN: 24 of 33 tiles, and the G_c columns of
// those tiles), and each entry of a block k > c is added at its own position and at its transpose's.
template <int NN, bool PADDED, bool SYM>
__global__ void __launch_bounds__(256) jacobian_kernel_g(CellData cd, AsmIO io) {
  constexpr int NDL = 3 * NN;
  constexpr int MT = (NN + 7) / 8, NT = (NDL + 7) / 8;
  static_assert(MT == 4, "eight warps: four row bands x two column-tile sets");
  extern __shared__ __align__(16) double sm[];
  const int np = io.np, ldg = io.ldg;
  const int R = 3 * np, ksteps = (R + 3) / 4;
  double* A = sm;                       // NN * R
  double* xl = A + (size_t)NN * R;      // NDL
  double* Hs = xl + NDL;                // 9 np
  double* iJs = Hs + 9 * np;            // 9 np
  double* dVs = iJs + 9 * np;           // np
  double* Dh = dVs + np;                // 81 np
  double* G = Dh + 81 * np;             // 4 ksteps x ldg
  const int li = blockIdx.x;
  if (li >= cd.ncells_list) return;
  const int cell = cd.cells ? cd.cells[li] : li;
  const int32_t* gid = cd.ids + (size_t)cell * NDL;
  for (int i = threadIdx.x; i < NN * R; i += blockDim.x) A[i] = io.dNt[i];
  for (int j = threadIdx.x; j < NDL; j += blockDim.x) {
    const int32_t id = gid[j];
    xl[j] = id > 0 ? io.u[id - 1] : (id < 0 ? io.dvals[-id - 1] : 0.0);
  }
  if (PADDED) {  // the padding of G_c: columns NDL..NT*8-1 of every row, and the rows past R
    constexpr int W = NT * 8 - NDL;
    for (int i = threadIdx.x; i < R * W; i += blockDim.x) G[(i / W) * ldg + NDL + i % W] = 0.0;
    for (int i = threadIdx.x; i < (4 * ksteps - R) * NT * 8; i += blockDim.x)
      G[(R + i / (NT * 8)) * ldg + i % (NT * 8)] = 0.0;
  }
  __syncthreads();
  asm_point_phase<NN>(cd, io, cell, A, xl, Hs, iJs, dVs, Dh);
  const int32_t* pos = io.nzpos + (size_t)NDL * NDL * cell;
  asm_component<NN, PADDED, SYM, 0>(io, pos, A, Dh, G);
  asm_component<NN, PADDED, SYM, 1>(io, pos, A, Dh, G);
  asm_component<NN, PADDED, SYM, 2>(io, pos, A, Dh, G);
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

// with_g: G_c with row stride ldg and the rows of the padded k dimension (3 np rounded up to 4)
inline size_t asm_smem_bytes(int nn, int np, bool with_g, int ldg) {
  size_t v = (size_t)nn * 3 * np + 3 * nn + 9 * np + 9 * np + np + 81 * np;
  if (with_g) v += (size_t)((3 * np + 3) / 4 * 4) * ldg;
  return v * sizeof(double);
}

}  // namespace hfk
